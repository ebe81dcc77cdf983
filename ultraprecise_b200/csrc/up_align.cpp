// up_align.cpp — the reference's AlignOptimize expression rewrite.
#include "up_internal.h"

extern "C" up_status up_expr_align_optimize(const up_expr_node* in, int32_t n_in, int32_t root,
                                            const up_col_type* cols, int32_t n_cols, up_expr_node* out,
                                            int32_t cap, int32_t* n_out, int32_t* out_root) {
    return upi::fail(UP_ERR_UNSUPPORTED, "align_optimize not built yet");
}
