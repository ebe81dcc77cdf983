/*
 * ultraprecise_util.h — benchmark and test utilities of libultraprecise.so.
 *
 * These have no counterpart in the reference's decimal path: they produce the
 * seeded synthetic columns that stand in for the reference's datasets (the
 * TPC-H lineitem columns of its paper experiments and the data generators
 * under append_expr_info/gen_data/, which are not shipped as data), flush the
 * L2 cache between timed iterations, and measure the 32-bit integer
 * multiply-add peak used as the roofline of the wide-precision kernels.
 */
#ifndef ULTRAPRECISE_UTIL_H_
#define ULTRAPRECISE_UTIL_H_

#include "ultraprecise.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Seeded random compact decimals of precision p written to `out` (DEVICE,
 * rows * up_compact_bytes(p) bytes).  Every one of the p digits is uniform
 * 0-9 (the precision-sweep distribution); signs are +/- with equal odds when
 * signed_ != 0.  nonzero != 0 redraws an all-zero value (a zero divisor). */
up_status up_util_gen_digits(void* out, int64_t rows, int32_t precision, uint64_t seed,
                             int32_t signed_, int32_t nonzero, void* stream);

/* Seeded random compact decimals whose unscaled integer is
 * lo + step * U{0 .. (hi-lo)/step}; lo, hi, step must fit int64 and the value
 * must fit the compact width of p. */
up_status up_util_gen_range(void* out, int64_t rows, int32_t precision, int64_t lo, int64_t hi,
                            int64_t step, uint64_t seed, void* stream);

/* Write `bytes` of a scratch buffer (DEVICE) to evict L2. */
up_status up_util_flush_l2(void* buf, int64_t bytes, void* stream);

/* Measure the limb multiply-add throughput of the current device: 32 x 32
 * -> 64-bit products added to 64-bit accumulators (the operation the limb
 * multiply loops issue), eight independent chains per thread, nothing else
 * in the loop.  Returns multiply-adds per second. */
up_status up_util_imad_peak(double* madds_per_s, void* stream);

/* Make the bounded wait of the bulk-copy pipelines run out, on purpose and
 * safely: one block waits with `polls` polls (1 .. 2^24) on an mbarrier armed
 * for bytes that no copy ever delivers, then reports UP_ROWERR_TIMEOUT in
 * *err_word (DEVICE) the way the tile kernels do, and adds 1 to *done_word
 * (DEVICE) when it has returned.  Nothing is left in flight; the context stays
 * usable.  For testing the timeout path. */
up_status up_util_wait_timeout_probe(uint32_t polls, uint32_t* err_word, uint32_t* done_word, void* stream);

/* Compile a kernel source with the library's NVRTC settings without loading
 * it (no GPU needed).  Returns UP_OK or UP_ERR_COMPILE with the log in
 * up_last_error_message(). */
up_status up_util_compile_only(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                               const up_col_type* cols, int32_t n_cols, int32_t query,
                               const up_query_agg* aggs, int32_t n_aggs);

/* The same for a batch module (ultraprecise_batch.h): generate and compile
 * every task into one CUBIN without loading it. */
/* Compile an expression module with explicit options (e.g. threads per
 * value) into the cubin cache without loading it (no GPU needed). */
up_status up_util_compile_expr_only(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                                    const up_col_type* cols, int32_t n_cols, const up_compile_opts* opts);

/* The threads per value an automatic compile would choose (no compile, no
 * GPU): use_model 0 = the width rule, 1 = the default cost model when one is
 * set (else the rule). */
up_status up_util_auto_tpv(const up_expr_node* nodes, int32_t n_nodes, int32_t root, const up_col_type* cols,
                           int32_t n_cols, int32_t use_model, int32_t* threads_per_value);

/* Generated CUDA source of an expression module (no compile, no GPU):
 * returns its length; copies at most cap-1 bytes + NUL when buf != NULL. */
int64_t up_util_expr_source(const up_expr_node* nodes, int32_t n_nodes, int32_t root, const up_col_type* cols,
                            int32_t n_cols, const up_compile_opts* opts, char* buf, int64_t cap);

/* NVRTC-compile a batch module into the cubin cache (no GPU): tpv_of gives
 * each task's threads per value, NULL the automatic choice (tpv_policy 0). */
struct up_batch_task;
up_status up_util_compile_batch_only(const struct up_batch_task* tasks, int32_t n_tasks, const int32_t* tpv_of);

/* The threads per value the measured batch policy (tpv_policy 2) times for a
 * task: writes at most cap of them to out, returns the count (-1: bad
 * arguments).  One thread per value is always first. */
int32_t up_util_batch_tpv_candidates(const struct up_batch_task* task, int32_t* out, int32_t cap);

#ifdef __cplusplus
}
#endif
#endif
