// up_typing.cpp — result typing of expression nodes (the reference's
// ListToBinTree rules, AriesEngineShell.cpp:90-144).
#include <algorithm>
#include <vector>

#include "up_internal.h"

namespace upi {

static bool is_cmp(int k) { return k >= UP_NODE_LT && k <= UP_NODE_OR; }  // boolean nodes

// ADD/SUB: p = max(p1-s1, p2-s2) + 1 + max(s1, s2), s = max(s1, s2)  (:115-121)
// MUL:     p = (p1-s1) + (p2-s2) + s1 + s2,        s = s1 + s2       (:122-128)
// DIV:     p = p1 - p2 + s2 + 4 + 1,               s = s1 + 4        (:129-135)
// MOD:     p = p2,                                 s = 0             (:136-141)
// The reference stores these in uint16 fields; a DIV precision that comes
// out <= its scale (a divisor much wider than the dividend) wraps there and
// indexes past its byte table.  This path widens such a DIV result to
// p = s + 1 instead.
static void type_binary(int kind, int p1, int s1, int p2, int s2, int& p, int& s) {
    switch (kind) {
        case UP_NODE_ADD:
        case UP_NODE_SUB:
            p = std::max(p1 - s1, p2 - s2) + 1;
            s = std::max(s1, s2);
            p += s;
            break;
        case UP_NODE_MUL:
            p = (p1 - s1) + (p2 - s2);
            s = s1 + s2;
            p += s;
            break;
        case UP_NODE_DIV:
            p = p1 - p2 + s2 + 4 + 1;
            s = s1 + 4;
            if (p <= s) p = s + 1;
            break;
        case UP_NODE_MOD:
            p = p2;
            s = 0;
            break;
        default:
            p = 1;
            s = 0;
    }
}

up_status derive_types_impl(up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols, int n_cols) {
    std::vector<NodeFacts> f;
    std::vector<int> topo;
    up_status st = analyze_nodes(nodes, n_nodes, cols, n_cols, f, topo, {root});
    if (st != UP_OK) return st;
    for (int k : topo) {
        up_expr_node& nd = nodes[k];
        switch (nd.kind) {
            case UP_NODE_COLUMN:
                nd.precision = cols[nd.column].precision;
                nd.scale = cols[nd.column].scale;
                break;
            case UP_NODE_CONST:
                break;  // given by the caller (folded constants may carry precision 0)
            case UP_NODE_INT: {
                // Decimal(int32_t) / Decimal(int64_t) precisions, decimal.cu:291-309
                bool fits32 = nd.int_value >= -2147483648LL && nd.int_value <= 2147483647LL;
                nd.precision = fits32 ? 10 : 19;
                nd.scale = 0;
                break;
            }
            case UP_NODE_RESCALE:
                if (nd.precision < 1) return fail(UP_ERR_INVALID_ARG, "RESCALE node needs a target precision");
                break;
            default:
                if (is_cmp(nd.kind)) {
                    nd.precision = 1;
                    nd.scale = 0;
                } else {
                    const up_expr_node& a = nodes[nd.left];
                    const up_expr_node& b = nodes[nd.right];
                    int p, s;
                    type_binary(nd.kind, a.precision, a.scale, b.precision, b.scale, p, s);
                    nd.precision = p;
                    nd.scale = s;
                }
        }
        if (nd.kind != UP_NODE_CONST && nd.kind != UP_NODE_RESCALE && !is_cmp(nd.kind) &&
            nd.scale != f[k].scale)
            return fail(UP_ERR_INVALID_ARG, "internal: typed scale disagrees with evaluation scale");
        if (!is_cmp(nd.kind) && nd.precision > kMaxPrecision)
            return fail(UP_ERR_UNSUPPORTED, "result precision above " + std::to_string(kMaxPrecision));
    }
    return UP_OK;
}

}  // namespace upi

extern "C" up_status up_expr_derive_types(up_expr_node* nodes, int32_t n_nodes, int32_t root,
                                          const up_col_type* cols, int32_t n_cols) {
    if (!nodes || n_nodes <= 0) return upi::fail(UP_ERR_INVALID_ARG, "no nodes");
    if (n_cols > 0 && !cols) return upi::fail(UP_ERR_INVALID_ARG, "no column types");
    return upi::derive_types_impl(nodes, n_nodes, root, cols, n_cols);
}
