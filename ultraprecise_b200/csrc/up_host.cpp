// up_host.cpp — errors, layout tables, host big integers and node analysis.
#include <sys/stat.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "up_internal.h"

namespace upi {

// ---------------------------------------------------------------- errors
static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
up_status fail(up_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}
const char* last_error() { return g_last_error.c_str(); }

// ---------------------------------------------------------------- tables
// Compact bytes per precision, p = 0..299: the reference's __PREC_BYTE_ARRAY
// (src/datatypes/decimal.cu:92).  Kept identical because it is the storage
// format of every compact column.
static const uint8_t kPrecBytes[300] = {
    0, 1, 1, 2, 2, 3, 3, 4, 4, 4, 5, 5, 6, 6, 6, 7, 7, 8, 8, 9,
    9, 9, 10, 10, 11, 11, 11, 12, 12, 13, 13, 14, 14, 14, 15, 15, 16, 16, 16, 17,
    17, 18, 18, 19, 19, 19, 20, 20, 21, 21, 21, 22, 22, 23, 23, 24, 24, 24, 25, 25,
    26, 26, 26, 27, 27, 28, 28, 29, 29, 29, 30, 30, 31, 31, 31, 32, 32, 33, 33, 34,
    34, 34, 35, 35, 36, 36, 36, 37, 37, 38, 38, 38, 39, 39, 40, 40, 41, 41, 41, 42,
    42, 43, 43, 43, 44, 44, 45, 45, 46, 46, 46, 47, 47, 48, 48, 48, 49, 49, 50, 50,
    51, 51, 51, 52, 52, 53, 53, 53, 54, 54, 55, 55, 56, 56, 56, 57, 57, 58, 58, 58,
    59, 59, 60, 60, 61, 61, 61, 62, 62, 63, 63, 63, 64, 64, 65, 65, 66, 66, 66, 67,
    67, 68, 68, 68, 69, 69, 70, 70, 71, 71, 71, 72, 72, 73, 73, 73, 74, 74, 75, 75,
    76, 76, 76, 77, 77, 78, 78, 78, 79, 79, 80, 80, 81, 81, 81, 82, 82, 83, 83, 83,
    84, 84, 85, 85, 86, 86, 86, 87, 87, 88, 88, 88, 89, 89, 90, 90, 91, 91, 91, 92,
    92, 93, 93, 93, 94, 94, 95, 95, 96, 96, 96, 97, 97, 98, 98, 98, 99, 99, 100, 100,
    101, 101, 101, 102, 102, 103, 103, 103, 104, 104, 105, 105, 105, 106, 106, 107, 107, 108, 108, 108,
    109, 109, 110, 110, 110, 111, 111, 112, 112, 113, 113, 113, 114, 114, 115, 115, 115, 116, 116, 117,
    117, 118, 118, 118, 119, 119, 120, 120, 120, 121, 121, 122, 122, 123, 123, 123, 124, 124, 125, 125,
};

// 32-bit words per precision, p = 0..299: the reference's __PREC_WORD_ARRAY
// (src/AriesDataType.cu:7).  Only reported (up_precision_words); limb counts
// of this path come from value bounds.
static const uint8_t kPrecWords[300] = {
    0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 2, 3,
    3, 3, 3, 3, 3, 3, 3, 3, 3, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 5,
    5, 5, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 7, 7,
    7, 7, 7, 7, 7, 7, 7, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 9, 9, 9,
    9, 9, 9, 9, 9, 9, 9, 10, 10, 10, 10, 10, 10, 10, 10, 10, 11, 11, 11, 11,
    11, 11, 11, 11, 11, 11, 12, 12, 12, 12, 12, 12, 12, 12, 12, 12, 13, 13, 13, 13,
    13, 13, 13, 13, 13, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 15, 15, 15, 15, 15,
    15, 15, 15, 15, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 17, 17, 17, 17, 17, 17,
    17, 17, 17, 17, 18, 18, 18, 18, 18, 18, 18, 18, 18, 19, 19, 19, 19, 19, 19, 19,
    19, 19, 19, 20, 20, 20, 20, 20, 20, 20, 20, 20, 21, 21, 21, 21, 21, 21, 21, 21,
    21, 21, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 23, 23, 23, 23, 23, 23, 23, 23,
    23, 24, 24, 24, 24, 24, 24, 24, 24, 24, 24, 25, 25, 25, 25, 25, 25, 25, 25, 25,
    26, 26, 26, 26, 26, 26, 26, 26, 26, 26, 27, 27, 27, 27, 27, 27, 27, 27, 27, 27,
    28, 28, 28, 28, 28, 28, 28, 28, 28, 29, 29, 29, 29, 29, 29, 29, 29, 29, 29, 30,
    30, 30, 30, 30, 30, 30, 30, 30, 30, 31, 31, 31, 31, 31, 31, 31, 31, 31, 32, 32,
};

static int bitlen_pow10_minus1(int p) {
    Big x = big_pow10(p);
    // subtract one
    for (auto& w : x.m) {
        if (w--) break;
    }
    big_trim(x);
    return big_bitlen(x);
}

int compact_bytes(int p) {
    if (p < 1 || p > kMaxPrecision) return -1;
    if (p < 300) return kPrecBytes[p];
    // extension: one sign bit above the magnitude, rounded up to bytes
    return (bitlen_pow10_minus1(p) + 1 + 7) / 8;
}

int precision_words(int p) {
    if (p < 1 || p > kMaxPrecision) return -1;
    if (p < 300) return kPrecWords[p];
    return (bitlen_pow10_minus1(p) + 1 + 31) / 32;
}

// ------------------------------------------------------- host big integer
void big_trim(Big& a) {
    while (!a.m.empty() && a.m.back() == 0) a.m.pop_back();
}

Big big_from_u64(uint64_t v) {
    Big b;
    b.m = {(uint32_t)v, (uint32_t)(v >> 32)};
    big_trim(b);
    return b;
}

static void big_mul_small_inplace(Big& a, uint32_t k) {
    uint64_t c = 0;
    for (auto& w : a.m) {
        uint64_t t = (uint64_t)w * k + c;
        w = (uint32_t)t;
        c = t >> 32;
    }
    if (c) a.m.push_back((uint32_t)c);
}

Big big_pow10(int k) {
    Big r;
    r.m = {1u};
    while (k >= 9) {
        big_mul_small_inplace(r, 1000000000u);
        k -= 9;
    }
    static const uint32_t p10[9] = {1, 10, 100, 1000, 10000, 100000, 1000000, 10000000, 100000000};
    if (k > 0) big_mul_small_inplace(r, p10[k]);
    return r;
}

Big big_mul(const Big& a, const Big& b) {
    Big r;
    if (a.is_zero() || b.is_zero()) return r;
    r.m.assign(a.m.size() + b.m.size(), 0u);
    for (size_t i = 0; i < a.m.size(); i++) {
        uint64_t c = 0;
        for (size_t j = 0; j < b.m.size(); j++) {
            uint64_t t = (uint64_t)a.m[i] * b.m[j] + r.m[i + j] + c;
            r.m[i + j] = (uint32_t)t;
            c = t >> 32;
        }
        r.m[i + b.m.size()] = (uint32_t)c;
    }
    big_trim(r);
    return r;
}

Big big_add(const Big& a, const Big& b) {
    Big r;
    size_t n = std::max(a.m.size(), b.m.size());
    r.m.resize(n + 1);
    uint64_t c = 0;
    for (size_t i = 0; i < n; i++) {
        c += (uint64_t)(i < a.m.size() ? a.m[i] : 0) + (i < b.m.size() ? b.m[i] : 0);
        r.m[i] = (uint32_t)c;
        c >>= 32;
    }
    r.m[n] = (uint32_t)c;
    big_trim(r);
    return r;
}

Big big_sub(const Big& a, const Big& b) {
    Big r;
    r.m.resize(a.m.size());
    int64_t br = 0;
    for (size_t i = 0; i < a.m.size(); i++) {
        int64_t t = (int64_t)a.m[i] - (i < b.m.size() ? b.m[i] : 0) - br;
        br = t < 0;
        r.m[i] = (uint32_t)t;
    }
    big_trim(r);
    return r;
}

int big_cmp(const Big& a, const Big& b) {
    if (a.m.size() != b.m.size()) return a.m.size() < b.m.size() ? -1 : 1;
    for (size_t i = a.m.size(); i-- > 0;)
        if (a.m[i] != b.m[i]) return a.m[i] < b.m[i] ? -1 : 1;
    return 0;
}

int big_bitlen(const Big& a) {
    if (a.m.empty()) return 0;
    return 32 * (int)(a.m.size() - 1) + (32 - __builtin_clz(a.m.back()));
}

Big big_divmod_small(const Big& a, uint32_t d, uint32_t* rem) {
    Big q;
    q.m.resize(a.m.size());
    uint64_t r = 0;
    for (size_t i = a.m.size(); i-- > 0;) {
        uint64_t cur = (r << 32) | a.m[i];
        q.m[i] = (uint32_t)(cur / d);
        r = cur % d;
    }
    if (rem) *rem = (uint32_t)r;
    big_trim(q);
    return q;
}

uint64_t big_low64(const Big& a) {
    uint64_t v = 0;
    if (a.m.size() > 0) v |= a.m[0];
    if (a.m.size() > 1) v |= (uint64_t)a.m[1] << 32;
    return v;
}

std::string big_to_dec(const Big& a) {
    if (a.is_zero()) return "0";
    Big x = a;
    std::string s;
    while (!x.is_zero()) {
        uint32_t r;
        x = big_divmod_small(x, 1000000000u, &r);
        char buf[16];
        if (x.is_zero()) snprintf(buf, sizeof buf, "%u", r);
        else snprintf(buf, sizeof buf, "%09u", r);
        s = std::string(buf) + s;
    }
    return s;
}

Big big_from_dec(const std::string& s) {
    Big r;
    for (char ch : s) {
        if (ch < '0' || ch > '9') continue;
        big_mul_small_inplace(r, 10u);
        Big d = big_from_u64((uint64_t)(ch - '0'));
        r = big_add(r, d);
    }
    big_trim(r);
    return r;
}

void mkdir_if_missing(const std::string& dir) {
    if (!dir.empty()) mkdir(dir.c_str(), 0755);
}

// ------------------------------------------------------ node analysis
int limbs_for_bits(int bits) { return std::max(1, (bits + 31) / 32); }

// boolean-valued nodes: comparisons and AND/OR
static bool is_compare_kind(int k) { return k >= UP_NODE_LT && k <= UP_NODE_OR; }

// Static scale of each node as the reference evaluates it: columns carry
// their scale, constants theirs, integers 0; ADD/SUB take the larger scale
// (AlignAddSubData), MUL adds scales (AriesDecimal.hxx:319), DIV adds 4
// (DIV_FIX_EX_FRAC, :762), MOD is 0 (:959).  Bits bound every magnitude the
// node can hold given its operands' bounds.
up_status analyze_nodes(const up_expr_node* nodes, int n_nodes, const up_col_type* cols, int n_cols,
                        std::vector<NodeFacts>& facts, std::vector<int>& topo, const std::vector<int>& roots) {
    facts.assign(n_nodes, NodeFacts());
    topo.clear();
    std::vector<int> state(n_nodes, 0);  // 0 new, 1 visiting, 2 done
    // iterative post-order DFS over every root
    for (int root : roots) {
        if (root < 0 || root >= n_nodes) return fail(UP_ERR_INVALID_ARG, "root index out of range");
        std::vector<std::pair<int, int>> st;
        st.push_back({root, 0});
        while (!st.empty()) {
            const int idx = st.back().first;
            const int phase = st.back().second;
            if (idx < 0 || idx >= n_nodes) return fail(UP_ERR_INVALID_ARG, "child index out of range");
            if (phase == 0) {
                if (state[idx] == 2) {
                    st.pop_back();
                    continue;
                }
                if (state[idx] == 1) return fail(UP_ERR_INVALID_ARG, "expression graph has a cycle");
                state[idx] = 1;
                st.back().second = 1;
                const up_expr_node& nd = nodes[idx];
                int k = nd.kind;
                bool binary = (k >= UP_NODE_ADD && k <= UP_NODE_MOD) || is_compare_kind(k);
                bool unary = k == UP_NODE_RESCALE;
                int l = nd.left, r = nd.right;
                if (binary) {
                    st.push_back({r, 0});
                    st.push_back({l, 0});
                } else if (unary) {
                    st.push_back({l, 0});
                }
                continue;
            }
            // phase 1: children done
            const up_expr_node& nd = nodes[idx];
            NodeFacts& f = facts[idx];
            switch (nd.kind) {
                case UP_NODE_COLUMN: {
                    if (nd.column < 0 || nd.column >= n_cols)
                        return fail(UP_ERR_INVALID_ARG, "column index out of range");
                    const up_col_type& t = cols[nd.column];
                    int b = compact_bytes(t.precision);
                    if (b < 1) return fail(UP_ERR_INVALID_ARG, "column precision out of range");
                    if (t.scale < 0 || t.scale > t.precision)
                        return fail(UP_ERR_INVALID_ARG, "column scale out of range");
                    f.scale = t.scale;
                    f.bits = 8 * b - 1;
                    break;
                }
                case UP_NODE_CONST: {
                    if (nd.const_nlimbs < 0 || nd.const_nlimbs > UP_CONST_MAX_LIMBS)
                        return fail(UP_ERR_INVALID_ARG, "constant limb count out of range");
                    if (nd.scale < 0 || nd.scale > kMaxPrecision)
                        return fail(UP_ERR_INVALID_ARG, "constant scale out of range");
                    Big c;
                    c.m.assign(nd.const_limbs, nd.const_limbs + nd.const_nlimbs);
                    big_trim(c);
                    f.scale = nd.scale;
                    f.bits = std::max(1, big_bitlen(c));
                    break;
                }
                case UP_NODE_INT: {
                    uint64_t mag = nd.int_value < 0 ? (uint64_t)(-(nd.int_value + 1)) + 1u : (uint64_t)nd.int_value;
                    f.scale = 0;
                    f.bits = std::max(1, big_bitlen(big_from_u64(mag)));
                    break;
                }
                case UP_NODE_ADD:
                case UP_NODE_SUB: {
                    const NodeFacts& a = facts[nd.left];
                    const NodeFacts& b = facts[nd.right];
                    if (a.is_compare || b.is_compare) return fail(UP_ERR_INVALID_ARG, "arithmetic on a comparison");
                    int s = std::max(a.scale, b.scale);
                    int ba = a.bits + (s > a.scale ? big_bitlen(big_pow10(s - a.scale)) : 0);
                    int bb = b.bits + (s > b.scale ? big_bitlen(big_pow10(s - b.scale)) : 0);
                    f.scale = s;
                    f.bits = std::max(ba, bb) + 1;
                    break;
                }
                case UP_NODE_MUL: {
                    const NodeFacts& a = facts[nd.left];
                    const NodeFacts& b = facts[nd.right];
                    if (a.is_compare || b.is_compare) return fail(UP_ERR_INVALID_ARG, "arithmetic on a comparison");
                    f.scale = a.scale + b.scale;
                    f.bits = a.bits + b.bits;
                    break;
                }
                case UP_NODE_DIV: {
                    const NodeFacts& a = facts[nd.left];
                    const NodeFacts& b = facts[nd.right];
                    if (a.is_compare || b.is_compare) return fail(UP_ERR_INVALID_ARG, "arithmetic on a comparison");
                    f.scale = a.scale + 4;
                    int sh = b.scale + 4;
                    f.bits = std::max(64, a.bits + big_bitlen(big_pow10(sh)));
                    break;
                }
                case UP_NODE_MOD: {
                    const NodeFacts& a = facts[nd.left];
                    const NodeFacts& b = facts[nd.right];
                    if (a.is_compare || b.is_compare) return fail(UP_ERR_INVALID_ARG, "arithmetic on a comparison");
                    f.scale = 0;
                    f.bits = std::min(a.bits, b.bits);
                    break;
                }
                case UP_NODE_RESCALE: {
                    const NodeFacts& a = facts[nd.left];
                    if (a.is_compare) return fail(UP_ERR_INVALID_ARG, "rescale of a comparison");
                    if (nd.scale < 0 || nd.scale > kMaxPrecision)
                        return fail(UP_ERR_INVALID_ARG, "rescale target out of range");
                    f.scale = nd.scale;
                    if (nd.scale >= a.scale) {
                        f.bits = a.bits + (nd.scale > a.scale ? big_bitlen(big_pow10(nd.scale - a.scale)) : 0);
                    } else {
                        // |v| < 2^b and 10^d >= 2^(bitlen(10^d)-1), so the
                        // truncated quotient is below 2^(b - bitlen(10^d) + 1)
                        f.bits = std::max(1, a.bits - big_bitlen(big_pow10(a.scale - nd.scale)) + 1);
                    }
                    break;
                }
                default:
                    if (is_compare_kind(nd.kind)) {
                        const NodeFacts& a = facts[nd.left];
                        const NodeFacts& b = facts[nd.right];
                        const bool logic = nd.kind == UP_NODE_AND || nd.kind == UP_NODE_OR;
                        if (!logic && (a.is_compare || b.is_compare))
                            return fail(UP_ERR_INVALID_ARG, "comparison of comparisons");
                        if (logic && !(a.is_compare && b.is_compare))
                            return fail(UP_ERR_INVALID_ARG, "AND/OR of a non-boolean operand");
                        f.scale = 0;
                        f.bits = 1;
                        f.is_compare = true;
                        break;
                    }
                    return fail(UP_ERR_INVALID_ARG, "unknown node kind " + std::to_string(nd.kind));
            }
            f.limbs = limbs_for_bits(f.bits);
            state[idx] = 2;
            topo.push_back(idx);
            st.pop_back();
        }
    }
    return UP_OK;
}

}  // namespace upi
