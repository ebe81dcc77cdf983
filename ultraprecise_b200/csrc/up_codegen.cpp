// up_codegen.cpp — typed expression DAG -> CUDA C++ source for NVRTC.
//
// Plays the role of the reference's expression codegen
// (AriesCommonExpr::StringForDynamicCode, AriesCommonExpr.cpp:163-304, and
// AEExprCalcNode::GenerateCudaFunction / GenerateLoadDataCode /
// GenSaveDataCode, AriesExprCalcNode.cpp:76-106, 1285-1428), but emits
// straight-line limb code with every node's limb count and scale fixed at
// compile time instead of instantiating one AriesDecimal<LEN> for all nodes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <set>
#include <sstream>

#include "up_internal.h"

namespace upi {

namespace {

std::string hex32(uint32_t v) {
    char b[16];
    snprintf(b, sizeof b, "0x%08xu", v);
    return b;
}

std::string limbs_init(const Big& x, int n) {
    std::string s = "{";
    for (int i = 0; i < n; i++) {
        if (i) s += ", ";
        s += hex32(i < (int)x.m.size() ? x.m[i] : 0u);
    }
    return s + "}";
}

bool is_compare_kind(int k) { return k >= UP_NODE_LT && k <= UP_NODE_OR; }  // boolean nodes

// Emits the body of a per-row evaluation function for a set of nodes.
struct Emitter {
    const up_expr_node* nodes;
    const up_col_type* cols;
    const std::vector<NodeFacts>& f;
    std::ostringstream body;
    std::set<int> p10;
    int tmp = 0;
    bool out_of_line = false;  // call wide operations out of line (see wide_work)

    Emitter(const up_expr_node* n, const up_col_type* c, const std::vector<NodeFacts>& facts)
        : nodes(n), cols(c), f(facts) {}

    // Sum of limb-product sizes over the expression's wide operations; above
    // kOutOfLineWork the operations with at least kWideOp limb products are
    // called out of line.
    static constexpr long kOutOfLineWork = 16384;
    static constexpr long kWideOp = 256;
    long work = 0;  // limb-product work per row (a cost estimate)
    void plan(const std::vector<int>& topo) {
        work = 0;
        for (int k : topo) work += op_size(k);
        out_of_line = work > kOutOfLineWork;
    }
    long op_size(int k) const {
        const up_expr_node& nd = nodes[k];
        switch (nd.kind) {
            case UP_NODE_MUL: return (long)f[nd.left].limbs * f[nd.right].limbs;
            case UP_NODE_DIV: return (long)f[k].limbs * f[nd.right].limbs + (long)f[nd.left].limbs * 4;
            case UP_NODE_RESCALE:
                return nd.scale < f[nd.left].scale
                           ? (long)f[nd.left].limbs * limbs_for_bits(big_bitlen(big_pow10(f[nd.left].scale - nd.scale)))
                           : (long)f[k].limbs;
            case UP_NODE_ADD:
            case UP_NODE_SUB: return (long)f[k].limbs * 4;
            default: return 0;
        }
    }
    const char* sfx(long size) const { return (out_of_line && size >= kWideOp) ? "_ni" : ""; }

    std::string p10_name(int k) {
        p10.insert(k);
        return "P10_" + std::to_string(k);
    }

    std::string v(int k) { return "v" + std::to_string(k); }
    std::string s(int k) { return "s" + std::to_string(k); }

    // name of an array holding node a's magnitude at scale sc (sc >= scale(a))
    std::string aligned(int a, int sc) {
        const NodeFacts& fa = f[a];
        if (sc == fa.scale) return v(a);
        const int d = sc - fa.scale;
        Big p = big_pow10(d);
        const int L = limbs_for_bits(fa.bits + big_bitlen(p));
        std::string t = "t" + std::to_string(tmp++);
        body << "    u32 " << t << "[" << L << "];\n";
        if (p.m.size() == 1) body << "    mul_u32(" << t << ", " << v(a) << ", " << hex32(p.m[0]) << ");\n";
        else body << "    mul" << sfx((long)fa.limbs * (long)p.m.size()) << "(" << t << ", " << v(a) << ", "
                  << p10_name(d) << ");\n";
        return t;
    }

    void node(int k) {
        const up_expr_node& nd = nodes[k];
        const NodeFacts& fk = f[k];
        const int L = fk.limbs;
        body << "    // node " << k << ": kind " << nd.kind << ", scale " << fk.scale << ", <= " << fk.bits
             << " bits\n";
        switch (nd.kind) {
            case UP_NODE_COLUMN: {
                const int B = compact_bytes(cols[nd.column].precision);
                body << "    u32 " << v(k) << "[" << L << "]; u32 " << s(k) << ";\n";
                body << "    if (words) ld_compact_words<" << B << ", " << L << ">(in" << nd.column << ", " << v(k)
                     << ", " << s(k) << ");\n";
                body << "    else ld_compact_bytes<" << B << ", " << L << ">(in" << nd.column << ", " << v(k)
                     << ", " << s(k) << ");\n";
                break;
            }
            case UP_NODE_CONST: {
                Big c;
                c.m.assign(nd.const_limbs, nd.const_limbs + nd.const_nlimbs);
                big_trim(c);
                body << "    const u32 " << v(k) << "[" << L << "] = " << limbs_init(c, L) << "; u32 " << s(k)
                     << " = " << (nd.const_sign ? 1 : 0) << "u;\n";
                break;
            }
            case UP_NODE_INT: {
                uint64_t mag = nd.int_value < 0 ? (uint64_t)(-(nd.int_value + 1)) + 1u : (uint64_t)nd.int_value;
                body << "    const u32 " << v(k) << "[" << L << "] = " << limbs_init(big_from_u64(mag), L)
                     << "; u32 " << s(k) << " = " << (nd.int_value < 0 ? 1 : 0) << "u;\n";
                break;
            }
            case UP_NODE_ADD:
            case UP_NODE_SUB: {
                std::string A = aligned(nd.left, fk.scale);
                std::string Bn = aligned(nd.right, fk.scale);
                body << "    u32 " << v(k) << "[" << L << "]; u32 " << s(k) << ";\n";
                body << "    add_signed(" << v(k) << ", " << s(k) << ", " << A << ", " << s(nd.left) << ", " << Bn
                     << ", " << s(nd.right) << (nd.kind == UP_NODE_SUB ? " ^ 1u" : "") << ");\n";
                break;
            }
            case UP_NODE_MUL:
                body << "    u32 " << v(k) << "[" << L << "]; mul" << sfx(op_size(k)) << "(" << v(k) << ", "
                     << v(nd.left) << ", "
                     << v(nd.right) << "); u32 " << s(k) << " = " << s(nd.left) << " ^ " << s(nd.right) << ";\n";
                break;
            case UP_NODE_DIV: {
                const int sh = f[nd.right].scale + 4;
                Big p = big_pow10(sh);
                const int np = (int)p.m.size();
                char w[40];
                snprintf(w, sizeof w, "0x%016llxull", (unsigned long long)big_low64(p));
                body << "    u32 " << v(k) << "[" << L << "]; u32 " << s(k) << ";\n";
                body << "    err |= div_round" << sfx(op_size(k)) << "<" << L << ", " << f[nd.left].limbs << ", " << f[nd.right].limbs << ", "
                     << np << ", " << sh << "u, " << w << ">(" << v(k) << ", " << s(k) << ", " << v(nd.left)
                     << ", " << s(nd.left) << ", " << v(nd.right) << ", " << s(nd.right) << ", " << p10_name(sh)
                     << ");\n";
                break;
            }
            case UP_NODE_MOD:
                body << "    u32 " << v(k) << "[" << L << "]; u32 " << s(k) << ";\n";
                body << "    err |= mod(" << v(k) << ", " << s(k) << ", " << v(nd.left) << ", " << s(nd.left) << ", "
                     << v(nd.right) << ", " << s(nd.right) << ");\n";
                break;
            case UP_NODE_RESCALE: {
                const int sa = f[nd.left].scale;
                body << "    u32 " << v(k) << "[" << L << "]; u32 " << s(k) << " = " << s(nd.left) << ";\n";
                if (nd.scale >= sa) {
                    std::string A = aligned(nd.left, nd.scale);
                    body << "    copy_ext(" << v(k) << ", " << A << ");\n";
                } else {
                    body << "    trunc_div_pow10" << sfx(op_size(k)) << "(" << v(k) << ", " << v(nd.left) << ", "
                         << p10_name(sa - nd.scale)
                         << ");\n";
                }
                break;
            }
            default: {
                if (nd.kind == UP_NODE_AND || nd.kind == UP_NODE_OR) {
                    body << "    const u32 c" << k << " = c" << nd.left << (nd.kind == UP_NODE_AND ? " & " : " | ") << "c"
                         << nd.right << ";\n";
                    return;
                }
                // comparison
                const int sc = std::max(f[nd.left].scale, f[nd.right].scale);
                std::string A = aligned(nd.left, sc);
                std::string Bn = aligned(nd.right, sc);
                body << "    const u32 c" << k << " = compare(" << (nd.kind - UP_NODE_LT) << ", " << A << ", "
                     << s(nd.left) << ", " << Bn << ", " << s(nd.right) << ");\n";
                return;
            }
        }
        if (nd.reverse) body << "    " << s(k) << " ^= 1u;\n";
    }

    std::string constants() {
        std::ostringstream o;
        for (int k : p10) {
            Big p = big_pow10(k);
            o << "    const u32 P10_" << k << "[" << p.m.size() << "] = " << limbs_init(p, (int)p.m.size()) << ";\n";
        }
        return o.str();
    }
};

// The argument blocks themselves (UpArgs, UpQArgs, BTask, BArgs) are declared
// once, in up_kargs.h, which up_dev.cuh includes for the generated code.
std::string kargs_source() { return "\n"; }

// Query modules: UpQArgs with the group-key fields and the group lookup.
std::string query_kargs_source() {
    return R"(
UP_DI int q_group(const UpQArgs& a, i64 row) {
    if (a.key_mode == 0) return a.gid[row];
    u32 key;
    if (a.key_mode == 1) key = a.key0[row];
    else if (a.key_mode == 2) key = ((u32)a.key0[row] << 8) | a.key1[row];
    else key = ((u32)a.key0[2 * row] << 8) | a.key0[2 * row + 1];
    return __ldg(a.key_table + key);
}
// the key of row r of a staged tile of R rows (key bytes at t)
UP_DI u32 q_tile_key(const UpQArgs& a, const u8* t, int r, int R) {
    if (a.key_mode == 1) return t[r];
    if (a.key_mode == 2) return ((u32)t[r] << 8) | t[R + r];
    return ((u32)t[2 * r] << 8) | t[2 * r + 1];
}
// the group of row r of a staged tile (gid or key bytes at t)
UP_DI int q_tile_group(const UpQArgs& a, const u8* t, int r, int R) {
    if (a.key_mode == 0) return ((const int*)t)[r];
    return __ldg(a.key_table + q_tile_key(a, t, r, R));
}
// The group count: n_groups when it is >= 0; otherwise the count the key
// table holds (entry 131072), with -n_groups the capacity of the
// accumulators and outputs; -1 when the table's count exceeds it.
UP_DI int q_groups(const UpQArgs& a) {
    if (a.n_groups >= 0) return a.n_groups;
    const int n = *(volatile const int*)(a.key_table + 131072);
    return (n >= 0 && n <= -a.n_groups) ? n : -1;
}
// groups held in shared memory by a tile kernel of this mode (recomputed
// where needed, so that no register holds it through the row loop)
UP_DI int q_nsm(const UpQArgs& a, int mode, int gr) {
    const int n = q_groups(a);
    return mode == 0 ? (n < gr ? n : gr) : (mode == 1 ? n : 0);
}
)";
}

std::string params_decl(const std::vector<int>& used_cols) {
    std::string p;
    for (int c : used_cols) p += "const u8* __restrict__ in" + std::to_string(c) + ", ";
    return p;
}

// Cooperative row code (T threads per value, K limbs per thread): the same
// node numbering and semantics as Emitter, on the tpi_* primitives.
struct TEmitter {
    const up_expr_node* nodes;
    const up_col_type* cols;
    const std::vector<NodeFacts>& f;
    int T, K;
    std::ostringstream body, globals;
    std::set<int> p10;
    int tmp = 0;
    bool out_of_line = false;  // call multiplies and divisions out of line
    bool words = false;        // columns come from a padded shared-memory tile (word loads)

    TEmitter(const up_expr_node* n, const up_col_type* c, const std::vector<NodeFacts>& facts, int t, int k)
        : nodes(n), cols(c), f(facts), T(t), K(k) {}

    // More than this many multiplies / divisions: call them out of line, so
    // code size (and compile time) follows the number of distinct shapes.
    static constexpr int kOutOfLineOps = 6;
    void plan(const std::vector<int>& topo) {
        int ops = 0;
        for (int k : topo) {
            const int kind = nodes[k].kind;
            ops += kind == UP_NODE_MUL || kind == UP_NODE_DIV ||
                   (kind == UP_NODE_RESCALE && nodes[k].scale < f[nodes[k].left].scale);
        }
        out_of_line = ops > kOutOfLineOps;
    }
    const char* ni() const { return out_of_line ? "_ni" : ""; }

    std::string v(int k) { return "v" + std::to_string(k); }
    std::string s(int k) { return "s" + std::to_string(k); }
    std::string tk() { return std::to_string(T) + ", " + std::to_string(K); }
    std::string p10_name(int d) {
        p10.insert(d);
        return "P10_" + std::to_string(d);
    }
    std::string aligned(int a, int sc) {
        if (sc == f[a].scale) return v(a);
        const int d = sc - f[a].scale;
        const Big p = big_pow10(d);
        std::string t = "t" + std::to_string(tmp++);
        body << "    u32 " << t << "[" << K << "]; tpi_mul_const<" << tk() << ", " << f[a].limbs << ", " << p.m.size()
             << ">(" << t << ", " << v(a) << ", " << p10_name(d) << ");\n";
        return t;
    }
    void constant(int k, const Big& c, uint32_t sign) {
        globals << "__device__ const u32 C" << k << "[" << std::max<size_t>(1, c.m.size()) << "] = "
                << limbs_init(c, std::max<int>(1, (int)c.m.size())) << ";\n";
        body << "    u32 " << v(k) << "[" << K << "]; tpi_const<" << tk() << ">(" << v(k) << ", C" << k << ", "
             << c.m.size() << "); u32 " << s(k) << " = " << sign << "u;\n";
    }
    void node(int k) {
        const up_expr_node& nd = nodes[k];
        body << "    // node " << k << ": kind " << nd.kind << ", scale " << f[k].scale << ", <= " << f[k].bits
             << " bits\n";
        switch (nd.kind) {
            case UP_NODE_COLUMN: {
                const int B = compact_bytes(cols[nd.column].precision);
                body << "    u32 " << v(k) << "[" << K << "]; u32 " << s(k) << "; tpi_ld" << (words ? "_words" : "") << "<" << tk() << ", " << B
                     << ">(in" << nd.column << ", " << v(k) << ", " << s(k) << ");\n";
                break;
            }
            case UP_NODE_CONST: {
                Big cb;
                cb.m.assign(nd.const_limbs, nd.const_limbs + nd.const_nlimbs);
                big_trim(cb);
                constant(k, cb, nd.const_sign ? 1u : 0u);
                break;
            }
            case UP_NODE_INT: {
                const uint64_t mag =
                    nd.int_value < 0 ? (uint64_t)(-(nd.int_value + 1)) + 1u : (uint64_t)nd.int_value;
                Big cb = big_from_u64(mag);
                big_trim(cb);
                constant(k, cb, nd.int_value < 0 ? 1u : 0u);
                break;
            }
            case UP_NODE_ADD:
            case UP_NODE_SUB: {
                const std::string A = aligned(nd.left, f[k].scale);
                const std::string Bn = aligned(nd.right, f[k].scale);
                body << "    u32 " << v(k) << "[" << K << "]; u32 " << s(k) << "; tpi_add_signed<" << tk() << ">("
                     << v(k) << ", " << s(k) << ", " << A << ", " << s(nd.left) << ", " << Bn << ", " << s(nd.right)
                     << (nd.kind == UP_NODE_SUB ? " ^ 1u" : "") << ");\n";
                break;
            }
            case UP_NODE_MUL: {
                // the operand with fewer limbs is streamed limb by limb
                int a = nd.left, b = nd.right;
                if (f[a].limbs < f[b].limbs) std::swap(a, b);
                body << "    u32 " << v(k) << "[" << K << "]; tpi_mul" << ni() << "<" << tk() << ", " << f[a].limbs << ", "
                     << f[b].limbs
                     << ">(" << v(k)
                     << ", " << v(a) << ", " << v(b) << "); u32 " << s(k) << " = " << s(nd.left) << " ^ "
                     << s(nd.right) << ";\n";
                break;
            }
            case UP_NODE_RESCALE: {
                body << "    u32 " << v(k) << "[" << K << "]; u32 " << s(k) << " = " << s(nd.left) << ";\n";
                if (nd.scale >= f[nd.left].scale) {
                    const std::string A = aligned(nd.left, nd.scale);
                    body << "#pragma unroll\n    for (int i = 0; i < " << K << "; i++) " << v(k) << "[i] = " << A
                         << "[i];\n";
                } else {
                    const Big p = big_pow10(f[nd.left].scale - nd.scale);
                    globals << "__device__ const u32 R" << k << "[" << p.m.size() << "] = "
                            << limbs_init(p, (int)p.m.size()) << ";\n";
                    body << "    tpi_trunc_pow10" << ni() << "<" << tk() << ">(" << v(k) << ", " << v(nd.left) << ", R" << k
                         << ", "
                         << p.m.size() << ");\n";
                }
                break;
            }
            case UP_NODE_DIV: {
                const int sh = f[nd.right].scale + 4;
                const Big p = big_pow10(sh);
                char w[40];
                snprintf(w, sizeof w, "0x%016llxull", (unsigned long long)big_low64(p));
                body << "    u32 " << v(k) << "[" << K << "]; u32 " << s(k) << ";\n";
                body << "    err |= tpi_div_round" << ni() << "<" << tk() << ", " << f[nd.left].limbs << ", " << p.m.size()
                     << ", "
                     << sh << "u, " << w << ">(" << v(k) << ", " << s(k) << ", " << v(nd.left) << ", " << s(nd.left)
                     << ", " << v(nd.right) << ", " << s(nd.right) << ", " << p10_name(sh) << ");\n";
                break;
            }
            case UP_NODE_MOD:
                body << "    u32 " << v(k) << "[" << K << "]; u32 " << s(k) << ";\n";
                body << "    err |= tpi_mod<" << tk() << ">(" << v(k) << ", " << s(k) << ", " << v(nd.left) << ", "
                     << s(nd.left) << ", " << v(nd.right) << ", " << s(nd.right) << ");\n";
                break;
            default: {
                if (nd.kind == UP_NODE_AND || nd.kind == UP_NODE_OR) {
                    body << "    const u32 c" << k << " = c" << nd.left << (nd.kind == UP_NODE_AND ? " & " : " | ") << "c"
                         << nd.right << ";\n";
                    return;
                }
                const int sc = std::max(f[nd.left].scale, f[nd.right].scale);
                const std::string A = aligned(nd.left, sc);
                const std::string Bn = aligned(nd.right, sc);
                body << "    const u32 c" << k << " = tpi_compare<" << tk() << ">(" << (nd.kind - UP_NODE_LT) << ", "
                     << A << ", " << s(nd.left) << ", " << Bn << ", " << s(nd.right) << ");\n";
                return;
            }
        }
        if (nd.reverse) body << "    " << s(k) << " ^= 1u;\n";
    }
    std::string constants() {
        std::ostringstream o;
        for (int d : p10) {
            const Big p = big_pow10(d);
            o << "    const u32 P10_" << d << "[" << p.m.size() << "] = " << limbs_init(p, (int)p.m.size()) << ";\n";
        }
        return o.str();
    }
};

// Automatic cooperative evaluation starts at this width: measured on B200,
// a*b+c at p=600 (127 limbs) runs 1.26x faster cooperatively, while at p=300
// (64 limbs) and p=150 (32 limbs) one thread per value is faster.
constexpr int kCoopMinLimbs = 96;

// Widest limb count a cooperative evaluation of the expression needs (every
// node, every aligned operand, and the headroom of the long divisions), or 0
// when a node kind has no cooperative form.
int cooperative_width(const up_expr_node* nodes, const std::vector<NodeFacts>& f, const std::vector<int>& topo) {
    int w = 1;
    for (int k : topo) {
        const up_expr_node& nd = nodes[k];
        switch (nd.kind) {
            case UP_NODE_COLUMN:
            case UP_NODE_CONST:
            case UP_NODE_INT:
            case UP_NODE_ADD:
            case UP_NODE_SUB:
            case UP_NODE_MUL:
                w = std::max(w, f[k].limbs);
                break;
            case UP_NODE_RESCALE:
                w = std::max(w, f[k].limbs);
                if (nd.scale < f[nd.left].scale) {  // long division by 10^d: one limb of headroom each
                    w = std::max(w, f[nd.left].limbs + 1);
                    w = std::max(w, limbs_for_bits(big_bitlen(big_pow10(f[nd.left].scale - nd.scale))) + 1);
                }
                break;
            case UP_NODE_DIV: {  // dividend scaled by 10^(s_b+4), plus headroom for normalising
                const int np = (int)big_pow10(f[nd.right].scale + 4).m.size();
                w = std::max(w, f[k].limbs);
                w = std::max(w, f[nd.left].limbs + np + 1);
                w = std::max(w, f[nd.right].limbs + 1);
                break;
            }
            case UP_NODE_MOD:
                w = std::max(w, f[k].limbs);
                w = std::max(w, f[nd.left].limbs + 1);
                w = std::max(w, f[nd.right].limbs + 1);
                break;
            default:
                if (!is_compare_kind(nd.kind)) return 0;
                if (nd.kind == UP_NODE_AND || nd.kind == UP_NODE_OR) break;
                {
                    const int sc = std::max(f[nd.left].scale, f[nd.right].scale);
                    for (int o : {nd.left, nd.right}) {
                        const int d = sc - f[o].scale;
                        w = std::max(w, limbs_for_bits(f[o].bits + (d > 0 ? big_bitlen(big_pow10(d)) : 0)));
                    }
                }
        }
    }
    return w;
}

}  // namespace

// The width rule for threads per value (non-nullable inputs): cooperative
// from kCoopMinLimbs limbs, with the smallest group of at most 8 limbs per
// thread, except for divisions, which one thread per value runs 2-5x faster
// on B200 (each long-division step costs a group several broadcasts and
// ballots).  Automatic threads per value: with a learned cost model set, the
// model's choice (ultraprecise_costmodel.h), else the rule.  Both return 1
// for one thread per value.
int rule_threads_per_value(const up_expr_node* nodes, const std::vector<NodeFacts>& f, const std::vector<int>& topo) {
    const int w = cooperative_width(nodes, f, topo);
    if (w <= 0) return 1;
    bool has_div = false;
    for (int k : topo)
        has_div |= nodes[k].kind == UP_NODE_DIV || nodes[k].kind == UP_NODE_MOD ||
                   (nodes[k].kind == UP_NODE_RESCALE && nodes[k].scale < f[nodes[k].left].scale);
    if (w < kCoopMinLimbs || has_div) return 1;
    int t = 2;
    while (t < 32 && t * 8 < w) t *= 2;
    return t;
}

int auto_threads_per_value(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols, int n_cols,
                           const std::vector<NodeFacts>& f, const std::vector<int>& topo) {
    if (cooperative_width(nodes, f, topo) <= 0) return 1;
    const CostChoice cc = default_model_choose_tpv(nodes, n_nodes, root, cols, n_cols);
    if (cc.valid) return cc.tpv > 1 ? cc.tpv : 1;
    return rule_threads_per_value(nodes, f, topo);
}

int coop_width_of(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols, int n_cols) {
    std::vector<NodeFacts> f;
    std::vector<int> topo;
    if (analyze_nodes(nodes, n_nodes, cols, n_cols, f, topo, {root}) != UP_OK) return 0;
    return cooperative_width(nodes, f, topo);
}

// ------------------------------------------------- cost-model features
// Features of launching an expression (ultraprecise_costmodel.h): what the
// generated kernel's run time depends on — rows, threads per value, limb
// widths, the multiply and divide work per row, bytes moved per row.
up_status expr_cost_features(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols, int n_cols,
                             int tpv, int64_t rows, float* out, bool* coop_ok) {
    std::vector<NodeFacts> f;
    std::vector<int> topo;
    up_status st = analyze_nodes(nodes, n_nodes, cols, n_cols, f, topo, {root});
    if (st != UP_OK) return st;
    bool any_nullable = false;
    std::vector<int> used;
    int max_limbs = 1, n_mul = 0, n_div = 0, n_add = 0, div_limbs = 0;
    double mul_work = 0, div_work = 0;
    for (int k : topo) {
        const up_expr_node& nd = nodes[k];
        max_limbs = std::max(max_limbs, f[k].limbs);
        switch (nd.kind) {
            case UP_NODE_COLUMN:
                if (std::find(used.begin(), used.end(), nd.column) == used.end()) used.push_back(nd.column);
                any_nullable |= cols[nd.column].nullable != 0;
                break;
            case UP_NODE_MUL:
                n_mul++;
                mul_work += (double)f[nd.left].limbs * f[nd.right].limbs;
                break;
            case UP_NODE_DIV:
            case UP_NODE_MOD: {
                n_div++;
                const int lb = f[nd.right].limbs;
                div_limbs = std::max(div_limbs, lb);
                const int lx = nd.kind == UP_NODE_DIV
                                   ? f[nd.left].limbs + limbs_for_bits(big_bitlen(big_pow10(f[nd.right].scale + 4)))
                                   : f[nd.left].limbs;
                div_work += (double)(lx - f[nd.left].limbs) * f[nd.left].limbs + (double)std::max(1, lx - lb + 1) * lb;
                break;
            }
            case UP_NODE_RESCALE:
                if (nd.scale < f[nd.left].scale) {
                    n_div++;
                    const int lp = limbs_for_bits(big_bitlen(big_pow10(f[nd.left].scale - nd.scale)));
                    div_limbs = std::max(div_limbs, lp);
                    div_work += (double)std::max(1, f[nd.left].limbs - lp + 1) * lp;
                }
                break;
            case UP_NODE_ADD:
            case UP_NODE_SUB:
                n_add++;
                break;
            default:
                break;
        }
    }
    const bool cmp_root = is_compare_kind(nodes[root].kind);
    const int out_bytes = cmp_root ? 1 : compact_bytes(nodes[root].precision);
    int in_bytes = 0;
    for (int c : used) in_bytes += compact_bytes(cols[c].precision);
    const int w = cooperative_width(nodes, f, topo);
    if (coop_ok) *coop_ok = w > 0 && !any_nullable;
    const double T = std::max(1, tpv);
    const double work = mul_work + div_work + (double)n_add * max_limbs;
    auto lg = [](double x) { return (float)std::log2(std::max(x, 1.0)); };
    float* o = out;
    o[0] = lg((double)std::max<int64_t>(rows, 1));
    o[1] = lg(T);
    o[2] = lg(max_limbs);
    o[3] = lg(limbs_for_bits(std::max(1, 8 * out_bytes)));
    o[4] = lg(1.0 + mul_work);
    o[5] = lg(1.0 + div_work);
    o[6] = (float)n_mul;
    o[7] = (float)n_div;
    o[8] = (float)n_add;
    o[9] = lg(std::max(1, in_bytes));
    o[10] = lg(out_bytes);
    o[11] = n_div > 0 ? 1.f : 0.f;
    o[12] = lg(std::max(1, div_limbs));
    o[13] = lg(1.0 + work / T);
    o[14] = o[0] + lg(1.0 + work);
    o[15] = lg(tpv > 1 && w > 0 ? std::ceil((double)w / T) : (double)max_limbs);
    return UP_OK;
}

// --------------------------------------------------- expression modules
up_status generate_expr_module(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols,
                               int n_cols, const up_compile_opts* opts, GeneratedModule& out) {
    if (!nodes || n_nodes <= 0) return fail(UP_ERR_INVALID_ARG, "empty expression");
    if (n_cols < 0 || n_cols > 16) return fail(UP_ERR_INVALID_ARG, "at most 16 input columns");
    if (n_cols > 0 && !cols) return fail(UP_ERR_INVALID_ARG, "column types missing");
    std::vector<NodeFacts> f;
    std::vector<int> topo;
    up_status st = analyze_nodes(nodes, n_nodes, cols, n_cols, f, topo, {root});
    if (st != UP_OK) return st;
    const up_expr_node& rn = nodes[root];
    const bool cmp_root = is_compare_kind(rn.kind);
    int out_p = cmp_root ? 1 : rn.precision;
    int out_s = cmp_root ? 0 : f[root].scale;
    int BO = cmp_root ? 1 : compact_bytes(out_p);
    if (!cmp_root && BO < 1) return fail(UP_ERR_INVALID_ARG, "root precision not set (run up_expr_derive_types)");
    for (int k : topo) {
        if (f[k].limbs > 512) return fail(UP_ERR_UNSUPPORTED, "intermediate wider than 16384 bits");
    }

    std::vector<int> used;
    bool any_nullable = false;
    for (int k : topo)
        if (nodes[k].kind == UP_NODE_COLUMN) {
            if (std::find(used.begin(), used.end(), nodes[k].column) == used.end()) used.push_back(nodes[k].column);
            any_nullable |= cols[nodes[k].column].nullable != 0;
        }
    std::sort(used.begin(), used.end());

    Emitter em(nodes, cols, f);
    em.plan(topo);
    for (int k : topo) em.node(k);

    int T = (opts && opts->block_threads > 0) ? opts->block_threads : 256;
    int row_bytes = BO;
    for (int c : used) row_bytes += compact_bytes(cols[c].precision);
    // Narrow rows: two pipeline stages of R rows (inputs + outputs) within
    // ~48 KB of shared memory, R a power of two in [128, 1024], moved by bulk
    // copies.  Wide rows: one synchronously staged tile of R rows (R >= 32)
    // and a CTA of min(256, R) threads, so no thread idles at the barriers.
    int R = 1024;
    while (R > 128 && 2L * R * row_bytes > 48 * 1024) R /= 2;
    const bool staged = 2L * R * row_bytes <= 48 * 1024;
    if (!staged) {
        R = 1024;
        while (R > 32 && (long)R * row_bytes > 48 * 1024) R /= 2;
    }
    if (T > R) T = R;
    std::ostringstream src;
    src << "#include \"up_dev.cuh\"\nusing namespace up;\n" << kargs_source();
    src << "UP_DI u32 up_row(" << params_decl(used) << "u8* __restrict__ out, const bool words) {\n";
    src << "    u32 err = 0u;\n" << em.constants() << em.body.str();
    if (cmp_root) {
        src << "    out[0] = (u8)c" << root << ";\n";
    } else if (BO % 4 == 0) {
        src << "    if (words) err |= st_compact_words<" << BO << ">(out, v" << root << ", s" << root << ");\n";
        src << "    else err |= st_compact_bytes<" << BO << ">(out, v" << root << ", s" << root << ");\n";
    } else {
        src << "    err |= st_compact_bytes<" << BO << ">(out, v" << root << ", s" << root << ");\n";
    }
    src << "    return err;\n}\n\n";

    // Cooperative evaluation for wide expressions: T threads per value, K
    // limbs each (threads_per_value 0 = automatic: K = 8 and the smallest T
    // covering the widest intermediate, for expressions of at least kCoopMinLimbs limbs;
    // 1 = one thread per value).
    int tpiT = 0, tpiK = 0;
    {
        const int req = opts ? opts->threads_per_value : 0;
        const int w = cooperative_width(nodes, f, topo);
        if (req > 1 && w > 0 && !any_nullable) {
            if (req != 2 && req != 4 && req != 8 && req != 16 && req != 32)
                return fail(UP_ERR_INVALID_ARG, "threads_per_value must be 1, 2, 4, 8, 16 or 32");
            tpiT = req;
        } else if (req == 0 && !any_nullable) {
            const int t = auto_threads_per_value(nodes, n_nodes, root, cols, n_cols, f, topo);
            if (t > 1) tpiT = t;
        }
        if (tpiT > 0) tpiK = (w + tpiT - 1) / tpiT;
    }
    out.threads_per_value = tpiT > 0 ? tpiT : 1;

    // tile kernel: contiguous columns
    int smem = 0;
    if (tpiT > 0) {
        TEmitter te(nodes, cols, f, tpiT, tpiK);
        te.words = true;  // the columns are read from the staged tile below (padded by 16 bytes)
        te.plan(topo);
        for (int k : topo) te.node(k);
        const int CT = 256;               // CTA threads
        const int G = CT / tpiT;          // values in flight per CTA
        R = 1024;
        while (R > 16 && (long)R * row_bytes > 32 * 1024) R /= 2;
        std::vector<int> off;
        for (int c : used) {
            off.push_back(smem);
            smem += ((R * compact_bytes(cols[c].precision) + 16 + 15) / 16) * 16;
        }
        const int off_out = smem;
        smem += ((R * BO + 16 + 15) / 16) * 16;
        src << te.globals.str();
        src << "UP_DI u32 up_trow(" << params_decl(used) << "u8* __restrict__ out, const bool store) {\n";
        src << "    u32 err = 0u;\n" << te.constants() << te.body.str();
        if (cmp_root)
            src << "    if (store && tpi_rank<" << tpiT << ">() == 0) out[0] = (u8)c" << root << ";\n";
        else
            src << "    err |= tpi_st<" << tpiT << ", " << tpiK << ", " << BO << ">(out, v" << root << ", s" << root
                << ", store);\n";
        src << "    return err;\n}\n\n";
        // four CTAs per SM (at most 64 registers): measured on B200, p=600
        // a*b+c at 16 threads per value 2.27 -> 2.17 ms
        src << "extern \"C\" __global__ void __launch_bounds__(" << CT << ", 4) up_expr_tile(const UpArgs a) {\n";
        src << "    extern __shared__ __align__(16) u8 sm[];\n";
        src << "    constexpr int R = " << R << ";\n    constexpr int G = " << G << ";\n";
        src << "    const int grp = (int)threadIdx.x / " << tpiT << ";\n";
        src << "    const i64 ntiles = (a.rows + R - 1) / R;\n    u32 err = 0u;\n";
        src << "    for (i64 t = blockIdx.x; t < ntiles; t += gridDim.x) {\n";
        src << "        const i64 row0 = t * (i64)R;\n";
        src << "        const int nr = (a.rows - row0) < R ? (int)(a.rows - row0) : R;\n";
        for (size_t i = 0; i < used.size(); i++) {
            const int cc = used[i];
            const int B = compact_bytes(cols[cc].precision);
            src << "        tile_copy_in(sm + " << off[i] << ", a.col[" << cc << "].data + row0 * " << B << ", nr * " << B
                << ", a.vec_ok != 0);\n";
        }
        src << "        __syncthreads();\n";
        src << "        // every group runs the same number of slots, so warps stay converged around the shuffles\n";
        src << "        for (int base = 0; base < nr; base += G) {\n";
        src << "            const int r = base + grp;\n            const bool valid = r < nr;\n";
        src << "            const int rr = valid ? r : 0;\n";
        src << "            const u32 e = up_trow(";
        for (size_t i = 0; i < used.size(); i++)
            src << "sm + " << off[i] << " + rr * " << compact_bytes(cols[used[i]].precision) << ", ";
        src << "sm + " << off_out << " + rr * " << BO << ", valid);\n";
        src << "            if (valid) err |= e;\n        }\n";
        src << "        __syncthreads();\n";
        src << "        tile_copy_out(a.out + row0 * " << BO << ", sm + " << off_out << ", nr * " << BO
            << ", a.vec_ok != 0);\n";
        src << "        __syncthreads();\n    }\n";
        T = CT;
    } else if (staged) {
        // double-buffered bulk-copy pipeline: stage k&1 holds tile k's inputs;
        // the next tile's loads are issued before the current tile is
        // computed; outputs leave through a bulk store from a double buffer
        std::vector<int> off;
        for (int c : used) {
            off.push_back(smem);
            smem += ((R * compact_bytes(cols[c].precision) + 16 + 15) / 16) * 16;
        }
        const int stage_in = smem;
        const int out_bytes = ((R * BO + 16 + 15) / 16) * 16;
        const int off_out = 2 * stage_in;
        const int off_bar = off_out + 2 * out_bytes;
        smem = off_bar + 16;
        int tile_in_bytes = 0;
        for (int c : used) tile_in_bytes += R * compact_bytes(cols[c].precision);
        src << "extern \"C\" __global__ void __launch_bounds__(" << T << ") up_expr_tile(const UpArgs a) {\n";
        src << "    extern __shared__ __align__(128) u8 sm[];\n";
        src << "    constexpr int R = " << R << ";\n";
        src << "    u64* bar = (u64*)(sm + " << off_bar << ");\n";
        src << "    const i64 ntiles = (a.rows + R - 1) / R;\n";
        src << "    const i64 nfull = a.vec_ok ? a.rows / R : 0;  // tiles moved by bulk copies\n";
        src << "    u32 err = 0u;\n";
        src << "    if (threadIdx.x == 0) { mbar_init(&bar[0], 1); mbar_init(&bar[1], 1); mbar_init_fence(); }\n";
        src << "    __syncthreads();\n";
        src << "    auto issue = [&](i64 tt, int st) {\n";
        src << "        mbar_expect_tx(&bar[st], " << tile_in_bytes << "u);\n";
        for (size_t i = 0; i < used.size(); i++) {
            int c = used[i];
            int B = compact_bytes(cols[c].precision);
            src << "        bulk_load(sm + st * " << stage_in << " + " << off[i] << ", a.col[" << c
                << "].data + tt * (i64)(R * " << B << "), " << R * B << "u, &bar[st]);\n";
        }
        src << "    };\n";
        src << "    if (threadIdx.x == 0 && (i64)blockIdx.x < nfull) issue(blockIdx.x, 0);\n";
        src << "    int k = 0;\n";
        src << "    bool timed_out = false;\n    int to_st = 0;\n    u32 to_par = 0u;\n";
        src << "    for (i64 t = blockIdx.x; t < ntiles; t += gridDim.x, k++) {\n";
        src << "        const int st = k & 1;\n";
        src << "        const i64 row0 = t * (i64)R;\n";
        src << "        const int nr = (a.rows - row0) < R ? (int)(a.rows - row0) : R;\n";
        src << "        const bool bulk = t < nfull;\n";
        src << "        const i64 tn = t + gridDim.x;\n";
        src << "        if (threadIdx.x == 0 && tn < nfull) issue(tn, st ^ 1);\n";
        src << "        u8* in = sm + st * " << stage_in << ";\n";
        src << "        u8* ob = sm + " << off_out << " + st * " << out_bytes << ";\n";
        src << "        if (bulk) {\n";
        src << "            if (!mbar_wait(&bar[st], (u32)((k >> 1) & 1))) { timed_out = true; to_st = st; to_par = (u32)((k >> 1) & 1); }\n";
        src << "        } else {\n";
        for (size_t i = 0; i < used.size(); i++) {
            int c = used[i];
            int B = compact_bytes(cols[c].precision);
            src << "            tile_copy_in(in + " << off[i] << ", a.col[" << c << "].data + row0 * " << B << ", nr * "
                << B << ", a.vec_ok != 0);\n";
        }
        src << "            __syncthreads();\n";
        src << "        }\n";
        src << "        if (__syncthreads_or(timed_out)) break;\n";
        src << "        for (int r = threadIdx.x; r < nr; r += blockDim.x)\n";
        src << "            err |= up_row(";
        for (size_t i = 0; i < used.size(); i++) {
            int B = compact_bytes(cols[used[i]].precision);
            src << "in + " << off[i] << " + r * " << B << ", ";
        }
        src << "ob + r * " << BO << ", true);\n";
        src << "        if (bulk) {\n";
        src << "            fence_async_smem();\n";
        src << "            __syncthreads();\n";
        src << "            if (threadIdx.x == 0) {\n";
        src << "                bulk_store(a.out + row0 * " << BO << ", ob, " << R * BO << "u);\n";
        src << "                bulk_commit();\n";
        src << "                bulk_wait_read_1();\n";
        src << "            }\n";
        src << "        } else {\n";
        src << "            __syncthreads();\n";
        src << "            tile_copy_out(a.out + row0 * " << BO << ", ob, nr * " << BO << ", a.vec_ok != 0);\n";
        src << "        }\n";
        src << "        __syncthreads();\n";
        src << "    }\n";
        src << "    if (threadIdx.x == 0) {\n";
        src << "        bulk_wait_all();\n";
        src << "        if (timed_out) {\n";
        src << "            err |= ERR_TIMEOUT;\n";
        src << "            mbar_wait(&bar[to_st], to_par);  // bounded: let copies in flight land before exit\n";
        src << "        }\n";
        src << "    }\n";
    } else {
        // one synchronously staged tile per iteration (wide rows)
        std::vector<int> off;
        for (int c : used) {
            off.push_back(smem);
            smem += ((R * compact_bytes(cols[c].precision) + 16 + 15) / 16) * 16;
        }
        const int off_out = smem;
        smem += ((R * BO + 16 + 15) / 16) * 16;
        // Minimum resident CTAs per SM, measured on B200.  The widest rows
        // stage 64 per tile in a 64-thread CTA: six per SM caps registers at
        // 168 (p=300 a*b+c 1.50 -> 1.40 ms, p=600 a/b 1.24 -> 1.14 ms).
        // 128-thread CTAs without a division: five per SM, 102 registers
        // (p=150 a*b+c 0.636 -> 0.547 ms); with divisions the cap spills into
        // the local memory the digit loop already waits on (p=300 a/b 0.75
        // -> 0.81 ms), so none is asked for.
        bool has_div = false;
        for (int k : topo)
            has_div |= nodes[k].kind == UP_NODE_DIV || nodes[k].kind == UP_NODE_MOD ||
                       (nodes[k].kind == UP_NODE_RESCALE && nodes[k].scale < f[nodes[k].left].scale);
        const char* min_ctas = T <= 64 ? ", 6" : (T == 128 && !has_div ? ", 5" : "");
        src << "extern \"C\" __global__ void __launch_bounds__(" << T << min_ctas
            << ") up_expr_tile(const UpArgs a) {\n";
        src << "    extern __shared__ __align__(16) u8 sm[];\n";
        src << "    constexpr int R = " << R << ";\n";
        src << "    const i64 ntiles = (a.rows + R - 1) / R;\n    u32 err = 0u;\n";
        src << "    for (i64 t = blockIdx.x; t < ntiles; t += gridDim.x) {\n";
        src << "        const i64 row0 = t * (i64)R;\n";
        src << "        const int nr = (a.rows - row0) < R ? (int)(a.rows - row0) : R;\n";
        for (size_t i = 0; i < used.size(); i++) {
            int c = used[i];
            int B = compact_bytes(cols[c].precision);
            src << "        tile_copy_in(sm + " << off[i] << ", a.col[" << c << "].data + row0 * " << B << ", nr * "
                << B << ", a.vec_ok != 0);\n";
        }
        src << "        __syncthreads();\n";
        src << "        for (int r = threadIdx.x; r < nr; r += blockDim.x)\n";
        src << "            err |= up_row(";
        for (size_t i = 0; i < used.size(); i++) {
            int B = compact_bytes(cols[used[i]].precision);
            src << "sm + " << off[i] << " + r * " << B << ", ";
        }
        src << "sm + " << off_out << " + r * " << BO << ", true);\n";
        src << "        __syncthreads();\n";
        src << "        tile_copy_out(a.out + row0 * " << BO << ", sm + " << off_out << ", nr * " << BO
            << ", a.vec_ok != 0);\n";
        src << "        __syncthreads();\n    }\n";
    }
    src << "    err = __reduce_or_sync(0xffffffffu, err);\n";
    src << "    if ((threadIdx.x & 31) == 0 && err != 0u && a.err) atomicOr(a.err, err);\n}\n\n";

    // Merged launches (the serving loop): one kernel over several requests of
    // this module; virtual tiles of RM rows map to their request by a binary
    // search over the requests' first tiles; each tile is staged synchronously.
    out.multi_rows = 0;
    if (tpiT == 0 && !any_nullable && !em.out_of_line) {
        int RM = 1024;
        while (RM > 32 && (long)RM * row_bytes > 24 * 1024) RM /= 2;
        std::vector<int> moff;
        int msm = 0;
        for (int c : used) {
            moff.push_back(msm);
            msm += ((RM * compact_bytes(cols[c].precision) + 16 + 15) / 16) * 16;
        }
        const int moff_out = msm;
        msm += ((RM * BO + 16 + 15) / 16) * 16;
        const int TM = std::min(256, RM);
        src << "extern \"C\" __global__ void __launch_bounds__(" << TM << ") up_expr_multi(const UpMultiArgs a) {\n";
        src << "    extern __shared__ __align__(16) u8 sm[];\n";
        src << "    constexpr int R = " << RM << ";\n";
        src << "    for (i64 t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {\n";
        src << "        int lo = 0, hi = a.n_req - 1;\n";
        src << "        while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (a.req[mid].tile0 <= t) lo = mid; else hi = mid - 1; }\n";
        src << "        const UpMultiReq& q = a.req[lo];\n";
        src << "        const i64 row0 = (t - q.tile0) * (i64)R;\n";
        src << "        const int nr = (q.rows - row0) < R ? (int)(q.rows - row0) : R;\n";
        for (size_t i = 0; i < used.size(); i++) {
            const int c = used[i];
            const int B = compact_bytes(cols[c].precision);
            src << "        tile_copy_in(sm + " << moff[i] << ", q.col[" << c << "].data + row0 * " << B << ", nr * " << B
                << ", q.vec_ok != 0);\n";
        }
        src << "        __syncthreads();\n        u32 err = 0u;\n";
        src << "        for (int r = threadIdx.x; r < nr; r += blockDim.x)\n            err |= up_row(";
        for (size_t i = 0; i < used.size(); i++)
            src << "sm + " << moff[i] << " + r * " << compact_bytes(cols[used[i]].precision) << ", ";
        src << "sm + " << moff_out << " + r * " << BO << ", true);\n";
        src << "        __syncthreads();\n";
        src << "        tile_copy_out(q.out + row0 * " << BO << ", sm + " << moff_out << ", nr * " << BO
            << ", q.vec_ok != 0);\n";
        src << "        err = __reduce_or_sync(0xffffffffu, err);\n";
        src << "        if ((threadIdx.x & 31) == 0 && err != 0u && q.err) atomicOr(q.err, err);\n";
        src << "        __syncthreads();\n    }\n}\n\n";
        out.multi_rows = RM;
        out.multi_threads = TM;
        out.multi_smem = msm;
    }

    // generic kernel: blocks, indirection, nullable values
    const int OB = BO + (any_nullable ? 1 : 0);
    src << "extern \"C\" __global__ void __launch_bounds__(" << T << ") up_expr_generic(const UpArgs a) {\n";
    src << "    u32 err = 0u;\n";
    src << "    const i64 stride = (i64)gridDim.x * blockDim.x;\n";
    src << "    for (i64 row = (i64)blockIdx.x * blockDim.x + threadIdx.x; row < a.rows; row += stride) {\n";
    src << "        u8* o = a.out + row * " << OB << ";\n";
    src << "        bool isnull = false;\n";
    for (int c : used) {
        src << "        const u8* in" << c << " = col_ptr(a.col[" << c << "], row);\n";
        src << "        if (in" << c << " == nullptr) isnull = true;\n";
        if (cols[c].nullable) {
            src << "        else { if (in" << c << "[0] == 0) isnull = true; in" << c << " += 1; }\n";
        }
    }
    if (any_nullable) {
        src << "        o[0] = isnull ? 0 : 1;\n";
        src << "        if (isnull) { for (int i = 0; i < " << BO << "; i++) o[1 + i] = 0; continue; }\n";
        src << "        o += 1;\n";
    } else {
        src << "        if (isnull) { err |= ERR_DOMAIN; for (int i = 0; i < " << BO << "; i++) o[i] = 0; continue; }\n";
    }
    src << "        err |= up_row(";
    for (int c : used) src << "in" << c << ", ";
    src << "o, false);\n    }\n";
    src << "    err = __reduce_or_sync(0xffffffffu, err);\n";
    src << "    if ((threadIdx.x & 31) == 0 && err != 0u && a.err) atomicOr(a.err, err);\n}\n";

    out.source = src.str();
    out.kernels = {"up_expr_tile", "up_expr_generic"};
    if (out.multi_rows > 0) out.kernels.push_back("up_expr_multi");
    out.work_per_row = em.work + row_bytes;
    out.out_precision = out_p;
    out.out_scale = out_s;
    out.out_bytes = OB;
    out.out_is_compare = cmp_root;
    out.block_threads = T;
    out.tile_rows = R;
    out.smem_bytes = smem;
    out.in_bytes.assign(n_cols, 0);
    for (int c = 0; c < n_cols; c++) out.in_bytes[c] = compact_bytes(cols[c].precision) + (cols[c].nullable ? 1 : 0);
    return UP_OK;
}

// ------------------------------------------------------ query modules
// Fused expression + grouped aggregation: every aggregate's expression is
// evaluated per row and added exactly into per-group two's complement
// accumulators (SUM/AVG), with a per-group row count; a second kernel turns
// the accumulators into the reference's 133-byte nullable_type<Decimal>
// images (AggregateColumnData SUM, AriesSqlOperator_group.cu:360-424, and
// DivisionInt64 AVG, AriesSqlOperator_helpers.cu:717-763).
up_status generate_query_module(const up_expr_node* nodes, int n_nodes, const up_col_type* cols, int n_cols,
                                const up_query_agg* aggs, int n_aggs, const up_compile_opts* opts,
                                GeneratedModule& out) {
    if (!nodes || n_nodes <= 0) return fail(UP_ERR_INVALID_ARG, "empty query");
    if (n_aggs <= 0 || n_aggs > 16) return fail(UP_ERR_INVALID_ARG, "1..16 aggregates");
    if (n_cols < 0 || n_cols > 16) return fail(UP_ERR_INVALID_ARG, "at most 16 input columns");
    std::vector<int> roots;
    for (int a = 0; a < n_aggs; a++) {
        int k = aggs[a].kind;
        if (k != UP_AGG_COUNT && k != UP_AGG_SUM && k != UP_AGG_AVG)
            return fail(UP_ERR_INVALID_ARG, "unknown aggregate kind");
        if (k != UP_AGG_COUNT) roots.push_back(aggs[a].root);
    }
    std::vector<NodeFacts> f;
    std::vector<int> topo;
    if (!roots.empty()) {
        up_status st = analyze_nodes(nodes, n_nodes, cols, n_cols, f, topo, roots);
        if (st != UP_OK) return st;
    }
    for (int r : roots)
        if (f[r].is_compare) return fail(UP_ERR_INVALID_ARG, "cannot sum a comparison");

    std::vector<int> used;
    for (int k : topo)
        if (nodes[k].kind == UP_NODE_COLUMN &&
            std::find(used.begin(), used.end(), nodes[k].column) == used.end())
            used.push_back(nodes[k].column);
    std::sort(used.begin(), used.end());

    out.n_aggs = n_aggs;
    out.agg_kind.clear();
    out.agg_scale.clear();
    out.agg_acc_limbs.clear();
    out.agg_acc_offset.clear();
    // one accumulator per distinct aggregated expression (SUM(x) and AVG(x)
    // share one), sized for a sign bit and 2^40 rows above the value bound
    std::vector<int> acc_root, acc_limbs, acc_off;
    std::vector<int> agg_slot(n_aggs, -1);
    int accw = 0;
    for (int a = 0; a < n_aggs; a++) {
        out.agg_kind.push_back(aggs[a].kind);
        if (aggs[a].kind == UP_AGG_COUNT) {
            out.agg_scale.push_back(0);
            out.agg_acc_limbs.push_back(0);
            out.agg_acc_offset.push_back(0);
            continue;
        }
        const int r = aggs[a].root;
        const NodeFacts& fr = f[r];
        const int nacc = limbs_for_bits(fr.bits + 1 + 40);
        int slot = (int)(std::find(acc_root.begin(), acc_root.end(), r) - acc_root.begin());
        if (slot == (int)acc_root.size()) {
            acc_root.push_back(r);
            acc_limbs.push_back(nacc);
            acc_off.push_back(accw);
            accw += nacc;
        }
        out.agg_scale.push_back(fr.scale);
        out.agg_acc_limbs.push_back(nacc);
        out.agg_acc_offset.push_back(acc_off[slot]);
        agg_slot[a] = slot;
    }
    const int NR = (int)acc_root.size();
    // Nullable columns take SQL's aggregate semantics (agg_sum_t on
    // nullable_type, operators.hxx:1176-1193; COUNT of a nullable column
    // counts its non-null rows, AriesEngineAlgorithm.h:725-736): a row adds to
    // SUM/AVG of an expression only when none of that expression's columns is
    // NULL, and every accumulator keeps its own count of those rows (two words
    // per accumulator after a group's accumulators) for the SUM flag and the
    // AVG divisor.  COUNT stays the group's row count (COUNT(*)).
    bool any_nullable = false;
    for (int c : used) any_nullable |= cols[c].nullable != 0;
    std::vector<int> cnt_off;
    if (any_nullable) {
        for (int i = 0; i < NR; i++) cnt_off.push_back(accw + 2 * i);
        accw += 2 * NR;
    }
    out.acc_words_per_group = accw;

    Emitter em(nodes, cols, f);
    em.plan(topo);
    for (int k : topo) em.node(k);

    const int T = (opts && opts->block_threads > 0) ? opts->block_threads : 256;
    std::ostringstream src;
    src << "#include \"up_dev.cuh\"\nusing namespace up;\n" << query_kargs_source();
    // per row: every accumulated expression as a two's complement image
    src << "UP_DI u32 up_qvals(" << params_decl(used) << "const bool words";
    for (int i = 0; i < NR; i++) src << ", u32 (&qv" << i << ")[" << acc_limbs[i] << "]";
    src << ") {\n    u32 err = 0u;\n" << em.constants() << em.body.str();
    for (int i = 0; i < NR; i++)
        src << "    to_twos(qv" << i << ", v" << acc_root[i] << ", s" << acc_root[i] << ");\n";
    src << "    return err;\n}\n\n";
    auto decl_t = [&](const std::string& ind) {
        std::string d;
        for (int i = 0; i < NR; i++) d += ind + "u32 qv" + std::to_string(i) + "[" + std::to_string(acc_limbs[i]) + "];\n";
        return d;
    };
    auto targs = [&]() {
        std::string d;
        for (int i = 0; i < NR; i++) d += ", qv" + std::to_string(i);
        return d;
    };
    const int W = std::max(accw, 1);
    std::vector<std::pair<std::string, std::string>> qval_calls;  // per accumulator: NULL test, arguments

    // generic kernel: blocks, indirection, nullable values; global accumulators
    if (any_nullable) {
        // one evaluation function per accumulated expression, over its own
        // columns, so that a NULL in one expression's columns leaves the others
        for (int i = 0; i < NR; i++) {
            std::vector<int> sub;
            std::vector<char> reach(n_nodes, 0);
            reach[acc_root[i]] = 1;
            for (auto it = topo.rbegin(); it != topo.rend(); ++it) {
                if (!reach[*it]) continue;
                const up_expr_node& nd = nodes[*it];
                if (nd.left >= 0) reach[nd.left] = 1;
                if (nd.right >= 0) reach[nd.right] = 1;
            }
            std::vector<int> sub_cols;
            for (int k : topo)
                if (reach[k]) {
                    sub.push_back(k);
                    if (nodes[k].kind == UP_NODE_COLUMN &&
                        std::find(sub_cols.begin(), sub_cols.end(), nodes[k].column) == sub_cols.end())
                        sub_cols.push_back(nodes[k].column);
                }
            std::sort(sub_cols.begin(), sub_cols.end());
            Emitter ei(nodes, cols, f);
            ei.plan(sub);
            for (int k : sub) ei.node(k);
            src << "UP_DI u32 up_qval" << i << "(" << params_decl(sub_cols) << "const bool words, u32 (&qv)["
                << acc_limbs[i] << "]) {\n    u32 err = 0u;\n" << ei.constants() << ei.body.str();
            src << "    to_twos(qv, v" << acc_root[i] << ", s" << acc_root[i] << ");\n    return err;\n}\n\n";
            std::string null_test = "false", args;
            for (int c : sub_cols) {
                null_test += " || n" + std::to_string(c);
                args += "in" + std::to_string(c) + ", ";
            }
            qval_calls.push_back({null_test, args});
        }
    }
    src << "extern \"C\" __global__ void __launch_bounds__(" << T << ") up_query_acc(const UpQArgs a) {\n";
    src << "    u32 err = 0u;\n";
    src << "    const int ngr = q_groups(a);\n";
    src << "    if (ngr < 0) { if (threadIdx.x == 0 && blockIdx.x == 0 && a.err) atomicOr(a.err, ERR_DOMAIN); return; }\n";
    src << "    const i64 stride = (i64)gridDim.x * blockDim.x;\n";
    src << "    for (i64 row = (i64)blockIdx.x * blockDim.x + threadIdx.x; row < a.rows; row += stride) {\n";
    src << "        const int g = q_group(a, row);\n";
    src << "        if ((unsigned)g >= (unsigned)ngr) { err |= ERR_DOMAIN; continue; }\n";
    if (any_nullable) {
        // NULL: a nullable column's flag byte is 0, or a -1 row index
        for (int c : used) {
            src << "        const u8* in" << c << " = col_ptr(a.col[" << c << "], row);\n";
            src << "        bool n" << c << " = in" << c << " == nullptr;\n";
            if (cols[c].nullable)
                src << "        if (!n" << c << ") { n" << c << " = in" << c << "[0] == 0; in" << c << " += 1; }\n";
        }
        src << "        atomicAdd(a.cnt + g, 1ull);\n";
        for (int i = 0; i < NR; i++) {
            src << "        if (!(" << qval_calls[i].first << ")) {\n";
            src << "            u32 qv[" << acc_limbs[i] << "];\n";
            src << "            err |= up_qval" << i << "(" << qval_calls[i].second << "false, qv);\n";
            src << "            atomic_add_twos(a.acc + (i64)g * " << W << " + " << acc_off[i] << ", qv);\n";
            src << "            const u32 one[2] = {1u, 0u};\n";
            src << "            atomic_add_twos(a.acc + (i64)g * " << W << " + " << cnt_off[i] << ", one);\n";
            src << "        }\n";
        }
    } else {
        // a -1 row index on a column that is not nullable is outside the domain
        src << "        bool isnull = false;\n";
        for (int c : used) {
            src << "        const u8* in" << c << " = col_ptr(a.col[" << c << "], row);\n";
            src << "        if (in" << c << " == nullptr) isnull = true;\n";
        }
        src << "        if (isnull) { err |= ERR_DOMAIN; continue; }\n";
        src << "        atomicAdd(a.cnt + g, 1ull);\n";
        src << decl_t("        ");
        src << "        err |= up_qvals(";
        for (int c : used) src << "in" << c << ", ";
        src << "false" << targs() << ");\n";
        for (int i = 0; i < NR; i++)
            src << "        atomic_add_twos(a.acc + (i64)g * " << W << " + " << acc_off[i] << ", qv" << i << ");\n";
    }
    src << "    }\n";
    src << "    err = __reduce_or_sync(0xffffffffu, err);\n";
    src << "    if ((threadIdx.x & 31) == 0 && err != 0u && a.err) atomicOr(a.err, err);\n}\n\n";

    // Tile kernels (contiguous non-null columns): the decimal columns and the
    // group ids stream through shared memory by double-buffered bulk copies;
    // the accumulation strategy depends on the group count (chosen at launch):
    //   _r  per-thread register accumulators for the first GR groups, merged
    //       once per thread into shared memory and once per CTA into global;
    //   _s  per-CTA shared-memory accumulators (up to GS groups), merged once
    //       per CTA into global;
    //   _g  global accumulators (many groups: little contention).
    int row_bytes = 4;
    for (int c : used) row_bytes += compact_bytes(cols[c].precision);
    int R = 1024;
    while (R > 128 && 2L * R * row_bytes > 32 * 1024) R /= 2;
    const bool staged = 2L * R * row_bytes <= 32 * 1024 && !any_nullable;
    // register mode keeps per group a count and, per accumulator, its full
    // width when that is at most 4 limbs, else a 128-bit fast accumulator
    int reg_words = 1;
    for (int n : acc_limbs) reg_words += std::min(n, 4);
    int GR = 0;
    while (GR < 8 && (GR + 1) * reg_words <= 96) GR++;
    // a second register-mode kernel for fewer groups (the largest power of
    // two below GR): a row then runs the predicated updates of fewer groups
    int GRL = 0;
    if (GR >= 3) {
        GRL = 1;
        while (GRL * 2 < GR) GRL *= 2;
    }
    out.q_gr_lo = GRL;
    out.q_staged = staged;
    out.q_tile_rows = R;
    out.q_gr = GR;
    out.q_gs = 0;
    out.q_smem = 0;
    if (staged) {
        std::vector<int> off;
        int stage_in = 0;
        for (int c : used) {
            off.push_back(stage_in);
            stage_in += ((R * compact_bytes(cols[c].precision) + 16 + 15) / 16) * 16;
        }
        const int off_gid = stage_in;
        stage_in += R * 4 + 16;
        const int off_acc = 2 * stage_in;
        const int budget = 48 * 1024 - off_acc - 64;
        int GS = std::min(4096, budget / (W * 4 + 4));
        if (GS < GR) GS = GR;
        const int off_cnt = off_acc + ((GS * W * 4 + 15) / 16) * 16;
        const int off_bar = off_cnt + ((GS * 4 + 15) / 16) * 16;
        const int smem = off_bar + 16;
        out.q_gs = GS;
        out.q_smem = smem;
        int tile_in_bytes = R * 4;
        for (int c : used) tile_in_bytes += R * compact_bytes(cols[c].precision);
        // KEYS (register mode with key columns): a row's key is matched
        // against the present keys held in registers (the inverse half of the
        // key table), so no table lookup happens per row; rows matching none
        // are counted and flagged as a domain error at the end
        src << "template <int MODE, int KEYS, int GRV>\nUP_DI void up_query_tile_body(const UpQArgs& a, u8* sm) {\n";
        src << "    constexpr int R = " << R << ";\n    constexpr int W = " << W << ";\n";
        src << "    constexpr int GR = GRV;  // register groups of this kernel\n";
        // the full register kernel leaves the group counts of the smaller one to it
        src << "    constexpr int GR_BELOW = GRV == " << std::max(GR, 1) << " ? " << GRL << " : 0;\n";
        src << "    u64* bar = (u64*)(sm + " << off_bar << ");\n";
        src << "    u32* sacc = (u32*)(sm + " << off_acc << ");\n";
        src << "    u32* scnt = (u32*)(sm + " << off_cnt << ");\n";
        // the launch picks the mode by group count; with the count on the
        // device every mode is launched and all but one return here
        src << "    const int ng = q_groups(a);\n";
        src << "    if (ng < 0) { if (threadIdx.x == 0 && blockIdx.x == 0 && a.err) atomicOr(a.err, ERR_DOMAIN); return; }\n";
        src << "    if (MODE == 0 ? (ng > GR || ng <= GR_BELOW) : MODE == 1 ? ((" << GR << " > 0 && ng <= " << GR
            << ") || ng > " << GS << ") : ng <= " << GS << ") return;\n";
        src << "    const int nsm = MODE == 0 ? (ng < GR ? ng : GR) : (MODE == 1 ? ng : 0);\n";
        src << "    for (int i = threadIdx.x; i < nsm * W; i += blockDim.x) sacc[i] = 0u;\n";
        src << "    for (int i = threadIdx.x; i < nsm; i += blockDim.x) scnt[i] = 0u;\n";
        // register accumulators: the full width when it is at most 4 limbs, else a
        // 128-bit fast accumulator for values that fit 64 bits (the others go
        // straight to the shared-memory accumulators)
        auto ra_limbs = [&](int i) { return acc_limbs[i] <= 4 ? acc_limbs[i] : 4; };
        for (int i = 0; i < NR; i++)
            src << "    u32 ra" << i << "[MODE == 0 ? GR : 1][" << ra_limbs(i) << "];\n";
        src << "    u32 rc[MODE == 0 ? GR : 1];\n";
        src << "#pragma unroll\n    for (int j = 0; j < (MODE == 0 ? GR : 1); j++) {\n        rc[j] = 0u;\n";
        for (int i = 0; i < NR; i++)
            src << "#pragma unroll\n        for (int l = 0; l < " << ra_limbs(i) << "; l++) ra" << i << "[j][l] = 0u;\n";
        src << "    }\n";
        src << "    u32 kj[KEYS ? GR : 1];\n    u32 nrow = 0u;\n";
        src << "#pragma unroll\n    for (int j = 0; j < (KEYS ? GR : 1); j++)\n";
        src << "        kj[j] = (KEYS && j < nsm) ? (u32)__ldg(a.key_table + 65536 + j) : 0xffffffffu;\n";
        src << "    const i64 ntiles = (a.rows + R - 1) / R;\n";
        src << "    const i64 nfull = a.vec_ok ? a.rows / R : 0;  // tiles moved by bulk copies\n";
        src << "    u32 err = 0u;\n";
        src << "    if (threadIdx.x == 0) { mbar_init(&bar[0], 1); mbar_init(&bar[1], 1); mbar_init_fence(); }\n";
        src << "    __syncthreads();\n";
        src << "    auto issue = [&](i64 tt, int st) {\n";
        src << "        mbar_expect_tx(&bar[st], " << tile_in_bytes - R * 4
            << "u + (a.key_mode == 0 ? " << R * 4 << "u : a.key_mode == 1 ? " << R << "u : " << 2 * R << "u));\n";
        for (size_t i = 0; i < used.size(); i++) {
            int c = used[i];
            int B = compact_bytes(cols[c].precision);
            src << "        bulk_load(sm + st * " << stage_in << " + " << off[i] << ", a.col[" << c
                << "].data + tt * (i64)(R * " << B << "), " << R * B << "u, &bar[st]);\n";
        }
        src << "        if (a.key_mode == 0) bulk_load(sm + st * " << stage_in << " + " << off_gid
            << ", (const u8*)(a.gid + tt * (i64)R), " << R * 4 << "u, &bar[st]);\n";
        src << "        else if (a.key_mode == 3) bulk_load(sm + st * " << stage_in << " + " << off_gid
            << ", a.key0 + tt * (i64)" << 2 * R << ", " << 2 * R << "u, &bar[st]);\n";
        src << "        else {\n            bulk_load(sm + st * " << stage_in << " + " << off_gid << ", a.key0 + tt * (i64)R, "
            << R << "u, &bar[st]);\n";
        src << "            if (a.key_mode == 2) bulk_load(sm + st * " << stage_in << " + " << off_gid + R
            << ", a.key1 + tt * (i64)R, " << R << "u, &bar[st]);\n        }\n";
        src << "    };\n";
        src << "    if (threadIdx.x == 0 && (i64)blockIdx.x < nfull) issue(blockIdx.x, 0);\n";
        src << "    int k = 0;\n";
        src << "    bool timed_out = false;\n    int to_st = 0;\n    u32 to_par = 0u;\n";
        src << "    for (i64 t = blockIdx.x; t < ntiles; t += gridDim.x, k++) {\n";
        src << "        const int st = k & 1;\n";
        src << "        const i64 row0 = t * (i64)R;\n";
        src << "        const int nr = (a.rows - row0) < R ? (int)(a.rows - row0) : R;\n";
        src << "        const bool bulk = t < nfull;\n";
        src << "        const i64 tn = t + gridDim.x;\n";
        src << "        if (threadIdx.x == 0 && tn < nfull) issue(tn, st ^ 1);\n";
        src << "        u8* in = sm + st * " << stage_in << ";\n";
        src << "        if (bulk) {\n";
        src << "            if (!mbar_wait(&bar[st], (u32)((k >> 1) & 1))) { timed_out = true; to_st = st; to_par = (u32)((k >> 1) & 1); }\n";
        src << "        } else {\n";
        for (size_t i = 0; i < used.size(); i++) {
            int c = used[i];
            int B = compact_bytes(cols[c].precision);
            src << "            tile_copy_in(in + " << off[i] << ", a.col[" << c << "].data + row0 * " << B << ", nr * "
                << B << ", a.vec_ok != 0);\n";
        }
        src << "            if (a.key_mode == 0) tile_copy_in(in + " << off_gid
            << ", (const u8*)(a.gid + row0), nr * 4, a.vec_ok != 0);\n";
        src << "            else if (a.key_mode == 3) tile_copy_in(in + " << off_gid
            << ", a.key0 + row0 * 2, nr * 2, a.vec_ok != 0);\n";
        src << "            else {\n                tile_copy_in(in + " << off_gid << ", a.key0 + row0, nr, a.vec_ok != 0);\n";
        src << "                if (a.key_mode == 2) tile_copy_in(in + " << off_gid + R
            << ", a.key1 + row0, nr, a.vec_ok != 0);\n            }\n";
        src << "            __syncthreads();\n";
        src << "        }\n";
        src << "        if (__syncthreads_or(timed_out)) break;\n";
        src << "        const u8* tg = in + " << off_gid << ";\n";
        src << "        for (int r = threadIdx.x; r < nr; r += blockDim.x) {\n";
        src << "            const u32 key = KEYS ? q_tile_key(a, tg, r, R) : 0u;\n";
        src << "            const int g = KEYS ? 0 : q_tile_group(a, tg, r, R);\n";
        src << "            if (!KEYS && (unsigned)g >= (unsigned)ng) { err |= ERR_DOMAIN; continue; }\n";
        src << "            if (KEYS) nrow++;\n";
        src << decl_t("            ");
        if (NR > 0) {
            src << "            err |= up_qvals(";
            for (size_t i = 0; i < used.size(); i++)
                src << "in + " << off[i] << " + r * " << compact_bytes(cols[used[i]].precision) << ", ";
            src << "true" << targs() << ");\n";
        }
        src << "            if constexpr (MODE == 0) {\n";
        for (int i = 0; i < NR; i++)
            if (acc_limbs[i] > 4) {
                src << "                const bool f" << i << " = fits_twos64(qv" << i << ");\n";
                src << "                if (!f" << i << ") {  // rare: wider than 64 bits\n";
                src << "                    const int gw = KEYS ? __ldg(a.key_table + key) : g;\n";
                src << "                    if ((unsigned)gw < (unsigned)q_nsm(a, MODE, GR)) atomic_add_twos(sacc + gw * W + "
                    << acc_off[i]
                    << ", qv" << i << ");\n                }\n";
            }
        src << "#pragma unroll\n                for (int j = 0; j < GR; j++)\n";
        src << "                    if (KEYS ? key == kj[j] : g == j) {\n                        rc[j]++;\n";
        for (int i = 0; i < NR; i++) {
            if (acc_limbs[i] > 4)
                src << "                        if (f" << i << ") add_twos64(ra" << i << "[j], qv" << i << ");\n";
            else
                src << "                        add_twos(ra" << i << "[j], qv" << i << ");\n";
        }
        src << "                    }\n";
        src << "            } else if constexpr (MODE == 1) {\n";
        src << "                atomicAdd(scnt + g, 1u);\n";
        for (int i = 0; i < NR; i++)
            src << "                atomic_add_twos(sacc + g * W + " << acc_off[i] << ", qv" << i << ");\n";
        src << "            } else {\n";
        src << "                atomicAdd(a.cnt + g, 1ull);\n";
        for (int i = 0; i < NR; i++)
            src << "                atomic_add_twos(a.acc + (i64)g * W + " << acc_off[i] << ", qv" << i << ");\n";
        src << "            }\n";
        src << "        }\n";
        src << "        __syncthreads();\n";
        src << "    }\n";
        src << "    if (threadIdx.x == 0 && timed_out) {\n";
        src << "        err |= ERR_TIMEOUT;\n";
        src << "        mbar_wait(&bar[to_st], to_par);  // bounded: let copies in flight land before exit\n";
        src << "    }\n";
        src << "    if constexpr (MODE == 0 && KEYS) {\n        u32 matched = 0u;\n";
        src << "#pragma unroll\n        for (int j = 0; j < GR; j++) matched += rc[j];\n";
        src << "        if (matched != nrow) err |= ERR_DOMAIN;  // a key outside the table\n    }\n";
        src << "    if constexpr (MODE == 0) {\n";
        src << "#pragma unroll\n        for (int j = 0; j < GR; j++)\n";
        src << "            if (rc[j] != 0u) {\n";
        src << "                atomicAdd(scnt + j, rc[j]);\n";
        for (int i = 0; i < NR; i++) {
            if (acc_limbs[i] > 4) {
                src << "                {\n                    u32 wide[" << acc_limbs[i] << "];  // sign-extended 128-bit sum\n";
                src << "#pragma unroll\n                    for (int l = 0; l < " << acc_limbs[i] << "; l++) wide[l] = l < 4 ? ra"
                    << i << "[j][l < 4 ? l : 0] : ((ra" << i << "[j][3] >> 31) ? 0xffffffffu : 0u);\n";
                src << "                    atomic_add_twos(sacc + j * W + " << acc_off[i] << ", wide);\n                }\n";
            } else {
                src << "                atomic_add_twos(sacc + j * W + " << acc_off[i] << ", ra" << i << "[j]);\n";
            }
        }
        src << "            }\n";
        src << "    }\n";
        src << "    if constexpr (MODE != 2) {\n";
        src << "        __syncthreads();\n";
        src << "        const int nsm_end = q_nsm(a, MODE, GR);\n";
        src << "        for (int gg = threadIdx.x; gg < nsm_end; gg += blockDim.x) {\n";
        src << "            const u32 c = scnt[gg];\n";
        src << "            if (c == 0u) continue;\n";
        src << "            atomicAdd(a.cnt + gg, (u64)c);\n";
        for (int i = 0; i < NR; i++) {
            src << "            {\n                u32 m[" << acc_limbs[i] << "];\n";
            src << "#pragma unroll\n                for (int l = 0; l < " << acc_limbs[i] << "; l++) m[l] = sacc[gg * W + "
                << acc_off[i] << " + l];\n";
            src << "                atomic_add_twos(a.acc + (i64)gg * W + " << acc_off[i] << ", m);\n            }\n";
        }
        src << "        }\n";
        src << "    }\n";
        src << "    err = __reduce_or_sync(0xffffffffu, err);\n";
        src << "    if ((threadIdx.x & 31) == 0 && err != 0u && a.err) atomicOr(a.err, err);\n";
        src << "}\n\n";
        const char* names[6] = {"up_query_tile_r",  "up_query_tile_s",    "up_query_tile_g",
                                "up_query_tile_rk", "up_query_tile_r_lo", "up_query_tile_rk_lo"};
        for (int kn = 0; kn < 6; kn++) {
            const int mde = kn == 1 ? 1 : (kn == 2 ? 2 : 0);
            const int keys = (kn == 3 || kn == 5) ? 1 : 0;
            const int grv = kn >= 4 ? GRL : std::max(GR, 1);
            if (mde == 0 && GR == 0) continue;
            if (kn >= 4 && GRL == 0) continue;
            // two CTAs per SM for the register modes (the key-matching one
            // would otherwise take a few registers too many for that)
            src << "extern \"C\" __global__ void __launch_bounds__(" << T << (mde == 0 && T == 256 ? ", 2" : "") << ") "
                << names[kn] << "(const UpQArgs a) {\n    extern __shared__ __align__(128) u8 sm[];\n"
                << "    up_query_tile_body<" << mde << ", " << keys << ", " << grv << ">(a, sm);\n}\n\n";
        }
    }

    src << "extern \"C\" __global__ void __launch_bounds__(256) up_query_fin(const UpQArgs a) {\n";
    src << "    const int g = blockIdx.x * blockDim.x + threadIdx.x;\n";
    src << "    if (g >= q_groups(a)) return;\n";
    src << "    const u64 cnt = a.cnt[g];\n";
    src << "    const u32* acc = a.acc + (i64)g * " << std::max(accw, 1) << ";\n";
    src << "    const u32 P10_4[1] = {10000u};\n";
    for (int a = 0; a < n_aggs; a++) {
        int k = aggs[a].kind;
        src << "    {\n";
        if (k == UP_AGG_COUNT) {
            src << "        ((i64*)a.out[" << a << "])[g] = (i64)cnt;\n";
        } else {
            int n = out.agg_acc_limbs[a];
            if (any_nullable)  // the accumulator's own count of non-NULL rows
                src << "        const u64 cnt = (u64)acc[" << cnt_off[agg_slot[a]] << "] | ((u64)acc["
                    << cnt_off[agg_slot[a]] + 1 << "] << 32);\n";
            src << "        u32 m[" << n << "];\n";
            src << "        for (int i = 0; i < " << n << "; i++) m[i] = acc[" << out.agg_acc_offset[a] << " + i];\n";
            src << "        const u32 neg = m[" << n - 1 << "] >> 31;\n";
            src << "        if (neg) negate(m);\n";
            src << "        u8* img = a.out[" << a << "] + (i64)g * 133;\n";
            if (k == UP_AGG_SUM) {
                src << "        agg_image(img, cnt > 0 ? 1u : 0u, neg, " << out.agg_scale[a] << "u, m);\n";
            } else {
                int nq = n + 1;
                // a group without rows has a zero sum: the divide rule's zero-dividend case
                src << "        {\n";
                src << "            const u32 c2[2] = {(u32)cnt, (u32)(cnt >> 32)};\n";
                src << "            u32 q[" << nq << "]; u32 sq;\n";
                src << "            const u32 e = div_round<" << nq << ", " << n << ", 2, 1, 4u, 10000ull>(q, sq, m, neg, c2, 0u, P10_4);\n";
                src << "            avg_image(img, cnt > 0 ? 1u : 0u, cnt, is_zero(m), sq, " << out.agg_scale[a] + 4 << "u, q, e);\n";
                src << "        }\n";
            }
        }
        src << "    }\n";
    }
    src << "}\n";

    out.source = src.str();
    out.work_per_row = em.work + row_bytes;
    out.kernels = {"up_query_acc", "up_query_fin"};
    if (out.q_staged) {
        if (out.q_gr > 0) {
            out.kernels.push_back("up_query_tile_r");
            out.kernels.push_back("up_query_tile_rk");
        }
        if (out.q_gr_lo > 0) {
            out.kernels.push_back("up_query_tile_r_lo");
            out.kernels.push_back("up_query_tile_rk_lo");
        }
        out.kernels.push_back("up_query_tile_s");
        out.kernels.push_back("up_query_tile_g");
    }
    out.block_threads = T;
    out.in_bytes.assign(n_cols, 0);
    for (int c = 0; c < n_cols; c++) out.in_bytes[c] = compact_bytes(cols[c].precision) + (cols[c].nullable ? 1 : 0);
    return UP_OK;
}

}  // namespace upi

namespace upi {

// ----------------------------------------------------- batch modules
// Each distinct task becomes one relocatable unit whose functions are named
// by a hash of their body (so a unit compiled once is reused by every batch
// that contains the same task); a dispatcher unit holds, per precision band,
// a persistent kernel (in three block sizes) that pulls (task, tile) work
// items and calls the task's tile function, plus the finalisation kernel.
namespace {
const char* kBatchPrelude =
    "#define UP_MUL_UNROLL_PAIRS 1024\n"
    "#include \"up_dev.cuh\"\nusing namespace up;\n";  // BTask, BArgs: up_kargs.h

uint64_t text_hash(const std::string& s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

std::string replace_all(std::string s, const std::string& from, const std::string& to) {
    size_t p = 0;
    while ((p = s.find(from, p)) != std::string::npos) {
        s.replace(p, from.size(), to);
        p += to.size();
    }
    return s;
}
}  // namespace

up_status generate_batch_module(const BatchTaskDesc* tasks, int n_tasks, GeneratedBatch& out) {
    if (n_tasks <= 0 || n_tasks > 1024) return fail(UP_ERR_INVALID_ARG, "1..1024 tasks");
    out.tasks.assign(n_tasks, GeneratedBatch::Task());
    out.units.clear();
    std::vector<std::string> fname(n_tasks);
    std::map<std::string, int> unit_of;
    for (int k = 0; k < n_tasks; k++) {
        const BatchTaskDesc& t = tasks[k];
        if (t.n_cols < 1 || t.n_cols > 8) return fail(UP_ERR_INVALID_ARG, "tasks take 1..8 columns");
        std::vector<NodeFacts> f;
        std::vector<int> topo;
        up_status st = analyze_nodes(t.nodes, t.n_nodes, t.cols, t.n_cols, f, topo, {t.root});
        if (st != UP_OK) return st;
        GeneratedBatch::Task& gt = out.tasks[k];
        int max_limbs = 1;
        for (int n : topo) max_limbs = std::max(max_limbs, f[n].limbs);
        if (max_limbs > 128) return fail(UP_ERR_UNSUPPORTED, "task " + std::to_string(k) + " wider than 4096 bits");
        gt.band = max_limbs <= 4 ? 0 : (max_limbs <= 24 ? 1 : 2);
        gt.agg = t.agg_kind;
        const up_expr_node& rn = t.nodes[t.root];
        const bool cmp_root = is_compare_kind(rn.kind);
        std::vector<int> used;
        for (int n : topo)
            if (t.nodes[n].kind == UP_NODE_COLUMN &&
                std::find(used.begin(), used.end(), t.nodes[n].column) == used.end())
                used.push_back(t.nodes[n].column);
        std::sort(used.begin(), used.end());
        gt.in_bytes.assign(t.n_cols, 0);
        for (int c = 0; c < t.n_cols; c++) gt.in_bytes[c] = compact_bytes(t.cols[c].precision);
        Emitter em(t.nodes, t.cols, f);
        em.plan(topo);
        for (int n : topo) em.node(n);
        std::ostringstream src;
        src << kBatchPrelude;
        const int wco = cooperative_width(t.nodes, f, topo);
        gt.tpv = (t.agg_kind < 0 && t.tpv > 1 && wco > 0) ? t.tpv : 1;
        if (gt.tpv > 1) {
            // Cooperative projection: groups of T threads per row, K limbs
            // each; every group of the CTA runs the same number of slots, so
            // warps stay converged around the shuffles (a group past the last
            // row works on row r0 and stores nothing).
            const int TT = gt.tpv, KK = (wco + TT - 1) / TT;
            if (cmp_root) {
                gt.out_p = 1;
                gt.out_s = 0;
                gt.out_bytes = 1;
            } else {
                if (rn.precision < 1) return fail(UP_ERR_INVALID_ARG, "task root precision not set");
                gt.out_p = rn.precision;
                gt.out_s = f[t.root].scale;
                gt.out_bytes = compact_bytes(rn.precision);
            }
            const int BO = gt.out_bytes;
            TEmitter te(t.nodes, t.cols, f, TT, KK);
            te.plan(topo);
            for (int n : topo) te.node(n);
            src << "namespace {\n" << te.globals.str() << "}  // namespace\n";
            src << "UP_DI u32 trow(" << params_decl(used) << "u8* __restrict__ out, const bool store) {\n";
            src << "    u32 err = 0u;\n" << te.constants() << te.body.str();
            if (cmp_root)
                src << "    if (store && tpi_rank<" << TT << ">() == 0) out[0] = (u8)c" << t.root << ";\n";
            else
                src << "    err |= tpi_st<" << TT << ", " << KK << ", " << BO << ">(out, v" << t.root << ", s" << t.root
                    << ", store);\n";
            src << "    return err;\n}\n";
            src << "extern \"C\" __device__ __noinline__ u32 @@tile(const BTask& t, i64 tile, int tr) {\n";
            src << "    u32 err = 0u;\n    const i64 r0 = tile * tr;\n";
            src << "    const i64 r1 = (r0 + tr) < t.rows ? (r0 + tr) : t.rows;\n";
            src << "    const int grp = (int)threadIdx.x / " << TT << ";\n";
            src << "    const int G = (int)blockDim.x / " << TT << ";\n";
            src << "    for (i64 base = r0; base < r1; base += G) {\n";
            src << "        const i64 r = base + grp;\n        const bool valid = r < r1;\n";
            src << "        const i64 rr = valid ? r : r0;\n";
            src << "        const u32 e = trow(";
            for (int c : used) src << "t.col[" << c << "].data + rr * " << gt.in_bytes[c] << ", ";
            src << "t.out + rr * " << BO << ", valid);\n";
            src << "        if (valid) err |= e;\n    }\n    return err;\n}\n";
        } else if (t.agg_kind < 0) {
            if (cmp_root) {
                gt.out_p = 1;
                gt.out_s = 0;
                gt.out_bytes = 1;
            } else {
                if (rn.precision < 1) return fail(UP_ERR_INVALID_ARG, "task root precision not set");
                gt.out_p = rn.precision;
                gt.out_s = f[t.root].scale;
                gt.out_bytes = compact_bytes(rn.precision);
            }
            const int BO = gt.out_bytes;
            src << "UP_DI u32 row(" << params_decl(used) << "u8* __restrict__ out, const bool words) {\n";
            src << "    u32 err = 0u;\n" << em.constants() << em.body.str();
            if (cmp_root) src << "    out[0] = (u8)c" << t.root << ";\n";
            else src << "    err |= st_compact_bytes<" << BO << ">(out, v" << t.root << ", s" << t.root << ");\n";
            src << "    return err;\n}\n";
            src << "extern \"C\" __device__ __noinline__ u32 @@tile(const BTask& t, i64 tile, int tr) {\n";
            src << "    u32 err = 0u;\n    const i64 r0 = tile * tr;\n";
            src << "    const i64 r1 = (r0 + tr) < t.rows ? (r0 + tr) : t.rows;\n";
            src << "    for (i64 r = r0 + threadIdx.x; r < r1; r += blockDim.x) {\n";
            src << "        const bool words = t.words != 0 && r + 1 < t.rows;  // word reads stay inside the column\n";
            src << "        err |= row(";
            for (int c : used) src << "t.col[" << c << "].data + r * " << gt.in_bytes[c] << ", ";
            src << "t.out + r * " << BO << ", words);\n    }\n    return err;\n}\n";
        } else {
            if (cmp_root) return fail(UP_ERR_INVALID_ARG, "cannot aggregate a comparison");
            const NodeFacts& fr = f[t.root];
            gt.nacc = limbs_for_bits(fr.bits + 1 + 40);
            gt.agg_scale = fr.scale;
            src << "UP_DI u32 qrow(" << params_decl(used) << "u32* __restrict__ acc, const bool words) {\n";
            src << "    u32 err = 0u;\n" << em.constants() << em.body.str();
            if (t.agg_kind != UP_AGG_COUNT)
                src << "    atomic_acc_add<" << gt.nacc << ">(acc, v" << t.root << ", s" << t.root << ");\n";
            src << "    return err;\n}\n";
            src << "extern \"C\" __device__ __noinline__ u32 @@tile(const BTask& t, i64 tile, int tr) {\n";
            src << "    u32 err = 0u;\n    const i64 r0 = tile * tr;\n";
            src << "    const i64 r1 = (r0 + tr) < t.rows ? (r0 + tr) : t.rows;\n";
            src << "    for (i64 r = r0 + threadIdx.x; r < r1; r += blockDim.x) {\n";
            src << "        const int g = t.gid[r];\n";
            src << "        if ((unsigned)g >= (unsigned)t.n_groups) { err |= ERR_DOMAIN; continue; }\n";
            src << "        atomicAdd(t.cnt + g, 1ull);\n";
            if (t.agg_kind != UP_AGG_COUNT) {
                src << "        const bool words = t.words != 0 && r + 1 < t.rows;\n";
                src << "        err |= qrow(";
                for (int c : used) src << "t.col[" << c << "].data + r * " << gt.in_bytes[c] << ", ";
                src << "t.acc + (i64)g * " << gt.nacc << ", words);\n";
            }
            src << "    }\n    return err;\n}\n";
            src << "extern \"C\" __device__ __noinline__ void @@fin(const BTask& t, int g) {\n";
            src << "    const u64 cnt = t.cnt[g];\n";
            if (t.agg_kind == UP_AGG_COUNT) {
                src << "    ((i64*)t.out)[g] = (i64)cnt;\n";
            } else {
                const int n = gt.nacc;
                src << "    u32 m[" << n << "];\n";
                src << "    for (int i = 0; i < " << n << "; i++) m[i] = t.acc[(i64)g * " << n << " + i];\n";
                src << "    const u32 neg = m[" << n - 1 << "] >> 31;\n    if (neg) negate(m);\n";
                src << "    u8* img = t.out + (i64)g * 133;\n";
                if (t.agg_kind == UP_AGG_SUM) {
                    src << "    agg_image(img, cnt > 0 ? 1u : 0u, neg, " << gt.agg_scale << "u, m);\n";
                } else {
                    src << "    const u32 P10_4[1] = {10000u};\n";
                    src << "    const u32 c2[2] = {(u32)cnt, (u32)(cnt >> 32)};\n";
                    src << "    u32 q[" << n + 1 << "]; u32 sq;\n";
                    src << "    const u32 e = div_round<" << n + 1 << ", " << n << ", 2, 1, 4u, 10000ull>(q, sq, m, neg, c2, 0u, P10_4);\n";
                    src << "    avg_image(img, cnt > 0 ? 1u : 0u, cnt, is_zero(m), sq, " << gt.agg_scale + 4 << "u, q, e);\n";
                }
            }
            src << "}\n";
        }
        const std::string body = src.str();
        char hname[40];
        snprintf(hname, sizeof hname, "ut%016llx_", (unsigned long long)text_hash(body));
        fname[k] = hname;
        if (!unit_of.count(hname)) {
            unit_of[hname] = (int)out.units.size();
            out.units.push_back(replace_all(body, "@@", hname));
        }
    }
    // dispatcher unit
    std::ostringstream d;
    d << kBatchPrelude;
    std::set<std::string> declared;
    std::vector<int> aggs;
    for (int k = 0; k < n_tasks; k++) {
        if (out.tasks[k].agg >= 0) aggs.push_back(k);
        if (declared.insert(fname[k]).second) {
            d << "extern \"C\" __device__ u32 " << fname[k] << "tile(const BTask& t, i64 tile, int tr);\n";
            if (out.tasks[k].agg >= 0) d << "extern \"C\" __device__ void " << fname[k] << "fin(const BTask& t, int g);\n";
        }
    }
    static const int kThreads[3] = {64, 128, 256};
    out.kernels.clear();
    for (int b = 0; b < 3; b++) {
        std::ostringstream body;
        body << "    __shared__ i64 s_item;\n    u32 err = 0u;\n";
        body << "    for (;;) {\n";
        body << "        if (threadIdx.x == 0) s_item = (i64)atomicAdd(a.head, 1ull);\n";
        body << "        __syncthreads();\n        const i64 it = s_item;\n        __syncthreads();\n";
        body << "        if (it >= a.n_items) break;\n";
        body << "        const int task = a.item_task[it];\n        const i64 tile = a.item_tile[it];\n";
        body << "        switch (task) {\n";
        for (int k = 0; k < n_tasks; k++)
            if (out.tasks[k].band == b)
                body << "            case " << k << ": err |= " << fname[k] << "tile(a.tasks[" << k
                     << "], tile, a.tile_rows); break;\n";
        body << "            default: break;\n        }\n    }\n";
        body << "    err = __reduce_or_sync(0xffffffffu, err);\n";
        body << "    if ((threadIdx.x & 31) == 0 && err != 0u && a.err) atomicOr(a.err, err);\n";
        for (int ti = 0; ti < 3; ti++) {
            std::string name = "up_batch_b" + std::to_string(b) + "_t" + std::to_string(kThreads[ti]);
            d << "extern \"C\" __global__ void __launch_bounds__(" << kThreads[ti] << ") " << name
              << "(const BArgs a) {\n" << body.str() << "}\n";
            out.kernels.push_back(name);
        }
    }
    d << "extern \"C\" __global__ void __launch_bounds__(256) up_batch_fin(const BArgs a) {\n";
    d << "    const int g = blockIdx.x * blockDim.x + threadIdx.x;\n    switch (blockIdx.y) {\n";
    for (size_t i = 0; i < aggs.size(); i++)
        d << "        case " << i << ": if (g < a.tasks[" << aggs[i] << "].n_groups) " << fname[aggs[i]] << "fin(a.tasks["
          << aggs[i] << "], g); break;\n";
    d << "        default: break;\n    }\n}\n";
    out.kernels.push_back("up_batch_fin");
    out.units.push_back(d.str());
    out.agg_tasks = aggs;
    out.source.clear();
    for (const auto& u : out.units) out.source += u;
    return UP_OK;
}

}  // namespace upi
