// up_align.cpp — the reference's AlignOptimize expression rewrite
// (src/AriesEngineWrapper/AriesEngineShell.cpp:90-685), restated on
// up_expr_node trees.
//
// Steps, each following the reference function named:
//   ModifySubOperation (:244-281)  a-b -> a+(-b); reversal pushed to children
//   BinToMultiTree/getChild (:283-342)  flatten chains of the same operator
//   AlignOptMultiTree (:360-612)   ADD: addends sorted integers, decimal
//       constants (by scale), then columns/subtrees by scale; constants folded
//       (host Decimal arithmetic, 1024-bit); MUL: constants folded; DIV/MOD:
//       integer operands become decimal constants, a zero dividend folds to 0
//   RemoveZeroNode (:192-229)      zero subtrees removed (under MUL: all zero)
//   MultiToBinTree/ListToBinTree (:90-190)  left-deep rebuild, re-typed
//   AlignOptimizeNode (:615-644)   root precision capped at 288
// Typing and ordering follow the reference exactly (addends with equal sort
// keys keep their order, as libstdc++'s std::sort, an insertion sort below 17
// elements, leaves them; chains of MOD are flattened like the reference
// does).  Three value-changing defects of the reference are not reproduced:
// MUL folding ignores a constant's reversal flag (so a-2*b became a+2*b),
// DIV/MOD drop the reversal of an integer operand they convert, and
// RemoveZeroNode treats every INTEGER under MUL as zero (so x*1 became 0).
// A root that folds to a constant-only or zero tree, which the reference
// leaves malformed, becomes INT 0 here.
#include <algorithm>
#include <cstring>
#include <deque>
#include <functional>
#include <queue>
#include <vector>

#include "up_internal.h"

namespace upi {

up_status derive_types_impl(up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols, int n_cols);

namespace {

enum BKind { K_COL, K_INT, K_DEC, K_CALC };

// host Decimal value: sign, frac, magnitude (kept below 2^1024 like the
// reference's 32-limb Decimal), prec
struct HDec {
    uint32_t sign = 0;
    int frac = 0;
    int prec = 10;
    Big mag;
    bool is_zero() const { return mag.is_zero(); }
};

void trunc1024(Big& b) {
    if (b.m.size() > 32) b.m.resize(32);
    big_trim(b);
}

// Decimal(int32_t), decimal.cu:291-298 / Decimal(int64_t) :301-309
HDec dec_from_int(int64_t t) {
    HDec d;
    d.prec = (t >= -2147483648LL && t <= 2147483647LL) ? 10 : 19;
    d.sign = t < 0;
    uint64_t mag = t < 0 ? (uint64_t)(-(t + 1)) + 1u : (uint64_t)t;
    d.mag = big_from_u64(mag);
    return d;
}

// Decimal(int32_t t, int32_t scale, ...), decimal.cu:230-260: t * 10^scale
HDec dec_from_int_scaled(int64_t t, int scale) {
    HDec d = dec_from_int(t);
    d.prec = 10 + (scale > 10 ? scale : 0);
    d.frac = scale;
    d.mag = big_mul(d.mag, big_pow10(scale));
    trunc1024(d.mag);
    return d;
}

// AlignAddSubData (decimal.cu:2905-2919) on copies
void align(HDec& a, HDec& b) {
    if (a.frac < b.frac) {
        a.mag = big_mul(a.mag, big_pow10(b.frac - a.frac));
        trunc1024(a.mag);
        a.frac = b.frac;
    } else if (b.frac < a.frac) {
        b.mag = big_mul(b.mag, big_pow10(a.frac - b.frac));
        trunc1024(b.mag);
        b.frac = a.frac;
    }
}

// AddDecimalOnCpu, decimal.cu:1284-1321
void add_on_cpu(HDec& self, const HDec& d) {
    HDec added = d;
    align(added, self);
    if (self.sign == added.sign) {
        self.mag = big_add(self.mag, added.mag);
        trunc1024(self.mag);
    } else {
        int c = big_cmp(self.mag, added.mag);
        if (c >= 0) self.mag = big_sub(self.mag, added.mag);
        else self.mag = big_sub(added.mag, self.mag);
        self.sign = (c > 0 && !d.sign) || (c < 0 && d.sign);
    }
}

// MulDecimalOnCpu, decimal.cu:1323-1350
void mul_on_cpu(HDec& self, const HDec& d) {
    self.sign ^= d.sign;
    self.frac += d.frac;
    self.mag = big_mul(self.mag, d.mag);
    trunc1024(self.mag);
}

// Decimal == Decimal (decimal.cu:724-740): signs equal and aligned magnitudes equal
bool dec_eq(const HDec& a, const HDec& b) {
    if (a.sign != b.sign) return false;
    HDec x = a, y = b;
    align(x, y);
    return big_cmp(x.mag, y.mag) == 0;
}

// Decimal(Decimal t, int32_t scale, ...), decimal.cu:263-268
HDec dec_rescaled(const HDec& t, int scale) {
    HDec d = t;
    int gap = scale - t.frac;
    if (gap > 0) {
        d.mag = big_mul(d.mag, big_pow10(gap));
        trunc1024(d.mag);
    }
    d.frac = scale;
    d.prec = t.prec + gap;
    return d;
}

struct BNode {
    int kind = K_COL;
    int op = 0;  // UP_NODE_ADD .. UP_NODE_MOD for K_CALC
    bool reverse = false;
    int prec = 0, scale = 0;
    int column = 0;
    int64_t ival = 0;
    HDec dec;
    std::vector<BNode*> children;
};

struct MNode {
    int kind = K_COL;
    int op = 0;
    bool reverse = false;
    int prec = 0, scale = 0;
    int column = 0;
    int64_t ival = 0;
    HDec dec;
    std::vector<MNode*> childList;
    BNode* rootObj = nullptr;
    void copy_info(const MNode& o) {  // CopyNodeInfo, :74-82
        kind = o.kind;
        op = o.op;
        reverse = o.reverse;
        prec = o.prec;
        scale = o.scale;
        column = o.column;
        ival = o.ival;
        dec = o.dec;
        childList = o.childList;
    }
};

struct Arena {
    std::deque<BNode> b;
    std::deque<MNode> m;
    BNode* nb() {
        b.emplace_back();
        return &b.back();
    }
    MNode* nm() {
        m.emplace_back();
        return &m.back();
    }
    MNode* from(BNode* o) {  // MultipleTree(BinaryTree*), :63-70
        MNode* x = nm();
        x->rootObj = o;
        x->kind = o->kind;
        x->op = o->op;
        x->reverse = o->reverse;
        x->prec = o->prec;
        x->scale = o->scale;
        x->column = o->column;
        x->ival = o->ival;
        x->dec = o->dec;
        return x;
    }
};

bool is_calc_kind(int k) { return k >= UP_NODE_ADD && k <= UP_NODE_MOD; }

// ModifySubOperation, :244-281
void modify_sub(BNode* root) {
    std::queue<BNode*> q;
    q.push(root);
    while (!q.empty()) {
        BNode* n = q.front();
        if (n->kind == K_CALC) {
            if (n->op == UP_NODE_MUL && n->reverse) {
                n->children[0]->reverse = !n->children[0]->reverse;
            } else if (n->op == UP_NODE_DIV && n->reverse) {
                n->children[0]->reverse = !n->children[0]->reverse;
            } else if (n->op == UP_NODE_ADD && n->reverse) {
                n->children[0]->reverse = !n->children[0]->reverse;
                n->children[1]->reverse = !n->children[1]->reverse;
            } else if (n->op == UP_NODE_SUB) {
                if (!n->reverse) n->children[1]->reverse = !n->children[1]->reverse;
                if (n->reverse) n->children[0]->reverse = !n->children[0]->reverse;
                n->op = UP_NODE_ADD;
            }
            if (n->children.size() == 2) {
                q.push(n->children[0]);
                q.push(n->children[1]);
            }
        }
        q.pop();
    }
}

// getChild, :285-329
std::vector<MNode*> get_child(Arena& A, BNode* b, int symbol) {
    std::vector<MNode*> out;
    if (symbol == UP_NODE_DIV) {
        out.push_back(A.from(b->children[0]));
        out.push_back(A.from(b->children[1]));
        return out;
    }
    for (int k = 0; k < 2; k++) {
        BNode* c = b->children[k];
        if (c->kind != K_CALC) {
            out.push_back(A.from(c));
        } else if (c->op == symbol) {
            auto sub = get_child(A, c, symbol);
            out.insert(out.end(), sub.begin(), sub.end());
        } else {
            out.push_back(A.from(c));
        }
    }
    return out;
}

// BinToMultiTree, :331-342
void bin_to_multi(Arena& A, BNode* b, MNode* m) {
    m->childList = get_child(A, b, m->rootObj->op);
    for (MNode* c : m->childList) {
        if (c->rootObj && c->rootObj->kind == K_CALC && c->rootObj->children.size() == 2)
            bin_to_multi(A, c->rootObj, c);
    }
}

// CmpByScale, :344-356
bool cmp_by_scale(const MNode* a, const MNode* b) {
    if (a->kind == K_INT) return true;
    if (b->kind == K_INT) return false;
    if (a->kind == K_DEC && b->kind == K_DEC) return a->scale < b->scale;
    if (a->kind == K_DEC) return true;
    if (b->kind == K_DEC) return false;
    return a->scale < b->scale;
}

// std::sort as libstdc++ performs it for short ranges (insertion sort)
void insertion_sort(std::vector<MNode*>& v) {
    for (size_t i = 1; i < v.size(); i++) {
        MNode* val = v[i];
        if (cmp_by_scale(val, v[0])) {
            for (size_t j = i; j > 0; j--) v[j] = v[j - 1];
            v[0] = val;
        } else {
            size_t j = i;
            while (cmp_by_scale(val, v[j - 1])) {
                v[j] = v[j - 1];
                j--;
            }
            v[j] = val;
        }
    }
}

void make_const(MNode* n, const HDec& d, int prec, int scale) {
    n->kind = K_DEC;
    n->dec = d;
    n->prec = prec;
    n->scale = scale;
    n->reverse = false;
    n->childList.clear();
    n->rootObj = nullptr;
}

// AlignOptMultiTree, :360-612
void align_opt(Arena& A, MNode* root) {
    std::queue<MNode*> q;
    q.push(root);
    int guard = 0;
    while (!q.empty() && guard++ < 1 << 20) {
        MNode* node = q.front();
        if (node->kind == K_CALC) {
            if (node->op == UP_NODE_ADD) {
                insertion_sort(node->childList);
                int64_t nodeInt = 0;
                HDec nodeDec = dec_from_int(0);
                size_t index = 0;
                const size_t n = node->childList.size();
                for (index = 0; index < n; index++) {
                    MNode* c = node->childList[index];
                    if (c->kind == K_INT) {
                        int64_t t = c->ival;
                        if (c->reverse) t = -t;
                        nodeInt += t;
                    } else if (c->kind == K_DEC) {
                        HDec d = c->dec;
                        if (c->reverse) d.sign = 1;
                        add_on_cpu(nodeDec, d);
                    } else {
                        break;
                    }
                }
                if (index == 0)
                    for (MNode* c : node->childList)
                        if (c->kind == K_CALC) q.push(c);
                std::vector<MNode*> nl;
                if (nodeInt == 0 && nodeDec.is_zero()) {
                    if (n > 0 && index == n - 1) {
                        node->copy_info(*node->childList[index]);
                    } else {
                        for (; index < n; index++) {
                            nl.push_back(node->childList[index]);
                            if (node->childList[index]->kind == K_CALC) q.push(node->childList[index]);
                        }
                        node->childList = nl;
                    }
                } else {
                    if (nodeDec.is_zero()) {
                        MNode* nn = A.nm();
                        const int nearScale = index < n ? node->childList[index]->scale : 0;
                        make_const(nn, dec_from_int_scaled(nodeInt, nearScale), 0, nearScale);
                        nl.push_back(nn);
                        for (; index < n; index++) {
                            nl.push_back(node->childList[index]);
                            if (node->childList[index]->kind == K_CALC) q.push(node->childList[index]);
                        }
                    } else {
                        bool opt_insert = true;
                        if (nodeInt != 0) add_on_cpu(nodeDec, dec_from_int(nodeInt));
                        for (; index < n; index++) {
                            MNode* c = node->childList[index];
                            if (c->scale > nodeDec.frac && opt_insert) {
                                opt_insert = false;
                                HDec d = dec_rescaled(nodeDec, c->scale);
                                MNode* nn = A.nm();
                                make_const(nn, d, 0, d.frac);
                                nl.push_back(nn);
                            }
                            nl.push_back(c);
                            if (c->kind == K_CALC) q.push(c);
                        }
                        if (opt_insert) {
                            MNode* nn = A.nm();
                            make_const(nn, nodeDec, nodeDec.frac, nodeDec.frac);
                            nl.push_back(nn);
                        }
                    }
                    node->childList = nl;
                }
            } else if (node->op == UP_NODE_MUL) {
                int64_t nodeInt = 1;
                HDec nodeDec = dec_from_int(1);
                std::vector<MNode*> nl;
                for (MNode* c : node->childList) {
                    // a constant's reversal flag is honoured here (the reference ignores it and
                    // so turns a-2*b into a+2*b)
                    if (c->kind == K_INT) nodeInt *= c->reverse ? -c->ival : c->ival;
                    else if (c->kind == K_DEC) {
                        HDec d = c->dec;
                        if (c->reverse) d.sign ^= 1u;
                        mul_on_cpu(nodeDec, d);
                    } else nl.push_back(c);
                }
                if (nodeInt != 1 || !dec_eq(nodeDec, dec_from_int(1))) {
                    if (nodeInt == 0 || nodeDec.is_zero()) {
                        node->kind = K_INT;
                        node->ival = 0;
                    } else {
                        mul_on_cpu(nodeDec, dec_from_int(nodeInt));
                        if (!dec_eq(nodeDec, dec_from_int(1))) {
                            MNode* nn = A.nm();
                            make_const(nn, nodeDec, 0, nodeDec.frac);
                            nl.push_back(nn);
                        }
                        node->childList = nl;
                    }
                }
                for (MNode* c : node->childList)
                    if (c->kind == K_CALC) q.push(c);
            } else if (node->op == UP_NODE_DIV || node->op == UP_NODE_MOD) {
                if (!node->childList.empty() && node->childList[0]->kind == K_INT && node->childList[0]->ival == 0) {
                    node->kind = K_INT;
                    node->ival = 0;
                } else {
                    for (size_t i = 0; i < node->childList.size(); i++) {
                        MNode* c = node->childList[i];
                        if (c->kind == K_CALC) q.push(c);
                        if (c->kind == K_INT) {
                            HDec d = dec_from_int(c->ival);
                            MNode* nn = A.nm();
                            make_const(nn, d, d.prec, d.frac);
                            nn->reverse = c->reverse;  // kept (the reference's fresh node drops it)
                            node->childList[i] = nn;
                        }
                    }
                }
            } else {
                for (MNode* c : node->childList)
                    if (c->kind == K_CALC) q.push(c);
            }
        }
        q.pop();
    }
}

// RemoveZeroNode, :192-229
MNode* remove_zero(MNode* m) {
    std::vector<MNode*> nl;
    for (size_t i = 0; i < m->childList.size(); i++) {
        MNode* c = m->childList[i];
        if (c->kind == K_INT) {
            if (c->ival != 0) {
                nl.push_back(c);  // a nonzero integer is not a zero (the reference zeroes x*1 here)
            } else if (m->op == UP_NODE_MUL) {
                m->kind = K_INT;
                m->ival = 0;
                return m;
            }
        } else if (c->kind == K_CALC) {
            m->childList[i] = remove_zero(c);
            if (m->childList[i]->kind == K_INT) {
                if (m->op == UP_NODE_MUL) {
                    m->kind = K_INT;
                    m->ival = 0;
                    return m;
                }
            } else {
                nl.push_back(m->childList[i]);
            }
        } else {
            nl.push_back(c);
        }
    }
    m->childList = nl;
    return m;
}

BNode* leaf_copy(Arena& A, const MNode* m) {
    BNode* b = A.nb();
    b->kind = m->kind;
    b->op = m->op;
    b->reverse = m->reverse;
    b->prec = m->prec;
    b->scale = m->scale;
    b->column = m->column;
    b->ival = m->ival;
    b->dec = m->dec;
    return b;
}

// ListToBinTree, :90-144: left-deep, re-typed
BNode* list_to_bin(Arena& A, std::vector<BNode*>& list, int index, int op) {
    if (index == 0) return list[0];
    BNode* l = list_to_bin(A, list, index - 1, op);
    BNode* r = list[index];
    BNode* t = A.nb();
    t->kind = K_CALC;
    const int p1 = l->prec, s1 = l->scale, p2 = r->prec, s2 = r->scale;
    if (op == UP_NODE_ADD) {
        if (r->reverse) {
            r->reverse = false;
            t->op = UP_NODE_SUB;
        } else {
            t->op = UP_NODE_ADD;
        }
        t->prec = std::max(p1 - s1, p2 - s2) + 1;
        t->scale = std::max(s1, s2);
        t->prec += t->scale;
    } else if (op == UP_NODE_MUL) {
        t->op = UP_NODE_MUL;
        t->prec = (p1 - s1) + (p2 - s2);
        t->scale = s1 + s2;
        t->prec += t->scale;
    } else if (op == UP_NODE_DIV) {
        t->op = UP_NODE_DIV;
        t->prec = p1 - p2 + s2 + 4 + 1;
        t->scale = s1 + 4;
        if (t->prec <= t->scale) t->prec = t->scale + 1;  // the reference wraps here (uint16)
    } else {
        t->op = UP_NODE_MOD;
        t->prec = p2;
        t->scale = 0;
    }
    t->children = {l, r};
    return t;
}

// MultiToBinTree, :146-190
BNode* multi_to_bin(Arena& A, MNode* m) {
    std::vector<BNode*> temp;
    for (MNode* c : m->childList) {
        if (c->kind != K_CALC) temp.push_back(leaf_copy(A, c));
        else temp.push_back(multi_to_bin(A, c));
    }
    if (m->kind != K_CALC || m->childList.empty()) return leaf_copy(A, m);
    if (m->childList.size() == 1) {
        if (m->childList[0]->kind == K_CALC) return temp[0];
        return temp[0];
    }
    return list_to_bin(A, temp, (int)temp.size() - 1, m->op);
}

BNode* clone_in(Arena& A, const up_expr_node* nodes, int idx, const up_col_type* cols) {
    const up_expr_node& nd = nodes[idx];
    BNode* b = A.nb();
    b->reverse = nd.reverse != 0;
    b->prec = nd.precision;
    b->scale = nd.scale;
    switch (nd.kind) {
        case UP_NODE_COLUMN:
            b->kind = K_COL;
            b->column = nd.column;
            b->prec = cols[nd.column].precision;
            b->scale = cols[nd.column].scale;
            break;
        case UP_NODE_INT:
            b->kind = K_INT;
            b->ival = nd.int_value;
            break;
        case UP_NODE_CONST:
            b->kind = K_DEC;
            b->dec.sign = nd.const_sign ? 1 : 0;
            b->dec.frac = nd.scale;
            b->dec.prec = nd.precision;
            b->dec.mag.m.assign(nd.const_limbs, nd.const_limbs + nd.const_nlimbs);
            big_trim(b->dec.mag);
            break;
        default:
            b->kind = K_CALC;
            b->op = nd.kind;
            b->children = {clone_in(A, nodes, nd.left, cols), clone_in(A, nodes, nd.right, cols)};
    }
    return b;
}

int emit(const BNode* b, std::vector<up_expr_node>& out) {
    up_expr_node nd;
    memset(&nd, 0, sizeof nd);
    nd.left = nd.right = -1;
    nd.reverse = b->reverse ? 1 : 0;
    nd.precision = b->prec;
    nd.scale = b->scale;
    switch (b->kind) {
        case K_COL:
            nd.kind = UP_NODE_COLUMN;
            nd.column = b->column;
            break;
        case K_INT:
            nd.kind = UP_NODE_INT;
            nd.int_value = b->ival;
            nd.precision = 0;
            nd.scale = 0;
            break;
        case K_DEC:
            nd.kind = UP_NODE_CONST;
            nd.const_sign = (int)b->dec.sign;
            nd.const_nlimbs = (int)std::min<size_t>(b->dec.mag.m.size(), UP_CONST_MAX_LIMBS);
            for (int i = 0; i < nd.const_nlimbs; i++) nd.const_limbs[i] = b->dec.mag.m[i];
            nd.scale = b->dec.frac;
            break;
        default: {
            int l = emit(b->children[0], out);
            int r = emit(b->children[1], out);
            nd.kind = b->op;
            nd.left = l;
            nd.right = r;
        }
    }
    out.push_back(nd);
    return (int)out.size() - 1;
}

}  // namespace

up_status align_optimize_impl(const up_expr_node* in, int n_in, int root, const up_col_type* cols, int n_cols,
                              std::vector<up_expr_node>& out, int& out_root) {
    // the frontend's typing of the original tree (CmpByScale reads it)
    std::vector<up_expr_node> typed(in, in + n_in);
    for (auto& nd : typed)
        if (nd.kind == UP_NODE_INT) nd.precision = nd.scale = 0;
    up_status st = derive_types_impl(typed.data(), n_in, root, cols, n_cols);
    if (st != UP_OK) return st;
    for (int k = 0; k < n_in; k++) {
        int kd = typed[k].kind;
        if (!(kd == UP_NODE_COLUMN || kd == UP_NODE_INT || kd == UP_NODE_CONST || is_calc_kind(kd)))
            return fail(UP_ERR_UNSUPPORTED, "align_optimize rewrites arithmetic trees only");
    }
    Arena A;
    BNode* b = clone_in(A, typed.data(), root, cols);
    out.clear();
    if (b->kind != K_CALC) {
        out_root = emit(b, out);
        return UP_OK;
    }
    modify_sub(b);
    MNode* m = A.from(b);
    bin_to_multi(A, b, m);
    align_opt(A, m);
    m = remove_zero(m);
    BNode* r;
    if (m->kind == K_INT || (m->kind == K_CALC && m->childList.empty())) {
        r = A.nb();
        r->kind = K_INT;
        r->ival = 0;
    } else {
        r = multi_to_bin(A, m);
    }
    if (r->kind == K_CALC && r->prec > 288) r->prec = 288;  // SUPPORTED_MAX_PRECISION, :634-636
    out_root = emit(r, out);
    return UP_OK;
}

}  // namespace upi

extern "C" up_status up_expr_align_optimize(const up_expr_node* in, int32_t n_in, int32_t root,
                                            const up_col_type* cols, int32_t n_cols, up_expr_node* out,
                                            int32_t cap, int32_t* n_out, int32_t* out_root) {
    if (!in || n_in <= 0 || !out || !n_out || !out_root) return upi::fail(UP_ERR_INVALID_ARG, "NULL arguments");
    std::vector<up_expr_node> res;
    int r = -1;
    up_status st = upi::align_optimize_impl(in, n_in, root, cols, n_cols, res, r);
    if (st != UP_OK) return st;
    if ((int)res.size() > cap) return upi::fail(UP_ERR_INVALID_ARG, "output capacity too small");
    memcpy(out, res.data(), res.size() * sizeof(up_expr_node));
    *n_out = (int32_t)res.size();
    *out_root = r;
    return UP_OK;
}
