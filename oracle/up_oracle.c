/*
 * up_oracle.c — CPU oracle for UltraPrecise's exact-decimal path.
 *
 * TEST INFRASTRUCTURE ONLY (see up_oracle.h).  Checker, never product.
 *
 * Restated semantics: AriesDecimal<LEN> (src/datatypes/AriesDecimal.hxx)
 * evaluated with LEN large enough that no intermediate is truncated, i.e.
 * every add, subtract, multiply and alignment is exact, and the divide keeps
 * the reference's three-branch rule with its two integer-width effects:
 *   - the 64-bit branch computes (|a|*10^shift) mod 2^64 and doubles the
 *     remainder mod 2^64 (AriesDecimal.hxx:581-596, 822-825);
 *   - the one-limb-divisor branch doubles the remainder mod 2^32
 *     (AriesDecimal.hxx:598-626, 827-829).
 * Grouped SUM follows decimal.cu:3319-3376 (exact sign-magnitude add) with a
 * zero result normalised to +0; AVG follows decimal.cu:2201-2446 (same
 * branch rule with the divisor a scale-0 integer count).
 */
#define _GNU_SOURCE
#include "up_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ tables */
/* Bytes per compact value.  The reference's table (decimal.cu:92, p < 300)
 * equals ceil((bitlen(10^p-1)+1)/8) except at the precisions below, where it
 * holds one byte more.  Written here as formula + exceptions so the oracle
 * does not share the product's table text. */
static const int16_t k_byte_plus_one[] = {
    31, 43, 55, 67, 79, 96, 108, 120, 132, 144, 149, 156, 161, 168,
    173, 180, 185, 192, 197, 204, 209, 214, 216, 221, 226, 228, 233, 238,
    240, 245, 250, 257, 262, 267, 269, 274, 279, 281, 286, 291, 293, 298};
/* Same idea for the word table (AriesDataType.cu:7): ceil((bitlen+1)/32)
 * plus one at these precisions. */
static const int16_t k_word_plus_one[] = {67, 96, 144, 173, 192, 221, 240, 250, 269, 279, 298};

static int32_t bitlen_pow10_minus1(int32_t p) {
    /* bitlen(10^p - 1) by exact big arithmetic on a small buffer */
    uint32_t m[ORC_MAXL];
    int n = 1;
    m[0] = 1;
    for (int i = 0; i < p; i++) {
        uint64_t c = 0;
        for (int k = 0; k < n; k++) {
            uint64_t t = (uint64_t)m[k] * 10u + c;
            m[k] = (uint32_t)t;
            c = t >> 32;
        }
        if (c) m[n++] = (uint32_t)c;
    }
    /* subtract one */
    for (int k = 0; k < n; k++) {
        if (m[k]--) break;
    }
    while (n > 0 && m[n - 1] == 0) n--;
    if (n == 0) return 0;
    return 32 * (n - 1) + (32 - __builtin_clz(m[n - 1]));
}

int32_t orc_compact_bytes(int32_t p) {
    if (p < 1) return -1;
    int32_t b = (bitlen_pow10_minus1(p) + 1 + 7) / 8;
    if (p < 300)
        for (size_t i = 0; i < sizeof(k_byte_plus_one) / sizeof(k_byte_plus_one[0]); i++)
            if (k_byte_plus_one[i] == p) b += 1;
    return b;
}

int32_t orc_precision_words(int32_t p) {
    if (p < 1) return -1;
    int32_t w = (bitlen_pow10_minus1(p) + 1 + 31) / 32;
    if (p < 300)
        for (size_t i = 0; i < sizeof(k_word_plus_one) / sizeof(k_word_plus_one[0]); i++)
            if (k_word_plus_one[i] == p) w += 1;
    return w;
}

/* ----------------------------------------------------- limb arithmetic */
static int bn_trim(const uint32_t* a, int n) {
    while (n > 0 && a[n - 1] == 0) n--;
    return n;
}

static int bn_cmp(const uint32_t* a, int na, const uint32_t* b, int nb) {
    na = bn_trim(a, na);
    nb = bn_trim(b, nb);
    if (na != nb) return na < nb ? -1 : 1;
    for (int i = na - 1; i >= 0; i--)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}

static int bn_add(uint32_t* r, const uint32_t* a, int na, const uint32_t* b, int nb) {
    if (na < nb) {
        const uint32_t* t = a; a = b; b = t;
        int tn = na; na = nb; nb = tn;
    }
    uint64_t c = 0;
    for (int i = 0; i < na; i++) {
        uint64_t t = (uint64_t)a[i] + (i < nb ? b[i] : 0) + c;
        r[i] = (uint32_t)t;
        c = t >> 32;
    }
    int n = na;
    if (c) r[n++] = (uint32_t)c;
    return bn_trim(r, n);
}

/* r = a - b, requires a >= b */
static int bn_sub(uint32_t* r, const uint32_t* a, int na, const uint32_t* b, int nb) {
    int64_t br = 0;
    for (int i = 0; i < na; i++) {
        int64_t t = (int64_t)a[i] - (i < nb ? b[i] : 0) - br;
        br = t < 0;
        r[i] = (uint32_t)t;
    }
    return bn_trim(r, na);
}

static int bn_mul(uint32_t* r, const uint32_t* a, int na, const uint32_t* b, int nb) {
    if (na == 0 || nb == 0) return 0;
    uint32_t tmp[2 * ORC_MAXL];
    memset(tmp, 0, sizeof(uint32_t) * (size_t)(na + nb));
    for (int i = 0; i < na; i++) {
        uint64_t c = 0;
        for (int j = 0; j < nb; j++) {
            uint64_t t = (uint64_t)a[i] * b[j] + tmp[i + j] + c;
            tmp[i + j] = (uint32_t)t;
            c = t >> 32;
        }
        tmp[i + nb] = (uint32_t)c;
    }
    int n = bn_trim(tmp, na + nb);
    if (n > ORC_MAXL) abort();
    memcpy(r, tmp, sizeof(uint32_t) * (size_t)n);
    return n;
}

static int bn_mul_u32(uint32_t* r, const uint32_t* a, int na, uint32_t k) {
    uint64_t c = 0;
    for (int i = 0; i < na; i++) {
        uint64_t t = (uint64_t)a[i] * k + c;
        r[i] = (uint32_t)t;
        c = t >> 32;
    }
    int n = na;
    if (c) r[n++] = (uint32_t)c;
    return bn_trim(r, n);
}

/* r = a * 10^k */
static int bn_mul_pow10(uint32_t* r, const uint32_t* a, int na, int k) {
    if (r != a) memmove(r, a, sizeof(uint32_t) * (size_t)na);
    int n = na;
    while (k >= 9) {
        n = bn_mul_u32(r, r, n, 1000000000u);
        k -= 9;
    }
    static const uint32_t p10[9] = {1, 10, 100, 1000, 10000, 100000, 1000000, 10000000, 100000000};
    if (k > 0) n = bn_mul_u32(r, r, n, p10[k]);
    if (n > ORC_MAXL) abort();
    return n;
}

static int bn_bitlen(const uint32_t* a, int n) {
    n = bn_trim(a, n);
    if (n == 0) return 0;
    return 32 * (n - 1) + (32 - __builtin_clz(a[n - 1]));
}

/* Knuth, TAOCP vol. 2, 4.3.1, Algorithm D (base 2^32).
 * q = a / b, rem = a % b; b != 0.  Returns nq, sets *nr. */
static int bn_divmod(uint32_t* q, uint32_t* rem, int* nr, const uint32_t* a, int na,
                     const uint32_t* b, int nb) {
    na = bn_trim(a, na);
    nb = bn_trim(b, nb);
    if (nb == 0) abort();
    if (bn_cmp(a, na, b, nb) < 0) {
        memmove(rem, a, sizeof(uint32_t) * (size_t)na);
        *nr = na;
        return 0;
    }
    if (nb == 1) {
        uint64_t r = 0;
        for (int i = na - 1; i >= 0; i--) {
            uint64_t cur = (r << 32) | a[i];
            q[i] = (uint32_t)(cur / b[0]);
            r = cur % b[0];
        }
        rem[0] = (uint32_t)r;
        *nr = r ? 1 : 0;
        return bn_trim(q, na);
    }
    uint32_t un[ORC_MAXL + 2], vn[ORC_MAXL + 1];
    int s = __builtin_clz(b[nb - 1]);
    for (int i = nb - 1; i > 0; i--)
        vn[i] = s ? (b[i] << s) | (b[i - 1] >> (32 - s)) : b[i];
    vn[0] = b[0] << s;
    un[na] = s ? a[na - 1] >> (32 - s) : 0;
    for (int i = na - 1; i > 0; i--)
        un[i] = s ? (a[i] << s) | (a[i - 1] >> (32 - s)) : a[i];
    un[0] = a[0] << s;
    for (int j = na - nb; j >= 0; j--) {
        uint64_t num = ((uint64_t)un[j + nb] << 32) | un[j + nb - 1];
        uint64_t qhat = num / vn[nb - 1];
        uint64_t rhat = num % vn[nb - 1];
        while (qhat >> 32 || qhat * vn[nb - 2] > ((rhat << 32) | un[j + nb - 2])) {
            qhat--;
            rhat += vn[nb - 1];
            if (rhat >> 32) break;
        }
        /* multiply and subtract */
        int64_t borrow = 0;
        uint64_t carry = 0;
        for (int i = 0; i < nb; i++) {
            uint64_t p = qhat * vn[i] + carry;
            carry = p >> 32;
            int64_t t = (int64_t)un[i + j] - (int64_t)(uint32_t)p - borrow;
            un[i + j] = (uint32_t)t;
            borrow = t < 0;
        }
        int64_t t = (int64_t)un[j + nb] - (int64_t)carry - borrow;
        un[j + nb] = (uint32_t)t;
        if (t < 0) {
            /* add back */
            qhat--;
            uint64_t c = 0;
            for (int i = 0; i < nb; i++) {
                uint64_t s2 = (uint64_t)un[i + j] + vn[i] + c;
                un[i + j] = (uint32_t)s2;
                c = s2 >> 32;
            }
            un[j + nb] += (uint32_t)c;
        }
        q[j] = (uint32_t)qhat;
    }
    for (int i = 0; i < nb; i++)
        rem[i] = s ? (un[i] >> s) | (un[i + 1] << (32 - s)) : un[i];
    *nr = bn_trim(rem, nb);
    return bn_trim(q, na - nb + 1);
}

/* ------------------------------------------------------ decimal values */
static void dec_zero(orc_dec* d) {
    d->sign = 0;
    d->frac = 0;
    d->n = 0;
}

static void dec_copy(orc_dec* d, const orc_dec* s) {
    d->sign = s->sign;
    d->frac = s->frac;
    d->n = s->n;
    memcpy(d->m, s->m, sizeof(uint32_t) * (size_t)s->n);
}

/* AriesDecimal(const CompactDecimal*, p, s), AriesDecimal.hxx:105-114:
 * copy the bytes, sign = bit 7 of the last byte, which is then cleared. */
void orc_decode(const uint8_t* bytes, int32_t nbytes, int32_t frac, orc_dec* out) {
    int nl = (nbytes + 3) / 4;
    memset(out->m, 0, sizeof(uint32_t) * (size_t)nl);
    for (int i = 0; i < nbytes; i++) out->m[i / 4] |= (uint32_t)bytes[i] << (8 * (i % 4));
    int top = nbytes - 1;
    out->sign = (bytes[top] >> 7) & 1u;
    out->m[top / 4] &= ~(0x80u << (8 * (top % 4)));
    out->frac = frac;
    out->n = bn_trim(out->m, nl);
}

/* ToCompactDecimal, AriesDecimal.hxx:308-313 with SET_SIGN_BIT
 * (decimal.hxx:91): low nbytes bytes of the magnitude, then the sign OR-ed
 * into bit 7 of the last byte. */
uint32_t orc_encode(const orc_dec* v, int32_t nbytes, uint8_t* out) {
    for (int i = 0; i < nbytes; i++) {
        int li = i / 4;
        out[i] = li < v->n ? (uint8_t)(v->m[li] >> (8 * (i % 4))) : 0;
    }
    out[nbytes - 1] |= (uint8_t)(v->sign << 7);
    return bn_bitlen(v->m, v->n) > 8 * nbytes - 1 ? UP_ROWERR_OVERFLOW : 0u;
}

/* AlignAddSubData + operator<<, AriesDecimal.hxx:116-168: the operand with
 * the smaller scale is multiplied by 10^(difference). */
static void dec_align(orc_dec* a, orc_dec* b) {
    if (a->frac < b->frac) {
        a->n = bn_mul_pow10(a->m, a->m, a->n, b->frac - a->frac);
        a->frac = b->frac;
    } else if (b->frac < a->frac) {
        b->n = bn_mul_pow10(b->m, b->m, b->n, a->frac - b->frac);
        b->frac = a->frac;
    }
}

/* operator+=, AriesDecimal.hxx:171-223 */
void orc_add(orc_dec* r, const orc_dec* a, const orc_dec* b) {
    orc_dec xs, ys;
    orc_dec* x = &xs;
    orc_dec* y = &ys;
    dec_copy(x, a);
    dec_copy(y, b);
    dec_align(x, y);
    r->frac = x->frac;
    if (x->sign == y->sign) {
        r->n = bn_add(r->m, x->m, x->n, y->m, y->n);
        r->sign = x->sign;
    } else {
        int c = bn_cmp(x->m, x->n, y->m, y->n);
        if (c >= 0) r->n = bn_sub(r->m, x->m, x->n, y->m, y->n);
        else r->n = bn_sub(r->m, y->m, y->n, x->m, x->n);
        r->sign = (c > 0 && !b->sign) || (c < 0 && b->sign);
    }
}

/* operator-=, AriesDecimal.hxx:234-289 */
void orc_sub(orc_dec* r, const orc_dec* a, const orc_dec* b) {
    orc_dec xs, ys;
    orc_dec* x = &xs;
    orc_dec* y = &ys;
    dec_copy(x, a);
    dec_copy(y, b);
    dec_align(x, y);
    r->frac = x->frac;
    if (y->sign != x->sign) {
        r->n = bn_add(r->m, x->m, x->n, y->m, y->n);
        r->sign = x->sign;
    } else {
        int c = bn_cmp(x->m, x->n, y->m, y->n);
        if (c >= 0) r->n = bn_sub(r->m, x->m, x->n, y->m, y->n);
        else r->n = bn_sub(r->m, y->m, y->n, x->m, x->n);
        r->sign = (c > 0 && y->sign) || (c < 0 && !y->sign);
    }
}

/* operator*=, AriesDecimal.hxx:316-404: sign XOR (so -x*0 is -0), scales add. */
void orc_mul(orc_dec* r, const orc_dec* a, const orc_dec* b) {
    uint32_t sign = a->sign ^ b->sign;
    int32_t frac = a->frac + b->frac;
    r->n = bn_mul(r->m, a->m, a->n, b->m, b->n);
    r->sign = sign;
    r->frac = frac;
}

/* DivOrMod(d, false), AriesDecimal.hxx:748-878 (and Decimal::DivOrMod,
 * decimal.cu:2201-2331, which has the same branch structure). */
uint32_t orc_div(orc_dec* r, const orc_dec* a, const orc_dec* b) {
    uint32_t sign = a->sign ^ b->sign;
    int32_t frac = a->frac + 4; /* DIV_FIX_EX_FRAC, decimal.hxx:56 */
    if (a->n == 0) { /* :767-771 dividend zero -> +0 */
        r->sign = 0;
        r->frac = frac;
        r->n = 0;
        return 0;
    }
    if (b->n == 0) { /* :774-777 divisor zero: value unchanged, error flag */
        if (r != a) dec_copy(r, a);
        r->sign = sign;
        r->frac = frac;
        return UP_ROWERR_DIV_BY_ZERO;
    }
    uint32_t shift = (uint32_t)b->frac + 4u;
    uint32_t hDt = (uint32_t)bn_bitlen(a->m, a->n);
    uint32_t hShift = (shift / 3) * 10 + (shift % 3 == 1 ? 4u : shift % 3 == 2 ? 7u : 0u);
    uint32_t hDs = (uint32_t)bn_bitlen(b->m, b->n);
    uint32_t q[ORC_MAXL], x[ORC_MAXL], rem[ORC_MAXL], dbl[ORC_MAXL + 1];
    int nq;
    if (hDt + hShift - 1 <= 64 && hDs <= 64) {
        /* DivByInt64, :581-596: all arithmetic in uint64 (wraps mod 2^64) */
        uint64_t dvs = (uint64_t)a->m[0] + (a->n > 1 ? (uint64_t)a->m[1] << 32 : 0);
        uint32_t sh = shift;
        while (sh > 9) {
            dvs *= 1000000000ull;
            sh -= 9;
        }
        static const uint64_t p10[10] = {1ull, 10ull, 100ull, 1000ull, 10000ull, 100000ull,
                                         1000000ull, 10000000ull, 100000000ull, 1000000000ull};
        dvs *= p10[sh];
        uint64_t dvt = (uint64_t)b->m[0] + (b->n > 1 ? (uint64_t)b->m[1] << 32 : 0);
        uint64_t res = dvs / dvt + (((dvs % dvt) << 1) >= dvt ? 1u : 0u);
        q[0] = (uint32_t)res;
        q[1] = (uint32_t)(res >> 32);
        nq = bn_trim(q, 2);
    } else {
        int nx = bn_mul_pow10(x, a->m, a->n, (int)shift);
        int nr = 0;
        nq = bn_divmod(q, rem, &nr, x, nx, b->m, b->n);
        int up;
        if (b->n == 1) {
            /* DivByInt, :598-626: remainder*2 evaluated in uint32 */
            uint32_t r32 = nr ? rem[0] : 0u;
            up = (uint32_t)(r32 * 2u) >= b->m[0];
        } else {
            /* chunked long division + doubleDivitend >= divisor, :791-873 */
            int nd = bn_add(dbl, rem, nr, rem, nr);
            up = bn_cmp(dbl, nd, b->m, b->n) >= 0;
        }
        if (up) {
            uint32_t one = 1;
            nq = bn_add(q, q, nq, &one, 1);
        }
    }
    memcpy(r->m, q, sizeof(uint32_t) * (size_t)nq);
    r->n = nq;
    r->sign = sign;
    r->frac = frac;
    return 0;
}

/* ModCalc, AriesDecimal.hxx:953-1012: magnitudes taken without alignment,
 * result scale 0, sign XOR, zero dividend -> +0.  A zero divisor is outside
 * the reference's defined behaviour; reported as DIV_BY_ZERO with value 0. */
uint32_t orc_mod(orc_dec* r, const orc_dec* a, const orc_dec* b) {
    uint32_t sign = a->sign ^ b->sign;
    if (a->n == 0) {
        r->sign = 0;
        r->frac = 0;
        r->n = 0;
        return 0;
    }
    if (b->n == 0) {
        r->sign = sign;
        r->frac = 0;
        r->n = 0;
        return UP_ROWERR_DIV_BY_ZERO;
    }
    uint32_t q[ORC_MAXL], rem[ORC_MAXL];
    int nr = 0;
    bn_divmod(q, rem, &nr, a->m, a->n, b->m, b->n);
    memcpy(r->m, rem, sizeof(uint32_t) * (size_t)nr);
    r->n = nr;
    r->sign = sign;
    r->frac = 0;
    return 0;
}

/* Extension beyond the reference's operators: change the scale by
 * truncation toward zero (or exact widening), sign kept.  Follows the
 * truncating Decimal::cast (decimal.cu:471-533). */
void orc_rescale(orc_dec* r, const orc_dec* a, int32_t scale) {
    if (r != a) dec_copy(r, a);
    if (scale > r->frac) {
        r->n = bn_mul_pow10(r->m, r->m, r->n, scale - r->frac);
    } else if (scale < r->frac) {
        uint32_t p[ORC_MAXL], q[ORC_MAXL], rem[ORC_MAXL];
        uint32_t one = 1;
        int np = bn_mul_pow10(p, &one, 1, r->frac - scale);
        int nr;
        int nq = bn_divmod(q, rem, &nr, r->m, r->n, p, np);
        memcpy(r->m, q, sizeof(uint32_t) * (size_t)nq);
        r->n = nq;
    }
    r->frac = scale;
}

/* operator< / > / == (AriesDecimal.hxx:458-570, 1023-1061): different signs
 * decide by sign alone (so -0 < +0 and -0 != +0); otherwise aligned
 * magnitudes, reversed for negatives. */
int32_t orc_compare(int32_t op, const orc_dec* a, const orc_dec* b) {
    int lt, gt, eq;
    if (a->sign != b->sign) {
        lt = a->sign == 1;
        gt = a->sign == 0;
        eq = 0;
    } else {
        orc_dec xs, ys;
        dec_copy(&xs, a);
        dec_copy(&ys, b);
        dec_align(&xs, &ys);
        int c = bn_cmp(xs.m, xs.n, ys.m, ys.n);
        eq = c == 0;
        lt = a->sign == 0 ? c < 0 : c > 0;
        gt = a->sign == 0 ? c > 0 : c < 0;
    }
    switch (op) {
        case UP_NODE_LT: return lt;
        case UP_NODE_LE: return !gt;
        case UP_NODE_GT: return gt;
        case UP_NODE_GE: return !lt;
        case UP_NODE_EQ: return eq;
        case UP_NODE_NE: return !eq;
        default: return -1;
    }
}

/* ------------------------------------------------ expression evaluation */
typedef struct {
    const up_expr_node* nodes;
    int32_t n_nodes;
    const up_col_type* col_types;
    const uint8_t* const* cols;
    orc_dec* vals;
    uint8_t* done;   /* 0 not yet evaluated, 1 a value, 2 NULL */
    uint32_t err;
} eval_ctx;

enum { EV_VALUE = 1, EV_NULL = 2 };

/* boolean nodes: comparisons, and AND/OR of booleans (AEExprAndOrNode,
 * AriesExprCalcNode.cpp:667-760; non-null values only) */
static int is_compare(int32_t k) { return k >= UP_NODE_LT && k <= UP_NODE_OR; }

static int col_value_bytes(const up_col_type* t) {
    return orc_compact_bytes(t->precision) + (t->nullable ? 1 : 0);
}

/* returns 0 on success, -1 on a malformed tree */
/* NULL propagates: a nullable column's value is NULL when its flag byte
 * (the leading byte of nullable_type, aries_types.hxx:298-330) is 0, and any
 * operator with a NULL operand is NULL without being evaluated (no row error
 * is raised for it). */
static int eval_node(eval_ctx* c, int32_t idx, int64_t row) {
    if (idx < 0 || idx >= c->n_nodes) return -1;
    if (c->done[idx]) return 0;
    const up_expr_node* nd = &c->nodes[idx];
    orc_dec* out = &c->vals[idx];
    if (nd->left >= 0 || nd->right >= 0) {
        if (nd->left >= 0 && eval_node(c, nd->left, row)) return -1;
        if (nd->right >= 0 && eval_node(c, nd->right, row)) return -1;
        if ((nd->left >= 0 && c->done[nd->left] == EV_NULL) || (nd->right >= 0 && c->done[nd->right] == EV_NULL)) {
            dec_zero(out);
            c->done[idx] = EV_NULL;
            return 0;
        }
    }
    switch (nd->kind) {
        case UP_NODE_COLUMN: {
            const up_col_type* t = &c->col_types[nd->column];
            int vb = col_value_bytes(t);
            const uint8_t* p = c->cols[nd->column] + row * vb;
            if (t->nullable) {
                if (p[0] == 0) {
                    dec_zero(out);
                    c->done[idx] = EV_NULL;
                    return 0;
                }
                p += 1;
            }
            orc_decode(p, orc_compact_bytes(t->precision), t->scale, out);
            break;
        }
        case UP_NODE_CONST:
            out->sign = (uint32_t)(nd->const_sign != 0);
            out->frac = nd->scale;
            out->n = bn_trim(nd->const_limbs, nd->const_nlimbs);
            memcpy(out->m, nd->const_limbs, sizeof(uint32_t) * (size_t)out->n);
            break;
        case UP_NODE_INT: {
            /* AriesDecimal(int32_t), AriesDecimal.hxx:896-904 (magnitude, sign) */
            int64_t v = nd->int_value;
            uint64_t mag = v < 0 ? (uint64_t)(-(v + 1)) + 1u : (uint64_t)v;
            out->sign = v < 0;
            out->frac = 0;
            out->m[0] = (uint32_t)mag;
            out->m[1] = (uint32_t)(mag >> 32);
            out->n = bn_trim(out->m, 2);
            break;
        }
        case UP_NODE_ADD: case UP_NODE_SUB: case UP_NODE_MUL: case UP_NODE_DIV:
        case UP_NODE_MOD: {
            if (eval_node(c, nd->left, row) || eval_node(c, nd->right, row)) return -1;
            const orc_dec* a = &c->vals[nd->left];
            const orc_dec* b = &c->vals[nd->right];
            if (nd->kind == UP_NODE_ADD) orc_add(out, a, b);
            else if (nd->kind == UP_NODE_SUB) orc_sub(out, a, b);
            else if (nd->kind == UP_NODE_MUL) orc_mul(out, a, b);
            else if (nd->kind == UP_NODE_DIV) c->err |= orc_div(out, a, b);
            else c->err |= orc_mod(out, a, b);
            break;
        }
        case UP_NODE_RESCALE:
            if (eval_node(c, nd->left, row)) return -1;
            orc_rescale(out, &c->vals[nd->left], nd->scale);
            break;
        default:
            if (is_compare(nd->kind)) {
                if (eval_node(c, nd->left, row) || eval_node(c, nd->right, row)) return -1;
                int v;
                if (nd->kind == UP_NODE_AND || nd->kind == UP_NODE_OR) {
                    const int l = c->vals[nd->left].n != 0, r = c->vals[nd->right].n != 0;
                    v = nd->kind == UP_NODE_AND ? (l && r) : (l || r);
                } else {
                    v = orc_compare(nd->kind, &c->vals[nd->left], &c->vals[nd->right]);
                }
                dec_zero(out);
                out->m[0] = (uint32_t)v;
                out->n = v ? 1 : 0;
                break;
            }
            return -1;
    }
    if (nd->reverse) out->sign ^= 1u; /* operator-(), AriesDecimal.hxx:291-300 */
    c->done[idx] = EV_VALUE;
    return 0;
}

/* 1 when a nullable column is reachable from node idx */
static int reaches_nullable(const up_expr_node* nodes, int32_t n_nodes, const up_col_type* col_types, int32_t idx,
                            int depth) {
    if (idx < 0 || idx >= n_nodes || depth > n_nodes) return 0;
    const up_expr_node* nd = &nodes[idx];
    if (nd->kind == UP_NODE_COLUMN) return col_types[nd->column].nullable != 0;
    return reaches_nullable(nodes, n_nodes, col_types, nd->left, depth + 1) ||
           reaches_nullable(nodes, n_nodes, col_types, nd->right, depth + 1);
}

int32_t orc_eval_expr(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                      const up_col_type* col_types, const uint8_t* const* cols,
                      int64_t row_begin, int64_t row_end,
                      uint8_t* out, int32_t out_bytes, uint32_t* err, uint8_t* row_err) {
    eval_ctx c;
    c.nodes = nodes;
    c.n_nodes = n_nodes;
    c.col_types = col_types;
    c.cols = cols;
    c.vals = (orc_dec*)malloc(sizeof(orc_dec) * (size_t)n_nodes);
    c.done = (uint8_t*)malloc((size_t)n_nodes);
    uint32_t all = 0;
    int rc = 0;
    int cmp = is_compare(nodes[root].kind);
    /* a nullable result (any nullable column in the tree) is a flag byte, 1
     * for a value, then the value; a NULL row stores flag 0 and zero bytes */
    const int nullable = reaches_nullable(nodes, n_nodes, col_types, root, 0);
    for (int64_t row = row_begin; row < row_end; row++) {
        memset(c.done, 0, (size_t)n_nodes);
        c.err = 0;
        if (eval_node(&c, root, row)) {
            rc = -1;
            break;
        }
        uint8_t* o = out + row * out_bytes;
        int vbytes = out_bytes;
        if (nullable) {
            o[0] = c.done[root] == EV_NULL ? 0 : 1;
            o += 1;
            vbytes -= 1;
            if (c.done[root] == EV_NULL) {
                memset(o, 0, (size_t)vbytes);
                if (row_err) row_err[row] = 0;
                continue;
            }
        }
        if (cmp) {
            o[0] = (uint8_t)(c.vals[root].n != 0);
        } else {
            c.err |= orc_encode(&c.vals[root], vbytes, o);
        }
        if (row_err) row_err[row] = (uint8_t)c.err;
        all |= c.err;
    }
    free(c.vals);
    free(c.done);
    if (err) *err |= all;
    return rc;
}

typedef struct {
    const up_expr_node* nodes;
    int32_t n_nodes, root;
    const up_col_type* col_types;
    const uint8_t* const* cols;
    int64_t b, e;
    uint8_t* out;
    int32_t out_bytes;
    uint32_t err;
    int32_t rc;
} eval_job;

static void* eval_thread(void* arg) {
    eval_job* j = (eval_job*)arg;
    j->err = 0;
    j->rc = orc_eval_expr(j->nodes, j->n_nodes, j->root, j->col_types, j->cols, j->b, j->e,
                          j->out, j->out_bytes, &j->err, NULL);
    return NULL;
}

int32_t orc_eval_expr_mt(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                         const up_col_type* col_types, const uint8_t* const* cols,
                         int64_t rows, uint8_t* out, int32_t out_bytes, uint32_t* err,
                         int32_t threads) {
    if (threads < 1) threads = 1;
    eval_job* jobs = (eval_job*)calloc((size_t)threads, sizeof(eval_job));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    int64_t chunk = (rows + threads - 1) / threads;
    for (int t = 0; t < threads; t++) {
        eval_job* j = &jobs[t];
        j->nodes = nodes;
        j->n_nodes = n_nodes;
        j->root = root;
        j->col_types = col_types;
        j->cols = cols;
        j->b = t * chunk < rows ? t * chunk : rows;
        j->e = (t + 1) * chunk < rows ? (t + 1) * chunk : rows;
        j->out = out;
        j->out_bytes = out_bytes;
        pthread_create(&th[t], NULL, eval_thread, j);
    }
    int32_t rc = 0;
    for (int t = 0; t < threads; t++) {
        pthread_join(th[t], NULL);
        if (err) *err |= jobs[t].err;
        if (jobs[t].rc) rc = jobs[t].rc;
    }
    free(jobs);
    free(th);
    return rc;
}

/* ------------------------------------------------ grouped aggregation */
/* nullable_type<Decimal> image (decimal.hxx:130-140 + flag byte):
 * [0] flag, [1] sign, [2] prec, [3] frac, [4] error, [5..133) v[32]. */
static void write_agg_image(uint8_t* img, int flag, const orc_dec* v) {
    memset(img, 0, UP_AGG_DECIMAL_BYTES);
    img[0] = (uint8_t)flag;
    img[1] = (uint8_t)v->sign;
    img[2] = 0;
    img[3] = (uint8_t)v->frac;
    img[4] = 0;
    for (int i = 0; i < 32 && i < v->n; i++) memcpy(img + 5 + 4 * i, &v->m[i], 4);
}

static void read_agg_image(const uint8_t* img, orc_dec* v) {
    v->sign = img[1];
    v->frac = img[3];
    for (int i = 0; i < 32; i++) memcpy(&v->m[i], img + 5 + 4 * i, 4);
    v->n = bn_trim(v->m, 32);
}

static void count_to_dec(int64_t cnt, orc_dec* d) {
    /* Decimal(int64_t), decimal.cu:301-309: scale 0 */
    d->sign = 0;
    d->frac = 0;
    d->m[0] = (uint32_t)cnt;
    d->m[1] = (uint32_t)((uint64_t)cnt >> 32);
    d->n = bn_trim(d->m, 2);
}

/* nullable_type<Decimal> /= int64 (aries_types.hxx:626-631): the value is
 * divided by Decimal::DivOrMod (decimal.cu:2200-2228) and the flag survives
 * only a nonzero divisor.  DivOrMod raises frac by 4 first; a zero dividend
 * then returns +0 with prec = frac + 1; a zero divisor leaves the value and
 * sets error = ERR_DIV_BY_ZERO (decimal.hxx:28). */
static void write_avg_image(uint8_t* img, int sum_flag, int64_t count, const orc_dec* dividend,
                            const orc_dec* r, uint32_t e) {
    write_agg_image(img, sum_flag && count != 0, r);
    if (dividend->n == 0) {
        img[1] = 0;
        img[2] = (uint8_t)(r->frac + 1);
    }
    if (e & UP_ROWERR_DIV_BY_ZERO) img[4] = 2;
}

void orc_division_int64(const uint8_t* sum_img, int64_t count, uint8_t* out_img) {
    orc_dec* s = (orc_dec*)malloc(3 * sizeof(orc_dec));
    orc_dec* c = s + 1;
    orc_dec* r = s + 2;
    read_agg_image(sum_img, s);
    count_to_dec(count, c);
    uint32_t e = orc_div(r, s, c);
    write_avg_image(out_img, sum_img[0] != 0, count, s, r, e);
    free(s);
}

/* accumulate into per-group sign-magnitude sums, then finalize */
static void finalize_group(uint8_t* out, int32_t kind, orc_dec* sum, int64_t cnt, int32_t g) {
    if (kind == UP_AGG_COUNT) {
        memcpy(out + 8 * (int64_t)g, &cnt, 8);
        return;
    }
    if (sum->n == 0) sum->sign = 0; /* -0 from cancellation normalised to +0 */
    uint8_t* img = out + (int64_t)UP_AGG_DECIMAL_BYTES * g;
    if (kind == UP_AGG_SUM) {
        write_agg_image(img, cnt > 0, sum);
        return;
    }
    /* AVG = DivisionInt64 of the SUM by the count; a group without rows has a
     * zero sum, which the divide rule's zero-dividend case handles */
    orc_dec* c = (orc_dec*)malloc(2 * sizeof(orc_dec));
    orc_dec* r = c + 1;
    count_to_dec(cnt, c);
    uint32_t e = orc_div(r, sum, c);
    write_avg_image(img, cnt > 0, cnt, sum, r, e);
    free(c);
}

int32_t orc_group_agg(const uint8_t* vals, int32_t value_bytes, int32_t scale,
                      int32_t kind, const int32_t* group_ids, int64_t rows,
                      int32_t n_groups, uint8_t* out) {
    orc_dec* sums = (orc_dec*)calloc((size_t)n_groups, sizeof(orc_dec));
    int64_t* cnts = (int64_t*)calloc((size_t)n_groups, sizeof(int64_t));
    orc_dec* v = (orc_dec*)malloc(2 * sizeof(orc_dec));
    orc_dec* t = v + 1;
    for (int32_t g = 0; g < n_groups; g++) sums[g].frac = scale;
    for (int64_t i = 0; i < rows; i++) {
        int32_t g = group_ids[i];
        if (g < 0 || g >= n_groups) continue;
        cnts[g]++;
        if (kind == UP_AGG_COUNT) continue;
        orc_decode(vals + i * value_bytes, value_bytes, scale, v);
        orc_add(t, &sums[g], v);
        dec_copy(&sums[g], t);
    }
    for (int32_t g = 0; g < n_groups; g++) finalize_group(out, kind, &sums[g], cnts[g], g);
    free(v);
    free(sums);
    free(cnts);
    return 0;
}

typedef struct {
    const up_expr_node* nodes;
    int32_t n_nodes;
    const up_col_type* col_types;
    const uint8_t* const* cols;
    const up_query_agg* aggs;
    int32_t n_aggs;
    const int32_t* group_ids;
    int64_t b, e;
    int32_t n_groups;
    orc_dec* sums;   /* [n_aggs][n_groups] */
    int64_t* cnts;   /* [n_groups]: rows of the group (COUNT(*)) */
    int64_t* acnts;  /* [n_aggs][n_groups]: rows whose aggregated expression is not NULL */
} query_job;

static void* query_thread(void* arg) {
    query_job* j = (query_job*)arg;
    eval_ctx c;
    c.nodes = j->nodes;
    c.n_nodes = j->n_nodes;
    c.col_types = j->col_types;
    c.cols = j->cols;
    c.vals = (orc_dec*)malloc(sizeof(orc_dec) * (size_t)(j->n_nodes + 1));
    c.done = (uint8_t*)malloc((size_t)j->n_nodes);
    orc_dec* t = &c.vals[j->n_nodes];
    for (int64_t row = j->b; row < j->e; row++) {
        int32_t g = j->group_ids[row];
        if (g < 0 || g >= j->n_groups) continue;
        memset(c.done, 0, (size_t)j->n_nodes);
        j->cnts[g]++;
        for (int32_t a = 0; a < j->n_aggs; a++) {
            if (j->aggs[a].kind == UP_AGG_COUNT) continue;
            c.err = 0;
            eval_node(&c, j->aggs[a].root, row);
            /* SUM/AVG skip NULLs (agg_sum_t on nullable_type, operators.hxx:1176-1193) */
            if (c.done[j->aggs[a].root] == EV_NULL) continue;
            j->acnts[(int64_t)a * j->n_groups + g]++;
            orc_dec* s = &j->sums[(int64_t)a * j->n_groups + g];
            orc_add(t, s, &c.vals[j->aggs[a].root]);
            dec_copy(s, t);
        }
    }
    free(c.vals);
    free(c.done);
    return NULL;
}

int32_t orc_query(const up_expr_node* nodes, int32_t n_nodes,
                  const up_col_type* col_types, const uint8_t* const* cols,
                  const up_query_agg* aggs, int32_t n_aggs,
                  const int32_t* group_ids, int64_t rows, int32_t n_groups,
                  uint8_t* const* outs, int32_t threads) {
    if (threads < 1) threads = 1;
    query_job* jobs = (query_job*)calloc((size_t)threads, sizeof(query_job));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    int64_t chunk = (rows + threads - 1) / threads;
    /* per-aggregate result scale: the root's scale as the evaluation yields it */
    for (int t = 0; t < threads; t++) {
        query_job* j = &jobs[t];
        j->nodes = nodes;
        j->n_nodes = n_nodes;
        j->col_types = col_types;
        j->cols = cols;
        j->aggs = aggs;
        j->n_aggs = n_aggs;
        j->group_ids = group_ids;
        j->b = t * chunk < rows ? t * chunk : rows;
        j->e = (t + 1) * chunk < rows ? (t + 1) * chunk : rows;
        j->n_groups = n_groups;
        j->sums = (orc_dec*)calloc((size_t)n_aggs * (size_t)n_groups, sizeof(orc_dec));
        j->cnts = (int64_t*)calloc((size_t)n_groups, sizeof(int64_t));
        j->acnts = (int64_t*)calloc((size_t)n_aggs * (size_t)n_groups, sizeof(int64_t));
        for (int32_t a = 0; a < n_aggs; a++)
            for (int32_t g = 0; g < n_groups; g++)
                j->sums[(int64_t)a * n_groups + g].frac = nodes[aggs[a].root].scale;
        pthread_create(&th[t], NULL, query_thread, j);
    }
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    /* merge thread partials exactly, in thread order */
    orc_dec* tmp = (orc_dec*)malloc(sizeof(orc_dec));
    for (int t = 1; t < threads; t++) {
        for (int32_t g = 0; g < n_groups; g++) jobs[0].cnts[g] += jobs[t].cnts[g];
        for (int64_t k = 0; k < (int64_t)n_aggs * n_groups; k++) jobs[0].acnts[k] += jobs[t].acnts[k];
        for (int64_t k = 0; k < (int64_t)n_aggs * n_groups; k++) {
            orc_add(tmp, &jobs[0].sums[k], &jobs[t].sums[k]);
            dec_copy(&jobs[0].sums[k], tmp);
        }
    }
    free(tmp);
    for (int32_t a = 0; a < n_aggs; a++)
        for (int32_t g = 0; g < n_groups; g++)
            finalize_group(outs[a], aggs[a].kind, &jobs[0].sums[(int64_t)a * n_groups + g],
                           aggs[a].kind == UP_AGG_COUNT ? jobs[0].cnts[g] : jobs[0].acnts[(int64_t)a * n_groups + g],
                           g);
    for (int t = 0; t < threads; t++) {
        free(jobs[t].sums);
        free(jobs[t].cnts);
        free(jobs[t].acnts);
    }
    free(jobs);
    free(th);
    return 0;
}
