// up_dev.cuh — device arithmetic on compact decimals for sm_100a.
//
// Compiled two ways: embedded into every NVRTC-generated expression kernel,
// and included by the precompiled .cu files.  Uses no standard headers.
//
// Values are sign-magnitude: a little-endian base-2^32 magnitude held in a
// fixed-size register array whose length is a compile-time bound derived from
// the operands' bit widths, plus a sign word; the scale is static (it is part
// of the expression type), so it never appears at run time.
//
// Semantics follow UltraPrecise's AriesDecimal<LEN> (src/datatypes/
// AriesDecimal.hxx) with LEN large enough that nothing is truncated:
//   add/sub sign rules    AriesDecimal.hxx:171-289
//   multiply              AriesDecimal.hxx:316-404  (sign XOR: -x*0 = -0)
//   divide                AriesDecimal.hxx:581-626, 748-878 (three branches)
//   compare               AriesDecimal.hxx:458-570, 1023-1061
//   compact load/store    AriesDecimal.hxx:105-114, 308-313; decimal.hxx:91-92
#ifndef UP_DEV_CUH_
#define UP_DEV_CUH_

#include "up_kargs.h"

namespace up {

typedef unsigned int u32;
typedef unsigned long long u64;
typedef long long i64;
typedef unsigned char u8;

#define UP_DI __device__ __forceinline__

#ifndef UP_MUL_UNROLL_PAIRS
#define UP_MUL_UNROLL_PAIRS 4096
#endif
constexpr int kMulUnrollPairs = UP_MUL_UNROLL_PAIRS;

enum : u32 { ERR_OVERFLOW = 1u, ERR_DIV0 = 2u, ERR_DOMAIN = 4u };

// ----------------------------------------------------------------- limbs
template <int N>
UP_DI u32 at(const u32 (&a)[N], int i) {
    return (i >= 0 && i < N) ? a[(i >= 0 && i < N) ? i : 0] : 0u;
}

template <int N>
UP_DI void zero(u32 (&r)[N]) {
#pragma unroll
    for (int i = 0; i < N; i++) r[i] = 0u;
}

template <int N, int M>
UP_DI void copy_ext(u32 (&r)[N], const u32 (&a)[M]) {
#pragma unroll
    for (int i = 0; i < N; i++) r[i] = at(a, i);
}

template <int N>
UP_DI bool is_zero(const u32 (&a)[N]) {
    u32 o = 0;
#pragma unroll
    for (int i = 0; i < N; i++) o |= a[i];
    return o == 0u;
}

// number of significant bits (0 for zero)
template <int N>
UP_DI u32 bitlen(const u32 (&a)[N]) {
    u32 r = 0;
#pragma unroll
    for (int i = 0; i < N; i++) r = a[i] ? 32u * i + 32u - (u32)__clz(a[i]) : r;
    return r;
}

// -1, 0, 1 comparing magnitudes
template <int NA, int NB>
UP_DI int cmp(const u32 (&a)[NA], const u32 (&b)[NB]) {
    constexpr int M = NA > NB ? NA : NB;
    int r = 0;
#pragma unroll
    for (int i = 0; i < M; i++) {
        u32 x = at(a, i), y = at(b, i);
        r = x != y ? (x < y ? -1 : 1) : r;
    }
    return r;
}

// r = a + b over N limbs; returns the carry out of limb N-1
template <int N, int NA, int NB>
UP_DI u32 add(u32 (&r)[N], const u32 (&a)[NA], const u32 (&b)[NB]) {
    u64 c = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        c += (u64)at(a, i) + at(b, i);
        r[i] = (u32)c;
        c >>= 32;
    }
    return (u32)c;
}

// r = a - b over N limbs (two's complement); returns 1 when a < b
template <int N, int NA, int NB>
UP_DI u32 sub(u32 (&r)[N], const u32 (&a)[NA], const u32 (&b)[NB]) {
    u64 c = 1;
#pragma unroll
    for (int i = 0; i < N; i++) {
        c += (u64)at(a, i) + (u64)(~at(b, i));
        r[i] = (u32)c;
        c >>= 32;
    }
    return (u32)(c ^ 1u);
}

template <int N>
UP_DI void negate(u32 (&r)[N]) {
    u64 c = 1;
#pragma unroll
    for (int i = 0; i < N; i++) {
        c += (u64)(~r[i]);
        r[i] = (u32)c;
        c >>= 32;
    }
}

// r += k (small), over N limbs
template <int N>
UP_DI void add_small(u32 (&r)[N], u32 k) {
    u64 c = k;
#pragma unroll
    for (int i = 0; i < N; i++) {
        c += r[i];
        r[i] = (u32)c;
        c >>= 32;
    }
}

// Signed add with AriesDecimal operator+= rules (AriesDecimal.hxx:171-223):
// equal signs add magnitudes and keep the sign; different signs subtract the
// smaller magnitude from the larger, the sign follows the larger, and equal
// magnitudes give +0.  Subtraction is this with b's sign flipped (the
// operator-= rules, AriesDecimal.hxx:234-289, reduce to exactly that).
template <int N, int NA, int NB>
UP_DI void add_signed(u32 (&r)[N], u32& sr, const u32 (&a)[NA], u32 sa, const u32 (&b)[NB], u32 sb) {
    const bool same = sa == sb;
    const u32 x = same ? 0u : 0xffffffffu;
    u64 c = same ? 0u : 1u;
#pragma unroll
    for (int i = 0; i < N; i++) {
        c += (u64)at(a, i) + (u64)(at(b, i) ^ x);
        r[i] = (u32)c;
        c >>= 32;
    }
    const bool neg = !same && c == 0u;  // a < b
    if (neg) negate(r);
    const bool nz = !is_zero(r);
    sr = same ? sa : (nz ? (neg ? sb : (sb ^ 1u)) : 0u);
}

// r = a * b (low N limbs of the product)
template <int N, int NA, int NB>
UP_DI void mul(u32 (&r)[N], const u32 (&a)[NA], const u32 (&b)[NB]) {
    zero(r);
    // products above UP_MUL_UNROLL_PAIRS limb pairs keep the outer loop rolled
    // (compile time)
#pragma unroll((NA * NB <= kMulUnrollPairs) ? NA : 1)
    for (int i = 0; i < NA; i++) {
        if (i >= N) break;
        u64 c = 0;
#pragma unroll
        for (int j = 0; j < NB; j++) {
            if (i + j < N) {
                u64 t = (u64)a[i] * b[j] + r[i + j] + c;
                r[i + j] = (u32)t;
                c = t >> 32;
            }
        }
        if (i + NB < N) r[i + NB] = (u32)c;
    }
}

// r = a * k (k one limb)
template <int N, int NA>
UP_DI void mul_u32(u32 (&r)[N], const u32 (&a)[NA], u32 k) {
    u64 c = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        u64 t = (u64)at(a, i) * k + c;
        r[i] = (u32)t;
        c = t >> 32;
    }
}

// ----------------------------------------------------------- shifts
// r = a << s (bits, dynamic s in [0, 32*N)), truncated to N limbs
template <int N>
UP_DI void shl_bits(u32 (&r)[N], const u32 (&a)[N], u32 s) {
    u32 t[N];
    copy_ext(t, a);
    // limb shift by s/32, done as a barrel of static shifts (skipped as a
    // whole when s < 32, the usual case of a normalising shift)
    const u32 ls = s >> 5;
    if (ls != 0u) {
#pragma unroll
        for (int k = 1; k < N; k <<= 1) {
            if (ls & (u32)k) {
#pragma unroll
                for (int i = N - 1; i >= 0; i--) t[i] = i >= k ? t[i >= k ? i - k : 0] : 0u;
            }
        }
    }
    const u32 bs = s & 31u;
#pragma unroll
    for (int i = N - 1; i >= 0; i--) r[i] = __funnelshift_l(i > 0 ? t[i > 0 ? i - 1 : 0] : 0u, t[i], bs);
}

// r = a >> s (bits, dynamic s in [0, 32*N))
template <int N>
UP_DI void shr_bits(u32 (&r)[N], const u32 (&a)[N], u32 s) {
    u32 t[N];
    copy_ext(t, a);
    const u32 ls = s >> 5;
    if (ls != 0u) {
#pragma unroll
        for (int k = 1; k < N; k <<= 1) {
            if (ls & (u32)k) {
#pragma unroll
                for (int i = 0; i < N; i++) t[i] = i + k < N ? t[i + k < N ? i + k : 0] : 0u;
            }
        }
    }
    const u32 bs = s & 31u;
#pragma unroll
    for (int i = 0; i < N; i++) r[i] = __funnelshift_r(t[i], i + 1 < N ? t[i + 1 < N ? i + 1 : 0] : 0u, bs);
}

// ------------------------------------------------------------ division
// Integer division runs its quotient-digit estimates on the FP64 pipe (idle
// in these kernels) instead of 64-bit integer divides, which the GPU has no
// instruction for: each estimate is a few double operations and is then made
// exact by integer multiply-subtract and at most one correction.

// Exact double of a 32-bit value without a conversion instruction: the
// value's bits as the mantissa of 2^52 + x, minus 2^52 (exact).
UP_DI double u32_to_f64(u32 x) { return __dadd_rn(__hiloint2double(0x43300000, (int)x), -4503599627370496.0); }

// floor(e) for 0 <= e < 2^32, or 0xffffffff when floor(e) >= 2^32: adding
// 2^52 rounded toward -inf leaves floor(e) in the low mantissa bits.
UP_DI u32 f64_floor_u32_sat(double e) {
    const double y = __dadd_rd(e, 4503599627370496.0);
    return __double2hiint(y) == 0x43300000 ? (u32)__double2loint(y) : 0xffffffffu;
}

// Reciprocal of a normalised divisor d (top bit set) for the 2/1 division of
// Moller & Granlund, "Improved division by invariant integers" (IEEE Trans.
// Computers, 2011): v = floor((2^64 - 1) / d) - 2^32.  The double estimate
// 2^64/d - 2^32 is within 2^-19 of the exact quotient; taking one less and
// stepping up while (2^32 + v + 1) * d < 2^64 makes it exact in at most two
// steps.
UP_DI u32 reciprocal_u32(u32 d) {
    const double r = __drcp_rn(u32_to_f64(d));                      // 1/d, correctly rounded
    const double e = __fma_rn(r, 18446744073709551616.0, -4294967296.0);  // ~ 2^64/d - 2^32, in [0, 2^32]
    u32 v = f64_floor_u32_sat(e);
    v = v ? v - 1u : 0u;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        // (2^32 + v + 1) * d = d * 2^32 + (v + 1) * d; below 2^64 when the sum does not carry
        const u64 lo = (u64)(v + 1u) * d;
        const u64 hi = (u64)d << 32;
        const bool below = v != 0xffffffffu && lo + hi >= hi;
        v += below ? 1u : 0u;
    }
    return v;
}

// 2/1 division by a normalised 32-bit divisor with its reciprocal v (Moller
// & Granlund 2011, Algorithm 4); u1 < d; returns floor((u1*2^32 + u0)/d) and
// the remainder in r.
UP_DI u32 div2by1(u32 u1, u32 u0, u32 d, u32 v, u32& r) {
    u64 q = (u64)v * u1;
    q += ((u64)u1 << 32) | u0;
    u32 q1 = (u32)(q >> 32) + 1u;
    const u32 q0 = (u32)q;
    u32 rr = u0 - q1 * d;
    if (rr > q0) {
        q1 -= 1u;
        rr += d;
    }
    if (rr >= d) {
        q1 += 1u;
        rr -= d;
    }
    r = rr;
    return q1;
}

// Quotient digits of Knuth's Algorithm D from the FP64 pipe.  With the
// divisor normalised (its top limb vtop has the top bit set) and the current
// remainder window w[0..n] < divisor * 2^32, the digit is
// floor(window / divisor) < 2^32.  The estimate is (w[n]:w[n-1]) * 2^32 /
// (vtop:vnext) in doubles: its relative error is below 2^-51 (four roundings)
// and the limbs it leaves out move it by less than 2^-31, so it is within
// 2^-18.9 of the exact quotient; biased up by 2^-18 and floored it is the
// digit or the digit + 1, which Algorithm D's add-back corrects.
struct QuotEst {
    double rcp;  // 2^32 / (vtop:vnext), correctly rounded
    UP_DI void init(u32 vtop, u32 vnext) {
        const double vd = __fma_rn(u32_to_f64(vtop), 4294967296.0, u32_to_f64(vnext));
        rcp = __dmul_rn(__drcp_rn(vd), 4294967296.0);
    }
    UP_DI u32 digit(u32 u1, u32 u0) const {
        const double t = __fma_rn(u32_to_f64(u1), 4294967296.0, u32_to_f64(u0));
        return f64_floor_u32_sat(__fma_rn(t, rcp, 3.814697265625e-06));  // + 2^-18
    }
};

// One step of Algorithm D on the window w[0..NB]: subtract qhat * bn, add
// back once when qhat was one too large; returns the digit.
template <int NB>
UP_DI u32 knuth_step(u32 (&w)[NB + 1], const u32 (&bn)[NB], u32 qhat) {
    u64 carry = 0;
    i64 borrow = 0;
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const u64 p = (u64)qhat * bn[i] + carry;
        carry = p >> 32;
        const i64 t = (i64)w[i] - (i64)(u32)p + borrow;
        w[i] = (u32)t;
        borrow = t >> 32;  // 0 or -1
    }
    const i64 t = (i64)w[NB] - (i64)carry + borrow;
    w[NB] = (u32)t;
    if (t < 0) {
        qhat--;
        u64 c = 0;
#pragma unroll
        for (int i = 0; i < NB; i++) {
            c += (u64)w[i] + bn[i];
            w[i] = (u32)c;
            c >>= 32;
        }
        w[NB] += (u32)c;
    }
    return qhat;
}

// Knuth, TAOCP vol. 2, 4.3.1, Algorithm D in base 2^32 with static array
// sizes: the divisor is normalised to exactly NB limbs (top bit set) by a
// dynamic left shift s applied to both operands; the nx - nb + 1 quotient
// digits that can be nonzero are produced (nx, nb: the operands' significant
// limbs), each estimated by QuotEst.  q = floor(x / b); rn = (x mod b) << s
// and bn = b << s (the normalised remainder and divisor, which is all a
// rounding decision needs).  Requires b != 0.
template <int NX, int NB>
UP_DI void divmod_norm(u32 (&q)[NX], u32 (&rn)[NB], u32 (&bn)[NB], u32& s, const u32 (&x)[NX],
                       const u32 (&b)[NB]) {
    if constexpr (NB == 1) {
        const u32 sh = (u32)__clz(b[0]);
        const u32 d = b[0] << sh;
        const u32 v = reciprocal_u32(d);
        u32 r = sh ? (x[NX - 1] >> (32u - sh)) : 0u;
#pragma unroll
        for (int i = NX - 1; i >= 0; i--) {
            const u32 lo = sh ? __funnelshift_l(i > 0 ? x[i > 0 ? i - 1 : 0] : 0u, x[i], sh) : x[i];
            q[i] = div2by1(r, lo, d, v, r);
        }
        rn[0] = r;
        bn[0] = d;
        s = sh;
    } else {
    // the shift reaches past a limb when b's value is narrower than NB limbs
    constexpr int NU = NX + NB + 1;
    constexpr bool kUnroll = (NX + 1) * NB <= 96;
    const u32 bl = bitlen(b);
    s = 32u * NB - bl;  // normalising shift
    u32 un[NU];
    if constexpr (kUnroll) {
        shl_bits(bn, b, s);
        u32 xe[NU];
        copy_ext(xe, x);
        shl_bits(un, xe, s);
    } else {
        // Wide operands: un is indexed by the digit loop (local memory), so
        // it is written limb by limb at its shifted position, and a limb
        // shift of b (a divisor narrower than NB limbs) goes through a local
        // copy; a barrel of static shifts would hold several copies of the
        // operands in registers at once.
        const u32 ls = s >> 5, bs = s & 31u;
        // zero the limbs the shifted dividend leaves free, below and above it
        for (int i = 0; i < (int)ls; i++) un[i] = 0u;
        for (int i = NX + 1 + (int)ls; i < NU; i++) un[i] = 0u;
#pragma unroll
        for (int i = 0; i <= NX; i++) {
            const u32 hi = i < NX ? x[i < NX ? i : 0] : 0u;
            const u32 lo = i > 0 ? x[i > 0 ? i - 1 : 0] : 0u;
            un[i + ls] = __funnelshift_l(lo, hi, bs);
        }
        if (ls == 0u) {
#pragma unroll
            for (int i = 0; i < NB; i++) bn[i] = __funnelshift_l(i > 0 ? b[i > 0 ? i - 1 : 0] : 0u, b[i], bs);
        } else {
            u32 bt[NB];
#pragma unroll
            for (int i = 0; i < NB; i++) bt[i] = b[i];
#pragma unroll
            for (int i = 0; i < NB; i++) {
                const int k = i - (int)ls;
                const u32 hi = k >= 0 ? bt[k >= 0 ? k : 0] : 0u;
                const u32 lo = k >= 1 ? bt[k >= 1 ? k - 1 : 0] : 0u;
                bn[i] = __funnelshift_l(lo, hi, bs);
            }
        }
    }
    QuotEst est;
    est.init(bn[NB - 1], bn[NB - 2]);
    // digits j = jmax .. 0 with jmax = nx - nb; the window of digit j is un[j .. j+NB]
    const int jmax = (int)((bitlen(x) + 31u) >> 5) - (int)((bl + 31u) >> 5);
#pragma unroll
    for (int i = 0; i < NX; i++) q[i] = 0u;
    if (jmax < 0) {  // x < b: the remainder is x itself
#pragma unroll
        for (int i = 0; i < NB; i++) rn[i] = un[i];
        return;
    }
    if constexpr (!kUnroll && NB <= 64) {
        // Wide operands: the rolled loop keeps the current remainder window
        // un[j .. j+NB] in registers (static indices) and moves it down one
        // limb per quotient digit, reading a single dividend limb per step
        // (windows above 16 limbs one digit per iteration: measured on B200
        // the two-digit body, which saves the moves, was slower there and
        // faster below).
        u32 w[NB + 1];
#pragma unroll
        for (int i = 0; i <= NB; i++) w[i] = un[jmax + i];
        // the next dividend limb is loaded one step ahead (local-memory
        // latency overlaps the multiply-subtract)
        int j = jmax;
        if constexpr (NB > 16) {
            u32 nxt = j >= 1 ? un[j - 1] : 0u;
#pragma unroll 1
            for (; j >= 1; j--) {
                const u32 cur = nxt;
                nxt = j >= 2 ? un[j - 2] : 0u;
                q[j < NX ? j : 0] = knuth_step<NB>(w, bn, est.digit(w[NB], w[NB - 1]));
#pragma unroll
                for (int i = NB; i > 0; i--) w[i] = w[i - 1];
                w[0] = cur;
            }
            q[0] = knuth_step<NB>(w, bn, est.digit(w[NB], w[NB - 1]));
        } else {
            // narrow windows: two digits per iteration (half the moves are renamings)
#pragma unroll 1
            for (; j >= 1; j -= 2) {
                const u32 n1 = un[j - 1];
                const u32 n2 = j >= 2 ? un[j - 2] : 0u;
                q[j < NX ? j : 0] = knuth_step<NB>(w, bn, est.digit(w[NB], w[NB - 1]));
#pragma unroll
                for (int i = NB; i > 0; i--) w[i] = w[i - 1];
                w[0] = n1;
                q[j - 1] = knuth_step<NB>(w, bn, est.digit(w[NB], w[NB - 1]));
                if (j >= 2) {
#pragma unroll
                    for (int i = NB; i > 0; i--) w[i] = w[i - 1];
                    w[0] = n2;
                }
            }
            if (j == 0) q[0] = knuth_step<NB>(w, bn, est.digit(w[NB], w[NB - 1]));
        }
#pragma unroll
        for (int i = 0; i < NB; i++) rn[i] = w[i];
        return;
    }
    // Static window positions: digit j uses un[j .. j+NB], j <= jmax <= NX - 1.
#pragma unroll(kUnroll ? NX : 1)
    for (int j = NX - 1; j >= 0; j--) {
        if (j > jmax) continue;
        u32 w[NB + 1];
#pragma unroll
        for (int i = 0; i <= NB; i++) w[i] = un[j + i];
        const u32 qd = knuth_step<NB>(w, bn, est.digit(w[NB], w[NB - 1]));
#pragma unroll
        for (int i = 0; i <= NB; i++) un[j + i] = w[i];
        q[j] = qd;
    }
    // the remainder (< bn) sits in un[0..NB)
#pragma unroll
    for (int i = 0; i < NB; i++) rn[i] = un[i];
    }
}

// q = floor(x / b), rem = x mod b.  Requires b != 0.
template <int NX, int NB>
UP_DI void divmod(u32 (&q)[NX], u32 (&rem)[NB], const u32 (&x)[NX], const u32 (&b)[NB]) {
    u32 rn[NB], bn[NB], s;
    divmod_norm(q, rn, bn, s, x, b);
    shr_bits(rem, rn, s);  // undo the normalising shift
}

// Quotients below 2^48 of narrow operands (NX + NB <= 12 limbs, divisor
// wider than one limb, bitlen(x) <= bitlen(b) + 47): q = floor(x / b) from
// one double division, made exact by one multiply-subtract and at most one
// correction; up = (2 * (x - q*b) >= b), the half-up decision.  x and b enter
// as doubles by Horner's rule from the top limb (each of the NX + NB - 2
// fused steps, the reciprocal and the product round once: relative error
// below (NX + NB) * 2^-53), so for q < 2^48 the double quotient is within
// 12/32 of x/b and its floor is q - 1, q or q + 1.
template <int NX, int NB>
UP_DI void div_small_quotient(u32 (&q)[NX], bool& up, const u32 (&x)[NX], const u32 (&b)[NB]) {
    static_assert(NX + NB <= 12, "the error bound needs narrow operands");
    double X = 0.0, D = 0.0;
#pragma unroll
    for (int i = NX - 1; i >= 0; i--) X = __fma_rn(X, 4294967296.0, u32_to_f64(x[i]));
#pragma unroll
    for (int i = NB - 1; i >= 0; i--) D = __fma_rn(D, 4294967296.0, u32_to_f64(b[i]));
    const double Q = __dmul_rn(X, __drcp_rn(D));
    // floor(Q) (0 <= Q < 2^49) in the low mantissa bits of Q + 2^52 rounded down
    const double Y = __dadd_rd(Q, 4503599627370496.0);
    u32 qv[2] = {(u32)__double2loint(Y), (u32)__double2hiint(Y) & 0xfffffu};
    // r = x - qv * b over NB + 2 limbs, two's complement (|r| < 2b)
    u32 t[NB + 2], rr[NB + 2];
    mul(t, b, qv);
    sub(rr, x, t);
    if (rr[NB + 1] >> 31) {  // one too large
        add(rr, rr, b);
        u32 one[1] = {1u};
        sub(qv, qv, one);
    } else if (cmp(rr, b) >= 0) {  // one too small
        sub(rr, rr, b);
        add_small(qv, 1u);
    }
    u32 dbl[NB + 2];
    add(dbl, rr, rr);
    up = cmp(dbl, b) >= 0;
#pragma unroll
    for (int i = 0; i < NX; i++) q[i] = i < 2 ? qv[i < 2 ? i : 0] : 0u;
}

// Bit length of 10^k estimated the way the reference does before choosing
// the 64-bit divide branch (AriesDecimal.hxx:799-804).
__host__ __device__ constexpr u32 ref_shift_bits(u32 shift) {
    return (shift / 3u) * 10u + (shift % 3u == 1u ? 4u : (shift % 3u == 2u ? 7u : 0u));
}

// Decimal divide with the reference's rule (DivOrMod, AriesDecimal.hxx:748-878):
//   sign = sa ^ sb; dividend 0 -> +0; divisor 0 -> dividend unchanged + ERR_DIV0;
//   shift = scale(b) + 4 (compile time: SHIFT);
//   if bitlen(a) + ref_shift_bits(SHIFT) - 1 <= 64 and bitlen(b) <= 64:
//       64-bit arithmetic: q = (a*10^SHIFT mod 2^64) / b, half-up with the
//       doubled remainder taken mod 2^64                         (:581-596)
//   else q = floor(a*10^SHIFT / b), half-up on 2*rem >= b, where a one-limb
//       divisor doubles the remainder mod 2^32                   (:598-626, :862-873)
// p10 holds the NP limbs of 10^SHIFT; P10W is 10^SHIFT mod 2^64.
template <int NR, int NA, int NB, int NP, u32 SHIFT, u64 P10W>
UP_DI u32 div_round(u32 (&r)[NR], u32& sr, const u32 (&a)[NA], u32 sa, const u32 (&b)[NB], u32 sb,
                    const u32 (&p10)[NP]) {
    sr = sa ^ sb;
    if (is_zero(a)) {
        zero(r);
        sr = 0u;
        return 0u;
    }
    if (is_zero(b)) {
        copy_ext(r, a);
        return ERR_DIV0;
    }
    const u32 hdt = bitlen(a);
    const u32 hds = bitlen(b);
    if (hdt + ref_shift_bits(SHIFT) - 1u <= 64u && hds <= 64u) {
        const u64 dvs = ((u64)at(a, 0) | ((u64)at(a, 1) << 32)) * P10W;
        const u64 dvt = (u64)at(b, 0) | ((u64)at(b, 1) << 32);
        u64 q = dvs / dvt;
        const u64 rm = dvs - q * dvt;
        q += ((rm << 1) >= dvt) ? 1u : 0u;
        zero(r);
        r[0] = (u32)q;
        if (NR > 1) r[NR > 1 ? 1 : 0] = (u32)(q >> 32);
        return 0u;
    }
    constexpr int NX = NA + NP;
    u32 x[NX];
    mul(x, a, p10);
    u32 q[NX];
    bool up;
    bool small = false;
    // (taken where 10^SHIFT leaves at least 16 bits of the 48 for a / b, so
    // that a warp's rows rarely split between this path and Algorithm D)
    if constexpr (NX + NB <= 12 && SHIFT <= 9) small = hds > 32u && bitlen(x) <= hds + 47u;
    if constexpr (NB == 1) {
        // one-limb divisor: 2/1 steps; the reference doubles this remainder
        // modulo 2^32 (only this path is compiled: long series inline many
        // such divisions)
        u32 r1[1];
        divmod<NX, 1>(q, r1, x, b);
        up = (u32)(r1[0] * 2u) >= b[0];
    } else if (small) {
        if constexpr (NX + NB <= 12 && SHIFT <= 9) div_small_quotient(q, up, x, b);
    } else if (hds <= 32u) {
        // a one-limb divisor value: 2/1 steps whatever NB is (the same
        // doubling modulo 2^32)
        const u32 b1[1] = {b[0]};
        u32 r1[1];
        divmod<NX, 1>(q, r1, x, b1);
        up = (u32)(r1[0] * 2u) >= b[0];
    } else {
        // 2 * rem >= b  <=>  2 * (rem << s) >= (b << s): decided on the
        // normalised remainder and divisor, so b itself is not kept
        u32 rn[NB], bn[NB], s;
        divmod_norm(q, rn, bn, s, x, b);
        u32 dbl[NB + 1];
        add(dbl, rn, rn);
        up = cmp(dbl, bn) >= 0;
    }
    copy_ext(r, q);
    if (up) add_small(r, 1u);
    return 0u;
}

// MOD with ModCalc rules (AriesDecimal.hxx:953-1012): raw magnitudes (no
// alignment), scale 0, sign XOR, zero dividend -> +0.  A zero divisor is
// undefined in the reference; here it yields 0 with ERR_DIV0.
template <int NR, int NA, int NB>
UP_DI u32 mod(u32 (&r)[NR], u32& sr, const u32 (&a)[NA], u32 sa, const u32 (&b)[NB], u32 sb) {
    sr = sa ^ sb;
    if (is_zero(a)) {
        zero(r);
        sr = 0u;
        return 0u;
    }
    if (is_zero(b)) {
        zero(r);
        return ERR_DIV0;
    }
    u32 q[NA];
    u32 rem[NB];
    divmod(q, rem, a, b);
    copy_ext(r, rem);
    return 0u;
}

// Truncate toward zero by 10^K (RESCALE to a smaller scale).
template <int NR, int NA, int NP>
UP_DI void trunc_div_pow10(u32 (&r)[NR], const u32 (&a)[NA], const u32 (&p10)[NP]) {
    u32 q[NA];
    u32 rem[NP];
    divmod(q, rem, a, p10);
    copy_ext(r, q);
}

// Out-of-line instances of the wide operations.  A module whose expression
// repeats many wide operations (long series, deep trees of 1000-digit values)
// calls one instance per operand shape instead of inlining every use: the
// limb arrays of such widths live in local memory either way, and compile
// time stays proportional to the number of distinct shapes.
template <int N, int NA, int NB>
__device__ __noinline__ void mul_ni(u32 (&r)[N], const u32 (&a)[NA], const u32 (&b)[NB]) {
    mul(r, a, b);
}

template <int NR, int NA, int NB, int NP, u32 SHIFT, u64 P10W>
__device__ __noinline__ u32 div_round_ni(u32 (&r)[NR], u32& sr, const u32 (&a)[NA], u32 sa, const u32 (&b)[NB],
                                         u32 sb, const u32 (&p10)[NP]) {
    return div_round<NR, NA, NB, NP, SHIFT, P10W>(r, sr, a, sa, b, sb, p10);
}

template <int NR, int NA, int NP>
__device__ __noinline__ void trunc_div_pow10_ni(u32 (&r)[NR], const u32 (&a)[NA], const u32 (&p10)[NP]) {
    trunc_div_pow10(r, a, p10);
}

// Comparison with the reference rules: different signs decide by sign
// alone (-0 < +0), else aligned magnitudes reversed for negatives.
// op: 0 <, 1 <=, 2 >, 3 >=, 4 ==, 5 !=
template <int NA, int NB>
UP_DI u32 compare(int op, const u32 (&a)[NA], u32 sa, const u32 (&b)[NB], u32 sb) {
    bool lt, gt, eq;
    if (sa != sb) {
        lt = sa == 1u;
        gt = sa == 0u;
        eq = false;
    } else {
        const int c = cmp(a, b);
        eq = c == 0;
        lt = sa == 0u ? c < 0 : c > 0;
        gt = sa == 0u ? c > 0 : c < 0;
    }
    switch (op) {
        case 0: return lt;
        case 1: return !gt;
        case 2: return gt;
        case 3: return !lt;
        case 4: return eq;
        default: return !eq;
    }
}

// ----------------------------------------------------- compact layout
// Load a B-byte compact value from 4-byte-readable memory (shared-memory
// tiles are padded so the word past the value is readable).
template <int B, int N>
UP_DI void ld_compact_words(const u8* p, u32 (&m)[N], u32& sign) {
    static_assert(N * 4 >= B, "limbs too few for the compact width");
    const unsigned long long addr = (unsigned long long)p;
    const u32 off = (u32)(addr & 3u);
    const u32* w = (const u32*)(p - off);
    const u32 sh = off * 8u;
    constexpr int W = (B + 3) / 4;
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (i < W) {
            const u32 lo = w[i];
            const u32 hi = (off != 0u) ? w[i + 1] : 0u;
            m[i] = __funnelshift_r(lo, hi, sh);
        } else {
            m[i] = 0u;
        }
    }
    constexpr int TOPL = (B - 1) / 4;
    constexpr int TOPB = ((B - 1) % 4) * 8 + 7;
    sign = (m[TOPL] >> TOPB) & 1u;
    m[TOPL] &= (TOPB == 31) ? 0x7fffffffu : ((1u << TOPB) - 1u);
}

// Byte-granular load (any alignment, never reads past the value).
template <int B, int N>
UP_DI void ld_compact_bytes(const u8* p, u32 (&m)[N], u32& sign) {
    zero(m);
#pragma unroll
    for (int i = 0; i < B; i++) m[i / 4] |= (u32)p[i] << (8 * (i % 4));
    constexpr int TOPL = (B - 1) / 4;
    constexpr int TOPB = ((B - 1) % 4) * 8 + 7;
    sign = (m[TOPL] >> TOPB) & 1u;
    m[TOPL] &= (TOPB == 31) ? 0x7fffffffu : ((1u << TOPB) - 1u);
}

// Overflow test: any magnitude bit at or above 8*B-1 would be lost or would
// collide with the sign bit.
template <int B, int N>
UP_DI u32 compact_overflow(const u32 (&m)[N]) {
    constexpr int BIT = 8 * B - 1;
    u32 o = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (32 * i + 32 <= BIT) continue;
        const u32 mask = (32 * i >= BIT) ? 0xffffffffu : ~((1u << (BIT - 32 * i)) - 1u);
        o |= m[i] & mask;
    }
    return o ? ERR_OVERFLOW : 0u;
}

// Store with ToCompactDecimal + SET_SIGN_BIT: low B bytes, then the sign
// OR-ed into bit 7 of the last byte.  Byte stores (any alignment).
template <int B, int N>
UP_DI u32 st_compact_bytes(u8* p, const u32 (&m)[N], u32 sign) {
#pragma unroll
    for (int i = 0; i < B; i++) {
        u32 byte = (at(m, i / 4) >> (8 * (i % 4))) & 0xffu;
        if (i == B - 1) byte |= sign << 7;
        p[i] = (u8)byte;
    }
    return compact_overflow<B>(m);
}

// Same, 4-byte aligned p and B % 4 == 0: word stores.
template <int B, int N>
UP_DI u32 st_compact_words(u8* p, const u32 (&m)[N], u32 sign) {
    static_assert(B % 4 == 0, "word store needs B % 4 == 0");
    u32* w = (u32*)p;
#pragma unroll
    for (int i = 0; i < B / 4; i++) {
        u32 v = at(m, i);
        if (i == B / 4 - 1) v |= sign << 31;
        w[i] = v;
    }
    return compact_overflow<B>(m);
}

#ifndef UP_HOST_TEST  // the host build of the arithmetic (CPU tests) stops here
// ------------------------------------------------ cooperative values
// T threads (T a power of two dividing 32; a group is T consecutive lanes of
// one warp) hold one value: the thread of rank g holds limbs [g*K, g*K + K).
// Carries and borrows between threads move by warp shuffles and ballots.
// Every shuffle and ballot below runs on all 32 lanes with the same control
// flow (callers keep whole warps converged: a group without a row works on
// zeros and skips its stores).
constexpr u32 kFull = 0xffffffffu;

template <int T>
UP_DI int tpi_rank() { return (int)(threadIdx.x & (T - 1)); }

template <int T>
UP_DI u32 tpi_ballot(bool p) {
    const u32 b = __ballot_sync(kFull, p);
    if constexpr (T == 32) return b;
    else return (b >> ((threadIdx.x & 31u) & ~(u32)(T - 1))) & ((1u << T) - 1u);
}

// Carry into each thread from per-thread generate (a carry leaves the
// thread regardless of its input) and propagate (an incoming carry passes
// through) flags: the carries of the binary sum (G|P) + G.
template <int T>
UP_DI u32 tpi_carry_in(bool gen, bool prop) {
    const u32 G = tpi_ballot<T>(gen);
    const u32 A = G | tpi_ballot<T>(prop);
    const u32 cin = (A + G) ^ A ^ G;
    return (cin >> tpi_rank<T>()) & 1u;
}

// x += cin (0 or 1) at this thread's lowest limb
template <int K>
UP_DI void tpi_inc_local(u32 (&x)[K], u32 cin) {
    u32 c = cin;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const u32 t = x[i] + c;
        c = (c != 0u && t == 0u) ? 1u : 0u;
        x[i] = t;
    }
}

// r = a + b (magnitudes; the carry out of the top thread is dropped)
template <int T, int K>
UP_DI void tpi_add(u32 (&r)[K], const u32 (&a)[K], const u32 (&b)[K]) {
    u64 c = 0;
    u32 all = kFull;
#pragma unroll
    for (int i = 0; i < K; i++) {
        c += (u64)a[i] + b[i];
        r[i] = (u32)c;
        c >>= 32;
        all &= r[i];
    }
    tpi_inc_local(r, tpi_carry_in<T>(c != 0, all == kFull));
}

// r = a - b for magnitudes a >= b
template <int T, int K>
UP_DI void tpi_sub(u32 (&r)[K], const u32 (&a)[K], const u32 (&b)[K]) {
    u64 br = 0;
    u32 any = 0;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const u64 d = (u64)a[i] - b[i] - br;
        r[i] = (u32)d;
        br = d >> 63;
        any |= r[i];
    }
    u32 bin = tpi_carry_in<T>(br != 0, any == 0u);
#pragma unroll
    for (int i = 0; i < K; i++) {
        const u32 t = r[i] - bin;
        bin = (bin != 0u && r[i] == 0u) ? 1u : 0u;
        r[i] = t;
    }
}

// Magnitude comparison: -1, 0 or 1 on every thread of the group.
template <int T, int K>
UP_DI int tpi_cmp(const u32 (&a)[K], const u32 (&b)[K]) {
    int lc = 0;
#pragma unroll
    for (int i = K - 1; i >= 0; i--)
        if (lc == 0 && a[i] != b[i]) lc = a[i] > b[i] ? 1 : -1;
    const u32 m = tpi_ballot<T>(lc != 0);
    const int top = m ? 31 - __clz((int)m) : 0;
    const int v = __shfl_sync(kFull, lc, top, T);
    return m ? v : 0;
}

template <int T, int K>
UP_DI bool tpi_is_zero(const u32 (&a)[K]) {
    u32 o = 0;
#pragma unroll
    for (int i = 0; i < K; i++) o |= a[i];
    return tpi_ballot<T>(o != 0u) == 0u;
}

// Signed add with the sign rules of add_signed (equal magnitudes of opposite
// sign give +0).
template <int T, int K>
UP_DI void tpi_add_signed(u32 (&r)[K], u32& sr, const u32 (&a)[K], u32 sa, const u32 (&b)[K], u32 sb) {
    const int c = tpi_cmp<T, K>(a, b);
    u32 x[K], y[K], sum[K], dif[K];
#pragma unroll
    for (int i = 0; i < K; i++) {
        x[i] = c >= 0 ? a[i] : b[i];
        y[i] = c >= 0 ? b[i] : a[i];
    }
    tpi_add<T, K>(sum, a, b);
    tpi_sub<T, K>(dif, x, y);
    const bool same = sa == sb;
#pragma unroll
    for (int i = 0; i < K; i++) r[i] = same ? sum[i] : dif[i];
    sr = same ? sa : (c == 0 ? 0u : (c > 0 ? sa : sb));
}

// Signed comparison with the rules of compare (-0 < +0).
template <int T, int K>
UP_DI u32 tpi_compare(int op, const u32 (&a)[K], u32 sa, const u32 (&b)[K], u32 sb) {
    const int c = tpi_cmp<T, K>(a, b);
    bool lt, gt, eq;
    if (sa != sb) {
        lt = sa == 1u;
        gt = sa == 0u;
        eq = false;
    } else {
        eq = c == 0;
        lt = sa == 0u ? c < 0 : c > 0;
        gt = sa == 0u ? c > 0 : c < 0;
    }
    switch (op) {
        case 0: return lt;
        case 1: return !gt;
        case 2: return gt;
        case 3: return !lt;
        case 4: return eq;
        default: return !eq;
    }
}

// Multiplication streams one operand limb by limb through a window that
// holds the running partial product of the other operand a (LA nonzero
// limbs).  The window needs LA+1 limbs, so it uses KA limbs per thread, the
// smallest divisor of K with T*KA >= LA+1: no thread multiplies limbs that
// are known to be zero.
template <int T, int K, int LA>
__host__ __device__ constexpr int tpi_window_limbs() {
    for (int d = 1; d <= K; d++)
        if (K % d == 0 && T * d >= LA + 1) return d;
    return K;
}

// a in the K-limb layout -> the KA-limb layout (KA divides K)
template <int T, int K, int KA>
UP_DI void tpi_pack(u32 (&aw)[KA], const u32 (&a)[K]) {
    if constexpr (KA == K) {
#pragma unroll
        for (int i = 0; i < K; i++) aw[i] = a[i];
    } else {
        const int g = tpi_rank<T>();
        const int sel = ((g * KA) % K) / KA;
#pragma unroll
        for (int i = 0; i < KA; i++) {
            const int src = (g * KA + i) / K;
            u32 v = 0u;
#pragma unroll
            for (int m = 0; m < K / KA; m++) {
                const u32 t = __shfl_sync(kFull, a[m * KA + i], src, T);
                if (sel == m) v = t;
            }
            aw[i] = v;
        }
    }
}

// One window step: acc += a * bj (pending carry bits e from the thread
// below enter at limb 0); returns product limb j (final, from rank 0) and
// moves the window down one limb.
template <int T, int KA>
UP_DI u32 tpi_window_step(u32 (&acc)[KA], u32& e, const u32 (&aw)[KA], u32 bj) {
    const int g = tpi_rank<T>();
    u32 ein = __shfl_up_sync(kFull, e, 1, T);
    if (g == 0) ein = 0u;
    u64 c = ein;
#pragma unroll
    for (int i = 0; i < KA; i++) {
        const u64 t = (u64)aw[i] * bj + acc[i] + c;
        acc[i] = (u32)t;
        c = t >> 32;
    }
    const u32 out = __shfl_sync(kFull, acc[0], 0, T);
    u32 nx = __shfl_down_sync(kFull, acc[0], 1, T);
    if (g == T - 1) nx = 0u;
#pragma unroll
    for (int i = 0; i < KA - 1; i++) acc[i] = acc[i + 1];
    const u64 top = (u64)nx + c;
    acc[KA - 1] = (u32)top;
    e = (u32)(top >> 32);
    return out;
}

// After LB steps: resolve the pending carry bits and move the window (product
// limbs LB.., KA layout) to positions >= LB of r (K layout).
template <int T, int K, int KA, int LB>
UP_DI void tpi_window_out(u32 (&r)[K], u32 (&acc)[KA], u32 e) {
    const int g = tpi_rank<T>();
    u32 ein = __shfl_up_sync(kFull, e, 1, T);
    if (g == 0) ein = 0u;
    u32 c = ein, all = kFull;
#pragma unroll
    for (int i = 0; i < KA; i++) {
        const u32 t = acc[i] + c;
        c = (c != 0u && t == 0u) ? 1u : 0u;
        acc[i] = t;
        all &= t;
    }
    tpi_inc_local(acc, tpi_carry_in<T>(c != 0u, all == kFull));
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int lidx = (((i - LB) % KA) + KA) % KA;
        const int q = g * K + i - LB;
        const int src = q >= 0 ? q / KA : 0;
        const u32 v = __shfl_sync(kFull, acc[lidx], src < T ? src : 0, T);
        if (q >= 0 && src < T) r[i] = v;
    }
}

// r = a * b (low T*K limbs); a has at most LA nonzero limbs, b at most LB.
template <int T, int K, int LA, int LB>
UP_DI void tpi_mul(u32 (&r)[K], const u32 (&a)[K], const u32 (&b)[K]) {
    constexpr int KA = tpi_window_limbs<T, K, LA>();
    const int g = tpi_rank<T>();
    u32 aw[KA], acc[KA];
    tpi_pack<T, K, KA>(aw, a);
#pragma unroll
    for (int i = 0; i < KA; i++) acc[i] = 0u;
#pragma unroll
    for (int i = 0; i < K; i++) r[i] = 0u;
    u32 e = 0u;
#pragma unroll
    for (int j = 0; j < LB; j++) {
        const u32 bj = __shfl_sync(kFull, b[j % K], j / K, T);
        const u32 out = tpi_window_step<T, KA>(acc, e, aw, bj);
        if (g == j / K) r[j % K] = out;
    }
    tpi_window_out<T, K, KA, LB>(r, acc, e);
}

// r = a * p for a static multiplier p of NP limbs (alignment by 10^d).
template <int T, int K, int LA, int NP>
UP_DI void tpi_mul_const(u32 (&r)[K], const u32 (&a)[K], const u32 (&p)[NP]) {
    constexpr int KA = tpi_window_limbs<T, K, LA>();
    const int g = tpi_rank<T>();
    u32 aw[KA], acc[KA];
    tpi_pack<T, K, KA>(aw, a);
#pragma unroll
    for (int i = 0; i < KA; i++) acc[i] = 0u;
#pragma unroll
    for (int i = 0; i < K; i++) r[i] = 0u;
    u32 e = 0u;
#pragma unroll
    for (int j = 0; j < NP; j++) {
        const u32 out = tpi_window_step<T, KA>(acc, e, aw, p[j]);
        if (g == j / K) r[j % K] = out;
    }
    tpi_window_out<T, K, KA, NP>(r, acc, e);
}

// Limb `pos` (the same position on every thread of the group; 0 when out of
// range) broadcast to the whole group.
template <int T, int K>
UP_DI u32 tpi_limb(const u32 (&v)[K], int pos) {
    const bool in = pos >= 0 && pos < T * K;
    const int src = in ? pos / K : 0;
    const int li = in ? pos % K : 0;
    u32 mine = 0u;
#pragma unroll
    for (int l = 0; l < K; l++)
        if (l == li) mine = v[l];
    const u32 r = __shfl_sync(kFull, mine, src, T);
    return in ? r : 0u;
}

// Index of the highest nonzero limb (-1 for zero), on every thread.
template <int T, int K>
UP_DI int tpi_top_limb(const u32 (&v)[K]) {
    int li = -1;
#pragma unroll
    for (int i = 0; i < K; i++)
        if (v[i] != 0u) li = i;
    const u32 m = tpi_ballot<T>(li >= 0);
    const int h = m ? 31 - __clz((int)m) : 0;
    const int top = __shfl_sync(kFull, tpi_rank<T>() * K + li, h, T);
    return m ? top : -1;
}

template <int T, int K>
UP_DI u32 tpi_bitlen(const u32 (&v)[K]) {
    const int t = tpi_top_limb<T, K>(v);
    const u32 w = tpi_limb<T, K>(v, t);
    return t < 0 ? 0u : (u32)(32 * t) + (32u - (u32)__clz((int)w));
}

// r = v << s bits (0 <= s < 32, the same on every thread; top bits dropped)
template <int T, int K>
UP_DI void tpi_shl_bits(u32 (&r)[K], const u32 (&v)[K], u32 s) {
    u32 below = __shfl_up_sync(kFull, v[K - 1], 1, T);
    if (tpi_rank<T>() == 0) below = 0u;
#pragma unroll
    for (int i = K - 1; i >= 0; i--) {
        const u32 lo = i > 0 ? v[i - 1] : below;
        r[i] = s ? ((v[i] << s) | (lo >> (32u - s))) : v[i];
    }
}

// r = v >> s bits (0 <= s < 32)
template <int T, int K>
UP_DI void tpi_shr_bits(u32 (&r)[K], const u32 (&v)[K], u32 s) {
    u32 above = __shfl_down_sync(kFull, v[0], 1, T);
    if (tpi_rank<T>() == T - 1) above = 0u;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const u32 hi = i < K - 1 ? v[i + 1] : above;
        r[i] = s ? ((v[i] >> s) | (hi << (32u - s))) : v[i];
    }
}

// Long division x = q*b + rem (Knuth's algorithm D) on values spread over the
// group; b != 0 and x has a zero top limb (room for the normalising shift).
// The divisor stays in place, normalised so its top bit is set; a window of
// n+1 remainder limbs aligned with it moves down the dividend one limb per
// quotient limb.  Each step estimates the quotient limb from three window
// limbs and two divisor limbs, subtracts quotient x divisor (carry words move
// up one thread, bit borrows resolve by ballot lookahead), and adds the
// divisor back when the estimate was one too large.  Groups of a warp may
// need different step counts: the warp runs the largest, and groups that
// are done keep their state.
template <int T, int K>
UP_DI void tpi_divmod(u32 (&q)[K], u32 (&rem)[K], const u32 (&x)[K], const u32 (&b)[K]) {
    const int g = tpi_rank<T>();
    const int n = tpi_top_limb<T, K>(b) + 1;
    const u32 sh = (u32)__clz((int)tpi_limb<T, K>(b, n - 1));
    u32 v[K], u[K], R[K];
    tpi_shl_bits<T, K>(v, b, sh);
    tpi_shl_bits<T, K>(u, x, sh);
    const int m = tpi_top_limb<T, K>(u) + 1;
    const int steps = m >= n ? m - n + 1 : 0;
    const int j0 = m - n;
#pragma unroll
    for (int i = 0; i < K; i++) q[i] = 0u;
    // window R = u[j0 .. j0+n]; with no steps the remainder is u itself
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int li = ((i + j0) % K + K) % K;
        u32 mine = 0u;
#pragma unroll
        for (int l = 0; l < K; l++)
            if (l == li) mine = u[l];
        const int pos = g * K + i + j0;
        const int src = pos >= 0 && pos < T * K ? pos / K : 0;
        const u32 w = __shfl_sync(kFull, mine, src, T);
        R[i] = steps == 0 ? u[i] : ((g * K + i <= n && pos >= 0 && pos < T * K) ? w : 0u);
    }
    const u32 vt1 = tpi_limb<T, K>(v, n - 1);
    const u32 vt2 = tpi_limb<T, K>(v, n - 2);
    const u32 rcp = reciprocal_u32(vt1);
    const int S = __reduce_max_sync(kFull, (u32)steps);
    for (int t = 0; t < S; t++) {
        const bool active = t < steps;
        const int j = j0 - t;
        const u32 r2 = tpi_limb<T, K>(R, n);
        const u32 r1 = tpi_limb<T, K>(R, n - 1);
        const u32 r0 = tpi_limb<T, K>(R, n - 2);
        // quotient limb estimate, at most 2^32-1, refined against vt2
        u32 qh, rh;
        bool rh_big = false;
        if (r2 >= vt1) {
            qh = 0xffffffffu;
            const u64 rr = (((u64)r2 << 32) | r1) - (u64)qh * vt1;
            rh_big = (rr >> 32) != 0;
            rh = (u32)rr;
        } else {
            qh = div2by1(r2, r1, vt1, rcp, rh);
        }
#pragma unroll 1
        for (int c = 0; c < 2; c++) {
            if (rh_big) break;
            if ((u64)qh * vt2 <= (((u64)rh << 32) | r0)) break;
            qh--;
            const u64 nr = (u64)rh + vt1;
            rh_big = (nr >> 32) != 0;
            rh = (u32)nr;
        }
        if (!active) qh = 0u;
        // R -= qh * v: local chains, then carry words up one thread, then bit borrows
        u32 loc[K];
        u64 c = 0;
        u32 br = 0u;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const u64 p = (u64)qh * v[i] + c;
            c = p >> 32;
            const u64 d = (u64)R[i] - (u32)p - br;
            loc[i] = (u32)d;
            br = (u32)(d >> 63);
        }
        const u64 owe = c + br;  // <= 2^32, owed to the next thread's limb 0
        u32 wlo = __shfl_up_sync(kFull, (u32)owe, 1, T);
        u32 whi = __shfl_up_sync(kFull, (u32)(owe >> 32), 1, T);
        if (g == 0) wlo = whi = 0u;
        u64 win = ((u64)whi << 32) | wlo;
        u32 any = 0u;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const u64 d = (u64)loc[i] - win;
            loc[i] = (u32)d;
            win = (d >> 63) ? 1u : 0u;
            any |= loc[i];
        }
        // bit borrows across threads; a borrow out of the top thread means the
        // estimate was one too large
        const u32 G = tpi_ballot<T>(win != 0u);
        const u32 A = G | tpi_ballot<T>(any == 0u);
        const u64 sum = (u64)A + G;
        u32 bin = (u32)(((sum ^ A ^ G) >> g) & 1u);
        const bool negative = ((sum >> T) & 1u) != 0u;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const u32 t2 = loc[i] - bin;
            bin = (bin != 0u && loc[i] == 0u) ? 1u : 0u;
            loc[i] = t2;
        }
        // add the divisor back when negative
        {
            u64 cc = 0;
            u32 all = kFull;
#pragma unroll
            for (int i = 0; i < K; i++) {
                cc += (u64)loc[i] + (negative ? v[i] : 0u);
                loc[i] = (u32)cc;
                cc >>= 32;
                all &= loc[i];
            }
            tpi_inc_local(loc, tpi_carry_in<T>(cc != 0, all == kFull));
        }
        if (negative) qh--;
        if (active) {
#pragma unroll
            for (int i = 0; i < K; i++) R[i] = loc[i];
            if (j >= 0 && g == j / K) {
#pragma unroll
                for (int l = 0; l < K; l++)
                    if (l == j % K) q[l] = qh;
            }
        }
        // next window: up one limb, u[j-1] enters at the bottom
        const u32 nxt = tpi_limb<T, K>(u, j - 1);
        u32 up1 = __shfl_up_sync(kFull, R[K - 1], 1, T);
        if (active && t + 1 < steps) {
#pragma unroll
            for (int i = K - 1; i > 0; i--) R[i] = R[i - 1];
            R[0] = g == 0 ? nxt : up1;
        }
    }
    tpi_shr_bits<T, K>(rem, R, sh);
}

// Decimal divide with the rule of div_round (the reference's DivOrMod,
// AriesDecimal.hxx:748-878) on values spread over the group; LA = limbs of a,
// p10 = 10^SHIFT (NP limbs), P10W = 10^SHIFT mod 2^64.
template <int T, int K, int LA, int NP, u32 SHIFT, u64 P10W>
UP_DI u32 tpi_div_round(u32 (&r)[K], u32& sr, const u32 (&a)[K], u32 sa, const u32 (&b)[K], u32 sb,
                        const u32 (&p10)[NP]) {
    const int g = tpi_rank<T>();
    sr = sa ^ sb;
    const bool za = tpi_is_zero<T, K>(a);
    const bool zb = tpi_is_zero<T, K>(b);
    const u32 hdt = tpi_bitlen<T, K>(a);
    const u32 hds = tpi_bitlen<T, K>(b);
    // general path (a zero divisor is replaced by 1 to keep it defined)
    u32 x[K], bb[K], qv[K], rv[K];
    tpi_mul_const<T, K, LA, NP>(x, a, p10);
#pragma unroll
    for (int i = 0; i < K; i++) bb[i] = zb ? ((g == 0 && i == 0) ? 1u : 0u) : b[i];
    tpi_divmod<T, K>(qv, rv, x, bb);
    u32 dbl[K];
    tpi_add<T, K>(dbl, rv, rv);
    const bool up_wide = tpi_cmp<T, K>(dbl, bb) >= 0;
    const u32 rem0 = tpi_limb<T, K>(rv, 0), b0 = tpi_limb<T, K>(bb, 0);
    const bool up = hds <= 32u ? (u32)(rem0 * 2u) >= b0 : up_wide;
    {
        u32 c = (g == 0 && up) ? 1u : 0u, all = kFull;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const u32 t2 = qv[i] + c;
            c = (c != 0u && t2 == 0u) ? 1u : 0u;
            qv[i] = t2;
            all &= t2;
        }
        tpi_inc_local(qv, tpi_carry_in<T>(c != 0u, all == kFull));
    }
    // the 64-bit branch
    const u64 a64 = (u64)tpi_limb<T, K>(a, 0) | ((u64)tpi_limb<T, K>(a, 1) << 32);
    const u64 b64 = (u64)tpi_limb<T, K>(b, 0) | ((u64)tpi_limb<T, K>(b, 1) << 32);
    const bool br64 = hdt + ref_shift_bits(SHIFT) - 1u <= 64u && hds <= 64u;
    u64 q64 = 0;
    if (br64 && !za && !zb) {
        const u64 dvs = a64 * P10W;
        q64 = dvs / b64;
        const u64 rm = dvs - q64 * b64;
        q64 += ((rm << 1) >= b64) ? 1u : 0u;
    }
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int pos = g * K + i;
        const u32 w64 = pos == 0 ? (u32)q64 : (pos == 1 ? (u32)(q64 >> 32) : 0u);
        r[i] = za ? 0u : (zb ? a[i] : (br64 ? w64 : qv[i]));
    }
    if (za) sr = 0u;
    return (!za && zb) ? ERR_DIV0 : 0u;
}

// MOD with the rule of mod (ModCalc): raw magnitudes, scale 0, sign XOR, zero
// dividend -> +0, zero divisor -> 0 with ERR_DIV0.
template <int T, int K>
UP_DI u32 tpi_mod(u32 (&r)[K], u32& sr, const u32 (&a)[K], u32 sa, const u32 (&b)[K], u32 sb) {
    const int g = tpi_rank<T>();
    sr = sa ^ sb;
    const bool za = tpi_is_zero<T, K>(a);
    const bool zb = tpi_is_zero<T, K>(b);
    u32 bb[K], qv[K], rv[K];
#pragma unroll
    for (int i = 0; i < K; i++) bb[i] = zb ? ((g == 0 && i == 0) ? 1u : 0u) : b[i];
    tpi_divmod<T, K>(qv, rv, a, bb);
#pragma unroll
    for (int i = 0; i < K; i++) r[i] = (za || zb) ? 0u : rv[i];
    if (za) sr = 0u;
    return (!za && zb) ? ERR_DIV0 : 0u;
}

// A distributed copy of a constant held in device memory (nl limbs).
template <int T, int K>
UP_DI void tpi_const(u32 (&x)[K], const u32* __restrict__ c, int nl) {
    const int g = tpi_rank<T>();
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int l = g * K + i;
        x[i] = l < nl ? c[l] : 0u;
    }
}

// Truncation toward zero by 10^d (a RESCALE to a smaller scale); c = the limbs
// of 10^d in device memory.
template <int T, int K>
UP_DI void tpi_trunc_pow10(u32 (&r)[K], const u32 (&a)[K], const u32* __restrict__ c, int nl) {
    u32 p[K], rv[K];
    tpi_const<T, K>(p, c, nl);
    tpi_divmod<T, K>(r, rv, a, p);
}

// Out-of-line instances of the cooperative wide operations, for expressions
// that repeat them many times (one instance per operand shape).
template <int T, int K, int LA, int LB>
__device__ __noinline__ void tpi_mul_ni(u32 (&r)[K], const u32 (&a)[K], const u32 (&b)[K]) {
    tpi_mul<T, K, LA, LB>(r, a, b);
}
template <int T, int K, int LA, int NP, u32 SHIFT, u64 P10W>
__device__ __noinline__ u32 tpi_div_round_ni(u32 (&r)[K], u32& sr, const u32 (&a)[K], u32 sa, const u32 (&b)[K],
                                             u32 sb, const u32 (&p10)[NP]) {
    return tpi_div_round<T, K, LA, NP, SHIFT, P10W>(r, sr, a, sa, b, sb, p10);
}
template <int T, int K>
__device__ __noinline__ void tpi_trunc_pow10_ni(u32 (&r)[K], const u32 (&a)[K], const u32* __restrict__ c, int nl) {
    tpi_trunc_pow10<T, K>(r, a, c, nl);
}

// Compact value of B bytes -> this thread's K limbs and the sign.
template <int T, int K, int B>
UP_DI void tpi_ld(const u8* __restrict__ p, u32 (&x)[K], u32& sign) {
    const int g = tpi_rank<T>();
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int o = 4 * (g * K + i);
        u32 w = 0u;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (o + k < B) w |= (u32)p[o + k] << (8 * k);
        x[i] = w;
    }
    sign = (u32)(p[B - 1] >> 7);
    constexpr int TOPL = (B - 1) / 4;
    constexpr u32 CLR = ~(0x80u << (8 * ((B - 1) % 4)));
    if (g == TOPL / K) x[TOPL % K] &= CLR;
}

// tpi_ld from 4-byte-readable memory (a staged shared-memory tile, padded
// past its last value): one funnel shift of two aligned words per limb
// instead of four byte loads; the bytes past the value are masked off.
// Measured on B200: p=600 a*b+c at 16 threads per value 2.18 -> 1.97 ms.
template <int T, int K, int B>
UP_DI void tpi_ld_words(const u8* __restrict__ p, u32 (&x)[K], u32& sign) {
    const int g = tpi_rank<T>();
    const u32 off = (u32)((unsigned long long)p & 3u);
    const u32* w = (const u32*)(p - off);
    const u32 sh = off * 8u;
    constexpr int W = (B + 3) / 4;  // limbs holding bytes of the value
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int L = g * K + i;
        x[i] = L < W ? __funnelshift_r(w[L], w[L + 1], sh) : 0u;
    }
    sign = (u32)(p[B - 1] >> 7);
    constexpr int TOPL = (B - 1) / 4;
    constexpr int TOPB = ((B - 1) % 4) * 8 + 7;  // the sign bit; the bits above it belong to the next value
    if (g == TOPL / K) x[TOPL % K] &= (TOPB == 31) ? 0x7fffffffu : ((1u << TOPB) - 1u);
}

// This thread's limbs -> bytes [4gK, 4gK+4K) of a B-byte compact value with
// the sign in bit 7 of byte B-1; ERR_OVERFLOW when a magnitude bit at or
// above 8*B-1 is set (the same rule as st_compact_bytes).  `store` false
// computes the error word only.
template <int T, int K, int B>
UP_DI u32 tpi_st(u8* __restrict__ p, const u32 (&x)[K], u32 sign, bool store) {
    const int g = tpi_rank<T>();
    bool over = false;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int o = 4 * (g * K + i);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            u32 byte = (x[i] >> (8 * k)) & 0xffu;
            if (o + k < B) {
                if (o + k == B - 1) {
                    over |= (byte & 0x80u) != 0u;
                    byte |= sign << 7;
                }
                if (store) p[o + k] = (u8)byte;
            } else {
                over |= byte != 0u;
            }
        }
    }
    // a declared width beyond the group's limbs: zero bytes, then the sign
    if constexpr (B > 4 * T * K) {
        if (store)
            for (int o = 4 * T * K + g; o < B; o += T) p[o] = (u8)(o == B - 1 ? sign << 7 : 0u);
    }
    return tpi_ballot<T>(over) ? ERR_OVERFLOW : 0u;
}

#endif  // UP_HOST_TEST
// ------------------------------------------------------ column access
// Per-column kernel argument: the AriesColumnDataIterator shape
// (AriesColumnDataIterator.hxx:8-41).
typedef ::UpKCol KCol;  // up_kargs.h

// Row -> value pointer for the block/indirection path
// (AriesColumnDataIterator::operator[], AriesColumnDataIterator.cu:60-115).
// Returns nullptr for a NULL index.
UP_DI const u8* col_ptr(const KCol& c, i64 row) {
    i64 r = row;
    if (c.indices) {
        const int j = c.indices[row];
        if (j < 0) return nullptr;
        r = j;
    }
    if (c.n_blocks == 0) return c.data + r * (i64)c.value_bytes;
    int lo = 0, hi = c.n_blocks;  // upper-bound search over prefix[0..n_blocks]
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (c.prefix[mid] <= r) lo = mid + 1;
        else hi = mid;
    }
    const int blk = lo - 1;
    return c.blocks[blk] + (r - c.prefix[blk]) * (i64)c.value_bytes;
}

// ------------------------------------------------- tile staging helpers
// Cooperative copy of n bytes global -> shared.  16-byte vectors when both
// ends allow it, bytes otherwise.
UP_DI void tile_copy_in(u8* __restrict__ dst, const u8* __restrict__ src, int n, bool vec_ok) {
    if (vec_ok && (n & 15) == 0) {
        const uint4* s = (const uint4*)src;
        uint4* d = (uint4*)dst;
        for (int i = threadIdx.x; i < (n >> 4); i += blockDim.x) d[i] = s[i];
    } else {
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    }
}

UP_DI void tile_copy_out(u8* __restrict__ dst, const u8* __restrict__ src, int n, bool vec_ok) {
    if (vec_ok && (n & 15) == 0) {
        const uint4* s = (const uint4*)src;
        uint4* d = (uint4*)dst;
        for (int i = threadIdx.x; i < (n >> 4); i += blockDim.x) d[i] = s[i];
    } else {
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    }
}

// ------------------------------------------- exact group accumulators
// Two's complement accumulation of a sign-magnitude value into NACC limbs in
// memory with 32-bit atomics, carries propagated limb by limb.  Exact as long
// as the true sum fits NACC limbs signed (the host sizes NACC for that).
template <int NACC>
UP_DI void atomic_add_twos(u32* acc, const u32 (&t)[NACC]) {
    u32 carry = 0;
#pragma unroll
    for (int i = 0; i < NACC; i++) {
        const u32 v = t[i];
        u32 add = v + carry;
        u32 c1 = (add < v) ? 1u : 0u;  // v + carry wrapped
        if (add != 0u) {
            const u32 old = atomicAdd(acc + i, add);
            c1 |= (old + add < old) ? 1u : 0u;
        }
        carry = c1;
    }
}

// True when a two's complement value of N limbs equals the sign extension of
// its low 64 bits.
template <int N>
UP_DI bool fits_twos64(const u32 (&t)[N]) {
    if constexpr (N <= 2) {
        return true;
    } else {
        const u32 ext = (t[1] >> 31) ? 0xffffffffu : 0u;
        bool f = true;
#pragma unroll
        for (int i = 2; i < N; i++) f &= t[i] == ext;
        return f;
    }
}

// 128-bit two's complement accumulator r (4 limbs) += the sign-extended low
// 64 bits of t.
template <int N>
UP_DI void add_twos64(u32 (&r)[4], const u32 (&t)[N]) {
    const u64 lo = (u64)t[0] | (N > 1 ? ((u64)t[N > 1 ? 1 : 0] << 32) : 0ull);
    const u64 ext = (N > 1 ? (t[N > 1 ? 1 : 0] >> 31) : (t[0] >> 31)) ? ~0ull : 0ull;
    const u64 a0 = (u64)r[0] | ((u64)r[1] << 32);
    const u64 a1 = (u64)r[2] | ((u64)r[3] << 32);
    const u64 s0 = a0 + lo;
    const u64 s1 = a1 + ext + (s0 < a0 ? 1ull : 0ull);
    r[0] = (u32)s0;
    r[1] = (u32)(s0 >> 32);
    r[2] = (u32)s1;
    r[3] = (u32)(s1 >> 32);
}

// Two's complement image over N limbs of a sign-magnitude value.
template <int N, int M>
UP_DI void to_twos(u32 (&t)[N], const u32 (&m)[M], u32 sign) {
    copy_ext(t, m);
    if (sign) negate(t);
}

// r += t modulo 2^(32N) (two's complement accumulate in registers).
template <int N>
UP_DI void add_twos(u32 (&r)[N], const u32 (&t)[N]) {
    u64 c = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        c += (u64)r[i] + t[i];
        r[i] = (u32)c;
        c >>= 32;
    }
}

template <int NACC, int N>
UP_DI void atomic_acc_add(u32* acc, const u32 (&m)[N], u32 sign) {
    u32 t[NACC];
    to_twos(t, m, sign);
    atomic_add_twos(acc, t);
}

// The reference's nullable_type<Decimal> image of a SUM/AVG result
// (decimal.hxx:130-140 plus the leading flag; kernel_segreduce.hxx:609-612):
// [0] flag, [1] sign, [2] prec, [3] frac, [4] error, [5..133) v[32] LE.
// prec and error are left 0 (the reference leaves them unwritten).
template <int N>
UP_DI void agg_image(u8* img, u32 flag, u32 sign, u32 frac, const u32 (&m)[N]) {
    img[0] = (u8)flag;
    img[1] = (u8)sign;
    img[2] = 0;
    img[3] = (u8)frac;
    img[4] = 0;
#pragma unroll 4
    for (int i = 0; i < 32; i++) {
        const u32 w = i < N ? m[i < N ? i : 0] : 0u;
        img[5 + 4 * i] = (u8)w;
        img[6 + 4 * i] = (u8)(w >> 8);
        img[7 + 4 * i] = (u8)(w >> 16);
        img[8 + 4 * i] = (u8)(w >> 24);
    }
}

// The AVG image: the nullable SUM divided by its int64 count the way
// nullable_type<Decimal>::operator/=(int64_t) does (aries_types.hxx:626-631 ->
// Decimal::DivOrMod, decimal.cu:2200-2228): the flag survives only a nonzero
// count; a zero dividend gives +0 with prec = frac + 1 (frac already raised by
// 4); a zero count with a nonzero dividend keeps the dividend and sets error
// ERR_DIV_BY_ZERO (2).  q, sign, err: the div_round result for the dividend.
template <int N>
UP_DI void avg_image(u8* img, u32 sum_flag, u64 count, bool dividend_zero, u32 sign, u32 frac,
                     const u32 (&q)[N], u32 err) {
    agg_image(img, (sum_flag && count != 0ull) ? 1u : 0u, dividend_zero ? 0u : sign, frac, q);
    if (dividend_zero) img[2] = (u8)(frac + 1u);
    img[4] = (err & ERR_DIV0) ? 2 : 0;
}

#ifndef UP_HOST_TEST
// ------------------------------------------------- bulk-copy pipeline
// 1-D bulk copies (cp.async.bulk, the TMA engine without a tensor map) between
// global and shared memory, completed through an mbarrier.  Sizes are
// multiples of 16 bytes and both addresses 16-byte aligned (the callers only
// use them for full tiles of 16-byte-aligned columns).  No multicast.
enum : u32 { ERR_TIMEOUT = 8u };

UP_DI u32 smem_addr(const void* p) {
    u32 r;
    asm volatile("{ .reg .u64 t; cvta.to.shared.u64 t, %1; cvt.u32.u64 %0, t; }" : "=r"(r) : "l"(p));
    return r;
}

UP_DI void mbar_init(u64* bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

UP_DI void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

UP_DI void mbar_expect_tx(u64* bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

UP_DI void bulk_load(void* dst_smem, const void* src_gmem, u32 bytes, u64* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Wait for the mbarrier phase with the given parity; gives up after `polls`
// polls and returns false (the caller records ERR_TIMEOUT).
UP_DI bool mbar_wait(u64* bar, u32 parity, u32 polls = 1u << 24) {
    const u32 a = smem_addr(bar);
    for (u32 it = 0; it < polls; it++) {
        u32 done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

UP_DI void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

UP_DI void bulk_store(void* dst_gmem, const void* src_smem, u32 bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem),
                 "r"(smem_addr(src_smem)), "r"(bytes)
                 : "memory");
}

UP_DI void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
UP_DI void bulk_wait_read_1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
UP_DI void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
#endif  // UP_HOST_TEST

}  // namespace up

#endif  // UP_DEV_CUH_
