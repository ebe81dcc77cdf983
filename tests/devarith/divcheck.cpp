// divcheck.cpp — TEST INFRASTRUCTURE: the device division code of
// ultraprecise_b200/csrc/up_dev.cuh, compiled for the host (host_shims.h),
// run on many seeded inputs:
//   * reciprocal_u32 against the exact floor((2^64 - 1) / d) - 2^32;
//   * divmod<NX, NB> checked by x == q*b + r and r < b (schoolbook multiply
//     and compare written here, independent of the code under test), on
//     random, structured and constructed operands (quotient digits of all
//     ones, divisors with leading zero limbs, x < b, b = 1 ...);
//   * div_round (the reference's decimal divide rule) against the C oracle's
//     orc_div on the precision-sweep shapes.
// Prints one line per check, "name cases failures"; exit status 1 on any failure.
#include "host_shims.h"
#include "../../ultraprecise_b200/csrc/up_dev.cuh"
extern "C" {
#include "../../oracle/up_oracle.h"
}

#include <cstdio>
#include <cstdlib>

using namespace up;

struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    u32 u32v() { return (u32)next(); }
    int below(int n) { return (int)(next() % (uint64_t)n); }
};

static u32 limb_of(Rng& g, int kind) {
    switch (kind) {
        case 0: return g.u32v();
        case 1: return 0xffffffffu;
        case 2: return 0u;
        case 3: return 0x80000000u;
        case 4: return 0x7fffffffu;
        default: return g.u32v() | 0x80000000u;
    }
}

// a value of `len` significant limbs (len <= N) with a random limb pattern
template <int N>
static void gen(Rng& g, u32 (&a)[N], int len) {
    const int kind = g.below(7);
    for (int i = 0; i < N; i++) a[i] = i < len ? limb_of(g, kind == 6 ? g.below(6) : kind) : 0u;
    if (len > 0 && a[len - 1] == 0u) a[len - 1] = 1u + (g.u32v() >> (g.below(32)));
}

// r = a * b + c (exact, NA + NB limbs; plain loops)
template <int NA, int NB, int NR>
static void mul_add(u32 (&r)[NR], const u32 (&a)[NA], const u32 (&b)[NB], const u32* c, int nc) {
    uint64_t t[NA + NB + 1] = {0};
    for (int i = 0; i < nc && i < NA + NB; i++) t[i] = c[i];
    for (int i = 0; i < NA; i++) {
        uint64_t carry = 0;
        for (int j = 0; j < NB; j++) {
            const uint64_t p = (uint64_t)a[i] * b[j] + (t[i + j] & 0xffffffffull) + carry;
            t[i + j] = p & 0xffffffffull;
            carry = p >> 32;
        }
        for (int k = i + NB; carry && k < NA + NB + 1; k++) {
            const uint64_t s = t[k] + carry;
            t[k] = s & 0xffffffffull;
            carry = s >> 32;
        }
    }
    for (int i = 0; i < NR; i++) r[i] = i < NA + NB ? (u32)t[i] : 0u;
}

template <int N, int M>
static int cmp_n(const u32 (&a)[N], const u32 (&b)[M]) {
    const int L = N > M ? N : M;
    for (int i = L - 1; i >= 0; i--) {
        const u32 x = i < N ? a[i] : 0u, y = i < M ? b[i] : 0u;
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

template <int NX, int NB>
static long check_divmod(Rng& g, long n) {
    long bad = 0;
    for (long c = 0; c < n; c++) {
        u32 x[NX], b[NB];
        const int mode = g.below(4);
        gen(g, b, 1 + g.below(NB));
        if (mode == 0) {
            // constructed x = q*b + r with chosen quotient digits and r < b
            u32 q[NX], r[NB];
            int nq = NX - NB + 1;
            if (nq < 1) nq = 1;
            gen(g, q, g.below(nq + 1));
            for (int i = 0; i < NB; i++) r[i] = g.below(2) ? b[i] : g.u32v();
            // make r < b: r = (r mod b) by one subtraction-free choice
            if (cmp_n(r, b) >= 0) {
                for (int i = 0; i < NB; i++) r[i] = 0u;
                r[0] = b[0] ? b[0] - 1u : 0u;
                if (cmp_n(r, b) >= 0) r[0] = 0u;
            }
            u32 full[NX + NB];
            mul_add<NX, NB>(full, q, b, r, NB);
            bool fits = true;
            for (int i = NX; i < NX + NB; i++) fits &= full[i] == 0u;
            if (!fits) continue;
            for (int i = 0; i < NX; i++) x[i] = full[i];
        } else {
            gen(g, x, g.below(NX + 1));
        }
        u32 q[NX], rem[NB];
        divmod(q, rem, x, b);
        u32 back[NX + NB];
        mul_add<NX, NB>(back, q, b, rem, NB);
        bool ok = cmp_n(rem, b) < 0;
        for (int i = 0; i < NX + NB; i++) ok &= back[i] == (i < NX ? x[i] : 0u);
        if (!ok) {
            if (bad < 3) {
                std::printf("divmod<%d,%d> mismatch: x=", NX, NB);
                for (int i = NX - 1; i >= 0; i--) std::printf("%08x", x[i]);
                std::printf(" b=");
                for (int i = NB - 1; i >= 0; i--) std::printf("%08x", b[i]);
                std::printf("\n");
            }
            bad++;
        }
    }
    std::printf("divmod<%d,%d> %ld %ld\n", NX, NB, n, bad);
    return bad;
}

static long check_reciprocal(Rng& g, long n) {
    long bad = 0;
    for (long c = 0; c < n; c++) {
        u32 d;
        switch (c % 8) {
            case 0: d = 0x80000000u + (u32)c; break;
            case 1: d = 0xffffffffu - (u32)c; break;
            case 2: d = 0x80000000u | (1u << (c % 31)); break;
            default: d = g.u32v() | 0x80000000u;
        }
        const unsigned __int128 num = ~(uint64_t)0;
        const u32 want = (u32)((uint64_t)(num / d) - (1ull << 32));
        if (reciprocal_u32(d) != want) {
            if (bad < 3) std::printf("reciprocal_u32(%08x) = %08x, want %08x\n", d, reciprocal_u32(d), want);
            bad++;
        }
    }
    std::printf("reciprocal_u32 %ld %ld\n", n, bad);
    return bad;
}

// p random decimal digits as limbs
template <int N>
static void digits(Rng& g, u32 (&a)[N], int p) {
    for (int i = 0; i < N; i++) a[i] = 0u;
    int left = p;
    while (left > 0) {
        const int d = left >= 9 ? 9 : left;
        left -= d;
        u32 mul = 1;
        for (int k = 0; k < d; k++) mul *= 10u;
        uint64_t carry = g.next() % mul;
        for (int i = 0; i < N; i++) {
            const uint64_t t = (uint64_t)a[i] * mul + carry;
            a[i] = (u32)t;
            carry = t >> 32;
        }
    }
    if (g.below(16) == 0) {  // short values too (small dividends, one-limb divisors)
        const int keep = g.below(N) + 1;
        for (int i = keep; i < N; i++) a[i] = 0u;
    }
}

// 10^k modulo 2^64
constexpr uint64_t pow10_mod64(int k) {
    uint64_t v = 1;
    for (int i = 0; i < k; i++) v *= 10u;
    return v;
}

template <int NA, int NP, u32 SHIFT, uint64_t P10W>
static long check_div_round(Rng& g, long n, int p, int s) {
    constexpr int NR = NA + NP + 1;
    u32 p10[NP];
    {
        for (int i = 0; i < NP; i++) p10[i] = 0u;
        p10[0] = 1u;
        for (u32 k = 0; k < SHIFT; k++) {
            uint64_t c = 0;
            for (int i = 0; i < NP; i++) {
                const uint64_t t = (uint64_t)p10[i] * 10u + c;
                p10[i] = (u32)t;
                c = t >> 32;
            }
        }
    }
    static orc_dec oa, ob, orr;
    long bad = 0;
    for (long c = 0; c < n; c++) {
        u32 a[NA], b[NA];
        digits(g, a, p);
        digits(g, b, p);
        const u32 sa = (u32)g.below(2), sb = (u32)g.below(2);
        if (g.below(64) == 0) for (int i = 0; i < NA; i++) b[i] = 0u;  // a zero divisor now and then
        u32 r[NR], sr;
        const u32 err = div_round<NR, NA, NA, NP, SHIFT, P10W>(r, sr, a, sa, b, sb, p10);
        oa.sign = sa; oa.frac = s; oa.n = NA; ob.sign = sb; ob.frac = s; ob.n = NA;
        for (int i = 0; i < NA; i++) { oa.m[i] = a[i]; ob.m[i] = b[i]; }
        while (oa.n > 0 && oa.m[oa.n - 1] == 0u) oa.n--;
        while (ob.n > 0 && ob.m[ob.n - 1] == 0u) ob.n--;
        const uint32_t oerr = orc_div(&orr, &oa, &ob);
        bool ok = (err != 0) == (oerr != 0);
        for (int i = 0; i < NR; i++) ok &= r[i] == (i < orr.n ? orr.m[i] : 0u);
        for (int i = NR; i < orr.n; i++) ok &= orr.m[i] == 0u;
        const bool zero = orr.n == 0;
        ok &= zero ? true : (sr == orr.sign);
        if (!ok) {
            if (bad < 3) std::printf("div_round p=%d mismatch\n", p);
            bad++;
        }
    }
    std::printf("div_round_p%d %ld %ld\n", p, n, bad);
    return bad;
}

// div_small_quotient on x = q*b + r built from a chosen quotient (below 2^48,
// boundaries included) and remainder (0, 1, b/2 - 1, b/2, b - 1, random).
template <int NX, int NB>
static long check_div_small(Rng& g, long n) {
    long bad = 0, ran = 0;
    for (long c = 0; c < n; c++) {
        u32 b[NB];
        const int len = 2 + g.below(NB - 1);  // wider than one limb
        gen(g, b, len);
        uint64_t qq;
        switch (c % 6) {
            case 0: qq = (1ull << 48) - 1 - (g.next() % 3); break;
            case 1: qq = g.next() % 4; break;
            case 2: qq = 1ull << (g.below(48)); break;
            default: qq = g.next() & ((1ull << 48) - 1);
        }
        // r in [0, b): 0, 1, b - 1, b/2 - 1, b/2 or random below b
        u32 r[NB], half[NB];
        for (int i = 0; i < NB; i++) half[i] = (b[i] >> 1) | (i + 1 < NB ? b[i + 1] << 31 : 0u);
        const int rk = g.below(6);
        for (int i = 0; i < NB; i++) r[i] = 0u;
        if (rk == 1) r[0] = 1u;
        else if (rk == 2) { u32 one[1] = {1u}; sub(r, b, one); }
        else if (rk == 3) { u32 one[1] = {1u}; sub(r, half, one); }
        else if (rk == 4) { for (int i = 0; i < NB; i++) r[i] = half[i]; }
        else if (rk == 5) { gen(g, r, len); if (cmp_n(r, b) >= 0) for (int i = 0; i < NB; i++) r[i] = half[i]; }
        u32 qv[2] = {(u32)qq, (u32)(qq >> 32)};
        u32 xw[NX + NB + 2];
        mul_add(xw, b, qv, r, NB);
        bool fits = true;
        for (int i = NX; i < NX + NB + 2; i++) fits &= xw[i] == 0u;
        if (!fits) continue;  // q*b + r wider than the dividend's static width
        u32 x[NX];
        for (int i = 0; i < NX; i++) x[i] = xw[i];
        // skip inputs the caller would not route here (quotient bound by bit lengths)
        if (!(bitlen(x) <= bitlen(b) + 47u) || bitlen(b) <= 32u) continue;
        u32 q[NX];
        bool up;
        ran++;
        div_small_quotient(q, up, x, b);
        u32 dbl[NB + 1];
        add(dbl, r, r);
        const bool want_up = cmp_n(dbl, b) >= 0;
        bool ok = up == want_up && q[0] == qv[0] && q[1] == qv[1];
        for (int i = 2; i < NX; i++) ok &= q[i] == 0u;
        if (!ok) {
            if (bad < 3) std::printf("div_small<%d,%d> mismatch q=%llu\n", NX, NB, (unsigned long long)qq);
            bad++;
        }
    }
    std::printf("div_small<%d,%d> %ld %ld\n", NX, NB, ran, bad);
    return bad + (ran < n / 8 ? 1 : 0);  // the constructed cases must mostly reach the path
}

int main(int argc, char** argv) {
    const long n = argc > 1 ? std::atol(argv[1]) : 100000;
    Rng g{argc > 2 ? (uint64_t)std::atoll(argv[2]) : 20261203ull};
    long bad = 0;
    bad += check_reciprocal(g, n);
    bad += check_divmod<2, 1>(g, n);
    bad += check_divmod<3, 2>(g, n);
    bad += check_divmod<4, 2>(g, n);
    bad += check_divmod<6, 4>(g, n);
    bad += check_divmod<5, 4>(g, n);
    bad += check_divmod<11, 8>(g, n);
    bad += check_divmod<9, 3>(g, n);
    bad += check_divmod<21, 16>(g, n / 4);
    bad += check_divmod<41, 32>(g, n / 16);
    bad += check_divmod<24, 5>(g, n / 8);
    bad += check_divmod<72, 63>(g, n / 64);
    bad += check_div_small<3, 2>(g, n);
    bad += check_div_small<6, 4>(g, n);
    bad += check_div_small<8, 4>(g, n);
    bad += check_div_round<2, 1, 8u, 100000000ull>(g, n, 18, 4);
    bad += check_div_round<4, 2, 13u, 10000000000000ull>(g, n, 38, 9);
    bad += check_div_round<8, 3, 23u, 0x2c7e14af6800000ull>(g, n / 2, 76, 19);
    bad += check_div_round<16, 5, 41u, pow10_mod64(41)>(g, n / 8, 150, 37);
    bad += check_div_round<32, 9, 79u, pow10_mod64(79)>(g, n / 32, 300, 75);
    bad += check_div_round<63, 17, 154u, pow10_mod64(154)>(g, n / 128, 600, 150);
    return bad ? 1 : 0;
}
