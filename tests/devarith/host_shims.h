// host_shims.h — TEST INFRASTRUCTURE: lets the arithmetic part of
// ultraprecise_b200/csrc/up_dev.cuh compile as host C++ (g++), so the CPU
// tests can run the device division and multiply code on millions of inputs.
// Each CUDA intrinsic the arithmetic uses is restated from its documented
// meaning (CUDA Math API: integer and type-casting intrinsics, double
// intrinsics with explicit rounding); IEEE-754 host arithmetic gives the
// same results for the correctly rounded operations used.
#ifndef UP_HOST_SHIMS_H_
#define UP_HOST_SHIMS_H_
#include <cfenv>
#include <cmath>
#include <cstdint>
#include <cstring>

#define UP_HOST_TEST 1
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__

struct up_dim3_shim { unsigned x, y, z; };
static const up_dim3_shim threadIdx = {0, 0, 0};
static const up_dim3_shim blockDim = {1, 1, 1};
static const up_dim3_shim blockIdx = {0, 0, 0};
static const up_dim3_shim gridDim = {1, 1, 1};
struct uint4 { unsigned x, y, z, w; };

inline int __clz(unsigned x) { return x ? __builtin_clz(x) : 32; }
inline int __clz(int x) { return __clz((unsigned)x); }
// hi:lo shifted left by (s & 31), the upper 32 bits
inline unsigned __funnelshift_l(unsigned lo, unsigned hi, unsigned s) {
    s &= 31u;
    return s ? (hi << s) | (lo >> (32u - s)) : hi;
}
// hi:lo shifted right by (s & 31), the lower 32 bits
inline unsigned __funnelshift_r(unsigned lo, unsigned hi, unsigned s) {
    s &= 31u;
    return s ? (lo >> s) | (hi << (32u - s)) : lo;
}
inline unsigned __umulhi(unsigned a, unsigned b) { return (unsigned)(((uint64_t)a * b) >> 32); }
inline double __hiloint2double(int hi, int lo) {
    const uint64_t u = ((uint64_t)(uint32_t)hi << 32) | (uint32_t)lo;
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}
inline int __double2hiint(double d) {
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return (int)(uint32_t)(u >> 32);
}
inline int __double2loint(double d) {
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return (int)(uint32_t)u;
}
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __fma_rn(double a, double b, double c) { return std::fma(a, b, c); }
inline double __drcp_rn(double x) { return 1.0 / x; }
inline double __dadd_rd(double a, double b) {
    const int old = std::fegetround();
    std::fesetround(FE_DOWNWARD);
    volatile double va = a, vb = b;
    const double r = va + vb;
    std::fesetround(old);
    return r;
}
inline unsigned atomicAdd(unsigned* p, unsigned v) {
    const unsigned o = *p;
    *p = o + v;
    return o;
}
#endif
