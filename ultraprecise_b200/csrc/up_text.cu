// up_text.cu — decimal text in and out on the GPU.
//
// Parsing follows the reference's string constructor of a typed decimal
// (Decimal::Decimal(precision, scale, mode, str), decimal.cu:158-165): the
// text is read by StringToDecimal (decimal.cu:2980-3025) — an optional
// leading '-', digits and at most one '.'; the magnitude is every digit, the
// scale is the number of digits after the '.' — and then cast to the column's
// scale (Decimal::cast, decimal.cu:471-533): more fraction digits than the
// column keeps are cut off (truncation toward zero, no rounding), fewer are
// padded with zeros.  The compact value keeps the low B(p) bytes with the
// sign in bit 7 of the last byte (ToCompactDecimal, decimal.cu:337-341).
// Where the reference reads past the text or turns other characters into
// digits (a second '.', any non-digit), this parser flags UP_ROWERR_DOMAIN and
// stores 0; lost magnitude bits flag UP_ROWERR_OVERFLOW.
//
// Formatting writes one fixed-width slot per row: either the reference's
// output image (Decimal::GetDecimal, decimal.cu:362-398: '+' or '-', eight
// upper-case hex digits per 32-bit limb from the highest nonzero limb down,
// then the scale as "(fff)"), or the plain decimal string ("-123.4500": a '-'
// when the sign bit is set, the digits, a '.' before the last `scale`
// digits).  The decimal string parses back to the same compact bytes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/ultraprecise.h"
#include "up_internal.h"

namespace upi {
namespace {

using u8 = uint8_t;
using u32 = uint32_t;
using u64 = uint64_t;

constexpr int kMaxPrecisionText = 1000;
constexpr int kMaxDigits = 1500;  // digits of one field
// 8960 bits: 1500 digits plus up to 1000 zeros of scale padding
constexpr int kMaxLimbs = 280;

__device__ __forceinline__ void mul_add_small(u32* m, int& nl, u32 k, u32 add) {
    u64 c = add;
    for (int i = 0; i < nl; i++) {
        const u64 t = (u64)m[i] * k + c;
        m[i] = (u32)t;
        c = t >> 32;
    }
    if (c && nl < kMaxLimbs) m[nl++] = (u32)c;
}

// m = floor(m / d), d < 2^32
__device__ __forceinline__ u32 div_small(u32* m, int& nl, u32 d) {
    u64 r = 0;
    for (int i = nl - 1; i >= 0; i--) {
        const u64 cur = (r << 32) | m[i];
        m[i] = (u32)(cur / d);
        r = cur % d;
    }
    while (nl > 1 && m[nl - 1] == 0u) nl--;
    return (u32)r;
}

__device__ __forceinline__ u32 pow10_u32(int k) {
    u32 p = 1;
    for (int i = 0; i < k; i++) p *= 10u;
    return p;
}

__global__ void k_parse_decimal(const char* __restrict__ text, const int64_t* __restrict__ off, int64_t rows,
                                int scale, int B, u8* __restrict__ out, u32* __restrict__ err_word) {
    u32 err = 0u;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += stride) {
        const char* s = text + off[r];
        const int64_t n = off[r + 1] - off[r];
        u32 m[kMaxLimbs];
        int nl = 1;
        m[0] = 0u;
        u32 sign = 0u;
        int64_t i = 0;
        if (n > 0 && s[0] == '-') {
            sign = 1u;
            i = 1;
        }
        bool dot = false, bad = false;
        int frac = 0, digits = 0, clen = 0;
        u32 chunk = 0;
        for (; i < n; i++) {
            const char c = s[i];
            if (c == '.' && !dot) {
                dot = true;
                continue;
            }
            if (c < '0' || c > '9' || digits >= kMaxDigits) {
                bad = true;
                break;
            }
            chunk = chunk * 10u + (u32)(c - '0');
            clen++;
            digits++;
            if (dot) frac++;
            if (clen == 9) {
                mul_add_small(m, nl, 1000000000u, chunk);
                chunk = 0u;
                clen = 0;
            }
        }
        if (!bad && clen) mul_add_small(m, nl, pow10_u32(clen), chunk);
        if (!bad) {
            // to the column's scale: pad with zeros or cut digits off
            for (int d = scale - frac; d > 0; d -= 9) mul_add_small(m, nl, pow10_u32(d < 9 ? d : 9), 0u);
            for (int d = frac - scale; d > 0; d -= 9) div_small(m, nl, pow10_u32(d < 9 ? d : 9));
        }
        u8* o = out + r * B;
        if (bad) {
            err |= UP_ROWERR_DOMAIN;
            for (int b = 0; b < B; b++) o[b] = 0;
            continue;
        }
        // low B bytes; magnitude bits at or above 8B-1 are lost (sign bit)
        bool lost = false;
        for (int b = 0; b < 4 * nl; b++) {
            const u32 byte = (m[b >> 2] >> (8 * (b & 3))) & 0xffu;
            if (b < B) {
                u32 v = byte;
                if (b == B - 1) {
                    lost |= (v & 0x80u) != 0u;
                    v |= sign << 7;
                }
                o[b] = (u8)v;
            } else {
                lost |= byte != 0u;
            }
        }
        for (int b = 4 * nl; b < B; b++) o[b] = (u8)(b == B - 1 ? sign << 7 : 0u);
        if (lost) err |= UP_ROWERR_OVERFLOW;
    }
    if (err && err_word) atomicOr(err_word, err);
}

__global__ void k_format_decimal(const u8* __restrict__ in, int64_t rows, int B, int scale, int hex,
                                 char* __restrict__ out, int width, int32_t* __restrict__ out_len) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += stride) {
        const u8* p = in + r * B;
        u32 m[kMaxLimbs];
        const int nl0 = (B + 3) / 4;
        for (int i = 0; i < nl0; i++) m[i] = 0u;
        for (int b = 0; b < B; b++) m[b >> 2] |= (u32)p[b] << (8 * (b & 3));
        const u32 sign = (u32)(p[B - 1] >> 7);
        m[(B - 1) >> 2] &= ~(0x80u << (8 * ((B - 1) & 3)));
        char* o = out + r * width;
        int len = 0;
        auto put = [&](char c) {
            if (len < width) o[len] = c;
            len++;
        };
        if (hex) {
            // Decimal::GetDecimal: sign, 8 hex digits per limb from the highest
            // nonzero one, then "(fff)"
            const char* dig = "0123456789ABCDEF";
            put(sign ? '-' : '+');
            int top = nl0 - 1;
            while (top >= 0 && m[top] == 0u) top--;
            for (int i = top; i >= 0; i--)
                for (int j = 7; j >= 0; j--) put(dig[(m[i] >> (4 * j)) & 0xfu]);
            put('(');
            put((char)('0' + scale / 100 % 10));
            put((char)('0' + scale / 10 % 10));
            put((char)('0' + scale % 10));
            put(')');
        } else {
            // decimal digits, least significant first, in base 10^9 chunks
            int nl = nl0;
            while (nl > 1 && m[nl - 1] == 0u) nl--;
            char rev[kMaxDigits + 16];
            int nd = 0;
            do {
                u32 rem = div_small(m, nl, 1000000000u);
                const bool last = nl == 1 && m[0] == 0u;
                for (int k = 0; k < 9 && (nd < kMaxDigits + 16); k++) {
                    rev[nd++] = (char)('0' + rem % 10u);
                    rem /= 10u;
                    if (last && rem == 0u) break;
                }
                if (last) break;
            } while (true);
            while (nd > 1 && rev[nd - 1] == '0') nd--;  // no leading zeros
            while (nd < scale + 1) rev[nd++] = '0';      // at least "0." before the fraction
            if (sign) put('-');
            for (int k = nd - 1; k >= 0; k--) {
                put(rev[k]);
                if (k == scale && scale > 0) put('.');
            }
        }
        out_len[r] = len <= width ? len : -1;
    }
}

int grid_for(int64_t rows) {
    const int64_t blocks = (rows + 127) / 128;
    const int sms = std::max(1, sm_count_current());
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)sms * 16));
}

}  // namespace
}  // namespace upi

using namespace upi;

extern "C" {

up_status up_parse_decimal(const char* text, const int64_t* offsets, int64_t rows, int32_t precision, int32_t scale,
                           void* out, uint32_t* err_word, void* stream) {
    if (rows < 0) return fail(UP_ERR_INVALID_ARG, "negative row count");
    if (precision < 1 || precision > kMaxPrecisionText || scale < 0 || scale > precision)
        return fail(UP_ERR_INVALID_ARG, "precision 1..1000 and 0 <= scale <= precision");
    if (rows == 0) return UP_OK;
    if (!text || !offsets || !out) return fail(UP_ERR_INVALID_ARG, "NULL buffers");
    const int B = compact_bytes(precision);
    k_parse_decimal<<<grid_for(rows), 128, 0, (cudaStream_t)stream>>>(text, offsets, rows, scale, B, (u8*)out,
                                                                      err_word);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? UP_ERR_NO_DEVICE : UP_ERR_CUDA,
                    std::string("parse launch: ") + cudaGetErrorString(e));
    return UP_OK;
}

int32_t up_format_width(int32_t precision, int32_t hex) {
    if (precision < 1 || precision > kMaxPrecisionText) return -1;
    const int B = compact_bytes(precision);
    if (hex) return 1 + 8 * ((B + 3) / 4) + 5;
    // digits of the largest magnitude B bytes can hold (2^(8B-1) - 1), a sign,
    // a '.' and a leading 0
    const int digits = (int)std::floor((8.0 * B - 1.0) * std::log10(2.0)) + 1;
    return digits + 3;
}

up_status up_format_decimal(const void* compact, int64_t rows, int32_t precision, int32_t scale, int32_t hex,
                            char* out_text, int32_t width, int32_t* out_len, void* stream) {
    if (rows < 0 || width < 1) return fail(UP_ERR_INVALID_ARG, "negative row count or width");
    if (precision < 1 || precision > kMaxPrecisionText || scale < 0 || scale > precision)
        return fail(UP_ERR_INVALID_ARG, "precision 1..1000 and 0 <= scale <= precision");
    if (rows == 0) return UP_OK;
    if (!compact || !out_text || !out_len) return fail(UP_ERR_INVALID_ARG, "NULL buffers");
    const int B = compact_bytes(precision);
    k_format_decimal<<<grid_for(rows), 128, 0, (cudaStream_t)stream>>>((const u8*)compact, rows, B, scale, hex ? 1 : 0,
                                                                       out_text, width, out_len);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? UP_ERR_NO_DEVICE : UP_ERR_CUDA,
                    std::string("format launch: ") + cudaGetErrorString(e));
    return UP_OK;
}

}  // extern "C"
