// ref_agg_harness.cu — TEST INFRASTRUCTURE: runs the reference's own 32-limb
// Decimal code (src/datatypes/decimal.cu, compiled from the reference sources
// where they lie by oracle/ref/Makefile) on the GPU, for the parts of the
// exact-decimal path that the AriesDecimal<LEN> harness (ref_harness.cu) does
// not reach:
//
//   * grouped SUM: every segment's values are turned into Decimal by the
//     constructor the aggregation uses (Decimal(CompactDecimal*, p, s),
//     decimal.cu:168-177; AriesEngineAlgorithm.h:836-840) and added, four
//     threads per value, by the XMP operator_add of the segmented reduction
//     (decimal.cu:3319-3376, called at kernel_segreduce.hxx:131,199); the
//     group's image is the reduction's store of sign and limbs
//     (kernel_segreduce.hxx:208-219) followed by the host fill of flag = 1
//     and frac = input scale (kernel_segreduce.hxx:609-612);
//   * AVG: the do_div body (kernel_util.hxx:426-438) — a
//     nullable_type<Decimal> copy of the SUM image divided by the int64 count
//     (aries_types.hxx:626-631 -> Decimal::operator/=(int64_t),
//     decimal.cu:2469-2472 -> DivOrMod, :2200-2331);
//   * decimal text in: the CSV import's Decimal(p, s, STRICT, str) followed
//     by ToCompactDecimal (importCsvFile.cpp:1885-1904; decimal.cu:158-165,
//     337-341), with the constructor's error code per row;
//   * decimal text out: Decimal::GetDecimal (decimal.cu:362-398) of each
//     compact value.
//
// Safety (nothing here may fault or hang a GPU): the harness entry points
// refuse precisions above 299 digits (its byte table's end) and text fields of more than 200
// characters (the reference reads its NUL-terminated copy of the field);
// each thread's stack is fitted to the kernels' measured frames before the
// first launch; the reference is compiled at -O0 (its optimised build of
// decimal.cu does not finish in reasonable time), which changes no result.
#include <cuda_runtime.h>
#include <stdint.h>

#include "AriesDefinition.h"
#include "datatypes/decimal.hxx"
#include "datatypes/aries_types.hxx"

using aries_acc::CompactDecimal;
using aries_acc::Decimal;
using aries_acc::nullable_type;

static_assert(sizeof(nullable_type<Decimal>) == 133, "the SUM/AVG output image is 133 bytes");

namespace {

constexpr int kMaxPrec = 299;  // the reference byte table ends at 299
constexpr int kMaxField = 200;

// One XMP instance (TPI threads, LIMBS limbs each) per segment.
__global__ void k_xmp_sum(const char* data, int len, int prec, int sca, const int* assoc, const int* starts,
                          int n_groups, int64_t rows, nullable_type<Decimal>* out) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t g = tid / TPI;
    const int lane = (int)(threadIdx.x & (TPI - 1));
    if (g >= n_groups) return;  // every thread of an instance leaves together
    const int64_t b = starts[g];
    const int64_t e = g + 1 < n_groups ? starts[g + 1] : rows;
    if (e <= b) return;
    uint32_t acc[LIMBS];
    uint8_t sign = 0;
    for (int64_t i = b; i < e; i++) {
        const int64_t row = assoc ? assoc[i] : i;
        Decimal d((const CompactDecimal*)(data + row * len), prec, sca);
        uint32_t x[LIMBS];
        for (int k = 0; k < LIMBS; k++) x[k] = d.v[lane * LIMBS + k];
        if (i == b) {
            for (int k = 0; k < LIMBS; k++) acc[k] = x[k];
            sign = d.sign;
        } else {
            sign = aries_acc::operator_add(acc, acc, x, 0, sign, d.sign);
        }
    }
    nullable_type<Decimal>& o = out[g];
    if (lane == 0) o.value.sign = sign;
    for (int k = 0; k < LIMBS; k++) o.value.v[lane * LIMBS + k] = acc[k];
    if (lane == 0) {
        o.flag = 1;
        o.value.frac = (uint8_t)sca;
    }
}

__global__ void k_div_int64(const nullable_type<Decimal>* sums, const int64_t* counts, int n,
                            nullable_type<Decimal>* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    nullable_type<Decimal> r(sums[i]);
    r /= counts[i];
    out[i] = r;
}

__global__ void k_parse(const char* text, const int64_t* offsets, int64_t rows, int prec, int sca, int nbytes,
                        char* out, uint8_t* err) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    char buf[kMaxField + 1];
    const int64_t a = offsets[r], n = offsets[r + 1] - a;
    for (int64_t i = 0; i < n; i++) buf[i] = text[a + i];
    buf[n] = '\0';
    Decimal v((uint32_t)prec, (uint32_t)sca, ARIES_MODE_STRICT_ALL_TABLES, buf);
    v.ToCompactDecimal(out + r * nbytes, nbytes);
    err[r] = (uint8_t)v.GetError();
}

__global__ void k_format(const char* compact, int64_t rows, int prec, int sca, int nbytes, char* out, int width) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    Decimal d((const CompactDecimal*)(compact + r * nbytes), prec, sca);
    char buf[8 * NUM_TOTAL_DIG + 8];
    d.GetDecimal(buf);
    char* o = out + r * width;
    int i = 0;
    for (; i < width - 1 && buf[i]; i++) o[i] = buf[i];
    for (; i < width; i++) o[i] = '\0';
}

// Fit the per-thread stack to the largest kernel frame (plus the calls it
// makes: the reference's functions are not inlined at -O0).
int fit_stack() {
    static int done = 0;
    if (done) return 0;
    size_t need = 0;
    const void* ks[] = {(const void*)k_xmp_sum, (const void*)k_div_int64, (const void*)k_parse,
                        (const void*)k_format};
    for (const void* k : ks) {
        cudaFuncAttributes at;
        if (cudaFuncGetAttributes(&at, k) != cudaSuccess) return -3;
        if (at.localSizeBytes > need) need = at.localSizeBytes;
    }
    size_t cur = 0;
    cudaDeviceGetLimit(&cur, cudaLimitStackSize);
    const size_t want = need + 32768;
    if (cur < want && cudaDeviceSetLimit(cudaLimitStackSize, want) != cudaSuccess) return -4;
    done = 1;
    return 0;
}

int finish() {
    const cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // namespace

// Bytes per compact value of the reference's table (decimal.cu:92,464-467).
extern "C" int refagg_compact_bytes(int prec) {
    if (prec < 1 || prec > kMaxPrec) return -1;
    return aries_acc::GetDecimalRealBytes((uint16_t)prec, 0);
}

// Grouped SUM of a compact DECIMAL(prec, sca) column.  Segment g covers the
// visiting positions [starts[g], starts[g+1]) (the last one ends at rows);
// position i reads row assoc[i] (or i when assoc is NULL).  out receives
// n_groups 133-byte images and must be zero-filled by the caller (prec and
// error are left as they were, as in the reference).  Device pointers.
extern "C" int refagg_sum(const void* data, int prec, int sca, const int* assoc, const int* starts, int n_groups,
                          int64_t rows, void* out) {
    if (prec < 1 || prec > kMaxPrec || n_groups < 0 || rows < 0) return -2;
    if (int rc = fit_stack()) return rc;
    if (n_groups == 0) return 0;
    const int len = aries_acc::GetDecimalRealBytes((uint16_t)prec, (uint16_t)sca);
    const int64_t threads = (int64_t)n_groups * TPI;
    const unsigned blocks = (unsigned)((threads + 31) / 32);
    k_xmp_sum<<<blocks, 32>>>((const char*)data, len, prec, sca, assoc, starts, n_groups, rows,
                              (nullable_type<Decimal>*)out);
    return finish();
}

// AVG images: the SUM images divided by the counts.  Device pointers.
extern "C" int refagg_div_int64(const void* sums, const int64_t* counts, int n, void* out) {
    if (n < 0) return -2;
    if (int rc = fit_stack()) return rc;
    if (n == 0) return 0;
    k_div_int64<<<(unsigned)((n + 63) / 64), 64>>>((const nullable_type<Decimal>*)sums, counts, n,
                                                 (nullable_type<Decimal>*)out);
    return finish();
}

// Text fields -> compact DECIMAL(prec, sca) + the constructor's error code per
// row.  Field r is text[offsets[r] .. offsets[r+1]) and must be at most 200
// characters (checked on the host copy of the offsets given in host_offsets).
extern "C" int refagg_parse(const char* text, const int64_t* offsets, const int64_t* host_offsets, int64_t rows,
                            int prec, int sca, void* out, uint8_t* err) {
    if (prec < 1 || prec > kMaxPrec || rows < 0) return -2;
    for (int64_t r = 0; r < rows; r++)
        if (host_offsets[r + 1] - host_offsets[r] > kMaxField || host_offsets[r + 1] < host_offsets[r]) return -2;
    if (int rc = fit_stack()) return rc;
    if (rows == 0) return 0;
    const int nbytes = aries_acc::GetDecimalRealBytes((uint16_t)prec, (uint16_t)sca);
    k_parse<<<(unsigned)((rows + 63) / 64), 64>>>(text, offsets, rows, prec, sca, nbytes, (char*)out, err);
    return finish();
}

// Compact DECIMAL(prec, sca) -> GetDecimal text in slots of `width` bytes
// (NUL-padded; width >= 8 * 32 + 8 holds any value).
extern "C" int refagg_format(const void* compact, int64_t rows, int prec, int sca, char* out, int width) {
    if (prec < 1 || prec > kMaxPrec || rows < 0 || width < 2) return -2;
    if (int rc = fit_stack()) return rc;
    if (rows == 0) return 0;
    const int nbytes = aries_acc::GetDecimalRealBytes((uint16_t)prec, (uint16_t)sca);
    k_format<<<(unsigned)((rows + 63) / 64), 64>>>((const char*)compact, rows, prec, sca, nbytes, out, width);
    return finish();
}
