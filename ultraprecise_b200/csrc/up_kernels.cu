// up_kernels.cu — precompiled sm_100a kernels: segment ids, AVG division,
// small-key grouping, and the benchmark utilities of ultraprecise_util.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/ultraprecise.h"
#include "../../include/ultraprecise_util.h"
#include "up_dev.cuh"
#include "up_internal.h"
#include "up_kernels.h"

namespace upi {

using up::u32;
using up::u64;
using up::u8;

// ------------------------------------------------ segment starts -> ids
// group of row position i = (last start <= i); the reference's segments
// (AriesSqlOperator_group.cu:14-54) are ascending starts into `associated`.
__global__ void k_fill_segment_gids(const int32_t* __restrict__ starts, int32_t n_groups, int64_t rows,
                                    int32_t* __restrict__ gid) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += stride) {
        int lo = 0, hi = n_groups;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if ((int64_t)starts[mid] <= i) lo = mid + 1;
            else hi = mid;
        }
        gid[i] = lo - 1;
    }
}

cudaError_t launch_fill_segment_gids(const int32_t* starts, int32_t n_groups, int64_t rows, int32_t* gid,
                                     cudaStream_t s) {
    if (rows <= 0) return cudaSuccess;
    int64_t blocks = std::min<int64_t>((rows + 255) / 256, 148 * 16);
    k_fill_segment_gids<<<(unsigned)blocks, 256, 0, s>>>(starts, n_groups, rows, gid);
    return cudaGetLastError();
}

// ------------------------------------------------------ AVG division
// DivisionInt64 (AriesSqlOperator_helpers.cu:717-763 -> do_div,
// kernel_util.hxx:426-438): Decimal(sum) /= int64 count, i.e. the divide
// rule with the divisor a scale-0 integer: scale + 4, half-up.
__global__ void k_division_int64(const u8* __restrict__ sums, const int64_t* __restrict__ counts, int32_t n,
                                 u8* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u8* img = sums + (int64_t)i * UP_AGG_DECIMAL_BYTES;
    u32 m[32];
#pragma unroll
    for (int k = 0; k < 32; k++)
        m[k] = (u32)img[5 + 4 * k] | ((u32)img[6 + 4 * k] << 8) | ((u32)img[7 + 4 * k] << 16) |
               ((u32)img[8 + 4 * k] << 24);
    const u32 sign = img[1] ? 1u : 0u;
    const u64 cnt = (u64)counts[i];
    const u32 c2[2] = {(u32)cnt, (u32)(cnt >> 32)};
    const u32 p10[1] = {10000u};
    u32 q[34];
    u32 sq;
    const u32 err = up::div_round<34, 32, 2, 1, 4u, 10000ull>(q, sq, m, sign, c2, 0u, p10);
    u8* o = out + (int64_t)i * UP_AGG_DECIMAL_BYTES;
    up::avg_image(o, img[0], cnt, up::is_zero(m), sq, (u32)img[3] + 4u, q, err);
}

cudaError_t launch_division_int64(const uint8_t* sums, const int64_t* counts, int32_t n, uint8_t* out,
                                  cudaStream_t s) {
    k_division_int64<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(sums, counts, n, out);
    return cudaGetLastError();
}

// --------------------------------------------------- small-key grouping
// Keys of at most 2 bytes in total.  A row's key is its key bytes in column
// order, most significant first, so ascending keys are the order of the
// reference's sort-based GroupColumns (AriesSqlOperator_group.cu:14-54).
// The key table maps each of the 65536 possible keys to its dense group id
// (-1 for an absent key); its second half lists the present keys by id, and
// entry 131072 holds the group count.
struct KeyCols {
    const u8* col[4];
    int bytes[4];
    int n;
    int fast16;  // 1 or 2 one-byte key columns, 16-byte aligned
};

__device__ __forceinline__ u32 row_key(const KeyCols& k, int64_t row) {
    u32 key = 0;
    for (int c = 0; c < k.n; c++)
        for (int b = 0; b < k.bytes[c]; b++) key = (key << 8) | k.col[c][row * k.bytes[c] + b];
    return key;
}

constexpr int kKeyWords = 65536 / 32;  // words of the key presence bitmap

__device__ __forceinline__ void mark_key(u32* sb, u32 key) {
    const u32 m = 1u << (key & 31u);
    if (!(sb[key >> 5] & m)) atomicOr(&sb[key >> 5], m);
}

// Every block marks the keys of its rows in a shared-memory bitmap (one-byte
// key columns are read 16 rows per 16-byte load), then ORs its nonzero words
// into the global bitmap.
__global__ void __launch_bounds__(256) k_mark_keys(KeyCols k, int64_t rows, u32* __restrict__ bits) {
    __shared__ u32 sb[kKeyWords];
    for (int i = threadIdx.x; i < kKeyWords; i += blockDim.x) sb[i] = 0u;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t done = 0;
    if (k.fast16) {
        const int64_t nvec = rows / 16;
        const uint4* a = (const uint4*)k.col[0];
        const uint4* b = (const uint4*)k.col[1];
        // two vectors per column in flight per thread, then 32 marks
        for (int64_t v = tid; v < nvec; v += 2 * stride) {
            const bool two = v + stride < nvec;
            uint4 x[2], y[2];
            x[0] = a[v];
            x[1] = two ? a[v + stride] : x[0];
            y[0] = k.n == 2 ? b[v] : make_uint4(0u, 0u, 0u, 0u);
            y[1] = k.n == 2 && two ? b[v + stride] : y[0];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const u32 xw[4] = {x[h].x, x[h].y, x[h].z, x[h].w}, yw[4] = {y[h].x, y[h].y, y[h].z, y[h].w};
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    if (k.n == 2) {
                        // two 16-bit keys per word: bytes (lo, hi) of rows 0-1, then rows 2-3
                        const u32 p01 = __byte_perm(xw[w], yw[w], 0x1504u);
                        const u32 p23 = __byte_perm(xw[w], yw[w], 0x3726u);
                        mark_key(sb, p01 & 0xffffu);
                        mark_key(sb, p01 >> 16);
                        mark_key(sb, p23 & 0xffffu);
                        mark_key(sb, p23 >> 16);
                    } else {
#pragma unroll
                        for (int j = 0; j < 4; j++) mark_key(sb, (xw[w] >> (8 * j)) & 0xffu);
                    }
                }
            }
        }
        done = nvec * 16;
    }
    for (int64_t i = done + tid; i < rows; i += stride) mark_key(sb, row_key(k, i));
    __syncthreads();
    for (int i = threadIdx.x; i < kKeyWords; i += blockDim.x)
        if (sb[i]) atomicOr(&bits[i], sb[i]);
}

// one block: dense ids in key order from the presence bitmap, the key table,
// the group count and the distinct keys.  The bitmap and the exclusive count
// before each 64-key range are staged in shared memory, then thread t writes
// the table entries of keys t, t + 1024, ... (coalesced).
__global__ void __launch_bounds__(1024) k_scan_keys(const u32* __restrict__ bits, int32_t* __restrict__ table,
                                                    int32_t* __restrict__ n_out, u8* __restrict__ keys_out,
                                                    int key_bytes) {
    __shared__ u32 sbits[kKeyWords];
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const u32 w0 = bits[2 * t], w1 = bits[2 * t + 1];
    sbits[2 * t] = w0;
    sbits[2 * t + 1] = w1;
    const int c = __popc(w0) + __popc(w1);
    part[t] = c;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    const int total = part[1023];
    __syncthreads();
    part[t] -= c;  // exclusive count before range t
    __syncthreads();
    for (int i = 0; i < 64; i++) {
        const int key = i * 1024 + t;
        const int range = key >> 6, b = key & 63;
        const u32 lo = sbits[2 * range], hi = sbits[2 * range + 1];
        const u32 wb = b < 32 ? lo : hi;
        const bool present = ((wb >> (b & 31)) & 1u) != 0u;
        int id = -1;
        if (present) {
            const u32 below = (1u << (b & 31)) - 1u;
            id = part[range] + (b < 32 ? __popc(lo & below) : __popc(lo) + __popc(hi & below));
            table[65536 + id] = key;
            if (keys_out)
                for (int k = 0; k < key_bytes; k++)
                    keys_out[(int64_t)id * key_bytes + k] = (u8)(key >> (8 * (key_bytes - 1 - k)));
        }
        table[key] = id;
    }
    if (t == 0) *n_out = total;
}

__global__ void k_map_keys(KeyCols k, int64_t rows, const int32_t* __restrict__ table, int32_t* __restrict__ gid) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += stride)
        gid[i] = __ldg(table + row_key(k, i));
}

namespace {

KeyCols key_cols_of(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys, int* total) {
    KeyCols k;
    *total = 0;
    bool fast = n_keys <= 2;
    for (int c = 0; c < 4; c++) {
        k.col[c] = c < n_keys ? (const u8*)key_cols[c] : nullptr;
        k.bytes[c] = c < n_keys ? key_bytes[c] : 0;
        *total += k.bytes[c];
        if (c < n_keys) fast = fast && key_bytes[c] == 1 && ((uintptr_t)key_cols[c] & 15u) == 0u;
    }
    k.n = n_keys;
    k.fast16 = fast ? 1 : 0;
    return k;
}

// mark + scan into `table`; the group count lands in *dn (device)
cudaError_t group_table_async(const KeyCols& k, int total, int64_t rows, int32_t* table, int32_t* dn, u32* bits,
                              void* group_keys, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(bits, 0, kKeyWords * 4, s);
    if (e != cudaSuccess) return e;
    if (rows > 0) {
        const int sms = std::max(1, sm_count_current());
        const int64_t work = k.fast16 ? (rows + 15) / 16 : rows;
        const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)sms * 8));
        k_mark_keys<<<(unsigned)blocks, 256, 0, s>>>(k, rows, bits);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    k_scan_keys<<<1, 1024, 0, s>>>(bits, table, dn, (u8*)group_keys, total);
    return cudaGetLastError();
}

}  // namespace

// The key table: kTableKeys forward entries (key -> id), kTableKeys entries
// of the id -> key list, then the group count at entry kTableCount.
constexpr int kTableKeys = 65536;
constexpr int kTableCount = 2 * kTableKeys;
constexpr int kTableEntries = kTableCount + 16;

cudaError_t launch_group_table_small_keys_async(const void* const* key_cols, const int32_t* key_bytes,
                                                int32_t n_keys, int64_t rows, int32_t* table, void* group_keys,
                                                cudaStream_t s) {
    int total = 0;
    const KeyCols k = key_cols_of(key_cols, key_bytes, n_keys, &total);
    void* scratch = nullptr;
    cudaError_t e = cudaMallocAsync(&scratch, kKeyWords * 4, s);
    if (e != cudaSuccess) return e;
    e = group_table_async(k, total, rows, table, table + kTableCount, (u32*)scratch, group_keys, s);
    const cudaError_t e2 = cudaFreeAsync(scratch, s);
    return e != cudaSuccess ? e : e2;
}

cudaError_t launch_group_table_small_keys(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                                          int64_t rows, int32_t* table, int32_t* n_groups, void* group_keys,
                                          cudaStream_t s) {
    cudaError_t e = launch_group_table_small_keys_async(key_cols, key_bytes, n_keys, rows, table, group_keys, s);
    int32_t hn = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hn, table + kTableCount, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) *n_groups = hn;
    return e;
}

cudaError_t launch_group_ids_small_keys(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                                        int64_t rows, int32_t* gid, int32_t* n_groups, void* group_keys,
                                        cudaStream_t s) {
    int total = 0;
    const KeyCols k = key_cols_of(key_cols, key_bytes, n_keys, &total);
    void* scratch = nullptr;
    // a whole key table (forward entries, id -> key list, count), then the bitmap
    cudaError_t e = cudaMallocAsync(&scratch, (size_t)kTableEntries * 4 + kKeyWords * 4, s);
    if (e != cudaSuccess) return e;
    int32_t* table = (int32_t*)scratch;
    u32* bits = (u32*)((u8*)scratch + (size_t)kTableEntries * 4);
    int32_t* dn = table + kTableCount;
    e = group_table_async(k, total, rows, table, dn, bits, group_keys, s);
    if (e == cudaSuccess && rows > 0) {
        const int sms = std::max(1, sm_count_current());
        const int64_t blocks = std::min<int64_t>((rows + 255) / 256, (int64_t)sms * 8);
        k_map_keys<<<(unsigned)blocks, 256, 0, s>>>(k, rows, table, gid);
        e = cudaGetLastError();
    }
    int32_t hn = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hn, dn, 4, cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(scratch, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) *n_groups = hn;
    return e;
}

// ---------------------------------------------------------- utilities
__device__ __forceinline__ u64 splitmix64(u64 x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

constexpr int kGenMaxLimbs = 160;  // p up to ~1500 digits

__global__ void k_gen_digits(u8* __restrict__ out, int64_t rows, int p, int bytes, u64 seed, int signed_,
                             int nonzero) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int L = (bytes + 3) / 4;
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += stride) {
        u32 m[kGenMaxLimbs];
        u64 st = seed ^ ((u64)row * 0xd1b54a32d192ed03ull);
        u32 sign = 0;
        for (int attempt = 0; attempt < 64; attempt++) {
            for (int i = 0; i < L; i++) m[i] = 0;
            int left = p;
            bool nz = false;
            while (left > 0) {
                const int d = left >= 9 ? 9 : left;
                left -= d;
                u32 pw = 1;
                for (int j = 0; j < d; j++) pw *= 10u;
                st = splitmix64(st);
                const u32 chunk = (u32)(((unsigned __int128)st * pw) >> 64);
                nz |= chunk != 0;
                u64 c = chunk;
                for (int i = 0; i < L; i++) {
                    u64 t = (u64)m[i] * pw + c;
                    m[i] = (u32)t;
                    c = t >> 32;
                }
            }
            st = splitmix64(st);
            sign = signed_ ? (u32)(st >> 63) : 0u;
            if (!nonzero || nz) break;
        }
        u8* o = out + row * bytes;
        for (int i = 0; i < bytes; i++) o[i] = (u8)(m[i / 4] >> (8 * (i % 4)));
        o[bytes - 1] |= (u8)(sign << 7);
    }
}

__global__ void k_gen_range(u8* __restrict__ out, int64_t rows, int bytes, long long lo, u64 n, long long step,
                            u64 seed) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += stride) {
        const u64 r = splitmix64(seed ^ ((u64)row * 0xd1b54a32d192ed03ull));
        const u64 idx = (u64)(((unsigned __int128)r * n) >> 64);
        const long long v = lo + (long long)idx * step;
        const u64 mag = v < 0 ? (u64)(-(v + 1)) + 1u : (u64)v;
        u8* o = out + row * bytes;
        for (int i = 0; i < bytes; i++) o[i] = i < 8 ? (u8)(mag >> (8 * i)) : 0;
        o[bytes - 1] |= (u8)((v < 0 ? 1u : 0u) << 7);
    }
}

__global__ void k_flush(uint4* __restrict__ buf, int64_t n, u32 salt) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        buf[i] = make_uint4(salt, (u32)i, salt ^ 1u, (u32)(i >> 32));
}

// The limb multiply-add (32 x 32 -> 64 plus a 64-bit addend, one wide
// integer multiply-add instruction) at full rate: 8 independent chains per
// thread and nothing else in the loop.  Each step multiplies by the high word
// of its own accumulator, so the recurrence is not affine (the loop cannot be
// folded into a closed form) and needs no instruction besides the
// multiply-add itself.
__global__ void __launch_bounds__(256) k_imad(u64* __restrict__ sink, int iters, u32 seed) {
    u32 x[8];
    u64 acc[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        x[k] = (seed * (threadIdx.x + 1u) + 977u * k) | 1u;
        acc[k] = ((u64)(seed + k) << 32) | (threadIdx.x * 31u + k);
    }
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) acc[k] = (u64)x[k] * (u32)(acc[k] >> 32) + acc[k];
    }
    u64 s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s ^= acc[k];
    if (s == 0x123456789ull) sink[0] = s;
}

// The bounded wait of the bulk-copy pipelines, made to run out: an mbarrier
// armed for `bytes` of transfer that nothing ever sends (no copy is issued),
// waited on with `polls` polls by the same code the tile kernels use; the
// timeout is reported the way they report it (ERR_TIMEOUT in the error word).
// Nothing is left in flight: the barrier lives in this block's shared memory.
__global__ void k_wait_timeout_probe(u32 polls, u32 bytes, u32* __restrict__ err_word,
                                     u32* __restrict__ done_word) {
    __shared__ __align__(8) u64 bar;
    if (threadIdx.x == 0) {
        up::mbar_init(&bar, 1);
        up::mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0) up::mbar_expect_tx(&bar, bytes);
    __syncthreads();
    const bool ok = up::mbar_wait(&bar, 0u, polls);
    const bool all_timed_out = __syncthreads_and(!ok);
    if (threadIdx.x == 0) {
        if (all_timed_out) atomicOr(err_word, up::ERR_TIMEOUT);
        atomicAdd(done_word, 1u);
    }
}

}  // namespace upi

using namespace upi;

extern "C" {

up_status up_util_wait_timeout_probe(uint32_t polls, uint32_t* err_word, uint32_t* done_word, void* stream) {
    if (!err_word || !done_word) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    if (polls == 0 || polls > (1u << 24)) return fail(UP_ERR_INVALID_ARG, "polls must be 1 .. 2^24");
    k_wait_timeout_probe<<<1, 32, 0, (cudaStream_t)stream>>>(polls, 256u, err_word, done_word);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? UP_OK : fail(UP_ERR_CUDA, cudaGetErrorString(e));
}

up_status up_util_gen_digits(void* out, int64_t rows, int32_t precision, uint64_t seed, int32_t signed_,
                             int32_t nonzero, void* stream) {
    const int b = compact_bytes(precision);
    if (b < 1 || (b + 3) / 4 > kGenMaxLimbs) return fail(UP_ERR_INVALID_ARG, "precision out of generator range");
    if (rows < 0 || (rows > 0 && !out)) return fail(UP_ERR_INVALID_ARG, "bad output");
    if (rows == 0) return UP_OK;
    int64_t blocks = std::min<int64_t>((rows + 127) / 128, 148 * 16);
    k_gen_digits<<<(unsigned)blocks, 128, 0, (cudaStream_t)stream>>>((u8*)out, rows, precision, b, seed, signed_,
                                                                      nonzero);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? UP_OK : fail(UP_ERR_CUDA, cudaGetErrorString(e));
}

up_status up_util_gen_range(void* out, int64_t rows, int32_t precision, int64_t lo, int64_t hi, int64_t step,
                            uint64_t seed, void* stream) {
    const int b = compact_bytes(precision);
    if (b < 1 || step <= 0 || hi < lo) return fail(UP_ERR_INVALID_ARG, "bad range");
    if (rows < 0 || (rows > 0 && !out)) return fail(UP_ERR_INVALID_ARG, "bad output");
    if (rows == 0) return UP_OK;
    const u64 n = (u64)((hi - lo) / step) + 1u;
    int64_t blocks = std::min<int64_t>((rows + 255) / 256, 148 * 16);
    k_gen_range<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>((u8*)out, rows, b, lo, n, step, seed);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? UP_OK : fail(UP_ERR_CUDA, cudaGetErrorString(e));
}

up_status up_util_flush_l2(void* buf, int64_t bytes, void* stream) {
    if (!buf || bytes < 16) return fail(UP_ERR_INVALID_ARG, "bad buffer");
    static u32 salt = 1;
    k_flush<<<148 * 4, 256, 0, (cudaStream_t)stream>>>((uint4*)buf, bytes / 16, salt++);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? UP_OK : fail(UP_ERR_CUDA, cudaGetErrorString(e));
}

up_status up_util_imad_peak(double* madds_per_s, void* stream) {
    if (!madds_per_s) return fail(UP_ERR_INVALID_ARG, "NULL result");
    cudaStream_t s = (cudaStream_t)stream;
    int sms = sm_count_current();
    if (sms <= 0) return fail(UP_ERR_NO_DEVICE, "no CUDA device");
    u64* sink = nullptr;
    if (cudaMallocAsync((void**)&sink, 8, s) != cudaSuccess) return fail(UP_ERR_NO_MEMORY, "sink");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    k_imad<<<blocks, threads, 0, s>>>(sink, 64, 7u);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(a, s);
        k_imad<<<blocks, threads, 0, s>>>(sink, iters, 11u + rep);
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFreeAsync(sink, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(UP_ERR_CUDA, cudaGetErrorString(e));
    *madds_per_s = (double)blocks * threads * 8.0 * iters / (best * 1e-3);
    return UP_OK;
}

}  // extern "C"
