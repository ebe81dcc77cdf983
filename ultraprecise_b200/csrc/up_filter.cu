// up_filter.cu — row selection from a boolean column (the reference's
// FilterFlags / FilterAssociated, AriesSqlOperator_filter.h:15-19): the
// indices of the rows whose flag byte is nonzero, in row order.
//
// Three launches: every block of kTile rows counts its selected rows (16
// flags per thread from one 16-byte load); one block scans the counts into
// starting offsets (and writes the total); every block then ranks its kept
// rows by a block scan, stages their indices in shared memory in row order and
// stores them contiguously at its offset.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/ultraprecise.h"
#include "up_internal.h"

namespace upi {
namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 16;                // one 16-byte load of flags
constexpr int kTile = kThreads * kPerThread;  // rows per block

// number of nonzero bytes of w
__device__ __forceinline__ int nonzero_bytes(uint32_t w) {
    w |= w >> 4;
    w |= w >> 2;
    w |= w >> 1;
    return __popc(w & 0x01010101u);
}

// the 16 flags of thread t of block b as a 16-bit mask (bit j = row 16t+j kept)
__device__ __forceinline__ uint32_t thread_mask(const uint8_t* __restrict__ flags, int64_t rows, int64_t row0,
                                                bool vec) {
    uint32_t m = 0u;
    if (vec && row0 + kPerThread <= rows) {
        const uint4 v = *(const uint4*)(flags + row0);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) m |= (((w[i] >> (8 * j)) & 0xffu) != 0u ? 1u : 0u) << (4 * i + j);
    } else {
        for (int j = 0; j < kPerThread; j++)
            if (row0 + j < rows && flags[row0 + j] != 0) m |= 1u << j;
    }
    return m;
}

// exclusive scan of v over the block (256 threads); *total receives the sum
__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    int before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; w++) {
        const int ws = warp_sums[w];
        before += w < warp ? ws : 0;
        all += ws;
    }
    *total = all;
    return before + x - v;
}

__global__ void __launch_bounds__(kThreads) k_count_flags(const uint8_t* __restrict__ flags, int64_t rows, int vec,
                                                          int32_t* __restrict__ counts) {
    const int64_t row0 = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kPerThread;
    int c = 0;
    if (vec && row0 + kPerThread <= rows) {
        const uint4 v = *(const uint4*)(flags + row0);
        c = nonzero_bytes(v.x) + nonzero_bytes(v.y) + nonzero_bytes(v.z) + nonzero_bytes(v.w);
    } else {
        for (int j = 0; j < kPerThread; j++) c += (row0 + j < rows && flags[row0 + j] != 0) ? 1 : 0;
    }
    __shared__ int part[kThreads / 32];
    c = (int)__reduce_add_sync(0xffffffffu, (unsigned)c);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kThreads / 32; w++) s += part[w];
        counts[blockIdx.x] = s;
    }
}

// one block of 1024 threads: exclusive scan of n counts into offsets (each
// thread owns a contiguous chunk), total into *count
__global__ void __launch_bounds__(1024) k_scan_counts(const int32_t* __restrict__ counts, int64_t n,
                                                      int64_t* __restrict__ offsets, int64_t* __restrict__ count) {
    __shared__ int64_t warp_sums[32];
    const int64_t per = (n + 1023) / 1024;
    const int64_t lo = (int64_t)threadIdx.x * per, hi = lo + per < n ? lo + per : n;
    int64_t local = 0;
    for (int64_t i = lo; i < hi; i++) local += counts[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    int64_t before = 0;
    for (int w = 0; w < warp; w++) before += warp_sums[w];
    int64_t run = before + x - local;
    for (int64_t i = lo; i < hi; i++) {
        offsets[i] = run;
        run += counts[i];
    }
    if (threadIdx.x == 1023) *count = before + x;
}

// every block: its kept rows' indices in row order, staged in shared memory
// and stored contiguously at the block's offset
__global__ void __launch_bounds__(kThreads) k_scatter_flags(const uint8_t* __restrict__ flags, int64_t rows, int vec,
                                                            const int64_t* __restrict__ offsets,
                                                            int32_t* __restrict__ indices) {
    __shared__ int32_t sidx[kTile];
    __shared__ int warp_sums[kThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kTile;
    const int64_t row0 = base + (int64_t)threadIdx.x * kPerThread;
    uint32_t m = thread_mask(flags, rows, row0, vec != 0);
    int total = 0;
    int pos = block_exclusive_scan(__popc(m), warp_sums, &total);
    while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1u;
        sidx[pos++] = (int32_t)(row0 + j);
    }
    __syncthreads();
    int32_t* dst = indices + offsets[blockIdx.x];
    for (int i = threadIdx.x; i < total; i += kThreads) dst[i] = sidx[i];
}

}  // namespace
}  // namespace upi

using namespace upi;

extern "C" {

up_status up_filter_flags(const uint8_t* flags, int64_t rows, int32_t* indices, int64_t* count, void* stream) {
    if (rows < 0 || rows > INT32_MAX) return fail(UP_ERR_INVALID_ARG, "0 <= rows <= 2^31-1");
    if (!count || (rows > 0 && (!flags || !indices))) return fail(UP_ERR_INVALID_ARG, "NULL buffers");
    cudaStream_t s = (cudaStream_t)stream;
    if (rows == 0) {
        cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int64_t), s);
        return e == cudaSuccess ? UP_OK : fail(UP_ERR_CUDA, std::string("memset: ") + cudaGetErrorString(e));
    }
    const int64_t nb = (rows + kTile - 1) / kTile;
    void* scratch = nullptr;
    cudaError_t e = cudaMallocAsync(&scratch, (size_t)nb * (sizeof(int32_t) + sizeof(int64_t)) + 16, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? UP_ERR_NO_MEMORY : UP_ERR_CUDA,
                    std::string("filter scratch: ") + cudaGetErrorString(e));
    }
    int64_t* offsets = (int64_t*)scratch;
    int32_t* counts = (int32_t*)((uint8_t*)scratch + (size_t)nb * sizeof(int64_t));
    const int vec = ((uintptr_t)flags & 15u) == 0u ? 1 : 0;
    k_count_flags<<<(unsigned)nb, kThreads, 0, s>>>(flags, rows, vec, counts);
    k_scan_counts<<<1, 1024, 0, s>>>(counts, nb, offsets, count);
    k_scatter_flags<<<(unsigned)nb, kThreads, 0, s>>>(flags, rows, vec, offsets, indices);
    e = cudaGetLastError();
    cudaFreeAsync(scratch, s);
    if (e != cudaSuccess)
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? UP_ERR_NO_DEVICE : UP_ERR_CUDA,
                    std::string("filter launch: ") + cudaGetErrorString(e));
    return UP_OK;
}

}  // extern "C"
