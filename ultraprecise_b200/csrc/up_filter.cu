// up_filter.cu — row selection from a boolean column (the reference's
// FilterFlags / FilterAssociated, AriesSqlOperator_filter.h:15-19): the
// indices of the rows whose flag byte is nonzero, in row order.
//
// Three launches: every block of kTile rows counts its selected rows; one
// block scans the counts into starting offsets (and writes the total); every
// block then writes its rows' indices at its offset, ordered inside the block
// by warp ballots.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/ultraprecise.h"
#include "up_internal.h"

namespace upi {
namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 16;
constexpr int kTile = kThreads * kPerThread;  // rows per block

__global__ void __launch_bounds__(kThreads) k_count_flags(const uint8_t* __restrict__ flags, int64_t rows,
                                                          int32_t* __restrict__ counts) {
    const int64_t base = (int64_t)blockIdx.x * kTile;
    int c = 0;
    for (int k = 0; k < kPerThread; k++) {
        const int64_t r = base + (int64_t)k * kThreads + threadIdx.x;
        c += (r < rows && flags[r] != 0) ? 1 : 0;
    }
    __shared__ int part[kThreads / 32];
    c = __reduce_add_sync(0xffffffffu, (unsigned)c);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kThreads / 32; w++) s += part[w];
        counts[blockIdx.x] = s;
    }
}

// one block: exclusive scan of n counts into offsets, total into *count
__global__ void __launch_bounds__(1024) k_scan_counts(const int32_t* __restrict__ counts, int64_t n,
                                                      int64_t* __restrict__ offsets, int64_t* __restrict__ count) {
    __shared__ int64_t buf[1024];
    int64_t carry = 0;
    for (int64_t base = 0; base < n; base += 1024) {
        const int64_t i = base + threadIdx.x;
        const int64_t v = i < n ? counts[i] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const int64_t t = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < n) offsets[i] = carry + buf[threadIdx.x] - v;
        const int64_t chunk = buf[1023];
        __syncthreads();
        carry += chunk;
    }
    if (threadIdx.x == 0) *count = carry;
}

__global__ void __launch_bounds__(kThreads) k_scatter_flags(const uint8_t* __restrict__ flags, int64_t rows,
                                                            const int64_t* __restrict__ offsets,
                                                            int32_t* __restrict__ indices) {
    __shared__ int wsum[kThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kTile;
    int64_t at = offsets[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < kPerThread; k++) {
        const int64_t r = base + (int64_t)k * kThreads + threadIdx.x;
        const bool sel = r < rows && flags[r] != 0;
        const unsigned m = __ballot_sync(0xffffffffu, sel);
        if (lane == 0) wsum[warp] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < kThreads / 32; w++) {
            before += w < warp ? wsum[w] : 0;
            total += wsum[w];
        }
        if (sel) indices[at + before + __popc(m & ((1u << lane) - 1u))] = (int32_t)r;
        at += total;
        __syncthreads();
    }
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
    k_count_flags<<<(unsigned)nb, kThreads, 0, s>>>(flags, rows, counts);
    k_scan_counts<<<1, 1024, 0, s>>>(counts, nb, offsets, count);
    k_scatter_flags<<<(unsigned)nb, kThreads, 0, s>>>(flags, rows, offsets, indices);
    e = cudaGetLastError();
    cudaFreeAsync(scratch, s);
    if (e != cudaSuccess)
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? UP_ERR_NO_DEVICE : UP_ERR_CUDA,
                    std::string("filter launch: ") + cudaGetErrorString(e));
    return UP_OK;
}

}  // extern "C"
