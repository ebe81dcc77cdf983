// up_noalloc.cu — the grouped-aggregate launch for callers that cannot
// allocate device memory.
//
// up_query_launch obtains its accumulator scratch with cudaMallocAsync.  Some
// callers cannot allocate at launch time: code running inside another
// runtime's memory budget (a database or an inference server that owns every
// device allocation and forbids allocations behind its back), callers on a
// hot path that must never touch the allocator, or callers that pre-plan all
// device memory up front.  up_query_launch_noalloc serves them: the same two
// kernels (accumulate, finalize) run with their scratch in the file-scope
// array below, so the call allocates nothing.
//
// Limits and sharing:
//   * the array is kNoAllocScratchBytes (8 MiB); a request whose accumulators
//     (n_groups x accumulator words x 4 bytes, 16-byte padded, plus 8 bytes of
//     count per group) do not fit is rejected with UP_ERR_INVALID_ARG;
//   * every GPU that loads this library holds the array until the process
//     exits;
//   * every call shares the array and it keeps the previous call's contents:
//     each call clears the bytes it uses (cudaMemsetAsync on the caller's
//     stream) before accumulating; two calls whose work overlaps on the GPU
//     (different streams, no ordering between them) race on the array and
//     give wrong results — order them on one stream or with events;
//   * the first call on a device looks up the array's device address for that
//     device (cudaGetSymbolAddress, which also loads this library's module on
//     that device if it is not loaded yet); make that first call before any
//     stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/ultraprecise.h"
#include "up_internal.h"

namespace upi {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices];

// Device address of g_noalloc_scratch on the current device, looked up once
// per device with that device current.  In host code the symbol's name is a
// host-side stand-in, never a device address.
up_status noalloc_scratch(void** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(UP_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    }
    if (dev < 0 || dev >= kMaxDevices) return fail(UP_ERR_UNSUPPORTED, "device index above 63");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(UP_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                         cudaGetErrorString(e));
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return UP_OK;
}

// Kernel argument block of the generated query kernels (UpQArgs).
struct NaCol {
    const void* data;
    const void* const* blocks;
    const int64_t* prefix;
    const int32_t* indices;
    int32_t n_blocks;
    int32_t value_bytes;
};
struct NaQArgs {
    NaCol col[16];
    uint8_t* out[16];
    int64_t rows;
    const int32_t* gid;
    uint32_t* acc;
    uint64_t* cnt;
    uint32_t* err;
    int32_t n_groups;
    int32_t vec_ok;
    const uint8_t* key0;  // key modes are not used here (group ids only)
    const uint8_t* key1;
    const int32_t* key_table;
    int32_t key_mode;
};
static_assert(sizeof(NaQArgs) == 848, "UpQArgs layout");

up_status na_cuda(cudaError_t e, const char* what) {
    cudaGetLastError();
    return fail(UP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace upi

using namespace upi;

extern "C" up_status up_query_launch_noalloc(up_module* m, const up_column* in, int32_t n_in, int64_t rows,
                                             const int32_t* group_ids, int32_t n_groups, void* const* outs,
                                             uint32_t* err_word, void* stream) {
    if (!m || !m->is_query) return fail(UP_ERR_INVALID_ARG, "not a query module");
    if (rows < 0 || n_groups < 0) return fail(UP_ERR_INVALID_ARG, "negative size");
    if (n_groups == 0) return UP_OK;
    if (rows > 0 && !group_ids) return fail(UP_ERR_INVALID_ARG, "group ids are NULL");
    if (!outs) return fail(UP_ERR_INVALID_ARG, "outputs are NULL");
    const GeneratedModule& g = m->jm.gen;
    if ((int)g.in_bytes.size() > n_in || n_in > 16 || (n_in > 0 && !in))
        return fail(UP_ERR_INVALID_ARG, "input columns do not match the compiled query");
    const size_t accw = (size_t)std::max(g.acc_words_per_group, 1);
    const size_t acc_bytes = (((size_t)n_groups * accw * 4u) + 15u) & ~(size_t)15u;
    const size_t need = acc_bytes + (size_t)n_groups * 8u;
    if (need > kNoAllocScratchBytes)
        return fail(UP_ERR_INVALID_ARG, "no-alloc scratch too small: " + std::to_string(n_groups) + " groups need " +
                                            std::to_string(need) + " bytes, the static array holds " +
                                            std::to_string(kNoAllocScratchBytes));
    NaQArgs a;
    memset(&a, 0, sizeof a);
    for (int c = 0; c < (int)g.in_bytes.size(); c++) {
        const up_column& col = in[c];
        if (col.value_bytes != g.in_bytes[c]) return fail(UP_ERR_INVALID_ARG, "column width differs from compiled");
        if (!col.data && col.n_blocks <= 0) return fail(UP_ERR_INVALID_ARG, "column has neither data nor blocks");
        if (col.n_blocks > 0 && (!col.blocks || !col.block_prefix))
            return fail(UP_ERR_INVALID_ARG, "block column without block arrays");
        a.col[c] = {col.data, col.blocks, col.block_prefix, col.indices, col.n_blocks > 0 ? col.n_blocks : 0,
                    col.value_bytes};
    }
    for (int k = 0; k < g.n_aggs; k++) {
        if (!outs[k]) return fail(UP_ERR_INVALID_ARG, "output is NULL");
        a.out[k] = (uint8_t*)outs[k];
    }
    void* scratch = nullptr;
    up_status st = noalloc_scratch(&scratch);
    if (st != UP_OK) return st;
    const int sms = sm_count_current();
    if (sms <= 0) return fail(UP_ERR_NO_DEVICE, "no CUDA device");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(scratch, 0, need, s);
    if (e != cudaSuccess) return na_cuda(e, "cudaMemsetAsync(no-alloc scratch)");
    a.rows = rows;
    a.gid = group_ids;
    a.acc = (uint32_t*)scratch;
    a.cnt = (uint64_t*)((uint8_t*)scratch + acc_bytes);
    a.err = err_word;
    a.n_groups = n_groups;
    a.vec_ok = 0;
    void* args[1] = {&a};
    if (rows > 0) {
        void* k = jit_kernel(*m->jm.ks, "up_query_acc");
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)k, g.block_threads, 0) != cudaSuccess) {
            cudaGetLastError();
            occ = 1;
        }
        const int64_t blocks = (rows + g.block_threads - 1) / g.block_threads;
        const int64_t cap = (int64_t)sms * std::max(occ, 1) * 4;
        e = cudaLaunchKernel((const void*)k, dim3((unsigned)std::min<int64_t>(blocks, cap)), dim3(g.block_threads),
                             args, 0, s);
        if (e != cudaSuccess) return na_cuda(e, "up_query_acc");
    }
    void* k = jit_kernel(*m->jm.ks, "up_query_fin");
    e = cudaLaunchKernel((const void*)k, dim3((unsigned)((n_groups + 255) / 256)), dim3(256), args, 0, s);
    if (e != cudaSuccess) return na_cuda(e, "up_query_fin");
    return UP_OK;
}
