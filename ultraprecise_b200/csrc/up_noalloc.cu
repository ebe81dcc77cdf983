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
// array below, so the call allocates nothing.  It runs the launch path of
// up_query_launch with that array as its scratch: the same column checks and
// the same kernels (the staged tile kernels with register, shared-memory or
// global accumulators for contiguous columns; the generic kernel otherwise).
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
//   * every call looks up the array's device address in the current context
//     (cudaGetSymbolAddress, which also loads this library's module there the
//     first time); make the first call on a device before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "../../include/ultraprecise.h"
#include "up_internal.h"

namespace upi {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Device address of g_noalloc_scratch in the current context, looked up on
// every call (cheap), so that a reset device or another context never sees a
// stale address.  In host code the symbol's name is a host-side stand-in,
// never a device address.
up_status noalloc_scratch(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? UP_ERR_NO_DEVICE : UP_ERR_CUDA,
                    std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
    }
    *out = p;
    return UP_OK;
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
    const size_t need = query_scratch_bytes(m->jm.gen, n_groups);
    if (need > kNoAllocScratchBytes)
        return fail(UP_ERR_INVALID_ARG, "no-alloc scratch too small: " + std::to_string(n_groups) + " groups need " +
                                            std::to_string(need) + " bytes, the static array holds " +
                                            std::to_string(kNoAllocScratchBytes));
    void* scratch = nullptr;
    up_status st = noalloc_scratch(&scratch);
    if (st != UP_OK) return st;
    // the launch path of up_query_launch (same column checks, same choice of
    // the staged tile kernels or the generic one) over the static array
    return query_launch_ex(m, in, n_in, rows, group_ids, n_groups, outs, err_word, stream, false, nullptr, scratch,
                           kNoAllocScratchBytes);
}
