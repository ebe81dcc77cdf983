// up_abi.cpp — the C entry points of libultraprecise.so (include/ultraprecise.h).
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ultraprecise_util.h"
#include "up_internal.h"
#include "up_kernels.h"

using namespace upi;

namespace {

// The kernels' argument blocks (UpKCol, UpArgs, UpQArgs) come from
// up_kargs.h, the header the generated kernels include as well.
constexpr int kMaxCols = UP_MAX_COLS;
constexpr int kMaxAggs = UP_MAX_AGGS;
using HKCol = UpKCol;
using HUpArgs = UpArgs;
using HUpQArgs = UpQArgs;

up_status cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    up_status s = (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? UP_ERR_NO_DEVICE
                  : (e == cudaErrorMemoryAllocation)                           ? UP_ERR_NO_MEMORY
                                                                               : UP_ERR_CUDA;
    return fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define UP_CUDA(call)                                  \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

struct ModCols {
    std::vector<up_col_type> cols;
};

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

up_status check_columns(const up_module* m, const up_column* in, int n_in, HKCol* kc, bool& all_contig,
                        bool& vec_ok) {
    const GeneratedModule& g = m->jm.gen;
    if ((int)g.in_bytes.size() > n_in) return fail(UP_ERR_INVALID_ARG, "fewer input columns than compiled");
    if (n_in > kMaxCols) return fail(UP_ERR_INVALID_ARG, "at most 16 input columns");
    all_contig = true;
    vec_ok = true;
    for (int c = 0; c < (int)g.in_bytes.size(); c++) {
        const up_column& col = in[c];
        if (col.value_bytes != g.in_bytes[c])
            return fail(UP_ERR_INVALID_ARG, "column " + std::to_string(c) + ": value_bytes " +
                                                std::to_string(col.value_bytes) + " != compiled " +
                                                std::to_string(g.in_bytes[c]));
        if (!col.data && col.n_blocks <= 0) return fail(UP_ERR_INVALID_ARG, "column has neither data nor blocks");
        if (col.n_blocks > 0 && (!col.blocks || !col.block_prefix))
            return fail(UP_ERR_INVALID_ARG, "block column without block arrays");
        kc[c].data = (const unsigned char*)col.data;
        kc[c].blocks = (const unsigned char* const*)col.blocks;
        kc[c].prefix = (const long long*)col.block_prefix;
        kc[c].indices = col.indices;
        kc[c].n_blocks = col.n_blocks > 0 ? col.n_blocks : 0;
        kc[c].value_bytes = col.value_bytes;
        if (col.n_blocks > 0 || col.indices || col.nullable || !col.data) all_contig = false;
        if (!aligned16(col.data)) vec_ok = false;
    }
    return UP_OK;
}

int occupancy(void* kernel, int threads, int smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, (const void*)kernel, threads, (size_t)smem) != cudaSuccess) {
        cudaGetLastError();
        n = 1;
    }
    return n < 1 ? 1 : n;
}

// Resident CTAs per SM for a tile kernel whose grid loops over tiles: the
// occupancy limit, except for kernels with large per-thread local memory
// (long expressions of wide values keep many limb arrays there), which keep
// at most kLocalHeavyThreads threads per SM.  Measured on B200 with the sin
// series: at p=300 (13 KB of local memory per thread, 128-thread CTAs) two
// CTAs per SM ran in 27 ms, three (the register limit) in 66 ms and one in
// 50 ms; at p=1000 (32-thread CTAs) eight CTAs per SM ran in 418 ms and
// three in 1277 ms.  Kernels with a few KB or less (the divisions) are
// unaffected.
constexpr int kLocalHeavyBytes = 4096;
constexpr int kLocalHeavyThreads = 256;
int resident_ctas(void* kernel, int threads, int smem) {
    int n = occupancy(kernel, threads, smem);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, (const void*)kernel) != cudaSuccess) {
        cudaGetLastError();
        return n;
    }
    if (fa.localSizeBytes >= (size_t)kLocalHeavyBytes) n = std::max(1, std::min(n, kLocalHeavyThreads / threads));
    return n;
}

up_status set_smem(void* kernel, int smem) {
    if (smem > 48 * 1024) {
        UP_CUDA(cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    }
    return UP_OK;
}

}  // namespace

namespace upi {
int sm_count_current() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}
}  // namespace upi

extern "C" {

const char* up_status_string(up_status s) {
    switch (s) {
        case UP_OK: return "ok";
        case UP_ERR_INVALID_ARG: return "invalid argument";
        case UP_ERR_UNSUPPORTED: return "unsupported";
        case UP_ERR_CUDA: return "CUDA error";
        case UP_ERR_COMPILE: return "compile error";
        case UP_ERR_NO_MEMORY: return "out of memory";
        case UP_ERR_TIMEOUT: return "timeout";
        case UP_ERR_QUEUE_FULL: return "queue full";
        case UP_ERR_NOT_READY: return "not ready";
        case UP_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char* up_last_error_message(void) { return last_error(); }
int32_t up_abi_version(void) { return UP_ABI_VERSION; }
int32_t up_compact_bytes(int32_t p) { return compact_bytes(p); }
int32_t up_precision_words(int32_t p) { return precision_words(p); }
int32_t up_max_precision(void) { return kMaxPrecision; }

up_status up_module_compile(const up_expr_node* nodes, int32_t n_nodes, int32_t root, const up_col_type* cols,
                            int32_t n_cols, const up_compile_opts* opts, up_module** out) {
    if (!out) return fail(UP_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    GeneratedModule gen;
    up_status st = generate_expr_module(nodes, n_nodes, root, cols, n_cols, opts, gen);
    if (st != UP_OK) return st;
    std::shared_ptr<JitKernelSet> ks;
    st = jit_get(gen, ks);
    if (st != UP_OK) return st;
    up_module* m = new up_module();
    m->jm.ks = ks;
    m->jm.gen = std::move(gen);
    m->is_query = false;
    *out = m;
    return UP_OK;
}

int32_t up_module_threads_per_value(const up_module* m) { return m ? m->jm.gen.threads_per_value : 0; }

up_status up_expr_launch_many(up_module* m, const up_column* in, int32_t n_in, const int64_t* rows, int32_t n_req,
                              void* const* outs, uint32_t* const* errs, void* stream) {
    if (!m || m->is_query) return fail(UP_ERR_INVALID_ARG, "not an expression module");
    if (n_req < 0 || (n_req > 0 && (!rows || !outs || (n_in > 0 && !in))))
        return fail(UP_ERR_INVALID_ARG, "bad request arrays");
    const GeneratedModule& g = m->jm.gen;
    std::vector<UpMultiReq> reqs;
    std::vector<int> alone;
    long long tiles = 0;
    for (int k = 0; k < n_req; k++) {
        if (rows[k] < 0) return fail(UP_ERR_INVALID_ARG, "negative row count");
        if (rows[k] == 0) continue;
        if (!outs[k]) return fail(UP_ERR_INVALID_ARG, "output is NULL");
        UpMultiReq q;
        memset(&q, 0, sizeof q);
        bool contig = true, vec_ok = true;
        up_status st = check_columns(m, in + (size_t)k * n_in, n_in, q.col, contig, vec_ok);
        if (st != UP_OK) return st;
        if (g.multi_rows == 0 || !contig) {
            alone.push_back(k);
            continue;
        }
        q.rows = rows[k];
        q.out = (unsigned char*)outs[k];
        q.err = errs ? errs[k] : nullptr;
        q.tile0 = tiles;
        q.vec_ok = (vec_ok && aligned16(outs[k])) ? 1 : 0;
        tiles += (rows[k] + g.multi_rows - 1) / g.multi_rows;
        reqs.push_back(q);
    }
    cudaStream_t s = (cudaStream_t)stream;
    for (int k : alone) {
        up_status st = expr_launch_ex(m, in + (size_t)k * n_in, n_in, rows[k], outs[k], errs ? errs[k] : nullptr,
                                      stream, false);
        if (st != UP_OK) return st;
    }
    if (reqs.empty()) return UP_OK;
    const int sms = sm_count_current();
    if (sms <= 0) return fail(UP_ERR_NO_DEVICE, "no CUDA device");
    void* k = jit_kernel(*m->jm.ks, "up_expr_multi");
    if (!k) return fail(UP_ERR_CUDA, "module has no up_expr_multi kernel");
    up_status st = set_smem(k, g.multi_smem);
    if (st != UP_OK) return st;
    UpMultiReq* d = nullptr;
    const size_t bytes = reqs.size() * sizeof(UpMultiReq);
    UP_CUDA(cudaMallocAsync((void**)&d, bytes, s));
    cudaError_t e = cudaMemcpyAsync(d, reqs.data(), bytes, cudaMemcpyHostToDevice, s);
    UpMultiArgs a;
    memset(&a, 0, sizeof a);
    a.req = d;
    a.n_tiles = tiles;
    a.n_req = (int)reqs.size();
    void* args[1] = {&a};
    if (e == cudaSuccess) {
        const int64_t cap = (int64_t)sms * occupancy(k, g.multi_threads, g.multi_smem);
        e = cudaLaunchKernel((const void*)k, dim3((unsigned)std::min<int64_t>(tiles, cap)), dim3(g.multi_threads),
                             args, (size_t)g.multi_smem, s);
    }
    cudaError_t e2 = cudaFreeAsync(d, s);
    if (e != cudaSuccess) return cuda_fail(e, "up_expr_multi");
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaFreeAsync");
    return UP_OK;
}

up_status up_module_result_type(const up_module* m, int32_t* precision, int32_t* scale, int32_t* value_bytes) {
    if (!m) return fail(UP_ERR_INVALID_ARG, "module is NULL");
    if (precision) *precision = m->jm.gen.out_precision;
    if (scale) *scale = m->jm.gen.out_scale;
    if (value_bytes) *value_bytes = m->jm.gen.out_bytes;
    return UP_OK;
}

int64_t up_module_source(const up_module* m, char* buf, int64_t cap) {
    if (!m) return -1;
    const std::string& s = m->jm.gen.source;
    if (buf && cap > 0) {
        int64_t n = std::min<int64_t>(cap - 1, (int64_t)s.size());
        memcpy(buf, s.data(), (size_t)n);
        buf[n] = 0;
    }
    return (int64_t)s.size();
}

void up_module_release(up_module* m) { delete m; }

int32_t up_module_cache_size(int32_t clear) { return jit_cache_size(clear != 0); }

up_status up_expr_launch(up_module* m, const up_column* in, int32_t n_in, int64_t rows, void* out,
                         uint32_t* err_word, void* stream) {
    return expr_launch_ex(m, in, n_in, rows, out, err_word, stream, false);
}

}  // extern "C"

up_status expr_launch_ex(up_module* m, const up_column* in, int32_t n_in, int64_t rows, void* out,
                         uint32_t* err_word, void* stream, bool spread) {
    if (!m || m->is_query) return fail(UP_ERR_INVALID_ARG, "not an expression module");
    if (rows < 0) return fail(UP_ERR_INVALID_ARG, "negative row count");
    if (rows == 0) return UP_OK;
    if (!out) return fail(UP_ERR_INVALID_ARG, "out is NULL");
    if (n_in > 0 && !in) return fail(UP_ERR_INVALID_ARG, "inputs are NULL");
    const GeneratedModule& g = m->jm.gen;
    HUpArgs a;
    memset(&a, 0, sizeof a);
    bool contig = true, vec_ok = true;
    up_status st = check_columns(m, in, n_in, a.col, contig, vec_ok);
    if (st != UP_OK) return st;
    a.rows = rows;
    a.out = (uint8_t*)out;
    a.err = err_word;
    a.out_nullable = g.out_bytes != (g.out_is_compare ? 1 : compact_bytes(g.out_precision));
    vec_ok = vec_ok && aligned16(out);
    a.vec_ok = vec_ok ? 1 : 0;
    const int sms = sm_count_current();
    if (sms <= 0) return fail(UP_ERR_NO_DEVICE, "no CUDA device");
    void* args[1] = {&a};
    cudaStream_t s = (cudaStream_t)stream;
    if (contig && !a.out_nullable) {
        void* k = jit_kernel(*m->jm.ks, "up_expr_tile");
        st = set_smem(k, g.smem_bytes);
        if (st != UP_OK) return st;
        const int64_t ntiles = (rows + g.tile_rows - 1) / g.tile_rows;
        const int64_t cap =
            spread ? (int64_t)INT32_MAX : (int64_t)sms * resident_ctas(k, g.block_threads, g.smem_bytes);
        const unsigned grid = (unsigned)std::min<int64_t>(ntiles, cap);
        UP_CUDA(cudaLaunchKernel((const void*)k, dim3(grid), dim3(g.block_threads), args, (size_t)g.smem_bytes, s));
    } else {
        void* k = jit_kernel(*m->jm.ks, "up_expr_generic");
        const int64_t blocks = (rows + g.block_threads - 1) / g.block_threads;
        const int64_t cap = spread ? (int64_t)INT32_MAX : (int64_t)sms * occupancy(k, g.block_threads, 0) * 4;
        const unsigned grid = (unsigned)std::min<int64_t>(blocks, cap);
        UP_CUDA(cudaLaunchKernel((const void*)k, dim3(grid), dim3(g.block_threads), args, 0, s));
    }
    return UP_OK;
}

extern "C" {


up_status up_expr_launch_host(up_module* m, const up_column* host_in, int32_t n_in, int64_t rows, void* host_out,
                              uint32_t* err_word, int64_t chunk_rows) {
    if (!m || m->is_query) return fail(UP_ERR_INVALID_ARG, "not an expression module");
    if (rows < 0 || chunk_rows < 0) return fail(UP_ERR_INVALID_ARG, "negative size");
    if (err_word) *err_word = 0u;
    if (rows == 0) return UP_OK;
    if (!host_out || (n_in > 0 && !host_in)) return fail(UP_ERR_INVALID_ARG, "NULL buffers");
    const GeneratedModule& g = m->jm.gen;
    const int nc = (int)g.in_bytes.size();
    if (n_in < nc) return fail(UP_ERR_INVALID_ARG, "fewer input columns than compiled");
    int64_t in_row = 0;
    for (int c = 0; c < nc; c++) {
        const up_column& col = host_in[c];
        if (!col.data || col.n_blocks > 0 || col.indices || col.nullable || col.value_bytes != g.in_bytes[c])
            return fail(UP_ERR_INVALID_ARG, "host launch takes contiguous non-null columns of the compiled width");
        in_row += col.value_bytes;
    }
    const int64_t out_row = g.out_bytes;
    if (chunk_rows == 0) chunk_rows = std::max<int64_t>(4096, ((int64_t)64 << 20) / std::max<int64_t>(in_row, 1));
    chunk_rows = std::max<int64_t>(1, std::min(chunk_rows, rows));
    constexpr int NB = HostStaging::kSets;
    const int64_t nchunks = (rows + chunk_rows - 1) / chunk_rows;
    // one buffer set: every input column + the output, 256-byte aligned
    std::vector<int64_t> col_off(nc);
    int64_t set_bytes = 0;
    for (int c = 0; c < nc; c++) {
        col_off[c] = set_bytes;
        set_bytes += (chunk_rows * g.in_bytes[c] + 255) / 256 * 256;
    }
    const int64_t out_off = set_bytes;
    set_bytes += (chunk_rows * out_row + 255) / 256 * 256;
    // the module keeps its staging buffers, streams and events between calls
    std::lock_guard<std::mutex> lk(m->host_mu);
    HostStaging& hs = m->host;
    up_status st = hs.ensure((size_t)(NB * set_bytes + 256));
    if (st != UP_OK) return st;
    cudaError_t e = cudaSuccess;
    uint32_t* derr = (uint32_t*)((uint8_t*)hs.dev + NB * set_bytes);
    e = cudaMemsetAsync(derr, 0, 4, hs.s_k);
    // the previous call finished (it synchronised), so every buffer set is free
    std::vector<up_column> dcol(host_in, host_in + n_in);
    for (int64_t ch = 0; ch < nchunks && e == cudaSuccess && st == UP_OK; ch++) {
        const int b = (int)(ch % NB);
        const int64_t r0 = ch * chunk_rows;
        const int64_t nr = std::min(chunk_rows, rows - r0);
        uint8_t* base = (uint8_t*)hs.dev + b * set_bytes;
        // inputs: this buffer set is free once the kernel of chunk ch-NB has run
        if (ch >= NB) e = cudaStreamWaitEvent(hs.s_in, hs.ev_k[b], 0);
        for (int c = 0; c < nc && e == cudaSuccess; c++) {
            const int64_t w = g.in_bytes[c];
            e = cudaMemcpyAsync(base + col_off[c], (const uint8_t*)host_in[c].data + r0 * w, (size_t)(nr * w),
                                cudaMemcpyHostToDevice, hs.s_in);
            dcol[c].data = base + col_off[c];
        }
        if (e == cudaSuccess) e = cudaEventRecord(hs.ev_in[b], hs.s_in);
        // kernel: after its inputs landed and the copy-out of chunk ch-NB left the output buffer
        if (e == cudaSuccess) e = cudaStreamWaitEvent(hs.s_k, hs.ev_in[b], 0);
        if (e == cudaSuccess && ch >= NB) e = cudaStreamWaitEvent(hs.s_k, hs.ev_out[b], 0);
        if (e == cudaSuccess) st = expr_launch_ex(m, dcol.data(), n_in, nr, base + out_off, derr, hs.s_k, false);
        if (e == cudaSuccess && st == UP_OK) e = cudaEventRecord(hs.ev_k[b], hs.s_k);
        // outputs
        if (e == cudaSuccess && st == UP_OK) e = cudaStreamWaitEvent(hs.s_out, hs.ev_k[b], 0);
        if (e == cudaSuccess && st == UP_OK)
            e = cudaMemcpyAsync((uint8_t*)host_out + r0 * out_row, base + out_off, (size_t)(nr * out_row),
                                cudaMemcpyDeviceToHost, hs.s_out);
        if (e == cudaSuccess && st == UP_OK) e = cudaEventRecord(hs.ev_out[b], hs.s_out);
    }
    uint32_t herr = 0;
    if (e == cudaSuccess && st == UP_OK) {
        e = cudaStreamWaitEvent(hs.s_out, hs.ev_k[(nchunks - 1) % NB], 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, hs.s_out);
    }
    // always leave the staging idle before returning
    const cudaError_t e1 = cudaStreamSynchronize(hs.s_out);
    const cudaError_t e2 = cudaStreamSynchronize(hs.s_k);
    const cudaError_t e3 = cudaStreamSynchronize(hs.s_in);
    if (st != UP_OK) return st;
    for (cudaError_t x : {e, e1, e2, e3})
        if (x != cudaSuccess) return cuda_fail(x, "host launch");
    if (err_word) *err_word = herr;
    return UP_OK;
}

up_status up_query_compile(const up_expr_node* nodes, int32_t n_nodes, const up_col_type* cols, int32_t n_cols,
                           const up_query_agg* aggs, int32_t n_aggs, const up_compile_opts* opts, up_module** out) {
    if (!out) return fail(UP_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    GeneratedModule gen;
    up_status st = generate_query_module(nodes, n_nodes, cols, n_cols, aggs, n_aggs, opts, gen);
    if (st != UP_OK) return st;
    std::shared_ptr<JitKernelSet> ks;
    st = jit_get(gen, ks);
    if (st != UP_OK) return st;
    up_module* m = new up_module();
    m->jm.ks = ks;
    m->jm.gen = std::move(gen);
    m->is_query = true;
    *out = m;
    return UP_OK;
}

up_status up_query_launch(up_module* m, const up_column* in, int32_t n_in, int64_t rows, const int32_t* group_ids,
                          int32_t n_groups, void* const* outs, uint32_t* err_word, void* stream) {
    return query_launch_ex(m, in, n_in, rows, group_ids, n_groups, outs, err_word, stream, false);
}

}  // extern "C"

size_t query_scratch_bytes(const GeneratedModule& g, int32_t n_groups) {
    const size_t accw = (size_t)std::max(g.acc_words_per_group, 1);
    // the int64 counts follow the accumulators: keep them 16-byte aligned
    const size_t acc_bytes = (((size_t)n_groups * accw * 4u) + 15u) & ~(size_t)15u;
    return acc_bytes + (size_t)n_groups * 8u;
}

up_status query_launch_ex(up_module* m, const up_column* in, int32_t n_in, int64_t rows, const int32_t* group_ids,
                          int32_t n_groups, void* const* outs, uint32_t* err_word, void* stream, bool spread,
                          const QueryKeys* keys, void* caller_scratch, size_t caller_scratch_bytes) {
    if (!m || !m->is_query) return fail(UP_ERR_INVALID_ARG, "not a query module");
    const bool device_count = keys && keys->capacity > 0;
    if (device_count) n_groups = keys->capacity;  // accumulators and outputs sized for the capacity
    if (rows < 0 || n_groups < 0) return fail(UP_ERR_INVALID_ARG, "negative size");
    if (n_groups == 0) return UP_OK;
    if (rows > 0 && !keys && !group_ids) return fail(UP_ERR_INVALID_ARG, "group ids are NULL");
    if (!outs) return fail(UP_ERR_INVALID_ARG, "outputs are NULL");
    const GeneratedModule& g = m->jm.gen;
    HUpQArgs a;
    memset(&a, 0, sizeof a);
    bool contig = true, vec_ok = true;
    up_status st = check_columns(m, in, n_in, a.col, contig, vec_ok);
    if (st != UP_OK) return st;
    for (int k = 0; k < g.n_aggs; k++) {
        if (!outs[k]) return fail(UP_ERR_INVALID_ARG, "output " + std::to_string(k) + " is NULL");
        a.out[k] = (uint8_t*)outs[k];
    }
    const int sms = sm_count_current();
    if (sms <= 0) return fail(UP_ERR_NO_DEVICE, "no CUDA device");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t accw = (size_t)std::max(g.acc_words_per_group, 1);
    const size_t acc_bytes = (((size_t)n_groups * accw * 4u) + 15u) & ~(size_t)15u;
    const size_t need = query_scratch_bytes(g, n_groups);
    void* scratch = caller_scratch;
    if (caller_scratch) {
        if (need > caller_scratch_bytes)
            return fail(UP_ERR_INVALID_ARG, "scratch too small: " + std::to_string(n_groups) + " groups need " +
                                                std::to_string(need) + " bytes, " +
                                                std::to_string(caller_scratch_bytes) + " given");
    } else {
        UP_CUDA(cudaMallocAsync(&scratch, need, s));
    }
    cudaError_t e = cudaMemsetAsync(scratch, 0, need, s);
    a.rows = rows;
    a.gid = group_ids;
    a.acc = (uint32_t*)scratch;
    a.cnt = (unsigned long long*)((uint8_t*)scratch + acc_bytes);
    a.err = err_word;
    a.n_groups = device_count ? -n_groups : n_groups;
    a.vec_ok = vec_ok ? 1 : 0;
    bool keys_aligned = aligned16(group_ids);
    if (keys) {
        a.key0 = keys->key0;
        a.key1 = keys->key1;
        a.key_table = keys->table;
        a.key_mode = keys->mode;
        keys_aligned = aligned16(keys->key0) && (keys->mode != 2 || aligned16(keys->key1));
    }
    void* args[1] = {&a};
    if (e == cudaSuccess && rows > 0) {
        if (contig && g.q_staged) {
            // staged tiles; accumulators in registers, shared memory or global
            // memory by group count
            const bool reg = g.q_gr > 0 && n_groups <= g.q_gr;
            const bool reg_lo = g.q_gr_lo > 0 && n_groups <= g.q_gr_lo;
            const char* reg_name = keys ? "up_query_tile_rk" : "up_query_tile_r";
            const char* lo_name = keys ? "up_query_tile_rk_lo" : "up_query_tile_r_lo";
            const char* name = reg_lo ? lo_name : reg ? reg_name : (n_groups <= g.q_gs) ? "up_query_tile_s"
                                                                                        : "up_query_tile_g";
            a.vec_ok = (vec_ok && keys_aligned) ? 1 : 0;
            const int64_t ntiles = (rows + g.q_tile_rows - 1) / g.q_tile_rows;
            auto launch_tile = [&](const char* kname) -> cudaError_t {
                void* k = jit_kernel(*m->jm.ks, kname);
                if (set_smem(k, g.q_smem) != UP_OK) return cudaErrorInvalidValue;  // layout kept within 48 KB
                // the register and shared-memory modes merge once per CTA, so a
                // spread launch keeps a bounded grid of several waves
                const int64_t cap = (int64_t)sms * occupancy(k, g.block_threads, g.q_smem) * (spread ? 8 : 1);
                return cudaLaunchKernel((const void*)k, dim3((unsigned)std::min<int64_t>(ntiles, cap)),
                                        dim3(g.block_threads), args, (size_t)g.q_smem, s);
            };
            if (device_count) {
                // the mode follows the count on the device: every applicable
                // mode kernel is launched and all but one return at once
                if (g.q_gr_lo > 0) e = launch_tile(lo_name);
                if (e == cudaSuccess && g.q_gr > 0 && n_groups > g.q_gr_lo) e = launch_tile(reg_name);
                if (e == cudaSuccess && (g.q_gr == 0 || n_groups > g.q_gr)) e = launch_tile("up_query_tile_s");
                if (e == cudaSuccess && n_groups > g.q_gs) e = launch_tile("up_query_tile_g");
            } else {
                e = launch_tile(name);
            }
        } else {
            void* k = jit_kernel(*m->jm.ks, "up_query_acc");
            const int64_t blocks = (rows + g.block_threads - 1) / g.block_threads;
            const int64_t cap = (int64_t)sms * occupancy(k, g.block_threads, 0) * 4;
            e = cudaLaunchKernel((const void*)k, dim3((unsigned)std::min<int64_t>(blocks, cap)), dim3(g.block_threads),
                                 args, 0, s);
        }
    }
    if (e == cudaSuccess) {
        void* k = jit_kernel(*m->jm.ks, "up_query_fin");
        e = cudaLaunchKernel((const void*)k, dim3((unsigned)((n_groups + 255) / 256)), dim3(256), args, 0, s);
    }
    cudaError_t e2 = caller_scratch ? cudaSuccess : cudaFreeAsync(scratch, s);
    if (e != cudaSuccess) return cuda_fail(e, "query launch");
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaFreeAsync");
    return UP_OK;
}

extern "C" {


up_status up_group_agg(const up_column* vals, const int32_t* kinds, int32_t n_vals, const int32_t* group_ids,
                       int32_t n_groups, int64_t rows, void* const* outs, uint32_t* err_word, void* stream) {
    if (n_vals <= 0 || n_vals > kMaxAggs) return fail(UP_ERR_INVALID_ARG, "1..16 aggregates");
    if (!vals || !kinds) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    std::vector<up_expr_node> nodes(n_vals);
    std::vector<up_col_type> cols(n_vals);
    std::vector<up_query_agg> aggs(n_vals);
    for (int k = 0; k < n_vals; k++) {
        memset(&nodes[k], 0, sizeof(up_expr_node));
        nodes[k].kind = UP_NODE_COLUMN;
        nodes[k].left = nodes[k].right = -1;
        nodes[k].column = k;
        nodes[k].precision = vals[k].precision;
        nodes[k].scale = vals[k].scale;
        cols[k].precision = vals[k].precision;
        cols[k].scale = vals[k].scale;
        cols[k].nullable = vals[k].nullable;
        aggs[k].kind = kinds[k];
        aggs[k].root = k;
    }
    up_module* m = nullptr;
    up_status st = up_query_compile(nodes.data(), n_vals, cols.data(), n_vals, aggs.data(), n_vals, nullptr, &m);
    if (st != UP_OK) return st;
    st = up_query_launch(m, vals, n_vals, rows, group_ids, n_groups, outs, err_word, stream);
    up_module_release(m);
    return st;
}

up_status up_aggregate_column_data(const up_column* src, int32_t kind, const int32_t* associated,
                                   const int32_t* group_starts, int32_t n_groups, int64_t rows, void* out,
                                   uint32_t* err_word, void* stream) {
    if (!src || !out) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    if (n_groups < 0 || rows < 0) return fail(UP_ERR_INVALID_ARG, "negative size");
    if (n_groups == 0) return UP_OK;
    if (rows > 0 && !group_starts) return fail(UP_ERR_INVALID_ARG, "group starts are NULL");
    if (associated && src->indices) return fail(UP_ERR_UNSUPPORTED, "column already has an indirection");
    cudaStream_t s = (cudaStream_t)stream;
    int32_t* gid = nullptr;
    if (rows > 0) {
        UP_CUDA(cudaMallocAsync((void**)&gid, (size_t)rows * 4u, s));
        cudaError_t e = launch_fill_segment_gids(group_starts, n_groups, rows, gid, s);
        if (e != cudaSuccess) {
            cudaFreeAsync(gid, s);
            return cuda_fail(e, "fill segment ids");
        }
    }
    up_column c = *src;
    if (associated) c.indices = associated;
    void* outs[1] = {out};
    up_status st = up_group_agg(&c, &kind, 1, gid, n_groups, rows, outs, err_word, stream);
    if (gid) cudaFreeAsync(gid, s);
    return st;
}

up_status up_division_int64(const void* sums, const int64_t* counts, int32_t n, void* out, void* stream) {
    if (n < 0) return fail(UP_ERR_INVALID_ARG, "negative size");
    if (n == 0) return UP_OK;
    if (!sums || !counts || !out) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    UP_CUDA(launch_division_int64((const uint8_t*)sums, counts, n, (uint8_t*)out, (cudaStream_t)stream));
    return UP_OK;
}

up_status up_group_ids_from_keys(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys, int64_t rows,
                                 int32_t* group_ids, int32_t* n_groups, void* group_keys, void* stream) {
    if (!key_cols || !key_bytes || !group_ids || !n_groups) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    if (n_keys < 1 || n_keys > 4) return fail(UP_ERR_INVALID_ARG, "1..4 key columns");
    int total = 0;
    for (int k = 0; k < n_keys; k++) {
        if (key_bytes[k] < 1) return fail(UP_ERR_INVALID_ARG, "key width < 1");
        total += key_bytes[k];
    }
    if (total > 2) return fail(UP_ERR_UNSUPPORTED, "direct key table supports at most 2 key bytes in total");
    cudaStream_t s = (cudaStream_t)stream;
    UP_CUDA(launch_group_ids_small_keys(key_cols, key_bytes, n_keys, rows, group_ids, n_groups, group_keys, s));
    return UP_OK;
}

up_status up_group_table_from_keys(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                                   int64_t rows, int32_t* key_table, int32_t* n_groups, void* group_keys,
                                   void* stream) {
    if (!key_cols || !key_bytes || !key_table || !n_groups) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    if (rows < 0) return fail(UP_ERR_INVALID_ARG, "negative row count");
    if (n_keys < 1 || n_keys > 4) return fail(UP_ERR_INVALID_ARG, "1..4 key columns");
    int total = 0;
    for (int k = 0; k < n_keys; k++) {
        if (key_bytes[k] < 1) return fail(UP_ERR_INVALID_ARG, "key width < 1");
        if (rows > 0 && !key_cols[k]) return fail(UP_ERR_INVALID_ARG, "key column is NULL");
        total += key_bytes[k];
    }
    if (total > 2) return fail(UP_ERR_UNSUPPORTED, "direct key table supports at most 2 key bytes in total");
    UP_CUDA(launch_group_table_small_keys(key_cols, key_bytes, n_keys, rows, key_table, n_groups, group_keys,
                                          (cudaStream_t)stream));
    return UP_OK;
}

static up_status query_keys_of(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                               const int32_t* key_table, int64_t rows, QueryKeys& k) {
    if (!key_cols || !key_bytes || !key_table) return fail(UP_ERR_INVALID_ARG, "NULL key arguments");
    if (n_keys == 1 && key_bytes[0] == 1) k.mode = 1;
    else if (n_keys == 2 && key_bytes[0] == 1 && key_bytes[1] == 1) k.mode = 2;
    else if (n_keys == 1 && key_bytes[0] == 2) k.mode = 3;
    else return fail(UP_ERR_UNSUPPORTED, "key columns: one of 1 or 2 bytes, or two of 1 byte");
    k.key0 = (const uint8_t*)key_cols[0];
    k.key1 = k.mode == 2 ? (const uint8_t*)key_cols[1] : nullptr;
    k.table = key_table;
    if (rows > 0 && (!k.key0 || (k.mode == 2 && !k.key1))) return fail(UP_ERR_INVALID_ARG, "key column is NULL");
    return UP_OK;
}

up_status up_query_launch_keys(up_module* m, const up_column* in, int32_t n_in, int64_t rows,
                               const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                               const int32_t* key_table, int32_t n_groups, void* const* outs, uint32_t* err_word,
                               void* stream) {
    QueryKeys k;
    const up_status st = query_keys_of(key_cols, key_bytes, n_keys, key_table, rows, k);
    if (st != UP_OK) return st;
    return query_launch_ex(m, in, n_in, rows, nullptr, n_groups, outs, err_word, stream, false, &k);
}

up_status up_query_launch_keys_async(up_module* m, const up_column* in, int32_t n_in, int64_t rows,
                                     const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                                     const int32_t* key_table, int32_t max_groups, void* const* outs,
                                     uint32_t* err_word, void* stream) {
    if (max_groups < 1 || max_groups > 65536) return fail(UP_ERR_INVALID_ARG, "max_groups must be 1..65536");
    QueryKeys k;
    const up_status st = query_keys_of(key_cols, key_bytes, n_keys, key_table, rows, k);
    if (st != UP_OK) return st;
    k.capacity = max_groups;
    return query_launch_ex(m, in, n_in, rows, nullptr, max_groups, outs, err_word, stream, false, &k);
}

up_status up_group_table_from_keys_async(const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                                         int64_t rows, int32_t* key_table, void* group_keys, void* stream) {
    if (!key_cols || !key_bytes || !key_table) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    if (rows < 0) return fail(UP_ERR_INVALID_ARG, "negative row count");
    if (n_keys < 1 || n_keys > 4) return fail(UP_ERR_INVALID_ARG, "1..4 key columns");
    int total = 0;
    for (int k = 0; k < n_keys; k++) {
        if (key_bytes[k] < 1) return fail(UP_ERR_INVALID_ARG, "key width < 1");
        if (rows > 0 && !key_cols[k]) return fail(UP_ERR_INVALID_ARG, "key column is NULL");
        total += key_bytes[k];
    }
    if (total > 2) return fail(UP_ERR_UNSUPPORTED, "direct key table supports at most 2 key bytes in total");
    UP_CUDA(launch_group_table_small_keys_async(key_cols, key_bytes, n_keys, rows, key_table, group_keys,
                                                (cudaStream_t)stream));
    return UP_OK;
}

up_status up_util_compile_only(const up_expr_node* nodes, int32_t n_nodes, int32_t root, const up_col_type* cols,
                               int32_t n_cols, int32_t query, const up_query_agg* aggs, int32_t n_aggs) {
    GeneratedModule gen;
    up_status st = query ? generate_query_module(nodes, n_nodes, cols, n_cols, aggs, n_aggs, nullptr, gen)
                         : generate_expr_module(nodes, n_nodes, root, cols, n_cols, nullptr, gen);
    if (st != UP_OK) return st;
    std::vector<char> cubin;
    return jit_compile_cubin(gen.source, cubin);
}

up_status up_util_compile_expr_only(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                                    const up_col_type* cols, int32_t n_cols, const up_compile_opts* opts) {
    GeneratedModule gen;
    up_status st = generate_expr_module(nodes, n_nodes, root, cols, n_cols, opts, gen);
    if (st != UP_OK) return st;
    std::vector<char> cubin;
    return jit_compile_cubin(gen.source, cubin);
}

up_status up_util_auto_tpv(const up_expr_node* nodes, int32_t n_nodes, int32_t root, const up_col_type* cols,
                           int32_t n_cols, int32_t use_model, int32_t* threads_per_value) {
    if (!nodes || n_nodes <= 0 || !threads_per_value) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    std::vector<NodeFacts> f;
    std::vector<int> topo;
    up_status st = analyze_nodes(nodes, n_nodes, cols, n_cols, f, topo, {root});
    if (st != UP_OK) return st;
    for (int c = 0; c < n_cols; c++)
        if (cols[c].nullable) {
            *threads_per_value = 1;
            return UP_OK;
        }
    *threads_per_value = use_model ? auto_threads_per_value(nodes, n_nodes, root, cols, n_cols, f, topo)
                                   : rule_threads_per_value(nodes, f, topo);
    return UP_OK;
}

int64_t up_util_expr_source(const up_expr_node* nodes, int32_t n_nodes, int32_t root, const up_col_type* cols,
                            int32_t n_cols, const up_compile_opts* opts, char* buf, int64_t cap) {
    GeneratedModule gen;
    if (generate_expr_module(nodes, n_nodes, root, cols, n_cols, opts, gen) != UP_OK) return -1;
    const int64_t n = (int64_t)gen.source.size();
    if (buf && cap > 0) {
        const int64_t k = std::min(n, cap - 1);
        memcpy(buf, gen.source.data(), (size_t)k);
        buf[k] = '\0';
    }
    return n;
}

up_status up_device_query(int32_t device, up_device_info* info) {
    if (!info) return fail(UP_ERR_INVALID_ARG, "info is NULL");
    memset(info, 0, sizeof *info);
    cudaDeviceProp p;
    UP_CUDA(cudaGetDeviceProperties(&p, device));
    info->sm_count = p.multiProcessorCount;
    info->cc_major = p.major;
    info->cc_minor = p.minor;
    strncpy(info->name, p.name, sizeof(info->name) - 1);
    int cur = 0;
    UP_CUDA(cudaGetDevice(&cur));
    if (cur == device) {
        size_t fr = 0, tot = 0;
        UP_CUDA(cudaMemGetInfo(&fr, &tot));
        info->free_bytes = (int64_t)fr;
        info->total_bytes = (int64_t)tot;
    }
    return UP_OK;
}

}  // extern "C"
