// up_internal.h — host-side internals shared by the C++ sources of
// libultraprecise.so (not part of the public ABI).
#ifndef UP_INTERNAL_H_
#define UP_INTERNAL_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ultraprecise.h"
#include "up_kargs.h"

namespace upi {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
up_status fail(up_status s, const std::string& msg);
const char* last_error();

// ---------------------------------------------------------------- tables
int compact_bytes(int precision);    // B(p) with the extension rule
int precision_words(int precision);  // W(p) with the extension rule
constexpr int kMaxPrecision = 4000;

// ------------------------------------------------------- host big integer
// Little-endian base-2^32 magnitude, trimmed (no leading zero limbs).
struct Big {
    std::vector<uint32_t> m;
    bool is_zero() const { return m.empty(); }
};
void big_trim(Big& a);
Big big_from_u64(uint64_t v);
Big big_pow10(int k);
Big big_mul(const Big& a, const Big& b);
Big big_add(const Big& a, const Big& b);
Big big_sub(const Big& a, const Big& b);  // a >= b
int big_cmp(const Big& a, const Big& b);
int big_bitlen(const Big& a);
Big big_divmod_small(const Big& a, uint32_t d, uint32_t* rem);
uint64_t big_low64(const Big& a);  // a mod 2^64
std::string big_to_dec(const Big& a);
Big big_from_dec(const std::string& s);

// ------------------------------------------------------ expression typing
// Per-node facts the code generator needs: the evaluation scale (static),
// an upper bound on magnitude bits, hence the limb count.
struct NodeFacts {
    int scale = 0;
    int bits = 1;
    int limbs = 1;
    bool is_compare = false;
};
up_status analyze_nodes(const up_expr_node* nodes, int n_nodes, const up_col_type* cols, int n_cols,
                        std::vector<NodeFacts>& facts, std::vector<int>& topo, const std::vector<int>& roots);
int limbs_for_bits(int bits);
// Cost-model features of an expression launch (ultraprecise_costmodel.h).
up_status expr_cost_features(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols, int n_cols,
                             int tpv, int64_t rows, float* out, bool* coop_ok);
// The process-wide model up_module_compile consults for automatic threads per
// value (NULL: the width rule); set by up_costmodel_set_default.
struct CostChoice {
    bool valid = false;
    int tpv = 1;
};
CostChoice default_model_choose_tpv(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols,
                                    int n_cols);
// Automatic threads per value of an expression over non-nullable columns:
// the default cost model's choice when one is set, else the width rule.
// Returns 1 for one thread per value.
int auto_threads_per_value(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols, int n_cols,
                           const std::vector<NodeFacts>& f, const std::vector<int>& topo);
// The width rule alone (no cost model).
int rule_threads_per_value(const up_expr_node* nodes, const std::vector<NodeFacts>& f, const std::vector<int>& topo);
// Widest limb count of a cooperative evaluation (0: no cooperative form).
int coop_width_of(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols, int n_cols);

// ------------------------------------------------------------ code generation
struct GeneratedModule {
    std::string source;
    std::vector<std::string> kernels;
    // expression modules
    int out_precision = 0, out_scale = 0, out_bytes = 0;
    bool out_is_compare = false;
    int block_threads = 256;
    int tile_rows = 256;
    int smem_bytes = 0;
    std::vector<int> in_bytes;  // per referenced input column: value bytes
    // query modules
    int n_aggs = 0;
    std::vector<int> agg_kind, agg_scale, agg_acc_limbs, agg_acc_offset;
    int acc_words_per_group = 0;  // one accumulator per distinct aggregated expression
    bool q_staged = false;        // tile kernels (bulk-copy staged inputs) were generated
    int q_tile_rows = 0;          // rows per tile of the tile kernels
    int q_gr = 0;                 // up_query_tile_r handles n_groups <= q_gr
    int q_gr_lo = 0;              // up_query_tile_r_lo handles n_groups <= q_gr_lo (0: no such kernel)
    int q_gs = 0;                 // up_query_tile_s handles n_groups <= q_gs
    int q_smem = 0;               // dynamic shared memory of the tile kernels
    long work_per_row = 0;        // limb-product work + bytes per row (scheduling cost estimate)
    int threads_per_value = 1;    // threads cooperating on one value in the tile kernel
    // up_expr_multi (merged launches of several requests): rows per virtual
    // tile (0: the module has no such kernel), CTA threads, shared memory
    int multi_rows = 0, multi_threads = 0, multi_smem = 0;
};
up_status generate_expr_module(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols,
                               int n_cols, const up_compile_opts* opts, GeneratedModule& out);
up_status generate_query_module(const up_expr_node* nodes, int n_nodes, const up_col_type* cols, int n_cols,
                                const up_query_agg* aggs, int n_aggs, const up_compile_opts* opts,
                                GeneratedModule& out);

// batch modules (one source, every task; persistent band kernels)
struct BatchTaskDesc {
    const up_expr_node* nodes;
    int n_nodes;
    int root;
    const up_col_type* cols;
    int n_cols;
    int agg_kind;  // -1 projection
    int tpv;       // threads per value of a projection task (1: one thread; 2..32: cooperative)
};
struct GeneratedBatch {
    struct Task {
        int band = 0;
        int agg = -1;
        int out_p = 0, out_s = 0, out_bytes = 0;
        int nacc = 0, agg_scale = 0;
        int tpv = 1;  // threads per value the task's tile function runs with
        std::vector<int> in_bytes;
    };
    std::vector<Task> tasks;
    std::vector<int> agg_tasks;
    std::vector<std::string> units;  // one relocatable unit per distinct task, then the dispatcher
    std::string source;              // all units concatenated (cache key of the batch)
    std::vector<std::string> kernels;
};
up_status generate_batch_module(const BatchTaskDesc* tasks, int n_tasks, GeneratedBatch& out);

// ------------------------------------------------------------------ JIT
struct JitKernelSet;  // opaque: loaded library + kernel handles
struct JitModule {
    std::shared_ptr<JitKernelSet> ks;
    GeneratedModule gen;
};
// Compile (or fetch from the cache) and load.  Thread-safe.
up_status jit_compile_cubin(const std::string& src, std::vector<char>& cubin);
up_status jit_compile_linked(const std::vector<std::string>& units, std::vector<char>& linked);
up_status jit_load(const std::vector<char>& cubin, const std::vector<std::string>& kernels,
                   std::shared_ptr<JitKernelSet>& out);
up_status jit_get(const GeneratedModule& gen, std::shared_ptr<JitKernelSet>& out);
void* jit_kernel(const JitKernelSet& ks, const std::string& name);  // cudaKernel_t as void*
int jit_cache_size(bool clear);
const std::string& device_header_source();

// ------------------------------------------------------------ devices
int sm_count_current();
void mkdir_if_missing(const std::string& dir);

}  // namespace upi

// Device staging of up_expr_launch_host, kept by the module between calls:
// kSets buffer sets in rotation, the three streams and their events.
struct HostStaging {
    static constexpr int kSets = 3;
    void* dev = nullptr;
    size_t bytes = 0;
    cudaStream_t s_in = nullptr, s_k = nullptr, s_out = nullptr;
    cudaEvent_t ev_in[kSets] = {}, ev_k[kSets] = {}, ev_out[kSets] = {};
    up_status ensure(size_t need) {
        if (!s_in) {
            for (cudaStream_t* sp : {&s_in, &s_k, &s_out})
                if (cudaStreamCreateWithFlags(sp, cudaStreamNonBlocking) != cudaSuccess) return bad();
            for (int i = 0; i < kSets; i++)
                for (cudaEvent_t* ep : {&ev_in[i], &ev_k[i], &ev_out[i]})
                    if (cudaEventCreateWithFlags(ep, cudaEventDisableTiming) != cudaSuccess) return bad();
        }
        if (need > bytes) {
            if (dev) cudaFree(dev);
            dev = nullptr;
            bytes = 0;
            if (cudaMalloc(&dev, need) != cudaSuccess) {
                cudaGetLastError();
                return upi::fail(UP_ERR_NO_MEMORY, "host launch staging");
            }
            bytes = need;
        }
        return UP_OK;
    }
    up_status bad() {
        cudaGetLastError();
        return upi::fail(UP_ERR_CUDA, "host launch streams");
    }
    ~HostStaging() {
        for (cudaStream_t s : {s_in, s_k, s_out})
            if (s) cudaStreamSynchronize(s);
        if (dev) cudaFree(dev);
        for (int i = 0; i < kSets; i++)
            for (cudaEvent_t ev : {ev_in[i], ev_k[i], ev_out[i]})
                if (ev) cudaEventDestroy(ev);
        for (cudaStream_t s : {s_in, s_k, s_out})
            if (s) cudaStreamDestroy(s);
    }
};

struct up_module {
    upi::JitModule jm;
    bool is_query = false;
    std::mutex host_mu;   // one host launch at a time per module
    HostStaging host;
};

// Launch variants used by the serving loop: `spread` launches one CTA per
// tile instead of a persistent grid, so that a long request's CTAs retire
// often and higher-priority streams get SMs between them.
up_status expr_launch_ex(up_module* m, const up_column* in, int32_t n_in, int64_t rows, void* out,
                         uint32_t* err_word, void* stream, bool spread);
// Group keys read by the query kernel itself (key_mode 1..3 of the generated
// UpQArgs) instead of a group id array.
struct QueryKeys {
    const uint8_t* key0 = nullptr;
    const uint8_t* key1 = nullptr;
    const int32_t* table = nullptr;
    int mode = 0;
    // > 0: the group count is read on the device from the key table (entry
    // 131072) and may be at most `capacity`, which sizes the accumulators
    int capacity = 0;
};
// Scratch of a query launch for n_groups groups: the accumulators (16-byte
// padded) followed by one int64 count per group.
size_t query_scratch_bytes(const upi::GeneratedModule& g, int32_t n_groups);
// scratch: caller-provided device memory of scratch_bytes (at least
// query_scratch_bytes, 16-byte aligned) used instead of a stream-ordered
// allocation; the launch clears what it uses on `stream`.
up_status query_launch_ex(up_module* m, const up_column* in, int32_t n_in, int64_t rows, const int32_t* group_ids,
                          int32_t n_groups, void* const* outs, uint32_t* err_word, void* stream, bool spread,
                          const QueryKeys* keys = nullptr, void* scratch = nullptr, size_t scratch_bytes = 0);

#endif  // UP_INTERNAL_H_
