// up_batch.cpp — batched persistent-kernel mode (include/ultraprecise_batch.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ultraprecise_batch.h"
#include "../../include/ultraprecise_util.h"
#include "up_internal.h"

using namespace upi;

namespace {

// the generated kernels' task and argument blocks (up_kargs.h)
using HBTask = BTask;
using HBArgs = BArgs;

const int kThreads[3] = {64, 128, 256};
constexpr int kSoloStreams = 1;

up_status cuda_err(cudaError_t e, const std::string& what) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? UP_ERR_NO_MEMORY : UP_ERR_CUDA, what + ": " + cudaGetErrorString(e));
}

#define UPB_CUDA(call)                                     \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_err(e_, #call); \
    } while (0)

struct Shape {
    int threads_idx = 2;  // index into kThreads
    int ctas_per_sm = 4;
    int tile_rows = 1024;
    double tuned_ms = 0.0;
};

std::string autotune_path() {
    const char* p = getenv("UP_AUTOTUNE_CACHE");
    if (p && *p) return p;
    const char* d = getenv("UP_JIT_CACHE_DIR");
    if (d && *d) return std::string(d) + "/autotune.txt";
    const char* home = getenv("HOME");
    return std::string(home && *home ? home : "/tmp") + "/.cache/ultraprecise_b200/autotune.txt";
}

uint64_t fnv(const std::string& s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

}  // namespace

struct up_batch {
    GeneratedBatch gen;
    // per task: a copy of its typed tree (for the per-task module of a solo task)
    std::vector<std::vector<up_expr_node>> t_nodes;
    std::vector<std::vector<up_col_type>> t_cols;
    std::vector<int> t_root, t_agg;
    std::vector<std::vector<up_column>> t_in;  // bound columns
    std::vector<bool> solo;                    // runs as its own kernel this step
    std::vector<up_module*> solo_mod;
    cudaStream_t solo_side[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t solo_join[4] = {nullptr, nullptr, nullptr, nullptr};
    std::shared_ptr<JitKernelSet> ks;
    up_batch_opts opts{};
    std::vector<HBTask> host_tasks;
    std::vector<bool> bound;
    std::vector<double> cost;  // per-row cost estimate per task
    void* d_tasks = nullptr;
    int64_t n_items[3] = {0, 0, 0};
    int32_t* item_task[3] = {nullptr, nullptr, nullptr};
    int64_t* item_tile[3] = {nullptr, nullptr, nullptr};
    int items_tile_rows[3] = {0, 0, 0};
    unsigned long long* heads = nullptr;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    int max_groups = 0;
    bool prepared = false;
    Shape shape[3];
    bool tuned = false;
    std::vector<int> tpv;      // threads per value per task (the batch module and the solo modules use it)
    bool tpv_tuned = false;
    bool tpv_dirty = false;    // a pinned threads per value is not in the loaded module yet
    std::vector<bool> tpv_pinned;
    std::string tpv_key;       // the batch's key before any threads-per-value change (tuning cache)
    cudaGraphExec_t gexec = nullptr;
    uint32_t* graph_err = nullptr;
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaStream_t cap = nullptr;  // private stream the step is captured on (the caller's may be the legacy stream)
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
    std::string key;
    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
    }
    void drop_device() {
        drop_graph();
        if (d_tasks) cudaFree(d_tasks);
        if (heads) cudaFree(heads);
        if (scratch) cudaFree(scratch);
        d_tasks = nullptr;
        heads = nullptr;
        scratch = nullptr;
        for (int band = 0; band < 3; band++) {
            if (item_task[band]) cudaFree(item_task[band]);
            item_task[band] = nullptr;
            item_tile[band] = nullptr;
            items_tile_rows[band] = 0;
        }
        prepared = false;
    }
    ~up_batch() {
        drop_device();
        for (auto* m : solo_mod)
            if (m) up_module_release(m);
        for (int i = 0; i < 4; i++) {
            if (solo_side[i]) cudaStreamDestroy(solo_side[i]);
            if (solo_join[i]) cudaEventDestroy(solo_join[i]);
        }
        if (cap) cudaStreamDestroy(cap);
        for (int i = 0; i < 2; i++) {
            if (side[i]) cudaStreamDestroy(side[i]);
            if (join[i]) cudaEventDestroy(join[i]);
        }
        if (fork) cudaEventDestroy(fork);
    }
};

namespace {

// (Re)build one band's work list for a given rows-per-item: every item of a
// costlier task precedes the items of cheaper ones (longest-processing-time
// order), tiles of a task in order.
up_status build_items(up_batch* b, int band, int tile_rows) {
    if (b->items_tile_rows[band] == tile_rows && b->item_task[band]) return UP_OK;
    std::vector<int> order;
    for (size_t k = 0; k < b->gen.tasks.size(); k++)
        if (b->gen.tasks[k].band == band && b->host_tasks[k].rows > 0 && !b->solo[k]) order.push_back((int)k);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->cost[x] > b->cost[y]; });
    std::vector<int32_t> it;
    std::vector<int64_t> tl;
    for (int k : order) {
        const int64_t nt = (b->host_tasks[k].rows + tile_rows - 1) / tile_rows;
        for (int64_t t = 0; t < nt; t++) {
            it.push_back(k);
            tl.push_back(t);
        }
    }
    if (b->item_task[band]) {
        cudaFree(b->item_task[band]);
        b->item_task[band] = nullptr;
        b->item_tile[band] = nullptr;
    }
    b->n_items[band] = (int64_t)it.size();
    b->items_tile_rows[band] = tile_rows;
    if (it.empty()) return UP_OK;
    void* mem = nullptr;
    const size_t bytes_t = ((it.size() * 4) + 15) & ~size_t(15), bytes_l = tl.size() * 8;
    UPB_CUDA(cudaMalloc(&mem, bytes_t + bytes_l));
    b->item_task[band] = (int32_t*)mem;
    b->item_tile[band] = (int64_t*)((uint8_t*)mem + bytes_t);
    UPB_CUDA(cudaMemcpy(b->item_task[band], it.data(), it.size() * 4, cudaMemcpyHostToDevice));
    UPB_CUDA(cudaMemcpy(b->item_tile[band], tl.data(), bytes_l, cudaMemcpyHostToDevice));
    return UP_OK;
}

HBArgs band_args(up_batch* b, int band, uint32_t* err) {
    HBArgs a;
    memset(&a, 0, sizeof a);
    a.tasks = (BTask*)b->d_tasks;
    a.item_task = b->item_task[band];
    a.item_tile = (const long long*)b->item_tile[band];
    a.n_items = b->n_items[band];
    a.head = b->heads + band;
    a.err = err;
    a.tile_rows = b->items_tile_rows[band];
    return a;
}

up_status launch_band(up_batch* b, int band, uint32_t* err, cudaStream_t s) {
    if (b->n_items[band] == 0) return UP_OK;
    const Shape& sh = b->shape[band];
    const std::string name = "up_batch_b" + std::to_string(band) + "_t" + std::to_string(kThreads[sh.threads_idx]);
    void* k = jit_kernel(*b->ks, name);
    if (!k) return fail(UP_ERR_CUDA, "missing kernel " + name);
    HBArgs a = band_args(b, band, err);
    void* args[1] = {&a};
    const int sms = std::max(1, sm_count_current());
    int64_t grid = std::min<int64_t>((int64_t)sms * sh.ctas_per_sm, b->n_items[band]);
    UPB_CUDA(cudaLaunchKernel((const void*)k, dim3((unsigned)std::max<int64_t>(grid, 1)),
                              dim3(kThreads[sh.threads_idx]), args, 0, s));
    return UP_OK;
}

up_status launch_fin(up_batch* b, uint32_t* err, cudaStream_t s) {
    if (b->gen.agg_tasks.empty() || b->max_groups == 0) return UP_OK;
    void* k = jit_kernel(*b->ks, "up_batch_fin");
    HBArgs a = band_args(b, 0, err);
    void* args[1] = {&a};
    dim3 grid((unsigned)((b->max_groups + 255) / 256), (unsigned)b->gen.agg_tasks.size());
    UPB_CUDA(cudaLaunchKernel((const void*)k, grid, dim3(256), args, 0, s));
    return UP_OK;
}

up_status clear_state(up_batch* b, cudaStream_t s) {
    UPB_CUDA(cudaMemsetAsync(b->heads, 0, 3 * sizeof(unsigned long long), s));
    if (b->scratch_bytes) UPB_CUDA(cudaMemsetAsync(b->scratch, 0, b->scratch_bytes, s));
    return UP_OK;
}

// one full step: clear, the three bands forked across streams, finalise
up_status run_step(up_batch* b, uint32_t* err, cudaStream_t s) {
    up_status st = clear_state(b, s);
    if (st != UP_OK) return st;
    UPB_CUDA(cudaEventRecord(b->fork, s));
    for (int i = 0; i < 2; i++) UPB_CUDA(cudaStreamWaitEvent(b->side[i], b->fork, 0));
    if ((st = launch_band(b, 0, err, s)) != UP_OK) return st;
    if ((st = launch_band(b, 1, err, b->side[0])) != UP_OK) return st;
    if ((st = launch_band(b, 2, err, b->side[1])) != UP_OK) return st;
    // tasks with many rows: their own kernels, one after another on a further
    // forked stream (each fills the GPU; running them concurrently measured
    // slower), overlapping the band kernels of the small tasks
    int nsolo = 0;
    for (size_t k = 0; k < b->solo.size(); k++) {
        if (!b->solo[k]) continue;
        const int q = nsolo++ % kSoloStreams;
        cudaStream_t ss = b->solo_side[q];
        if (nsolo <= kSoloStreams) UPB_CUDA(cudaStreamWaitEvent(ss, b->fork, 0));
        const HBTask& h = b->host_tasks[k];
        const auto& in = b->t_in[k];
        if (b->t_agg[k] < 0) {
            st = up_expr_launch(b->solo_mod[k], in.data(), (int32_t)in.size(), h.rows, h.out, err, ss);
        } else {
            void* outs[1] = {h.out};
            st = up_query_launch(b->solo_mod[k], in.data(), (int32_t)in.size(), h.rows, h.gid, h.n_groups, outs, err,
                                 ss);
        }
        if (st != UP_OK) return st;
    }
    for (int i = 0; i < 2; i++) {
        UPB_CUDA(cudaEventRecord(b->join[i], b->side[i]));
        UPB_CUDA(cudaStreamWaitEvent(s, b->join[i], 0));
    }
    for (int q = 0; q < std::min(nsolo, kSoloStreams); q++) {
        UPB_CUDA(cudaEventRecord(b->solo_join[q], b->solo_side[q]));
        UPB_CUDA(cudaStreamWaitEvent(s, b->solo_join[q], 0));
    }
    return launch_fin(b, err, s);
}

up_status prepare(up_batch* b) {
    if (b->prepared) return UP_OK;
    const size_t nt = b->host_tasks.size();
    // tasks with many rows run as their own per-task kernels
    const int64_t solo_rows = b->opts.solo_rows == 0 ? (int64_t)262144 : b->opts.solo_rows;
    for (size_t k = 0; k < nt; k++) {
        b->solo[k] = solo_rows > 0 && b->host_tasks[k].rows >= solo_rows;
        if (!b->solo[k] || b->solo_mod[k]) continue;
        up_module* m = nullptr;
        up_status st;
        if (b->t_agg[k] < 0) {
            up_compile_opts mo;
            memset(&mo, 0, sizeof mo);
            mo.threads_per_value = b->tpv[k];
            st = up_module_compile(b->t_nodes[k].data(), (int32_t)b->t_nodes[k].size(), b->t_root[k],
                                   b->t_cols[k].data(), (int32_t)b->t_cols[k].size(), &mo, &m);
        } else {
            up_query_agg qa = {b->t_agg[k], b->t_root[k]};
            st = up_query_compile(b->t_nodes[k].data(), (int32_t)b->t_nodes[k].size(), b->t_cols[k].data(),
                                  (int32_t)b->t_cols[k].size(), &qa, 1, nullptr, &m);
        }
        if (st != UP_OK) return st;
        b->solo_mod[k] = m;
    }
    size_t off = 0;
    std::vector<size_t> acc_off(nt, 0), cnt_off(nt, 0);
    b->max_groups = 0;
    for (size_t k = 0; k < nt; k++) {
        const auto& gt = b->gen.tasks[k];
        if (gt.agg < 0 || b->solo[k]) continue;
        const int G = b->host_tasks[k].n_groups;
        b->max_groups = std::max(b->max_groups, G);
        acc_off[k] = off;
        off += (((size_t)G * std::max(gt.nacc, 1) * 4u) + 15u) & ~size_t(15);
        cnt_off[k] = off;
        off = (off + (size_t)G * 8u + 15u) & ~size_t(15);
    }
    b->scratch_bytes = off;
    if (off) UPB_CUDA(cudaMalloc(&b->scratch, off));
    std::vector<HBTask> dev_tasks = b->host_tasks;
    for (size_t k = 0; k < nt; k++) {
        if (b->solo[k]) {  // neither the bands nor the finalisation touch it
            dev_tasks[k].rows = 0;
            dev_tasks[k].n_groups = 0;
            continue;
        }
        if (b->gen.tasks[k].agg < 0) continue;
        dev_tasks[k].acc = (uint32_t*)((uint8_t*)b->scratch + acc_off[k]);
        dev_tasks[k].cnt = (unsigned long long*)((uint8_t*)b->scratch + cnt_off[k]);
    }
    UPB_CUDA(cudaMalloc(&b->d_tasks, nt * sizeof(HBTask)));
    UPB_CUDA(cudaMemcpy(b->d_tasks, dev_tasks.data(), nt * sizeof(HBTask), cudaMemcpyHostToDevice));
    UPB_CUDA(cudaMalloc((void**)&b->heads, 3 * sizeof(unsigned long long)));
    for (int i = 0; i < 2; i++) {
        if (!b->side[i]) UPB_CUDA(cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking));
        if (!b->join[i]) UPB_CUDA(cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming));
    }
    for (int i = 0; i < 4; i++) {
        if (!b->solo_side[i]) UPB_CUDA(cudaStreamCreateWithFlags(&b->solo_side[i], cudaStreamNonBlocking));
        if (!b->solo_join[i]) UPB_CUDA(cudaEventCreateWithFlags(&b->solo_join[i], cudaEventDisableTiming));
    }
    if (!b->fork) UPB_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    if (!b->cap) UPB_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    for (int band = 0; band < 3; band++) {
        up_status st = build_items(b, band, b->shape[band].tile_rows);
        if (st != UP_OK) return st;
    }
    b->prepared = true;
    return UP_OK;
}

// ------------------------------------------------------------ autotuner
bool load_tuned(up_batch* b) {
    std::ifstream f(autotune_path());
    if (!f) return false;
    std::string line;
    int found = 0;
    Shape tmp[3];
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::string key;
        int band, ti, ctas, tr;
        double ms;
        if (!(ss >> key >> band >> ti >> ctas >> tr >> ms)) continue;
        if (key != b->key || band < 0 || band > 2 || ti < 0 || ti > 2 || ctas < 1 || tr < 1) continue;
        tmp[band] = Shape{ti, ctas, tr, ms};
        found |= 1 << band;
    }
    if (found != 7) return false;
    for (int i = 0; i < 3; i++) b->shape[i] = tmp[i];
    return true;
}

void save_tuned(up_batch* b) {
    const std::string p = autotune_path();
    const std::string dir = p.substr(0, p.rfind('/'));
    for (size_t i = 1; i <= dir.size(); i++)
        if (i == dir.size() || dir[i] == '/') mkdir_if_missing(dir.substr(0, i));
    std::ofstream f(p, std::ios::app);
    for (int band = 0; band < 3; band++) {
        const Shape& s = b->shape[band];
        f << b->key << " " << band << " " << s.threads_idx << " " << s.ctas_per_sm << " " << s.tile_rows << " "
          << s.tuned_ms << "\n";
    }
}

// Sweep block size x CTAs per SM x rows per work item for each band, timing
// that band's kernel alone with CUDA events; keep the fastest shape.
up_status autotune(up_batch* b, cudaStream_t s) {
    if (load_tuned(b)) {
        for (int band = 0; band < 3; band++) {
            up_status st = build_items(b, band, b->shape[band].tile_rows);
            if (st != UP_OK) return st;
        }
        b->tuned = true;
        return UP_OK;
    }
    cudaEvent_t e0, e1;
    UPB_CUDA(cudaEventCreate(&e0));
    UPB_CUDA(cudaEventCreate(&e1));
    static const int kCtas[] = {1, 2, 4, 8};
    static const int kTiles[] = {256, 1024, 4096};
    up_status st = UP_OK;
    for (int band = 0; band < 3 && st == UP_OK; band++) {
        bool any = false;
        for (size_t k = 0; k < b->gen.tasks.size(); k++)
            if (b->gen.tasks[k].band == band && b->host_tasks[k].rows > 0 && !b->solo[k]) any = true;
        if (!any) continue;
        Shape best = b->shape[band];
        best.tuned_ms = 1e30;
        for (int tr : kTiles) {
            if ((st = build_items(b, band, tr)) != UP_OK) break;
            for (int ti = 0; ti < 3 && st == UP_OK; ti++)
                for (int c : kCtas) {
                    b->shape[band] = Shape{ti, c, tr, 0.0};
                    double best_rep = 1e30;
                    for (int rep = 0; rep < 2; rep++) {
                        if ((st = clear_state(b, s)) != UP_OK) break;
                        cudaEventRecord(e0, s);
                        if ((st = launch_band(b, band, nullptr, s)) != UP_OK) break;
                        cudaEventRecord(e1, s);
                        cudaEventSynchronize(e1);
                        float ms = 0;
                        cudaEventElapsedTime(&ms, e0, e1);
                        best_rep = std::min(best_rep, (double)ms);
                    }
                    if (st != UP_OK) break;
                    if (best_rep < best.tuned_ms) best = Shape{ti, c, tr, best_rep};
                }
        }
        b->shape[band] = best;
        if (st == UP_OK) st = build_items(b, band, best.tile_rows);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != UP_OK) return st;
    b->tuned = true;
    save_tuned(b);
    return UP_OK;
}

// Threads per value before any measurement: automatic for projections (the
// default cost model, else the width rule) unless one thread is asked for;
// aggregates one thread per value.
std::vector<int> initial_tpv(const up_batch_task* tasks, int n_tasks, int policy) {
    std::vector<int> tpv(n_tasks, 1);
    for (int k = 0; k < n_tasks && policy != 1; k++) {
        if (tasks[k].agg_kind >= 0) continue;
        std::vector<NodeFacts> f;
        std::vector<int> topo;
        if (analyze_nodes(tasks[k].nodes, tasks[k].n_nodes, tasks[k].cols, tasks[k].n_cols, f, topo,
                          {tasks[k].root}) != UP_OK)
            continue;  // reported by the module build
        bool nullable = false;
        for (int c = 0; c < tasks[k].n_cols; c++) nullable |= tasks[k].cols[c].nullable != 0;
        if (!nullable)
            tpv[k] = auto_threads_per_value(tasks[k].nodes, tasks[k].n_nodes, tasks[k].root, tasks[k].cols,
                                            tasks[k].n_cols, f, topo);
    }
    return tpv;
}

// (Re)generate, compile and load the batch module for the current
// threads-per-value choices.
up_status build_module(up_batch* b) {
    const int n = (int)b->t_nodes.size();
    std::vector<BatchTaskDesc> desc(n);
    for (int k = 0; k < n; k++)
        desc[k] = BatchTaskDesc{b->t_nodes[k].data(), (int)b->t_nodes[k].size(), b->t_root[k], b->t_cols[k].data(),
                                (int)b->t_cols[k].size(), b->t_agg[k], b->tpv[k]};
    GeneratedBatch gen;
    up_status st = generate_batch_module(desc.data(), n, gen);
    if (st != UP_OK) return st;
    std::vector<char> cubin;
    if ((st = jit_compile_linked(gen.units, cubin)) != UP_OK) return st;
    std::shared_ptr<JitKernelSet> ks;
    if ((st = jit_load(cubin, gen.kernels, ks)) != UP_OK) return st;
    b->gen = std::move(gen);
    b->ks = ks;
    for (int k = 0; k < n; k++) b->tpv[k] = b->gen.tasks[k].tpv;
    b->tpv_dirty = false;
    char key[40];
    snprintf(key, sizeof key, "%016llx", (unsigned long long)fnv(b->gen.source));
    b->key = key;
    return UP_OK;
}

// Candidate threads per value of a projection task: one thread, and the
// groups that leave each thread 2..16 limbs of its widest intermediate (a
// single limb per thread is all shuffles; more than 16 spill).  Tasks narrower
// than 16 limbs run one thread per value.
constexpr double kTpvMargin = 0.9;  // a cooperative choice must time below 0.9 x one thread per value

std::vector<int> tpv_candidates(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols,
                                int n_cols, int agg) {
    std::vector<int> c = {1};
    if (agg >= 0) return c;
    const int w = coop_width_of(nodes, n_nodes, root, cols, n_cols);
    if (w < 16) return c;
    for (int t : {2, 4, 8, 16, 32}) {
        const int kk = (w + t - 1) / t;
        if (kk >= 2 && kk <= 16) c.push_back(t);
    }
    return c;
}

// The measured threads-per-value policy: time each projection task's own
// module at every candidate on its bound inputs (at most 1M rows, into its
// own output), keep the fastest; the choices are cached with the rows.
up_status tune_tpv(up_batch* b, cudaStream_t s) {
    const int n = (int)b->t_nodes.size();
    std::vector<int> chosen = b->tpv;
    std::vector<bool> have(n, false);
    {
        std::ifstream f(autotune_path());
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream ss(line);
            std::string tag, key;
            int task, tpv;
            long long rows;
            double ms;
            if (!(ss >> tag >> key >> task >> rows >> tpv >> ms)) continue;
            if (tag != "tpv" || key != b->tpv_key || task < 0 || task >= n || b->tpv_pinned[task]) continue;
            if (rows != (long long)b->host_tasks[task].rows) continue;
            chosen[task] = tpv;
            have[task] = true;
        }
    }
    cudaEvent_t e0, e1;
    UPB_CUDA(cudaEventCreate(&e0));
    UPB_CUDA(cudaEventCreate(&e1));
    std::ostringstream lines;
    up_status st = UP_OK;
    for (int k = 0; k < n && st == UP_OK; k++) {
        if (have[k] || b->tpv_pinned[k] || b->t_agg[k] >= 0 || b->host_tasks[k].rows == 0) continue;
        const std::vector<int> cand = tpv_candidates(b->t_nodes[k].data(), (int)b->t_nodes[k].size(), b->t_root[k],
                                                     b->t_cols[k].data(), (int)b->t_cols[k].size(), b->t_agg[k]);
        if (cand.size() < 2) {
            chosen[k] = 1;
            continue;
        }
        const int64_t rows = std::min<int64_t>(b->host_tasks[k].rows, (int64_t)1 << 20);
        double best_ms = 1e30, one_ms = 1e30;
        int best = 1;
        for (int t : cand) {
            up_compile_opts mo;
            memset(&mo, 0, sizeof mo);
            mo.threads_per_value = t;
            up_module* m = nullptr;
            if (up_module_compile(b->t_nodes[k].data(), (int32_t)b->t_nodes[k].size(), b->t_root[k],
                                  b->t_cols[k].data(), (int32_t)b->t_cols[k].size(), &mo, &m) != UP_OK)
                continue;  // no cooperative form at this width: not a candidate
            const auto& in = b->t_in[k];
            double ms_best = 1e30;
            for (int rep = 0; rep < 3 && st == UP_OK; rep++) {
                cudaEventRecord(e0, s);
                st = up_expr_launch(m, in.data(), (int32_t)in.size(), rows, b->host_tasks[k].out, nullptr, s);
                cudaEventRecord(e1, s);
                if (cudaEventSynchronize(e1) != cudaSuccess) st = fail(UP_ERR_CUDA, "threads-per-value timing");
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) ms_best = std::min(ms_best, (double)ms);  // the first launch warms up
            }
            up_module_release(m);
            if (t == 1) one_ms = ms_best;
            if (ms_best < best_ms) {
                best_ms = ms_best;
                best = t;
            }
        }
        // a group of threads has to beat one thread per value by kTpvMargin:
        // timed alone, smaller gains did not survive running beside the other
        // tasks of the step
        if (best != 1 && one_ms < 1e30 && best_ms > kTpvMargin * one_ms) {
            best = 1;
            best_ms = one_ms;
        }
        chosen[k] = best;
        lines << "tpv " << b->tpv_key << " " << k << " " << b->host_tasks[k].rows << " " << best << " " << best_ms
              << "\n";
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != UP_OK) return st;
    if (!lines.str().empty()) {
        const std::string p = autotune_path();
        const std::string dir = p.substr(0, p.rfind('/'));
        for (size_t i = 1; i <= dir.size(); i++)
            if (i == dir.size() || dir[i] == '/') mkdir_if_missing(dir.substr(0, i));
        std::ofstream f(p, std::ios::app);
        f << lines.str();
    }
    b->tpv_tuned = true;
    if (chosen == b->tpv && !b->tpv_dirty) return UP_OK;
    b->tpv = chosen;
    b->drop_device();  // the work lists and the graph belong to the old module
    for (auto*& m : b->solo_mod)
        if (m) {
            up_module_release(m);
            m = nullptr;
        }
    return build_module(b);
}

}  // namespace

extern "C" {

up_status up_batch_create(const up_batch_task* tasks, int32_t n_tasks, const up_batch_opts* opts, up_batch** out) {
    if (!tasks || !out || n_tasks <= 0) return fail(UP_ERR_INVALID_ARG, "no tasks");
    *out = nullptr;
    if (opts && (opts->tpv_policy < 0 || opts->tpv_policy > 2)) return fail(UP_ERR_INVALID_ARG, "bad tpv_policy");
    auto* b = new up_batch();
    if (opts) b->opts = *opts;
    else b->opts.use_graph = 1;
    for (int k = 0; k < n_tasks; k++) {
        b->t_nodes.emplace_back(tasks[k].nodes, tasks[k].nodes + tasks[k].n_nodes);
        b->t_cols.emplace_back(tasks[k].cols, tasks[k].cols + tasks[k].n_cols);
        b->t_root.push_back(tasks[k].root);
        b->t_agg.push_back(tasks[k].agg_kind);
    }
    b->tpv = initial_tpv(tasks, n_tasks, b->opts.tpv_policy);
    b->tpv_pinned.assign(n_tasks, false);
    up_status st = build_module(b);
    if (st != UP_OK) {
        delete b;
        return st;
    }
    b->tpv_key = b->key;
    b->host_tasks.assign(n_tasks, HBTask());
    memset(b->host_tasks.data(), 0, sizeof(HBTask) * n_tasks);
    b->bound.assign(n_tasks, false);
    b->cost.assign(n_tasks, 1.0);
    b->solo.assign(n_tasks, false);
    b->solo_mod.assign(n_tasks, nullptr);
    b->t_in.assign(n_tasks, {});
    for (int k = 0; k < n_tasks; k++) {
        // per-row cost estimate: limb products of every node
        std::vector<NodeFacts> f;
        std::vector<int> topo;
        analyze_nodes(tasks[k].nodes, tasks[k].n_nodes, tasks[k].cols, tasks[k].n_cols, f, topo, {tasks[k].root});
        double c = 0;
        for (int n : topo) c += (double)f[n].limbs * f[n].limbs;
        b->cost[k] = c;
    }
    for (int band = 0; band < 3; band++) {
        Shape& s = b->shape[band];
        if (b->opts.block_threads == 64) s.threads_idx = 0;
        else if (b->opts.block_threads == 128) s.threads_idx = 1;
        else if (b->opts.block_threads == 256) s.threads_idx = 2;
        else s.threads_idx = band == 2 ? 0 : 2;
        s.ctas_per_sm = b->opts.ctas_per_sm > 0 ? b->opts.ctas_per_sm : (band == 2 ? 8 : 4);
        s.tile_rows = b->opts.tile_rows > 0 ? b->opts.tile_rows : (band == 2 ? 256 : 1024);
    }
    *out = b;
    return UP_OK;
}

up_status up_batch_bind(up_batch* b, int32_t task, const up_column* in, int32_t n_in, int64_t rows,
                        const int32_t* group_ids, int32_t n_groups, void* out) {
    if (!b || task < 0 || task >= (int)b->gen.tasks.size()) return fail(UP_ERR_INVALID_ARG, "bad task");
    const auto& gt = b->gen.tasks[task];
    if (n_in < (int)gt.in_bytes.size() || (n_in > 0 && !in)) return fail(UP_ERR_INVALID_ARG, "too few columns");
    if (rows < 0 || !out) return fail(UP_ERR_INVALID_ARG, "bad rows or output");
    if (gt.agg >= 0 && (n_groups < 0 || (rows > 0 && !group_ids))) return fail(UP_ERR_INVALID_ARG, "bad groups");
    HBTask& h = b->host_tasks[task];
    memset(&h.col, 0, sizeof h.col);
    bool words = true;
    for (int c = 0; c < (int)gt.in_bytes.size(); c++) {
        if (in[c].value_bytes != gt.in_bytes[c] || !in[c].data || in[c].n_blocks > 0 || in[c].indices ||
            in[c].nullable)
            return fail(UP_ERR_INVALID_ARG, "batch tasks take contiguous non-null columns of the compiled width");
        h.col[c].data = (const unsigned char*)in[c].data;
        h.col[c].value_bytes = in[c].value_bytes;
        if (((uintptr_t)in[c].data & 3u) != 0) words = false;
    }
    b->t_in[task].assign(in, in + gt.in_bytes.size());
    h.rows = rows;
    h.out = (uint8_t*)out;
    h.gid = group_ids;
    h.n_groups = gt.agg >= 0 ? n_groups : 0;
    h.words = words ? 1 : 0;
    b->bound[task] = true;
    b->drop_device();  // device copies and the graph are rebuilt on the next launch
    return UP_OK;
}

up_status up_batch_launch(up_batch* b, uint32_t* err_word, void* stream) {
    if (!b) return fail(UP_ERR_INVALID_ARG, "batch is NULL");
    for (size_t k = 0; k < b->bound.size(); k++)
        if (!b->bound[k]) return fail(UP_ERR_INVALID_ARG, "task " + std::to_string(k) + " is not bound");
    cudaStream_t s = (cudaStream_t)stream;
    up_status st;
    if (b->opts.tpv_policy == 2 && !b->tpv_tuned) {
        if ((st = tune_tpv(b, s)) != UP_OK) return st;
    }
    if (b->tpv_dirty) {  // pinned threads per value: the module, work lists, solo modules and graph are rebuilt
        b->drop_device();
        for (auto*& m : b->solo_mod)
            if (m) {
                up_module_release(m);
                m = nullptr;
            }
        if ((st = build_module(b)) != UP_OK) return st;
    }
    b->tpv_dirty = false;
    st = prepare(b);
    if (st != UP_OK) return st;
    if (b->opts.autotune && !b->tuned) {
        if ((st = autotune(b, s)) != UP_OK) return st;
    }
    if (!b->opts.use_graph) return run_step(b, err_word, s);
    if (b->gexec && b->graph_err != err_word) b->drop_graph();
    if (!b->gexec) {
        cudaGraph_t g = nullptr;
        UPB_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
        up_status st2 = run_step(b, err_word, b->cap);
        cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (st2 != UP_OK) {
            if (g) cudaGraphDestroy(g);
            return st2;
        }
        if (e != cudaSuccess) return cuda_err(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_err(e, "cudaGraphInstantiate");
        b->graph_err = err_word;
    }
    UPB_CUDA(cudaGraphLaunch(b->gexec, s));
    return UP_OK;
}

up_status up_batch_shape(const up_batch* b, int32_t band, int32_t* block_threads, int32_t* ctas_per_sm,
                         int32_t* tile_rows, double* tuned_ms) {
    if (!b || band < 0 || band > 2) return fail(UP_ERR_INVALID_ARG, "bad band");
    const Shape& s = b->shape[band];
    if (block_threads) *block_threads = kThreads[s.threads_idx];
    if (ctas_per_sm) *ctas_per_sm = s.ctas_per_sm;
    if (tile_rows) *tile_rows = s.tile_rows;
    if (tuned_ms) *tuned_ms = s.tuned_ms;
    return UP_OK;
}

up_status up_batch_task_type(const up_batch* b, int32_t task, int32_t* precision, int32_t* scale,
                             int32_t* value_bytes, int32_t* band) {
    if (!b || task < 0 || task >= (int)b->gen.tasks.size()) return fail(UP_ERR_INVALID_ARG, "bad task");
    const auto& t = b->gen.tasks[task];
    if (precision) *precision = t.out_p;
    if (scale) *scale = t.out_s;
    if (value_bytes) *value_bytes = t.out_bytes;
    if (band) *band = t.band;
    return UP_OK;
}

up_status up_batch_set_task_tpv(up_batch* b, int32_t task, int32_t threads_per_value) {
    if (!b || task < 0 || task >= (int)b->tpv.size()) return fail(UP_ERR_INVALID_ARG, "bad task");
    const int t = threads_per_value;
    if (t != 1 && t != 2 && t != 4 && t != 8 && t != 16 && t != 32)
        return fail(UP_ERR_INVALID_ARG, "threads_per_value must be 1, 2, 4, 8, 16 or 32");
    b->tpv_pinned[task] = true;
    if (b->tpv[task] != t) {
        b->tpv[task] = t;
        b->tpv_dirty = true;
    }
    return UP_OK;
}

up_status up_batch_task_tpv(const up_batch* b, int32_t task, int32_t* threads_per_value) {
    if (!b || task < 0 || task >= (int)b->tpv.size() || !threads_per_value)
        return fail(UP_ERR_INVALID_ARG, "bad task");
    *threads_per_value = b->tpv[task];
    return UP_OK;
}

void up_batch_release(up_batch* b) { delete b; }

int32_t up_util_batch_tpv_candidates(const up_batch_task* task, int32_t* out, int32_t cap) {
    if (!task || !out || cap <= 0) return -1;
    const std::vector<int> c =
        tpv_candidates(task->nodes, task->n_nodes, task->root, task->cols, task->n_cols, task->agg_kind);
    int n = 0;
    for (int t : c)
        if (n < cap) out[n++] = t;
    return n;
}

up_status up_util_compile_batch_only(const up_batch_task* tasks, int32_t n_tasks, const int32_t* tpv_of) {
    if (!tasks || n_tasks <= 0) return fail(UP_ERR_INVALID_ARG, "no tasks");
    const std::vector<int> auto_tpv = initial_tpv(tasks, n_tasks, 0);
    std::vector<BatchTaskDesc> desc(n_tasks);
    for (int k = 0; k < n_tasks; k++)
        desc[k] = BatchTaskDesc{tasks[k].nodes, tasks[k].n_nodes, tasks[k].root, tasks[k].cols, tasks[k].n_cols,
                                tasks[k].agg_kind, tpv_of ? tpv_of[k] : auto_tpv[k]};
    GeneratedBatch gen;
    up_status st = generate_batch_module(desc.data(), n_tasks, gen);
    if (st != UP_OK) return st;
    std::vector<char> cubin;
    return jit_compile_linked(gen.units, cubin);
}

}  // extern "C"
