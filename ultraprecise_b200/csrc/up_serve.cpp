// up_serve.cpp — serving loop (include/ultraprecise_serve.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ultraprecise_serve.h"
#include "up_internal.h"

using namespace upi;

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    int64_t id = 0;
    up_module* module = nullptr;
    std::vector<up_column> in;
    int64_t rows = 0;
    const int32_t* group_ids = nullptr;
    int32_t n_groups = 0;
    double arrival_ms = 0.0;
    double done_ms = 0.0;
    int32_t state = UP_REQ_QUEUED;
    int64_t bytes = 0;                  // outputs + query scratch, for admission
    std::vector<int64_t> part_off, part_bytes;
    int64_t out_bytes = 0;              // the allocation: err word slot + outputs
    bool heavy = false;                 // work above opts.heavy_work: low-priority stream, spread grid
    void* mem = nullptr;
    cudaStream_t stream = nullptr;
    uint32_t* host_err = nullptr;       // pinned slot the err word is copied to
    up_serve* owner = nullptr;
};

constexpr int64_t kAlign = 256;
int64_t pad(int64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

}  // namespace

struct up_serve {
    int device = 0;
    Clock::time_point t0;
    up_serve_opts opts{};
    std::vector<cudaStream_t> streams;        // high priority: ordinary requests
    std::vector<cudaStream_t> heavy_streams;  // low priority: long requests
    size_t next_stream = 0, next_heavy = 0;
    uint32_t* pinned = nullptr;         // one err slot per in-flight request
    std::vector<int> free_slots;
    std::unordered_map<int64_t, std::unique_ptr<Req>> reqs;
    std::unordered_map<uint32_t*, int> slot_of;
    std::deque<Req*> queue;
    std::mutex mu;
    std::condition_variable cv;        // scheduler wake-ups
    std::condition_variable done_cv;   // request completions
    std::thread worker;
    bool stop = false;
    int64_t next_id = 1;
    int64_t budget = 0, outstanding = 0, max_outstanding = 0;
    int32_t inflight = 0, max_inflight_seen = 0;
    int64_t submitted = 0, completed = 0, failed = 0, deferred = 0;
    std::atomic<int64_t> merged_launches{0}, merged_requests{0};
    std::vector<double> lat;           // completed since the last stats reset

    double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
};

namespace {

void CUDART_CB on_done(void* p) {
    Req* r = (Req*)p;
    up_serve* s = r->owner;
    const double t = s->now_ms();
    {
        std::lock_guard<std::mutex> g(s->mu);
        r->done_ms = t;
        r->state = UP_REQ_DONE;
        s->inflight--;
        s->completed++;
        s->lat.push_back(t - r->arrival_ms);
    }
    s->done_cv.notify_all();
    s->cv.notify_all();
}

// Bytes a request needs while it runs: its outputs (plus the err slot) and,
// for queries, the accumulator scratch up_query_launch allocates.
void size_request(Req& r, double heavy_work) {
    const GeneratedModule& g = r.module->jm.gen;
    r.part_off.clear();
    r.part_bytes.clear();
    int64_t off = kAlign;  // the first 256 bytes hold the err word
    if (!r.module->is_query) {
        r.part_off.push_back(off);
        r.part_bytes.push_back(r.rows * (int64_t)g.out_bytes);
        off += pad(r.rows * (int64_t)g.out_bytes);
        r.bytes = off;
    } else {
        for (int k = 0; k < g.n_aggs; k++) {
            const int64_t w = g.agg_kind[k] == UP_AGG_COUNT ? 8 : UP_AGG_DECIMAL_BYTES;
            r.part_off.push_back(off);
            r.part_bytes.push_back((int64_t)r.n_groups * w);
            off += pad((int64_t)r.n_groups * w);
        }
        const int64_t accw = std::max(g.acc_words_per_group, 1);
        r.bytes = off + pad((int64_t)r.n_groups * accw * 4 + 16) + pad((int64_t)r.n_groups * 8);
    }
    r.out_bytes = off;
    r.heavy = heavy_work > 0 && (double)r.rows * (double)g.work_per_row > heavy_work;
}

// Launch one admitted request on its stream (scheduler thread, lock not held).
void launch(up_serve* s, Req* r) {
    cudaStream_t st = r->stream;
    up_status status = UP_OK;
    cudaError_t e = cudaMallocAsync(&r->mem, (size_t)r->out_bytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r->mem, 0, 4, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        status = UP_ERR_CUDA;
        r->mem = nullptr;
    }
    uint32_t* err = (uint32_t*)r->mem;
    if (status == UP_OK) {
        if (!r->module->is_query) {
            status = expr_launch_ex(r->module, r->in.data(), (int32_t)r->in.size(), r->rows,
                                    (uint8_t*)r->mem + r->part_off[0], err, st, r->heavy);
        } else {
            std::vector<void*> outs;
            for (size_t k = 0; k < r->part_off.size(); k++) outs.push_back((uint8_t*)r->mem + r->part_off[k]);
            status = query_launch_ex(r->module, r->in.data(), (int32_t)r->in.size(), r->rows, r->group_ids,
                                     r->n_groups, outs.data(), err, st, r->heavy);
        }
    }
    if (status == UP_OK) {
        e = cudaMemcpyAsync(r->host_err, err, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaLaunchHostFunc(st, on_done, r);
        if (e != cudaSuccess) {
            cudaGetLastError();
            status = UP_ERR_CUDA;
        }
    }
    if (status != UP_OK) {
        std::lock_guard<std::mutex> g(s->mu);
        r->state = UP_REQ_FAILED;
        r->done_ms = s->now_ms();
        s->inflight--;
        s->failed++;
        s->done_cv.notify_all();
    }
}

// Launch requests of one expression module as one merged kernel on the
// first request's stream (scheduler thread, lock not held).
void launch_merged(up_serve* s, std::vector<Req*>& g) {
    cudaStream_t st = g[0]->stream;
    std::vector<up_column> in;
    std::vector<int64_t> rows;
    std::vector<void*> outs;
    std::vector<uint32_t*> errs;
    std::vector<Req*> ok;
    for (Req* r : g) {
        r->stream = st;
        cudaError_t e = cudaMallocAsync(&r->mem, (size_t)r->out_bytes, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(r->mem, 0, 4, st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            r->mem = nullptr;
            std::lock_guard<std::mutex> lk(s->mu);
            r->state = UP_REQ_FAILED;
            r->done_ms = s->now_ms();
            s->inflight--;
            s->failed++;
            s->done_cv.notify_all();
            continue;
        }
        in.insert(in.end(), r->in.begin(), r->in.end());
        rows.push_back(r->rows);
        outs.push_back((uint8_t*)r->mem + r->part_off[0]);
        errs.push_back((uint32_t*)r->mem);
        ok.push_back(r);
    }
    if (ok.empty()) return;
    const int n_in = (int)ok[0]->in.size();
    up_status status = up_expr_launch_many(ok[0]->module, in.data(), n_in, rows.data(), (int32_t)ok.size(),
                                           outs.data(), errs.data(), st);
    s->merged_launches++;
    s->merged_requests += (int64_t)ok.size();
    for (Req* r : ok) {
        cudaError_t e = status == UP_OK ? cudaMemcpyAsync(r->host_err, r->mem, 4, cudaMemcpyDeviceToHost, st)
                                        : cudaErrorUnknown;
        if (e == cudaSuccess) e = cudaLaunchHostFunc(st, on_done, r);
        if (e != cudaSuccess) {
            cudaGetLastError();
            std::lock_guard<std::mutex> lk(s->mu);
            r->state = UP_REQ_FAILED;
            r->done_ms = s->now_ms();
            s->inflight--;
            s->failed++;
            s->done_cv.notify_all();
        }
    }
}

// Same-module expression requests of one dispatch (at least two, contiguous
// columns, not heavy) become merged launches; the rest launch one by one.
void dispatch(up_serve* s, std::vector<Req*>& batch) {
    if (!s->opts.merge) {
        for (Req* r : batch) launch(s, r);
        return;
    }
    std::unordered_map<up_module*, std::vector<Req*>> by_mod;
    std::vector<Req*> single;
    for (Req* r : batch) {
        bool mergeable = !r->module->is_query && !r->heavy && r->rows > 0 && r->module->jm.gen.multi_rows > 0;
        for (const up_column& c : r->in)
            mergeable = mergeable && c.data && c.n_blocks <= 0 && !c.indices && !c.nullable;
        if (mergeable) by_mod[r->module].push_back(r);
        else single.push_back(r);
    }
    for (auto& kv : by_mod) {
        if (kv.second.size() >= 2) launch_merged(s, kv.second);
        else single.push_back(kv.second[0]);
    }
    for (Req* r : single) launch(s, r);
}

void scheduler(up_serve* s) {
    cudaSetDevice(s->device);
    std::vector<Req*> batch;
    for (;;) {
        batch.clear();
        {
            std::unique_lock<std::mutex> lk(s->mu);
            bool waited_for_memory = false;
            bool window_used = false;
            for (;;) {
                if (s->stop) return;
                // admit in arrival order while memory and the in-flight cap allow
                while (!s->queue.empty() && s->inflight < s->opts.max_inflight && !s->free_slots.empty()) {
                    Req* r = s->queue.front();
                    if (s->outstanding + r->bytes > s->budget) {
                        if (!waited_for_memory) s->deferred++;
                        waited_for_memory = true;
                        break;
                    }
                    s->queue.pop_front();
                    s->outstanding += r->bytes;
                    s->max_outstanding = std::max(s->max_outstanding, s->outstanding);
                    s->inflight++;
                    s->max_inflight_seen = std::max(s->max_inflight_seen, s->inflight);
                    const int slot = s->free_slots.back();
                    s->free_slots.pop_back();
                    r->host_err = s->pinned + slot;
                    *r->host_err = 0u;
                    s->slot_of[r->host_err] = slot;
                    r->stream = r->heavy ? s->heavy_streams[s->next_heavy++ % s->heavy_streams.size()]
                                         : s->streams[s->next_stream++ % s->streams.size()];
                    r->state = UP_REQ_RUNNING;
                    batch.push_back(r);
                    if ((int)batch.size() >= s->opts.max_batch) break;
                }
                if (!batch.empty()) {
                    // continuous batching window: wait a little for more arrivals to admit with these
                    if (s->opts.batch_window_us > 0 && (int)batch.size() < s->opts.max_batch && !window_used) {
                        window_used = true;
                        s->cv.wait_for(lk, std::chrono::duration<double, std::micro>(s->opts.batch_window_us));
                        continue;
                    }
                    break;
                }
                s->cv.wait(lk);
            }
        }
        dispatch(s, batch);
    }
}

}  // namespace

extern "C" {

up_status up_serve_create(const up_serve_opts* opts, up_serve** out) {
    if (!out) return fail(UP_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    auto s = std::make_unique<up_serve>();
    if (opts) s->opts = *opts;
    if (s->opts.n_streams <= 0) s->opts.n_streams = 8;
    if (s->opts.max_inflight <= 0) s->opts.max_inflight = 1024;
    if (s->opts.reserve_bytes <= 0) s->opts.reserve_bytes = 2ll << 30;
    if (s->opts.max_batch <= 0) s->opts.max_batch = 256;
    cudaError_t e = cudaGetDevice(&s->device);
    size_t fr = 0, tot = 0;
    if (e == cudaSuccess) e = cudaMemGetInfo(&fr, &tot);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(UP_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    s->budget = std::max<int64_t>(0, (int64_t)fr - s->opts.reserve_bytes);
    if (s->opts.memory_cap_bytes > 0) s->budget = std::min(s->budget, s->opts.memory_cap_bytes);
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    // n_streams in total (the hardware has 8 work queues by default; more
    // streams alias onto them): a quarter low-priority for heavy requests
    const int n_heavy = s->opts.heavy_work > 0 ? std::max(1, s->opts.n_streams / 4) : 0;
    const int n_light = std::max(1, s->opts.n_streams - n_heavy);
    for (int i = 0; i < n_light + n_heavy; i++) {
        cudaStream_t st;
        const bool hv = i >= n_light;
        if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hv ? least : greatest) != cudaSuccess) {
            cudaGetLastError();
            for (auto x : s->streams) cudaStreamDestroy(x);
            for (auto x : s->heavy_streams) cudaStreamDestroy(x);
            return fail(UP_ERR_CUDA, "cudaStreamCreate failed");
        }
        (hv ? s->heavy_streams : s->streams).push_back(st);
    }
    if (cudaMallocHost((void**)&s->pinned, sizeof(uint32_t) * (size_t)s->opts.max_inflight) != cudaSuccess) {
        cudaGetLastError();
        for (auto x : s->streams) cudaStreamDestroy(x);
        return fail(UP_ERR_NO_MEMORY, "pinned error slots");
    }
    for (int i = s->opts.max_inflight - 1; i >= 0; i--) s->free_slots.push_back(i);
    s->t0 = Clock::now();
    up_serve* raw = s.release();
    raw->worker = std::thread(scheduler, raw);
    *out = raw;
    return UP_OK;
}

double up_serve_clock_ms(const up_serve* s) { return s ? s->now_ms() : 0.0; }

up_status up_serve_submit(up_serve* s, const up_serve_request* req, int64_t* id) {
    if (!s || !req || !id || !req->module) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    if (req->rows < 0 || req->n_in < 0 || (req->n_in > 0 && !req->in)) return fail(UP_ERR_INVALID_ARG, "bad inputs");
    if (req->module->is_query && (req->n_groups < 0 || (req->rows > 0 && !req->group_ids)))
        return fail(UP_ERR_INVALID_ARG, "query request without group ids");
    auto r = std::make_unique<Req>();
    r->module = req->module;
    r->in.assign(req->in, req->in + req->n_in);
    r->rows = req->rows;
    r->group_ids = req->group_ids;
    r->n_groups = req->n_groups;
    r->owner = s;
    size_request(*r, s->opts.heavy_work);
    std::lock_guard<std::mutex> g(s->mu);
    if (r->bytes > s->budget) return fail(UP_ERR_NO_MEMORY, "request larger than the session's memory budget");
    r->arrival_ms = req->arrival_ms >= 0 ? req->arrival_ms : s->now_ms();
    r->id = s->next_id++;
    *id = r->id;
    s->queue.push_back(r.get());
    s->reqs[r->id] = std::move(r);
    s->submitted++;
    s->cv.notify_all();
    return UP_OK;
}

up_status up_serve_poll(up_serve* s, int64_t id, int32_t* state, double* latency_ms) {
    if (!s) return fail(UP_ERR_INVALID_ARG, "session is NULL");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(UP_ERR_INVALID_ARG, "unknown request");
    const Req& r = *it->second;
    if (state) *state = r.state;
    if (latency_ms) *latency_ms = (r.state == UP_REQ_DONE || r.state == UP_REQ_FAILED) ? r.done_ms - r.arrival_ms : -1;
    return UP_OK;
}

up_status up_serve_wait(up_serve* s, int64_t id, double timeout_ms, int32_t* state) {
    if (!s) return fail(UP_ERR_INVALID_ARG, "session is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(UP_ERR_INVALID_ARG, "unknown request");
    Req* r = it->second.get();
    auto done = [&] { return r->state == UP_REQ_DONE || r->state == UP_REQ_FAILED; };
    if (timeout_ms < 0) s->done_cv.wait(lk, done);
    else s->done_cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done);
    if (state) *state = r->state;
    return UP_OK;
}

up_status up_serve_result(up_serve* s, int64_t id, int32_t part, void** out, int64_t* bytes, uint32_t* err_word) {
    if (!s) return fail(UP_ERR_INVALID_ARG, "session is NULL");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(UP_ERR_INVALID_ARG, "unknown request");
    const Req& r = *it->second;
    if (r.state != UP_REQ_DONE) return fail(UP_ERR_INVALID_ARG, "request not finished");
    if (part < 0 || part >= (int)r.part_off.size()) return fail(UP_ERR_INVALID_ARG, "no such output part");
    if (out) *out = (uint8_t*)r.mem + r.part_off[part];
    if (bytes) *bytes = r.part_bytes[part];
    if (err_word) *err_word = *r.host_err;
    return UP_OK;
}

up_status up_serve_release(up_serve* s, int64_t id) {
    if (!s) return fail(UP_ERR_INVALID_ARG, "session is NULL");
    std::unique_ptr<Req> r;
    {
        std::lock_guard<std::mutex> g(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) return fail(UP_ERR_INVALID_ARG, "unknown request");
        if (it->second->state == UP_REQ_QUEUED || it->second->state == UP_REQ_RUNNING)
            return fail(UP_ERR_INVALID_ARG, "request still pending");
        r = std::move(it->second);
        s->reqs.erase(it);
        if (r->host_err) {
            s->free_slots.push_back(s->slot_of[r->host_err]);
            s->slot_of.erase(r->host_err);
        }
        if (r->stream) s->outstanding -= r->bytes;
    }
    if (r->mem) cudaFreeAsync(r->mem, r->stream);
    s->cv.notify_all();
    return UP_OK;
}

up_status up_serve_stats_get(up_serve* s, int32_t reset, up_serve_stats* out) {
    if (!s || !out) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    std::vector<double> v;
    {
        std::lock_guard<std::mutex> g(s->mu);
        memset(out, 0, sizeof *out);
        out->submitted = s->submitted;
        out->completed = s->completed;
        out->failed = s->failed;
        out->deferred = s->deferred;
        out->outstanding_bytes = s->outstanding;
        out->max_outstanding_bytes = s->max_outstanding;
        out->budget_bytes = s->budget;
        out->max_inflight_seen = s->max_inflight_seen;
        out->merged_launches = s->merged_launches.load();
        out->merged_requests = s->merged_requests.load();
        v = s->lat;
        if (reset) {
            s->lat.clear();
            s->max_inflight_seen = s->inflight;
            s->max_outstanding = s->outstanding;
            s->deferred = 0;
        }
    }
    if (!v.empty()) {
        std::sort(v.begin(), v.end());
        auto q = [&](double f) { return v[std::min(v.size() - 1, (size_t)(f * (double)(v.size() - 1) + 0.5))]; };
        double sum = 0;
        for (double x : v) sum += x;
        out->p50_ms = q(0.50);
        out->p95_ms = q(0.95);
        out->p99_ms = q(0.99);
        out->mean_ms = sum / (double)v.size();
        out->max_ms = v.back();
    }
    return UP_OK;
}

void up_serve_destroy(up_serve* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    std::vector<cudaStream_t> all = s->streams;
    all.insert(all.end(), s->heavy_streams.begin(), s->heavy_streams.end());
    for (auto st : all) cudaStreamSynchronize(st);
    for (auto& kv : s->reqs)
        if (kv.second->mem) cudaFreeAsync(kv.second->mem, kv.second->stream);
    for (auto st : all) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (s->pinned) cudaFreeHost(s->pinned);
    delete s;
}

}  // extern "C"
