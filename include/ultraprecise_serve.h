/*
 * ultraprecise_serve.h — serving loop for decimal queries over resident columns.
 *
 * No counterpart in the reference (its engine runs one query at a time and
 * synchronises after every kernel, DynamicKernel.cu:281-338).  A session keeps
 * a pool of CUDA streams and one scheduler thread.  Clients submit requests
 * (a compiled expression or query module over device columns that stay
 * resident in HBM); the scheduler admits them in arrival order while the
 * session's device-memory budget (free memory at creation minus a reserve,
 * optionally capped) covers their outputs and scratch, and launches every
 * admitted request at once across the streams, while earlier ones still run
 * (continuous batching); requests of the same expression module admitted in
 * one dispatch share one merged launch (opts.merge), and an optional window
 * lets a dispatch wait briefly for more arrivals to merge.  Each request's completion time is stamped by a host
 * callback on its stream; latency = completion - arrival.  Results are
 * byte-identical to launching the same module alone.
 */
#ifndef ULTRAPRECISE_SERVE_H_
#define ULTRAPRECISE_SERVE_H_

#include "ultraprecise.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct up_serve up_serve;

typedef struct up_serve_opts {
    int32_t n_streams;         /* launch streams in total, a quarter of them for heavy requests (0 = 8) */
    int32_t max_inflight;      /* launched, not yet completed (0 = 1024) */
    int64_t memory_cap_bytes;  /* cap on outstanding request memory (0 = the free-memory budget) */
    int64_t reserve_bytes;     /* device memory left free (0 = 2 GiB) */
    double heavy_work;         /* > 0: estimated limb work (rows x per-row work) above which a request runs on a
                                  low-priority stream with one CTA per tile; <= 0: off (all streams equal) */
    int32_t merge;             /* 1: requests of one expression module admitted together run as one merged
                                  launch (up_expr_launch_many); 0: one launch per request */
    int32_t max_batch;         /* most requests the scheduler admits per dispatch (0 = 256) */
    double batch_window_us;    /* > 0: after the first request of a dispatch, wait up to this long for more
                                  arrivals to admit with it (continuous batching window); 0: dispatch at once */
} up_serve_opts;

typedef struct up_serve_request {
    up_module* module;         /* from up_module_compile or up_query_compile; kept alive by the caller */
    const up_column* in;       /* resident device columns (the descriptors are copied) */
    int32_t n_in;
    int64_t rows;
    const int32_t* group_ids;  /* query modules: DEVICE int32 ids in [0, n_groups) */
    int32_t n_groups;
    double arrival_ms;         /* arrival on the session clock; < 0 means "now" */
} up_serve_request;

enum { UP_REQ_QUEUED = 0, UP_REQ_RUNNING = 1, UP_REQ_DONE = 2, UP_REQ_FAILED = 3 };

up_status up_serve_create(const up_serve_opts* opts, up_serve** out);

/* Milliseconds since the session was created (the clock of arrival_ms). */
double up_serve_clock_ms(const up_serve* s);

/* Queue a request; *id identifies it until up_serve_release.  Requests whose
 * memory exceeds the whole budget fail with UP_ERR_NO_MEMORY at submit. */
up_status up_serve_submit(up_serve* s, const up_serve_request* req, int64_t* id);

/* State and, once done, latency (completion - arrival) in ms. */
up_status up_serve_poll(up_serve* s, int64_t id, int32_t* state, double* latency_ms);

/* Block until the request is done or failed, or timeout_ms passes (< 0: no limit). */
up_status up_serve_wait(up_serve* s, int64_t id, double timeout_ms, int32_t* state);

/* Output `part` of a finished request (0 for an expression; aggregate k of a
 * query) as a device pointer and byte size, and the request's row-error word. */
up_status up_serve_result(up_serve* s, int64_t id, int32_t part, void** out, int64_t* bytes,
                          uint32_t* err_word);

/* Free a finished request's memory (stream-ordered) and forget it. */
up_status up_serve_release(up_serve* s, int64_t id);

typedef struct up_serve_stats {
    int64_t submitted, completed, failed;
    int64_t deferred;              /* admission checks that had to wait for memory */
    int64_t outstanding_bytes, max_outstanding_bytes, budget_bytes;
    int32_t max_inflight_seen;
    int32_t pad;
    double p50_ms, p95_ms, p99_ms, mean_ms, max_ms;   /* over requests completed since the last reset */
    int64_t merged_launches;       /* merged launches so far, and the requests they ran */
    int64_t merged_requests;
} up_serve_stats;

up_status up_serve_stats_get(up_serve* s, int32_t reset, up_serve_stats* out);

/* Stop the scheduler, wait for launched work, free everything. */
void up_serve_destroy(up_serve* s);

#ifdef __cplusplus
}
#endif
#endif
