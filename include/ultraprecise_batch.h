/*
 * ultraprecise_batch.h — batched persistent-kernel mode and its autotuner.
 *
 * No counterpart in the reference (it launches one JIT kernel per expression
 * and synchronises after each, DynamicKernel.cu:281-338).  Many independent
 * decimal tasks (projections, or grouped SUM/AVG/COUNT of an expression) are
 * compiled into one module; per precision band a persistent kernel pulls
 * (task, row tile) work items from a device queue, costliest tasks first, and
 * the whole step (queue reset, the band kernels on forked streams, the
 * aggregate finalisation) is captured once as a CUDA graph and replayed.
 * Tasks with many rows (opts.solo_rows) run as their own per-task kernels on
 * further forked streams of the same step, concurrently with the bands.
 * Results are byte-identical to running each task alone through
 * up_expr_launch / up_query_launch.
 */
#ifndef ULTRAPRECISE_BATCH_H_
#define ULTRAPRECISE_BATCH_H_

#include "ultraprecise.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct up_batch_task {
    const up_expr_node* nodes;
    int32_t n_nodes;
    int32_t root;
    const up_col_type* cols;
    int32_t n_cols;            /* <= 8 */
    int32_t agg_kind;          /* -1: projection (compact output); else UP_AGG_SUM/AVG/COUNT by group */
} up_batch_task;

typedef struct up_batch_opts {
    int32_t autotune;          /* 1: sweep launch shapes per band on the first launch (cached on disk) */
    int32_t block_threads;     /* 0 = default; else 64, 128 or 256 */
    int32_t ctas_per_sm;       /* 0 = default */
    int32_t tile_rows;         /* 0 = default rows per work item */
    int32_t use_graph;         /* 1: capture the step once as a CUDA graph and replay it */
    int32_t tpv_policy;        /* threads per value of projection tasks (aggregate tasks run one thread per
                                  value): 0 = automatic (the default cost model's choice when one is set,
                                  else the width rule); 1 = one thread per value; 2 = measured: the first
                                  launch times each projection task alone at every candidate threads per
                                  value on its bound inputs and keeps the fastest (cached on disk) */
    int64_t solo_rows;         /* tasks with at least this many rows run as their own kernels inside the
                                  same step (on forked streams); 0 = 262144, < 0 = never */
} up_batch_opts;

typedef struct up_batch up_batch;

/* Compile every task into one module (NVRTC, sm_100a; cached). */
up_status up_batch_create(const up_batch_task* tasks, int32_t n_tasks, const up_batch_opts* opts,
                          up_batch** out);

/* Bind a task's device buffers.  Projection: `out` holds rows * value_bytes.
 * Aggregate: group_ids (rows int32 in [0, n_groups)) and `out` holds
 * n_groups * 133 bytes (SUM/AVG) or n_groups int64 (COUNT).  Rebinding after
 * a launch drops the captured graph (the next launch captures again). */
up_status up_batch_bind(up_batch* b, int32_t task, const up_column* in, int32_t n_in, int64_t rows,
                        const int32_t* group_ids, int32_t n_groups, void* out);

/* Run every task once, stream-ordered.  The first launch after binding
 * allocates the work queue and aggregate scratch, tunes when asked, and
 * captures the graph; later launches replay it.  err_word may be NULL. */
up_status up_batch_launch(up_batch* b, uint32_t* err_word, void* stream);

/* Launch shape in use for a band (0 narrow, 1 mid, 2 wide): block threads,
 * CTAs per SM, rows per work item, and the tuned time in ms (0 if untuned). */
up_status up_batch_shape(const up_batch* b, int32_t band, int32_t* block_threads, int32_t* ctas_per_sm,
                         int32_t* tile_rows, double* tuned_ms);

/* Band (0..2) of a task and the result type of a projection task. */
up_status up_batch_task_type(const up_batch* b, int32_t task, int32_t* precision, int32_t* scale,
                             int32_t* value_bytes, int32_t* band);

/* Pin a projection task's threads per value (1, 2, 4, 8, 16 or 32; an
 * expression without a cooperative form stays at 1).  The module is rebuilt
 * on the next launch; the measured policy leaves pinned tasks alone. */
up_status up_batch_set_task_tpv(up_batch* b, int32_t task, int32_t threads_per_value);

/* Threads per value a task runs with (after the first launch under the
 * measured policy). */
up_status up_batch_task_tpv(const up_batch* b, int32_t task, int32_t* threads_per_value);

void up_batch_release(up_batch* b);

#ifdef __cplusplus
}
#endif
#endif
