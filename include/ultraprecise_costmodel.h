/*
 * ultraprecise_costmodel.h — the learned cost model of the decimal kernels.
 *
 * No counterpart in the reference (it picks one kernel shape per expression
 * with fixed rules: AriesDecimal<LEN> with LEN from a width table,
 * AriesEngineShell.cpp:678-684, and the XMP threads-per-instance fixed at
 * compile time, decimal.hxx:61).  Here a small multilayer perceptron predicts
 * the run time of an expression launch from features of the expression and
 * the launch (rows, threads per value, limb widths, multiply and divide work,
 * bytes per row); it is trained on the GPU by this library's own forward,
 * backward and Adam kernels on kernel times measured on the device, and it
 * chooses the threads per value of an expression (one thread per value or a
 * cooperative group of 2..32) by the lowest predicted time.  It never touches
 * the arithmetic: every choice computes the same bytes.
 *
 * Network: UP_CM_FEATURES inputs -> UP_CM_HIDDEN -> UP_CM_HIDDEN -> 1, SiLU
 * activations, fp32; inputs and target (natural log of milliseconds) are
 * standardised with statistics taken at training time.
 */
#ifndef ULTRAPRECISE_COSTMODEL_H_
#define ULTRAPRECISE_COSTMODEL_H_

#include "ultraprecise.h"

#ifdef __cplusplus
extern "C" {
#endif

#define UP_CM_FEATURES 16
#define UP_CM_HIDDEN 64
/* parameters: W1[F][H], b1[H], W2[H][H], b2[H], W3[H], b3 */
#define UP_CM_PARAMS (UP_CM_FEATURES * UP_CM_HIDDEN + UP_CM_HIDDEN + UP_CM_HIDDEN * UP_CM_HIDDEN + UP_CM_HIDDEN + \
                      UP_CM_HIDDEN + 1)
#define UP_CM_BATCH_MAX 128

typedef struct up_costmodel up_costmodel;

/* A model with seeded random parameters (He-style scaling). */
up_status up_costmodel_create(uint64_t seed, up_costmodel** out);
void up_costmodel_release(up_costmodel* m);

/* Features of launching an expression over `rows` rows with
 * `threads_per_value` threads per value (1, 2, 4, 8, 16 or 32).  No GPU
 * needed.  *coop_ok (may be NULL) receives 1 when the expression has a
 * cooperative form (threads_per_value > 1 is possible), else 0. */
up_status up_costmodel_expr_features(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                                     const up_col_type* cols, int32_t n_cols, int32_t threads_per_value,
                                     int64_t rows, float* features, int32_t* coop_ok);

/* Train on n samples (HOST arrays: features[n][UP_CM_FEATURES], targets[n] =
 * log(ms)): standardise both, then `epochs` passes of shuffled mini-batches of
 * `batch` samples (<= UP_CM_BATCH_MAX), one GPU kernel per step (forward,
 * backward and Adam update in one CTA).  *final_loss (may be NULL) receives
 * the mean squared error over all samples after training, in standardised
 * units.  Synchronises the model's stream. */
up_status up_costmodel_train(up_costmodel* m, const float* features, const float* targets, int32_t n,
                             int32_t epochs, int32_t batch, float lr, uint64_t seed, float* final_loss);

/* Predicted log(ms) of n samples (HOST arrays), by the GPU forward kernel. */
up_status up_costmodel_predict(up_costmodel* m, const float* features, int32_t n, float* log_ms);

/* Gradients of the mean squared error (mean over the n <= UP_CM_BATCH_MAX
 * samples) of the raw network (no standardisation) at the current
 * parameters, computed by the training kernel without the update: grads
 * receives UP_CM_PARAMS floats, *loss the error.  For checking the backward
 * pass. */
up_status up_costmodel_gradients(up_costmodel* m, const float* features, const float* targets, int32_t n,
                                 float* grads, float* loss);

/* Parameters (UP_CM_PARAMS floats, the layout above) and the standardisation
 * statistics (mean and std of each feature, then of the target). */
up_status up_costmodel_get_params(const up_costmodel* m, float* params, float* norm /* 2*F+2 or NULL */);
up_status up_costmodel_set_params(up_costmodel* m, const float* params, const float* norm /* or NULL */);

/* Threads per value with the lowest predicted time for launching the
 * expression over `rows` rows, among 1 and (when it has a cooperative form)
 * 2..32; *pred_ms (may be NULL) the predicted time. */
up_status up_costmodel_choose_tpv(up_costmodel* m, const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                                  const up_col_type* cols, int32_t n_cols, int64_t rows, int32_t* tpv,
                                  float* pred_ms);

/* Ensembles: add a copy of `other`'s trained network (and standardisation)
 * to `m`; predictions then average the log ms of m's network and every
 * member (independently trained networks disagree where data is thin). */
up_status up_costmodel_add_member(up_costmodel* m, const up_costmodel* other);

/* Guard the choice: up_costmodel_choose_tpv keeps the width rule's threads
 * per value unless the model predicts the best choice saves at least
 * `margin` (0 <= margin < 1) of the rule's time.  0 (the default): the
 * model's lowest prediction. */
up_status up_costmodel_set_guard(up_costmodel* m, float margin);

/* Make `m` (or NULL: none) the model that up_module_compile consults when
 * opts->threads_per_value is 0 (automatic): the threads per value with the
 * lowest predicted time for UP_CM_ROWS_HINT rows.  Without a model the
 * automatic choice is the width rule (cooperative from 96 limbs for
 * expressions without division).  The model must outlive its use here. */
#define UP_CM_ROWS_HINT (1 << 20)
up_status up_costmodel_set_default(up_costmodel* m);

#ifdef __cplusplus
}
#endif
#endif
