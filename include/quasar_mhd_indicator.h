/*
 * Learned troubled-cell indicator for the MP reconstruction.  No counterpart
 * in the reference; its labels are the reference limiter's own decisions
 * (numerics/mp_limiter.hpp:71-224) taken in the solver's reconstruction.
 *
 * Network: 200 -> 64 -> 64 -> 1 with GELU, BF16 weights, FP32 accumulation on
 * the tensor cores.  Inputs: the 8 primitives (rho, vx, vy, vz, p, bx, by, bz,
 * collocated field) of the 5 x 5 cell stencil, normalised by the centre cell:
 * (rho/rho_c - 1, (v - v_c)/a_c, p/p_c - 1, (B - B_c)/(sqrt(rho_c) a_c)),
 * a_c the centre sound speed; feature index = 8 * (5 * (dj + 2) + (di + 2)) + k.
 * Parameters (QMHD_INDICATOR_PARAMS floats): w1 [64][200], b1 [64],
 * w2 [64][64], b2 [64], w3 [64], b3.  Same status conventions as quasar_mhd.h.
 */
#ifndef QUASAR_MHD_INDICATOR_H
#define QUASAR_MHD_INDICATOR_H

#include <stddef.h>

#include "quasar_mhd.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QMHD_INDICATOR_FEATURES 200
#define QMHD_INDICATOR_HIDDEN 64
#define QMHD_INDICATOR_PARAMS 17089

typedef struct qmhd_indicator qmhd_indicator;

/* Glorot-uniform weights from `seed`, zero biases. */
int qmhd_indicator_create(unsigned long long seed, qmhd_indicator** out);
void qmhd_indicator_destroy(qmhd_indicator* ind);
int qmhd_indicator_get_params(qmhd_indicator* ind, float* params, size_t n);
int qmhd_indicator_set_params(qmhd_indicator* ind, const float* params, size_t n);

/* Logits of `rows` host feature rows (rows x 200 floats, rounded to BF16). */
int qmhd_indicator_forward(qmhd_indicator* ind, const float* features, long long rows,
                           float* logits);

/* Mean weighted binary cross-entropy of host rows (positives weighted by
 * pos_weight) and its gradient (QMHD_INDICATOR_PARAMS floats, parameter
 * packing), from the tensor-core backward pass; no parameter update. */
int qmhd_indicator_gradient(qmhd_indicator* ind, const float* features,
                            const unsigned char* labels, long long rows, float pos_weight,
                            float* grad, size_t n, double* loss);

/* Append every interior cell of the solver's live state to the training set:
 * its feature row and its label, 1 when a face state whose stencil is
 * centred on the cell, as the solver's own MP reconstruction (mp5/mp7)
 * limits it in characteristic fields, departs from the unlimited
 * component-wise interpolation by more than `tol` of the state's scale
 * (largest relative difference over rho, momentum against sqrt(2 rho E),
 * energy, field against sqrt(2 E)).  Where no face departs more than tol the
 * learned step's fast path reproduces the plain step within tol.  (The
 * early-accept test of numerics/mp_limiter.hpp:84-106 alone fails in nearly
 * every cell: near-constant fields fail it by sign noise while the limiter
 * moves them by rounding only.)  A negative tol selects the literal label
 * instead: 1 when the MP limiter fired (changed the unlimited value, the
 * negation of the early accept of mp_limiter.hpp:84-106) on any
 * characteristic field of such a face state. */
int qmhd_indicator_collect(qmhd_indicator* ind, qmhd_solver* solver, float tol);
long long qmhd_indicator_rows(const qmhd_indicator* ind);
/* The collected labels (n = qmhd_indicator_rows bytes, collection order:
 * per collected state its interior cells row by row). */
int qmhd_indicator_labels(const qmhd_indicator* ind, unsigned char* labels, long long n);
int qmhd_indicator_clear(qmhd_indicator* ind);

/* Adam (beta 0.9 / 0.999) over random 128-row tiles, `tiles_per_step` tiles
 * per step; one tile in `holdout`, chosen by a hash of the tile index, is held
 * out (0 = none).  *loss = mean
 * training loss of the last epoch. */
int qmhd_indicator_train(qmhd_indicator* ind, int epochs, int tiles_per_step, float lr,
                         float pos_weight, int holdout, unsigned long long seed, double* loss);
/* Recall of limiter firings and fraction of rows flagged (logit > threshold)
 * on the held-out tiles. */
int qmhd_indicator_evaluate(qmhd_indicator* ind, float threshold, int holdout, double* recall,
                            double* flagged, long long* positives, long long* total);
int qmhd_indicator_threshold_for_recall(qmhd_indicator* ind, double recall, int holdout,
                                        float* threshold);

/* Learned mode of a solver (mp5 / mp7): once per step the indicator scores
 * the live state; faces next to a cell scored above `threshold` (or without
 * a full stencil) keep the characteristic MP reconstruction in every stage,
 * all other faces take the unlimited component-wise interpolation, which
 * equals the characteristic result wherever the limiter would not fire.
 * ind = NULL restores the plain step.  The indicator must outlive this use. */
int qmhd_solver_set_indicator(qmhd_solver* solver, const qmhd_indicator* ind, float threshold);
/* The same learned mode for every instance of a batch (quasar_mhd_batch.h):
 * one batched indicator launch per step over all instances, their face lists
 * and the two reconstruction passes inside the batched step. */
struct qmhd_batch;
int qmhd_batch_set_indicator(struct qmhd_batch* batch, const qmhd_indicator* ind,
                             float threshold);
/* Faces on the full-reconstruction lists of the last learned step. */
int qmhd_solver_learned_face_counts(qmhd_solver* solver, long long* x_faces, long long* y_faces);

#ifdef __cplusplus
}
#endif

#endif /* QUASAR_MHD_INDICATOR_H */
