/*
 * Learned troubled-cell indicator for the MP reconstruction.  No counterpart
 * in the reference; its labels are the reference's own limiter decisions
 * (the negation of the MP early-accept test, numerics/mp_limiter.hpp:84-106).
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

#ifdef __cplusplus
}
#endif

#endif /* QUASAR_MHD_INDICATOR_H */
