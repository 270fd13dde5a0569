/*
 * Batched MHD instances on one GPU.  No counterpart in the reference, which
 * steps one instance per MhdSolver2D (physics/mhd/mhd_solver.hpp:85-173)
 * with host-driven launches (mhd_solver.cpp:1399-1409).
 *
 * A batch holds many independent instances (their own grid sizes, gamma and
 * boundaries; one reconstruction order, mp5 or mp7).  Each instance is a
 * full solver handle: seed, read, check and step it with the functions of
 * quasar_mhd.h.  qmhd_batch_advance steps every instance with its own
 * auto dt = min(cfl, 0.2) / max rate, with one persistent launch per phase
 * of each RK stage over all instances, the step replayed as a CUDA graph.
 * Each instance runs the device code of the single-instance step; inlined
 * into the batched kernels its multiply-adds may contract differently, so
 * results agree with stepping the instance alone to rounding.
 * Same status conventions as quasar_mhd.h.
 */
#ifndef QUASAR_MHD_BATCH_H
#define QUASAR_MHD_BATCH_H

#include "quasar_mhd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qmhd_batch qmhd_batch;

/* Tuned phases: 0 x reconstruction, 1 y reconstruction, 2 face flux, 3 cell
 * EMF, 4 corner EMF, 5 update, 6 collocation + admissibility, 7 x ghosts,
 * 8 y ghosts. */
#define QMHD_BATCH_PHASES 9

/* n >= 1 configurations; every reconstruction_order must be 5 or every one 7. */
int qmhd_batch_create(const qmhd_config* configs, int n, qmhd_batch** out);
void qmhd_batch_destroy(qmhd_batch* batch);
int qmhd_batch_size(const qmhd_batch* batch);
long long qmhd_batch_zones(const qmhd_batch* batch);

/* Instance i as a solver handle owned by the batch (qmhd_solver_destroy on
 * it does nothing); NULL for an index out of range. */
qmhd_solver* qmhd_batch_instance(qmhd_batch* batch, int i);

/* `steps` auto-dt steps of every instance.  An instance whose step needs the
 * positivity controller's retry completes it on the host, as
 * qmhd_solver_advance_auto does.  steps_taken (optional, n entries). */
int qmhd_batch_advance(qmhd_batch* batch, int steps, int* steps_taken);

/* Device time in ms of `steps` batched steps; *zone_updates = sum over
 * instances of nx * ny * steps taken on the device. */
int qmhd_batch_time_steps(qmhd_batch* batch, int steps, double* ms, long long* zone_updates);

/* Measure each phase's persistent grid (CTAs per SM, 0 = one CTA per tile)
 * on profiled steps of this batch and keep the fastest.  Every instance
 * advances by *trial_steps steps.  ctas_per_sm (optional) receives the
 * choice, QMHD_BATCH_PHASES entries. */
int qmhd_batch_autotune(qmhd_batch* batch, int* ctas_per_sm, int* trial_steps);
int qmhd_batch_set_tuning(qmhd_batch* batch, const int* ctas_per_sm);

/* One batched step with per-phase device times in ms (measurement hook, no
 * counterpart in the reference): entries 0 .. QMHD_BATCH_PHASES - 1 are the
 * tuned phases above, entry QMHD_BATCH_PHASES the rest (step begin and end;
 * in learned mode also the indicator and the face lists).
 * n >= QMHD_BATCH_PHASES + 1.  Every instance advances by one step. */
int qmhd_batch_profile_step(qmhd_batch* batch, double* ms_by_phase, int n);

#ifdef __cplusplus
}
#endif

#endif /* QUASAR_MHD_BATCH_H */
