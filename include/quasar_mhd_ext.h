/*
 * Measurement extensions of the B200 MHD solver (no counterpart in the
 * reference; used by bench.py).  Same status conventions as quasar_mhd.h.
 */
#ifndef QUASAR_MHD_EXT_H
#define QUASAR_MHD_EXT_H

#include "quasar_mhd.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QMHD_PROFILE_PHASES 8

/* Run `steps` device-resident auto-dt steps (CUDA graphs) bracketed by CUDA
 * events on the solver's stream; *ms = device time, *done = steps taken. */
int qmhd_solver_time_auto_steps(qmhd_solver* solver, int steps, double* ms, int* done);

/* One step with per-phase device times in ms (n >= QMHD_PROFILE_PHASES):
 * 0 control (step begin, dt), 1 reconstruction, 2 face flux, 3 cell EMF,
 * 4 corner EMF, 5 update, 6 ghost fill, 7 collocation + admissibility. */
int qmhd_solver_profile_step(qmhd_solver* solver, double* ms_by_phase, int n);

/* Measured FP64 FMA throughput of the current device in TFLOP/s. */
int qmhd_fp64_fma_peak(double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* QUASAR_MHD_EXT_H */
