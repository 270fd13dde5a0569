/*
 * Extensions of the B200 MHD solver with no counterpart in the reference:
 * measurement entry points used by bench.py and an allocation-free
 * diagnostic.  Same status conventions as quasar_mhd.h.
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
 * 0 control (step begin, dt; with an indicator attached also its inference
 * and the face lists), 1 reconstruction, 2 face flux, 3 cell EMF,
 * 4 corner EMF, 5 update, 6 ghost fill, 7 collocation + admissibility. */
int qmhd_solver_profile_step(qmhd_solver* solver, double* ms_by_phase, int n);

/* Measured FP64 FMA throughput of the current device in TFLOP/s. */
int qmhd_fp64_fma_peak(double* tflops);

/* Tile hooks of a decomposed domain (quasar_b200/tiles.py), the pieces the
 * reference's distributed runtime keeps inside its solver
 * (src/distributed/mhd_runtime.cpp: dt and admissibility reduced over the
 * owned cells, halos refreshed from the neighbours).
 *
 * qmhd_solver_set_owned_window: only interior cells [x0, x1) x [y0, y1)
 * (0 <= x0 < x1 <= nx, 0 <= y0 < y1 <= ny) enter the reductions that decide
 * dt (cfl_limit), positivity retries, the live-state preflights,
 * divergence_b_max and conserved_cell_totals; the other cells are halo.
 * The default window is every interior cell.
 *
 * qmhd_solver_write_halo: write a whole component (storage size, like
 * qmhd_solver_seed_state) whose interior values are finite and come from
 * the solver's own steps, e.g. the owned cells of neighbouring tiles: the
 * state stays solver-owned, so its solenoidality preflight stays the one of
 * a stepped state (a seeded state gets the stricter seeded-state test).
 * Ghost layers need not be finite; they are closed again before use. */
int qmhd_solver_set_owned_window(qmhd_solver* solver, int x0, int x1, int y0, int y1);
int qmhd_solver_write_halo(qmhd_solver* solver, const char* component, const double* values,
                           size_t n);

/* The halo exchange without the host round trip of whole components:
 *
 * qmhd_solver_gather_live: out[k] = live value of `component` at storage
 * index idx[k] (row-major padded storage, 0 <= idx[k] < storage size), for
 * k < n: what this tile sends to a neighbour.
 *
 * qmhd_solver_scatter_halo: live value at idx[k] = values[k], for k < n:
 * what this tile receives.  The values must be finite and come from the
 * solver's own steps (as for qmhd_solver_write_halo, the state stays
 * solver-owned); on a bad index or a non-finite value nothing is written
 * and the call fails with QMHD_INVALID_ARGUMENT.
 *
 * idx, out and values are DEVICE memory of the solver's device, each
 * inside one allocation (checked), and must be ready when the call is made
 * (their producer's stream synchronised).  Both calls return once the copy
 * finished. */
int qmhd_solver_gather_live(qmhd_solver* solver, const char* component, const long long* idx,
                            size_t n, double* out);
int qmhd_solver_scatter_halo(qmhd_solver* solver, const char* component, const long long* idx,
                             size_t n, const double* values);

/* Largest nx*ny accepted by qmhd_conserved_cell_totals_device. */
#define QMHD_TOTALS_DEVICE_MAX_CELLS 67108864LL

/* Mass and energy cell totals of caller-owned device arrays, allocating
 * nothing.  No counterpart in the reference: it is the compensated sum of
 * qmhd_solver_conserved_cell_totals (reference mhd_solver.cpp:1376-1382)
 * applied to the caller's own buffers instead of a solver's state.
 *
 * rho, energy: device memory of the calling thread's current device, in the
 *   solver's padded layout: (nx + 2 nghost) x (ny + 2 nghost) doubles, cell
 *   (i, j) at (i + nghost) + (nx + 2 nghost)(j + nghost); ghosts are ignored.
 * stream: a cudaStream_t of that device (NULL = the default stream).  The
 *   call orders its work after what is already queued on the stream, copies
 *   the two totals to *mass and *energy_total and synchronizes the stream.
 *
 * Scratch is a fixed 256 KiB device array inside the library (one per
 * device): nothing is allocated on the device, and nothing on the host
 * unless an error message is formatted.  nx*ny above
 * QMHD_TOTALS_DEVICE_MAX_CELLS returns QMHD_INVALID_ARGUMENT.  No part of the
 * scratch has to start at zero: each call writes every slot it reads.
 * rho and energy must be device or managed memory whose device is the
 * current one (managed memory whose device is another GPU is rejected).
 * Every call looks up the scratch address in the current context (a
 * cudaGetSymbolAddress, which allocates nothing), so a cudaDeviceReset
 * between calls is harmless.  Calls on one device share the one scratch
 * array: they hold a per-device lock from the lookup until their stream has
 * synchronized, so calls from several host threads take turns and never
 * overlap on the GPU (other processes have their own copy of the array).
 * Every call copies to pageable host memory and synchronizes its stream, so
 * it must not be made while any stream capture is active on the device. */
int qmhd_conserved_cell_totals_device(const double* rho, const double* energy, int nx, int ny,
                                      int nghost, void* stream, double* mass,
                                      double* energy_total);

#ifdef __cplusplus
}
#endif

#endif /* QUASAR_MHD_EXT_H */
