/*
 * C ABI of the B200 (sm_100a) 2-D ideal-MHD solver.
 *
 * Drop-in boundary for the reference's MHD solver binding: each entry point
 * replaces one method of quasar's `_core.mhd.MhdSolver2D`
 * (bindings/python/bind_mhd.cpp:589-647), which forwards to
 * quasar::mhd::MhdSolver2D (include/quasar/physics/mhd/mhd_solver.hpp:85-173).
 * Plain pointers and sizes only.  Host arrays are the reference's padded
 * storage: (nx + 2g) * (ny + 2g) doubles, flat index (i + g) + (nx + 2g)(j + g)
 * (include/quasar/core/grid.hpp:158-161), g = 4 for MP7, 3 for MP5, 2 for
 * MUSCL.
 *
 * Every function returns QMHD_OK or a negative status; qmhd_last_error()
 * gives the message of the calling thread's last failure.  The status codes
 * map the reference's exception types: std::invalid_argument ->
 * QMHD_INVALID_ARGUMENT, std::runtime_error -> QMHD_RUNTIME_ERROR; a CUDA
 * failure is QMHD_DEVICE_ERROR (the reference's DeviceError,
 * include/quasar/backend/device.hpp:23-35).
 */
#ifndef QUASAR_MHD_H
#define QUASAR_MHD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QMHD_OK 0
#define QMHD_INVALID_ARGUMENT (-1)
#define QMHD_RUNTIME_ERROR (-2)
#define QMHD_DEVICE_ERROR (-3)

#define QMHD_BC_PERIODIC 0
#define QMHD_BC_OUTFLOW 1
#define QMHD_BC_WALL 2

typedef struct qmhd_solver qmhd_solver;

/* Subset of quasar::mhd::MhdConfig (mhd_solver.hpp:50-83) that the device
 * evolution accepts: reconstruction "muscl_minmod" (2), "mp5" (5) or "mp7"
 * (7); riemann "hlld", ct "fd_ct_christlieb", integrator "ssprk3" and
 * positivity "troubled_cell" are implied.  boundary[] = x_lo, x_hi, y_lo,
 * y_hi, one QMHD_BC_* each, applied to both fluid and field
 * (boundary/mhd_boundary.hpp). */
typedef struct qmhd_config {
  int nx, ny;
  double lx, ly;
  double origin_x, origin_y;
  int reconstruction_order;
  double gamma;
  double cfl;
  int boundary[4];
} qmhd_config;

/* Last error message of the calling thread ("" if none). */
const char* qmhd_last_error(void);

/* MhdSolver2D(MhdConfig): mhd_solver.cpp:366-505. */
int qmhd_solver_create(const qmhd_config* config, qmhd_solver** out);
/* ~MhdSolver2D */
void qmhd_solver_destroy(qmhd_solver* solver);
/* grid(): extents and the resolved ghost width (mhd_solver.hpp:90). */
int qmhd_solver_grid(const qmhd_solver* solver, int* nx, int* ny, int* nghost);
/* grid().storage_size(): elements of one padded component array. */
long long qmhd_solver_storage_size(const qmhd_solver* solver);

/* seed_state(component, values): mhd_solver.cpp:521-541.  component is
 * "rho", "mx", "my", "mz", "energy", "bx"/"bx_face", "by"/"by_face",
 * "bz"/"bz_cell"; n must equal the storage size; values must be finite
 * (tested on the device after the copy; a rejected buffer leaves the live
 * state unchanged). */
int qmhd_solver_seed_state(qmhd_solver* solver, const char* component,
                           const double* values, size_t n);
/* state_component_to_host(component): mhd_solver.cpp:586-606.  "bx"/"by"
 * return the face-to-cell collocated field, "bx_face"/"by_face" the raw CT
 * arrays. */
int qmhd_solver_state_component_to_host(qmhd_solver* solver, const char* component,
                                        double* out, size_t n);

/* cfl_limit(): mhd_solver.cpp:1224-1321. */
int qmhd_solver_cfl_limit(qmhd_solver* solver, double* dt);
/* step(dt): rejects dt > cfl_limit() (mhd_solver.cpp:1384-1397). */
int qmhd_solver_step(qmhd_solver* solver, double dt);
/* step_unchecked(dt): mhd_solver.cpp:1399-1409. */
int qmhd_solver_step_unchecked(qmhd_solver* solver, double dt);
/* advance(t_end, dt): mhd_solver.cpp:1411-1441. */
int qmhd_solver_advance(qmhd_solver* solver, double t_end, double dt);
/* divergence_b_max(): mhd_solver.cpp:1323-1338. */
int qmhd_solver_divergence_b_max(qmhd_solver* solver, double* out);
/* conserved_cell_totals(): (mass, energy), mhd_solver.cpp:1376-1382. */
int qmhd_solver_conserved_cell_totals(qmhd_solver* solver, double* mass, double* energy);
/* last_positivity_substeps(): mhd_solver.hpp:99-101. */
int qmhd_solver_last_positivity_substeps(const qmhd_solver* solver);

/* Auto-dt run loop of the reference's CLI (python/quasar/mhd/cli.py:386-490:
 * dt = min(cfl_limit(), t_end - t); step_unchecked(dt); t += dt) run for up to
 * max_steps steps with dt kept on the device and the steps replayed as CUDA
 * graphs, so no host round trip happens per step.  *t is advanced in place;
 * *steps_taken receives the number of steps. */
int qmhd_solver_advance_auto(qmhd_solver* solver, double* t, double t_end, int max_steps,
                             int* steps_taken);

#ifdef __cplusplus
}
#endif

#endif /* QUASAR_MHD_H */
