/*
 * Per-kernel launch interface of the B200 MHD step: the C ABI of the
 * reference's backend seam, include/quasar/physics/mhd/kernels.hpp, whose
 * launch_mhd_* functions the reference solver calls for every kernel of a
 * step (src/physics/mhd/mhd_solver.cpp:680-800).  Each entry point below
 * names the declaration it replaces (kernels.hpp:line).  quasar_mhd.h is the
 * other seam (the solver class); both drive the same sm_100a kernels.
 * launch_mhd_split_energy_residual (kernels.hpp:320-329) has no entry here:
 * it does nothing when the background field is off (mhd_split_energy.hip:252),
 * the only mode this library runs, so a forwarding layer defines it as that
 * no-op.
 *
 * Conventions, as the reference states them (kernels.hpp:18-25):
 *   - every pointer is device memory of the calling thread's current device,
 *     owned by the caller; nothing is allocated;
 *   - arrays are the padded SoA layout (nx + 2 nghost) x (ny + 2 nghost)
 *     doubles, cell (i, j) at (i + nghost) + (nx + 2 nghost)(j + nghost);
 *     x-face i of row j and y-face j of column i share cell (i, j)'s index;
 *   - work is queued on `stream` (a cudaStream_t; NULL = the default
 *     stream); functions that return a host scalar synchronize the stream;
 *   - flags[4] are the boundary modes x_lo, x_hi, y_lo, y_hi: 0 periodic,
 *     1 outflow, 2 conducting wall (BoundaryFlags4, kernels.hpp:49-51; the
 *     reference's axis and internal-tile modes are not supported);
 *   - nghost is the solver's ghost width for the configured order: 4 for
 *     MP7, 3 for MP5, 2 for MUSCL; order 1 (the positivity retry) runs on
 *     any of them;
 *   - status codes and qmhd_last_error() as in quasar_mhd.h; a cylindrical
 *     grid, an active background field or a partial face ownership is
 *     QMHD_INVALID_ARGUMENT (out of scope).
 *
 * Reductions write into `scratch`: caller-owned device memory of at least
 * QMHD_LAUNCH_SCRATCH_BYTES, 8-byte aligned, whose content need not be
 * initialised (the reference's block-partials buffer, kernels.hpp:477-481).
 * Calls that share one scratch must be serialised by the caller.
 */
#ifndef QUASAR_MHD_LAUNCH_H
#define QUASAR_MHD_LAUNCH_H

#include "quasar_mhd.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QMHD_LAUNCH_SCRATCH_BYTES 64

/* Grid2D (include/quasar/core/grid.hpp): extents, ghost width, spacings. */
typedef struct qmhd_grid {
  int nx, ny, nghost;
  double dx, dy;
} qmhd_grid;

/* MhdField2D (physics/mhd/mhd_field.hpp): rho, mx, my, mz, energy, bx_face,
 * by_face, bz_cell.  Also the flux and residual (dudt) records. */
typedef struct qmhd_field {
  double* comp[8];
} qmhd_field;

/* MhdInterfaceStates (numerics/interface_states.hpp): the left and right
 * conserved states of every face normal to one direction, stored at the
 * index of the face's high cell. */
typedef struct qmhd_iface {
  double* left[8];
  double* right[8];
} qmhd_iface;

/* EmfField2D (physics/mhd/mhd_field.hpp) as this library forms it: the upwind
 * face E_z of each direction with its one-dimensional "no jump" proof, the
 * cell-average E_z, and the corner E_z at the lower-left corner of each cell
 * (the reference's ez_edge). */
typedef struct qmhd_emf {
  double* face_ez_x;
  double* face_ez_y;
  int* no_jump_x;
  int* no_jump_y;
  double* cell_ez;
  double* corner_ez;
} qmhd_emf;

/* ScaledCflRate (kernels.hpp:483-486): true max rate = scaled_max_rate /
 * rate_scale.  This library always reports rate_scale 1; an aggregate that
 * overflows reports +inf. */
typedef struct qmhd_cfl_rate {
  double scaled_max_rate;
  double rate_scale;
} qmhd_cfl_rate;

/* launch_mhd_reconstruct (kernels.hpp:162-166): left/right conserved states
 * of every face normal to dir (0 x, 1 y) for scheme_order 1, 2, 5 or 7.
 * cell_bx, cell_by: caller scratch (padded arrays) that receives the
 * face-to-cell collocated field of u, which the reconstruction reads.
 * rate_only (the CFL path's flag) gives the same states, as in the reference,
 * where it only picks an admissibility predicate that forwards to the other. */
int qmhd_launch_reconstruct(const qmhd_grid* grid, const qmhd_field* u, double* cell_bx,
                            double* cell_by, int dir, const qmhd_iface* out,
                            int scheme_order, const int flags[4], double gamma, void* stream,
                            int rate_only);

/* launch_mhd_hlld_flux (kernels.hpp:186-194): Gauss-point HLLD face flux
 * (MP5/MP7), the face-state HLLD (order 2) or the LF retry flux (order 1,
 * hll_only = 1; the reference solver passes hll_only = (order <= 1)).
 * ownership: NULL or all ones. */
int qmhd_launch_hlld_flux(const qmhd_grid* grid, const qmhd_iface* iface, int dir,
                          const qmhd_field* flux_out, const int flags[4], double gamma,
                          void* stream, int hll_only, int scheme_order, const int ownership[4]);

/* launch_mhd_flux_difference (kernels.hpp:203-205): dudt += -(F_hi - F_lo)/d
 * over the interior cells, all eight slots. */
int qmhd_launch_flux_difference(const qmhd_grid* grid, const qmhd_field* flux, int dir,
                                const qmhd_field* dudt, void* stream, int cylindrical);

/* launch_mhd_ct_emf_prepare (kernels.hpp:274-280): upwind face E_z and
 * no-jump proofs of both directions from the interface states, and the
 * cell-average E_z of u (tensor Gauss quadrature for MP5/MP7).  cell_bx,
 * cell_by: caller scratch as in qmhd_launch_reconstruct. */
int qmhd_launch_ct_emf_prepare(const qmhd_grid* grid, const qmhd_field* u, double* cell_bx,
                               double* cell_by, const qmhd_iface* ifx, const qmhd_iface* ify,
                               const int flags[4], const qmhd_emf* emf, double gamma,
                               void* stream, int scheme_order, int hll_only);

/* launch_mhd_ct_emf_finish (kernels.hpp:281-284): corner E_z. */
int qmhd_launch_ct_emf_finish(const qmhd_grid* grid, const int flags[4], const qmhd_emf* emf,
                              void* stream, int scheme_order, int cylindrical);

/* launch_mhd_emf_curl_rate (kernels.hpp:307-309): overwrite dudt.bx_face
 * (i <= nx, j < ny) and dudt.by_face (i < nx, j <= ny) with the curl of the
 * corner E_z. */
int qmhd_launch_emf_curl_rate(const qmhd_grid* grid, const qmhd_emf* emf, const qmhd_field* dudt,
                              void* stream, int cylindrical);

/* launch_mhd_rk_stage (kernels.hpp:336-338): out = a un + b ustage + c_dt dudt;
 * operands with a zero weight are not read; (1, 0, 0) copies exactly.  out
 * may alias ustage. */
int qmhd_launch_rk_stage(const qmhd_grid* grid, const qmhd_field* out, const qmhd_field* un,
                         const qmhd_field* ustage, const qmhd_field* dudt, double a, double b,
                         double c_dt, void* stream);

/* launch_mhd_admissible_fraction (kernels.hpp:361-366): largest theta in
 * [0, 1] with rho > rho_floor and p > p_floor on base + theta (candidate -
 * base) in every interior cell; collocation_order 0 high-order, 1 two-face. */
int qmhd_launch_admissible_fraction(const qmhd_grid* grid, const qmhd_field* base,
                                    const qmhd_field* candidate, double rho_floor,
                                    double p_floor, double gamma, void* scratch,
                                    double* host_theta, void* stream, int collocation_order);

/* launch_mhd_cfl_max_rate (kernels.hpp:488-495): max over interior cells of
 * 0.5 (alpha_xlo + alpha_xhi)/dx + 0.5 (alpha_ylo + alpha_yhi)/dy from the
 * interface states (and their Gauss points for MP5/MP7). */
int qmhd_launch_cfl_max_rate(const qmhd_grid* grid, const qmhd_iface* ifx, const qmhd_iface* ify,
                             double gamma, void* scratch, qmhd_cfl_rate* host_rate, void* stream,
                             int scheme_order, int cylindrical, const int flags[4]);

/* launch_mhd_ct_divb_linf (kernels.hpp:509-512): max interior |div B|. */
int qmhd_launch_ct_divb_linf(const qmhd_grid* grid, const qmhd_field* u, void* scratch,
                             double* host_linf, void* stream, int cylindrical);

/* launch_mhd_ct_divb_relative_linf (kernels.hpp:530-533): the live-state
 * solenoidality preflight ratio. */
int qmhd_launch_ct_divb_relative_linf(const qmhd_grid* grid, const qmhd_field* u, void* scratch,
                                      double* host_linf, void* stream, int cylindrical,
                                      int solver_owned);

/* launch_mhd_fill_ghosts_fluid / _field (kernels.hpp:545-558): one side
 * (0 x_lo, 1 x_hi, 2 y_lo, 3 y_hi) with mode 0 periodic, 1 outflow, 2 wall;
 * fluid = rho, momentum, energy, bz_cell; field = bx_face, by_face. */
int qmhd_launch_fill_ghosts_fluid(const qmhd_grid* grid, const qmhd_field* u, int side, int mode,
                                  void* stream);
int qmhd_launch_fill_ghosts_field(const qmhd_grid* grid, const qmhd_field* u, int side, int mode,
                                  void* stream);

/* launch_mhd_collocate_face_to_cell (kernels.hpp:735-738): cell average of
 * the face component `face` (axis 0 bx_face, 1 by_face) over the padded grid
 * with the nghost-matched rule; cell must not alias face. */
int qmhd_launch_collocate_face_to_cell(const qmhd_grid* grid, int axis, const double* face,
                                       double* cell, void* stream);

/* launch_mhd_conserved_cell_sums (kernels.hpp:412-414): compensated mass and
 * energy totals of the interior cells, returned to the host (this library
 * finishes the sum on the device; the scratch rule of
 * qmhd_conserved_cell_totals_device applies). */
int qmhd_launch_conserved_cell_sums(const qmhd_grid* grid, const qmhd_field* u, int cylindrical,
                                    void* stream, double* mass, double* energy);

/* MhdInitialConditionSpec (physics/mhd/initial_conditions.hpp:74-131), the
 * Cartesian fields: kind 0 brio_wu, 1 alfven_wave, 2 orszag_tang, 3 blast,
 * 4 rotor, 5 confined_blob; lx, ly, origin_x, origin_y of the spec's grid
 * (its extents, ghost width and spacings are the qmhd_grid); left/right in
 * the order rho, p, vx, vy, vz, bx, by, bz. */
typedef struct qmhd_ic_spec {
  int kind;
  double lx, ly, origin_x, origin_y;
  double gamma;
  double magnetic_scale;
  double interface_x;
  double left[8], right[8];
  double rho, pressure, b0, total_b0, amplitude;
  long long wavenumber;
  double magnetic_velocity_scale;
  double b_uniform[3];
  double center[2];
  double r_in, r0, r1, rho_in, rho_out, p_in, p_out, p_core, p_ambient, rho_ambient, u0,
      blob_half;
} qmhd_ic_spec;

/* launch_mhd_seed_initial_state (kernels.hpp:656-660): the padded initial
 * state of `spec` into `out` (cells and faces, ghosts included), in two
 * passes like the reference's kernels: the conserved state with the raw
 * magnetic half-norm in the energy (also written to raw_magnetic), then the
 * energy re-formed with the face-to-cell collocated field.  Seed errors are
 * or-ed into the device int *status with the reference's bits
 * (kMhdSeed*, kernels.hpp:650-655); the caller zeroes it and reads it back.
 * cell_bx, cell_by: caller scratch as in qmhd_launch_reconstruct (they end
 * holding the collocated field).  Cartesian only; sin, cos and hypot are
 * CUDA's, so the sine-based and radial states may differ from the
 * reference's CPU build in the last bits. */
int qmhd_launch_seed_initial_state(const qmhd_grid* grid, const qmhd_ic_spec* spec,
                                   const qmhd_field* out, double* raw_magnetic, double* cell_bx,
                                   double* cell_by, int* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QUASAR_MHD_LAUNCH_H */
