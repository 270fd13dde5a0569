// Kernel-side data structures and launch entry points of the sm_100a MHD step.
// Included by the kernels (.cu) and by the host solver.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace qb {

// Padded SoA grid: index (i+ng) + pitch*(j+ng), pitch = nx+2ng
// (reference core/grid.hpp:158-161).  bc[4] = x_lo, x_hi, y_lo, y_hi with
// 0 periodic, 1 outflow, 2 conducting wall (reference BoundaryFlags4,
// physics/mhd/kernels.hpp:49-51).
struct Grid {
  int nx, ny, ng, pitch;
  double dx, dy;
  int bc[4];
  __host__ __device__ long long idx(int i, int j) const {
    return (long long)(i + ng) + (long long)pitch * (long long)(j + ng);
  }
  __host__ __device__ long long size() const {
    return (long long)pitch * (long long)(ny + 2 * ng);
  }
};

// Eight conserved components plus the cell-collocated in-plane field of the
// same state (bxc, byc), which every consumer of a cell-centred B reads.
struct StateP {
  double* c[8];  // rho, mx, my, mz, energy, bx_face, by_face, bz_cell
  double* bxc;
  double* byc;
};

struct IfaceP {
  double* L[8];
  double* R[8];
};

struct FluxP {
  double* f[8];
};

// Step control block, resident in device memory.  Reduced scalars use the
// IEEE bit pattern of a non-negative double, whose integer order equals its
// numeric order, so atomicMax/atomicMin on uint64 reduce them.
struct Ctl {
  unsigned long long max_rate;     // CFL: max over cells of the additive face rate
  unsigned long long theta;        // min admissible fraction of the current stage
  unsigned long long divb_res;     // solenoidality: max unexplained |div|
  unsigned long long divb_scale;   // solenoidality: max directional scale
  unsigned long long live_theta;   // min admissible fraction of the live state (coll 0)
  unsigned long long anchor_theta; // same with the two-face (low-order) collocation
  int anchor_ok;                   // live state admissible under the low-order collocation
  double dt;                       // timestep used by the stage updates
  double t;                        // accumulated time (device-resident loop)
  double t_end;                    // clip target for the device-resident loop
  int status;                      // kStatus* bits; kernels return early when set
  int steps_done;                  // completed steps of the device-resident loop
};

enum : int {
  kStatusRetry = 1,          // a stage candidate left the admissible set
  kStatusCflNonFinite = 2,   // non-finite signal speed in the CFL reduction
  kStatusNotSolenoidal = 4,  // live field fails the discrete div B preflight
  kStatusNotAdmissible = 8,  // live state inadmissible before a step
  kStatusDone = 16,          // device-resident loop reached t_end
};

struct StageArgs {
  Grid g;
  double gamma;
  int order;       // 1 (low-order retry), 2, 5 or 7
  StateP u;        // stage input
  IfaceP ix, iy;   // interface states
  FluxP fx, fy;    // face fluxes
  double* xemf;    // x-face E_z table
  double* yemf;
  int* xnj;        // x-face "no jump" proofs
  int* ynj;
  double* xspd;    // per-face CFL signal speed (stage 0 only)
  double* yspd;
  double* cell_ez;
  double* ez;      // corner EMF
  Ctl* ctl;
};

// Launch wrappers (mhd_kernels.cu).  All take a stream and never allocate.
void launch_fill_ghosts(const Grid& g, const StateP& u, cudaStream_t s);
// theta_mask: bit0 admissibility vs base with the high-order collocation,
// bit1 with the two-face collocation, bit2 the latter only when the live
// state's low-order anchor is admissible.
void launch_colloc_check(const Grid& g, const StateP& cand, const StateP* base,
                         int theta_mask, bool anchor_check, bool live_checks,
                         bool solver_owned, double gamma, Ctl* ctl, cudaStream_t s);
void launch_reconstruct(const StageArgs& a, int dir, cudaStream_t s);
void launch_face_flux(const StageArgs& a, int dir, bool speeds, cudaStream_t s);
void launch_cell_emf(const StageArgs& a, bool cfl_reduce, cudaStream_t s);
void launch_corner_emf(const StageArgs& a, cudaStream_t s);
void launch_update(const StageArgs& a, const StateP& un, const StateP& us,
                   const StateP& out, int stage, const double* dt_dev, double dt_host,
                   cudaStream_t s);
void launch_step_begin(Ctl* ctl, int coll, int anchor_mode, cudaStream_t s);
void launch_reset_stats(Ctl* ctl, cudaStream_t s);
void launch_set_time(Ctl* ctl, double t, double t_end, cudaStream_t s);
void launch_dt(Ctl* ctl, double cfl_eff, double hmin, double hmax, int clip, cudaStream_t s);
void launch_step_end(Ctl* ctl, cudaStream_t s);
void launch_divb_linf(const Grid& g, const StateP& u, unsigned long long* out, cudaStream_t s);
// Per-block compensated partial sums (4 doubles per block: mass, mass error,
// energy, energy error).
void launch_cell_sums(const Grid& g, const StateP& u, double* partial, int blocks,
                      cudaStream_t s);

}  // namespace qb
