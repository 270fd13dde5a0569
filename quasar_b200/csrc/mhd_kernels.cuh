// Kernel-side data structures and launch entry points of the sm_100a MHD step.
// Included by the kernels (.cu) and by the host solver.
#pragma once

#include <cuda.h>
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
  // Owned window [wx0, wx1) x [wy0, wy1) of interior cells: the reductions
  // that decide dt, admissibility retries and the live-state preflights
  // consider these cells only (a tile of a decomposed domain owns part of
  // its interior; the rest is halo kept for the stencils).  Default: all.
  int wx0 = 0, wx1 = 1 << 30, wy0 = 0, wy1 = 1 << 30;
  __host__ __device__ bool in_window(int i, int j) const {
    return i >= wx0 && i < wx1 && j >= wy0 && j < wy1;
  }
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
  kStatusWaitExpired = 32,   // a bounded device wait (TMA tile) ran out
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
  // TMA descriptor of the stage input's register (its ten arrays c[0..7],
  // bxc, byc as one 3-D tensor), or null: the cell-EMF tile is then staged
  // by plain loads
  const CUtensorMap* cell_map = nullptr;
};

// The 3-D tensor map (x, y, array) of a state register whose ten arrays are
// consecutive in memory, with the box the cell-EMF tile stages; false where
// the layout or the TMA alignment rules do not allow one (odd pitch, orders
// other than 5 and 7, or no driver entry point).
bool make_state_tensor_map(const StateP& u, const Grid& g, int order, CUtensorMap* map);

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

// ---- per-kernel launch interface (launch_abi.cu) ---------------------------
// Device address of a zero control block that no kernel writes (the calling
// thread's current device; looked up once per device).
cudaError_t abi_zero_ctl(Ctl** out);
void launch_abi_flux_difference(const Grid& g, const FluxP& f, int dir, const FluxP& d,
                                cudaStream_t s);
void launch_abi_curl_rate(const Grid& g, const double* ez, double* dbx, double* dby,
                          cudaStream_t s);
void launch_abi_rk_stage(const Grid& g, const StateP& out, const StateP& un, const StateP& us,
                         const FluxP& d, double a, double b, double c, cudaStream_t s);
void launch_abi_collocate(const Grid& g, int axis, const double* face, double* cell,
                          cudaStream_t s);
// parts: 1 fluid components, 2 staggered field
void launch_abi_fill_side(const Grid& g, const StateP& u, int side, int mode, int parts,
                          cudaStream_t s);
// *theta: bits of the running minimum (start it at the bits of 1.0)
void launch_abi_admissible(const Grid& g, const StateP& base, const StateP& cand,
                           double rho_floor, double q_floor, int coll, unsigned long long* theta,
                           cudaStream_t s);
// acc[0], acc[1]: bits of the residual and scale maxima (start them at 0)
void launch_abi_divb_relative(const Grid& g, const StateP& u, int solver_owned,
                              unsigned long long* acc, cudaStream_t s);
// *max_rate: bits of the running maximum (start it at 0)
void launch_abi_cfl_rate(const Grid& g, const IfaceP& ix, const IfaceP& iy, int order,
                         double gamma, unsigned long long* max_rate, cudaStream_t s);
void launch_abi_set_u64(unsigned long long* p, int n, unsigned long long v, cudaStream_t s);

// Analytic initial state of the reference's Cartesian generators
// (MhdInitialConditionSpec, physics/mhd/initial_conditions.hpp:74-131):
// kind 0 brio_wu, 1 alfven_wave, 2 orszag_tang, 3 blast, 4 rotor,
// 5 confined_blob.
struct SeedSpec {
  int kind;
  double lx, ly, ox, oy, gamma, magnetic_scale;
  double interface_x, left[8], right[8];
  double rho, pressure, b0, total_b0, amplitude;
  long long wavenumber;
  double mvs, b_uniform[3], center[2];
  double r_in, r0, r1, rho_in, rho_out, p_in, p_out, p_core, p_ambient, rho_ambient, u0,
      blob_half;
};
// Both passes of launch_mhd_seed_initial_state over the padded grid: the
// conserved state with the raw magnetic half-norm in the energy (out.c,
// raw), the face-to-cell collocation of the seeded faces (out.bxc, out.byc),
// and the energy re-formed from the collocated field.  Seed errors are
// or-ed into *status with the reference's bit values.
void launch_abi_seed(const Grid& g, const SeedSpec& spec, const StateP& out, double* raw,
                     int* status, cudaStream_t s);

// ---- batched step: many independent instances per launch -----------------
// One record per instance and stage: the instance's stage arguments (a.u is
// the stage input), its live register (update and admissibility base) and the
// stage's output register, plus its dt parameters.
struct BatchRec {
  StageArgs a;
  StateP live, out;
  double cfl_eff, hmin, hmax;
};

// Tile phases of a batched stage.  A phase's prefix table maps a global tile
// index to (instance, tile within the instance): prefix[i] is the first tile
// of instance i, prefix[n] the total.
enum BatchPhase : int {
  kBpRecon0, kBpRecon1, kBpFlux, kBpCell, kBpCorner, kBpUpdate, kBpColloc, kBpFill0, kBpFill1,
  kBpCount
};
// Extra tile phases of the learned batched step (not autotuned): indicator
// tiles of 16 x 8 padded cells, and 256-cell chunks of the padded grid.
enum : int { kBpInd = kBpCount, kBpCells = kBpCount + 1, kBpAll = kBpCount + 2 };

// Learned-mode buffers of one instance (those of its MhdSolver2D).
struct BatchLearnRec {
  unsigned char* flag;  // per padded cell
  int* xlist;
  int* ylist;
  int* counts;          // [2]
};

struct BatchPlan {
  const int* prefix;  // device, n + 1 entries
  int n;              // instances
  int total;          // tiles over all instances
  int grid;           // CTAs of the persistent launch (<= total)
};

// Tiles of one instance in a phase (x count, y count); the same function
// drives the host plans and the device tile decode.
__host__ __device__ inline void batch_tiles(int phase, const Grid& g, int* tx, int* ty) {
  auto cd = [](int a, int b) { return (a + b - 1) / b; };
  switch (phase) {
    case kBpRecon0: *tx = cd(g.nx + 1, 32); *ty = cd(g.ny + 2 * g.ng, 4); break;
    case kBpRecon1: *tx = cd(g.nx + 2 * g.ng, 32); *ty = cd(g.ny + 1, 4); break;
    // face tiles of 8 x 4 (MP7, 4 ghosts) or 8 x 5 (MP5, 3 ghosts) faces
    case kBpFlux: *tx = cd(g.nx + 1, 8); *ty = cd(g.ny + 1, g.ng == 3 ? 5 : 4); break;
    case kBpCell: *tx = cd(g.nx + 1, 16); *ty = cd(g.ny + 1, 16); break;  // kCellTX x kCellTY
    case kBpCorner: *tx = cd(g.nx + 1, 32); *ty = cd(g.ny + 1, 4); break;
    case kBpUpdate: *tx = cd(g.nx + 1, 32); *ty = cd(g.ny + 1, 8); break;
    case kBpColloc: *tx = cd(g.nx + 2 * g.ng, 32); *ty = cd(g.ny + 2 * g.ng, 8); break;
    case kBpFill0: *tx = cd(2 * g.ng * (g.ny + 2 * g.ng), 256); *ty = 1; break;
    case kBpFill1: *tx = cd(2 * g.ng * (g.nx + 2 * g.ng), 256); *ty = 1; break;
    case kBpInd: *tx = cd(g.pitch, 16); *ty = cd(g.ny + 2 * g.ng, 8); break;
    default: *tx = int((g.size() + 255) / 256); *ty = 1; break;  // kBpCells
  }
}

#ifdef __CUDACC__
// Instance of global tile t (largest i with prefix[i] <= t) and the tile's
// index within that instance.
__device__ __forceinline__ int batch_locate(const BatchPlan& p, int t, int* local) {
  int lo = 0, hi = p.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(p.prefix + mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  *local = t - __ldg(p.prefix + lo);
  return lo;
}

__device__ __forceinline__ void batch_block(int phase, const Grid& g, int local, int* bx, int* by) {
  int tx, ty;
  batch_tiles(phase, g, &tx, &ty);
  *bx = local % tx;
  *by = local / tx;
}
#endif

// Threads per CTA of each phase's batched kernel and its resident CTAs per SM
// (queried once per process), for sizing persistent grids.
int batch_phase_threads(int phase);
int batch_phase_max_ctas_per_sm(int phase, int order);

// Batched launches: every record's instance in one persistent launch.  Records
// are indexed like the plan's prefix table.  All instances share `order`.
void launch_batch_reconstruct(const BatchRec* r, const BatchPlan& p, int dir, int order,
                              cudaStream_t s);
void launch_batch_face_flux(const BatchRec* r, const BatchPlan& p, int dir, int order,
                            bool speeds, cudaStream_t s);
void launch_batch_cell_emf(const BatchRec* r, const BatchPlan& p, int order, bool cfl_reduce,
                           cudaStream_t s);
void launch_batch_corner_emf(const BatchRec* r, const BatchPlan& p, int order, cudaStream_t s);
void launch_batch_update(const BatchRec* r, const BatchPlan& p, int stage, cudaStream_t s);
void launch_batch_fill_ghosts(const BatchRec* r, const BatchPlan& p, int axis, cudaStream_t s);
void launch_batch_colloc_check(const BatchRec* r, const BatchPlan& p, int order, int theta_mask,
                               bool live_checks, cudaStream_t s);
// Learned batched step: flags of every padded cell set to 1 and list counts
// cleared (cells plan), face lists of every instance, and the two
// reconstruction passes (component-wise over all faces, characteristic over
// each instance's list).
void launch_batch_learned_reset(const BatchRec* r, const BatchLearnRec* l, const BatchPlan& cells,
                                cudaStream_t s);
void launch_batch_face_lists(const BatchRec* r, const BatchLearnRec* l, const BatchPlan& cells,
                             cudaStream_t s);
void launch_batch_reconstruct_learned(const BatchRec* r, const BatchLearnRec* l,
                                      const BatchPlan& p, int dir, int order, int list_grid,
                                      cudaStream_t s);
// Per-instance control kernels (one thread per instance): 0 step_begin
// (collocation 0, anchor from the live state), 1 dt (clipped to t_end),
// 2 step_end, 3 set_time(t, t_end).
void launch_batch_ctl(const BatchRec* r, int n, int what, double t, double t_end, cudaStream_t s);

// ---- learned troubled-cell mode --------------------------------------------
// Limiter departures (per padded cell, float bits, max-reduced): how far a
// face state of a stencil centred on the cell, limited in characteristic
// fields, departs from the unlimited component-wise state, relative to the
// state's scale.  The array must start at zero.
void launch_reconstruct_label(const StageArgs& a, int dir, int* label, int literal,
                              cudaStream_t s);
// Unlimited component-wise reconstruction of every face, then the full
// characteristic path for the listed faces (count on the device).  Faces
// whose unlimited states are not admissible are appended to the list (flag:
// the per-cell flags the list was built from).
void launch_reconstruct_learned(const StageArgs& a, int dir, const unsigned char* flag, int* list,
                                int* count, int list_grid, cudaStream_t s);
// Faces adjacent to a flagged cell (flag per padded cell) -> x / y lists;
// counts[0..1] are reset first.
void launch_face_lists(const Grid& g, const unsigned char* flag, int* xlist, int* ylist,
                       int* counts, cudaStream_t s);

// *bad |= 1 if any of v[0..n) is not finite (*bad must start at zero).
void launch_flag_nonfinite(const double* v, long long n, unsigned long long* bad, cudaStream_t s);

// ---- tile halo exchange ----------------------------------------------------
// out[k] = src[idx[k]] and dst[idx[k]] = v[k] for k < n, indices checked
// against [0, size) and scattered values against non-finite ones; problems
// are OR-ed into *bad (1: index, 2: value) and a scatter with any problem
// writes nothing.  *bad must start at zero.
void launch_gather_values(const double* src, const long long* idx, long long n, long long size,
                          double* out, unsigned long long* bad, cudaStream_t s);
void launch_scatter_values(double* dst, const long long* idx, const double* v, long long n,
                           long long size, unsigned long long* bad, cudaStream_t s);

}  // namespace qb
