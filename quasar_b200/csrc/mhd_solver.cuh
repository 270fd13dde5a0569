// Host side of the B200 MHD solver: the reference's MhdSolver2D interface
// (physics/mhd/mhd_solver.hpp:85-173) over the sm_100a kernels.
//
// Device memory is allocated once, at construction; stepping allocates
// nothing.  Four state registers rotate (live U^n, stage outputs U1, U2 and
// the next state), so the Shu-Osher combine never needs a rollback copy: a
// rejected candidate is simply not promoted.  dt, the CFL reduction and the
// admissibility fractions live in a device control block; the API-mode step
// reads back one status word, the device-resident loop none.
#pragma once

#include "mhd_kernels.cuh"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace qb {

struct Config {
  int nx = 0, ny = 0;
  double lx = 1.0, ly = 1.0, ox = 0.0, oy = 0.0;
  int order = 7;  // 2 (muscl_minmod), 5 (mp5), 7 (mp7)
  double gamma = 5.0 / 3.0;
  double cfl = 0.4;
  int bc[4] = {0, 0, 0, 0};  // x_lo, x_hi, y_lo, y_hi: 0 periodic, 1 outflow, 2 wall
};

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class MhdBatch2D;
class Indicator;

class MhdSolver2D {
 public:
  explicit MhdSolver2D(const Config& cfg);
  ~MhdSolver2D();
  MhdSolver2D(const MhdSolver2D&) = delete;
  MhdSolver2D& operator=(const MhdSolver2D&) = delete;

  const Grid& grid() const { return g_; }
  const Config& config() const { return cfg_; }
  long long storage_size() const { return g_.size(); }

  // Reference-facing API (mhd_solver.hpp:111-173).
  void seed_state(int comp, const double* host, long long n);
  // comp 0..7 raw storage; 8 / 9 = the collocated cell bx / by.
  void state_component_to_host(int comp, double* host, long long n);
  double cfl_limit();
  void step(double dt);
  void step_unchecked(double dt);
  void advance(double t_end, double dt);
  double divergence_b_max();
  void conserved_cell_totals(double* mass, double* energy);
  int last_positivity_substeps() const { return last_substeps_; }

  // Device-resident auto-dt loop: up to `max_steps` steps of
  // dt = min(cfl_limit, t_end - t) without host round trips (replayed CUDA
  // graphs); a step the positivity controller must retry falls back to the
  // host controller.  Returns the steps taken; *t is advanced in place.
  int advance_auto(double* t, double t_end, int max_steps);

  // Measurement hooks (bench.py): `steps` device-resident auto-dt steps timed
  // with CUDA events on the solver stream (returns ms, *done = steps taken),
  // and one API step with per-phase device times (ms_by_phase[kPhases]).
  double time_auto_steps(int steps, int* done);
  void profile_step(double* ms_by_phase);
  static constexpr int kPhases = 8;

  // Device pointers of the live state (kernel-level C-ABI and tests).
  double* live_component(int comp) const;
  // Stage arguments of the live state after its preflight (ghosts filled,
  // field collocated), for kernels run on the solver's state from outside.
  StageArgs live_args();

  // Learned troubled-cell mode (mp5/mp7): once per step the indicator scores
  // the live state's cells; faces next to a cell scored above `threshold`
  // keep the characteristic MP reconstruction in every stage, all others
  // take the unlimited component-wise interpolation.  nullptr turns it off.
  // The indicator must outlive its use by this solver.
  void set_indicator(const Indicator* ind, float threshold);
  // Faces on the full-reconstruction lists of the last step, x and y.
  void learned_face_counts(long long* nx_faces, long long* ny_faces);
  cudaStream_t stream() const { return stream_; }

  // Tile of a decomposed domain (quasar_b200/tiles.py).  The owned window
  // [x0, x1) x [y0, y1) of interior cells restricts the reductions that
  // decide dt, retries and the live-state preflights to the cells this tile
  // owns.  write_halo writes a whole component like seed_state, but the
  // values are the solver's own (stepped on another tile), so the state
  // stays solver-owned and its preflight stays the one of a stepped state.
  void set_owned_window(int x0, int x1, int y0, int y1);
  void write_halo(int comp, const double* host, long long n);
  // The same exchange on the device: gather_live copies the live values at
  // storage indices idx[0..n) into out; scatter_halo writes v[k] to index
  // idx[k] (all finite; on any bad index or value it writes nothing and
  // throws) and keeps the state solver-owned like write_halo.  idx, out and
  // v are device memory of the solver's device, ready when called; both
  // return after the copy finished.
  void gather_live(int comp, const long long* idx, long long n, double* out);
  void scatter_halo(int comp, const long long* idx, long long n, const double* v);

 private:
  friend class MhdBatch2D;  // batched stage launches over the same registers
  struct Attempt {
    bool ok;
    double theta;
  };
  StageArgs stage_args(const StateP& u, int order) const;
  void ensure_live_ready();
  void refresh_live_stats();
  void front_impl(int order, int dt_mode, int anchor_mode);
  void finish_impl(int order, const double* dt_dev, double dt_host, bool step_end);
  Ctl read_ctl();
  void throw_status(int status);
  void promote();
  void copy_state(const StateP& src, const StateP& dst);
  void advance_positive(double dt);
  void controller(double dt, double theta, bool anchor);
  double cfl_limit_for(int coll);
  void check_cuda(const char* what);
  void build_graphs();

  Config cfg_;
  Grid g_;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  double* arena_ = nullptr;
  int* iarena_ = nullptr;
  Ctl* ctl_ = nullptr;
  Ctl* ctl_host_ = nullptr;  // pinned mirror
  double* sums_ = nullptr;
  unsigned long long* scalar_ = nullptr;
  int sum_blocks_ = 0;
  StateP st_[5];  // 0..3 rotating registers, 4 = request backup
  // TMA descriptors of the registers (each register's ten arrays as one 3-D
  // tensor) for the cell-EMF tile; tmap_ok_ false where none could be made
  alignas(64) CUtensorMap tmaps_[5];
  bool tmap_ok_[5] = {};
  bool halo_write_ = false;  // the live state was last written by write_halo
  int live_ = 0, s1_ = 1, s2_ = 2, next_ = 3;
  IfaceP ix_, iy_;
  FluxP fx_, fy_;
  double *xemf_, *yemf_, *xspd_, *yspd_, *cell_ez_, *ez_;
  int *xnj_, *ynj_;
  bool seeded_dirty_ = true;    // live state written externally since last check
  bool solver_owned_ = false;   // live state produced by an accepted step
  int front_order_ = 0;         // order of the cached stage-0 residual (0 = none)
  int front_dt_mode_ = 0;       // whether that residual also produced a device dt
  int anchor_mode_ = -1;        // forced low-order anchor flag inside the controller
  int low_order_ = 0;           // 1 while the positivity controller runs low order
  int last_substeps_ = 0;
  cudaGraphExec_t graph_[2] = {nullptr, nullptr};
  void release_graphs();
  void reconstruct_stage(const StageArgs& a, int order);
  // learned mode
  const Indicator* ind_ = nullptr;
  float ind_threshold_ = 0.f;
  unsigned char* flags_ = nullptr;   // per padded cell
  int* flists_ = nullptr;            // x list, y list (padded size each)
  int* fcounts_ = nullptr;           // [2]
  int* ind_status_ = nullptr;
  // per-phase event marks while profiling (phase, event after the launch)
  struct Mark {
    int phase;
    cudaEvent_t ev;
  };
  Mark* marks_ = nullptr;
  int nmarks_ = 0;
  void mark(int phase);
};

}  // namespace qb
