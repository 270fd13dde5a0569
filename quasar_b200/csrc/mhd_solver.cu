// Host solver: buffer ownership, stage sequencing, the positivity retry
// controller and the device-resident loop.  Mirrors the reference's
// MhdSolver2D (src/physics/mhd/mhd_solver.cpp) call for call where the
// semantics are observable: preflights, CFL cap, retry policy, errors.
#include "mhd_solver.cuh"
#include "indicator.cuh"

#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <sstream>
#include <vector>

namespace qb {

namespace {

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

double from_bits(unsigned long long b) {
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
}

int ghosts_for(int order) { return order == 7 ? 4 : order == 5 ? 3 : 2; }

// [p, p + bytes) must lie in one device allocation of `device` (the kernels
// that read or write it have no other way to know its extent).
void check_device_range(const void* p, size_t bytes, int device, const char* what) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess ||
      !(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ||
      a.device != device) {
    cudaGetLastError();
    throw std::invalid_argument(std::string(what) + " is not device memory of the solver's device");
  }
  using RangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
  static RangeFn range = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      range = reinterpret_cast<RangeFn>(fn);
  });
  if (!range) throw CudaError("cuMemGetAddressRange is unavailable");
  CUdeviceptr base = 0;
  size_t size = 0;
  if (range(&base, &size, reinterpret_cast<CUdeviceptr>(p)) != CUDA_SUCCESS)
    throw std::invalid_argument(std::string(what) + ": no device allocation holds it");
  const CUdeviceptr q = reinterpret_cast<CUdeviceptr>(p);
  if (q - base > size || bytes > size - (q - base))
    throw std::invalid_argument(std::string(what) + " runs past the end of its allocation");
}

}  // namespace

// Configuration checks of mhd_solver.cpp:56-208 that apply to this path.
MhdSolver2D::MhdSolver2D(const Config& c) : cfg_(c) {
  if (c.nx < 1 || c.ny < 1)
    throw std::invalid_argument("MhdSolver2D: grid extents must be positive");
  if (!(std::isfinite(c.lx) && c.lx > 0.0 && std::isfinite(c.ly) && c.ly > 0.0))
    throw std::invalid_argument("MhdSolver2D: grid lengths must be finite and positive");
  if (!(std::isfinite(c.gamma) && c.gamma > 1.0))
    throw std::invalid_argument("MhdSolver2D: gamma must be finite and greater than one");
  if (!(std::isfinite(c.cfl) && c.cfl > 0.0 && c.cfl <= 1.0))
    throw std::invalid_argument("MhdSolver2D: cfl must be finite and in (0,1]");
  if (c.order != 2 && c.order != 5 && c.order != 7)
    throw std::invalid_argument(
        "MhdSolver2D: device evolution supports only reconstruction='muscl_minmod', "
        "'mp5', or 'mp7'");
  for (int s = 0; s < 4; ++s)
    if (c.bc[s] < 0 || c.bc[s] > 2)
      throw std::invalid_argument("MhdSolver2D: boundary mode must be periodic, outflow or wall");
  for (int axis = 0; axis < 2; ++axis)
    if ((c.bc[2 * axis] == 0) != (c.bc[2 * axis + 1] == 0))
      throw std::invalid_argument(
          "MhdSolver2D: periodic boundaries must be selected on both sides of an axis");
  const int ng = ghosts_for(c.order);
  g_.nx = c.nx;
  g_.ny = c.ny;
  g_.ng = ng;
  g_.pitch = c.nx + 2 * ng;
  g_.dx = c.lx / c.nx;
  g_.dy = c.ly / c.ny;
  for (int s = 0; s < 4; ++s) g_.bc[s] = c.bc[s];

  ck(cudaGetDevice(&device_), "device");
  ck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  const long long n = g_.size();
  constexpr int kArrays = 5 * 10 + 32 + 16 + 6;
  ck(cudaMalloc(&arena_, sizeof(double) * n * kArrays), "state arena");
  ck(cudaMemsetAsync(arena_, 0, sizeof(double) * n * kArrays, stream_), "memset");
  ck(cudaMalloc(&iarena_, sizeof(int) * n * 2), "flag arena");
  ck(cudaMemsetAsync(iarena_, 0, sizeof(int) * n * 2, stream_), "memset");
  ck(cudaMalloc(&ctl_, sizeof(Ctl)), "control block");
  ck(cudaMallocHost(&ctl_host_, sizeof(Ctl)), "pinned control block");
  sum_blocks_ = int(std::min<long long>(1024, ((long long)c.nx * c.ny + 255) / 256));
  ck(cudaMalloc(&sums_, sizeof(double) * 4 * sum_blocks_), "sum scratch");
  ck(cudaMalloc(&scalar_, sizeof(unsigned long long)), "scalar scratch");
  double* p = arena_;
  auto take = [&]() {
    double* r = p;
    p += n;
    return r;
  };
  for (auto& s : st_) {
    for (auto& comp : s.c) comp = take();
    s.bxc = take();
    s.byc = take();
  }
  for (int k = 0; k < 8; ++k) ix_.L[k] = take();
  for (int k = 0; k < 8; ++k) ix_.R[k] = take();
  for (int k = 0; k < 8; ++k) iy_.L[k] = take();
  for (int k = 0; k < 8; ++k) iy_.R[k] = take();
  for (int k = 0; k < 8; ++k) fx_.f[k] = take();
  for (int k = 0; k < 8; ++k) fy_.f[k] = take();
  xemf_ = take();
  yemf_ = take();
  xspd_ = take();
  yspd_ = take();
  cell_ez_ = take();
  ez_ = take();
  xnj_ = iarena_;
  ynj_ = iarena_ + n;
  for (int k = 0; k < 5; ++k) tmap_ok_[k] = make_state_tensor_map(st_[k], g_, cfg_.order, &tmaps_[k]);
  Ctl init{};
  *ctl_host_ = init;
  ck(cudaMemcpyAsync(ctl_, ctl_host_, sizeof(Ctl), cudaMemcpyHostToDevice, stream_), "ctl init");
  ck(cudaStreamSynchronize(stream_), "init");
}

MhdSolver2D::~MhdSolver2D() {
  for (auto& ge : graph_)
    if (ge) cudaGraphExecDestroy(ge);
  cudaStreamSynchronize(stream_);
  cudaFree(flags_);
  cudaFree(flists_);
  cudaFree(fcounts_);
  cudaFree(ind_status_);
  cudaFree(arena_);
  cudaFree(iarena_);
  cudaFree(ctl_);
  cudaFreeHost(ctl_host_);
  cudaFree(sums_);
  cudaFree(scalar_);
  cudaStreamDestroy(stream_);
}

void MhdSolver2D::check_cuda(const char* what) { ck(cudaGetLastError(), what); }

double* MhdSolver2D::live_component(int comp) const {
  if (comp == 8) return st_[live_].bxc;
  if (comp == 9) return st_[live_].byc;
  return st_[live_].c[comp];
}

StageArgs MhdSolver2D::stage_args(const StateP& u, int order) const {
  StageArgs a;
  a.g = g_;
  a.gamma = cfg_.gamma;
  a.order = order;
  a.u = u;
  a.ix = ix_;
  a.iy = iy_;
  a.fx = fx_;
  a.fy = fy_;
  a.xemf = xemf_;
  a.yemf = yemf_;
  a.xnj = xnj_;
  a.ynj = ynj_;
  a.xspd = xspd_;
  a.yspd = yspd_;
  a.cell_ez = cell_ez_;
  a.ez = ez_;
  a.ctl = ctl_;
  for (int k = 0; k < 5; ++k)
    if (u.c[0] == st_[k].c[0] && tmap_ok_[k]) a.cell_map = &tmaps_[k];
  return a;
}

// mhd_solver.cpp:521-541.  seed_state performs no ghost refill; the next
// solver operation closes the boundary and runs the preflights.
void MhdSolver2D::seed_state(int comp, const double* host, long long n) {
  if (comp < 0 || comp > 7) throw std::invalid_argument("MhdSolver2D: unknown state component");
  if (n != g_.size()) {
    std::ostringstream m;
    m << "MhdSolver2D::seed_state: host buffer size (" << n
      << ") does not match the component storage size (" << g_.size() << ")";
    throw std::invalid_argument(m.str());
  }
  // The values land in the first stage register (scratch between steps),
  // are tested there on the device, and only then replace the live
  // component, so a rejected buffer leaves the state as it was (a host-side
  // scan of the buffer cost as much as the copy itself at large sizes).
  double* stage = st_[s1_].c[comp];
  ck(cudaMemcpyAsync(stage, host, sizeof(double) * n, cudaMemcpyHostToDevice, stream_),
     "seed copy");
  ck(cudaMemsetAsync(scalar_, 0, sizeof(unsigned long long), stream_), "memset");
  launch_flag_nonfinite(stage, n, scalar_, stream_);
  check_cuda("seed check launch");
  unsigned long long bad = 0;
  ck(cudaMemcpyAsync(&bad, scalar_, sizeof bad, cudaMemcpyDeviceToHost, stream_), "seed flag");
  ck(cudaStreamSynchronize(stream_), "seed");
  if (bad)
    throw std::invalid_argument(
        "MhdSolver2D::seed_state: host buffer must contain only finite values");
  ck(cudaMemcpyAsync(st_[live_].c[comp], stage, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                     stream_),
     "seed copy");
  ck(cudaStreamSynchronize(stream_), "seed");
  seeded_dirty_ = true;
  solver_owned_ = false;
  halo_write_ = false;
  front_order_ = 0;
}

void MhdSolver2D::set_owned_window(int x0, int x1, int y0, int y1) {
  if (!(0 <= x0 && x0 < x1 && x1 <= g_.nx && 0 <= y0 && y0 < y1 && y1 <= g_.ny))
    throw std::invalid_argument("MhdSolver2D::set_owned_window: need 0 <= x0 < x1 <= nx and "
                                "0 <= y0 < y1 <= ny");
  g_.wx0 = x0;
  g_.wx1 = x1;
  g_.wy0 = y0;
  g_.wy1 = y1;
  release_graphs();  // the captured launches hold the grid by value
  seeded_dirty_ = true;  // recompute the live preflights over the window
  halo_write_ = solver_owned_;
  front_order_ = 0;
}

void MhdSolver2D::write_halo(int comp, const double* host, long long n) {
  if (comp < 0 || comp > 7) throw std::invalid_argument("MhdSolver2D: unknown state component");
  if (n != g_.size())
    throw std::invalid_argument("MhdSolver2D::write_halo: host buffer size mismatch");
  // the interior must be finite; ghost layers are closed again before use
  for (int j = 0; j < g_.ny; ++j)
    for (int i = 0; i < g_.nx; ++i)
      if (!std::isfinite(host[g_.idx(i, j)]))
        throw std::invalid_argument("MhdSolver2D::write_halo: non-finite interior value");
  ck(cudaMemcpyAsync(st_[live_].c[comp], host, sizeof(double) * n, cudaMemcpyHostToDevice,
                     stream_),
     "halo copy");
  ck(cudaStreamSynchronize(stream_), "halo");
  if (!seeded_dirty_) halo_write_ = solver_owned_;
  seeded_dirty_ = true;
  front_order_ = 0;
}

void MhdSolver2D::gather_live(int comp, const long long* idx, long long n, double* out) {
  if (comp < 0 || comp > 7) throw std::invalid_argument("MhdSolver2D: unknown state component");
  if (n < 0) throw std::invalid_argument("MhdSolver2D::gather_live: negative count");
  if (n == 0) return;
  check_device_range(idx, sizeof(long long) * n, device_, "gather_live: index buffer");
  check_device_range(out, sizeof(double) * n, device_, "gather_live: output buffer");
  ck(cudaMemsetAsync(scalar_, 0, sizeof(unsigned long long), stream_), "memset");
  launch_gather_values(st_[live_].c[comp], idx, n, g_.size(), out, scalar_, stream_);
  check_cuda("gather launch");
  unsigned long long bad = 0;
  ck(cudaMemcpyAsync(&bad, scalar_, sizeof bad, cudaMemcpyDeviceToHost, stream_), "gather flag");
  ck(cudaStreamSynchronize(stream_), "gather");
  if (bad) throw std::invalid_argument("MhdSolver2D::gather_live: storage index out of range");
}

void MhdSolver2D::scatter_halo(int comp, const long long* idx, long long n, const double* v) {
  if (comp < 0 || comp > 7) throw std::invalid_argument("MhdSolver2D: unknown state component");
  if (n < 0) throw std::invalid_argument("MhdSolver2D::scatter_halo: negative count");
  if (n == 0) return;
  check_device_range(idx, sizeof(long long) * n, device_, "scatter_halo: index buffer");
  check_device_range(v, sizeof(double) * n, device_, "scatter_halo: value buffer");
  ck(cudaMemsetAsync(scalar_, 0, sizeof(unsigned long long), stream_), "memset");
  launch_scatter_values(st_[live_].c[comp], idx, v, n, g_.size(), scalar_, stream_);
  check_cuda("scatter launch");
  unsigned long long bad = 0;
  ck(cudaMemcpyAsync(&bad, scalar_, sizeof bad, cudaMemcpyDeviceToHost, stream_), "scatter flag");
  ck(cudaStreamSynchronize(stream_), "scatter");
  if (bad & 1ull)
    throw std::invalid_argument("MhdSolver2D::scatter_halo: storage index out of range");
  if (bad & 2ull) throw std::invalid_argument("MhdSolver2D::scatter_halo: non-finite value");
  if (!seeded_dirty_) halo_write_ = solver_owned_;
  seeded_dirty_ = true;
  front_order_ = 0;
}

void MhdSolver2D::state_component_to_host(int comp, double* host, long long n) {
  if (comp < 0 || comp > 9) throw std::invalid_argument("MhdSolver2D: unknown state component");
  if (n != g_.size()) throw std::invalid_argument("MhdSolver2D: host buffer size mismatch");
  if (comp >= 8) ensure_live_ready();
  ck(cudaMemcpyAsync(host, live_component(comp), sizeof(double) * n, cudaMemcpyDeviceToHost,
                     stream_),
     "read copy");
  ck(cudaStreamSynchronize(stream_), "read");
}

// Close the boundary of an externally written live state, collocate its
// field and compute its preflight statistics (admissibility under both
// collocations, discrete div B).
void MhdSolver2D::ensure_live_ready() {
  if (!seeded_dirty_) return;
  // a state the solver stepped (here or on another tile, written back by
  // write_halo) keeps the preflight of a stepped state; a seeded one gets
  // the seeded-state test
  const bool owned = halo_write_;
  launch_fill_ghosts(g_, st_[live_], stream_);
  launch_reset_stats(ctl_, stream_);
  launch_colloc_check(g_, st_[live_], nullptr, 0, false, true, owned, cfg_.gamma, ctl_, stream_);
  check_cuda("preflight launch");
  seeded_dirty_ = false;
  solver_owned_ = owned;
  halo_write_ = false;
  front_order_ = 0;
}

void MhdSolver2D::refresh_live_stats() {
  launch_reset_stats(ctl_, stream_);
  launch_colloc_check(g_, st_[live_], nullptr, 0, false, true, solver_owned_, cfg_.gamma, ctl_,
                      stream_);
  check_cuda("live stats launch");
}

// Stage-0 residual of the live state: reconstruction, face fluxes with CFL
// speeds, cell and corner EMF, and (dt_mode 1/2) the device dt.
void MhdSolver2D::front_impl(int order, int dt_mode, int anchor_mode) {
  launch_step_begin(ctl_, order <= 1 ? 1 : 0, anchor_mode, stream_);
  mark(0);
  const StageArgs a = stage_args(st_[live_], order);
  if (ind_ && order >= 5) {
    // score the live state once per step; unwritten flags stay 1 (full path)
    ck(cudaMemsetAsync(flags_, 1, size_t(g_.size()), stream_), "flags");
    ck(launch_indicator(g_, st_[live_], cfg_.gamma, ind_->dev(), ind_threshold_, flags_,
                        ind_status_, stream_),
       "indicator launch");
    launch_face_lists(g_, flags_, flists_, flists_ + g_.size(), fcounts_, stream_);
    mark(0);
  }
  reconstruct_stage(a, order);
  mark(1);
  const bool speeds = dt_mode != 0;
  launch_face_flux(a, 0, speeds, stream_);
  launch_face_flux(a, 1, speeds, stream_);
  mark(2);
  launch_cell_emf(a, speeds, stream_);
  mark(3);
  launch_corner_emf(a, stream_);
  mark(4);
  if (dt_mode != 0) {
    const double eff = order >= 5 ? std::min(cfg_.cfl, 0.2) : cfg_.cfl;
    launch_dt(ctl_, eff, std::min(g_.dx, g_.dy), std::max(g_.dx, g_.dy), dt_mode == 2 ? 1 : 0,
              stream_);
    mark(0);
  }
}

void MhdSolver2D::reconstruct_stage(const StageArgs& a, int order) {
  if (ind_ && order >= 5) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    launch_reconstruct_learned(a, 0, flags_, flists_, fcounts_, 4 * sms, stream_);
    launch_reconstruct_learned(a, 1, flags_, flists_ + g_.size(), fcounts_ + 1, 4 * sms, stream_);
  } else {
    launch_reconstruct(a, 0, stream_);
    launch_reconstruct(a, 1, stream_);
  }
}

StageArgs MhdSolver2D::live_args() {
  ensure_live_ready();
  return stage_args(st_[live_], cfg_.order);
}

void MhdSolver2D::release_graphs() {
  for (auto& ge : graph_) {
    if (ge) cudaGraphExecDestroy(ge);
    ge = nullptr;
  }
}

void MhdSolver2D::set_indicator(const Indicator* ind, float threshold) {
  if (ind && cfg_.order != 5 && cfg_.order != 7)
    throw std::invalid_argument("MhdSolver2D: the learned indicator needs mp5 or mp7");
  if (ind && !std::isfinite(threshold))
    throw std::invalid_argument("MhdSolver2D: indicator threshold must be finite");
  if (ind) ck(configure_indicator_kernels(), "indicator kernels");
  if (ind && !flags_) {
    ck(cudaMalloc(&flags_, size_t(g_.size())), "indicator flags");
    ck(cudaMalloc(&flists_, sizeof(int) * 2 * size_t(g_.size())), "face lists");
    ck(cudaMalloc(&fcounts_, sizeof(int) * 2), "face counts");
    ck(cudaMalloc(&ind_status_, sizeof(int)), "indicator status");
    ck(cudaMemsetAsync(fcounts_, 0, sizeof(int) * 2, stream_), "face counts");
    ck(cudaMemsetAsync(ind_status_, 0, sizeof(int), stream_), "indicator status");
  }
  ind_ = ind;
  ind_threshold_ = threshold;
  front_order_ = 0;
  release_graphs();
}

void MhdSolver2D::learned_face_counts(long long* nxf, long long* nyf) {
  int c[2] = {0, 0}, st = 0;
  if (fcounts_) {
    ck(cudaMemcpyAsync(c, fcounts_, sizeof c, cudaMemcpyDeviceToHost, stream_), "face counts");
    ck(cudaMemcpyAsync(&st, ind_status_, sizeof st, cudaMemcpyDeviceToHost, stream_), "status");
    ck(cudaStreamSynchronize(stream_), "face counts");
  }
  if (st) throw std::runtime_error("MhdSolver2D: indicator tensor-core wait ran out");
  *nxf = c[0];
  *nyf = c[1];
}

// Stages of one SSP-RK3 step after the cached stage-0 residual
// (mhd_solver.cpp:840-953).  Candidates go to U1, U2 and the next register;
// each is closed, collocated and checked against the live state.
void MhdSolver2D::finish_impl(int order, const double* dt_dev, double dt_host, bool step_end) {
  const StateP live = st_[live_], u1 = st_[s1_], u2 = st_[s2_], nxt = st_[next_];
  const int mask01 = order <= 1 ? 2 : 1;
  const int mask2 = order <= 1 ? 3 : (1 | 4);
  launch_update(stage_args(live, order), live, live, u1, 0, dt_dev, dt_host, stream_);
  mark(5);
  launch_fill_ghosts(g_, u1, stream_);
  mark(6);
  launch_colloc_check(g_, u1, &live, mask01, false, false, true, cfg_.gamma, ctl_, stream_);
  mark(7);
  for (int stage = 1; stage < 3; ++stage) {
    const StateP in = stage == 1 ? u1 : u2;
    const StateP out = stage == 1 ? u2 : nxt;
    const StageArgs a = stage_args(in, order);
    reconstruct_stage(a, order);
    mark(1);
    launch_face_flux(a, 0, false, stream_);
    launch_face_flux(a, 1, false, stream_);
    mark(2);
    launch_cell_emf(a, false, stream_);
    mark(3);
    launch_corner_emf(a, stream_);
    mark(4);
    launch_update(a, live, in, out, stage, dt_dev, dt_host, stream_);
    mark(5);
    launch_fill_ghosts(g_, out, stream_);
    mark(6);
    launch_colloc_check(g_, out, &live, stage == 1 ? mask01 : mask2, false, stage == 2, true,
                        cfg_.gamma, ctl_, stream_);
    mark(7);
  }
  if (step_end) launch_step_end(ctl_, stream_);
}

Ctl MhdSolver2D::read_ctl() {
  ck(cudaMemcpyAsync(ctl_host_, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, stream_), "ctl read");
  ck(cudaStreamSynchronize(stream_), "step");
  return *ctl_host_;
}

// Errors that the reference raises as exceptions (mhd_solver.cpp:1178-1222,
// 1306-1308).  The live register is untouched when they are raised.
void MhdSolver2D::throw_status(int status) {
  if (status & (kStatusNotAdmissible | kStatusNotSolenoidal | kStatusCflNonFinite)) {
    seeded_dirty_ = true;
    front_order_ = 0;
  }
  if (status & kStatusNotSolenoidal)
    throw std::invalid_argument(
        "MhdSolver2D: live magnetic field is not discretely divergence-free");
  if (status & kStatusNotAdmissible)
    throw std::invalid_argument(
        "MhdSolver2D: live state must have finite components, rho > 0, and gas pressure > 0 "
        "in every interior cell");
  if (status & kStatusCflNonFinite)
    throw std::runtime_error("MhdSolver2D: non-finite state encountered in CFL reduction");
}

}  // namespace qb

namespace qb {

void MhdSolver2D::promote() {
  std::swap(live_, next_);
  solver_owned_ = true;
  front_order_ = 0;
}

void MhdSolver2D::copy_state(const StateP& src, const StateP& dst) {
  const size_t bytes = sizeof(double) * size_t(g_.size());
  for (int c = 0; c < 8; ++c)
    ck(cudaMemcpyAsync(dst.c[c], src.c[c], bytes, cudaMemcpyDeviceToDevice, stream_), "copy");
  ck(cudaMemcpyAsync(dst.bxc, src.bxc, bytes, cudaMemcpyDeviceToDevice, stream_), "copy");
  ck(cudaMemcpyAsync(dst.byc, src.byc, bytes, cudaMemcpyDeviceToDevice, stream_), "copy");
}

// cfl_limit_for_collocation (mhd_solver.cpp:1228-1321): preflights, the
// order-matched reconstruction and the additive incident-face rate.  The
// stage-0 residual computed on the way is kept for the step that follows.
double MhdSolver2D::cfl_limit_for(int coll) {
  ensure_live_ready();
  const int order = coll > 0 ? 1 : cfg_.order;
  if (front_order_ != order || front_dt_mode_ == 0) {
    front_impl(order, 1, anchor_mode_);
    front_order_ = order;
    front_dt_mode_ = 1;
  }
  const Ctl c = read_ctl();
  if (c.status) {
    front_order_ = 0;
    throw_status(c.status);
  }
  if (!(c.dt > 0.0) || !std::isfinite(c.dt))
    throw std::runtime_error("MhdSolver2D: no finite positive CFL timestep is representable");
  return c.dt;
}

double MhdSolver2D::cfl_limit() { return cfl_limit_for(0); }

void MhdSolver2D::step_unchecked(double dt) {
  if (!(dt > 0.0) || !std::isfinite(dt))
    throw std::invalid_argument("MhdSolver2D: dt must be finite and positive");
  ensure_live_ready();
  advance_positive(dt);
}

void MhdSolver2D::step(double dt) {
  if (!(dt > 0.0) || !std::isfinite(dt))
    throw std::invalid_argument("MhdSolver2D: dt must be finite and positive");
  if (dt > cfl_limit())
    throw std::invalid_argument(
        "MhdSolver2D: dt exceeds the CFL stability limit for this grid and scheme");
  advance_positive(dt);
}

// mhd_solver.cpp:1411-1441
void MhdSolver2D::advance(double t_end, double dt) {
  if (!(t_end >= 0.0) || !std::isfinite(t_end))
    throw std::invalid_argument("MhdSolver2D::advance: t_end must be finite and non-negative");
  if (!(dt > 0.0) || !std::isfinite(dt))
    throw std::invalid_argument("MhdSolver2D::advance: dt must be finite and positive");
  double t = 0.0;
  while (t < t_end) {
    const double remaining = t_end - t;
    const double d = std::min(dt, remaining);
    if (!(d > 0.0) || !std::isfinite(d))
      throw std::runtime_error("MhdSolver2D::advance: timestep made no finite forward progress");
    step(d);
    if (d == remaining) {
      t = t_end;
    } else {
      const double nx = t + d;
      if (!(nx > t) || !std::isfinite(nx))
        throw std::runtime_error("MhdSolver2D::advance: timestep made no finite forward progress");
      t = nx;
    }
  }
}

// Fast path: one full-interval configured-order substep whose candidates
// are all admissible.  Anything else enters the reference's retry
// controller (mhd_solver.cpp:965-1143).
void MhdSolver2D::advance_positive(double dt) {
  const int prev = last_substeps_;
  if (front_order_ != cfg_.order) front_impl(cfg_.order, 0, -1);
  finish_impl(cfg_.order, nullptr, dt, false);
  front_order_ = 0;
  const Ctl c = read_ctl();
  if (c.status == 0) {
    promote();
    last_substeps_ = 1;
    return;
  }
  if (c.status & ~kStatusRetry) {
    last_substeps_ = prev;
    throw_status(c.status);
  }
  controller(dt, from_bits(c.theta), c.anchor_ok != 0);
}

// The positivity controller after a rejected full-interval high-order
// candidate: retry the interval with the low-order LF operator when the live
// state is admissible under the two-face collocation, otherwise shrink the
// substep by the admissible fraction; grow again after accepted substeps.
void MhdSolver2D::controller(double dt, double theta, bool anchor) {
  const int prev = last_substeps_;
  copy_state(st_[live_], st_[4]);
  try {
    double remaining = dt, trial = dt;
    bool low_interval = false, high = true, pending = true;
    int retries = 0, attempts = 1;
    last_substeps_ = 0;
    // message of mhd_solver.cpp:1009-1020, counters at the point of failure
    auto no_progress = [&](const char* what, double th) {
      low_order_ = 0;
      std::ostringstream m;
      m.precision(17);
      m << "MhdSolver2D: " << what << " cannot advance time (trial=" << trial
        << ", remaining=" << remaining << ", theta=" << th
        << ", low_order=" << (low_interval ? "true" : "false") << ", retries=" << retries
        << ", accepted_substeps=" << last_substeps_ << ", attempts=" << attempts << ")";
      return std::runtime_error(m.str());
    };
    while (remaining > 0.0) {
      if (pending) {
        pending = false;
        low_order_ = 0;
        refresh_live_stats();
        if (++retries > 80)
          throw std::runtime_error("MhdSolver2D: unable to find a positive conservative substep");
        bool switched = false;
        if (high) {
          const Ctl c = read_ctl();
          const double anchor_theta = from_bits(c.anchor_theta);
          if (anchor_theta >= 1.0) {
            anchor = true;
            low_interval = true;
            low_order_ = 1;
            anchor_mode_ = 1;
            trial = std::min(trial, cfl_limit_for(1));
            if (!(trial > 0.0) || !std::isfinite(trial) || !(remaining - trial < remaining))
              throw no_progress("low-order CFL substep", anchor_theta);
            switched = true;
          }
        }
        if (!switched) {
          trial *= std::max(0.05, std::min(0.8, 0.8 * theta));
          low_order_ = low_interval ? 1 : 0;
          if (!(trial > 0.0) || !std::isfinite(trial) || !(remaining - trial < remaining))
            throw no_progress("positive conservative substep", theta);
        }
      }
      if (++attempts > 100000)
        throw std::runtime_error("MhdSolver2D: positivity controller exceeded its substep limit");
      trial = std::min(trial, remaining);
      anchor_mode_ = anchor ? 1 : 0;
      const int order = low_order_ ? 1 : cfg_.order;
      if (front_order_ != order) front_impl(order, 0, anchor_mode_);
      finish_impl(order, nullptr, trial, false);
      front_order_ = 0;
      const Ctl c = read_ctl();
      if (c.status & ~kStatusRetry) throw_status(c.status);
      if (c.status & kStatusRetry) {
        high = low_order_ == 0;
        theta = from_bits(c.theta);
        pending = true;
        continue;
      }
      promote();
      retries = 0;
      ++last_substeps_;
      low_order_ = low_interval ? 1 : 0;
      if (trial == remaining) break;
      const double nr = remaining - trial;
      if (!(nr > 0.0) || !(nr < remaining))
        throw std::runtime_error("MhdSolver2D: positivity substep made no finite time progress");
      remaining = nr;
      trial = std::min(std::min(2.0 * trial, remaining), cfl_limit_for(low_interval ? 1 : 0));
    }
    low_order_ = 0;
    anchor_mode_ = -1;
  } catch (...) {
    low_order_ = 0;
    anchor_mode_ = -1;
    last_substeps_ = prev;
    copy_state(st_[4], st_[live_]);
    front_order_ = 0;
    refresh_live_stats();
    cudaStreamSynchronize(stream_);
    throw;
  }
}

// mhd_solver.cpp:1323-1338
double MhdSolver2D::divergence_b_max() {
  ensure_live_ready();
  launch_fill_ghosts(g_, st_[live_], stream_);
  ck(cudaMemsetAsync(scalar_, 0, sizeof(unsigned long long), stream_), "memset");
  launch_divb_linf(g_, st_[live_], scalar_, stream_);
  unsigned long long b = 0;
  ck(cudaMemcpyAsync(&b, scalar_, sizeof b, cudaMemcpyDeviceToHost, stream_), "divb read");
  ck(cudaStreamSynchronize(stream_), "divb");
  return from_bits(b);
}

// mhd_solver.cpp:1376-1382 (Cartesian cell sums, compensated)
void MhdSolver2D::conserved_cell_totals(double* mass, double* energy) {
  launch_cell_sums(g_, st_[live_], sums_, sum_blocks_, stream_);
  std::vector<double> h(4 * size_t(sum_blocks_));
  ck(cudaMemcpyAsync(h.data(), sums_, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream_),
     "sums read");
  ck(cudaStreamSynchronize(stream_), "sums");
  long double m = 0.0L, e = 0.0L;
  for (int b = 0; b < sum_blocks_; ++b) {
    m += (long double)h[4 * b] + (long double)h[4 * b + 1];
    e += (long double)h[4 * b + 2] + (long double)h[4 * b + 3];
  }
  *mass = double(m);
  *energy = double(e);
}

// One graph per register assignment: a complete auto-dt step from the live
// register into the next one (the roles swap each accepted step).
void MhdSolver2D::build_graphs() {
  if (graph_[0]) return;
  const int keep_live = live_, keep_next = next_;
  for (int k = 0; k < 2; ++k) {
    live_ = k == 0 ? 0 : 3;
    next_ = k == 0 ? 3 : 0;
    cudaGraph_t graph;
    ck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
    front_impl(cfg_.order, 2, -1);
    finish_impl(cfg_.order, &ctl_->dt, 0.0, true);
    ck(cudaStreamEndCapture(stream_, &graph), "capture end");
    ck(cudaGraphInstantiate(&graph_[k], graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);
  }
  live_ = keep_live;
  next_ = keep_next;
}

int MhdSolver2D::advance_auto(double* t_io, double t_end, int max_steps) {
  double t = *t_io;
  if (max_steps <= 0 || !(t < t_end)) return 0;
  ensure_live_ready();
  build_graphs();
  front_order_ = 0;
  int total = 0;
  while (total < max_steps && t < t_end) {
    launch_set_time(ctl_, t, t_end, stream_);
    const int batch = std::min(max_steps - total, 64);
    int lv = live_;
    for (int b = 0; b < batch; ++b) {
      ck(cudaGraphLaunch(graph_[lv == 0 ? 0 : 1], stream_), "graph launch");
      lv = lv == 0 ? 3 : 0;
    }
    const Ctl c = read_ctl();
    for (int s = 0; s < c.steps_done; ++s) promote();
    total += c.steps_done;
    t = c.t;
    last_substeps_ = c.steps_done > 0 ? 1 : last_substeps_;
    if (c.status & kStatusDone) break;
    if (c.status & kStatusRetry) {
      controller(c.dt, from_bits(c.theta), c.anchor_ok != 0);
      const double rem = t_end - t;
      t = c.dt == rem ? t_end : t + c.dt;
      ++total;
      continue;
    }
    if (c.status) throw_status(c.status);
  }
  *t_io = t;
  return total;
}

}  // namespace qb

namespace qb {

void MhdSolver2D::mark(int phase) {
  if (!marks_) return;
  cudaEvent_t e;
  ck(cudaEventCreate(&e), "event");
  ck(cudaEventRecord(e, stream_), "event record");
  marks_[nmarks_++] = Mark{phase, e};
}

// One API-mode step (cfl_limit + step_unchecked) with an event after every
// launch group; the elapsed time between consecutive events is charged to the
// group.  The step is a real step: the live state advances.
void MhdSolver2D::profile_step(double* ms) {
  ensure_live_ready();
  front_order_ = 0;
  Mark buf[64];
  marks_ = buf;
  nmarks_ = 0;
  cudaEvent_t start;
  ck(cudaEventCreate(&start), "event");
  ck(cudaEventRecord(start, stream_), "event record");
  try {
    front_impl(cfg_.order, 1, -1);
    finish_impl(cfg_.order, &ctl_->dt, 0.0, false);
  } catch (...) {
    marks_ = nullptr;
    throw;
  }
  marks_ = nullptr;
  const Ctl c = read_ctl();
  for (int p = 0; p < kPhases; ++p) ms[p] = 0.0;
  cudaEvent_t prev = start;
  for (int k = 0; k < nmarks_; ++k) {
    float t = 0.f;
    ck(cudaEventElapsedTime(&t, prev, buf[k].ev), "elapsed");
    ms[buf[k].phase] += t;
    prev = buf[k].ev;
  }
  for (int k = 0; k < nmarks_; ++k) cudaEventDestroy(buf[k].ev);
  cudaEventDestroy(start);
  front_order_ = 0;
  if (c.status) throw_status(c.status & ~kStatusRetry);
  if (c.status & kStatusRetry) throw std::runtime_error("MhdSolver2D: profiled step was rejected");
  promote();
}

double MhdSolver2D::time_auto_steps(int steps, int* done) {
  ensure_live_ready();
  build_graphs();
  front_order_ = 0;
  launch_set_time(ctl_, 0.0, std::numeric_limits<double>::infinity(), stream_);
  cudaEvent_t a, b;
  ck(cudaEventCreate(&a), "event");
  ck(cudaEventCreate(&b), "event");
  ck(cudaEventRecord(a, stream_), "event record");
  int lv = live_;
  for (int k = 0; k < steps; ++k) {
    ck(cudaGraphLaunch(graph_[lv == 0 ? 0 : 1], stream_), "graph launch");
    lv = lv == 0 ? 3 : 0;
  }
  ck(cudaEventRecord(b, stream_), "event record");
  const Ctl c = read_ctl();
  float ms = 0.f;
  ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  for (int s = 0; s < c.steps_done; ++s) promote();
  if (done) *done = c.steps_done;
  if (c.status & ~kStatusDone) throw_status(c.status & ~kStatusRetry);
  return ms;
}

}  // namespace qb
