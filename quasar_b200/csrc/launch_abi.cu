// extern "C" per-kernel launch interface (declarations:
// include/quasar_mhd_launch.h), the C ABI of the reference's backend seam
// include/quasar/physics/mhd/kernels.hpp.  Each function checks its
// arguments on the host, queues the kernels the fused step uses for the same
// work, and reports launch failures; reductions synchronize the stream and
// return their scalar.
#include "../../include/quasar_mhd_ext.h"
#include "../../include/quasar_mhd_launch.h"
#include "mhd_kernels.cuh"
#include "mhd_solver.cuh"
#include "noalloc.cuh"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>

namespace qb {
int capi_guarded(const std::function<void()>& f);
}

namespace {

using qb::FluxP;
using qb::Grid;
using qb::IfaceP;
using qb::StageArgs;
using qb::StateP;

[[noreturn]] void bad(const char* fn, const std::string& what) {
  throw std::invalid_argument(std::string(fn) + ": " + what);
}

void check_cuda(const char* fn, cudaError_t e) {
  if (e != cudaSuccess) throw qb::CudaError(std::string(fn) + ": " + cudaGetErrorString(e));
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

int ghost_width(int order) { return order == 7 ? 4 : order == 5 ? 3 : 2; }

Grid make_grid(const char* fn, const qmhd_grid* q, const int* flags) {
  if (!q) bad(fn, "null grid");
  if (q->nx < 1 || q->ny < 1) bad(fn, "grid extents must be positive");
  if (q->nghost < 2 || q->nghost > 4) bad(fn, "nghost must be 2, 3 or 4");
  if (!(std::isfinite(q->dx) && q->dx > 0.0 && std::isfinite(q->dy) && q->dy > 0.0))
    bad(fn, "grid spacings must be finite and positive");
  Grid g{};
  g.nx = q->nx;
  g.ny = q->ny;
  g.ng = q->nghost;
  g.pitch = q->nx + 2 * q->nghost;
  g.dx = q->dx;
  g.dy = q->dy;
  for (int s = 0; s < 4; ++s) {
    const int m = flags ? flags[s] : 0;
    if (m < 0 || m > 2)
      bad(fn, "boundary flag " + std::to_string(m) + " is not 0 periodic, 1 outflow or 2 wall");
    g.bc[s] = m;
  }
  if ((g.bc[0] == 0) != (g.bc[1] == 0) || (g.bc[2] == 0) != (g.bc[3] == 0))
    bad(fn, "a periodic side needs a periodic opposite side");
  return g;
}

void check_order(const char* fn, const Grid& g, int order) {
  if (order != 1 && order != 2 && order != 5 && order != 7)
    bad(fn, "scheme_order must be 1, 2, 5 or 7");
  if (order != 1 && ghost_width(order) != g.ng)
    bad(fn, "nghost " + std::to_string(g.ng) + " does not match scheme_order " +
                std::to_string(order) + " (needs " + std::to_string(ghost_width(order)) + ")");
}

void check_gamma(const char* fn, double gamma) {
  if (!(std::isfinite(gamma) && gamma > 1.0)) bad(fn, "gamma must be finite and > 1");
}

void check_dir(const char* fn, int dir) {
  if (dir != 0 && dir != 1) bad(fn, "dir must be 0 (x) or 1 (y)");
}

void cartesian_only(const char* fn, int cylindrical) {
  if (cylindrical) bad(fn, "cylindrical geometry is not supported");
}

StateP state_of(const char* fn, const qmhd_field* f, double* bxc = nullptr,
                double* byc = nullptr) {
  if (!f) bad(fn, "null field");
  StateP s{};
  for (int c = 0; c < 8; ++c) {
    if (!f->comp[c]) bad(fn, "null field component " + std::to_string(c));
    s.c[c] = f->comp[c];
  }
  s.bxc = bxc;
  s.byc = byc;
  return s;
}

FluxP flux_of(const char* fn, const qmhd_field* f) {
  const StateP s = state_of(fn, f);
  FluxP r{};
  for (int c = 0; c < 8; ++c) r.f[c] = s.c[c];
  return r;
}

IfaceP iface_of(const char* fn, const qmhd_iface* v) {
  if (!v) bad(fn, "null interface states");
  IfaceP r{};
  for (int c = 0; c < 8; ++c) {
    if (!v->left[c] || !v->right[c]) bad(fn, "null interface component " + std::to_string(c));
    r.L[c] = v->left[c];
    r.R[c] = v->right[c];
  }
  return r;
}

unsigned long long* scratch_of(const char* fn, void* scratch) {
  if (!scratch) bad(fn, "null scratch");
  if (reinterpret_cast<std::uintptr_t>(scratch) % 8 != 0) bad(fn, "scratch must be 8-byte aligned");
  return static_cast<unsigned long long*>(scratch);
}

qb::Ctl* zero_ctl(const char* fn) {
  qb::Ctl* z = nullptr;
  check_cuda(fn, qb::abi_zero_ctl(&z));
  return z;
}

double from_bits(unsigned long long b) {
  double d;
  static_assert(sizeof d == sizeof b, "64-bit double");
  std::memcpy(&d, &b, sizeof d);
  return d;
}

unsigned long long to_bits(double d) {
  unsigned long long b;
  std::memcpy(&b, &d, sizeof b);
  return b;
}

// Copy n reduced words back and wait for them.
void read_back(const char* fn, const unsigned long long* dev, unsigned long long* host, int n,
               cudaStream_t s) {
  check_cuda(fn, cudaGetLastError());
  check_cuda(fn, cudaMemcpyAsync(host, dev, n * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
  check_cuda(fn, cudaStreamSynchronize(s));
}

// Stage arguments of a standalone launch: grid, order, gamma and the zero
// control block; the caller fills the buffers the kernel reads.
StageArgs stage_args(const char* fn, const Grid& g, int order, double gamma) {
  StageArgs a{};
  a.g = g;
  a.order = order;
  a.gamma = gamma;
  a.ctl = zero_ctl(fn);
  return a;
}

}  // namespace

extern "C" {

int qmhd_launch_reconstruct(const qmhd_grid* grid, const qmhd_field* u, double* cell_bx,
                            double* cell_by, int dir, const qmhd_iface* out, int scheme_order,
                            const int flags[4], double gamma, void* stream, int rate_only) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_reconstruct";
    const Grid g = make_grid(fn, grid, flags);
    check_order(fn, g, scheme_order);
    check_dir(fn, dir);
    check_gamma(fn, gamma);
    // rate_only only selects reconstructed_rate_state_admissible, which
    // forwards to reconstructed_state_admissible (mhd_reconstruct.hip:449-452,
    // 654-659): the same reconstruction either way
    (void)rate_only;
    if (!cell_bx || !cell_by) bad(fn, "null collocation scratch");
    const StateP st = state_of(fn, u, cell_bx, cell_by);
    const IfaceP io = iface_of(fn, out);
    StageArgs a = stage_args(fn, g, scheme_order, gamma);
    a.u = st;
    (dir == 0 ? a.ix : a.iy) = io;
    const cudaStream_t s = as_stream(stream);
    qb::launch_abi_collocate(g, 0, a.u.c[5], cell_bx, s);
    qb::launch_abi_collocate(g, 1, a.u.c[6], cell_by, s);
    qb::launch_reconstruct(a, dir, s);
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_hlld_flux(const qmhd_grid* grid, const qmhd_iface* iface, int dir,
                          const qmhd_field* flux_out, const int flags[4], double gamma,
                          void* stream, int hll_only, int scheme_order, const int ownership[4]) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_hlld_flux";
    const Grid g = make_grid(fn, grid, flags);
    check_order(fn, g, scheme_order);
    check_dir(fn, dir);
    check_gamma(fn, gamma);
    if ((hll_only != 0) != (scheme_order <= 1))
      bad(fn, "hll_only must be set exactly for scheme_order 1 (the LF retry flux)");
    if (ownership)
      for (int q = 0; q < 4; ++q)
        if (ownership[q] != 1) bad(fn, "partial face ownership is not supported");
    const IfaceP in = iface_of(fn, iface);
    const FluxP fo = flux_of(fn, flux_out);
    StageArgs a = stage_args(fn, g, scheme_order, gamma);
    (dir == 0 ? a.ix : a.iy) = in;
    (dir == 0 ? a.fx : a.fy) = fo;
    qb::launch_face_flux(a, dir, false, as_stream(stream));
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_flux_difference(const qmhd_grid* grid, const qmhd_field* flux, int dir,
                                const qmhd_field* dudt, void* stream, int cylindrical) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_flux_difference";
    const Grid g = make_grid(fn, grid, nullptr);
    check_dir(fn, dir);
    cartesian_only(fn, cylindrical);
    qb::launch_abi_flux_difference(g, flux_of(fn, flux), dir, flux_of(fn, dudt),
                                   as_stream(stream));
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_ct_emf_prepare(const qmhd_grid* grid, const qmhd_field* u, double* cell_bx,
                               double* cell_by, const qmhd_iface* ifx, const qmhd_iface* ify,
                               const int flags[4], const qmhd_emf* emf, double gamma,
                               void* stream, int scheme_order, int hll_only) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_ct_emf_prepare";
    const Grid g = make_grid(fn, grid, flags);
    check_order(fn, g, scheme_order);
    check_gamma(fn, gamma);
    if ((hll_only != 0) != (scheme_order <= 1))
      bad(fn, "hll_only must be set exactly for scheme_order 1 (the LF retry flux)");
    if (!emf || !emf->face_ez_x || !emf->face_ez_y || !emf->no_jump_x || !emf->no_jump_y ||
        !emf->cell_ez)
      bad(fn, "null EMF table");
    if (!cell_bx || !cell_by) bad(fn, "null collocation scratch");
    const StateP st = state_of(fn, u, cell_bx, cell_by);
    const IfaceP vx = iface_of(fn, ifx), vy = iface_of(fn, ify);
    StageArgs a = stage_args(fn, g, scheme_order, gamma);
    a.u = st;
    a.ix = vx;
    a.iy = vy;
    a.xemf = emf->face_ez_x;
    a.yemf = emf->face_ez_y;
    a.xnj = emf->no_jump_x;
    a.ynj = emf->no_jump_y;
    a.cell_ez = emf->cell_ez;
    const cudaStream_t s = as_stream(stream);
    // face tables only: the flux records are not part of this launch
    qb::launch_face_flux(a, 0, false, s);
    qb::launch_face_flux(a, 1, false, s);
    qb::launch_abi_collocate(g, 0, a.u.c[5], cell_bx, s);
    qb::launch_abi_collocate(g, 1, a.u.c[6], cell_by, s);
    qb::launch_cell_emf(a, false, s);
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_ct_emf_finish(const qmhd_grid* grid, const int flags[4], const qmhd_emf* emf,
                              void* stream, int scheme_order, int cylindrical) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_ct_emf_finish";
    const Grid g = make_grid(fn, grid, flags);
    check_order(fn, g, scheme_order);
    cartesian_only(fn, cylindrical);
    if (!emf || !emf->face_ez_x || !emf->face_ez_y || !emf->no_jump_x || !emf->no_jump_y ||
        !emf->cell_ez || !emf->corner_ez)
      bad(fn, "null EMF table");
    StageArgs a = stage_args(fn, g, scheme_order, 5.0 / 3.0);
    a.xemf = emf->face_ez_x;
    a.yemf = emf->face_ez_y;
    a.xnj = emf->no_jump_x;
    a.ynj = emf->no_jump_y;
    a.cell_ez = emf->cell_ez;
    a.ez = emf->corner_ez;
    qb::launch_corner_emf(a, as_stream(stream));
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_emf_curl_rate(const qmhd_grid* grid, const qmhd_emf* emf, const qmhd_field* dudt,
                              void* stream, int cylindrical) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_emf_curl_rate";
    const Grid g = make_grid(fn, grid, nullptr);
    cartesian_only(fn, cylindrical);
    if (!emf || !emf->corner_ez) bad(fn, "null corner EMF");
    const StateP d = state_of(fn, dudt);
    qb::launch_abi_curl_rate(g, emf->corner_ez, d.c[5], d.c[6], as_stream(stream));
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_rk_stage(const qmhd_grid* grid, const qmhd_field* out, const qmhd_field* un,
                         const qmhd_field* ustage, const qmhd_field* dudt, double a, double b,
                         double c_dt, void* stream) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_rk_stage";
    const Grid g = make_grid(fn, grid, nullptr);
    if (!(std::isfinite(a) && std::isfinite(b) && std::isfinite(c_dt)))
      bad(fn, "stage weights must be finite");
    const StateP o = state_of(fn, out), n = state_of(fn, un);
    // operands with a zero weight are never read and may be absent
    const StateP us = b != 0.0 ? state_of(fn, ustage) : n;
    const FluxP d = c_dt != 0.0 ? flux_of(fn, dudt) : FluxP{{n.c[0], n.c[1], n.c[2], n.c[3],
                                                            n.c[4], n.c[5], n.c[6], n.c[7]}};
    qb::launch_abi_rk_stage(g, o, n, us, d, a, b, c_dt, as_stream(stream));
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_admissible_fraction(const qmhd_grid* grid, const qmhd_field* base,
                                    const qmhd_field* candidate, double rho_floor,
                                    double p_floor, double gamma, void* scratch,
                                    double* host_theta, void* stream, int collocation_order) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_admissible_fraction";
    const Grid g = make_grid(fn, grid, nullptr);
    check_gamma(fn, gamma);
    if (!host_theta) bad(fn, "null host_theta");
    if (collocation_order != 0 && collocation_order != 1)
      bad(fn, "collocation_order must be 0 or 1");
    if (!(std::isfinite(rho_floor) && std::isfinite(p_floor)))
      bad(fn, "floors must be finite");
    unsigned long long* acc = scratch_of(fn, scratch);
    const cudaStream_t s = as_stream(stream);
    // q = E - kinetic - magnetic bounds p / (gamma - 1) (mhd_reduce.hip:1044)
    const double q_floor = p_floor / (gamma - 1.0);
    qb::launch_abi_set_u64(acc, 1, to_bits(1.0), s);
    qb::launch_abi_admissible(g, state_of(fn, base), state_of(fn, candidate), rho_floor, q_floor,
                              collocation_order, acc, s);
    unsigned long long bits = 0;
    read_back(fn, acc, &bits, 1, s);
    *host_theta = from_bits(bits);
  });
}

int qmhd_launch_cfl_max_rate(const qmhd_grid* grid, const qmhd_iface* ifx, const qmhd_iface* ify,
                             double gamma, void* scratch, qmhd_cfl_rate* host_rate, void* stream,
                             int scheme_order, int cylindrical, const int flags[4]) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_cfl_max_rate";
    const Grid g = make_grid(fn, grid, flags);
    check_order(fn, g, scheme_order);
    check_gamma(fn, gamma);
    cartesian_only(fn, cylindrical);
    if (!host_rate) bad(fn, "null host_rate");
    unsigned long long* acc = scratch_of(fn, scratch);
    const cudaStream_t s = as_stream(stream);
    qb::launch_abi_set_u64(acc, 1, 0ull, s);
    qb::launch_abi_cfl_rate(g, iface_of(fn, ifx), iface_of(fn, ify), scheme_order, gamma, acc, s);
    unsigned long long bits = 0;
    read_back(fn, acc, &bits, 1, s);
    host_rate->scaled_max_rate = from_bits(bits);
    host_rate->rate_scale = 1.0;
  });
}

int qmhd_launch_ct_divb_linf(const qmhd_grid* grid, const qmhd_field* u, void* scratch,
                             double* host_linf, void* stream, int cylindrical) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_ct_divb_linf";
    const Grid g = make_grid(fn, grid, nullptr);
    cartesian_only(fn, cylindrical);
    if (!host_linf) bad(fn, "null host_linf");
    unsigned long long* acc = scratch_of(fn, scratch);
    const cudaStream_t s = as_stream(stream);
    qb::launch_abi_set_u64(acc, 1, 0ull, s);
    qb::launch_divb_linf(g, state_of(fn, u), acc, s);
    unsigned long long bits = 0;
    read_back(fn, acc, &bits, 1, s);
    *host_linf = from_bits(bits);
  });
}

int qmhd_launch_ct_divb_relative_linf(const qmhd_grid* grid, const qmhd_field* u, void* scratch,
                                      double* host_linf, void* stream, int cylindrical,
                                      int solver_owned) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_ct_divb_relative_linf";
    const Grid g = make_grid(fn, grid, nullptr);
    cartesian_only(fn, cylindrical);
    if (!host_linf) bad(fn, "null host_linf");
    unsigned long long* acc = scratch_of(fn, scratch);
    const cudaStream_t s = as_stream(stream);
    qb::launch_abi_set_u64(acc, 2, 0ull, s);
    qb::launch_abi_divb_relative(g, state_of(fn, u), solver_owned ? 1 : 0, acc, s);
    unsigned long long bits[2] = {0, 0};
    read_back(fn, acc, bits, 2, s);
    const double res = from_bits(bits[0]), scale = from_bits(bits[1]);
    *host_linf = res == 0.0 ? 0.0 : res / scale;
  });
}

static int fill_ghosts(const char* fn, const qmhd_grid* grid, const qmhd_field* u, int side,
                       int mode, void* stream, int parts) {
  return qb::capi_guarded([&] {
    const Grid g = make_grid(fn, grid, nullptr);
    if (side < 0 || side > 3) bad(fn, "side must be 0..3 (x_lo, x_hi, y_lo, y_hi)");
    if (mode < 0 || mode > 2) bad(fn, "mode must be 0 periodic, 1 outflow or 2 wall");
    qb::launch_abi_fill_side(g, state_of(fn, u), side, mode, parts, as_stream(stream));
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_fill_ghosts_fluid(const qmhd_grid* grid, const qmhd_field* u, int side, int mode,
                                  void* stream) {
  return fill_ghosts("qmhd_launch_fill_ghosts_fluid", grid, u, side, mode, stream, 1);
}

int qmhd_launch_fill_ghosts_field(const qmhd_grid* grid, const qmhd_field* u, int side, int mode,
                                  void* stream) {
  return fill_ghosts("qmhd_launch_fill_ghosts_field", grid, u, side, mode, stream, 2);
}

int qmhd_launch_collocate_face_to_cell(const qmhd_grid* grid, int axis, const double* face,
                                       double* cell, void* stream) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_collocate_face_to_cell";
    const Grid g = make_grid(fn, grid, nullptr);
    if (axis != 0 && axis != 1) bad(fn, "axis must be 0 (bx_face) or 1 (by_face)");
    if (!face || !cell) bad(fn, "null array");
    if (face == cell) bad(fn, "cell must not alias face");
    qb::launch_abi_collocate(g, axis, face, cell, as_stream(stream));
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_seed_initial_state(const qmhd_grid* grid, const qmhd_ic_spec* spec,
                                   const qmhd_field* out, double* raw_magnetic, double* cell_bx,
                                   double* cell_by, int* status, void* stream) {
  return qb::capi_guarded([&] {
    const char* fn = "qmhd_launch_seed_initial_state";
    const Grid g = make_grid(fn, grid, nullptr);
    if (!spec) bad(fn, "null spec");
    if (spec->kind < 0 || spec->kind > 5) bad(fn, "kind must be 0..5");
    check_gamma(fn, spec->gamma);
    if (!(std::isfinite(spec->magnetic_scale) && spec->magnetic_scale > 0.0))
      bad(fn, "magnetic unit scale must be finite and positive");
    if (!(std::isfinite(spec->lx) && spec->lx > 0.0 && std::isfinite(spec->ly) && spec->ly > 0.0))
      bad(fn, "lx and ly must be finite and positive");
    if (!raw_magnetic || !cell_bx || !cell_by || !status) bad(fn, "null scratch or status");
    const StateP st = state_of(fn, out, cell_bx, cell_by);
    qb::SeedSpec s{};
    s.kind = spec->kind;
    s.lx = spec->lx; s.ly = spec->ly; s.ox = spec->origin_x; s.oy = spec->origin_y;
    s.gamma = spec->gamma;
    s.magnetic_scale = spec->magnetic_scale;
    s.interface_x = spec->interface_x;
    for (int c = 0; c < 8; ++c) {
      s.left[c] = spec->left[c];
      s.right[c] = spec->right[c];
    }
    s.rho = spec->rho; s.pressure = spec->pressure; s.b0 = spec->b0;
    s.total_b0 = spec->total_b0; s.amplitude = spec->amplitude;
    s.wavenumber = spec->wavenumber; s.mvs = spec->magnetic_velocity_scale;
    for (int c = 0; c < 3; ++c) s.b_uniform[c] = spec->b_uniform[c];
    s.center[0] = spec->center[0]; s.center[1] = spec->center[1];
    s.r_in = spec->r_in; s.r0 = spec->r0; s.r1 = spec->r1;
    s.rho_in = spec->rho_in; s.rho_out = spec->rho_out; s.p_in = spec->p_in;
    s.p_out = spec->p_out; s.p_core = spec->p_core; s.p_ambient = spec->p_ambient;
    s.rho_ambient = spec->rho_ambient; s.u0 = spec->u0; s.blob_half = spec->blob_half;
    qb::launch_abi_seed(g, s, st, raw_magnetic, status, as_stream(stream));
    check_cuda(fn, cudaGetLastError());
  });
}

int qmhd_launch_conserved_cell_sums(const qmhd_grid* grid, const qmhd_field* u, int cylindrical,
                                    void* stream, double* mass, double* energy) {
  if (cylindrical) {
    return qb::capi_guarded([&] {
      bad("qmhd_launch_conserved_cell_sums", "cylindrical geometry is not supported");
    });
  }
  if (!grid || !u) {
    return qb::capi_guarded(
        [&] { bad("qmhd_launch_conserved_cell_sums", "null grid or field"); });
  }
  return qmhd_conserved_cell_totals_device(u->comp[0], u->comp[4], grid->nx, grid->ny,
                                           grid->nghost, stream, mass, energy);
}

}  // extern "C"
