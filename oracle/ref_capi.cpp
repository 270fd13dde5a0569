// C-ABI driver over the reference's OWN, unmodified MHD solver
// (quasar::mhd::MhdSolver2D, src/physics/mhd/mhd_solver.cpp) compiled for the
// host through oracle/shim.  Test infrastructure only: it is the parity oracle
// that pins oracle/mhd_oracle.cpp and the CUDA product, and the timed CPU
// baseline of bench.py.  It is built by oracle/build_ref.sh into oracle/_ref/.
//
// Component order everywhere: rho, mx, my, mz, energy, bx_face, by_face,
// bz_cell (mhd_field.hpp:17-29).  Arrays are padded storage of
// (nx+2g)*(ny+2g) doubles, index (i+g)+(nx+2g)*(j+g) (core/grid.hpp:158-161).

// The stage-debug entry points read the solver's interface/flux/EMF scratch,
// which the reference keeps private.  Opening them here is the harness's only
// intrusion; nothing in the reference's arithmetic changes.
#define private public
#include "quasar/physics/mhd/mhd_solver.hpp"
#undef private

#include "quasar/physics/mhd/initial_conditions.hpp"
#include "quasar/numerics/hlld_core.hpp"
#include "quasar/numerics/mhd_eigensystem.hpp"
#include "quasar/numerics/mp_limiter.hpp"
#include "quasar/numerics/mhd_background_metrics.hpp"
#include "quasar/physics/mhd/kernels.hpp"

#include <cstring>
#include <exception>
#include <string>
#include <vector>

using quasar::Real;
using quasar::mhd::MhdField2D;
using quasar::mhd::MhdSolver2D;

namespace {

thread_local std::string g_error;

int fail(const std::exception& e) {
  g_error = e.what();
  return -1;
}

const char* const kComp[8] = {"rho",    "mx",      "my",      "mz",
                              "energy", "bx_face", "by_face", "bz_cell"};

quasar::backend::DeviceBuffer<Real>& comp(MhdField2D<Real>& f, int c) {
  switch (c) {
    case 0: return f.rho;
    case 1: return f.mx;
    case 2: return f.my;
    case 3: return f.mz;
    case 4: return f.energy;
    case 5: return f.bx_face;
    case 6: return f.by_face;
    default: return f.bz_cell;
  }
}

const char* bc_name(int mode) {
  switch (mode) {
    case 0: return "periodic";
    case 1: return "outflow";
    default: return "wall";
  }
}

}  // namespace

extern "C" {

const char* qref_last_error() { return g_error.c_str(); }

// order: 2 (muscl_minmod), 5 (mp5) or 7 (mp7).  bc[4] = x_lo,x_hi,y_lo,y_hi
// modes 0 periodic, 1 outflow, 2 wall.
void* qref_create(int nx, int ny, double lx, double ly, double ox, double oy,
                  int order, double gamma, double cfl, const int* bc) {
  try {
    quasar::mhd::MhdConfig cfg;
    const int ng = order == 7 ? 4 : order == 5 ? 3 : 2;
    cfg.grid = quasar::Grid2D{nx, ny, lx, ly, ox, oy, ng};
    cfg.reconstruction = order == 7 ? "mp7" : order == 5 ? "mp5" : "muscl_minmod";
    cfg.gamma = gamma;
    cfg.cfl = cfl;
    for (int s = 0; s < 4; ++s) {
      cfg.boundary.fluid[s] = bc_name(bc[s]);
      cfg.boundary.field[s] = bc_name(bc[s]);
    }
    return new MhdSolver2D{cfg};
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

void qref_destroy(void* h) { delete static_cast<MhdSolver2D*>(h); }

int qref_grid(void* h, int* nx, int* ny, int* ng) {
  const auto g = static_cast<MhdSolver2D*>(h)->grid();
  *nx = g.nx;
  *ny = g.ny;
  *ng = g.nghost;
  return 0;
}

int qref_seed(void* h, int c, const double* data, size_t n) {
  try {
    static_cast<MhdSolver2D*>(h)->seed_state(
        kComp[c], std::vector<Real>(data, data + n));
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

// Raw storage read of the live register (face arrays NOT collocated).
int qref_read(void* h, int c, double* out, size_t n) {
  try {
    auto* s = static_cast<MhdSolver2D*>(h);
    auto& buf = comp(s->rk_[0], c);
    if (n != buf.size()) throw std::invalid_argument("qref_read: size");
    buf.copy_to_host(out, n);
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

int qref_cfl(void* h, double* dt) {
  try {
    *dt = static_cast<MhdSolver2D*>(h)->cfl_limit();
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

int qref_step(void* h, double dt) {
  try {
    static_cast<MhdSolver2D*>(h)->step_unchecked(dt);
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

int qref_substeps(void* h) {
  return static_cast<MhdSolver2D*>(h)->last_positivity_substeps();
}

// The solver's own live-state solenoidality measure (the quantity
// ensure_live_state_solenoidal, mhd_solver.cpp:1196-1222, compares with
// numerics::kDiscreteSolenoidalTolerance) on the live register after the
// boundary fill the preflight runs behind (mhd_solver.cpp:697-700), with the
// provenance given explicitly: solver_owned = 1 is the test of a state the
// solver stepped itself, 0 the stricter one of a seeded state.
int qref_divb_relative(void* h, int solver_owned, double* out) {
  try {
    auto* s = static_cast<MhdSolver2D*>(h);
    s->fill_ghosts(s->rk_[0]);
    Real v = Real{0};
    quasar::mhd::launch_mhd_ct_divb_relative_linf(s->rk_[0], s->divb_scratch_, &v, nullptr,
                                                  s->is_cylindrical(), solver_owned != 0);
    *out = v;
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

double qref_solenoidal_tolerance() { return quasar::numerics::kDiscreteSolenoidalTolerance; }

int qref_divb(void* h, double* out) {
  try {
    *out = static_cast<MhdSolver2D*>(h)->divergence_b_max();
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

int qref_totals(void* h, double* mass, double* energy) {
  try {
    const auto t = static_cast<MhdSolver2D*>(h)->conserved_cell_totals();
    *mass = t.mass;
    *energy = t.energy;
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

// One residual evaluation L(u) of an arbitrary padded state through the
// solver's own compute_residual (mhd_solver.cpp:665-670), on stage register 1.
// Outputs (each padded, NULL to skip):
//   dudt[8]             the residual, B slots = CT curl rate
//   ifx[16], ify[16]    reconstructed L (8) then R (8) interface states
//   fx[8], fy[8]        face fluxes
//   ez                  corner EMF; cell_ez, xface_ez, yface_ez  CT tables
int qref_residual(void* h, const double* const* in8, double* const* dudt,
                  double* const* ifx, double* const* ify, double* const* fx,
                  double* const* fy, double* ez, double* cell_ez,
                  double* xface_ez, double* yface_ez) {
  try {
    auto* s = static_cast<MhdSolver2D*>(h);
    s->internal_integrator_access_ = true;
    MhdField2D<Real>& u = s->rk_[1];
    for (int c = 0; c < 8; ++c) {
      auto& b = comp(u, c);
      b.copy_from_host(in8[c], b.size());
    }
    s->invalidate_interface_cache();
    s->compute_residual(u, s->residual_);
    s->internal_integrator_access_ = false;
    const size_t n = u.rho.size();
    if (dudt) for (int c = 0; c < 8; ++c) comp(s->residual_, c).copy_to_host(dudt[c], n);
    auto dump_iface = [&](const quasar::numerics::MhdInterfaceStates<Real>& st,
                          double* const* out) {
      if (!out) return;
      const quasar::backend::DeviceBuffer<Real>* b[16] = {
          &st.Lrho, &st.Lmx, &st.Lmy, &st.Lmz, &st.Lenergy, &st.Lbx, &st.Lby, &st.Lbz,
          &st.Rrho, &st.Rmx, &st.Rmy, &st.Rmz, &st.Renergy, &st.Rbx, &st.Rby, &st.Rbz};
      for (int c = 0; c < 16; ++c) b[c]->copy_to_host(out[c], n);
    };
    dump_iface(s->ifx_, ifx);
    dump_iface(s->ify_, ify);
    if (fx) for (int c = 0; c < 8; ++c) comp(s->flux_x_, c).copy_to_host(fx[c], n);
    if (fy) for (int c = 0; c < 8; ++c) comp(s->flux_y_, c).copy_to_host(fy[c], n);
    if (ez) s->emf_.ez_edge.copy_to_host(ez, n);
    if (cell_ez) s->emf_.cell_ez_average.copy_to_host(cell_ez, n);
    if (xface_ez) s->emf_.xface_ez.copy_to_host(xface_ez, n);
    if (yface_ez) s->emf_.yface_ez.copy_to_host(yface_ez, n);
    return 0;
  } catch (const std::exception& e) {
    static_cast<MhdSolver2D*>(h)->internal_integrator_access_ = false;
    return fail(e);
  }
}

// Pointwise kernels of the reference's numerics headers, for known-answer
// tests.  States are 8-vectors in component order.
int qref_hlld_flux_x(const double* l, const double* r, double gamma,
                     double* f) {
  using quasar::numerics::MhdState;
  const MhdState L{l[0], l[1], l[2], l[3], l[4], l[5], l[6], l[7]};
  const MhdState R{r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]};
  const auto F = quasar::numerics::hlld::hlld_flux_x(L, R, gamma);
  const double out[8] = {F.rho, F.mx, F.my, F.mz, F.energy, F.bx, F.by, F.bz};
  std::memcpy(f, out, sizeof out);
  return 0;
}

int qref_eigensystem(const double* s8, double gamma, double* l49,
                     double* r49, double* speeds7) {
  using quasar::numerics::MhdState;
  const MhdState s{s8[0], s8[1], s8[2], s8[3], s8[4], s8[5], s8[6], s8[7]};
  quasar::numerics::MhdEigensystem eig;
  eig.build(s, 0, gamma);
  for (int k = 0; k < 7; ++k) {
    const Real* row = eig.left_row(k);
    const Real* col = eig.right_col(k);
    for (int v = 0; v < 7; ++v) {
      l49[k * 7 + v] = row[v];
      r49[v * 7 + k] = col[v];
    }
    speeds7[k] = eig.wave_speed(k);
  }
  return 0;
}

double qref_mp5(const double* v) {
  return quasar::numerics::mp5_reconstruct(v[0], v[1], v[2], v[3], v[4]);
}

double qref_mp7(const double* v) {
  return quasar::numerics::mp7_reconstruct(v[0], v[1], v[2], v[3], v[4],
                                           v[5], v[6]);
}

// The reference's own deck initial state (build_initial_state,
// src/physics/mhd/initial_conditions.cpp, over the seed kernels of
// mhd_initial_conditions.hip).  kind: 0 brio_wu, 1 alfven_wave, 2
// orszag_tang, 3 blast, 4 rotor, 5 confined_blob.  par[40] in this order:
// interface, left[8], right[8] (rho, p, vx, vy, vz, bx, by, bz), rho,
// pressure, b0, total_b0, amplitude, wavenumber, magnetic_velocity_scale,
// b_uniform[3], center[2], r_in, r0, r1, rho_in, rho_out, p_in, p_out,
// p_core, p_ambient, rho_ambient, u0, blob_half, magnetic_scale.
// out8: the 8 padded components.
int qref_initial_state(int kind, int nx, int ny, double lx, double ly, double ox, double oy,
                       int ng, double gamma, int order, const double* par,
                       double* const* out8) {
  try {
    quasar::mhd::MhdInitialConditionSpec s;
    s.kind = static_cast<quasar::mhd::MhdInitialConditionKind>(kind);
    s.grid = quasar::Grid2D{nx, ny, lx, ly, ox, oy, ng};
    s.gamma = gamma;
    s.cylindrical = 0;
    s.scheme_order = order;
    int q = 0;
    s.interface = par[q++];
    for (int c = 0; c < 8; ++c) s.left[c] = par[q++];
    for (int c = 0; c < 8; ++c) s.right[c] = par[q++];
    s.rho = par[q++];
    s.pressure = par[q++];
    s.b0 = par[q++];
    s.total_b0 = par[q++];
    s.amplitude = par[q++];
    s.wavenumber = static_cast<std::int64_t>(par[q++]);
    s.magnetic_velocity_scale = par[q++];
    for (int c = 0; c < 3; ++c) s.b_uniform[c] = par[q++];
    for (int c = 0; c < 2; ++c) s.center[c] = par[q++];
    s.r_in = par[q++];
    s.r0 = par[q++];
    s.r1 = par[q++];
    s.rho_in = par[q++];
    s.rho_out = par[q++];
    s.p_in = par[q++];
    s.p_out = par[q++];
    s.p_core = par[q++];
    s.p_ambient = par[q++];
    s.rho_ambient = par[q++];
    s.u0 = par[q++];
    s.blob_half = par[q++];
    s.magnetic_scale = par[q++];
    MhdField2D<Real> out{s.grid};
    quasar::mhd::build_initial_state(s, out, nullptr);
    for (int c = 0; c < 8; ++c) comp(out, c).copy_to_host(out8[c], s.grid.storage_size());
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

}  // extern "C"
