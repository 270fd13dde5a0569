// ORACLE (test infrastructure, never shipped or called by the product):
// CPU restatement of the reference's 2-D ideal-MHD step, kernel by kernel, in
// plain binary64.  It checks the CUDA product in tests/, is the "port" CPU
// baseline of bench.py, and (instantiated with the Counted scalar) yields the
// algorithmic FLOP count used by the roofline.  It is pinned against the
// reference's own code built for the CPU (oracle/_ref) by
// tests/test_oracle_vs_reference.py.
//
// Layout: eight padded SoA arrays, index (i+g) + (nx+2g)*(j+g)
// (core/grid.hpp:158-161); bx_face(i,j) is the x-low face of cell (i,j),
// by_face(i,j) the y-low face (mhd_ct.hip:1-9).
#include "oracle_count.hpp"
#include "oracle_numerics.hpp"

#include <algorithm>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace qoracle {

struct Grid {
  int nx, ny, ng;
  double lx, ly;
  double dx() const { return lx / nx; }
  double dy() const { return ly / ny; }
  int pitch() const { return nx + 2 * ng; }
  int height() const { return ny + 2 * ng; }
  size_t size() const { return size_t(pitch()) * size_t(height()); }
  size_t idx(int i, int j) const {
    return size_t(i + ng) + size_t(pitch()) * size_t(j + ng);
  }
};

enum { RHO, MX, MY, MZ, EN, BX, BY, BZ };

struct Field {
  std::vector<double> c[8];
  void init(size_t n) {
    for (auto& v : c) v.assign(n, 0.0);
  }
};

struct Iface {
  std::vector<double> L[8], R[8];
  void init(size_t n) {
    for (int k = 0; k < 8; ++k) {
      L[k].assign(n, 0.0);
      R[k].assign(n, 0.0);
    }
  }
};

struct Config {
  int order;    // 2, 5 or 7 (1 = low-order retry operator)
  double gamma, cfl;
  int bc[4];    // x_lo, x_hi, y_lo, y_hi: 0 periodic, 1 outflow, 2 wall
};

template <class R>
class Solver {
 public:
  // The counting scalar keeps a per-thread counter, so it runs serially.
  static constexpr bool kPar = std::is_same_v<R, double>;
  Grid g;
  Config cfg;
  Field rk[3], step_backup, request_backup, residual, flux_x, flux_y;
  Iface ifx, ify;
  std::vector<double> cell_ez, xface_ez, yface_ez, ez;
  std::vector<int> xnj, ynj;
  bool solver_owned = false;
  int low_order = 0;  // positivity_reconstruction_order_
  bool control_active = false;
  bool anchor_available = false;
  int last_substeps = 0;

  Solver(int nx, int ny, double lx, double ly, Config c) : cfg(c) {
    const int ng = c.order == 7 ? 4 : c.order == 5 ? 3 : 2;
    g = Grid{nx, ny, ng, lx, ly};
    const size_t n = g.size();
    for (auto& f : rk) f.init(n);
    step_backup.init(n);
    request_backup.init(n);
    residual.init(n);
    flux_x.init(n);
    flux_y.init(n);
    ifx.init(n);
    ify.init(n);
    cell_ez.assign(n, 0.0);
    xface_ez.assign(n, 0.0);
    yface_ez.assign(n, 0.0);
    ez.assign(n, 0.0);
    xnj.assign(n, 0);
    ynj.assign(n, 0);
  }

  int order_now() const { return low_order > 0 ? low_order : cfg.order; }

  // ---- FLOP attribution (counting instance only) --------------------------
  // Phases: 0 collocation, 1 reconstruction, 2 face flux, 3 cell EMF,
  // 4 corner EMF, 5 update (flux difference, curl, combine), 6 CFL rates,
  // 7 admissibility, 8 work the reference repeats (not algorithmic).
  std::uint64_t phase_flops[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  bool colloc_free = false;  // per-load collocation is charged once per cell instead
  void charge(int p) {
    if constexpr (!kPar) {
      phase_flops[p] += flop_counter();
      flop_counter() = 0;
    }
  }
  void charge_collocation(const Field& u) {
    if constexpr (!kPar) {
      if (!colloc_free) return;
      charge(8);
      colloc_free = false;
      for (int j = -g.ng; j < g.ny + g.ng; ++j)
        for (int i = -g.ng; i < g.nx + g.ng; ++i) {
          (void)face_to_cell(u.c[BX], 0, i, j, 0);
          (void)face_to_cell(u.c[BY], 1, j, i, 0);
        }
      colloc_free = true;
      charge(0);
    }
  }

  // ---- staggered-B collocation: mhd_staggering.hpp:42-50, 77-236 -------
  static int colloc_width(int extent, int ng) {
    const int req = ng >= 4 ? 8 : ng >= 3 ? 6 : ng >= 2 ? 4 : 2;
    if (req >= 8 && extent >= 8) return 8;
    if (req >= 6 && extent >= 6) return 6;
    if (req >= 4 && extent >= 4) return 4;
    return extent >= 2 ? 2 : 1;
  }
  static double bary(int width, int k) {
    static const int w8[8] = {1, -7, 21, -35, 35, -21, 7, -1};
    static const int w6[6] = {1, -5, 10, -10, 5, -1};
    static const int w4[4] = {1, -3, 3, -1};
    if (width == 8) return w8[k];
    if (width == 6) return w6[k];
    if (width == 4) return w4[k];
    return k == 0 ? 1.0 : -1.0;
  }
  double axis_sample(const std::vector<double>& f, int axis, int q, int fixed) const {
    return axis == 0 ? f[g.idx(q, fixed)] : f[g.idx(fixed, q)];
  }
  R face_to_cell(const std::vector<double>& f, int axis, int cell, int fixed,
                 int coll) const {
    if constexpr (!kPar) {
      if (colloc_free) {
        const std::uint64_t saved = flop_counter();
        auto* self = const_cast<Solver*>(this);
        self->colloc_free = false;
        const R r = face_to_cell(f, axis, cell, fixed, coll);
        self->colloc_free = true;
        flop_counter() = saved;
        return r;
      }
    }
    const int n = axis == 0 ? g.nx : g.ny;
    const int lo = -g.ng, hi = n + g.ng - 1;
    if (coll == 1) {  // mhd_staggering.hpp:243-254
      const R lf = R(axis_sample(f, axis, cell, fixed));
      if (cell >= hi) return lf;
      return (lf + R(axis_sample(f, axis, cell + 1, fixed))) / R(2);
    }
    const int width = colloc_width(n + 2 * g.ng, g.ng);
    if (width == 1) return R(axis_sample(f, axis, cell, fixed));
    const int cs = cell - (width / 2 - 1);
    if (cs >= lo && cs + width - 1 <= hi) {
      static const int c8[8] = {-191, 1879, -9531, 68323, 68323, -9531, 1879, -191};
      static const int c6[6] = {11, -93, 802, 802, -93, 11};
      static const int c4[4] = {-1, 13, 13, -1};
      const int* c = width == 8 ? c8 : width == 6 ? c6 : width == 4 ? c4 : nullptr;
      const double den = width == 8 ? 120960.0 : width == 6 ? 1440.0 : width == 4 ? 24.0 : 2.0;
      double w[8];
      R x[8];
      for (int k = 0; k < width; ++k) {
        w[k] = c ? double(c[k]) : 1.0;
        x[k] = R(axis_sample(f, axis, cs + k, fixed));
      }
      return exact_dot(w, x, width) / R(den);
    }
    // One-sided outer-ghost closure: 4-point Gauss integral of the
    // barycentric interpolant (mhd_staggering.hpp:113-173).
    int start = cs;
    if (start < lo) start = lo;
    if (start + width - 1 > hi) start = hi - width + 1;
    static const double xq[4] = {0.0694318442029737124, 0.3300094782075718676,
                                 0.6699905217924281324, 0.9305681557970262876};
    static const double wq[4] = {0.1739274225687269287, 0.3260725774312730713,
                                 0.3260725774312730713, 0.1739274225687269287};
    const int rel = cell - start;
    R terms[32];
    int nt = 0;
    for (int q = 0; q < 4; ++q) {
      const R x = R(double(rel)) + R(xq[q]);
      R dt[8];
      for (int k = 0; k < width; ++k) dt[k] = R(bary(width, k)) / (x - R(double(k)));
      const R den = crsum(dt, width);
      for (int k = 0; k < width; ++k) {
        const R wb = R(wq[q]) * R(bary(width, k));
        terms[nt++] = ((wb * R(axis_sample(f, axis, start + k, fixed))) / (x - R(double(k)))) / den;
      }
    }
    return crsum(terms, nt);
  }
  // mhd_staggering.hpp:321-338
  State<R> load(const Field& u, int i, int j, int coll = 0) const {
    const size_t k = g.idx(i, j);
    State<R> s;
    s.rho = R(u.c[RHO][k]);
    s.mx = R(u.c[MX][k]);
    s.my = R(u.c[MY][k]);
    s.mz = R(u.c[MZ][k]);
    s.energy = R(u.c[EN][k]);
    s.bx = face_to_cell(u.c[BX], 0, i, j, coll);
    s.by = face_to_cell(u.c[BY], 1, j, i, coll);
    s.bz = R(u.c[BZ][k]);
    return s;
  }

  // ---- ghost fill: mhd_boundary_hip.hip:66-218, solver order :627-649 ----
  void ghost_idx(int n, int layer, bool lo, int mode, int& gi, int& si) const {
    gi = lo ? -layer : n - 1 + layer;
    if (mode == 0) si = lo ? n - layer : layer - 1;
    else if (mode == 1) si = lo ? 0 : n - 1;
    else si = lo ? layer - 1 : n - layer;
  }
  void fill_ghosts(Field& u) const {
    for (int side = 0; side < 4; ++side) {
      const int mode = cfg.bc[side];
      const bool xs = side < 2, lo = side == 0 || side == 2;
      const double sn = mode == 2 ? -1.0 : 1.0;
      const int n = xs ? g.nx : g.ny;
      const int lines = (xs ? g.ny : g.nx) + 2 * g.ng;
      // fluid
      for (int layer = 1; layer <= g.ng; ++layer)
        for (int l = 0; l < lines; ++l) {
          const int line = l - g.ng;
          int gi, si;
          ghost_idx(n, layer, lo, mode, gi, si);
          const size_t kd = xs ? g.idx(gi, line) : g.idx(line, gi);
          const size_t ks = xs ? g.idx(si, line) : g.idx(line, si);
          for (int c : {RHO, MX, MY, MZ, EN}) {
            const bool normal = (xs && c == MX) || (!xs && c == MY);
            u.c[c][kd] = (normal ? sn : 1.0) * u.c[c][ks];
          }
        }
      // field
      for (int layer = 1; layer <= g.ng; ++layer)
        for (int l = 0; l < lines; ++l) {
          const int line = l - g.ng;
          int gi, si;
          ghost_idx(n, layer, lo, mode, gi, si);
          std::vector<double>& bn = xs ? u.c[BX] : u.c[BY];
          std::vector<double>& bt = xs ? u.c[BY] : u.c[BX];
          auto at = [&](int a, int ln) { return xs ? g.idx(a, ln) : g.idx(ln, a); };
          bt[at(gi, line)] = bt[at(si, line)];
          u.c[BZ][at(gi, line)] = u.c[BZ][at(si, line)];
          if (mode == 2) {
            if (lo) {
              bn[at(0, line)] = 0.0;
              bn[at(-layer, line)] = -bn[at(layer, line)];
            } else if (layer == 1) {
              bn[at(n, line)] = 0.0;
            } else {
              bn[at(n + layer - 1, line)] = -bn[at(n - (layer - 1), line)];
            }
          } else if (mode == 1 && !lo) {
            if (layer > 1) bn[at(n - 1 + layer, line)] = bn[at(n, line)];
          } else {
            bn[at(gi, line)] = sn * bn[at(si, line)];
          }
        }
    }
  }

  // ---- reconstruction: mhd_reconstruct.hip:150-670 -----------------------
  static State<R> rotate_xy(const State<R>& v, int dir) {
    if (dir == 0) return v;
    State<R> r = v;
    r.mx = v.my;
    r.my = v.mx;
    r.bx = v.by;
    r.by = v.bx;
    return r;
  }
  static void set_normal_b(State<R>& s, int dir, R v) {
    R& bn = dir == 0 ? s.bx : s.by;
    s.energy = crsum3(s.energy * R(1), v * (R(0.5) * v), bn * (-R(0.5) * bn));
    bn = v;
  }
  static bool admissible(const State<R>& s, R gamma) {
    if (!(qfinite(s.rho) && s.rho > R(0))) return false;
    const Prim<R> w = to_primitive(s, gamma);
    if (!(qfinite(w.vx) && qfinite(w.vy) && qfinite(w.vz) && qfinite(w.p) && w.p > R(0)))
      return false;
    return qfinite(s.mx) && qfinite(s.my) && qfinite(s.mz) && qfinite(s.energy) &&
           qfinite(s.bx) && qfinite(s.by) && qfinite(s.bz);
  }
  static int slope_drop(int c, int n, int lo, int hi) {
    if (lo != 0 && lo != 4 && c <= 0) return -1;
    if (hi != 0 && hi != 4 && c >= n - 1) return +1;
    return 0;
  }
  static R limited_slope(R back, R fwd, int drop) {
    if (drop < 0) return fwd;
    if (drop > 0) return back;
    return minmod2(back, fwd);
  }
  static Prim<R> muscl_face(const Prim<R>& m, const Prim<R>& c, const Prim<R>& p,
                            R sign, int drop) {
    const R h = R(0.5) * sign;
    Prim<R> f;
    f.rho = c.rho + h * limited_slope(c.rho - m.rho, p.rho - c.rho, drop);
    f.vx = c.vx + h * limited_slope(c.vx - m.vx, p.vx - c.vx, drop);
    f.vy = c.vy + h * limited_slope(c.vy - m.vy, p.vy - c.vy, drop);
    f.vz = c.vz + h * limited_slope(c.vz - m.vz, p.vz - c.vz, drop);
    f.p = c.p + h * limited_slope(c.p - m.p, p.p - c.p, drop);
    f.bx = c.bx + h * limited_slope(c.bx - m.bx, p.bx - c.bx, drop);
    f.by = c.by + h * limited_slope(c.by - m.by, p.by - c.by, drop);
    f.bz = c.bz + h * limited_slope(c.bz - m.bz, p.bz - c.bz, drop);
    return f;
  }
  void muscl_pair(const Field& u, int dir, int i, int j, State<R>& ul, State<R>& ur) const {
    const R gamma = R(cfg.gamma);
    const int di = dir == 0, dj = dir == 1;
    const Prim<R> a = to_primitive(load(u, i - 2 * di, j - 2 * dj), gamma);
    const Prim<R> b = to_primitive(load(u, i - di, j - dj), gamma);
    const Prim<R> c = to_primitive(load(u, i, j), gamma);
    const Prim<R> d = to_primitive(load(u, i + di, j + dj), gamma);
    const int n = dir == 0 ? g.nx : g.ny;
    const int lo = dir == 0 ? cfg.bc[0] : cfg.bc[2];
    const int hi = dir == 0 ? cfg.bc[1] : cfg.bc[3];
    const int dm = slope_drop(dir == 0 ? i - 1 : j - 1, n, lo, hi);
    const int dp = slope_drop(dir == 0 ? i : j, n, lo, hi);
    ul = to_conserved(muscl_face(a, b, c, R(1), dm), gamma);
    ur = to_conserved(muscl_face(b, c, d, R(-1), dp), gamma);
  }
  // Characteristic MP5/MP7 pair at face (i,j): mhd_reconstruct.hip:217-349,
  // 525-616.  `fired` (optional) reports whether the MP limiter changed any
  // wave of either state.
  void mp_pair(const Field& u, int dir, int i, int j, int order, State<R>& ul,
               State<R>& ur, bool* fired = nullptr) const {
    const R gamma = R(cfg.gamma);
    const int di = dir == 0, dj = dir == 1;
    const State<R> cL = load(u, i - di, j - dj), cR = load(u, i, j);
    State<R> ref;
    ref.rho = R(0.5) * cL.rho + R(0.5) * cR.rho;
    ref.mx = R(0.5) * cL.mx + R(0.5) * cR.mx;
    ref.my = R(0.5) * cL.my + R(0.5) * cR.my;
    ref.mz = R(0.5) * cL.mz + R(0.5) * cR.mz;
    ref.energy = R(0.5) * cL.energy + R(0.5) * cR.energy;
    ref.bx = R(0.5) * cL.bx + R(0.5) * cR.bx;
    ref.by = R(0.5) * cL.by + R(0.5) * cR.by;
    ref.bz = R(0.5) * cL.bz + R(0.5) * cR.bz;
    const State<R> cref = rotate_xy(ref, dir);
    Eigen<R> eig;
    build_eigensystem(cref, gamma, eig);
    const int half = order == 5 ? 2 : 3, width = 2 * half + 1;
    R chars[8][7];
    for (int s = 0; s < 2 * half + 2; ++s) {
      const int off = -1 - half + s;
      const State<R> d = rotate_xy(load(u, i + off * di, j + off * dj), dir);
      const R u7[7] = {d.rho - cref.rho, d.mx - cref.mx, d.my - cref.my, d.mz - cref.mz,
                       d.energy - cref.energy, d.by - cref.by, d.bz - cref.bz};
      for (int k = 0; k < 7; ++k) {
        R acc = R(0);
        for (int v = 0; v < 7; ++v) acc = acc + eig.L[k * 7 + v] * u7[v];
        chars[s][k] = acc;
      }
    }
    bool any = false;
    auto recon = [&](int base, bool right) {
      R wf[7];
      for (int k = 0; k < 7; ++k) {
        R sc[7];
        for (int s = 0; s < width; ++s) sc[s] = chars[base + (right ? width - 1 - s : s)][k];
        bool f = false;
        wf[k] = mp_reconstruct(sc, width, &f);
        any = any || f;
      }
      R d7[7];
      for (int v = 0; v < 7; ++v) d7[v] = R(0);
      for (int k = 0; k < 7; ++k)
        for (int v = 0; v < 7; ++v) d7[v] = d7[v] + eig.Rm[v * 7 + k] * wf[k];
      State<R> s;
      s.rho = cref.rho + d7[0];
      s.mx = cref.mx + d7[1];
      s.my = cref.my + d7[2];
      s.mz = cref.mz + d7[3];
      s.energy = cref.energy + d7[4];
      s.bx = cref.bx + R(0);
      s.by = cref.by + d7[5];
      s.bz = cref.bz + d7[6];
      return rotate_xy(s, dir);
    };
    ul = recon(0, false);
    ur = recon(1, true);
    if (fired) *fired = any;
  }
  void reconstruct_face(const Field& u, int dir, int i, int j, int order,
                        State<R>& ul, State<R>& ur) const {
    const R gamma = R(cfg.gamma);
    const int di = dir == 0, dj = dir == 1;
    if (order <= 1) {
      ul = load(u, i - di, j - dj, 1);
      ur = load(u, i, j, 1);
    } else if (order != 2) {
      mp_pair(u, dir, i, j, order, ul, ur);
      if (!admissible(ul, gamma) || !admissible(ur, gamma)) muscl_pair(u, dir, i, j, ul, ur);
    } else {
      muscl_pair(u, dir, i, j, ul, ur);
    }
    const R bn = R((dir == 0 ? u.c[BX] : u.c[BY])[g.idx(i, j)]);
    set_normal_b(ul, dir, bn);
    set_normal_b(ur, dir, bn);
    if (!admissible(ul, gamma) || !admissible(ur, gamma)) {
      const int coll = order <= 1 ? 1 : 0;
      ul = load(u, i - di, j - dj, coll);
      ur = load(u, i, j, coll);
      set_normal_b(ul, dir, bn);
      set_normal_b(ur, dir, bn);
    }
    if (!admissible(ul, gamma) || !admissible(ur, gamma)) {
      const R nan = R(std::numeric_limits<double>::quiet_NaN());
      ul = State<R>{nan, nan, nan, nan, nan, nan, nan, nan};
      ur = ul;
    }
  }
  void reconstruct(const Field& u, int dir, int order, Iface& out) const {
    const int i0 = dir == 0 ? 0 : -g.ng, i1 = dir == 0 ? g.nx : g.nx + g.ng - 1;
    const int j0 = dir == 1 ? 0 : -g.ng, j1 = dir == 1 ? g.ny : g.ny + g.ng - 1;
#pragma omp parallel for collapse(2) schedule(dynamic, 16) if (kPar)
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) {
        State<R> ul, ur;
        reconstruct_face(u, dir, i, j, order, ul, ur);
        const size_t k = g.idx(i, j);
        const R l8[8] = {ul.rho, ul.mx, ul.my, ul.mz, ul.energy, ul.bx, ul.by, ul.bz};
        const R r8[8] = {ur.rho, ur.mx, ur.my, ur.mz, ur.energy, ur.bx, ur.by, ur.bz};
        for (int c = 0; c < 8; ++c) {
          out.L[c][k] = qval(l8[c]);
          out.R[c][k] = qval(r8[c]);
        }
      }
  }

  // ---- face quadrature + HLLD: mhd_face_quadrature.hpp:114-273 ----------
  State<R> iface_state(const Iface& v, size_t k, bool left) const {
    const auto& a = left ? v.L : v.R;
    return State<R>{R(a[0][k]), R(a[1][k]), R(a[2][k]), R(a[3][k]),
                    R(a[4][k]), R(a[5][k]), R(a[6][k]), R(a[7][k])};
  }
  static bool point_admissible(const State<R>& s, R gamma) {
    if (!(qfinite(s.rho) && s.rho > R(0) && qfinite(s.mx) && qfinite(s.my) && qfinite(s.mz) &&
          qfinite(s.energy) && qfinite(s.bx) && qfinite(s.by) && qfinite(s.bz)))
      return false;
    const R p = pressure(s, gamma);
    return qfinite(p) && p > R(0);
  }
  State<R> point_state(const Iface& v, int dir, int i, int j, int order, int node,
                       bool left) const {
    const int half = order >= 7 ? 3 : 2, taps = 2 * half + 1;
    const double* w = order >= 7 ? kPoint7[node] : kPoint5[node];
    const auto& a = left ? v.L : v.R;
    R out[8];
    for (int c = 0; c < 8; ++c) {
      R s[7];
      for (int k = 0; k < taps; ++k) {
        const int off = k - half;
        s[k] = R(a[c][dir == 0 ? g.idx(i, j + off) : g.idx(i + off, j)]);
      }
      out[c] = weighted_value(w, s, taps);
    }
    return State<R>{out[0], out[1], out[2], out[3], out[4], out[5], out[6], out[7]};
  }
  static Flux<R> riemann(const State<R>& l, const State<R>& r, int dir, bool hll_only,
                         R gamma) {
    const State<R> lr = rotate_xy(l, dir), rr = rotate_xy(r, dir);
    Flux<R> f = hll_only ? lax_friedrichs_flux_x(lr, rr, gamma) : hlld_flux_x(lr, rr, gamma);
    if (dir == 1) {
      std::swap(f.mx, f.my);
      std::swap(f.bx, f.by);
    }
    return f;
  }
  Flux<R> face_flux(const Iface& v, int dir, int i, int j, int order, bool hll_only) const {
    const R gamma = R(cfg.gamma);
    const size_t k = g.idx(i, j);
    const State<R> bl = iface_state(v, k, true), br = iface_state(v, k, false);
    if (order != 5 && order != 7) return riemann(bl, br, dir, hll_only, gamma);
    const int count = order == 5 ? 3 : 4;
    Flux<R> f[4];
    for (int q = 0; q < count; ++q) {
      const State<R> l = point_state(v, dir, i, j, order, q, true);
      const State<R> r = point_state(v, dir, i, j, order, q, false);
      if (!point_admissible(l, gamma) || !point_admissible(r, gamma))
        return riemann(bl, br, dir, hll_only, gamma);
      f[q] = riemann(l, r, dir, hll_only, gamma);
    }
    const double* w = count == 3 ? kGauss3 : kGauss4;
    auto avg = [&](R Flux<R>::*m) {
      R s[4];
      for (int q = 0; q < count; ++q) s[q] = f[q].*m;
      return weighted_value(w, s, count);
    };
    return Flux<R>{avg(&Flux<R>::rho), avg(&Flux<R>::mx), avg(&Flux<R>::my),
                   avg(&Flux<R>::mz), avg(&Flux<R>::energy), avg(&Flux<R>::bx),
                   avg(&Flux<R>::by), avg(&Flux<R>::bz)};
  }
  // mhd_riemann.hip:53-136
  void face_fluxes(const Iface& v, int dir, int order, Field& out) const {
    const bool hll_only = order <= 1;
#pragma omp parallel for collapse(2) schedule(dynamic, 16) if (kPar)
    for (int j = 0; j <= g.ny; ++j)
      for (int i = 0; i <= g.nx; ++i) {
        int si = i, sj = j;
        if (dir == 0 && i == g.nx && cfg.bc[0] == 0 && cfg.bc[1] == 0) si = 0;
        if (dir == 1 && j == g.ny && cfg.bc[2] == 0 && cfg.bc[3] == 0) sj = 0;
        const Flux<R> f = face_flux(v, dir, si, sj, order, hll_only);
        const R f8[8] = {f.rho, f.mx, f.my, f.mz, f.energy, f.bx, f.by, f.bz};
        const size_t k = g.idx(i, j);
        for (int c = 0; c < 8; ++c) out.c[c][k] = qval(f8[c]);
      }
  }
  // mhd_update.hip:21-105 (Cartesian)
  void flux_difference(const Field& f, int dir, Field& dudt) const {
    const double h = dir == 0 ? g.dx() : g.dy();
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        const size_t k = g.idx(i, j);
        const size_t kp = dir == 0 ? g.idx(i + 1, j) : g.idx(i, j + 1);
        for (int c = 0; c < 8; ++c) {
          const R d = R(f.c[c][kp]) / R(h) + (-R(f.c[c][k])) / R(h);
          dudt.c[c][k] = qval(R(dudt.c[c][k]) + (-d));
        }
      }
  }

  // ---- constrained transport: mhd_ct.hip:126-931 -------------------------
  static int face_index(int q, int n, int lo, int hi) {
    if (lo == 0 && hi == 0) {
      int w = q % n;
      if (w < 0) w += n;
      return w;
    }
    if (q < 0) return lo == 4 ? q : 0;
    if (q > n) return hi == 4 ? q : n;
    return q;
  }
  bool in_pad(int i, int j) const {
    return i >= -g.ng && i < g.nx + g.ng && j >= -g.ng && j < g.ny + g.ng;
  }
  bool face_no_jump(const Iface& v, int dir, int i, int j, int order) const {
    const int rh = order >= 7 ? 3 : order >= 5 ? 2 : 0;
    for (int off = -rh; off <= rh; ++off) {
      const int si = dir == 0 ? i : i + off, sj = dir == 0 ? j + off : j;
      const int mi = face_index(si, g.nx, cfg.bc[0], cfg.bc[1]);
      const int mj = face_index(sj, g.ny, cfg.bc[2], cfg.bc[3]);
      if (!in_pad(mi, mj)) return false;
      const size_t k = g.idx(mi, mj);
      for (int c = 0; c < 8; ++c)
        if (!(v.L[c][k] == v.R[c][k])) return false;
    }
    return true;
  }
  static R physical_ez(const State<R>& s) {
    const R vx = s.mx / s.rho, vy = s.my / s.rho;
    return vy * s.bx + vx * (-s.by);
  }
  R cell_average_ez(const Field& u, int i, int j, int order) const {
    const R gamma = R(cfg.gamma);
    const int coll = order <= 1 ? 1 : 0;
    const R fallback = physical_ez(load(u, i, j, coll));
    if (order != 5 && order != 7) return fallback;
    const int half = order == 5 ? 2 : 3, taps = 2 * half + 1, count = order == 5 ? 3 : 4;
    if (i - half < -g.ng || i + half > g.nx + g.ng - 1 || j - half < -g.ng ||
        j + half > g.ny + g.ng - 1)
      return fallback;
    R bxb[7][7], byb[7][7];
    for (int a = 0; a < taps; ++a)
      for (int b = 0; b < taps; ++b) {
        bxb[a][b] = face_to_cell(u.c[BX], 0, i + a - half, j + b - half, 0);
        byb[a][b] = face_to_cell(u.c[BY], 1, j + b - half, i + a - half, 0);
      }
    R point[4][4];
    for (int qx = 0; qx < count; ++qx) {
      const double* wx = order == 5 ? kPoint5[qx] : kPoint7[qx];
      R rows[8][7];
      for (int k = 0; k < taps; ++k) {
        const int oy = k - half;
        R s[8][7];
        for (int ox = -half; ox <= half; ++ox) {
          const size_t kk = g.idx(i + ox, j + oy);
          s[0][ox + half] = R(u.c[RHO][kk]);
          s[1][ox + half] = R(u.c[MX][kk]);
          s[2][ox + half] = R(u.c[MY][kk]);
          s[3][ox + half] = R(u.c[MZ][kk]);
          s[4][ox + half] = R(u.c[EN][kk]);
          s[5][ox + half] = bxb[ox + half][oy + half];
          s[6][ox + half] = byb[ox + half][oy + half];
          s[7][ox + half] = R(u.c[BZ][kk]);
        }
        for (int c = 0; c < 8; ++c) rows[c][k] = weighted_value(wx, s[c], taps);
      }
      for (int qy = 0; qy < count; ++qy) {
        const double* wy = order == 5 ? kPoint5[qy] : kPoint7[qy];
        R c8[8];
        for (int c = 0; c < 8; ++c) c8[c] = weighted_value(wy, rows[c], taps);
        const State<R> st{c8[0], c8[1], c8[2], c8[3], c8[4], c8[5], c8[6], c8[7]};
        if (!point_admissible(st, gamma)) return fallback;
        point[qy][qx] = physical_ez(st);
      }
    }
    const double* w = count == 3 ? kGauss3 : kGauss4;
    R row[4];
    for (int qy = 0; qy < count; ++qy) row[qy] = weighted_value(w, point[qy], count);
    return weighted_value(w, row, count);
  }
  static R edge_interp(const R* e, int order) {
    // scaled_face_average{,_to_edge5,_to_edge7}: mhd_ct.hip:50-97
    const int n = order >= 7 ? 8 : order >= 5 ? 6 : 2;
    bool same = true;
    for (int k = 1; k < n; ++k) same = same && (e[k] == e[0]);
    if (same) return e[0];
    if (n == 2) return (e[0] + e[1]) / R(2);
    static const double c6[6] = {1, -8, 37, 37, -8, 1};
    static const double c8[8] = {-3, 29, -139, 533, 533, -139, 29, -3};
    const double* c = n == 6 ? c6 : c8;
    return exact_dot(c, e, n) / R(n == 6 ? 60.0 : 840.0);
  }
  double tab(const std::vector<double>& t, int i, int j) const {
    return t[g.idx(face_index(i, g.nx, cfg.bc[0], cfg.bc[1]),
                   face_index(j, g.ny, cfg.bc[2], cfg.bc[3]))];
  }
  bool corner_no_jump(int dir, int i, int j, int order, const std::vector<int>& nj) const {
    const int lo = order >= 7 ? -4 : order >= 5 ? -3 : -1;
    const int hi = order >= 7 ? 3 : order >= 5 ? 2 : 0;
    for (int off = lo; off <= hi; ++off) {
      const int si = dir == 0 ? i : i + off, sj = dir == 0 ? j + off : j;
      const int ii = face_index(si, g.nx, cfg.bc[0], cfg.bc[1]);
      const int jj = face_index(sj, g.ny, cfg.bc[2], cfg.bc[3]);
      if (!in_pad(ii, jj) || nj[g.idx(ii, jj)] == 0) return false;
    }
    return true;
  }
  bool cell_const_along(int i, int j, int order, int axis) const {
    const int lo = order >= 7 ? -4 : order >= 5 ? -3 : -1;
    const int hi = order >= 7 ? 3 : order >= 5 ? 2 : 0;
    for (int va = lo; va <= hi; ++va) {
      const double ref = axis == 0 ? tab(cell_ez, i + lo, j + va) : tab(cell_ez, i + va, j + lo);
      for (int inv = lo + 1; inv <= hi; ++inv) {
        const double c = axis == 0 ? tab(cell_ez, i + inv, j + va) : tab(cell_ez, i + va, j + inv);
        if (c != ref) return false;
      }
    }
    return true;
  }
  void ct_emf(const Field& u, int order) {
    const bool hll_only = order <= 1;
    const bool phx = cfg.bc[1] != 0 && cfg.bc[1] != 4;
    const bool phy = cfg.bc[3] != 0 && cfg.bc[3] != 4;
#pragma omp parallel for collapse(2) schedule(dynamic, 16) if (kPar)
    for (int j = 0; j <= g.ny; ++j)
      for (int i = 0; i <= g.nx; ++i) {
        const size_t k = g.idx(i, j);
        if (!((i == g.nx && !phx) || (j == g.ny && !phy)))
          cell_ez[k] = qval(cell_average_ez(u, i, j, order));
      }
    charge(3);
    // Directional face EMFs: the reference re-solves every face problem here
    // (mhd_ct.hip:330-359); the fluxes above already hold the same values.
#pragma omp parallel for collapse(2) schedule(dynamic, 16) if (kPar)
    for (int j = 0; j <= g.ny; ++j)
      for (int i = 0; i <= g.nx; ++i) {
        const size_t k = g.idx(i, j);
        if (j < g.ny || (j == g.ny && phy)) {
          xface_ez[k] = qval(-face_flux(ifx, 0, i, j, order, hll_only).by);
          xnj[k] = face_no_jump(ifx, 0, i, j, order) ? 1 : 0;
        }
        if (i < g.nx || (i == g.nx && phx)) {
          yface_ez[k] = qval(face_flux(ify, 1, i, j, order, hll_only).bx);
          ynj[k] = face_no_jump(ify, 1, i, j, order) ? 1 : 0;
        }
      }
    charge(8);
#pragma omp parallel for collapse(2) schedule(static) if (kPar)
    for (int j = 0; j <= g.ny; ++j)
      for (int i = 0; i <= g.nx; ++i) {
        const size_t k = g.idx(i, j);
        const bool conducting = (i == 0 && cfg.bc[0] == 2) || (i == g.nx && cfg.bc[1] == 2) ||
                                (j == 0 && cfg.bc[2] == 2) || (j == g.ny && cfg.bc[3] == 2);
        if (conducting) {
          ez[k] = 0.0;
          continue;
        }
        const int lo = order >= 7 ? -4 : order >= 5 ? -3 : -1;
        const int n = order >= 7 ? 8 : order >= 5 ? 6 : 2;
        R ex_s[8], ey_s[8], line[8];
        for (int q = 0; q < n; ++q) {
          ex_s[q] = R(tab(xface_ez, i, j + lo + q));
          ey_s[q] = R(tab(yface_ez, i + lo + q, j));
        }
        const R ex = edge_interp(ex_s, order), ey = edge_interp(ey_s, order);
        for (int q = 0; q < n; ++q) {
          R c[8];
          for (int p = 0; p < n; ++p) c[p] = R(tab(cell_ez, i + lo + p, j + lo + q));
          line[q] = edge_interp(c, order);
        }
        const R centered = edge_interp(line, order);
        const bool x_only = corner_no_jump(1, i, j, order, ynj) && cell_const_along(i, j, order, 1);
        const bool y_only = corner_no_jump(0, i, j, order, xnj) && cell_const_along(i, j, order, 0);
        R e;
        if (x_only && !y_only) e = ex;
        else if (y_only && !x_only) e = ey;
        else e = crsum3(ex, ey, -centered);
        ez[k] = qval(e);
      }
    charge(4);
  }
  // mhd_ct.hip:893-931 (Cartesian)
  void curl_rate(Field& dudt) const {
    for (int j = 0; j <= g.ny; ++j)
      for (int i = 0; i <= g.nx; ++i) {
        const size_t k = g.idx(i, j);
        if (j < g.ny)
          dudt.c[BX][k] = qval(-R(ez[g.idx(i, j + 1)]) / R(g.dy()) + R(ez[k]) / R(g.dy()));
        if (i < g.nx)
          dudt.c[BY][k] = qval(R(ez[g.idx(i + 1, j)]) / R(g.dx()) + (-R(ez[k])) / R(g.dx()));
      }
  }

  // ---- residual: mhd_solver.cpp:665-826 -----------------------------------
  bool iface_cache_valid = false;
  const Field* iface_cache_src = nullptr;
  int iface_cache_order = -1;

  void compute_residual(Field& u, Field& dudt) {
    const int order = order_now();
    const bool current = iface_cache_valid && iface_cache_src == &u && iface_cache_order == order;
    fill_ghosts(u);
    if (&u == &rk[0]) {
      ensure_solenoidal();
      ensure_admissible(order <= 1 ? 1 : 0);
    }
    charge(7);
    for (auto& c : dudt.c) std::fill(c.begin(), c.end(), 0.0);
    if (!current) charge_collocation(u);
    if (!current) reconstruct(u, 0, order, ifx);
    charge(1);
    face_fluxes(ifx, 0, order, flux_x);
    charge(2);
    if (!current) reconstruct(u, 1, order, ify);
    charge(1);
    face_fluxes(ify, 1, order, flux_y);
    charge(2);
    iface_cache_valid = false;
    flux_difference(flux_x, 0, dudt);
    flux_difference(flux_y, 1, dudt);
    charge(5);
    ct_emf(u, order);
    curl_rate(dudt);
    charge(5);
  }

  // ---- SSP-RK3 combine: mhd_update.hip:113-206, mhd_solver.cpp:840-906 ---
  static R rk_sum(R a, R un, R b, R us, R c, R d) {
    const bool ua = a != R(0), ub = b != R(0), uc = c != R(0);
    if (ua) {
      if (ub) return uc ? crsum3(a * un, b * us, c * d) : a * un + b * us;
      return uc ? a * un + c * d : a * un;
    }
    if (ub) return uc ? b * us + c * d : b * us;
    return uc ? c * d : R(0);
  }
  void rk_stage(Field& out, const Field& un, const Field& us, const Field& d, double a,
                double b, double c) const {
    for (int j = 0; j <= g.ny; ++j)
      for (int i = 0; i <= g.nx; ++i) {
        const bool cell = i < g.nx && j < g.ny;
        const bool bxp = j < g.ny, byp = i < g.nx;
        const size_t k = g.idx(i, j);
        const bool copy = a == 1.0 && b == 0.0 && c == 0.0;
        for (int comp = 0; comp < 8; ++comp) {
          const bool active = comp == BX ? bxp : comp == BY ? byp : cell;
          if (!active) continue;
          out.c[comp][k] = copy ? un.c[comp][k]
                                : qval(rk_sum(R(a), R(un.c[comp][k]), R(b), R(us.c[comp][k]),
                                              R(c), R(d.c[comp][k])));
        }
      }
  }
  void copy_state(const Field& src, Field& dst) {
    rk_stage(dst, src, src, residual, 1.0, 0.0, 0.0);
    fill_ghosts(dst);
  }

  // ---- admissible fraction: mhd_reduce.hip:120-209 ----------------------
  static R convex_q(const State<R>& a, const State<R>& b, R th) {
    const R omt = R(1) - th;
    const R rho = omt * a.rho + th * b.rho;
    if (!(rho > R(0)) || !qfinite(rho)) return R(-std::numeric_limits<double>::infinity());
    const R mx = omt * a.mx + th * b.mx, my = omt * a.my + th * b.my, mz = omt * a.mz + th * b.mz;
    const R e = omt * a.energy + th * b.energy;
    const R bx = omt * a.bx + th * b.bx, by = omt * a.by + th * b.by, bz = omt * a.bz + th * b.bz;
    const R q = (e - kinetic_from_momentum(mx, my, mz, rho)) - half_squared_norm3(bx, by, bz);
    return qfinite(q) ? q : R(-std::numeric_limits<double>::infinity());
  }
  double admissible_fraction(const Field& base, const Field& cand, int coll) const {
    double theta = 1.0;
#pragma omp parallel for collapse(2) reduction(min : theta) if (kPar)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        const State<R> a = load(base, i, j, coll), b = load(cand, i, j, coll);
        const R qa = convex_q(a, b, R(0));
        double local;
        if (!(a.rho > R(0)) || !(qa > R(0)) || !qfinite(a.rho) || !qfinite(qa)) {
          local = 0.0;
        } else if (!(qfinite(b.rho) && qfinite(b.mx) && qfinite(b.my) && qfinite(b.mz) &&
                     qfinite(b.energy) && qfinite(b.bx) && qfinite(b.by) && qfinite(b.bz))) {
          local = 0.0;
        } else {
          R hi = R(1);
          if (b.rho <= R(0)) {
            const R den = a.rho - b.rho;
            hi = den > R(0) ? (a.rho - R(0)) / den : R(0);
            if (hi < R(0)) hi = R(0);
            if (hi > R(1)) hi = R(1);
          }
          if (convex_q(a, b, hi) > R(0)) {
            local = qval(hi);
          } else {
            R lo = R(0);
            for (int it = 0; it < 56; ++it) {
              const R mid = R(0.5) * (lo + hi);
              if (convex_q(a, b, mid) > R(0)) lo = mid; else hi = mid;
            }
            local = qval(lo);
          }
        }
        theta = std::min(theta, local);
      }
    return theta;
  }
  void ensure_admissible(int coll) const {
    if (!(admissible_fraction(rk[0], rk[0], coll) >= 1.0))
      throw std::invalid_argument(
          "MhdSolver2D: live state must have finite components, rho > 0, and gas "
          "pressure > 0 in every interior cell");
  }
  // Solenoidality preflight: mhd_reduce.hip:556-700, solver :1196-1222.
  static double ulp_of(double x) {
    if (!std::isfinite(x)) return std::numeric_limits<double>::infinity();
    const double m = std::fabs(x);
    if (m < std::numeric_limits<double>::min()) return std::numeric_limits<double>::denorm_min();
    int e = 0;
    (void)std::frexp(m, &e);
    return std::ldexp(0.5, e - 52);
  }
  void ensure_solenoidal() const {
    const Field& u = rk[0];
    double rmax = 0.0, smax = 0.0;
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        const double bxl = u.c[BX][g.idx(i, j)], bxh = u.c[BX][g.idx(i + 1, j)];
        const double byl = u.c[BY][g.idx(i, j)], byh = u.c[BY][g.idx(i, j + 1)];
        const double d1 = (bxh - bxl) / g.dx(), d2 = (byh - byl) / g.dy();
        const double res = d1 + d2, scale = std::fabs(d1) + std::fabs(d2);
        const double unc = (ulp_of(bxh) + ulp_of(bxl)) / g.dx() + (ulp_of(byh) + ulp_of(byl)) / g.dy();
        bool explained;
        if (solver_owned) {
          explained = std::fabs(res) <= 1024.0 * unc;
        } else {
          explained = d1 != 0.0 && d2 != 0.0 && std::signbit(d1) != std::signbit(d2) &&
                      std::fabs(res) <= 0.5 * scale && std::fabs(res) <= 1024.0 * unc;
        }
        rmax = std::max(rmax, explained ? 0.0 : std::fabs(res));
        smax = std::max(smax, scale);
      }
    const double rel = rmax == 0.0 ? 0.0 : rmax / smax;
    if (!(std::isfinite(rel) && rel <= 1024.0 * kEps))
      throw std::invalid_argument(
          "MhdSolver2D: live magnetic field is not discretely divergence-free");
  }

  // ---- CFL: mhd_reduce.hip:254-501, mhd_solver.cpp:1228-1321 -------------
  struct Speed {
    R v, f;
  };
  Speed speed_parts(const State<R>& s, int dir) const {
    const R gamma = R(cfg.gamma);
    const R p = pressure(s, gamma);
    const R inf = R(std::numeric_limits<double>::infinity());
    if (!(qfinite(s.rho) && s.rho > R(0) && qfinite(s.mx) && qfinite(s.my) && qfinite(s.mz) &&
          qfinite(s.energy) && qfinite(s.bx) && qfinite(s.by) && qfinite(s.bz) && qfinite(p) &&
          p > R(0)))
      return {inf, inf};
    const R sr = qsqrt(s.rho);
    const R sound = (qsqrt(gamma) * qsqrt(p)) / sr;
    const R ax = s.bx / sr, ay = s.by / sr, az = s.bz / sr;
    const R ca = scaled_norm3(ax, ay, az);
    const R can = qabs(dir == 0 ? ax : ay);
    const R scale = qmax(sound, ca);
    R fast = R(0);
    if (scale > R(0)) {
      const R an = sound / scale, bn = ca / scale, cn = can / scale;
      const R a2 = an * an, b2 = bn * bn, sum = a2 + b2;
      R disc = sum * sum - R(4) * a2 * cn * cn;
      if (disc < R(0)) disc = R(0);
      fast = scale * qsqrt(R(0.5) * (sum + qsqrt(disc)));
    }
    const R vel = qabs(dir == 0 ? s.mx : s.my) / s.rho;
    if (!(qfinite(vel) && qfinite(fast))) return {inf, inf};
    return {vel, fast};
  }
  R iface_speed(const Speed& l, const Speed& r, int order) const {
    const R rate = order <= 1 ? qmax(l.v + l.f, r.v + r.f) : qmax(l.v, r.v) + qmax(l.f, r.f);
    return qfinite(rate) ? rate : R(std::numeric_limits<double>::infinity());
  }
  R face_rate(const Iface& v, int dir, int fi, int fj, int order, double spacing) const {
    const R gamma = R(cfg.gamma);
    if (dir == 0 && fi == g.nx && cfg.bc[0] == 0 && cfg.bc[1] == 0) fi = 0;
    if (dir == 1 && fj == g.ny && cfg.bc[2] == 0 && cfg.bc[3] == 0) fj = 0;
    const size_t k = g.idx(fi, fj);
    auto rate = [&](const State<R>& l, const State<R>& r) {
      const R sp = iface_speed(speed_parts(l, dir), speed_parts(r, dir), order);
      if (!(qfinite(sp) && sp >= R(0))) return R(std::numeric_limits<double>::infinity());
      return (sp * R(0.5)) / R(spacing);
    };
    R mx = rate(iface_state(v, k, true), iface_state(v, k, false));
    if (order != 5 && order != 7) return mx;
    const int count = order == 5 ? 3 : 4;
    for (int q = 0; q < count; ++q) {
      const State<R> l = point_state(v, dir, fi, fj, order, q, true);
      const State<R> r = point_state(v, dir, fi, fj, order, q, false);
      if (!point_admissible(l, gamma) || !point_admissible(r, gamma)) return mx;
      mx = qmax(mx, rate(l, r));
    }
    return mx;
  }
  double cfl_limit(int coll = 0) {
    fill_ghosts(rk[0]);
    ensure_solenoidal();
    ensure_admissible(coll);
    const int order = coll > 0 ? 1 : cfg.order;
    charge(7);
    charge_collocation(rk[0]);
    reconstruct(rk[0], 0, order, ifx);
    reconstruct(rk[0], 1, order, ify);
    charge(1);
    iface_cache_valid = true;
    iface_cache_src = &rk[0];
    iface_cache_order = order;
    double maxrate = 0.0;
#pragma omp parallel for collapse(2) reduction(max : maxrate) if (kPar)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        const R a = face_rate(ifx, 0, i, j, order, g.dx()) + face_rate(ifx, 0, i + 1, j, order, g.dx());
        const R b = face_rate(ify, 1, i, j, order, g.dy()) + face_rate(ify, 1, i, j + 1, order, g.dy());
        double local = qval(a + b);
        local = std::isfinite(local) ? std::max(0.0, local) : std::numeric_limits<double>::infinity();
        maxrate = std::max(maxrate, local);
      }
    charge(6);
    const double eff = order >= 5 ? std::min(cfg.cfl, 0.2) : cfg.cfl;
    if (!std::isfinite(maxrate))
      throw std::runtime_error("MhdSolver2D: non-finite state encountered in CFL reduction");
    if (!(maxrate > 0.0)) {
      const double hmin = std::min(g.dx(), g.dy()), hmax = std::max(g.dx(), g.dy());
      return eff * (hmin / (1.0 + hmin / hmax));
    }
    return qval(R(eff) / R(maxrate));
  }

  // ---- positivity controller: mhd_solver.cpp:828-1143 --------------------
  struct Retry {
    double theta;
  };
  double stage_theta(int stage) {
    Field& out = rk[stage == 2 ? 0 : stage + 1];
    double th = 1.0;
    if (control_active) {
      th = admissible_fraction(step_backup, out, low_order);
      if (stage == 2 && low_order == 0 && anchor_available)
        th = std::min(th, admissible_fraction(step_backup, out, 1));
      else if (stage == 2 && low_order == 1)
        th = std::min(th, admissible_fraction(step_backup, out, 0));
    }
    return std::isfinite(th) ? th : 0.0;
  }
  void combine_stage(int stage, double dt) {
    Field* out;
    double a, b, c;
    if (stage == 0) { out = &rk[1]; a = 1.0; b = 0.0; c = dt; }
    else if (stage == 1) { out = &rk[2]; a = 3.0 / 4.0; b = 1.0 / 4.0; c = (1.0 / 4.0) * dt; }
    else { out = &rk[0]; a = 1.0 / 3.0; b = 2.0 / 3.0; c = (2.0 / 3.0) * dt; }
    const Field& us = stage == 2 ? rk[2] : rk[1];
    charge(8);
    rk_stage(*out, rk[0], us, residual, a, b, c);
    charge(5);
    fill_ghosts(*out);
    if (out == &rk[0]) iface_cache_valid = false;
    const double th = stage_theta(stage);
    charge(7);
    if (!(th >= 1.0)) throw Retry{std::isfinite(th) ? th : 0.0};
  }
  void integrate(double dt) {  // ssprk_integrator.cpp:40-53
    for (int s = 0; s < 3; ++s) {
      compute_residual(rk[s], residual);
      combine_stage(s, dt);
    }
  }
  void advance_positive(double dt) {
    copy_state(rk[0], request_backup);
    const int prev_sub = last_substeps;
    try {
      double remaining = dt, trial = dt;
      bool low_interval = false;
      int retries = 0, attempts = 0;
      last_substeps = 0;
      anchor_available = admissible_fraction(rk[0], rk[0], 1) >= 1.0;
      while (remaining > 0.0) {
        if (++attempts > 100000) throw std::runtime_error("MhdSolver2D: positivity controller exceeded its substep limit");
        trial = std::min(trial, remaining);
        copy_state(rk[0], step_backup);
        control_active = true;
        try {
          integrate(trial);
        } catch (const Retry& r) {
          const bool high = low_order == 0;
          control_active = false;
          low_order = 0;
          copy_state(step_backup, rk[0]);
          iface_cache_valid = false;
          if (++retries > 80) throw std::runtime_error("MhdSolver2D: unable to find a positive conservative substep");
          if (high) {
            if (admissible_fraction(rk[0], rk[0], 1) >= 1.0) {
              anchor_available = true;
              low_interval = true;
              low_order = 1;
              trial = std::min(trial, cfl_limit(1));
              if (!(trial > 0.0) || !std::isfinite(trial) || !(remaining - trial < remaining)) {
                low_order = 0;
                throw std::runtime_error("MhdSolver2D: low-order CFL substep cannot advance time");
              }
              continue;
            }
          }
          const double f = std::max(0.05, std::min(0.8, 0.8 * r.theta));
          trial *= f;
          low_order = low_interval ? 1 : 0;
          if (!(trial > 0.0) || !std::isfinite(trial) || !(remaining - trial < remaining)) {
            low_order = 0;
            throw std::runtime_error("MhdSolver2D: positive conservative substep cannot advance time");
          }
          continue;
        }
        control_active = false;
        solver_owned = true;
        retries = 0;
        ++last_substeps;
        low_order = low_interval ? 1 : 0;
        if (trial == remaining) break;
        const double next = remaining - trial;
        if (!(next > 0.0) || !(next < remaining)) throw std::runtime_error("MhdSolver2D: positivity substep made no finite time progress");
        remaining = next;
        trial = std::min(std::min(2.0 * trial, remaining), cfl_limit(low_interval ? 1 : 0));
      }
      low_order = 0;
      control_active = false;
      anchor_available = false;
    } catch (...) {
      control_active = false;
      anchor_available = false;
      low_order = 0;
      last_substeps = prev_sub;
      copy_state(request_backup, rk[0]);
      iface_cache_valid = false;
      throw;
    }
  }
  void step_unchecked(double dt) {
    if (!(dt > 0.0) || !std::isfinite(dt)) throw std::invalid_argument("MhdSolver2D: dt must be finite and positive");
    ensure_admissible(0);
    advance_positive(dt);
  }
};

}  // namespace qoracle

// ---------------------------------------------------------------------------
// C ABI (ctypes) -- component order rho,mx,my,mz,energy,bx_face,by_face,bz_cell
using qoracle::Solver;
using Oracle = Solver<double>;
using Counting = Solver<qoracle::Counted>;

namespace {
thread_local std::string g_err;
struct Handle {
  Oracle* s = nullptr;
  Counting* c = nullptr;
};
template <class S>
void seed_into(S* s, int comp, const double* d) {
  std::memcpy(s->rk[0].c[comp].data(), d, sizeof(double) * s->g.size());
  s->solver_owned = false;
  s->iface_cache_valid = false;
}
}  // namespace

extern "C" {

int qor_count_phases(void* p, int steps, double* out);

const char* qor_last_error() { return g_err.c_str(); }

// counting != 0 builds the FLOP-counting instance instead.
void* qor_create(int nx, int ny, double lx, double ly, int order, double gamma,
                 double cfl, const int* bc, int counting) {
  try {
    qoracle::Config c{order, gamma, cfl, {bc[0], bc[1], bc[2], bc[3]}};
    if (nx < 1 || ny < 1 || !(gamma > 1.0) || !(cfl > 0.0 && cfl <= 1.0) ||
        (order != 2 && order != 5 && order != 7))
      throw std::invalid_argument("qor_create: invalid configuration");
    auto* h = new Handle;
    if (counting) h->c = new Counting(nx, ny, lx, ly, c);
    else h->s = new Oracle(nx, ny, lx, ly, c);
    return h;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void qor_destroy(void* p) {
  auto* h = static_cast<Handle*>(p);
  delete h->s;
  delete h->c;
  delete h;
}

int qor_seed(void* p, int comp, const double* d, size_t n) {
  auto* h = static_cast<Handle*>(p);
  const size_t want = h->s ? h->s->g.size() : h->c->g.size();
  if (n != want || comp < 0 || comp > 7) {
    g_err = "qor_seed: size or component mismatch";
    return -1;
  }
  for (size_t k = 0; k < n; ++k)
    if (!std::isfinite(d[k])) {
      g_err = "qor_seed: host buffer must contain only finite values";
      return -1;
    }
  if (h->s) seed_into(h->s, comp, d);
  else seed_into(h->c, comp, d);
  return 0;
}

int qor_read(void* p, int comp, double* out, size_t n) {
  auto* h = static_cast<Handle*>(p);
  const auto& v = h->s ? h->s->rk[0].c[comp] : h->c->rk[0].c[comp];
  if (n != v.size()) {
    g_err = "qor_read: size";
    return -1;
  }
  std::memcpy(out, v.data(), sizeof(double) * n);
  return 0;
}

int qor_cfl(void* p, double* dt) {
  auto* h = static_cast<Handle*>(p);
  try {
    *dt = h->s ? h->s->cfl_limit() : h->c->cfl_limit();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int qor_step(void* p, double dt) {
  auto* h = static_cast<Handle*>(p);
  try {
    if (h->s) h->s->step_unchecked(dt);
    else h->c->step_unchecked(dt);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int qor_substeps(void* p) {
  auto* h = static_cast<Handle*>(p);
  return h->s ? h->s->last_substeps : h->c->last_substeps;
}

// One residual L(u) of an arbitrary padded state (stage register 1).
int qor_residual(void* p, const double* const* in8, double* const* dudt,
                 double* const* ifx, double* const* ify, double* const* fx,
                 double* const* fy, double* ez, double* cell_ez) {
  auto* h = static_cast<Handle*>(p);
  Oracle* s = h->s;
  if (!s) {
    g_err = "qor_residual: counting instance";
    return -1;
  }
  try {
    const size_t n = s->g.size();
    for (int c = 0; c < 8; ++c) std::memcpy(s->rk[1].c[c].data(), in8[c], n * sizeof(double));
    s->iface_cache_valid = false;
    s->compute_residual(s->rk[1], s->residual);
    auto put = [&](const std::vector<double>& v, double* o) {
      if (o) std::memcpy(o, v.data(), n * sizeof(double));
    };
    for (int c = 0; c < 8; ++c) {
      if (dudt) put(s->residual.c[c], dudt[c]);
      if (fx) put(s->flux_x.c[c], fx[c]);
      if (fy) put(s->flux_y.c[c], fy[c]);
    }
    for (int c = 0; c < 8; ++c) {
      if (ifx) { put(s->ifx.L[c], ifx[c]); put(s->ifx.R[c], ifx[8 + c]); }
      if (ify) { put(s->ify.L[c], ify[c]); put(s->ify.R[c], ify[8 + c]); }
    }
    put(s->ez, ez);
    put(s->cell_ez, cell_ez);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// FLOPs (oracle_count.hpp rules) per zone-step of `steps` full steps of the
// counting instance, cfl_limit included: *as_written counts every operation
// the reference's code performs, *algorithmic applies the de-duplication
// rules of qor_count_phases, *cfl is the CFL-rate share of the latter.
int qor_count_flops(void* p, int steps, double* as_written, double* algorithmic,
                    double* cfl) {
  auto* h = static_cast<Handle*>(p);
  Counting* s = h->c;
  if (!s) {
    g_err = "qor_count_flops: not a counting instance";
    return -1;
  }
  try {
    for (auto& v : s->phase_flops) v = 0;
    qoracle::flop_counter() = 0;
    s->colloc_free = false;
    for (int k = 0; k < steps; ++k) {
      const double dt = s->cfl_limit();
      s->charge(7);
      s->step_unchecked(dt);
      s->charge(7);
    }
    const double zones = double(s->g.nx) * double(s->g.ny) * double(steps);
    double total = 0;
    for (auto v : s->phase_flops) total += double(v);
    *as_written = total / zones;
    double ph[8];
    const int rc = qor_count_phases(p, steps, ph);
    if (rc != 0) return rc;
    double alg = 0;
    for (double v : ph) alg += v;
    *algorithmic = alg;
    *cfl = ph[6];
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// Per-phase algorithmic FLOPs per zone-step (phases as Solver::charge):
// collocation counted once per padded cell per stage (the reference repeats
// it for every load), the face-EMF re-solve not counted (it repeats the flux
// solve), and each CFL face rate once (the per-cell reduction evaluates every
// interior face twice).  out[0..7].
int qor_count_phases(void* p, int steps, double* out) {
  auto* h = static_cast<Handle*>(p);
  Counting* s = h->c;
  if (!s) {
    g_err = "qor_count_phases: not a counting instance";
    return -1;
  }
  try {
    s->colloc_free = true;
    for (auto& v : s->phase_flops) v = 0;
    qoracle::flop_counter() = 0;
    for (int k = 0; k < steps; ++k) {
      const double dt = s->cfl_limit();
      s->charge(7);
      s->step_unchecked(dt);
      s->charge(7);
    }
    const double zones = double(s->g.nx) * double(s->g.ny) * double(steps);
    for (int k = 0; k < 8; ++k) out[k] = double(s->phase_flops[k]) / zones;
    out[6] *= 0.5;
    s->colloc_free = false;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// Pointwise restatements for known-answer tests.
int qor_hlld_flux_x(const double* l, const double* r, double gamma, double* f) {
  using S = qoracle::State<double>;
  const S L{l[0], l[1], l[2], l[3], l[4], l[5], l[6], l[7]};
  const S R{r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]};
  const auto F = qoracle::hlld_flux_x(L, R, gamma);
  const double o[8] = {F.rho, F.mx, F.my, F.mz, F.energy, F.bx, F.by, F.bz};
  std::memcpy(f, o, sizeof o);
  return 0;
}

int qor_eigensystem(const double* s8, double gamma, double* l49, double* r49,
                    double* speeds7) {
  const qoracle::State<double> s{s8[0], s8[1], s8[2], s8[3], s8[4], s8[5], s8[6], s8[7]};
  qoracle::Eigen<double> e;
  qoracle::build_eigensystem(s, gamma, e);
  std::memcpy(l49, e.L, sizeof e.L);
  std::memcpy(r49, e.Rm, sizeof e.Rm);
  std::memcpy(speeds7, e.speeds, sizeof e.speeds);
  return 0;
}

double qor_mp5(const double* v) { return qoracle::mp_reconstruct(v, 5); }
double qor_mp7(const double* v) { return qoracle::mp_reconstruct(v, 7); }

}  // extern "C"
