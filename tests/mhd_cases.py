"""Shared test helpers: seeded initial states and ctypes bindings for the two
CPU checkers (the oracle restatement in oracle/ and, when it was built, the
reference's own code in oracle/_ref).  Test infrastructure only.

Arrays are padded SoA storage, shape (ny + 2g, nx + 2g) in C order, so that
flat index (i + g) + (nx + 2g) * (j + g) matches core/grid.hpp:158-161 of the
reference.  Component order: rho, mx, my, mz, energy, bx_face, by_face,
bz_cell.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libquasar_mhd_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libquasar_mhd_ref.so")

COMPONENTS = ("rho", "mx", "my", "mz", "energy", "bx_face", "by_face", "bz_cell")
PERIODIC = (0, 0, 0, 0)
OUTFLOW = (1, 1, 1, 1)


def nghost(order: int) -> int:
    return 4 if order == 7 else 3 if order == 5 else 2


# Initial states: the product's generators (quasar_b200/ics.py), so the
# checkers and the CUDA path are always seeded with the same arrays.
sys.path.insert(0, ROOT)
from quasar_b200.ics import blast, orszag_tang, rotor  # noqa: E402,F401


# --------------------------------------------------------------------------
# ctypes bindings
# --------------------------------------------------------------------------
_dp = ctypes.POINTER(ctypes.c_double)


def _ptrs(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


class _Lib:
    prefix = ""

    def __init__(self, path):
        self.lib = ctypes.CDLL(path)
        p = self.prefix
        L = self.lib
        getattr(L, p + "last_error").restype = ctypes.c_char_p
        for f in ("seed", "read"):
            getattr(L, p + f).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
        getattr(L, p + "cfl").argtypes = [ctypes.c_void_p, _dp]
        getattr(L, p + "step").argtypes = [ctypes.c_void_p, ctypes.c_double]
        getattr(L, p + "destroy").argtypes = [ctypes.c_void_p]
        getattr(L, p + "substeps").argtypes = [ctypes.c_void_p]
        getattr(L, p + "hlld_flux_x").argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        getattr(L, p + "mp5").argtypes = [ctypes.c_void_p]
        getattr(L, p + "mp5").restype = ctypes.c_double
        getattr(L, p + "mp7").argtypes = [ctypes.c_void_p]
        getattr(L, p + "mp7").restype = ctypes.c_double

    def err(self):
        return getattr(self.lib, self.prefix + "last_error")().decode()

    def hlld_flux_x(self, left, right, gamma):
        left = np.ascontiguousarray(left, dtype=np.float64)
        right = np.ascontiguousarray(right, dtype=np.float64)
        out = np.zeros(8)
        getattr(self.lib, self.prefix + "hlld_flux_x")(left.ctypes.data, right.ctypes.data, gamma, out.ctypes.data)
        return out

    def mp(self, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        f = self.prefix + ("mp5" if v.size == 5 else "mp7")
        return getattr(self.lib, f)(v.ctypes.data)


class CpuSolver:
    """Common driver over either checker: seed, cfl, step, read."""

    def __init__(self, lib: _Lib, handle, nx, ny, order):
        self.L = lib
        self.h = handle
        self.nx, self.ny, self.order = nx, ny, order
        self.ng = nghost(order)
        self.shape = (ny + 2 * self.ng, nx + 2 * self.ng)

    def __del__(self):
        try:
            getattr(self.L.lib, self.L.prefix + "destroy")(self.h)
        except Exception:
            pass

    def _call(self, name, *args):
        rc = getattr(self.L.lib, self.L.prefix + name)(self.h, *args)
        if rc != 0:
            raise RuntimeError(self.L.err())

    def seed(self, comps):
        for c, a in enumerate(comps):
            a = np.ascontiguousarray(a, dtype=np.float64)
            assert a.shape == self.shape
            self._call("seed", c, a.ctypes.data, a.size)

    def read(self):
        out = []
        for c in range(8):
            a = np.empty(self.shape)
            self._call("read", c, a.ctypes.data, a.size)
            out.append(a)
        return out

    def cfl(self):
        d = ctypes.c_double()
        self._call("cfl", ctypes.byref(d))
        return d.value

    def step(self, dt):
        self._call("step", dt)

    def substeps(self):
        return getattr(self.L.lib, self.L.prefix + "substeps")(self.h)

    def residual(self, comps):
        """L(u) of an arbitrary padded state: dict of dudt, ifx, ify, fx, fy, ez."""
        comps = [np.ascontiguousarray(a, dtype=np.float64) for a in comps]
        mk = lambda k: [np.zeros(self.shape) for _ in range(k)]  # noqa: E731
        out = dict(dudt=mk(8), ifx=mk(16), ify=mk(16), fx=mk(8), fy=mk(8),
                   ez=np.zeros(self.shape), cell_ez=np.zeros(self.shape))
        args = [_ptrs(comps), _ptrs(out["dudt"]), _ptrs(out["ifx"]), _ptrs(out["ify"]),
                _ptrs(out["fx"]), _ptrs(out["fy"]), ctypes.c_void_p(out["ez"].ctypes.data),
                ctypes.c_void_p(out["cell_ez"].ctypes.data)]
        if isinstance(self.L, RefLib):
            args += [None, None]
        self._call("residual", *args)
        return out


class OracleLib(_Lib):
    prefix = "qor_"

    def __init__(self, path=ORACLE_SO):
        super().__init__(path)
        L = self.lib
        L.qor_create.restype = ctypes.c_void_p
        L.qor_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.qor_residual.argtypes = [ctypes.c_void_p] * 9
        L.qor_count_flops.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp]
        L.qor_count_phases.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]

    def solver(self, nx, ny, order, gamma=5.0 / 3.0, cfl=0.4, bc=PERIODIC, lx=1.0, ly=1.0, counting=False):
        h = self.lib.qor_create(nx, ny, lx, ly, order, gamma, cfl, (ctypes.c_int * 4)(*bc), int(counting))
        if not h:
            raise RuntimeError(self.err())
        return CpuSolver(self, h, nx, ny, order)

    def count_flops(self, solver: CpuSolver, steps: int):
        """(as written, algorithmic, CFL share) FLOPs per zone-step."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        solver._call("count_flops", steps, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def count_phases(self, solver: CpuSolver, steps: int):
        """Algorithmic FLOPs per zone-step by phase (see qor_count_phases)."""
        out = np.zeros(8)
        solver._call("count_phases", steps, out.ctypes.data)
        return out


class RefLib(_Lib):
    prefix = "qref_"

    def __init__(self, path=REF_SO):
        super().__init__(path)
        L = self.lib
        L.qref_create.restype = ctypes.c_void_p
        L.qref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
        L.qref_residual.argtypes = [ctypes.c_void_p] * 11
        L.qref_divb.argtypes = [ctypes.c_void_p, _dp]
        if hasattr(L, "qref_divb_relative"):
            L.qref_divb_relative.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
            L.qref_solenoidal_tolerance.restype = ctypes.c_double

    def divb_relative(self, solver, solver_owned):
        """The reference's live-state solenoidality measure of the solver's
        live register, as a stepped (solver_owned) or a seeded state."""
        v = ctypes.c_double()
        if self.lib.qref_divb_relative(solver.h, int(solver_owned), ctypes.byref(v)) != 0:
            raise RuntimeError(self.err())
        return v.value

    def solenoidal_tolerance(self):
        return self.lib.qref_solenoidal_tolerance()

    def solver(self, nx, ny, order, gamma=5.0 / 3.0, cfl=0.4, bc=PERIODIC, lx=1.0, ly=1.0,
               ox=0.0, oy=0.0):
        h = self.lib.qref_create(nx, ny, lx, ly, ox, oy, order, gamma, cfl, (ctypes.c_int * 4)(*bc))
        if not h:
            raise RuntimeError(self.err())
        return CpuSolver(self, h, nx, ny, order)

    # Parameter order of qref_initial_state (oracle/ref_capi.cpp).
    IC_PARAMS = (["interface"] + [f"left_{k}" for k in range(8)] +
                 [f"right_{k}" for k in range(8)] +
                 ["rho", "pressure", "b0", "total_b0", "amplitude", "wavenumber",
                  "magnetic_velocity_scale", "bx", "by", "bz", "cx", "cy", "r_in", "r0", "r1",
                  "rho_in", "rho_out", "p_in", "p_out", "p_core", "p_ambient", "rho_ambient",
                  "u0", "blob_half", "magnetic_scale"])
    IC_DEFAULTS = dict(interface=0.5, rho=1.0, pressure=0.1, b0=1.0, total_b0=1.0,
                       amplitude=1e-6, wavenumber=1.0, magnetic_velocity_scale=1.0, r_in=0.1,
                       r0=0.1, r1=0.115, rho_in=10.0, rho_out=1.0, p_in=1.0, p_out=0.1,
                       p_core=10.0, p_ambient=0.1, rho_ambient=1.0, u0=2.0, magnetic_scale=1.0)

    def initial_state(self, kind, nx, ny, lx, ly, ox, oy, ng, gamma, order, **params):
        """The reference's own build_initial_state (8 padded components)."""
        vals = dict(self.IC_DEFAULTS, **params)
        par = np.array([float(vals.get(k, 0.0)) for k in self.IC_PARAMS])
        n = (nx + 2 * ng) * (ny + 2 * ng)
        out = [np.zeros(n) for _ in range(8)]
        L = self.lib
        L.qref_initial_state.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + \
            [ctypes.c_double] * 4 + [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_void_p]
        rc = L.qref_initial_state(kind, nx, ny, lx, ly, ox, oy, ng, gamma, order,
                                  par.ctypes.data, _ptrs(out))
        if rc != 0:
            raise ValueError(self.err())
        return out


def oracle_available():
    return os.path.exists(ORACLE_SO)


def ref_available():
    return os.path.exists(REF_SO)


# --------------------------------------------------------------------------
# Metrics
# --------------------------------------------------------------------------
def interior(a, ng):
    return a[ng:-ng, ng:-ng]


def rel_l1(a, b, ng):
    """Relative L1 over the interior: sum|a-b| / sum|b| (0 if both zero)."""
    x, y = interior(a, ng), interior(b, ng)
    den = np.abs(y).sum()
    num = np.abs(x - y).sum()
    return 0.0 if num == 0.0 else num / max(den, 1e-300)


def _evolved(a, c, ng, nx, ny):
    if c == 5:
        return a[ng:ng + ny, ng:ng + nx + 1]
    if c == 6:
        return a[ng:ng + ny + 1, ng:ng + nx]
    return a[ng:ng + ny, ng:ng + nx]


# Relative L1 is taken per physical group so that a component which is zero
# analytically (mz, bz in 2-D problems) is measured against its vector.
GROUPS = ((0,), (1, 2, 3), (4,), (5, 6, 7))


def state_rel_l1(sa, sb, ng, nx, ny):
    """Max over groups (rho, momentum, energy, field) of
    sum|a-b| / sum|b| on the evolved region (cells plus owned high faces)."""
    worst = 0.0
    for grp in GROUPS:
        num = sum(np.abs(_evolved(sa[c], c, ng, nx, ny) - _evolved(sb[c], c, ng, nx, ny)).sum() for c in grp)
        den = sum(np.abs(_evolved(sb[c], c, ng, nx, ny)).sum() for c in grp)
        if num == 0.0:
            continue
        worst = max(worst, num / den if den > 0 else np.inf)
    return worst


def summary_rel(state, fx, n, order):
    """Largest relative L1 gap, per physical group, between a state and a
    summary fixture (tests/golden/make_golden.py `summarize`): over the
    strided subsample, the row sums and the column sums.  A cell that
    differs shows in its row's and its column's sum (and in the subsample
    when it lies on the stride), so a local defect cannot hide."""
    ng = nghost(order)
    sub = int(fx["sub_stride"])
    worst = 0.0
    for grp in GROUPS:
        num = {"sub": 0.0, "row": 0.0, "col": 0.0}
        den = dict(num)
        for c in grp:
            name = COMPONENTS[c]
            a = _evolved(state[c], c, ng, n, n)
            num["sub"] += np.abs(a[::sub, ::sub] - fx[name + "_sub"]).sum()
            den["sub"] += np.abs(fx[name + "_sub"]).sum()
            num["row"] += np.abs(a.sum(axis=1) - fx[name + "_row_sum"]).sum()
            den["row"] += fx[name + "_row_abs"].sum()
            num["col"] += np.abs(a.sum(axis=0) - fx[name + "_col_sum"]).sum()
            den["col"] += fx[name + "_col_abs"].sum()
        for k in num:
            if num[k] > 0.0:
                worst = max(worst, num[k] / den[k] if den[k] > 0.0 else np.inf)
    return worst


def divb_max(s, ng, nx, ny, dx, dy):
    bx, by = s[5], s[6]
    d = ((bx[ng:ng + ny, ng + 1:ng + nx + 1] - bx[ng:ng + ny, ng:ng + nx]) / dx +
         (by[ng + 1:ng + ny + 1, ng:ng + nx] - by[ng:ng + ny, ng:ng + nx]) / dy)
    return float(np.abs(d).max())
