"""Python mirror of the reference's `_core.mhd` module
(bindings/python/bind_mhd.cpp:571-647) over the sm_100a C ABI.

    cfg = MhdConfig()
    cfg.grid = Grid2D(256, 256, 1.0, 1.0)
    cfg.reconstruction = "mp7"
    solver = MhdSolver2D(cfg)
    solver.seed_state("rho", rho_padded)      # storage-sized float64 arrays
    dt = solver.cfl_limit(); solver.step_unchecked(dt)
    rho = solver.state_component_to_host("rho")
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import _native

_ORDERS = {"muscl_minmod": 2, "mp5": 5, "mp7": 7}
_BC = {"periodic": 0, "outflow": 1, "wall": 2}


@dataclass
class Grid2D:
    """core/grid.hpp:84-161 (nghost 0 lets the solver size the halo)."""
    nx: int = 1
    ny: int = 1
    lx: float = 1.0
    ly: float = 1.0
    origin_x: float = 0.0
    origin_y: float = 0.0
    nghost: int = 0

    def dx(self) -> float:
        return self.lx / self.nx

    def dy(self) -> float:
        return self.ly / self.ny

    def pitch(self) -> int:
        return self.nx + 2 * self.nghost

    def storage_size(self) -> int:
        return (self.nx + 2 * self.nghost) * (self.ny + 2 * self.nghost)


def _side(side: int) -> int:
    # pybind11 maps the binding's std::out_of_range("side") to IndexError
    if not 0 <= int(side) <= 3:
        raise IndexError("side")
    return int(side)


@dataclass
class MhdBoundarySpec:
    """boundary/mhd_boundary.hpp: per-side registry names, [x_lo,x_hi,y_lo,y_hi],
    with the setters and getters of bind_mhd.cpp:503-545."""
    fluid: List[str] = field(default_factory=lambda: ["periodic"] * 4)
    field: List[str] = field(default_factory=lambda: ["periodic"] * 4)

    def set_fluid_all(self, kind: str) -> None:
        self.fluid = [kind] * 4

    def set_fluid_side(self, side: int, kind: str) -> None:
        self.fluid[_side(side)] = kind

    def fluid_side(self, side: int) -> str:
        return self.fluid[_side(side)]

    def set_field_all(self, kind: str) -> None:
        self.field = [kind] * 4

    def set_field_side(self, side: int, kind: str) -> None:
        self.field[_side(side)] = kind

    def field_side(self, side: int) -> str:
        return self.field[_side(side)]


@dataclass
class MhdBackgroundSpec:
    """physics/mhd/mhd_background.hpp:67-84.  This library runs the zero-background
    step only: a solver whose spec is enabled is refused."""
    enabled: bool = False
    profile: str = "uniform"
    bx0: float = 0.0
    by0: float = 0.0
    bz0: float = 0.0
    params: dict = field(default_factory=dict)
    profile_scale: float = 1.0
    curl_free: bool = False


@dataclass
class MhdConfig:
    """physics/mhd/mhd_solver.hpp:50-83."""
    grid: Grid2D = field(default_factory=Grid2D)
    gamma: float = 5.0 / 3.0
    geometry: str = "cartesian"
    reconstruction: str = "mp7"
    riemann: str = "hlld"
    integrator: str = "ssprk3"
    ct: str = "fd_ct_christlieb"
    positivity: str = "troubled_cell"
    rho_floor: float = 1e-8
    p_floor: float = 1e-9
    cfl: float = 0.4
    # restart/checkpoint identity of the dt policy (mhd_solver.hpp:70-76); kept,
    # not interpreted, as by the solver itself
    timestep_signature: str = ""
    boundary: MhdBoundarySpec = field(default_factory=MhdBoundarySpec)
    background: MhdBackgroundSpec = field(default_factory=MhdBackgroundSpec)


def _check_device_pair(idx, vals, what: str) -> None:
    import torch
    if not (isinstance(idx, torch.Tensor) and isinstance(vals, torch.Tensor)):
        raise TypeError(f"{what}: idx and values must be torch tensors")
    if idx.dtype != torch.int64 or vals.dtype != torch.float64:
        raise TypeError(f"{what}: idx must be int64 and values float64")
    if not (idx.is_cuda and vals.is_cuda and idx.is_contiguous() and vals.is_contiguous()):
        raise ValueError(f"{what}: idx and values must be contiguous CUDA tensors")
    if idx.numel() != vals.numel():
        raise ValueError(f"{what}: idx and values differ in length")


def _native_config(cfg: MhdConfig) -> _native.QmhdConfig:
    if cfg.geometry != "cartesian":
        raise ValueError("MhdSolver2D: geometry must be 'cartesian' in this library")
    if cfg.background.enabled:
        raise ValueError("MhdSolver2D: the field-split background is not supported in this library")
    if cfg.riemann != "hlld":
        raise ValueError("MhdSolver2D: device evolution supports only riemann='hlld'")
    if cfg.ct != "fd_ct_christlieb":
        raise ValueError("MhdSolver2D: device evolution supports only ct='fd_ct_christlieb'")
    if cfg.integrator != "ssprk3":
        raise ValueError(f"MhdSolver2D: unknown integrator '{cfg.integrator}'")
    if cfg.positivity != "troubled_cell":
        raise ValueError(f"MhdSolver2D: unknown positivity limiter '{cfg.positivity}'")
    if cfg.reconstruction not in _ORDERS:
        raise ValueError(
            "MhdSolver2D: device evolution supports only reconstruction='muscl_minmod', "
            "'mp5', or 'mp7'")
    order = _ORDERS[cfg.reconstruction]
    required = 4 if order == 7 else 3 if order == 5 else 2
    if cfg.grid.nghost > 0 and cfg.grid.nghost != required:
        raise ValueError(
            f"MhdSolver2D: grid nghost ({cfg.grid.nghost}) must equal the reconstruction "
            f"scheme's halo ({required}) in this library")
    bc = []
    for side in range(4):
        f, b = cfg.boundary.fluid[side], cfg.boundary.field[side]
        if f not in _BC or b not in _BC:
            raise ValueError(f"MhdSolver2D: unknown boundary '{f if f not in _BC else b}'")
        if f != b:
            raise ValueError("MhdSolver2D: fluid and field boundaries must match per side in this library")
        bc.append(_BC[f])
    c = _native.QmhdConfig()
    c.nx, c.ny = int(cfg.grid.nx), int(cfg.grid.ny)
    c.lx, c.ly = float(cfg.grid.lx), float(cfg.grid.ly)
    c.origin_x, c.origin_y = float(cfg.grid.origin_x), float(cfg.grid.origin_y)
    c.reconstruction_order = order
    c.gamma = float(cfg.gamma)
    c.cfl = float(cfg.cfl)
    for s in range(4):
        c.boundary[s] = bc[s]
    return c


class MhdSolver2D:
    """physics/mhd/mhd_solver.hpp:85-173 on the sm_100a kernels."""

    def __init__(self, config: MhdConfig, _handle=None, _owner=None):
        L = _native.lib()
        self._cfg = config
        self._owner = _owner  # a batch view keeps its batch alive
        if _handle is None:
            h = ctypes.c_void_p()
            _native.check(L.qmhd_solver_create(ctypes.byref(_native_config(config)), ctypes.byref(h)))
        else:
            h = _handle
        self._h = h
        nx, ny, ng = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _native.check(L.qmhd_solver_grid(self._h, ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(ng)))
        g = config.grid
        self._grid = Grid2D(nx.value, ny.value, g.lx, g.ly, g.origin_x, g.origin_y, ng.value)
        self._n = int(L.qmhd_solver_storage_size(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_owner", None) is None:
            _native.lib().qmhd_solver_destroy(h)
        self._h = None

    def grid(self) -> Grid2D:
        return self._grid

    def config(self) -> MhdConfig:
        return self._cfg

    def seed_state(self, component: str, values) -> None:
        a = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1))
        _native.check(_native.lib().qmhd_solver_seed_state(
            self._h, component.encode(), a.ctypes.data, a.size))

    def state_component_to_host(self, component: str) -> np.ndarray:
        out = np.empty(self._n, dtype=np.float64)
        _native.check(_native.lib().qmhd_solver_state_component_to_host(
            self._h, component.encode(), out.ctypes.data, out.size))
        return out

    def cfl_limit(self) -> float:
        d = ctypes.c_double()
        _native.check(_native.lib().qmhd_solver_cfl_limit(self._h, ctypes.byref(d)))
        return d.value

    def step(self, dt: float) -> None:
        _native.check(_native.lib().qmhd_solver_step(self._h, float(dt)))

    def step_unchecked(self, dt: float) -> None:
        _native.check(_native.lib().qmhd_solver_step_unchecked(self._h, float(dt)))

    def advance(self, t_end: float, dt: float) -> None:
        _native.check(_native.lib().qmhd_solver_advance(self._h, float(t_end), float(dt)))

    def divergence_b_max(self) -> float:
        d = ctypes.c_double()
        _native.check(_native.lib().qmhd_solver_divergence_b_max(self._h, ctypes.byref(d)))
        return d.value

    def set_owned_window(self, x0: int, x1: int, y0: int, y1: int) -> None:
        """Restrict dt, retry and preflight reductions to interior cells
        [x0, x1) x [y0, y1) (a tile of a decomposed domain; the rest is halo)."""
        _native.check(_native.lib().qmhd_solver_set_owned_window(self._h, int(x0), int(x1),
                                                                 int(y0), int(y1)))

    def write_halo(self, component: str, values) -> None:
        """Write a whole component whose values come from the solver's own
        steps (neighbouring tiles' owned cells); the state stays
        solver-owned."""
        a = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1))
        _native.check(_native.lib().qmhd_solver_write_halo(
            self._h, component.encode(), a.ctypes.data, a.size))

    def gather_live(self, component: str, idx, out) -> None:
        """out[k] = live value of `component` at storage index idx[k]; idx
        (int64) and out (float64) are contiguous CUDA tensors of the
        solver's device."""
        _check_device_pair(idx, out, "gather_live")
        _native.check(_native.lib().qmhd_solver_gather_live(
            self._h, component.encode(), idx.data_ptr(), idx.numel(), out.data_ptr()))

    def scatter_halo(self, component: str, idx, values) -> None:
        """Live value of `component` at storage index idx[k] = values[k]
        (finite, from the solver's own steps); the state stays
        solver-owned.  CUDA tensors as for gather_live."""
        _check_device_pair(idx, values, "scatter_halo")
        _native.check(_native.lib().qmhd_solver_scatter_halo(
            self._h, component.encode(), idx.data_ptr(), idx.numel(), values.data_ptr()))

    def divergence_b_relative(self) -> float:
        """Dimensionless solenoidality: max |div B| x dx / max |B_face| over
        the evolved faces, the measure the reference's own example tests
        assert (tests/python/test_examples.py:1985-2003: below 1e-11).  Not a
        method of the reference's solver; it reads the face field back."""
        g = self._grid
        ng, nx, ny = g.nghost, g.nx, g.ny
        shape = (ny + 2 * ng, nx + 2 * ng)
        bx = self.state_component_to_host("bx_face").reshape(shape)[ng:ng + ny, ng:ng + nx + 1]
        by = self.state_component_to_host("by_face").reshape(shape)[ng:ng + ny + 1, ng:ng + nx]
        bmax = float(max(np.abs(bx).max(), np.abs(by).max()))
        d = self.divergence_b_max()
        return d * g.dx() / bmax if bmax > 0.0 else d

    def conserved_cell_totals(self):
        m, e = ctypes.c_double(), ctypes.c_double()
        _native.check(_native.lib().qmhd_solver_conserved_cell_totals(
            self._h, ctypes.byref(m), ctypes.byref(e)))
        return (m.value, e.value)

    def has_background(self) -> bool:
        """Always False: this library runs the zero-background step."""
        return False

    def seed_background(self, component: str, values) -> None:
        # mhd_solver.cpp:543-549: a solver without an enabled background
        # refuses B0 (std::logic_error, RuntimeError in Python)
        raise RuntimeError(
            "MhdSolver2D::seed_background: the field-split background is not enabled "
            "(set background.enabled in the deck before seeding B0)")

    def last_positivity_substeps(self) -> int:
        return int(_native.lib().qmhd_solver_last_positivity_substeps(self._h))

    def advance_auto(self, t: float, t_end: float, max_steps: int):
        """Device-resident auto-dt loop; returns (t, steps_taken)."""
        tt, n = ctypes.c_double(float(t)), ctypes.c_int()
        _native.check(_native.lib().qmhd_solver_advance_auto(
            self._h, ctypes.byref(tt), float(t_end), int(max_steps), ctypes.byref(n)))
        return tt.value, n.value


class MhdBatch2D:
    """Many independent instances stepped together (include/quasar_mhd_batch.h).

    No counterpart in the reference, which runs one MhdSolver2D per instance.
    `instance(i)` is an MhdSolver2D view of instance i (seed, read, check or
    step it alone); `advance(steps)` steps every instance with its own auto dt
    in batched persistent launches replayed as CUDA graphs.
    """

    PHASES = 9

    def __init__(self, configs):
        L = _native.lib()
        configs = list(configs)
        arr = (_native.QmhdConfig * len(configs))(*[_native_config(c) for c in configs])
        h = ctypes.c_void_p()
        _native.check(L.qmhd_batch_create(arr, len(configs), ctypes.byref(h)))
        self._h = h
        self._views = [MhdSolver2D(c, _handle=ctypes.c_void_p(L.qmhd_batch_instance(h, i)),
                                   _owner=self) for i, c in enumerate(configs)]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            for v in getattr(self, "_views", []):
                v._h = None
            _native.lib().qmhd_batch_destroy(h)
            self._h = None

    def __len__(self) -> int:
        return len(self._views)

    def instance(self, i: int) -> MhdSolver2D:
        return self._views[i]

    def zones(self) -> int:
        return int(_native.lib().qmhd_batch_zones(self._h))

    def advance(self, steps: int) -> list:
        done = (ctypes.c_int * len(self))()
        _native.check(_native.lib().qmhd_batch_advance(self._h, int(steps), done))
        return list(done)

    def time_steps(self, steps: int):
        ms, zu = ctypes.c_double(), ctypes.c_longlong()
        _native.check(_native.lib().qmhd_batch_time_steps(
            self._h, int(steps), ctypes.byref(ms), ctypes.byref(zu)))
        return ms.value, zu.value

    def autotune(self):
        c = (ctypes.c_int * self.PHASES)()
        t = ctypes.c_int()
        _native.check(_native.lib().qmhd_batch_autotune(self._h, c, ctypes.byref(t)))
        return list(c), t.value

    def profile_step(self) -> dict:
        """One step of every instance with per-phase device times (ms)."""
        ms = (ctypes.c_double * (self.PHASES + 1))()
        _native.check(_native.lib().qmhd_batch_profile_step(self._h, ms, self.PHASES + 1))
        names = ["recon_x", "recon_y", "face_flux", "cell_emf", "corner_emf", "update",
                 "collocation", "ghosts_x", "ghosts_y", "control"]
        return dict(zip(names, ms[:]))

    def set_tuning(self, ctas_per_sm) -> None:
        c = (ctypes.c_int * self.PHASES)(*[int(x) for x in ctas_per_sm])
        _native.check(_native.lib().qmhd_batch_set_tuning(self._h, c))


# -- Registry introspection (bind_mhd.cpp:101-253) ---------------------------
# The names this library accepts, sorted like the binding's lists; the deck
# validators select against them.  The reference's "axis" boundary, its
# background profiles and its internal tile boundary are outside this library.
def registered_riemann_solvers() -> List[str]:
    return ["hlld"]


def registered_reconstructions() -> List[str]:
    return sorted(_ORDERS)


def registered_integrators() -> List[str]:
    return ["ssprk3"]


def registered_ct_schemes() -> List[str]:
    return ["fd_ct_christlieb"]


def registered_positivity_limiters() -> List[str]:
    return ["troubled_cell"]


def registered_mhd_fluid_boundaries() -> List[str]:
    return sorted(_BC)


def registered_mhd_field_boundaries() -> List[str]:
    return sorted(_BC)


def registered_mhd_background_profiles() -> List[str]:
    return []


def registered_initial_conditions() -> List[str]:
    """Built-in initial-condition generators, in the reference's kind order."""
    return ["brio_wu", "alfven_wave", "orszag_tang", "blast", "rotor", "confined_blob"]


def reconstruction_halo(name: str) -> int:
    """Ghost-cell halo of the named reconstruction (bind_mhd.cpp:133-147)."""
    if name not in _ORDERS:
        raise ValueError(f"unknown MHD reconstruction scheme '{name}'")
    order = _ORDERS[name]
    return 4 if order == 7 else 3 if order == 5 else 2


def reconstruction_order(name: str) -> int:
    """Formal order from the halo (flux_reconstruction.hpp:65-71)."""
    return {3: 5, 4: 7}.get(reconstruction_halo(name), 2)
