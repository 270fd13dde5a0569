"""Run the reference's ideal-MHD decks on the B200 solver.

    python -m quasar_b200.deck run path/to/input.yaml [--steps-override N]

Drop-in for `python -m quasar.mhd.cli run` (python/quasar/mhd/cli.py) on the
decks this library evolves: Cartesian geometry, no static background field,
reconstruction muscl_minmod / mp5 / mp7 with HLLD, CT, SSP-RK3 and the
troubled-cell positivity controller, periodic / outflow / wall boundaries
(the same per side for fluid and field).  Everything else is rejected with a
ValueError naming the feature.

* The deck schema and validation follow quasar.mhd.io (python/quasar/mhd/
  io.py:292-905): the same keys, defaults and error conditions.
* The initial states follow the reference's seed kernels
  (src/backend/hip/mhd/mhd_initial_conditions.hip:59-330): each generator is
  evaluated at the cell centre fma(i + 1/2, dx, x0) of every padded cell, the
  faces take the centre value, the energy is formed from the primitives with
  the raw magnetic half-norm and then re-formed as (E - raw) + |B_c|^2 / 2
  from the face-to-cell collocated field.  The arithmetic is restated here in
  float64 in the kernel's order; the collocation is this library's own
  (qmhd_launch_collocate_face_to_cell) on the analytic arrays.
* The run loop and the .npz archive follow quasar.mhd.cli (cli.py:110-492):
  the same dt policy (auto: cfl_limit() before every step, clipped to t_end),
  step/time termination, div B sampling and snapshot cadence, and the same
  archive keys (state_*, state_*_initial, divb_linf, snapshot_*, and the OT
  mass/energy invariants).
"""
from __future__ import annotations

import argparse
import copy
import math
import time
from dataclasses import dataclass, field
from fractions import Fraction
from pathlib import Path
from typing import Sequence, Union

import numpy as np

from . import mhd

STATE_COMPONENTS = ("rho", "mx", "my", "mz", "energy", "bx", "by", "bz")
_PRIMITIVE_KEYS = ("rho", "p", "vx", "vy", "vz", "bx", "by", "bz")
_TOP_LEVEL_KEYS = {"units", "domain", "geometry", "numerics", "initial", "time",
                   "diagnostics", "boundary", "background_field"}
INITIAL_TYPES = ("brio_wu", "alfven_wave", "orszag_tang", "blast", "rotor", "confined_blob")
MAX_GRID_DIM = 1 << 16  # cells per axis (io.py:83-84)
MAX_GRID_CELLS = 1 << 30
_KIND = {name: k for k, name in enumerate(INITIAL_TYPES)}
MU0 = 4.0e-7 * math.pi
SQRT_MU0 = math.sqrt(MU0)


# ---- deck schema (python/quasar/mhd/io.py:292-905) ---------------------------
@dataclass
class Domain:
    nx: int
    ny: int
    lx_m: float
    ly_m: float
    origin_x_m: float = 0.0
    origin_y_m: float = 0.0


@dataclass
class Numerics:
    gamma: float = 5.0 / 3.0
    reconstruction: str = "mp7"
    riemann: str = "hlld"
    integrator: str = "ssprk3"
    ct: str = "fd_ct_christlieb"
    positivity: str = "troubled_cell"
    rho_floor: float = 1.0e-8
    p_floor: float = 1.0e-9
    cfl: float = 0.4


@dataclass
class Initial:
    type: str
    params: dict = field(default_factory=dict)


@dataclass
class Time:
    dt_s: Union[float, str] = "auto"
    steps: int = 100
    t_end: Union[float, None] = None


@dataclass
class Diagnostics:
    output_path: str = "out.npz"
    cadence: int = 0
    fields: list = field(default_factory=lambda: list(STATE_COMPONENTS))
    divb: bool = True

    def __post_init__(self) -> None:
        self.fields = [str(name).lower() for name in self.fields]


@dataclass
class BoundaryConfig:
    fluid: tuple = ("periodic",) * 4
    field: tuple = ("periodic",) * 4


@dataclass
class MhdDeck:
    domain: Domain
    numerics: Numerics = field(default_factory=Numerics)
    initial: Union[Initial, None] = None
    time: Time = field(default_factory=Time)
    diagnostics: Diagnostics = field(default_factory=Diagnostics)
    boundary: BoundaryConfig = field(default_factory=BoundaryConfig)
    units: str = "normalized"
    geometry: str = "cartesian"
    raw: dict = field(default_factory=dict)
    source_dir: Union[Path, None] = None

    def validate(self) -> None:
        if self.units not in ("SI", "normalized"):
            raise ValueError("units must be 'SI' or 'normalized'")
        if self.geometry not in ("cartesian", "cylindrical"):
            raise ValueError("geometry must be 'cartesian' or 'cylindrical'")
        if self.geometry != "cartesian":
            raise ValueError("geometry 'cylindrical' is not supported by the B200 solver")
        d = self.domain
        nx, ny = _exact_int(d.nx, "domain.nx"), _exact_int(d.ny, "domain.ny")
        if nx <= 0 or ny <= 0:
            raise ValueError("domain.nx and domain.ny must be positive")
        if nx > MAX_GRID_DIM or ny > MAX_GRID_DIM:
            raise ValueError(f"domain.nx/ny must be <= {MAX_GRID_DIM} (got {nx}x{ny})")
        if nx * ny > MAX_GRID_CELLS:
            raise ValueError(f"domain.nx*ny must be <= {MAX_GRID_CELLS} cells")
        for name in ("lx_m", "ly_m"):
            v = getattr(d, name)
            if not (math.isfinite(v) and v > 0.0):
                raise ValueError(f"domain.{name} must be finite and positive")
        for name in ("origin_x_m", "origin_y_m"):
            if not math.isfinite(getattr(d, name)):
                raise ValueError(f"domain.{name} must be finite")
        # io.py:434-449: the grid must stay representable in binary64 (upper
        # bounds, spacings, and distinct first and last cell centres)
        x0, y0 = float(d.origin_x_m), float(d.origin_y_m)
        x1, y1 = x0 + float(d.lx_m), y0 + float(d.ly_m)
        for v, what in ((x1, "domain upper x bound"), (y1, "domain upper y bound")):
            if not math.isfinite(v):
                raise ValueError(f"{what} must be finite")
        dx, dy = float(d.lx_m) / nx, float(d.ly_m) / ny
        for v, what in ((dx, "domain x spacing"), (dy, "domain y spacing")):
            if not (math.isfinite(v) and v > 0.0):
                raise ValueError(f"{what} must be finite and positive")
        if (x0 + 0.5 * dx == x0 or x0 + (nx - 0.5) * dx == x1
                or y0 + 0.5 * dy == y0 or y0 + (ny - 0.5) * dy == y1):
            raise ValueError("domain cell coordinates collapse in floating-point precision")
        n = self.numerics
        if not (math.isfinite(n.gamma) and n.gamma > 1.0):
            raise ValueError("numerics.gamma must be finite and greater than one")
        for value, names, context in (
                (n.reconstruction, mhd.registered_reconstructions(), "numerics.reconstruction"),
                (n.riemann, mhd.registered_riemann_solvers(), "numerics.riemann"),
                (n.integrator, mhd.registered_integrators(), "numerics.integrator"),
                (n.ct, mhd.registered_ct_schemes(), "numerics.ct"),
                (n.positivity, mhd.registered_positivity_limiters(), "numerics.positivity")):
            if value not in names:
                raise ValueError(f"{context} {value!r} must be one of {sorted(names)}")
        if not (math.isfinite(n.cfl) and n.cfl > 0.0):
            raise ValueError("numerics.cfl must be finite and positive")
        if self.initial is None:
            raise ValueError("initial is required")
        if self.initial.type not in INITIAL_TYPES:
            raise ValueError(f"initial.type {self.initial.type!r} must be one of "
                             f"{sorted(INITIAL_TYPES)}")
        _VALIDATORS[self.initial.type](self, self.initial.params)
        t = self.time
        if not (isinstance(t.dt_s, str) and t.dt_s == "auto"):
            if isinstance(t.dt_s, str) or not (math.isfinite(t.dt_s) and t.dt_s > 0.0):
                raise ValueError("time.dt_s must be 'auto' or a positive finite number")
        if _exact_int(t.steps, "time.steps") <= 0:
            raise ValueError("time.steps must be positive")
        if t.t_end is not None and not (math.isfinite(t.t_end) and t.t_end > 0.0):
            raise ValueError("time.t_end must be positive and finite")
        if (not isinstance(self.diagnostics.output_path, str)
                or not self.diagnostics.output_path.strip()):
            raise ValueError("diagnostics.output_path must be a non-empty string")
        if _exact_int(self.diagnostics.cadence, "diagnostics.cadence") < 0:
            raise ValueError("diagnostics.cadence must be non-negative")
        for name in self.diagnostics.fields:
            if name not in STATE_COMPONENTS:
                raise ValueError(f"diagnostics.fields entry {name!r} must be one of "
                                 f"{list(STATE_COMPONENTS)}")
        kinds = set(mhd.registered_mhd_fluid_boundaries()) & set(
            mhd.registered_mhd_field_boundaries())
        fl, fd = self.boundary.fluid, self.boundary.field
        for side in range(4):
            for part, kind in (("fluid", fl[side]), ("field", fd[side])):
                if kind == "internal":
                    raise ValueError(f"boundary.{part}[{side}] = 'internal' is reserved for "
                                     "the distributed tile runtime")
                if kind not in kinds:
                    raise ValueError(f"boundary kind {kind!r} is not supported by the B200 "
                                     "solver (periodic, outflow, wall)")
        # io.py:550-564
        for side in range(4):
            if (fl[side] == "periodic") != (fd[side] == "periodic"):
                raise ValueError("fluid and field periodicity must match on every side")
        for lo in (0, 2):
            if ((fl[lo] == "periodic") != (fl[lo + 1] == "periodic")
                    or (fd[lo] == "periodic") != (fd[lo + 1] == "periodic")):
                raise ValueError("periodic boundaries must be selected on both sides of an axis")
        for side in range(4):
            if self.boundary.fluid[side] != self.boundary.field[side]:
                raise ValueError("fluid and field boundaries must match per side in the B200 "
                                 "solver")


def _exact_int(value, context: str) -> int:
    """An integer as YAML gives it (io.py:100-115): booleans and floats,
    integral-looking ones such as 16.0 included, are refused so a misspelt
    deck cannot silently change its grid, run length, cadence or mode."""
    if isinstance(value, (bool, np.bool_)):
        raise ValueError(f"{context} must be an integer, not a boolean")
    if isinstance(value, (int, np.integer)):
        return int(value)
    raise ValueError(f"{context} must be an integer")


def _mapping(value, context: str) -> dict:
    if value is None:
        return {}
    if not isinstance(value, dict):
        raise ValueError(f"{context} must be a mapping")
    return value


def _reject_unknown(d: dict, allowed, context: str) -> None:
    unknown = sorted(set(d) - set(allowed))
    if unknown:
        raise ValueError(f"{context}: unknown key(s) {unknown}")


def _finite(value, context: str) -> float:
    try:
        v = float(value)
    except (TypeError, ValueError):
        raise ValueError(f"{context} must be a finite number") from None
    if not math.isfinite(v):
        raise ValueError(f"{context} must be a finite number")
    return v


def _positive(value, context: str) -> float:
    v = _finite(value, context)
    if not v > 0.0:
        raise ValueError(f"{context} must be positive")
    return v


def _pair(value, context: str):
    if not isinstance(value, (list, tuple)) or len(value) != 2:
        raise ValueError(f"{context} must be a two-element list")
    return _finite(value[0], context), _finite(value[1], context)


def _v_brio_wu(deck, p):
    _reject_unknown(p, {"interface", "left", "right"}, "initial.params")
    if "interface" not in p:
        raise ValueError("initial.params: missing required key 'interface'")
    _finite(p["interface"], "initial.params.interface")
    for side in ("left", "right"):
        state = _mapping(p.get(side), f"initial.params.{side}")
        _reject_unknown(state, _PRIMITIVE_KEYS, f"initial.params.{side}")
        missing = [k for k in _PRIMITIVE_KEYS if k not in state]
        if missing:
            raise ValueError(f"initial.params.{side}: missing required field(s) {missing}")
        for k in _PRIMITIVE_KEYS:
            _finite(state[k], f"initial.params.{side}.{k}")
        _positive(state["rho"], f"initial.params.{side}.rho")
        _positive(state["p"], f"initial.params.{side}.p")
    if float(p["left"]["bx"]) != float(p["right"]["bx"]):
        raise ValueError("brio_wu requires a continuous normal magnetic field: "
                         "initial.params.left.bx must equal initial.params.right.bx")


def _v_alfven(deck, p):
    _reject_unknown(p, {"rho", "p", "b0", "amplitude", "wavenumber", "polarization"},
                    "initial.params")
    _positive(p.get("rho", 1.0), "initial.params.rho")
    _positive(p.get("p", 0.1), "initial.params.p")
    _finite(p.get("amplitude", 1.0e-6), "initial.params.amplitude")
    if _finite(p.get("b0", 1.0), "initial.params.b0") == 0.0:
        raise ValueError("alfven_wave requires a nonzero total axial background field")
    n = _exact_int(p.get("wavenumber", 1), "initial.params.wavenumber")
    if n <= 0:
        raise ValueError("initial.params.wavenumber must be positive")
    if 2 * n >= deck.domain.nx:
        raise ValueError("initial.params.wavenumber must be below the x-grid Nyquist mode")
    if p.get("polarization", "circular") != "circular":
        raise ValueError("alfven_wave currently supports only polarization='circular'")


def _v_orszag_tang(deck, p):
    _reject_unknown(p, {"b0"}, "initial.params")
    _finite(p.get("b0", 1.0), "initial.params.b0")


def _v_blast(deck, p):
    _reject_unknown(p, {"rho_ambient", "p_ambient", "p_core", "r_in", "center", "bx", "by", "bz"},
                    "initial.params")
    for k, dflt in (("rho_ambient", 1.0), ("p_ambient", 0.1), ("p_core", 10.0), ("r_in", 0.1)):
        _positive(p.get(k, dflt), f"initial.params.{k}")
    _pair(p.get("center", [0.0, 0.0]), "initial.params.center")
    for k in ("bx", "by", "bz"):
        _finite(p.get(k, 0.0), f"initial.params.{k}")


def _v_rotor(deck, p):
    _reject_unknown(p, {"center", "r0", "r1", "rho_in", "rho_out", "u0", "p", "bx", "by", "bz"},
                    "initial.params")
    _pair(p.get("center", [0.5, 0.5]), "initial.params.center")
    r0 = _finite(p.get("r0", 0.1), "initial.params.r0")
    r1 = _finite(p.get("r1", 0.115), "initial.params.r1")
    if r0 <= 0.0:
        raise ValueError("initial.params.r0 must be positive")
    if r1 <= r0:
        raise ValueError("initial.params.r1 must be greater than r0")
    for k, dflt in (("rho_in", 10.0), ("rho_out", 1.0), ("p", 1.0)):
        _positive(p.get(k, dflt), f"initial.params.{k}")
    for k, dflt in (("u0", 2.0), ("bx", 0.0), ("by", 0.0), ("bz", 0.0)):
        _finite(p.get(k, dflt), f"initial.params.{k}")


def _v_blob(deck, p):
    _reject_unknown(p, {"rho_in", "rho_out", "p_in", "p_out", "blob_half", "bz"},
                    "initial.params")
    for k, dflt in (("rho_in", 10.0), ("rho_out", 1.0), ("p_in", 1.0), ("p_out", 0.1)):
        _positive(p.get(k, dflt), f"initial.params.{k}")
    if "blob_half" in p:
        _positive(p["blob_half"], "initial.params.blob_half")
    _finite(p.get("bz", 0.1), "initial.params.bz")


_VALIDATORS = {"brio_wu": _v_brio_wu, "alfven_wave": _v_alfven, "orszag_tang": _v_orszag_tang,
               "blast": _v_blast, "rotor": _v_rotor, "confined_blob": _v_blob}


def _side_map(value, context: str):
    sides = ("x_lo", "x_hi", "y_lo", "y_hi")
    if value is None:
        return ("periodic",) * 4
    if isinstance(value, str):
        return (value,) * 4
    if isinstance(value, (list, tuple)):
        if len(value) != 4:
            raise ValueError(f"{context} must list four sides")
        return tuple(str(v) for v in value)
    if isinstance(value, dict):
        _reject_unknown(value, set(sides), context)
        return tuple(str(value.get(s, "periodic")) for s in sides)
    raise ValueError(f"{context} must be a name, a 4-list or a side map")


def parse(data: dict) -> MhdDeck:
    data = _mapping(data, "deck")
    _reject_unknown(data, _TOP_LEVEL_KEYS, "deck")
    if "domain" not in data:
        raise ValueError("deck: missing required key 'domain'")
    d = _mapping(data["domain"], "domain")
    _reject_unknown(d, {"nx", "ny", "lx_m", "ly_m", "origin_x_m", "origin_y_m"}, "domain")
    for k in ("nx", "ny", "lx_m", "ly_m"):
        if k not in d:
            raise ValueError(f"domain: missing required key {k!r}")
    domain = Domain(nx=_exact_int(d["nx"], "domain.nx"), ny=_exact_int(d["ny"], "domain.ny"),
                    lx_m=float(d["lx_m"]), ly_m=float(d["ly_m"]),
                    origin_x_m=float(d.get("origin_x_m", 0.0)),
                    origin_y_m=float(d.get("origin_y_m", 0.0)))
    n = _mapping(data.get("numerics"), "numerics")
    _reject_unknown(n, {"gamma", "reconstruction", "riemann", "integrator", "ct", "positivity",
                        "rho_floor", "p_floor", "cfl"}, "numerics")
    numerics = Numerics(gamma=float(n.get("gamma", 5.0 / 3.0)),
                        reconstruction=str(n.get("reconstruction", "mp7")),
                        riemann=str(n.get("riemann", "hlld")),
                        integrator=str(n.get("integrator", "ssprk3")),
                        ct=str(n.get("ct", "fd_ct_christlieb")),
                        positivity=str(n.get("positivity", "troubled_cell")),
                        rho_floor=float(n.get("rho_floor", 1.0e-8)),
                        p_floor=float(n.get("p_floor", 1.0e-9)),
                        cfl=float(n.get("cfl", 0.4)))
    initial = None
    if data.get("initial") is not None:
        i = _mapping(data["initial"], "initial")
        _reject_unknown(i, {"type", "params"}, "initial")
        if "type" not in i:
            raise ValueError("initial: missing required key 'type'")
        initial = Initial(type=str(i["type"]),
                          params=dict(_mapping(i.get("params", {}), "initial.params")))
    t = _mapping(data.get("time"), "time")
    _reject_unknown(t, {"dt_s", "steps", "t_end"}, "time")
    dt_raw = t.get("dt_s", "auto")
    tm = Time(dt_s=dt_raw if isinstance(dt_raw, str) else float(dt_raw),
              steps=_exact_int(t.get("steps", 100), "time.steps"),
              t_end=None if t.get("t_end") is None else float(t["t_end"]))
    g = _mapping(data.get("diagnostics"), "diagnostics")
    _reject_unknown(g, {"output_path", "cadence", "fields", "divb"}, "diagnostics")
    if not isinstance(g.get("output_path", "out.npz"), str):
        raise ValueError("diagnostics.output_path must be a string")
    divb = g.get("divb", True)
    if not isinstance(divb, bool):
        raise ValueError("diagnostics.divb must be a boolean")
    diagnostics = Diagnostics(output_path=g.get("output_path", "out.npz"),
                              cadence=_exact_int(g.get("cadence", 0), "diagnostics.cadence"),
                              fields=list(g.get("fields", list(STATE_COMPONENTS))), divb=divb)
    b = _mapping(data.get("boundary"), "boundary")
    _reject_unknown(b, {"fluid", "field"}, "boundary")
    boundary = BoundaryConfig(fluid=_side_map(b.get("fluid"), "boundary.fluid"),
                              field=_side_map(b.get("field"), "boundary.field"))
    bg = _mapping(data.get("background_field"), "background_field")
    _reject_unknown(bg, {"enabled", "profile", "bx0", "by0", "bz0", "params", "file", "a_file",
                         "conductors"}, "background_field")
    if not isinstance(bg.get("enabled", False), (bool, np.bool_)):
        raise ValueError("background_field.enabled must be a boolean")
    if bg.get("enabled", False):
        raise ValueError("background_field is not supported by the B200 solver "
                         "(field-split B0 is out of its scope)")
    deck = MhdDeck(domain=domain, numerics=numerics, initial=initial, time=tm,
                   diagnostics=diagnostics, boundary=boundary,
                   units=str(data.get("units", "normalized")),
                   geometry=str(data.get("geometry", "cartesian")), raw=data)
    deck.validate()
    return deck


def _yaml_load(text: str):
    """One YAML document with duplicate mapping keys refused (a later key
    would otherwise silently replace the earlier one)."""
    import yaml

    class Loader(yaml.SafeLoader):
        pass

    def mapping(loader, node, deep=False):
        seen = set()
        for key_node, _ in node.value:
            key = loader.construct_object(key_node, deep=deep)
            try:
                dup = key in seen
            except TypeError:
                dup = False
            if dup:
                raise ValueError(f"duplicate YAML key {key!r} at line "
                                 f"{key_node.start_mark.line + 1}")
            seen.add(key)
        return yaml.SafeLoader.construct_mapping(loader, node, deep=deep)

    Loader.add_constructor(yaml.resolver.BaseResolver.DEFAULT_MAPPING_TAG, mapping)
    return yaml.load(text, Loader=Loader)  # noqa: S506 (a SafeLoader subclass)


def load(path: Union[str, Path]) -> MhdDeck:
    with open(path) as fh:
        data = _yaml_load(fh.read())
    if not isinstance(data, dict):
        raise ValueError(f"{path}: top-level YAML must be a mapping")
    deck = parse(data)
    deck.source_dir = Path(path).resolve().parent
    return deck


# ---- initial states (mhd_initial_conditions.hip:59-330) ------------------------
def nghost(reconstruction: str) -> int:
    return mhd.reconstruction_halo(reconstruction)


def _centres(n: int, ng: int, spacing: float, origin: float) -> np.ndarray:
    """fma(i + 1/2, spacing, origin) for i in [-ng, n + ng), rounded once
    (core/grid.hpp:166-172)."""
    s, o = Fraction(spacing), Fraction(origin)
    return np.array([float(Fraction(2 * i + 1, 2) * s + o) for i in range(-ng, n + ng)])


def _half_squared_norm3(x, y, z):
    """numerics/mhd_state.hpp:98-106 elementwise."""
    scale = np.fmax(np.abs(x), np.fmax(np.abs(y), np.abs(z)))
    safe = np.where(scale == 0.0, 1.0, scale)
    xs, ys, zs = x / safe, y / safe, z / safe
    out = (0.5 * safe) * (safe * ((xs * xs + ys * ys) + zs * zs))
    return np.where(scale == 0.0, 0.0, out)


def _kinetic_from_velocity(rho, vx, vy, vz):
    """numerics/mhd_state.hpp:123-133 elementwise."""
    scale = np.fmax(np.abs(vx), np.fmax(np.abs(vy), np.abs(vz)))
    safe = np.where(scale == 0.0, 1.0, scale)
    xs, ys, zs = vx / safe, vy / safe, vz / safe
    q = np.sqrt(rho) * safe
    out = (0.5 * q) * (q * ((xs * xs + ys * ys) + zs * zs))
    return np.where(scale == 0.0, 0.0, out)


def _libm(fn, values: np.ndarray) -> np.ndarray:
    """The C library's function per element (the reference's device math is
    the correctly rounded libm result for sin/cos on these arguments)."""
    return np.array([fn(float(v)) for v in values])


def _primitives(deck: MhdDeck, ng: int):
    d, p, kind = deck.domain, deck.initial.params, deck.initial.type
    gamma = deck.numerics.gamma
    dx, dy = d.lx_m / d.nx, d.ly_m / d.ny
    xc1 = _centres(d.nx, ng, dx, d.origin_x_m)
    yc1 = _centres(d.ny, ng, dy, d.origin_y_m)
    shape = (yc1.size, xc1.size)
    X = np.broadcast_to(xc1[None, :], shape)
    Y = np.broadcast_to(yc1[:, None], shape)
    zero = np.zeros(shape)
    full = lambda v: np.full(shape, float(v))  # noqa: E731
    eoff = zero
    if kind == "brio_wu":
        left = np.array([float(p["left"][k]) for k in _PRIMITIVE_KEYS])
        right = np.array([float(p["right"][k]) for k in _PRIMITIVE_KEYS])
        side = X < float(p.get("interface", 0.5))
        w = [np.where(side, left[c], right[c]) for c in range(8)]
        rho, pr, vx, vy, vz, bx, by, bz = w
    elif kind == "alfven_wave":
        n = float(_exact_int(p.get("wavenumber", 1), "wavenumber"))
        amp = float(p.get("amplitude", 1.0e-6))
        rho0, p0, b0 = float(p.get("rho", 1.0)), float(p.get("p", 0.1)), float(p.get("b0", 1.0))
        mvs = 1.0 / SQRT_MU0 if deck.units == "SI" else 1.0
        k = 2.0 * math.pi * n / d.lx_m
        phase = k * (xc1 - d.origin_x_m)
        q = n / float(d.nx)
        fv = 1.0 if q == 0.0 else math.sin(math.pi * q) / (math.pi * q)
        inv = math.copysign(mvs, b0) / math.sqrt(rho0)
        s1, c1 = _libm(math.sin, phase), _libm(math.cos, phase)
        row = lambda a: np.broadcast_to(a[None, :], shape)  # noqa: E731
        rho, pr, vx = full(rho0), full(p0), zero
        vy = row(((-amp) * inv) * fv * s1)
        vz = row(((-amp) * inv) * fv * c1)
        bx = full(b0)
        by = row((amp * fv) * s1)
        bz = row((amp * fv) * c1)
        sa = amp * mvs
        eoff = full((sa * sa) * (1.0 - fv * fv))
    elif kind == "orszag_tang":
        two_pi = 2.0 * math.pi
        xi = (xc1 - d.origin_x_m) / d.lx_m
        eta = (yc1 - d.origin_y_m) / d.ly_m
        b0 = float(p.get("b0", 1.0))
        se = _libm(math.sin, two_pi * eta)
        sx = _libm(math.sin, two_pi * xi)
        s2x = _libm(math.sin, (2.0 * two_pi) * xi)
        rho, pr = full(gamma * gamma), full(gamma)
        vx = np.broadcast_to((-se)[:, None], shape)
        vy = np.broadcast_to(sx[None, :], shape)
        vz = zero
        bx = np.broadcast_to(((-b0) * se)[:, None], shape)
        by = np.broadcast_to((b0 * s2x)[None, :], shape)
        bz = zero
    elif kind == "blast":
        cx, cy = (float(v) for v in p.get("center", [0.0, 0.0]))
        r = np.hypot(X - cx, Y - cy)
        rho = full(p.get("rho_ambient", 1.0))
        pr = np.where(r < float(p.get("r_in", 0.1)), float(p.get("p_core", 10.0)),
                      float(p.get("p_ambient", 0.1)))
        vx = vy = vz = zero
        bx, by, bz = full(p.get("bx", 0.0)), full(p.get("by", 0.0)), full(p.get("bz", 0.0))
    elif kind == "rotor":
        cx, cy = (float(v) for v in p.get("center", [0.5, 0.5]))
        r0, r1 = float(p.get("r0", 0.1)), float(p.get("r1", 0.115))
        rin, rout = float(p.get("rho_in", 10.0)), float(p.get("rho_out", 1.0))
        u0 = float(p.get("u0", 2.0))
        rx, ry = X - cx, Y - cy
        r = np.hypot(rx, ry)
        f = np.fmin(np.fmax((r1 - r) / (r1 - r0), 0.0), 1.0)
        inside = r <= r0
        f = np.where(inside, 1.0, np.where(r >= r1, 0.0, f))
        taper = (~inside) & (r < r1)
        speed = np.where(inside, u0 / r0,
                         np.where(taper, (f * u0) / np.where(taper, r, 1.0), 0.0))
        rho = rout + f * (rin - rout)
        pr = full(p.get("p", 1.0))
        vx, vy, vz = (-speed) * ry, speed * rx, zero
        bx, by, bz = full(p.get("bx", 0.0)), full(p.get("by", 0.0)), full(p.get("bz", 0.0))
    else:  # confined_blob
        cx, cy = d.origin_x_m + 0.5 * d.lx_m, d.origin_y_m + 0.5 * d.ly_m
        half = float(p.get("blob_half", 0.25 * min(d.lx_m, d.ly_m)))
        inside = (np.abs(X - cx) <= half) & (np.abs(Y - cy) <= half)
        rho = np.where(inside, float(p.get("rho_in", 10.0)), float(p.get("rho_out", 1.0)))
        pr = np.where(inside, float(p.get("p_in", 1.0)), float(p.get("p_out", 0.1)))
        vx = vy = vz = bx = by = zero
        bz = full(p.get("bz", 0.1))
    return [np.ascontiguousarray(np.broadcast_to(a, shape), dtype=np.float64)
            for a in (rho, pr, vx, vy, vz, bx, by, bz, eoff)]


def build_initial_state_pass1(deck: MhdDeck, ng: int):
    """The seed kernel's first pass (mhd_initial_conditions.hip:211-271):
    conserved arrays with the raw magnetic half-norm in the energy, the
    magnetic components in the solver's B/sqrt(mu0) variable, and the raw
    half-norm itself.  Raises ValueError on the reference's seed errors."""
    rho, pr, vx, vy, vz, bx, by, bz, eoff = _primitives(deck, ng)
    gamma = deck.numerics.gamma
    if not (np.all(np.isfinite(rho)) and np.all(rho > 0.0)):
        raise ValueError("initial state must have strictly positive density everywhere")
    if not (np.all(np.isfinite(pr)) and np.all(pr > 0.0)):
        raise ValueError("initial state must have strictly positive gas pressure everywhere")
    kinetic = _kinetic_from_velocity(rho, vx, vy, vz)
    magnetic = _half_squared_norm3(bx, by, bz)
    energy = ((pr / (gamma - 1.0) + kinetic) + magnetic) + eoff
    mx, my, mz = rho * vx, rho * vy, rho * vz
    if not all(np.all(np.isfinite(m)) for m in (mx, my, mz, energy)):
        raise ValueError("initial state energy is not representable in float64")
    scale = 1.0 / SQRT_MU0 if deck.units == "SI" else 1.0
    state = {"rho": rho, "mx": mx, "my": my, "mz": mz, "energy": energy,
             "bx": scale * bx, "by": scale * by, "bz": scale * bz}
    return {k: v.reshape(-1) for k, v in state.items()}, magnetic.reshape(-1)


def build_initial_state(deck: MhdDeck, ng: int) -> dict:
    """{component: padded host array} as the reference's build_initial_state
    returns it: pass 1, then the energy re-formed from the collocated field
    (mhd_initial_conditions.hip:273-330) on the analytic (unfilled) arrays."""
    import torch
    from . import launch as L
    state, raw = build_initial_state_pass1(deck, ng)
    d = deck.domain
    grid = L.Grid(d.nx, d.ny, ng, d.lx_m / d.nx, d.ly_m / d.ny)
    dev = torch.device("cuda")
    faces = [torch.from_numpy(state[c]).to(dev) for c in ("bx", "by")]
    cells = [torch.empty_like(faces[0]) for _ in range(2)]
    for axis in range(2):
        L.collocate_face_to_cell(grid, axis, faces[axis], cells[axis])
    torch.cuda.synchronize()
    bxc, byc = (c.cpu().numpy() for c in cells)
    if not (np.all(np.isfinite(bxc)) and np.all(np.isfinite(byc))):
        raise ValueError("face-to-cell magnetic collocation is not representable")
    energy = (state["energy"] - raw) + _half_squared_norm3(bxc, byc, state["bz"])
    if not np.all(np.isfinite(energy)):
        raise ValueError("initial state energy is not representable in float64")
    state["energy"] = energy
    return state


# ---- run (python/quasar/mhd/cli.py:110-492) -------------------------------------
def _magnetic_to_output(value, units: str):
    arr = np.asarray(value, dtype=np.float64)
    return arr * SQRT_MU0 if units == "SI" else arr


def make_config(deck: MhdDeck) -> mhd.MhdConfig:
    cfg = mhd.MhdConfig()
    d = deck.domain
    cfg.grid = mhd.Grid2D(d.nx, d.ny, d.lx_m, d.ly_m, d.origin_x_m, d.origin_y_m)
    n = deck.numerics
    cfg.gamma, cfg.geometry, cfg.reconstruction = n.gamma, deck.geometry, n.reconstruction
    cfg.riemann, cfg.integrator, cfg.ct, cfg.positivity = n.riemann, n.integrator, n.ct, n.positivity
    cfg.rho_floor, cfg.p_floor, cfg.cfl = n.rho_floor, n.p_floor, n.cfl
    cfg.boundary = mhd.MhdBoundarySpec(list(deck.boundary.fluid), list(deck.boundary.field))
    return cfg


def prepare_run(deck: MhdDeck):
    """(solver, dt, dt_is_auto) as cli.py:110-161."""
    solver = mhd.MhdSolver2D(make_config(deck))
    ng = solver.grid().nghost
    for component, buf in build_initial_state(deck, ng).items():
        solver.seed_state(component, buf)
    cfl = solver.cfl_limit()
    if deck.time.dt_s == "auto":
        return solver, cfl, True
    dt = float(deck.time.dt_s)
    if dt > cfl:
        raise ValueError(f"time.dt_s ({dt:.6e}) exceeds the MHD CFL stability limit "
                         f"({cfl:.6e}) for this grid and seeded state; reduce dt_s or use "
                         "'auto'.")
    return solver, dt, False


def _padded(solver, deck: MhdDeck, component: str) -> np.ndarray:
    g = solver.grid()
    flat = np.asarray(solver.state_component_to_host(component))
    if component in ("bx", "by", "bz"):
        flat = _magnetic_to_output(flat, deck.units)
    return flat.reshape(deck.domain.ny + 2 * g.nghost, deck.domain.nx + 2 * g.nghost)


def _interior(solver, deck: MhdDeck, component: str) -> np.ndarray:
    g = solver.grid().nghost
    return _padded(solver, deck, component)[g:g + deck.domain.ny, g:g + deck.domain.nx]


def confine_output_path(directory: Path, relative: str) -> Path:
    """A relative output path that stays inside the deck's directory."""
    p = Path(relative)
    if p.is_absolute():
        raise ValueError("diagnostics.output_path must be relative to the deck")
    out = (Path(directory) / p).resolve()
    base = Path(directory).resolve()
    if base not in out.parents and out != base:
        raise ValueError("diagnostics.output_path must stay inside the deck's directory")
    return out


def run_loop(solver, deck: MhdDeck, dt: float, dt_is_auto: bool, out_path: Path,
             log_every: int = 0):
    """cli.py:386-492: the stepping policy, the diagnostics and the archive."""
    snapshots, divb_series, sim_time, t0 = [], [], 0.0, time.time()
    extra = {}
    if deck.initial.type == "orszag_tang":
        mass, energy = solver.conserved_cell_totals()
        extra = {"mass_initial": float(mass), "energy_initial": float(energy)}
    initial = {f"state_{c}_initial": _interior(solver, deck, c) for c in STATE_COMPONENTS}
    if deck.diagnostics.divb:
        divb_series.append(float(solver.divergence_b_max()))
    cadence, step, t_end = deck.diagnostics.cadence, 0, deck.time.t_end
    while step < deck.time.steps and (t_end is None or sim_time < float(t_end)):
        dt_limit = float(solver.cfl_limit()) if dt_is_auto else float(dt)
        if not np.isfinite(dt_limit) or not dt_limit > 0.0:
            raise RuntimeError("MHD timestep is not finite and strictly positive")
        dt_step, clipped = dt_limit, False
        if t_end is not None:
            remaining = float(t_end) - sim_time
            dt_step = min(dt_step, remaining)
            clipped = dt_step == remaining
        if not np.isfinite(dt_step) or not dt_step > 0.0:
            raise RuntimeError("MHD timestep cannot make positive finite progress")
        next_time = None
        if not clipped:
            next_time = sim_time + dt_step
            if not np.isfinite(next_time) or not next_time > sim_time:
                raise RuntimeError("MHD timestep is too small to advance simulation time")
        if dt_is_auto:
            solver.step_unchecked(dt_step)
        else:
            solver.step(dt_step)
        sim_time = float(t_end) if clipped else next_time
        step += 1
        last = step == deck.time.steps or (t_end is not None and sim_time >= float(t_end))
        on_cadence = cadence > 0 and step % cadence == 0
        need_divb = deck.diagnostics.divb and (
            on_cadence or last or (log_every > 0 and step % log_every == 0))
        divb_now = float(solver.divergence_b_max()) if need_divb else None
        if divb_now is not None:
            divb_series.append(divb_now)
        if on_cadence:
            snap = {"step": step, "time_s": sim_time,
                    "fields": {c: _interior(solver, deck, c) for c in deck.diagnostics.fields}}
            if deck.diagnostics.divb:
                snap["divb"] = divb_now
            snapshots.append(snap)
        if log_every > 0 and step % log_every == 0:
            elapsed = time.time() - t0
            rate = step / elapsed if elapsed > 0 else 0.0
            msg = f"step {step}/{deck.time.steps}  t={sim_time:.6e}  rate={rate:.0f} step/s"
            if deck.diagnostics.divb:
                msg += f"  |divB|inf={divb_now:.3e}"
            print(msg, flush=True)
    flat = {"final_step": np.array([step]), "final_time_s": np.array([sim_time]),
            "nx": np.array([deck.domain.nx]), "ny": np.array([deck.domain.ny]),
            "lx_m": np.array([deck.domain.lx_m]), "ly_m": np.array([deck.domain.ly_m]),
            "nghost": np.array([solver.grid().nghost]), "units": np.array([deck.units]),
            "geometry": np.array([deck.geometry]), "gamma": np.array([deck.numerics.gamma])}
    for c in STATE_COMPONENTS:
        flat[f"state_{c}"] = _interior(solver, deck, c)
    if deck.diagnostics.divb:
        out = _magnetic_to_output(np.asarray(divb_series, dtype=np.float64), deck.units)
        flat["divb_linf"] = out
        flat["divb_linf_final"] = np.array([out[-1]])
    if snapshots:
        flat["snapshot_steps"] = np.array([s["step"] for s in snapshots])
        flat["snapshot_times_s"] = np.array([s["time_s"] for s in snapshots])
        for c in deck.diagnostics.fields:
            flat[f"snapshot_state_{c}"] = np.stack([s["fields"][c] for s in snapshots])
        if deck.diagnostics.divb:
            flat["snapshot_divb_linf"] = _magnetic_to_output(
                np.array([s["divb"] for s in snapshots], dtype=np.float64), deck.units)
    for k, v in extra.items():
        flat[k] = np.array([v])
    flat.update(initial)
    with Path(out_path).open("wb") as stream:
        np.savez(stream, **flat)
    return step, sim_time


def run(input_deck, steps_override: int | None = None, verbose: bool = False,
        print_config: bool = False, log_every: int = 0):
    """cli.run for the serial path: returns (final_step, final_time, path)."""
    if steps_override is not None and (isinstance(steps_override, bool) or
                                       not isinstance(steps_override, int) or
                                       steps_override <= 0):
        raise ValueError("steps_override must be a positive integer")
    if isinstance(input_deck, MhdDeck):
        deck, deck_dir = input_deck, Path.cwd()
    else:
        deck_path = Path(input_deck).resolve()
        deck, deck_dir = load(deck_path), deck_path.parent
    if steps_override is not None:
        deck = copy.deepcopy(deck)
        deck.time = Time(dt_s=deck.time.dt_s, steps=steps_override, t_end=deck.time.t_end)
        deck.validate()
    solver, dt, auto = prepare_run(deck)
    if print_config:
        print(f"grid    : {deck.domain.nx}x{deck.domain.ny}  nghost={solver.grid().nghost}")
        print(f"schemes : recon={deck.numerics.reconstruction} riemann={deck.numerics.riemann}")
        print(f"initial : {deck.initial.type}")
        print(f"dt      : {dt:.6e}    steps: {deck.time.steps}")
    out = confine_output_path(deck_dir, deck.diagnostics.output_path)
    step, t = run_loop(solver, deck, dt, auto, out, log_every)
    if print_config or verbose:
        print(f"wrote   : {out}")
    return step, t, out


def main(argv: Sequence[str] | None = None) -> int:
    ap = argparse.ArgumentParser(prog="quasar-b200-mhd", description="B200 ideal-MHD driver.")
    sub = ap.add_subparsers(dest="command", required=True)
    r = sub.add_parser("run", help="Run an MHD simulation from a YAML deck.")
    r.add_argument("input")
    r.add_argument("--verbose", action="store_true")
    r.add_argument("--print-config", action="store_true")
    r.add_argument("--steps-override", type=int, default=None)
    r.add_argument("--log-every", type=int, default=0)
    a = ap.parse_args(argv)
    run(a.input, steps_override=a.steps_override, verbose=a.verbose,
        print_config=a.print_config, log_every=a.log_every)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
