"""Deck validation of quasar_b200.deck against the behaviour of the reference's
deck layer (python/quasar/mhd/io.py): the same decks are refused, with the
same kind of message, and the same decks pass.  Host logic only."""
import copy
import math

import pytest

from quasar_b200 import deck as Q


def _base():
    return {"units": "normalized", "geometry": "cartesian",
            "domain": {"nx": 8, "ny": 8, "lx_m": 1.0, "ly_m": 1.0},
            "numerics": {"gamma": 5.0 / 3.0},
            "initial": {"type": "orszag_tang", "params": {}},
            "time": {"dt_s": "auto", "steps": 2},
            "diagnostics": {"cadence": 0, "divb": True},
            "boundary": {"fluid": "periodic", "field": "periodic"},
            "background_field": {"enabled": False}}


def _set(path, value):
    def mutate(d):
        for k in path[:-1]:
            d = d[k]
        d[path[-1]] = value
    return mutate


_L = {"rho": 1.0, "p": 1.0, "vx": 0.0, "vy": 0.0, "vz": 0.0, "bx": 0.75, "by": 1.0, "bz": 0.0}
_R = dict(_L, rho=0.125, p=0.1, by=-1.0)
_TINY = float.fromhex("0x0.0000000000001p-1022")
_HUGE = float.fromhex("0x1.fffffffffffffp+1023")


def _collapse(d):
    # the last cell centre x0 + (nx - 1/2) dx rounds onto the upper bound
    d["domain"].update(nx=2, origin_x_m=float.fromhex("0x1.58be77ab34af0p-1002"),
                       lx_m=float.fromhex("0x0.0000000373a5dp-1022"))


REFUSED = [
    # boundaries
    (_set(["boundary"], {"fluid": "internal", "field": "internal"}), "reserved"),
    (_set(["boundary"], {"fluid": ["periodic", "outflow", "periodic", "periodic"],
                         "field": ["periodic", "outflow", "periodic", "periodic"]}), "both sides"),
    (_set(["boundary"], {"fluid": "periodic",
                         "field": ["outflow", "outflow", "periodic", "periodic"]}),
     "periodicity must match"),
    (_set(["boundary", "fluid"], {"x_low": "wall"}), "unknown key"),
    (_set(["boundary"], {"fluid": ["periodic", "outflow"], "field": "periodic"}), "four sides"),
    (_set(["boundary"], {"fluid": ["periodic", "reflecting", "periodic", "periodic"],
                         "field": "periodic"}), "not supported"),
    # unknown keys at every level
    (_set(["geometery"], "cylindrical"), "unknown key"),
    (_set(["domain", "nxx"], 16), "unknown key"),
    (_set(["numerics", "cfl_number"], 0.2), "unknown key"),
    (_set(["initial", "kind"], "rotor"), "unknown key"),
    (_set(["time", "step"], 10), "unknown key"),
    (_set(["diagnostics", "div_b"], True), "unknown key"),
    (_set(["boundary", "fields"], "wall"), "unknown key"),
    (_set(["background_field", "enable"], True), "unknown key"),
    (_set(["background_field", "enabled"], "yes"), "boolean"),
    # gamma and grid
    (_set(["numerics", "gamma"], 0.5), "gamma"),
    (_set(["numerics", "gamma"], 1.0), "gamma"),
    (_set(["numerics", "gamma"], math.nan), "gamma"),
    (_set(["domain", "nx"], 0), "positive"),
    (_set(["domain", "nx"], -8), "positive"),
    (_set(["domain", "nx"], 8.0), "integer"),
    (_set(["domain", "nx"], 8.5), "integer"),
    (_set(["domain", "nx"], True), "integer"),
    (_set(["domain", "nx"], 1 << 17), "<="),
    (_set(["domain", "ny"], 0), "positive"),
    (_set(["domain", "lx_m"], 0.0), "lx_m"),
    (_set(["domain", "ly_m"], math.inf), "ly_m"),
    (lambda d: d["domain"].update(origin_x_m=_HUGE, lx_m=_HUGE), "upper x bound"),
    (lambda d: d["domain"].update(nx=2, lx_m=_TINY), "x spacing"),
    (_collapse, "coordinates collapse"),
    # scheme names against the registry queries
    (_set(["numerics", "reconstruction"], "weno5"), "numerics.reconstruction"),
    (_set(["numerics", "riemann"], "roe"), "numerics.riemann"),
    (_set(["numerics", "integrator"], "rk4"), "numerics.integrator"),
    (_set(["numerics", "ct"], "gardiner"), "numerics.ct"),
    (_set(["numerics", "positivity"], "none"), "numerics.positivity"),
    # initial conditions
    (_set(["initial", "type"], "not_a_real_ic"), "initial.type"),
    (_set(["initial"], {"type": "alfven_wave", "params": {"wavenumber": 1.0}}), "integer"),
    (_set(["initial"], {"type": "alfven_wave", "params": {"wavenumber": 1.5}}), "integer"),
    (_set(["initial"], {"type": "alfven_wave", "params": {"wavenumber": True}}), "integer"),
    (_set(["initial"], {"type": "alfven_wave", "params": {"b0": 0.0}}), "nonzero"),
    (_set(["initial"], {"type": "alfven_wave", "params": {"b0": 1.0, "wavenumber": 0}}),
     "wavenumber"),
    (_set(["initial"], {"type": "alfven_wave", "params": {"b0": 1.0, "wavenumber": 8}}),
     "Nyquist"),
    (_set(["initial"], {"type": "alfven_wave", "params": {"rho": 0.0, "p": 1.0}}), "rho"),
    (_set(["initial"], {"type": "alfven_wave", "params": {"rho": 1.0, "p": 0.0}}), "p must"),
    (_set(["initial"], {"type": "brio_wu", "params": {"interface": 0.5}}), "left"),
    (_set(["initial"], {"type": "brio_wu", "params": {"interface": 0.5, "left": [1.0, 2.0],
                                                      "right": _R}}), "mapping"),
    (_set(["initial"], {"type": "brio_wu", "params": {"interface": math.nan, "left": _L,
                                                      "right": _R}}), "interface"),
    (_set(["initial"], {"type": "brio_wu", "params": {"interface": 0.5, "left": _L,
                                                      "right": dict(_R, bx=0.5)}}),
     "continuous normal"),
    (_set(["initial"], {"type": "blast", "params": {"center": [0.0], "r_in": 0.1}}), "center"),
    (_set(["initial"], {"type": "blast", "params": {"center": [0.0, 0.0], "r_in": 0.0}}),
     "r_in"),
    (_set(["initial"], {"type": "rotor", "params": {"r0": 0.0, "r1": 0.2}}), "r0"),
    (_set(["initial"], {"type": "rotor", "params": {"r0": 0.2, "r1": 0.2}}), "r1"),
    (_set(["initial"], {"type": "rotor", "params": {"center": [0.0, math.inf]}}), "center"),
    (_set(["initial"], {"type": "confined_blob", "params": {"blob_half": 0.0}}), "blob_half"),
    # time and diagnostics
    (_set(["time", "steps"], 0), "steps"),
    (_set(["time", "steps"], 5.0), "integer"),
    (_set(["time", "steps"], True), "integer"),
    (_set(["time", "dt_s"], "fast"), "dt_s"),
    (_set(["time", "dt_s"], -1.0e-3), "dt_s"),
    (_set(["diagnostics", "output_path"], ""), "output_path"),
    (_set(["diagnostics", "output_path"], "   "), "output_path"),
    (_set(["diagnostics", "output_path"], 123), "output_path"),
    (_set(["diagnostics", "cadence"], -1), "cadence"),
    (_set(["diagnostics", "cadence"], 1.0), "integer"),
    (_set(["diagnostics", "divb"], "false"), "divb"),
]


@pytest.mark.parametrize("mutate,match", REFUSED)
def test_refused_like_the_reference(mutate, match):
    d = _base()
    mutate(d)
    with pytest.raises(ValueError, match=match):
        Q.parse(d)


@pytest.mark.parametrize("mutate", [
    lambda d: None,
    _set(["numerics", "gamma"], 1.4),
    _set(["time", "dt_s"], 1.0e6),  # no CFL check before a solver exists
    _set(["boundary"], {"fluid": ["outflow", "outflow", "wall", "wall"],
                        "field": ["outflow", "outflow", "wall", "wall"]}),
    _set(["boundary"], {"fluid": {"x_lo": "outflow", "x_hi": "outflow", "y_lo": "periodic",
                                  "y_hi": "periodic"},
                        "field": ["outflow", "outflow", "periodic", "periodic"]}),
    _set(["background_field"], {"enabled": False, "profile": "uniform", "bx0": 2.0}),
])
def test_accepted_like_the_reference(mutate):
    d = _base()
    mutate(d)
    deck = Q.parse(copy.deepcopy(d))
    assert deck.domain.nx == 8


def test_boundary_forms_map_to_four_sides():
    d = _base()
    d["boundary"] = {"fluid": ["wall", "wall", "periodic", "periodic"],
                     "field": ["wall", "wall", "periodic", "periodic"]}
    deck = Q.parse(d)
    assert tuple(deck.boundary.fluid) == ("wall", "wall", "periodic", "periodic")
    d = _base()
    d["boundary"] = {"fluid": "outflow", "field": "outflow"}
    assert tuple(Q.parse(d).boundary.field) == ("outflow",) * 4
    d = _base()
    del d["boundary"]
    assert tuple(Q.parse(d).boundary.fluid) == ("periodic",) * 4


def test_duplicate_yaml_keys_are_refused(tmp_path):
    p = tmp_path / "deck.yaml"
    p.write_text("units: normalized\nunits: normalized\n")
    with pytest.raises(ValueError, match=r"duplicate YAML key 'units'.*line 2"):
        Q.load(p)
    p.write_text("domain: {nx: 8, ny: 8, lx_m: 1.0, ly_m: 1.0}\n"
                 "initial: {type: orszag_tang}\n")
    assert Q.load(p).domain.nx == 8
