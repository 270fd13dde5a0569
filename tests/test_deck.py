"""Deck front end (quasar_b200/deck.py) on the CPU: the reference's deck
schema and its errors, and the first pass of the initial-state generators
against the reference's own seed (oracle/_ref, built from the reference's
sources) bit for bit.  The energy, which needs the collocation on the GPU,
and the full runs are in test_gpu_deck.py."""
import copy

import numpy as np
import pytest

import deck_cases as D
import mhd_cases as M
from quasar_b200 import deck as Q

ORDER = {"mp5": 5, "mp7": 7, "muscl_minmod": 2}


def test_decks_parse_and_defaults():
    for name, raw in D.decks().items():
        d = Q.parse(copy.deepcopy(raw))
        assert d.initial.type == name
        assert d.time.dt_s == "auto" and d.diagnostics.cadence == 4
    d = Q.parse({"domain": {"nx": 8, "ny": 8, "lx_m": 1.0, "ly_m": 1.0},
                 "initial": {"type": "orszag_tang"}})
    assert d.numerics.reconstruction == "mp7" and d.numerics.cfl == 0.4
    assert d.boundary.fluid == ("periodic",) * 4 and d.time.steps == 100
    assert d.diagnostics.fields == list(Q.STATE_COMPONENTS)


@pytest.mark.parametrize("mutate,match", [
    (lambda r: r.update(geometry="cylindrical"), "cylindrical"),
    (lambda r: r.update(background_field={"enabled": True, "bx0": 1.0}), "background_field"),
    (lambda r: r.update(bogus=1), "unknown key"),
    (lambda r: r["numerics"].update(gamma=1.0), "gamma"),
    (lambda r: r["initial"].update(type="tearing"), "initial.type"),
    (lambda r: r["initial"]["params"].update(extra=2), "unknown key"),
    (lambda r: r["boundary"].update(fluid="wall"), "periodicity must match"),
    (lambda r: r["boundary"].update(fluid="wall", field="outflow"), "match per side"),
    (lambda r: r["boundary"].update(fluid="axis", field="axis"), "not supported"),
    (lambda r: r["time"].update(steps=0), "time.steps"),
    (lambda r: r["diagnostics"].update(fields=["temperature"]), "diagnostics.fields"),
])
def test_deck_errors(mutate, match):
    raw = copy.deepcopy(D.decks()["orszag_tang"])
    mutate(raw)
    with pytest.raises(ValueError, match=match):
        Q.parse(raw)


def test_rotor_and_brio_wu_parameter_rules():
    raw = copy.deepcopy(D.decks()["rotor"])
    raw["initial"]["params"]["r1"] = 0.05
    with pytest.raises(ValueError, match="r1 must be greater"):
        Q.parse(raw)
    raw = copy.deepcopy(D.decks()["brio_wu"])
    raw["initial"]["params"]["right"]["bx"] = 0.5
    with pytest.raises(ValueError, match="continuous normal"):
        Q.parse(raw)


def test_output_path_is_confined(tmp_path):
    assert Q.confine_output_path(tmp_path, "a/out.npz") == (tmp_path / "a" / "out.npz").resolve()
    for bad in ("../out.npz", "/tmp/out.npz"):
        with pytest.raises(ValueError):
            Q.confine_output_path(tmp_path, bad)


@pytest.mark.skipif(not M.ref_available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("name", ["orszag_tang", "rotor", "blast", "brio_wu", "alfven_wave"])
@pytest.mark.parametrize("recon", ["mp5", "mp7"])
@pytest.mark.parametrize("units", ["normalized", "SI"])
def test_first_pass_matches_reference_seed_bitwise(ref, name, recon, units):
    """SI decks carry B in tesla: the seed scales it (and, for the Alfven
    wave, its velocity eigen-relation) by 1/sqrt(mu0)."""
    raw = copy.deepcopy(D.decks(recon=recon)[name])
    raw["units"] = units
    d = Q.parse(raw)
    ng = Q.nghost(recon)
    ours, _ = Q.build_initial_state_pass1(d, ng)
    dm = d.domain
    want = ref.initial_state(Q._KIND[name], dm.nx, dm.ny, dm.lx_m, dm.ly_m, dm.origin_x_m,
                             dm.origin_y_m, ng, d.numerics.gamma, ORDER[recon], **D.ref_params(d))
    for c, comp in enumerate(Q.STATE_COMPONENTS):
        if comp == "energy":
            continue  # re-formed from the collocated field: test_gpu_deck.py
        assert np.array_equal(ours[comp], want[c]), (name, comp)
