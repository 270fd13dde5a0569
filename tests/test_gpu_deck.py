"""Deck runs on the GPU (quasar_b200/deck.py): the full initial state,
energy re-formed from the collocated field included, against the reference's
own seed (oracle/_ref), and a deck run through the CLI loop against the
reference's solver seeded with its own initial state and stepped with its
own dt."""
import copy

import numpy as np
import pytest
import yaml

import deck_cases as D
import mhd_cases as M
from quasar_b200 import deck as Q

pytestmark = pytest.mark.gpu
ORDER = {"mp5": 5, "mp7": 7}


def _ref_state(ref, d, recon):
    dm = d.domain
    return ref.initial_state(Q._KIND[d.initial.type], dm.nx, dm.ny, dm.lx_m, dm.ly_m,
                             dm.origin_x_m, dm.origin_y_m, Q.nghost(recon), d.numerics.gamma,
                             ORDER[recon], **D.ref_params(d))


@pytest.mark.parametrize("name", ["orszag_tang", "rotor", "blast", "brio_wu", "alfven_wave"])
@pytest.mark.parametrize("recon", ["mp5", "mp7"])
@pytest.mark.parametrize("units", ["normalized", "SI"])
def test_initial_state_matches_reference_seed(ref, name, recon, units):
    raw = copy.deepcopy(D.decks(recon=recon)[name])
    raw["units"] = units
    d = Q.parse(raw)
    ours = Q.build_initial_state(d, Q.nghost(recon))
    want = _ref_state(ref, d, recon)
    for c, comp in enumerate(Q.STATE_COMPONENTS):
        assert np.array_equal(ours[comp], want[c]), (name, comp,
                                                     float(np.max(np.abs(ours[comp] - want[c]))))


@pytest.mark.parametrize("name,recon", [("orszag_tang", "mp5"), ("rotor", "mp7"),
                                        ("brio_wu", "mp5")])
def test_deck_run_matches_reference_solver(ref, tmp_path, name, recon):
    raw = copy.deepcopy(D.decks(n=32, recon=recon)[name])
    path = tmp_path / "input.yaml"
    path.write_text(yaml.safe_dump(raw))
    steps, t, out = Q.run(path, steps_override=6)
    z = np.load(out)
    assert steps == 6 and int(z["final_step"][0]) == 6 and out.parent == tmp_path
    d = Q.parse(raw)
    dm, ng = d.domain, Q.nghost(recon)
    bc = tuple({"periodic": 0, "outflow": 1, "wall": 2}[s] for s in d.boundary.fluid)
    s = ref.solver(dm.nx, dm.ny, ORDER[recon], gamma=d.numerics.gamma, cfl=d.numerics.cfl, bc=bc,
                   ox=dm.origin_x_m, oy=dm.origin_y_m)
    sl = (slice(ng, ng + dm.ny), slice(ng, ng + dm.nx))
    shape = (dm.ny + 2 * ng, dm.nx + 2 * ng)
    s.seed([a.reshape(shape) for a in _ref_state(ref, d, recon)])
    init = [np.asarray(a).reshape(shape) for a in s.read()]
    for c in (0, 1, 2, 3, 4, 7):
        comp = Q.STATE_COMPONENTS[c]
        assert np.array_equal(z[f"state_{comp}_initial"], init[c][sl]), comp
    time_ref = 0.0
    for _ in range(6):
        dt = s.cfl()
        s.step(dt)
        time_ref += dt
    assert abs(float(z["final_time_s"][0]) - time_ref) <= 1e-13 * time_ref
    got = [np.asarray(a).reshape(shape) for a in s.read()]
    for c in (0, 1, 2, 3, 4, 7):
        comp = Q.STATE_COMPONENTS[c]
        a, b = z[f"state_{comp}"], got[c][sl]
        scale = max(float(np.sum(np.abs(b))), 1e-300)
        assert float(np.sum(np.abs(a - b))) / scale <= 1e-12 or float(np.max(np.abs(a - b))) <= 1e-14, comp
    assert z["divb_linf"].shape == (1 + 6 // 4 + 1,) and float(z["divb_linf_final"][0]) <= 1e-12
    assert z["snapshot_steps"].tolist() == [4] and z["snapshot_state_rho"].shape == (1, dm.ny, dm.nx)
    if name == "orszag_tang":
        assert "mass_initial" in z and "energy_initial" in z


def test_explicit_dt_above_cfl_limit_fails_before_output(tmp_path):
    """An explicit dt far above the CFL limit passes deck validation (no
    solver exists there) and is refused by the solver's checked step before
    any archive is written, as in the reference's CLI."""
    data = copy.deepcopy(D.decks(16, "mp5")["orszag_tang"])
    data["time"]["dt_s"] = 1.0e6
    path = tmp_path / "deck.yaml"
    path.write_text(yaml.safe_dump(data))
    with pytest.raises(ValueError, match="CFL"):
        Q.run(str(path))
    assert not (tmp_path / "out.npz").exists()
