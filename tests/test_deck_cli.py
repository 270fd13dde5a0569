"""The deck CLI's run loop and exit behaviour against those of the
reference's (python/quasar/mhd/cli.py): time accounting with a stand-in
solver, divergence diagnostics switched off, the archive path, and invalid
decks refused before any stepping or output.  Host logic only."""
import math
import subprocess
import sys

import numpy as np
import pytest
import yaml

from quasar_b200 import deck as Q


class _Grid:
    nghost = 0


class _Solver:
    """Just enough of MhdSolver2D for the run loop: scripted CFL limits."""

    def __init__(self, nx, ny, limits):
        self._state = np.zeros(nx * ny)
        self._limits = iter(limits)
        self.dts = []
        self.divergence_calls = 0

    def grid(self):
        return _Grid()

    def state_component_to_host(self, _component):
        return self._state.copy()

    def divergence_b_max(self):
        self.divergence_calls += 1
        return 0.0

    def cfl_limit(self):
        return next(self._limits)

    def step_unchecked(self, dt):
        self.dts.append(float(dt))

    def step(self, dt):
        self.dts.append(float(dt))


def _deck(t_end, steps=8, divb=True, cadence=0, output_path="out.npz"):
    return Q.parse({"domain": {"nx": 2, "ny": 2, "lx_m": 1.0, "ly_m": 1.0},
                    "initial": {"type": "blast", "params": {}},
                    "time": {"dt_s": "auto", "steps": steps, "t_end": t_end},
                    "diagnostics": {"output_path": output_path, "cadence": cadence,
                                    "fields": [], "divb": divb}})


def test_endpoint_is_the_exact_sum_of_the_steps_taken(tmp_path):
    # 0.3 is not a multiple of binary64 0.1: the last step is the exact
    # floating residual and the archived time is t_end itself
    solver = _Solver(2, 2, [0.1] * 4)
    Q.run_loop(solver, _deck(0.3), 0.1, True, tmp_path / "out.npz")
    with np.load(tmp_path / "out.npz") as out:
        final = float(np.asarray(out["final_time_s"]).ravel()[0])
    assert len(solver.dts) == 3
    assert solver.dts[-1] == 0.3 - (solver.dts[0] + solver.dts[1])
    assert math.fsum(solver.dts) == 0.3 and final == 0.3


def test_unrepresentable_time_progress_raises(tmp_path):
    solver = _Solver(2, 2, [1.0e16, 0.5])
    with pytest.raises(RuntimeError, match="too small to advance"):
        Q.run_loop(solver, _deck(2.0e16), 1.0e16, True, tmp_path / "out.npz")
    assert solver.dts == [1.0e16]


def test_divergence_off_means_no_reductions_and_no_keys(tmp_path):
    solver = _Solver(2, 2, [0.1, 0.1])
    Q.run_loop(solver, _deck(0.2, steps=2, divb=False, cadence=1), 0.1, True,
               tmp_path / "out.npz", log_every=1)
    with np.load(tmp_path / "out.npz") as out:
        assert not [k for k in out.files if "divb" in k]
    assert solver.divergence_calls == 0


def test_suffixless_output_path_is_used_exactly(tmp_path):
    solver = _Solver(2, 2, [0.1, 0.1])
    Q.run_loop(solver, _deck(0.2, steps=2, output_path="result"), 0.1, True,
               tmp_path / "result")
    assert (tmp_path / "result").exists() and not (tmp_path / "result.npz").exists()


@pytest.mark.parametrize("section,key,value", [
    ("numerics", "gamma", 0.5), ("numerics", "reconstruction", "nope"),
    ("domain", "nx", 0), ("initial", "type", "not_a_real_ic")])
def test_invalid_deck_exits_nonzero_before_output(tmp_path, section, key, value):
    data = {"domain": {"nx": 16, "ny": 16, "lx_m": 1.0, "ly_m": 1.0},
            "numerics": {"gamma": 5.0 / 3.0, "reconstruction": "mp5"},
            "initial": {"type": "orszag_tang"},
            "time": {"dt_s": "auto", "steps": 2},
            "diagnostics": {"output_path": "out.npz"}}
    data[section][key] = value
    path = tmp_path / "deck.yaml"
    path.write_text(yaml.safe_dump(data))
    res = subprocess.run([sys.executable, "-m", "quasar_b200.deck", "run", str(path)],
                         capture_output=True, text=True, timeout=300,
                         cwd=str(__import__("pathlib").Path(Q.__file__).parents[1]))
    assert res.returncode != 0
    text = (res.stdout + res.stderr).lower()
    assert "no module named" not in text and "valueerror" in text
    assert not (tmp_path / "out.npz").exists()
