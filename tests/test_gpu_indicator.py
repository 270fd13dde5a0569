"""Tensor-core troubled-cell indicator against its numpy restatement
(oracle/mlp_oracle.py), through the C ABI."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


def random_rows(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((n, O.FEAT)) * 0.7).astype(np.float32)


@pytest.mark.parametrize("rows", [1, 127, 128, 1000, 40000])
def test_forward_matches_oracle(rows):
    from quasar_b200.indicator import TroubledCellIndicator
    ind = TroubledCellIndicator(seed=3)
    p = ind.params()
    rng = np.random.default_rng(4)
    p[O.HID * O.FEAT:O.HID * O.FEAT + O.HID] = rng.standard_normal(O.HID) * 0.1  # b1
    ind.set_params(p)
    x = random_rows(rows, rows)
    got = ind.forward(x)
    want, _ = O.forward(p, x)
    scale = np.max(np.abs(want)) + 1e-30
    assert np.max(np.abs(got - want)) <= 2e-3 * scale, np.max(np.abs(got - want)) / scale
