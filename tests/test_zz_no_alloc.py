"""Allocation-free conserved totals (qmhd_conserved_cell_totals_device).

Runs last (file name) so it is also exercised after every other GPU test has
used the device.  The entry point is called through the C ABI on device
copies of a solver's state and compared with qmhd_solver_conserved_cell_totals
on the same state, twice in a row.
"""
import ctypes

import numpy as np
import pytest

import mhd_cases as M

pytestmark = pytest.mark.gpu

REL = 1e-13  # both sides are compensated sums of the same cells


def _solver(n):
    from quasar_b200 import mhd
    cfg = mhd.MhdConfig()
    cfg.grid = mhd.Grid2D(n, n, 1.0, 1.0)
    cfg.reconstruction = "mp5"
    s = mhd.MhdSolver2D(cfg)
    for name, a in zip(M.COMPONENTS, M.orszag_tang(n, order=5)):
        s.seed_state(name, a)
    return s


def _device_totals(rho, energy, nx, ny, ng, stream=0):
    from quasar_b200 import _native
    L = _native.lib()
    m, e = ctypes.c_double(), ctypes.c_double()
    rc = L.qmhd_conserved_cell_totals_device(
        ctypes.c_void_p(rho.data_ptr()), ctypes.c_void_p(energy.data_ptr()), nx, ny, ng,
        ctypes.c_void_p(stream), ctypes.byref(m), ctypes.byref(e))
    return rc, m.value, e.value


def _close(a, b):
    return abs(a - b) <= REL * max(abs(a), abs(b))


@pytest.mark.parametrize("n", [64, 200])
def test_matches_solver_totals_on_two_consecutive_calls(n):
    import torch
    from quasar_b200 import _native
    s = _solver(n)
    ng = 3
    for step in range(3):
        ref = s.conserved_cell_totals()
        rho = torch.from_numpy(s.state_component_to_host("rho")).to("cuda:0")
        energy = torch.from_numpy(s.state_component_to_host("energy")).to("cuda:0")
        st = torch.cuda.Stream(device="cuda:0")
        st.wait_stream(torch.cuda.current_stream())
        first = _device_totals(rho, energy, n, n, ng, st.cuda_stream)
        second = _device_totals(rho, energy, n, n, ng, st.cuda_stream)
        for rc, m, e in (first, second):
            assert rc == _native.QMHD_OK, _native.lib().qmhd_last_error().decode()
            assert _close(m, ref[0]), (step, m, ref[0])
            assert _close(e, ref[1]), (step, e, ref[1])
        assert first == second
        s.step_unchecked(s.cfl_limit())


def test_default_stream_and_ragged_chunk():
    """A cell count that is not a multiple of the 8192-cell chunk, default stream."""
    import torch
    from quasar_b200 import _native
    nx, ny, ng = 131, 67, 2
    rng = np.random.default_rng(7)
    rho = rng.uniform(0.5, 2.0, (ny + 2 * ng) * (nx + 2 * ng))
    energy = rng.uniform(1.0, 3.0, rho.size)
    core = (slice(ng, ng + ny), slice(ng, ng + nx))
    want_m = float(np.sum(rho.reshape(ny + 2 * ng, nx + 2 * ng)[core], dtype=np.longdouble))
    want_e = float(np.sum(energy.reshape(ny + 2 * ng, nx + 2 * ng)[core], dtype=np.longdouble))
    dr = torch.from_numpy(rho).to("cuda:0")
    de = torch.from_numpy(energy).to("cuda:0")
    torch.cuda.synchronize()
    for _ in range(2):
        rc, m, e = _device_totals(dr, de, nx, ny, ng)
        assert rc == _native.QMHD_OK, _native.lib().qmhd_last_error().decode()
        assert _close(m, want_m) and _close(e, want_e), (m, want_m, e, want_e)


def test_rejects_sizes_beyond_the_scratch_and_host_pointers():
    import torch
    from quasar_b200 import _native
    L = _native.lib()
    d = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    side = 8193  # 8193 * 8192 cells is one row past QMHD_TOTALS_DEVICE_MAX_CELLS
    assert side * 8192 > _native.TOTALS_DEVICE_MAX_CELLS
    rc, _, _ = _device_totals(d, d, side, 8192, 0)
    assert rc == _native.QMHD_INVALID_ARGUMENT
    assert "scratch limit" in L.qmhd_last_error().decode()
    rc, _, _ = _device_totals(d, d, 0, 4, 0)
    assert rc == _native.QMHD_INVALID_ARGUMENT
    host = torch.zeros(16, dtype=torch.float64)
    rc, _, _ = _device_totals(host, host, 4, 4, 0)
    assert rc == _native.QMHD_INVALID_ARGUMENT
    assert "not device memory" in L.qmhd_last_error().decode()
    # the device is still usable after the rejected calls
    rc, m, _ = _device_totals(d, d, 4, 4, 0)
    assert rc == _native.QMHD_OK and m == 0.0
