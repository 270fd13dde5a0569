"""The C-ABI library loads and exports every entry point include/quasar_mhd.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(header="quasar_mhd.h"):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qmhd_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_solver_surface():
    syms = declared_symbols()
    for name in ("qmhd_solver_create", "qmhd_solver_seed_state", "qmhd_solver_cfl_limit",
                 "qmhd_solver_step_unchecked", "qmhd_solver_state_component_to_host",
                 "qmhd_solver_divergence_b_max", "qmhd_solver_conserved_cell_totals"):
        assert name in syms


def test_library_exports_every_declared_symbol():
    from quasar_b200 import _native
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(_native.EXPORTS)
    batch = declared_symbols("quasar_mhd_batch.h")
    assert set(batch) == set(_native.BATCH_EXPORTS)
    assert all(hasattr(lib, s) for s in batch)
    ind = declared_symbols("quasar_mhd_indicator.h")
    assert set(ind) == set(_native.INDICATOR_EXPORTS)
    assert all(hasattr(lib, s) for s in ind)
    ext = declared_symbols("quasar_mhd_ext.h")
    assert set(ext) == set(_native.EXT_EXPORTS)
    assert all(hasattr(lib, s) for s in ext)


def test_python_config_validation_matches_reference_errors():
    import pytest
    from quasar_b200 import mhd
    cfg = mhd.MhdConfig()
    cfg.reconstruction = "weno5"
    with pytest.raises(ValueError):
        mhd._native_config(cfg)
    cfg = mhd.MhdConfig()
    cfg.riemann = "hll"
    with pytest.raises(ValueError):
        mhd._native_config(cfg)
    cfg = mhd.MhdConfig()
    cfg.boundary.fluid = ["periodic", "outflow", "periodic", "periodic"]
    cfg.boundary.field = list(cfg.boundary.fluid)
    c = mhd._native_config(cfg)  # the periodic pairing is checked natively
    assert list(c.boundary) == [0, 1, 0, 0]
