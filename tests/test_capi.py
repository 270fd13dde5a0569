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
    launch = declared_symbols("quasar_mhd_launch.h")
    assert set(launch) == set(_native.LAUNCH_EXPORTS)
    assert all(hasattr(lib, s) for s in launch)


def test_launch_interface_names_every_reference_seam_entry():
    # kernels.hpp entry points of the Cartesian, zero-background hot path
    want = ("reconstruct", "hlld_flux", "flux_difference", "ct_emf_prepare", "ct_emf_finish",
            "emf_curl_rate", "rk_stage", "admissible_fraction", "cfl_max_rate", "ct_divb_linf",
            "ct_divb_relative_linf", "fill_ghosts_fluid", "fill_ghosts_field",
            "collocate_face_to_cell", "conserved_cell_sums", "seed_initial_state")
    assert set("qmhd_launch_" + w for w in want) == set(declared_symbols("quasar_mhd_launch.h"))


def test_launch_interface_rejects_bad_arguments_before_any_launch():
    """Host-side validation (null device pointers throughout, so nothing could
    be launched even if a check were missing)."""
    import pytest
    from quasar_b200 import launch as L
    g = L.Grid(16, 16, 4, 1 / 16, 1 / 16)
    u, iface = L.Field(), L.Iface()
    per = L.flags((0, 0, 0, 0))
    with pytest.raises(ValueError, match="dir"):
        L.reconstruct(g, u, None, None, 2, iface, 7, per, 5 / 3, stream=0)
    with pytest.raises(ValueError, match="nghost"):
        L.reconstruct(g, u, None, None, 0, iface, 5, per, 5 / 3, stream=0)
    with pytest.raises(ValueError, match="periodic"):
        L.reconstruct(g, u, None, None, 0, iface, 7, L.flags((0, 1, 0, 0)), 5 / 3, stream=0)
    with pytest.raises(ValueError, match="boundary flag"):
        L.hlld_flux(g, iface, 0, u, L.flags((3, 3, 0, 0)), 5 / 3, 7, stream=0)
    with pytest.raises(ValueError, match="gamma"):
        L.hlld_flux(g, iface, 0, u, per, 1.0, 7, stream=0)
    with pytest.raises(ValueError, match="null"):
        L.hlld_flux(g, iface, 0, u, per, 5 / 3, 7, stream=0)
    with pytest.raises(ValueError, match="null"):
        L.flux_difference(g, u, 0, u, stream=0)
    import ctypes
    from quasar_b200 import _native
    lib = _native.lib()
    with pytest.raises(ValueError, match="side"):
        _native.check(lib.qmhd_launch_fill_ghosts_fluid(ctypes.byref(g), ctypes.byref(u), 5, 0,
                                                        None))
    with pytest.raises(ValueError, match="mode"):
        _native.check(lib.qmhd_launch_fill_ghosts_field(ctypes.byref(g), ctypes.byref(u), 1, 3,
                                                        None))
    with pytest.raises(ValueError, match="nghost must be"):
        L.collocate_face_to_cell(L.Grid(16, 16, 6, 1 / 16, 1 / 16), 0, None, None, stream=0)
    with pytest.raises(ValueError, match="scratch"):
        L.ct_divb_linf(g, u, None, stream=0)
    with pytest.raises(ValueError, match="cylindrical"):
        _native.check(lib.qmhd_launch_flux_difference(ctypes.byref(g), ctypes.byref(u), 0,
                                                      ctypes.byref(u), None, 1))
    # rate_only is accepted (same states as the reference): the call gets as
    # far as the scratch check
    with pytest.raises(ValueError, match="collocation scratch"):
        _native.check(lib.qmhd_launch_reconstruct(ctypes.byref(g), ctypes.byref(u), None, None, 0,
                                                  ctypes.byref(iface), 7, per, 5 / 3, None, 1))
    spec = L.IcSpec()
    spec.kind, spec.gamma, spec.magnetic_scale, spec.lx, spec.ly = 9, 5 / 3, 1.0, 1.0, 1.0
    seed = lambda: _native.check(lib.qmhd_launch_seed_initial_state(  # noqa: E731
        ctypes.byref(g), ctypes.byref(spec), ctypes.byref(u), None, None, None, None, None))
    with pytest.raises(ValueError, match="kind"):
        seed()
    spec.kind, spec.gamma = 2, 1.0
    with pytest.raises(ValueError, match="gamma"):
        seed()
    spec.gamma, spec.magnetic_scale = 5 / 3, 0.0
    with pytest.raises(ValueError, match="magnetic unit scale"):
        seed()
    spec.magnetic_scale = 1.0
    with pytest.raises(ValueError, match="null scratch or status"):
        seed()
    with pytest.raises(ValueError, match="ownership"):
        _native.check(lib.qmhd_launch_hlld_flux(ctypes.byref(g), ctypes.byref(iface), 0,
                                                ctypes.byref(u), per, 5 / 3, None, 0, 7,
                                                L.flags((1, 0, 1, 1))))
    with pytest.raises(ValueError, match="hll_only"):
        _native.check(lib.qmhd_launch_hlld_flux(ctypes.byref(g), ctypes.byref(iface), 0,
                                                ctypes.byref(u), per, 5 / 3, None, 1, 7, None))


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


def test_seam_build_loads_and_reports_a_missing_device_as_the_reference_does():
    """oracle/_ref/libquasar_mhd_seam.so (the reference's own MhdSolver2D
    linked over this library's launch interface) loads, binds every
    kernels.hpp entry point at link time, and without a GPU its solver
    constructor fails with the reference's DeviceError text instead of
    crashing."""
    import pytest
    import torch
    import mhd_cases as M
    so = os.path.join(ROOT, "oracle", "_ref", "libquasar_mhd_seam.so")
    if not os.path.exists(so):
        pytest.skip("seam build absent (oracle/build_seam.sh)")
    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU tests cover the seam")
    lib = M.RefLib(so)
    with pytest.raises(RuntimeError, match="device error"):
        lib.solver(16, 16, 5)


def test_seam_and_cpu_reference_builds_load_into_one_process():
    """Both builds carry the reference's registry singletons and register the
    same factory names at load time.  The seam library keeps its copies
    local, so loading it after the CPU build (as the GPU tests do) must not
    end the process with a duplicate-registration error.  Run in a child
    process, since that error aborts."""
    import subprocess
    import sys
    import pytest
    seam = os.path.join(ROOT, "oracle", "_ref", "libquasar_mhd_seam.so")
    cpu = os.path.join(ROOT, "oracle", "_ref", "libquasar_mhd_ref.so")
    if not (os.path.exists(seam) and os.path.exists(cpu)):
        pytest.skip("reference builds absent (oracle/build_ref.sh, oracle/build_seam.sh)")
    code = ("import ctypes; ctypes.CDLL(%r); ctypes.CDLL(%r); print('both loaded')" % (cpu, seam))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "both loaded" in r.stdout
