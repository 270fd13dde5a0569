"""The Python mirror of the reference's `_core.mhd` module
(bindings/python/bind_mhd.cpp): boundary-spec setters and getters, the
background spec, registry introspection and the halo/order helpers.  Host
logic only (no device calls)."""
import pytest

from quasar_b200 import mhd


def test_boundary_spec_setters_and_getters():
    b = mhd.MhdBoundarySpec()
    assert [b.fluid_side(s) for s in range(4)] == ["periodic"] * 4
    b.set_fluid_all("outflow")
    b.set_field_all("outflow")
    b.set_fluid_side(2, "wall")
    b.set_field_side(2, "wall")
    assert b.fluid == ["outflow", "outflow", "wall", "outflow"]
    assert b.field_side(2) == "wall" and b.field_side(3) == "outflow"
    for bad in (-1, 4):
        with pytest.raises(IndexError, match="side"):
            b.fluid_side(bad)
        with pytest.raises(IndexError, match="side"):
            b.set_field_side(bad, "wall")


def test_config_carries_background_and_timestep_signature():
    cfg = mhd.MhdConfig()
    assert cfg.timestep_signature == ""
    assert cfg.background.enabled is False and cfg.background.profile == "uniform"
    cfg.timestep_signature = "auto"
    cfg.background.enabled = True
    cfg.grid = mhd.Grid2D(16, 16, 1.0, 1.0)
    # refused before any device call
    with pytest.raises(ValueError, match="background"):
        mhd._native_config(cfg)


def test_registry_introspection_names_what_this_build_accepts():
    assert mhd.registered_reconstructions() == ["mp5", "mp7", "muscl_minmod"]
    assert mhd.registered_riemann_solvers() == ["hlld"]
    assert mhd.registered_integrators() == ["ssprk3"]
    assert mhd.registered_ct_schemes() == ["fd_ct_christlieb"]
    assert mhd.registered_positivity_limiters() == ["troubled_cell"]
    assert mhd.registered_mhd_fluid_boundaries() == ["outflow", "periodic", "wall"]
    assert mhd.registered_mhd_field_boundaries() == ["outflow", "periodic", "wall"]
    assert mhd.registered_mhd_background_profiles() == []
    from quasar_b200 import deck
    assert tuple(mhd.registered_initial_conditions()) == deck.INITIAL_TYPES
    # every accepted name passes the configuration check
    for rec in mhd.registered_reconstructions():
        for bc in mhd.registered_mhd_fluid_boundaries():
            cfg = mhd.MhdConfig()
            cfg.grid = mhd.Grid2D(16, 16, 1.0, 1.0)
            cfg.reconstruction = rec
            cfg.boundary.set_fluid_all(bc)
            cfg.boundary.set_field_all(bc)
            mhd._native_config(cfg)


def test_reconstruction_halo_and_order():
    assert [mhd.reconstruction_halo(n) for n in ("muscl_minmod", "mp5", "mp7")] == [2, 3, 4]
    assert [mhd.reconstruction_order(n) for n in ("muscl_minmod", "mp5", "mp7")] == [2, 5, 7]
    with pytest.raises(ValueError, match="unknown MHD reconstruction scheme 'weno5'"):
        mhd.reconstruction_halo("weno5")
