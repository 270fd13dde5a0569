"""ctypes view of the per-kernel launch interface (include/quasar_mhd_launch.h):
the C ABI of the reference's MHD backend seam
(include/quasar/physics/mhd/kernels.hpp), one function per launch_mhd_* entry
point, with the reference's argument order.

Device arrays are CUDA float64 tensors in the padded layout
(nx + 2 nghost) x (ny + 2 nghost); torch only allocates them and supplies the
stream.  Every call runs kernels of the in-tree library and raises ValueError
or RuntimeError on a failed status, as the reference's binding does.
"""
from __future__ import annotations

import ctypes

from . import _native

_vp, _i, _d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double


class Grid(ctypes.Structure):
    """Grid2D: extents, ghost width and spacings."""
    _fields_ = [("nx", _i), ("ny", _i), ("nghost", _i), ("dx", _d), ("dy", _d)]


class Field(ctypes.Structure):
    """MhdField2D: rho, mx, my, mz, energy, bx_face, by_face, bz_cell."""
    _fields_ = [("comp", _vp * 8)]


class Iface(ctypes.Structure):
    """MhdInterfaceStates of one direction."""
    _fields_ = [("left", _vp * 8), ("right", _vp * 8)]


class Emf(ctypes.Structure):
    """Face E_z and no-jump proofs per direction, cell and corner E_z."""
    _fields_ = [("face_ez_x", _vp), ("face_ez_y", _vp), ("no_jump_x", _vp), ("no_jump_y", _vp),
                ("cell_ez", _vp), ("corner_ez", _vp)]


class CflRate(ctypes.Structure):
    """ScaledCflRate: true max rate = scaled_max_rate / rate_scale."""
    _fields_ = [("scaled_max_rate", _d), ("rate_scale", _d)]


class IcSpec(ctypes.Structure):
    """MhdInitialConditionSpec, Cartesian fields (kind 0 brio_wu, 1 alfven_wave,
    2 orszag_tang, 3 blast, 4 rotor, 5 confined_blob)."""
    _fields_ = [("kind", _i), ("lx", _d), ("ly", _d), ("origin_x", _d), ("origin_y", _d),
                ("gamma", _d), ("magnetic_scale", _d), ("interface_x", _d),
                ("left", _d * 8), ("right", _d * 8),
                ("rho", _d), ("pressure", _d), ("b0", _d), ("total_b0", _d), ("amplitude", _d),
                ("wavenumber", ctypes.c_longlong), ("magnetic_velocity_scale", _d),
                ("b_uniform", _d * 3), ("center", _d * 2),
                ("r_in", _d), ("r0", _d), ("r1", _d), ("rho_in", _d), ("rho_out", _d),
                ("p_in", _d), ("p_out", _d), ("p_core", _d), ("p_ambient", _d),
                ("rho_ambient", _d), ("u0", _d), ("blob_half", _d)]


_P = ctypes.POINTER
_flags = _P(_i)


def declare(L) -> None:
    """argtypes of the launch entry points (called by _native.lib())."""
    g, f, v, e = _P(Grid), _P(Field), _P(Iface), _P(Emf)
    L.qmhd_launch_reconstruct.argtypes = [g, f, _vp, _vp, _i, v, _i, _flags, _d, _vp, _i]
    L.qmhd_launch_hlld_flux.argtypes = [g, v, _i, f, _flags, _d, _vp, _i, _i, _flags]
    L.qmhd_launch_flux_difference.argtypes = [g, f, _i, f, _vp, _i]
    L.qmhd_launch_ct_emf_prepare.argtypes = [g, f, _vp, _vp, v, v, _flags, e, _d, _vp, _i, _i]
    L.qmhd_launch_ct_emf_finish.argtypes = [g, _flags, e, _vp, _i, _i]
    L.qmhd_launch_emf_curl_rate.argtypes = [g, e, f, _vp, _i]
    L.qmhd_launch_rk_stage.argtypes = [g, f, f, f, f, _d, _d, _d, _vp]
    L.qmhd_launch_admissible_fraction.argtypes = [g, f, f, _d, _d, _d, _vp, _P(_d), _vp, _i]
    L.qmhd_launch_cfl_max_rate.argtypes = [g, v, v, _d, _vp, _P(CflRate), _vp, _i, _i, _flags]
    L.qmhd_launch_ct_divb_linf.argtypes = [g, f, _vp, _P(_d), _vp, _i]
    L.qmhd_launch_ct_divb_relative_linf.argtypes = [g, f, _vp, _P(_d), _vp, _i, _i]
    L.qmhd_launch_fill_ghosts_fluid.argtypes = [g, f, _i, _i, _vp]
    L.qmhd_launch_fill_ghosts_field.argtypes = [g, f, _i, _i, _vp]
    L.qmhd_launch_collocate_face_to_cell.argtypes = [g, _i, _vp, _vp, _vp]
    L.qmhd_launch_conserved_cell_sums.argtypes = [g, f, _i, _vp, _P(_d), _P(_d)]
    L.qmhd_launch_seed_initial_state.argtypes = [g, _P(IcSpec), f, _vp, _vp, _vp, _vp, _vp]


def _ptr(t) -> int | None:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    assert t.is_cuda and t.is_contiguous(), "device arrays are contiguous CUDA tensors"
    return t.data_ptr()


def field(arrays) -> Field:
    return Field((_vp * 8)(*[_ptr(a) for a in arrays]))


def iface(left, right) -> Iface:
    return Iface((_vp * 8)(*[_ptr(a) for a in left]), (_vp * 8)(*[_ptr(a) for a in right]))


def emf(face_ez_x, face_ez_y, no_jump_x, no_jump_y, cell_ez, corner_ez) -> Emf:
    return Emf(*[_ptr(a) for a in (face_ez_x, face_ez_y, no_jump_x, no_jump_y, cell_ez, corner_ez)])


def flags(modes) -> ctypes.Array:
    return (_i * 4)(*modes)


def _stream(stream):
    if stream is not None:
        return stream
    import torch
    return torch.cuda.current_stream().cuda_stream


def reconstruct(grid, u, cell_bx, cell_by, dir, out, order, bflags, gamma, stream=None):
    _native.check(_native.lib().qmhd_launch_reconstruct(
        ctypes.byref(grid), ctypes.byref(u), _ptr(cell_bx), _ptr(cell_by), dir, ctypes.byref(out),
        order, bflags, gamma, _stream(stream), 0))


def hlld_flux(grid, iface_states, dir, flux_out, bflags, gamma, order, stream=None):
    _native.check(_native.lib().qmhd_launch_hlld_flux(
        ctypes.byref(grid), ctypes.byref(iface_states), dir, ctypes.byref(flux_out), bflags, gamma,
        _stream(stream), 1 if order <= 1 else 0, order, None))


def flux_difference(grid, flux, dir, dudt, stream=None):
    _native.check(_native.lib().qmhd_launch_flux_difference(
        ctypes.byref(grid), ctypes.byref(flux), dir, ctypes.byref(dudt), _stream(stream), 0))


def ct_emf_prepare(grid, u, cell_bx, cell_by, ifx, ify, bflags, table, gamma, order, stream=None):
    _native.check(_native.lib().qmhd_launch_ct_emf_prepare(
        ctypes.byref(grid), ctypes.byref(u), _ptr(cell_bx), _ptr(cell_by), ctypes.byref(ifx),
        ctypes.byref(ify), bflags, ctypes.byref(table), gamma, _stream(stream), order,
        1 if order <= 1 else 0))


def ct_emf_finish(grid, bflags, table, order, stream=None):
    _native.check(_native.lib().qmhd_launch_ct_emf_finish(
        ctypes.byref(grid), bflags, ctypes.byref(table), _stream(stream), order, 0))


def emf_curl_rate(grid, table, dudt, stream=None):
    _native.check(_native.lib().qmhd_launch_emf_curl_rate(
        ctypes.byref(grid), ctypes.byref(table), ctypes.byref(dudt), _stream(stream), 0))


def rk_stage(grid, out, un, ustage, dudt, a, b, c_dt, stream=None):
    _native.check(_native.lib().qmhd_launch_rk_stage(
        ctypes.byref(grid), ctypes.byref(out), ctypes.byref(un), ctypes.byref(ustage),
        ctypes.byref(dudt), a, b, c_dt, _stream(stream)))


def admissible_fraction(grid, base, candidate, rho_floor, p_floor, gamma, scratch,
                        collocation_order=0, stream=None) -> float:
    theta = ctypes.c_double()
    _native.check(_native.lib().qmhd_launch_admissible_fraction(
        ctypes.byref(grid), ctypes.byref(base), ctypes.byref(candidate), rho_floor, p_floor, gamma,
        _ptr(scratch), ctypes.byref(theta), _stream(stream), collocation_order))
    return theta.value


def cfl_max_rate(grid, ifx, ify, gamma, scratch, order, bflags, stream=None) -> CflRate:
    rate = CflRate()
    _native.check(_native.lib().qmhd_launch_cfl_max_rate(
        ctypes.byref(grid), ctypes.byref(ifx), ctypes.byref(ify), gamma, _ptr(scratch),
        ctypes.byref(rate), _stream(stream), order, 0, bflags))
    return rate


def ct_divb_linf(grid, u, scratch, stream=None) -> float:
    out = ctypes.c_double()
    _native.check(_native.lib().qmhd_launch_ct_divb_linf(
        ctypes.byref(grid), ctypes.byref(u), _ptr(scratch), ctypes.byref(out), _stream(stream), 0))
    return out.value


def ct_divb_relative_linf(grid, u, scratch, solver_owned=False, stream=None) -> float:
    out = ctypes.c_double()
    _native.check(_native.lib().qmhd_launch_ct_divb_relative_linf(
        ctypes.byref(grid), ctypes.byref(u), _ptr(scratch), ctypes.byref(out), _stream(stream), 0,
        1 if solver_owned else 0))
    return out.value


def fill_ghosts(grid, u, modes, stream=None) -> None:
    """The solver's closure (mhd_solver.cpp:627-631): per side, fluid then field."""
    L = _native.lib()
    for side in range(4):
        _native.check(L.qmhd_launch_fill_ghosts_fluid(ctypes.byref(grid), ctypes.byref(u), side,
                                                      modes[side], _stream(stream)))
        _native.check(L.qmhd_launch_fill_ghosts_field(ctypes.byref(grid), ctypes.byref(u), side,
                                                      modes[side], _stream(stream)))


def collocate_face_to_cell(grid, axis, face, cell, stream=None) -> None:
    _native.check(_native.lib().qmhd_launch_collocate_face_to_cell(
        ctypes.byref(grid), axis, _ptr(face), _ptr(cell), _stream(stream)))


def conserved_cell_sums(grid, u, stream=None) -> tuple[float, float]:
    m, e = ctypes.c_double(), ctypes.c_double()
    _native.check(_native.lib().qmhd_launch_conserved_cell_sums(
        ctypes.byref(grid), ctypes.byref(u), 0, _stream(stream), ctypes.byref(m), ctypes.byref(e)))
    return m.value, e.value


def seed_initial_state(grid, spec, out, raw_magnetic, cell_bx, cell_by, status,
                       stream=None) -> None:
    """launch_mhd_seed_initial_state; status: a device int32 tensor the
    caller zeroes and reads back (the reference's kMhdSeed* bits)."""
    _native.check(_native.lib().qmhd_launch_seed_initial_state(
        ctypes.byref(grid), ctypes.byref(spec), ctypes.byref(out), _ptr(raw_magnetic),
        _ptr(cell_bx), _ptr(cell_by), _ptr(status), _stream(stream)))
