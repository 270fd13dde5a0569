"""Deck dictionaries in the reference's YAML schema (python/quasar/mhd/io.py)
for the five Cartesian, zero-background initial-state generators, at small
sizes, and their parameters lowered for the reference's own seed
(oracle/ref_capi.cpp qref_initial_state)."""
import math


def decks(n=24, recon="mp5"):
    base = lambda init, gamma=5.0 / 3.0, bc="periodic", nx=n, ny=n, ox=0.0, oy=0.0, units="normalized": {  # noqa: E731
        "units": units, "geometry": "cartesian",
        "domain": {"nx": nx, "ny": ny, "lx_m": 1.0, "ly_m": 1.0, "origin_x_m": ox, "origin_y_m": oy},
        "numerics": {"gamma": gamma, "reconstruction": recon, "riemann": "hlld",
                     "integrator": "ssprk3", "ct": "fd_ct_christlieb", "positivity": "troubled_cell",
                     "cfl": 0.3},
        "initial": init,
        "time": {"dt_s": "auto", "steps": 12},
        "diagnostics": {"output_path": "out.npz", "cadence": 4, "divb": True},
        "boundary": {"fluid": bc, "field": bc}}
    left = {"rho": 1.0, "p": 1.0, "vx": 0.0, "vy": 0.0, "vz": 0.0, "bx": 0.75, "by": 1.0, "bz": 0.0}
    right = {"rho": 0.125, "p": 0.1, "vx": 0.0, "vy": 0.0, "vz": 0.0, "bx": 0.75, "by": -1.0, "bz": 0.0}
    return {
        "orszag_tang": base({"type": "orszag_tang", "params": {"b0": 1.0}}),
        "rotor": base({"type": "rotor", "params": {"center": [0.5, 0.5], "r0": 0.1, "r1": 0.115,
                                                   "rho_in": 10.0, "rho_out": 1.0, "u0": 2.0,
                                                   "p": 1.0, "bx": 5.0 / math.sqrt(4 * math.pi)}},
                      gamma=1.4, bc="outflow"),
        "blast": base({"type": "blast", "params": {"center": [0.5, 0.5], "r_in": 0.1,
                                                   "p_core": 10.0, "p_ambient": 0.1,
                                                   "bx": 1.0 / math.sqrt(2), "by": 1.0 / math.sqrt(2)}},
                      bc="outflow"),
        "brio_wu": base({"type": "brio_wu", "params": {"interface": 0.5, "left": left,
                                                       "right": right}},
                        gamma=2.0, bc={"x_lo": "outflow", "x_hi": "outflow", "y_lo": "periodic",
                                       "y_hi": "periodic"}, ny=8),
        "alfven_wave": base({"type": "alfven_wave", "params": {"rho": 1.0, "p": 0.1, "b0": 1.0,
                                                               "amplitude": 1e-6, "wavenumber": 1}},
                            ny=8, ox=-0.25, oy=0.5),
    }


def ref_params(deck):
    """The reference's spec scalars for a parsed deck (io.py:922-995)."""
    p, t = deck.initial.params, deck.initial.type
    # SI decks give B in tesla and the solver evolves B / sqrt(mu0)
    inv_sqrt_mu0 = 1.0 / math.sqrt(4.0e-7 * math.pi) if deck.units == "SI" else 1.0
    out = {"magnetic_scale": inv_sqrt_mu0}
    if t == "brio_wu":
        keys = ("rho", "p", "vx", "vy", "vz", "bx", "by", "bz")
        out["interface"] = float(p.get("interface", 0.5))
        for k, key in enumerate(keys):
            out[f"left_{k}"] = float(p["left"][key])
            out[f"right_{k}"] = float(p["right"][key])
    elif t == "alfven_wave":
        out.update(rho=float(p.get("rho", 1.0)), pressure=float(p.get("p", 0.1)),
                   b0=float(p.get("b0", 1.0)), total_b0=float(p.get("b0", 1.0)),
                   amplitude=float(p.get("amplitude", 1e-6)),
                   wavenumber=float(p.get("wavenumber", 1)),
                   magnetic_velocity_scale=inv_sqrt_mu0)
    elif t == "orszag_tang":
        out.update(bx=float(p.get("b0", 1.0)))
    elif t == "blast":
        c = p.get("center", [0.0, 0.0])
        out.update(cx=float(c[0]), cy=float(c[1]), rho_ambient=float(p.get("rho_ambient", 1.0)),
                   p_ambient=float(p.get("p_ambient", 0.1)), p_core=float(p.get("p_core", 10.0)),
                   r_in=float(p.get("r_in", 0.1)), bx=float(p.get("bx", 0.0)),
                   by=float(p.get("by", 0.0)), bz=float(p.get("bz", 0.0)))
    elif t == "rotor":
        c = p.get("center", [0.5, 0.5])
        out.update(cx=float(c[0]), cy=float(c[1]), r0=float(p.get("r0", 0.1)),
                   r1=float(p.get("r1", 0.115)), rho_in=float(p.get("rho_in", 10.0)),
                   rho_out=float(p.get("rho_out", 1.0)), u0=float(p.get("u0", 2.0)),
                   p_ambient=float(p.get("p", 1.0)), bx=float(p.get("bx", 0.0)),
                   by=float(p.get("by", 0.0)), bz=float(p.get("bz", 0.0)))
    return out
