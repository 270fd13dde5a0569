"""Algorithmic FLOP table of the MHD step, written to profiles/flop_counts.json
(read by bench.py for the roofline).  Test infrastructure: runs the counting
instance of the oracle restatement (oracle/mhd_oracle.cpp, Counted scalar).

    python oracle/count_flops.py [n] [steps]

Counting rules (oracle/oracle_count.hpp): add, sub, mul, div, sqrt = 1;
compare, min, max, abs = 0; the reference's exact-expansion sums count as
their plain products and sums.  Work the reference repeats counts once:
the face-to-cell collocation (once per padded cell per stage, not per load),
the face-EMF Riemann re-solve (not counted: it equals the flux solve) and the
CFL face rate (once per face, not once per adjacent cell).
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))
import mhd_cases as M  # noqa: E402

PHASES = ["collocation", "reconstruction", "face_flux", "cell_emf", "corner_emf", "update",
          "cfl_rate", "admissibility"]
WORKLOADS = {
    "rotor_mp7": (M.rotor, 7, M.OUTFLOW),
    "blast_mp7": (M.blast, 7, M.OUTFLOW),
    "orszag_tang_mp5": (M.orszag_tang, 5, M.PERIODIC),
    "orszag_tang_mp7": (M.orszag_tang, 7, M.PERIODIC),
}


def main(n=128, steps=3):
    O = M.OracleLib()
    table = {"rules": __doc__.split("Counting rules")[1].strip(), "n": n, "steps": steps,
             "phases": PHASES, "workloads": {}}
    for name, (ic, order, bc) in WORKLOADS.items():
        t0 = time.time()
        s = O.solver(n, n, order, bc=bc, counting=True)
        s.seed(ic(n, order=order))
        ph = O.count_phases(s, steps)
        s2 = O.solver(n, n, order, bc=bc, counting=True)
        s2.seed(ic(n, order=order))
        as_written, alg, cfl = O.count_flops(s2, steps)
        table["workloads"][name] = {
            "per_zone_step": {p: float(v) for p, v in zip(PHASES, ph)},
            "algorithmic_total": float(sum(ph)),
            "as_written_total": float(as_written),
        }
        print(f"{name}: algorithmic {sum(ph):.0f} flop/zone-step, as written {as_written:.0f} "
              f"({time.time() - t0:.1f}s)", flush=True)
    out = os.path.join(ROOT, "profiles", "flop_counts.json")
    with open(out, "w") as f:
        json.dump(table, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main(*(int(a) for a in sys.argv[1:3]))
