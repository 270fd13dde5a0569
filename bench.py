#!/usr/bin/env python
"""Benchmark: MHD zone-updates/s of the plain FP64 step on one B200.

Workload (default): MHD rotor, 4096^2, MP7 + HLLD + upwind CT, SSP-RK3,
outflow boundaries, gamma 5/3, CFL 0.4 (capped to 0.2 by the MP limiter as in
the reference); seeded synthetic analytic initial state.  One step = one
auto-dt SSP-RK3 step (cfl_limit + step), dt kept on the device.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--case rotor|blast]
                    [--n 4096] [--impl b200|reference]

N > 1 (torchrun, one process per GPU): the headline single-instance step
runs as N independent replicas (it is not domain-decomposed here); the batched
lines split their independent instances over the ranks, zones balanced
(quasar_b200/shard.py), with no data-path exchange.  Either way the value is
the zone-updates summed over ranks over the time taken as the max over ranks.

Printed JSON line: value = device-timed zone-updates/s with the state resident
in HBM; e2e = the same metric through the public C ABI with host buffers
(seed from pinned host memory, per-step cfl_limit read-back, final state read
back); roofline = the reconstruction kernel (the largest share of the step)
against the FP64 FMA peak measured on the same GPU; cpu_baseline = the
reference's own MHD path built for the CPU, on a bounded sample.
Beside the plain line: `learned` = the same workload with the shipped
troubled-cell indicator (quasar_b200/data/indicator_mp{5,7}.npz), its speed-up
and the density L1 gap to the plain run after the same steps; `batched` = 256
seeded independent MP5 instances on uneven grids stepped together, against
the same instances stepped one after another, and (`batched.learned`) batched
with the shipped MP5 indicator, with its density L1 gap to the plain batch;
`batched_learned` = one batch of Orszag-Tang 8192^2 MP7 and 64 rotor/blast
instances, plain and then learned (--no-learned / --no-batch skip them).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
WORLD = int(os.environ.get("WORLD_SIZE", "1"))
RANK = int(os.environ.get("RANK", "0"))
LOCAL_RANK = int(os.environ.get("LOCAL_RANK", "0"))

def pin_rank_device(env, local_rank):
    """One GPU per rank: the solver library carries its own CUDA runtime and
    uses device 0 of what it sees, so narrow CUDA_VISIBLE_DEVICES to this
    rank's GPU (the local_rank-th listed one, or local_rank itself when the
    variable is unset) before any CUDA initialisation in this process."""
    listed = [d for d in env.get("CUDA_VISIBLE_DEVICES", "").split(",") if d.strip()]
    if "CUDA_VISIBLE_DEVICES" not in env:
        env["CUDA_VISIBLE_DEVICES"] = str(local_rank)
    elif local_rank < len(listed):
        env["CUDA_VISIBLE_DEVICES"] = listed[local_rank].strip()


if WORLD > 1:
    pin_rank_device(os.environ, LOCAL_RANK)
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PHASES = ["control", "reconstruction", "face_flux", "cell_emf", "corner_emf", "update",
          "ghost_fill", "collocation"]
# kernels per auto-dt step: step_begin, 2 reconstruct, 2 face_flux, cell_emf,
# corner_emf, dt | stage 0 update, 2 ghost, colloc_check | 2 x (2 reconstruct,
# 2 face_flux, cell_emf, corner_emf, update, 2 ghost, colloc_check) | step_end
LAUNCHES_PER_STEP = 8 + 4 + 2 * 10 + 1
CPU_SAMPLE_N = 512  # side of the CPU baseline's sample of the workload
FLOP_PHASE = {"reconstruction": "reconstruction", "face_flux": "face_flux", "cell_emf": "cell_emf",
              "corner_emf": "corner_emf", "update": "update", "collocation": "collocation"}


# ---------------------------------------------------------------------------
def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--case", default="rotor", choices=["rotor", "blast"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--order", type=int, default=7, choices=[5, 7])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-indicator run")
    ap.add_argument("--no-batch", action="store_true", help="skip the 256-instance batched run")
    ap.add_argument("--no-other", action="store_true", help="skip the second single-instance case")
    return ap.parse_args()


class Dist:
    """Barrier and max/sum over ranks (gloo on host scalars)."""

    def __init__(self):
        self.pg = None
        if WORLD > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if WORLD > 1:
            self.dist.barrier()

    def reduce(self, x, op):
        if WORLD == 1:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if WORLD > 1:
            self.dist.destroy_process_group()


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during a region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        dev = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
        rows = [l.split(", ") for l in self.lines if l]
        rows = [r for r in rows if len(r) >= 9 and (r[0] == dev or not dev.isdigit())]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows)}


# ---------------------------------------------------------------------------
def reference_cpu(case, order, steps, warmup, n=CPU_SAMPLE_N):
    """The reference's own MHD path built for the CPU (oracle/_ref), all host
    threads, on an n^2 sample of the workload; falls back to the oracle port.
    Per-zone cost is size-independent on the GPU but not on the CPU (it rises
    with n up to a few hundred: thread blocks amortise better), so the
    baseline is sampled at 512^2, the largest size whose steps stay within
    seconds, and reported per zone."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import mhd_cases as M
    from quasar_b200 import ics
    ic = ics.GENERATORS[case](n, order=order)
    bc = (1, 1, 1, 1)
    if M.ref_available():
        lib, kind = M.RefLib(), "reference"
    else:
        lib, kind = M.OracleLib(), "port"
    s = lib.solver(n, n, order, bc=bc)
    s.seed(ic)
    for _ in range(warmup):
        s.step(s.cfl())
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step(s.cfl())
    wall = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": n * n * steps / wall, "unit": "zone-updates/s", "cores": cores, "kind": kind,
            "sample": f"{case} {n}^2 MP{order} outflow, {warmup} untimed + {steps} timed steps "
                      f"(cfl_limit + step_unchecked), {cores} OpenMP threads; per-zone rate "
                      f"extrapolated to the workload's size"}


def workload_config(a):
    """The `config` object both arms report."""
    return {"workload": f"{a.case} {a.n}^2 MP{a.order}+HLLD+upwind CT, SSP-RK3, outflow, "
                        "gamma 5/3, CFL 0.4 (0.2 effective)",
            "n": a.n, "order": a.order, "parallelism": f"replicas x{WORLD}",
            "l2": "state 1 GB+ per register, larger than L2"}


def run_reference_arm(a):
    if RANK != 0:
        return
    steps, warmup = max(1, min(a.steps, 3)), max(0, min(a.warmup, 1))
    cpu = reference_cpu(a.case, a.order, steps, warmup)
    line = {"impl": "reference", "metric": "MHD zone-updates/s (plain FP64 step)",
            "value": cpu["value"], "unit": "zone-updates/s", "n_gpus": a.gpus, "steps": steps,
            "warmup": warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(a), sample_n=CPU_SAMPLE_N,
                           sample=f"each step a {CPU_SAMPLE_N}^2 instance of the workload on the "
                                  "host cores (per-zone rate)"),
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def make_solver(a):
    from quasar_b200 import mhd
    cfg = mhd.MhdConfig()
    cfg.grid = mhd.Grid2D(a.n, a.n, 1.0, 1.0)
    cfg.reconstruction = "mp7" if a.order == 7 else "mp5"
    cfg.boundary = mhd.MhdBoundarySpec(["outflow"] * 4, ["outflow"] * 4)
    return mhd.MhdSolver2D(cfg)


def make_batch(insts, order):
    from quasar_b200 import mhd
    cfgs = []
    for x in insts:
        c = mhd.MhdConfig()
        c.grid = mhd.Grid2D(x["nx"], x["ny"], x["lx"], x["ly"])
        c.reconstruction = "mp7" if order == 7 else "mp5"
        c.gamma = x["gamma"]
        side = "periodic" if x["bc"] == 0 else "outflow"
        c.boundary = mhd.MhdBoundarySpec([side] * 4, [side] * 4)
        cfgs.append(c)
    b = mhd.MhdBatch2D(cfgs)
    for i, x in enumerate(insts):
        for name, arr in zip(ics_components(), x["arrays"]()):
            b.instance(i).seed_state(name, arr)
    return b


def sequential_instances(insts, steps):
    """Each instance alone, one after another: its own solver's device-timed
    auto-dt graph loop over `steps` steps after 3 warm-up steps.  Returns
    (summed device ms, zone-updates)."""
    import ctypes

    from quasar_b200 import _native, mhd
    L = _native.lib()
    ms, done = ctypes.c_double(), ctypes.c_int()
    total_ms, zu = 0.0, 0
    for x in insts:
        c = mhd.MhdConfig()
        c.grid = mhd.Grid2D(x["nx"], x["ny"], x["lx"], x["ly"])
        c.reconstruction = "mp5"
        c.gamma = x["gamma"]
        side = "periodic" if x["bc"] == 0 else "outflow"
        c.boundary = mhd.MhdBoundarySpec([side] * 4, [side] * 4)
        s = mhd.MhdSolver2D(c)
        for name, arr in zip(ics_components(), x["arrays"]()):
            s.seed_state(name, arr)
        for k in (3, steps):
            _native.check(L.qmhd_solver_time_auto_steps(s._h, k, ctypes.byref(ms), ctypes.byref(done)))
            if done.value != k:
                raise RuntimeError(f"sequential instance stopped after {done.value} of {k} steps")
        total_ms += ms.value
        zu += x["nx"] * x["ny"] * steps
        del s
    return total_ms, zu


def ics_components():
    from quasar_b200.ics import COMPONENTS
    return COMPONENTS


def seed(s, comps):
    from quasar_b200.ics import COMPONENTS
    for name, arr in zip(COMPONENTS, comps):
        s.seed_state(name, arr)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference_arm(a)
        return
    import ctypes

    from quasar_b200 import _native, ics
    L = _native.lib()
    dist = Dist()
    comps = ics.GENERATORS[a.case](a.n, order=a.order)
    s = make_solver(a)
    seed(s, comps)
    ms, done = ctypes.c_double(), ctypes.c_int()

    def timed(k):
        _native.check(L.qmhd_solver_time_auto_steps(s._h, k, ctypes.byref(ms), ctypes.byref(done)))
        if done.value != k:
            raise RuntimeError(f"device loop stopped after {done.value} of {k} steps")
        return ms.value

    timed(max(a.warmup, 3))
    dist.barrier()
    clocks = Clocks()
    clocks.start()
    t_ms = timed(a.steps)
    clk = clocks.stop()
    dist.barrier()
    t_ms = dist.reduce(t_ms, "max")
    zones = a.n * a.n
    value = zones * a.steps * WORLD / (t_ms * 1e-3)

    # per-phase device times of one step, for the roofline
    ph = (ctypes.c_double * 8)()
    _native.check(L.qmhd_solver_profile_step(s._h, ph, 8))
    phase_ms = dict(zip(PHASES, list(ph)))
    peak = ctypes.c_double()
    _native.check(L.qmhd_fp64_fma_peak(ctypes.byref(peak)))
    flops = {}
    fpath = os.path.join(ROOT, "profiles", "flop_counts.json")
    if os.path.exists(fpath):
        table = json.load(open(fpath))["workloads"].get(f"{a.case}_mp{a.order}", {})
        flops = table.get("per_zone_step", {})
    dom = "reconstruction"
    achieved = flops.get(dom, 0.0) * zones / (phase_ms[dom] * 1e-3) / 1e12 if phase_ms[dom] > 0 else None
    step_flops = sum(flops.values()) if flops else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        tt = json.load(open(tpath)).get(f"{a.case}_mp{a.order}_reconstruction")
        if tt:  # DRAM bytes of one reconstruction launch (6 launches per step)
            traffic = tt["bytes_per_zone_step"] / 6.0 * zones
    roofline = {"bound": "fp64", "kernel": "k_reconstruct (x and y, 3 stages; achieved over "
                                          "the phase, traffic per launch)",
                "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": (achieved / peak.value) if achieved else None, "traffic": traffic,
                "peak_source": "FP64 FMA probe on this GPU (qmhd_fp64_fma_peak); "
                               "MEASURED_PEAKS.json holds no FP64 figure",
                "step_flop_per_zone": step_flops,
                "step_achieved_tflops": (step_flops * value / WORLD / 1e12) if step_flops else None,
                "phase_ms_per_step": {k: round(v, 4) for k, v in phase_ms.items()}}

    div_b = {"max": s.divergence_b_max(), "rel": s.divergence_b_relative()}

    # the other single-instance workload of the benchmark configuration
    # (blast beside rotor, same size and order), plain step
    other = None
    if not a.no_other:
        oc = "blast" if a.case == "rotor" else "rotor"
        # the blast's first steps take positivity retries, which the
        # graph-only timing loop stops on: run the device-resident loop with
        # its retry controller (advance_auto) and time it on the host clock
        so = make_solver(a)
        seed(so, ics.GENERATORS[oc](a.n, order=a.order))
        t_sim, _ = so.advance_auto(0.0, float("inf"), max(a.warmup, 3))
        dist.barrier()
        w0 = time.perf_counter()
        t_sim, taken = so.advance_auto(t_sim, float("inf"), a.steps)
        to = dist.reduce((time.perf_counter() - w0) * 1e3, "max")
        other = {"workload": f"{oc} {a.n}^2 MP{a.order}, outflow, same step as the headline",
                 "value": zones * taken * WORLD / (to * 1e-3), "unit": "zone-updates/s",
                 "ms_per_step": to / max(taken, 1), "steps": taken, "t": t_sim,
                 "how": "advance_auto (device-resident graph steps plus the positivity "
                        "controller's retries), host wall clock after warm-up",
                 "div_b": {"max": so.divergence_b_max(), "rel": so.divergence_b_relative()}}
        del so

    # end to end through the public API with host buffers
    e2e = None
    if not a.no_e2e:
        import torch
        pinned = []
        for arr in comps:
            t = torch.empty(arr.size, dtype=torch.float64, pin_memory=True)
            t.numpy()[:] = arr.reshape(-1)
            pinned.append(t)
        out = [torch.empty(arr.size, dtype=torch.float64, pin_memory=True) for arr in comps]
        s2 = make_solver(a)
        names = ics.COMPONENTS
        k_e2e = a.steps
        dist.barrier()
        t0 = time.perf_counter()
        for name, t in zip(names, pinned):
            _native.check(L.qmhd_solver_seed_state(s2._h, name.encode(), t.data_ptr(), t.numel()))
        dt = ctypes.c_double()
        for _ in range(k_e2e):
            _native.check(L.qmhd_solver_cfl_limit(s2._h, ctypes.byref(dt)))
            _native.check(L.qmhd_solver_step_unchecked(s2._h, dt.value))
        for name, t in zip(names, out):
            _native.check(L.qmhd_solver_state_component_to_host(s2._h, name.encode(), t.data_ptr(),
                                                                t.numel()))
        wall = time.perf_counter() - t0
        wall = dist.reduce(wall, "max")
        bytes_state = sum(arr.nbytes for arr in comps)
        e2e = {"value": zones * k_e2e * WORLD / wall, "unit": "zone-updates/s",
               "h2d_bytes_per_step": bytes_state / k_e2e,
               "d2h_bytes_per_step": bytes_state / k_e2e + 8,
               "how": "seed_state x8 from pinned host once, then per step cfl_limit (8-byte dt "
                      "read back) + step_unchecked, then state_component_to_host x8 once: the "
                      "state crosses PCIe once each way per run of K steps (the reference CLI's "
                      "seed-once, step-many use), so the per-step bytes are the state / K; "
                      "host wall clock"}
        del s2

    # the same workload with the learned troubled-cell indicator (shipped
    # weights), from the same initial state and for the same number of steps,
    # with the density L1 gap to the plain run
    learned = None
    if not a.no_learned:
        from quasar_b200 import train_indicator
        from quasar_b200.indicator import learned_face_counts
        ind, thr = train_indicator.load(order=a.order)
        s3 = make_solver(a)
        seed(s3, comps)
        ind.attach(s3, thr)

        def timed3(k):
            _native.check(L.qmhd_solver_time_auto_steps(s3._h, k, ctypes.byref(ms), ctypes.byref(done)))
            if done.value != k:
                raise RuntimeError(f"learned loop stopped after {done.value} of {k} steps")
            return ms.value

        timed3(max(a.warmup, 3))
        dist.barrier()
        tl = dist.reduce(timed3(a.steps), "max")
        ph3 = (ctypes.c_double * 8)()
        _native.check(L.qmhd_solver_profile_step(s3._h, ph3, 8))  # matches the profiled plain step
        fx, fy = learned_face_counts(s3)
        nfaces = (a.n + 1) * (a.n + 2 * ics.nghost(a.order))
        r_plain = s.state_component_to_host("rho")
        r_learn = s3.state_component_to_host("rho")
        l1 = float(np.sum(np.abs(r_learn - r_plain)) / np.sum(np.abs(r_plain)))
        learned = {"value": zones * a.steps * WORLD / (tl * 1e-3), "unit": "zone-updates/s",
                   "ms_per_step": tl / a.steps, "speedup_vs_plain": t_ms / tl,
                   "phase_ms_per_step": {k: round(v, 4) for k, v in zip(PHASES, list(ph3))},
                   "phase_note": "control holds the indicator inference and the face lists",
                   "indicator": f"quasar_b200/data/indicator_mp{a.order}.npz",
                   "threshold": thr, "full_path_face_fraction": (fx + fy) / (2.0 * nfaces),
                   "rho_l1_vs_plain": l1, "steps_compared": max(a.warmup, 3) + a.steps + 1,
                   "div_b_max": s3.divergence_b_max(), "div_b_max_plain": s.divergence_b_max(),
                   "div_b_rel": s3.divergence_b_relative(),
                   "div_b_rel_plain": s.divergence_b_relative(),
                   "div_b_rel_note": "max|div B| dx / max|B_face|, the reference's own measure "
                                     "(bound 1e-11 in its example tests)"}
        del s3

    # batched steps: the 256-instance MP5 batch (plain), and the combined
    # batch (OT 8192^2 MP7 + 64 rotor/blast instances) plain then learned
    batched = combined = None
    if not a.no_batch:
        kb = max(10, a.steps // 10)
        from quasar_b200 import shard
        every = ics.batch_instances(count=256, seed=0, order=5)
        # instance-parallel over the ranks: each steps its share, no exchange
        insts = shard.rank_share(every, [x["nx"] * x["ny"] for x in every], RANK, WORLD)
        b = make_batch(insts, 5)
        ctas, trials = b.autotune()
        b.time_steps(3)
        bms, bzu = b.time_steps(kb)
        bms, bzu = dist.reduce(bms, "max"), dist.reduce(bzu, "sum")
        seq_ms, seq_zu = sequential_instances(insts, kb)
        seq_ms, seq_zu = dist.reduce(seq_ms, "max"), dist.reduce(seq_zu, "sum")
        batched = {"workload": "256 seeded MP5 instances, sides log-uniform in [64, 512], "
                               "Orszag-Tang / oblique Brio-Wu / linear fast or Alfven waves",
                   "zones": sum(x["nx"] * x["ny"] for x in every),
                   "value": bzu / (bms * 1e-3), "unit": "zone-updates/s",
                   "parallelism": f"instance-parallel over {WORLD} rank(s), zones balanced "
                                  "(quasar_b200/shard.py); zone-updates summed, time max",
                   "ms_per_step": bms / kb, "autotuned_ctas_per_sm": ctas,
                   "autotune_steps": trials,
                   "sequential": {"value": seq_zu / (seq_ms * 1e-3),
                                  "ms_per_step": seq_ms / kb,
                                  "how": "the same instances stepped one after another, each "
                                         "its own solver's device-resident graph loop of the "
                                         "same steps, device times summed"},
                   "batch_over_sequential": (bzu / bms) / (seq_zu / seq_ms)}
        if not a.no_learned:
            # the same instances batched in learned mode (shipped MP5
            # indicator), from the same initial states, with the plain
            # batch's tuning and as many steps as it took (autotune trials,
            # warm-up, timed), then the density L1 gap between the two runs
            from quasar_b200 import train_indicator
            from quasar_b200.indicator import attach_batch
            bl = make_batch(insts, 5)
            bl.set_tuning(ctas)
            ind5, thr5 = train_indicator.load(order=5)
            attach_batch(ind5, bl, thr5)
            bl.time_steps(trials + 3)
            lms, lzu = bl.time_steps(kb)
            num = den = 0.0
            dvb = {"max": 0.0, "rel": 0.0, "max_plain": 0.0, "rel_plain": 0.0}
            for i, x in enumerate(insts):
                shape = (x["ny"] + 2 * ics.nghost(5), x["nx"] + 2 * ics.nghost(5))
                g = ics.nghost(5)
                rp = b.instance(i).state_component_to_host("rho").reshape(shape)[g:-g, g:-g]
                rl = bl.instance(i).state_component_to_host("rho").reshape(shape)[g:-g, g:-g]
                num += float(np.abs(rl - rp).sum())
                den += float(np.abs(rp).sum())
                for key, s_ in (("", bl.instance(i)), ("_plain", b.instance(i))):
                    dvb["max" + key] = max(dvb["max" + key], s_.divergence_b_max())
                    dvb["rel" + key] = max(dvb["rel" + key], s_.divergence_b_relative())
            del bl
            lms, lzu = dist.reduce(lms, "max"), dist.reduce(lzu, "sum")
            num, den = dist.reduce(num, "sum"), dist.reduce(den, "sum")
            dvb = {k: dist.reduce(v, "max") for k, v in dvb.items()}
            batched["learned"] = {
                "value": lzu / (lms * 1e-3), "ms_per_step": lms / kb,
                "over_plain_batched": (lzu / lms) / (bzu / bms),
                "over_sequential_plain": (lzu / lms) / (seq_zu / seq_ms),
                "density_l1_vs_plain_batched": num / den,
                "div_b": dict(dvb, note="max over instances of max|div B| and of the reference's "
                                        "relative measure max|div B| dx / max|B_face|, learned "
                                        "and plain batch after the same steps"),
                "how": "shipped MP5 indicator on every instance; L1 = sum |rho_learned - "
                       "rho_plain| / sum |rho_plain| over every interior cell after the same "
                       "steps from the same initial states"}
        del b
        if not a.no_learned:
            from quasar_b200 import train_indicator
            from quasar_b200.indicator import attach_batch
            every = ics.combined_instances(seed=2, order=7)
            mine = shard.rank_share(every, [x["nx"] * x["ny"] for x in every], RANK, WORLD)
            b = make_batch(mine, 7)
            ctas, trials = b.autotune()
            b.time_steps(3)
            pms, pzu = b.time_steps(kb)
            ind, thr = train_indicator.load(order=7)
            attach_batch(ind, b, thr)
            b.time_steps(3)
            lms, lzu = b.time_steps(kb)
            pms, lms = dist.reduce(pms, "max"), dist.reduce(lms, "max")
            pzu, lzu = dist.reduce(pzu, "sum"), dist.reduce(lzu, "sum")
            combined = {"workload": "one batch: Orszag-Tang 8192^2 MP7 + 64 seeded rotor/blast MP7 "
                                    "instances, sides log-uniform in [256, 1024]",
                        "zones": sum(x["nx"] * x["ny"] for x in every), "unit": "zone-updates/s",
                        "plain_batched": pzu / (pms * 1e-3),
                        "learned_batched": lzu / (lms * 1e-3),
                        "speedup": (lzu / lms) / (pzu / pms),
                        "ms_per_step_plain": pms / kb, "ms_per_step_learned": lms / kb,
                        "note": "plain steps first, then the learned steps continue the same "
                                "batch; the density L1 gap is measured by the `learned` line "
                                "and tests/test_gpu_batch.py"}
            del b

    cpu = None
    if RANK == 0 and WORLD == 1 and not a.no_cpu:
        cpu = reference_cpu(a.case, a.order, 2, 1)
        small = reference_cpu(a.case, a.order, 3, 1, n=128)
        cpu["small_sample"] = {"value": small["value"], "sample": small["sample"]}

    if RANK == 0:
        line = {"metric": "MHD zone-updates/s (plain FP64 step)", "value": value,
                "unit": "zone-updates/s", "n_gpus": WORLD, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": t_ms / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(a),
                "gpu_launches": LAUNCHES_PER_STEP * a.steps,
                "clocks": clk, "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu,
                "div_b": div_b, "other_case": other,
                "learned": learned, "batched": batched, "batched_learned": combined}
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
