"""The multi-process host path of bench.py (N > 1 replicas, one process per
GPU): barrier and max / sum reductions over gloo, world size 2, on CPU."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    os.environ.pop("CUDA_VISIBLE_DEVICES", None)
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.barrier()
    mx = d.reduce(1.0 + rank, "max")
    sm = d.reduce(1.0 + rank, "sum")
    d.barrier()
    d.close()
    q.put((rank, mx, sm, os.environ.get("CUDA_VISIBLE_DEVICES")))


def test_two_rank_reductions_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [(r, mx, sm) for r, mx, sm, _ in out] == [(0, 2.0, 3.0), (1, 2.0, 3.0)]
    # each replica is pinned to its own GPU
    assert [dev for _, _, _, dev in out] == ["0", "1"]


def test_rank_device_pinning():
    sys.path.insert(0, ROOT)
    from bench import pin_rank_device
    env = {}
    pin_rank_device(env, 3)
    assert env["CUDA_VISIBLE_DEVICES"] == "3"
    env = {"CUDA_VISIBLE_DEVICES": "4,5,6,7"}
    pin_rank_device(env, 2)
    assert env["CUDA_VISIBLE_DEVICES"] == "6"
    env = {"CUDA_VISIBLE_DEVICES": ""}  # no GPU visible: left alone
    pin_rank_device(env, 1)
    assert env["CUDA_VISIBLE_DEVICES"] == ""
