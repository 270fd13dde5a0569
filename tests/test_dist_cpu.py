"""The multi-process host path of bench.py (one process per GPU): barrier
and max / sum reductions over gloo, and the instance-parallel sharding of a
batch (quasar_b200/shard.py), world size 2, on CPU."""
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


def _shard_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    os.environ.pop("CUDA_VISIBLE_DEVICES", None)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    from quasar_b200 import ics, shard
    d = bench.Dist()
    insts = ics.batch_instances(count=256, seed=0, order=5)  # descriptions only
    zones = [x["nx"] * x["ny"] for x in insts]
    mine = shard.rank_share(list(range(len(insts))), zones, rank, world)
    # every rank's share, gathered over gloo: a partition of all instances
    got = [None] * world
    dist.all_gather_object(got, mine)
    # throughput the way bench.py forms it: zone-updates summed, time max
    zu = d.reduce(float(sum(zones[i] for i in mine)), "sum")
    ms = d.reduce(10.0 + rank, "max")
    d.close()
    q.put((rank, got, zu, ms))


def test_two_rank_instance_sharding_over_gloo():
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    from quasar_b200 import ics
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    zones = [x["nx"] * x["ny"] for x in ics.batch_instances(count=256, seed=0, order=5)]
    (_, got0, zu0, ms0), (_, got1, zu1, ms1) = out
    assert got0 == got1  # both ranks computed the same partition
    flat = sorted(i for part in got0 for i in part)
    assert flat == list(range(256))  # each instance on exactly one rank
    loads = [sum(zones[i] for i in part) for part in got0]
    assert abs(loads[0] - loads[1]) <= max(zones)  # balanced to one instance
    assert zu0 == zu1 == float(sum(zones)) and ms0 == ms1 == 11.0


def test_partition_rules():
    sys.path.insert(0, ROOT)
    from quasar_b200 import shard
    assert shard.partition([5, 3, 3, 1], 2) == [[0, 3], [1, 2]]
    assert shard.partition([4, 4], 3) == [[0], [1], []]
    assert shard.partition([7, 1, 1, 1], 1) == [[0, 1, 2, 3]]
    assert shard.imbalance([1] * 8, 4) == 1.0
    with pytest.raises(ValueError):
        shard.partition([1], 0)
