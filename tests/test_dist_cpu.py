"""The multi-process host path of bench.py (one process per GPU): barrier
and max / sum reductions over gloo, and the instance-parallel sharding of a
batch (quasar_b200/shard.py), world size 2, on CPU."""
import os
import socket
import sys

import numpy as np
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


class _ArraySolver:
    """Stand-in for a tile's local solver on the CPU: numpy arrays behind
    state_component_to_host / write_halo."""

    def __init__(self, arrays):
        self.arrays = arrays

    def state_component_to_host(self, name):
        return self.arrays[name].copy()

    def write_halo(self, name, values):
        self.arrays[name] = np.asarray(values, dtype=np.float64).copy()

    # the device exchange's calls, on CPU tensors
    def gather_live(self, name, idx, out):
        import torch
        out.copy_(torch.from_numpy(self.arrays[name])[idx])

    def scatter_halo(self, name, idx, values):
        v = values.numpy()
        if not np.all(np.isfinite(v)):
            raise ValueError("scatter_halo: non-finite value")
        self.arrays[name][idx.numpy()] = v


def _tile_rank(rank, world, port, q, nx, ny, bc, px, py, halo, mode):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch.distributed as dist

    from quasar_b200 import tiles
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ng = 3
    lay = tiles.TileLayout(nx, ny, bc, px, py, halo)
    rng = np.random.default_rng(7)
    glob = {n: rng.standard_normal((ny + 2 * ng) * (nx + 2 * ng)) for n in tiles.COMPONENTS}
    t = lay.tiles[rank]
    loc = {n: tiles.extract_local(lay, rank, glob[n], n, ng) for n in tiles.COMPONENTS}
    want = {n: a.copy() for n, a in loc.items()}
    # every position this tile does not own is stale before the exchange
    lp = t.nxl + 2 * ng
    for n in tiles.COMPONENTS:
        kind = lay.kind_of(n)
        il, jl = lay.positions(t, kind)
        gi, gj = lay._global(t, il, jl, kind)
        stale = ~((lay.owner(gi, gj, kind) == rank) & lay._owned_here(t, il, jl, kind))
        loc[n][(il[stale] + ng) + lp * (jl[stale] + ng)] = np.nan
    ts = tiles.TiledSolver.__new__(tiles.TiledSolver)
    ts.dist, ts.group, ts.device, ts.rank = dist, None, "cpu", rank
    ts.layout, ts.tile, ts.ng = lay, t, ng
    ts.local = _ArraySolver(loc)
    ts.plans = [lay.exchange_plan(r, ng) for r in range(world)]
    ts.exchange_mode, ts._xplan = mode, None
    if mode == "device":
        import torch
        ts.xdev = torch.device("cpu")
    ts.exchange()
    ok = True
    for n in tiles.COMPONENTS:
        il, jl = lay.positions(t, lay.kind_of(n))
        k = (il + ng) + lp * (jl + ng)
        ok = ok and np.array_equal(ts.local.arrays[n][k], want[n][k])
    g = {n: ts.gather(n) for n in ("rho", "bx_face", "by_face")}
    pitch = nx + 2 * ng
    gat = True
    for n, kind in (("rho", "cell"), ("bx_face", "xface"), ("by_face", "yface")):
        gp, ref = g[n].reshape(-1, pitch), glob[n].reshape(-1, pitch)
        ni, nj = nx + (kind == "xface"), ny + (kind == "yface")
        sub, rsub = gp[ng:ng + nj, ng:ng + ni], ref[ng:ng + nj, ng:ng + ni]
        if kind == "xface" and bc[0] == "periodic":
            sub, rsub = sub[:, :nx], rsub[:, :nx]
        if kind == "yface" and bc[2] == "periodic":
            sub, rsub = sub[:ny], rsub[:ny]
        gat = gat and np.array_equal(sub, rsub)
    dist.destroy_process_group()
    q.put((rank, bool(ok), bool(gat)))


@pytest.mark.parametrize("mode", ["host", "device"])
@pytest.mark.parametrize("nx,ny,bc,px,py,halo", [
    (24, 20, ("periodic",) * 4, 2, 1, 6),
    (24, 20, ("outflow",) * 4, 1, 2, 5),
    (17, 13, ("periodic", "periodic", "outflow", "outflow"), 2, 2, 4),
    (10, 12, ("periodic",) * 4, 2, 2, 7),   # halos wider than a tile: periodic images
])
def test_tile_halo_exchange_over_gloo(nx, ny, bc, px, py, halo, mode):
    """The tile runtime's exchange (quasar_b200/tiles.py) on gloo ranks with
    numpy arrays in place of the solvers: every position a tile does not own
    (cells and both face fields, periodic images included) comes back equal
    to the whole domain's value, and gathering the owned values rebuilds the
    whole domain.  "device" runs the packed gather / send / scatter exchange
    with CPU tensors standing in for the device buffers (the stale positions
    hold NaN, so a position the plan missed or scattered twice from a stale
    source shows)."""
    import torch.multiprocessing as mp
    world = px * py
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_tile_rank, args=(r, world, port, q, nx, ny, bc, px, py, halo, mode))
             for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok and gat for _, ok, gat in out), out
