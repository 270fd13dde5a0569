"""One MHD instance decomposed over ranks: 2-D tiles with deep halos (the
"next" multi-GPU row: the reference's distributed runtime,
src/distributed/mhd_runtime.cpp, exchanges halos, face records and CT
tables every stage and reduces dt and the admissible fraction over ranks).

Design.  Rank r of a px x py process grid owns a block of cells and steps a
local MhdSolver2D over that block plus a halo of `halo` cells on every side
that is not a physical boundary.  The halo is deep enough for a whole SSP-RK3
step: each stage's residual at a cell depends on cells at most about 15 away
(MP7: the normal stencil, the transverse Gauss recovery, the collocated
field and the corner EMF interpolation), so three stages stay inside 48
cells and the owned cells come out of the local step bit for bit as in the
undecomposed run.  What crosses ranks per step:

* dt: every rank's cfl_limit() over its owned cells only (the solver's owned
  window), reduced with MIN: the same dt as the whole domain's;
* after the step, the halo: every local position another rank owns is
  refreshed from that rank (cells and both face fields; a face belongs to
  the owner of the cell above it, the domain's last face to its last cell),
  written back with write_halo so that the state stays solver-owned;
* agreement flags (MAX) around each collective so that a rank that fails
  (a preflight, a positivity retry) takes every rank down with the same
  error instead of leaving them waiting in the next collective.

Positivity retries are not coordinated: a step that needs one on any rank
raises on every rank.  The kernels never wait on another rank: the exchange
is a host step between launches.  exchange="host" reads whole components
back, patches the halo on the host and writes them with write_halo;
exchange="device" gathers only the positions peers need into one packed
device buffer per peer (gather_live), sends those buffers over the process
group (CUDA tensors under NCCL, staged through host memory under gloo) and
scatters the received ones into the halo (scatter_halo), so per step only
the halo's bytes move.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Tuple

import numpy as np

from . import mhd

CELL = ("rho", "mx", "my", "mz", "energy", "bz_cell")
COMPONENTS = ("rho", "mx", "my", "mz", "energy", "bx_face", "by_face", "bz_cell")
DEFAULT_HALO = 48


def _split(n: int, parts: int, k: int) -> Tuple[int, int]:
    return (k * n) // parts, ((k + 1) * n) // parts


@dataclasses.dataclass
class Tile:
    """Rank `rank`'s piece: owned cells [x0, x1) x [y0, y1) of the global
    interior and the local domain [lx0, lx0 + nxl) x [ly0, ly0 + nyl) in
    global cell coordinates (periodic axes may run past the edges)."""
    rank: int
    x0: int
    x1: int
    y0: int
    y1: int
    lx0: int
    ly0: int
    nxl: int
    nyl: int
    bc: Tuple[str, str, str, str]

    def window(self) -> Tuple[int, int, int, int]:
        """The owned cells in local interior coordinates."""
        return (self.x0 - self.lx0, self.x1 - self.lx0, self.y0 - self.ly0, self.y1 - self.ly0)


class TileLayout:
    """px x py decomposition of an nx x ny domain with side boundaries `bc`
    (x_lo, x_hi, y_lo, y_hi: 'periodic', 'outflow' or 'wall')."""

    def __init__(self, nx: int, ny: int, bc, px: int, py: int, halo: int = DEFAULT_HALO):
        if px < 1 or py < 1 or px > nx or py > ny:
            raise ValueError("process grid must be 1 <= px <= nx, 1 <= py <= ny")
        if (bc[0] == "periodic") != (bc[1] == "periodic") or (bc[2] == "periodic") != (bc[3] == "periodic"):
            raise ValueError("periodic sides come in pairs")
        self.nx, self.ny, self.px, self.py, self.halo = nx, ny, px, py, halo
        self.bc = tuple(bc)
        self.perx, self.pery = bc[0] == "periodic", bc[2] == "periodic"
        self.tiles = [self._tile(r) for r in range(px * py)]

    @property
    def world(self) -> int:
        return self.px * self.py

    def _axis(self, n, parts, k, periodic, lo_bc, hi_bc):
        a, b = _split(n, parts, k)
        if parts == 1:
            return a, b, 0, n, (lo_bc, hi_bc)
        if periodic:
            h = self.halo
            return a, b, a - h, (b - a) + 2 * h, ("outflow", "outflow")
        hl, hh = min(self.halo, a), min(self.halo, n - b)
        return a, b, a - hl, (b - a) + hl + hh, (lo_bc if hl == 0 else "outflow",
                                                  hi_bc if hh == 0 else "outflow")

    def _tile(self, r: int) -> Tile:
        rx, ry = r % self.px, r // self.px
        x0, x1, lx0, nxl, (bxl, bxh) = self._axis(self.nx, self.px, rx, self.perx, self.bc[0], self.bc[1])
        y0, y1, ly0, nyl, (byl, byh) = self._axis(self.ny, self.py, ry, self.pery, self.bc[2], self.bc[3])
        return Tile(r, x0, x1, y0, y1, lx0, ly0, nxl, nyl, (bxl, bxh, byl, byh))

    def _bounds(self, n: int, parts: int) -> np.ndarray:
        return np.array([(k * n) // parts for k in range(parts + 1)])

    def owner(self, gi, gj, kind: str):
        """Rank owning global positions (arrays or scalars): a cell's tile; a
        face, the tile of the cell above it (the domain's last face: its
        last cell's)."""
        gi, gj = np.asarray(gi), np.asarray(gj)
        ci = np.minimum(gi, self.nx - 1) if kind == "xface" else gi
        cj = np.minimum(gj, self.ny - 1) if kind == "yface" else gj
        ox = np.searchsorted(self._bounds(self.nx, self.px), ci, side="right") - 1
        oy = np.searchsorted(self._bounds(self.ny, self.py), cj, side="right") - 1
        r = ox + self.px * oy
        return int(r) if r.ndim == 0 else r

    def positions(self, t: Tile, kind: str):
        """Local interior positions (il, jl) of `kind` the local step evolves,
        row by row, as two index arrays."""
        ni = t.nxl + (1 if kind == "xface" else 0)
        nj = t.nyl + (1 if kind == "yface" else 0)
        jl, il = np.meshgrid(np.arange(nj), np.arange(ni), indexing="ij")
        return il.ravel(), jl.ravel()

    def _global(self, t: Tile, il, jl, kind: str):
        """Global positions of local interior positions of `kind` ('cell',
        'xface', 'yface'), wrapped on periodic axes."""
        gi, gj = np.asarray(il) + t.lx0, np.asarray(jl) + t.ly0
        if self.perx:
            gi = gi % self.nx
        if self.pery:
            gj = gj % self.ny
        return gi, gj

    def _owned_here(self, t: Tile, il, jl, kind: str):
        """Whether local positions are the owner's own copy (inside the owned
        block, not a periodic image of it)."""
        gi, gj = np.asarray(il) + t.lx0, np.asarray(jl) + t.ly0
        xi = (t.x0 <= gi) & (gi < t.x1)
        yj = (t.y0 <= gj) & (gj < t.y1)
        if kind == "xface" and not self.perx and t.x1 == self.nx:
            xi = xi | (gi == self.nx)
        if kind == "yface" and not self.pery and t.y1 == self.ny:
            yj = yj | (gj == self.ny)
        return xi & yj

    def exchange_plan(self, rank: int, ng: int) -> Dict[int, Dict[str, Tuple[np.ndarray, np.ndarray]]]:
        """For every peer p (this rank included for wrapped copies):
        plan[p][kind] = (indices into this rank's padded local arrays that
        receive from p, indices into p's padded local arrays that p sends),
        in one agreed order (this rank's positions row by row)."""
        t = self.tiles[rank]
        pitch = t.nxl + 2 * ng
        plan: Dict[int, Dict[str, Tuple[np.ndarray, np.ndarray]]] = {}
        for kind in ("cell", "xface", "yface"):
            il, jl = self.positions(t, kind)
            gi, gj = self._global(t, il, jl, kind)
            own = self.owner(gi, gj, kind)
            take = ~((own == rank) & self._owned_here(t, il, jl, kind))
            il, jl, gi, gj, own = il[take], jl[take], gi[take], gj[take], own[take]
            dst_all = (il + ng) + pitch * (jl + ng)
            for p in np.unique(own):
                sel = own == p
                src = self.tiles[int(p)]
                # the owner's local coordinates of the positions it owns
                src_k = (gi[sel] - src.lx0 + ng) + (src.nxl + 2 * ng) * (gj[sel] - src.ly0 + ng)
                plan.setdefault(int(p), {})[kind] = (dst_all[sel].astype(np.int64),
                                                     src_k.astype(np.int64))
        return plan

    def local_grid_config(self, cfg: mhd.MhdConfig, rank: int) -> mhd.MhdConfig:
        t = self.tiles[rank]
        g = cfg.grid
        dx, dy = g.lx / g.nx, g.ly / g.ny
        c = dataclasses.replace(cfg)
        c.grid = mhd.Grid2D(t.nxl, t.nyl, t.nxl * dx, t.nyl * dy,
                            g.origin_x + t.lx0 * dx, g.origin_y + t.ly0 * dy)
        c.boundary = mhd.MhdBoundarySpec(list(t.bc), list(t.bc))
        return c

    def kind_of(self, name: str) -> str:
        return "xface" if name == "bx_face" else "yface" if name == "by_face" else "cell"


def extract_local(layout: TileLayout, rank: int, global_padded: np.ndarray, name: str,
                  ng: int) -> np.ndarray:
    """This rank's padded local array cut from a global padded array (the
    global array's ghost layers must hold at least ng cells; periodic axes
    wrap through the interior)."""
    t = layout.tiles[rank]
    gp = np.asarray(global_padded).reshape(layout.ny + 2 * ng, layout.nx + 2 * ng)
    gi = np.arange(-ng, t.nxl + ng) + t.lx0
    gj = np.arange(-ng, t.nyl + ng) + t.ly0
    if layout.perx:
        gi = gi % layout.nx
    if layout.pery:
        gj = gj % layout.ny
    okx = (gi >= -ng) & (gi < layout.nx + ng)
    oky = (gj >= -ng) & (gj < layout.ny + ng)
    out = np.zeros((t.nyl + 2 * ng, t.nxl + 2 * ng))
    out[np.ix_(oky, okx)] = gp[np.ix_(gj[oky] + ng, gi[okx] + ng)]
    return out.reshape(-1)


class TiledSolver:
    """The rank's tile of a decomposed MhdSolver2D over a process group
    (torch.distributed, initialised by the caller).  Every rank calls every
    method in the same order."""

    def __init__(self, cfg: mhd.MhdConfig, px: int, py: int, halo: int = DEFAULT_HALO,
                 group=None, device: str = "cpu", exchange: str = "host"):
        import torch.distributed as dist
        if exchange not in ("host", "device"):
            raise ValueError("exchange must be 'host' or 'device'")
        self.dist, self.group, self.device = dist, group, device
        self.exchange_mode = exchange
        self._xplan = None
        self.rank = dist.get_rank(group)
        world = dist.get_world_size(group)
        g = cfg.grid
        side = list(cfg.boundary.fluid)
        self.layout = TileLayout(g.nx, g.ny, side, px, py, halo)
        if self.layout.world != world:
            raise ValueError(f"process grid {px}x{py} needs {px * py} ranks, the group has {world}")
        self.cfg = cfg
        self.local = mhd.MhdSolver2D(self.layout.local_grid_config(cfg, self.rank))
        self.ng = self.local.grid().nghost
        self.tile = self.layout.tiles[self.rank]
        self.local.set_owned_window(*self.tile.window())
        self.plans = [self.layout.exchange_plan(r, self.ng) for r in range(world)]
        if exchange == "device":
            import torch
            # where the solver's state lives: the gathered and scattered halo
            # values stay there; only the packed halo crosses the group
            self.xdev = torch.device("cuda", torch.cuda.current_device())

    # ---- agreement and reductions -------------------------------------------
    def _reduce(self, value: float, op: str) -> float:
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        o = self.dist.ReduceOp.MIN if op == "min" else self.dist.ReduceOp.MAX if op == "max" else \
            self.dist.ReduceOp.SUM
        self.dist.all_reduce(t, op=o, group=self.group)
        return float(t.item())

    def _agree(self, fn):
        """Run fn on every rank; if it raised anywhere, raise everywhere."""
        err, out = None, None
        try:
            out = fn()
        except (RuntimeError, ValueError) as e:
            err = e
        if self._reduce(1.0 if err else 0.0, "max") > 0.0:
            raise err if err else RuntimeError("tiled solver: another rank failed")
        return out

    # ---- seeding and stepping ------------------------------------------------
    def seed_global(self, name: str, global_padded) -> None:
        """Seed component `name` from the whole domain's padded array (every
        rank passes the same array)."""
        arr = extract_local(self.layout, self.rank, np.asarray(global_padded, dtype=np.float64),
                            name, self.ng)
        self._agree(lambda: self.local.seed_state(name, arr))

    def cfl_limit(self) -> float:
        dt = self._agree(self.local.cfl_limit)
        return self._reduce(dt, "min")

    def step_unchecked(self, dt: float) -> None:
        def run():
            self.local.step_unchecked(dt)
            if self.local.last_positivity_substeps() > 1:
                raise RuntimeError("tiled solver: a positivity retry is not coordinated across "
                                   "tiles; step the undecomposed solver")
        self._agree(run)
        self.exchange()

    def advance_steps(self, steps: int) -> float:
        t = 0.0
        for _ in range(steps):
            dt = self.cfl_limit()
            self.step_unchecked(dt)
            t += dt
        return t

    # ---- halo exchange ------------------------------------------------------
    def _pairwise(self, sends, recvs) -> None:
        """Blocking send / recv with every peer, pairwise in rank order: the
        lower rank of a pair sends first, so no two ranks wait on each other."""
        for p in sorted(set(sends) | set(recvs)):
            if self.rank < p:
                if p in sends:
                    self.dist.send(sends[p], dst=p, group=self.group)
                if p in recvs:
                    self.dist.recv(recvs[p], src=p, group=self.group)
            else:
                if p in recvs:
                    self.dist.recv(recvs[p], src=p, group=self.group)
                if p in sends:
                    self.dist.send(sends[p], dst=p, group=self.group)

    def exchange(self) -> None:
        """Refresh every local position another rank owns from that rank."""
        if getattr(self, "exchange_mode", "host") == "device":
            self._exchange_device()
        else:
            self._exchange_host()

    def _device_plan(self):
        """The exchange plan as device index tensors, built once: per peer
        the (component, indices) this rank packs for it and unpacks from it,
        in the agreed order (components in COMPONENTS order, positions in the
        receiver's order), and the periodic self-images."""
        if self._xplan is not None:
            return self._xplan
        import torch
        kinds = {n: self.layout.kind_of(n) for n in COMPONENTS}

        cache = {}

        def dev(a):
            # components of one kind share their index arrays: upload each once
            key = id(a)
            if key not in cache:
                cache[key] = (a, torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64),
                                                 device=self.xdev))
            return cache[key][1]
        send, recv, images = {}, {}, []
        for p in range(self.layout.world):
            if p == self.rank:
                continue
            need = self.plans[p].get(self.rank, {})
            items = [(n, dev(need[kinds[n]][1])) for n in COMPONENTS if kinds[n] in need]
            if items:
                send[p] = items
        mine = self.plans[self.rank]
        for p, have in mine.items():
            items = [(n, dev(have[kinds[n]][0])) for n in COMPONENTS if kinds[n] in have]
            if p == self.rank:
                images = [(n, dev(have[kinds[n]][1]), idx) for n, idx in items]
            elif items:
                recv[p] = items
        self._xplan = (send, recv, images)
        return self._xplan

    def _sync(self) -> None:
        import torch
        if self.xdev.type == "cuda":
            torch.cuda.synchronize(self.xdev)

    def _exchange_device(self) -> None:
        """The exchange without whole components crossing to the host: each
        rank gathers what its peers need into one packed device buffer per
        peer, the buffers cross the group (directly as CUDA tensors under
        NCCL, staged through host memory under gloo), and the receiver
        scatters them into its halo positions."""
        import torch
        send, recv, images = self._device_plan()
        f64 = torch.float64
        packed, image_vals = {}, []

        def pack():
            self._sync()
            for p, items in send.items():
                buf = torch.empty(sum(int(i.numel()) for _, i in items), dtype=f64,
                                  device=self.xdev)
                off = 0
                for n, idx in items:
                    self.local.gather_live(n, idx, buf[off:off + idx.numel()])
                    off += idx.numel()
                packed[p] = buf
            for n, src, dst in images:
                v = torch.empty(src.numel(), dtype=f64, device=self.xdev)
                self.local.gather_live(n, src, v)
                image_vals.append((n, dst, v))
        self._agree(pack)
        sends = {p: b.to(self.device) for p, b in packed.items()}
        recvs = {p: torch.empty(sum(int(i.numel()) for _, i in items), dtype=f64,
                                device=self.device) for p, items in recv.items()}
        self._pairwise(sends, recvs)

        def unpack():
            bufs = {p: b.to(self.xdev) for p, b in recvs.items()}
            self._sync()
            for p, items in recv.items():
                off = 0
                for n, idx in items:
                    self.local.scatter_halo(n, idx, bufs[p][off:off + idx.numel()])
                    off += idx.numel()
            for n, dst, v in image_vals:
                self.local.scatter_halo(n, dst, v)
        self._agree(unpack)

    def _exchange_host(self) -> None:
        import torch
        arrays = {n: self.local.state_component_to_host(n) for n in COMPONENTS}
        world = self.layout.world
        kinds = {n: self.layout.kind_of(n) for n in COMPONENTS}
        sends, recvs = {}, {}
        for p in range(world):
            # what p needs from me, in p's order
            need = self.plans[p].get(self.rank, {})
            parts = [arrays[n][need[kinds[n]][1]] for n in COMPONENTS if kinds[n] in need]
            if p == self.rank:
                continue
            if parts:
                buf = torch.from_numpy(np.concatenate(parts)).to(self.device)
                sends[p] = buf
        mine = self.plans[self.rank]
        for p in range(world):
            if p == self.rank or p not in mine:
                continue
            size = sum(len(mine[p][kinds[n]][0]) for n in COMPONENTS if kinds[n] in mine[p])
            recvs[p] = torch.empty(size, dtype=torch.float64, device=self.device)
        self._pairwise(sends, recvs)
        for p, buf in recvs.items():
            data, off = buf.cpu().numpy(), 0
            for n in COMPONENTS:
                k = kinds[n]
                if k not in mine[p]:
                    continue
                dst = mine[p][k][0]
                arrays[n][dst] = data[off:off + len(dst)]
                off += len(dst)
        if self.rank in mine:  # periodic images of this rank's own cells
            for n in COMPONENTS:
                k = kinds[n]
                if k in mine[self.rank]:
                    dst, src = mine[self.rank][k]
                    arrays[n][dst] = arrays[n][src]
        self._agree(lambda: [self.local.write_halo(n, arrays[n]) for n in COMPONENTS])

    # ---- gathering -----------------------------------------------------------
    def owned_block(self, name: str) -> np.ndarray:
        """This rank's owned values of `name` in local storage order
        (cells, or the faces the rank owns)."""
        return self.local.state_component_to_host(name)

    def gather(self, name: str) -> np.ndarray:
        """The whole domain's padded array of `name` on every rank (interior
        cells and evolved faces filled from their owners; ghosts zero)."""
        import torch
        ng, lay = self.ng, self.layout
        kind = lay.kind_of(name)
        pitch = lay.nx + 2 * ng
        local = self.local.state_component_to_host(name)
        t = self.tile
        lp = t.nxl + 2 * ng
        il, jl = lay.positions(t, kind)
        gi, gj = lay._global(t, il, jl, kind)
        mine = (lay.owner(gi, gj, kind) == self.rank) & lay._owned_here(t, il, jl, kind)
        gidx = ((gi[mine] + ng) + pitch * (gj[mine] + ng)).tolist()
        vals = local[(il[mine] + ng) + lp * (jl[mine] + ng)].tolist()
        n = torch.tensor([len(gidx)], dtype=torch.int64)
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(lay.world)]
        self.dist.all_gather(sizes, n, group=self.group)
        m = int(max(s.item() for s in sizes))
        gi_t = torch.full((m,), -1, dtype=torch.int64)
        gi_t[:len(gidx)] = torch.tensor(gidx, dtype=torch.int64)
        v_t = torch.zeros(m, dtype=torch.float64)
        v_t[:len(vals)] = torch.tensor(vals, dtype=torch.float64)
        all_i = [torch.empty(m, dtype=torch.int64) for _ in range(lay.world)]
        all_v = [torch.empty(m, dtype=torch.float64) for _ in range(lay.world)]
        self.dist.all_gather(all_i, gi_t, group=self.group)
        self.dist.all_gather(all_v, v_t, group=self.group)
        out = np.zeros((lay.ny + 2 * ng) * pitch)
        for a, b in zip(all_i, all_v):
            a, b = a.numpy(), b.numpy()
            keep = a >= 0
            out[a[keep]] = b[keep]
        # a periodic axis's last face is the image of its first
        o = out.reshape(lay.ny + 2 * ng, pitch)
        if kind == "xface" and lay.perx:
            o[ng:ng + lay.ny, ng + lay.nx] = o[ng:ng + lay.ny, ng]
        if kind == "yface" and lay.pery:
            o[ng + lay.ny, ng:ng + lay.nx] = o[ng, ng:ng + lay.nx]
        return out
