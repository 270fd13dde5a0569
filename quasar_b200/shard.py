"""Instance-parallel sharding of independent MHD instances over ranks (one
process per GPU).  No counterpart in the reference, which runs one
MhdSolver2D per process.

Independent instances need no exchange while they step: each rank builds an
MhdBatch2D of its own share and advances it; only the throughput figures
(zone-updates summed, device time as the maximum over ranks) cross ranks,
over the host process group.  The split balances zones, the work per step:
instances in decreasing zone count, each to the rank with the fewest zones so
far (the lowest rank on ties), so the partition is deterministic and every
rank computes it alone.
"""
from __future__ import annotations

from typing import List, Sequence


def partition(zones: Sequence[int], world: int) -> List[List[int]]:
    """Instance indices per rank (each list in ascending order)."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(zones)), key=lambda i: (-int(zones[i]), i))
    load = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(zones[i])
    return [sorted(p) for p in parts]


def rank_share(items: Sequence, zones: Sequence[int], rank: int, world: int) -> list:
    """The items (instance descriptions) rank `rank` steps."""
    return [items[i] for i in partition(zones, world)[rank]]


def imbalance(zones: Sequence[int], world: int) -> float:
    """Largest rank load over the mean load (1 = perfect balance)."""
    parts = partition(zones, world)
    loads = [sum(int(zones[i]) for i in p) for p in parts]
    mean = sum(loads) / world
    return max(loads) / mean if mean > 0 else 1.0
