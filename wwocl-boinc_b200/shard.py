"""Multi-GPU sharding of the search path: one process per GPU, no data-path
collective.  Ranges split into contiguous per-rank pieces (aligned to 30 so
every piece starts on a wheel boundary); the only exchange is one 64-bit sum
of checksums and PRP counts, and a gather of the hit lists, at the end.
Checksums are sums modulo 2^64, so the split never changes them."""
from __future__ import annotations

import numpy as np


def split_range(lo: int, hi: int, world: int, rank: int, align: int = 30) -> tuple[int, int]:
    """The rank's contiguous piece of [lo, hi); pieces tile the range."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    width = hi - lo

    def cut(k: int) -> int:
        if k == 0:
            return lo
        if k == world:
            return hi
        c = lo + width * k // world
        return max(lo, min(hi, c - c % align))

    return cut(rank), cut(rank + 1)


def split_units(units: list[tuple[int, int]], world: int, rank: int) -> list[int]:
    """Indices of the units a rank runs: greedy balance by width (largest
    first to the least loaded rank), deterministic on every rank."""
    order = sorted(range(len(units)), key=lambda i: (-(units[i][1] - units[i][0]), i))
    load = [0] * world
    owner = [0] * len(units)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += units[i][1] - units[i][0]
    return [i for i in range(len(units)) if owner[i] == rank]


def reduce_sums(checksum: int, prp_count: int, group=None) -> tuple[int, int]:
    """Sum (checksum mod 2^64, PRP count) over the ranks of `group`."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([np.int64(np.uint64(checksum % 2**64)), prp_count], dtype=torch.int64)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, group=group)
    c, n = (int(x) for x in t.cpu().tolist())
    return c % 2**64, n


def gather_hits(hits: list[tuple], group=None) -> list[tuple]:
    """Every rank's hit records, merged and sorted by p (Wieferich first)."""
    import torch.distributed as dist

    if dist.is_initialized() and dist.get_world_size(group) > 1:
        out = [None] * dist.get_world_size(group)
        dist.all_gather_object(out, list(hits), group=group)
        hits = [h for part in out for h in part]
    return sorted(hits, key=lambda h: (h[0], h[1] != 1093))
