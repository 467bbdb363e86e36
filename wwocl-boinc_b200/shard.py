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


def gpu_searcher(device: int = 0, unit_width: int = 1 << 30, max_hits: int = 1 << 16):
    """A per-rank searcher on one GPU: the rank's piece cut into unit_width
    units (the reference's checkpoint cadence) and run as one batched launch.
    Returns f(a, b) -> (checksum mod 2^64, PRP count, hits as (p, result,
    rem, quot))."""
    import wwcuda

    ctx = wwcuda.Context(device, max_prps=1 << 20, max_hits=15000)
    batch = wwcuda.Batch(ctx, max_hits=max_hits)

    def search(a: int, b: int) -> tuple[int, int, list[tuple[int, int, int, int]]]:
        if b <= a:
            return 0, 0, []
        units = [(s, min(s + unit_width, b)) for s in range(a, b, unit_width)]
        res = batch.run(units)
        if batch.hit_count > max_hits:
            raise RuntimeError(f"{batch.hit_count} hits overflowed the {max_hits}-record buffer")
        hits = [h[1:] for h in batch.hits()]
        return sum(r["checksum"] for r in res) % 2**64, sum(r["prp_count"] for r in res), hits

    search.close = ctx.close
    return search


def search_range(lo: int, hi: int, searcher, group=None) -> dict:
    """Search [lo, hi) across the ranks of `group` (or alone when no process
    group is initialised): each rank runs `searcher` on its contiguous piece,
    then one all-reduce of (checksum, PRP count) and one gather of the hits.
    The result is the same on every rank and equals a single-process search
    of the whole range."""
    import torch.distributed as dist

    if dist.is_initialized():
        world, rank = dist.get_world_size(group), dist.get_rank(group)
    else:
        world, rank = 1, 0
    a, b = split_range(lo, hi, world, rank)
    cks, cnt, hits = searcher(a, b)
    cks, cnt = reduce_sums(cks, cnt, group)
    return {"checksum": cks, "prp_count": cnt, "hits": gather_hits(hits, group), "piece": (a, b)}


def main(argv=None) -> int:
    """torchrun entry point: python -m torch.distributed.run --nproc-per-node N
    shard.py START END [--results FILE].  One rank per GPU; rank 0 prints the
    summary as one JSON line and, with --results, writes the reference's
    results file (prime hits, then the 16-digit hex checksum)."""
    import argparse
    import datetime
    import json
    import os

    import torch
    import torch.distributed as dist

    import wwcuda

    ap = argparse.ArgumentParser()
    ap.add_argument("start")
    ap.add_argument("end")
    ap.add_argument("--results", default="")
    args = ap.parse_args(argv)
    lo, hi = wwcuda.parse_number(args.start), wwcuda.parse_number(args.end)
    lo = max(lo, 127)  # the search starts at 127, as the reference's does (main.cpp:1264-1268)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    searcher = gpu_searcher(local)
    out = search_range(lo, hi, searcher)
    searcher.close()
    rank = dist.get_rank() if dist.is_initialized() else 0
    if rank == 0:
        text, dropped = wwcuda.format_hits(out["hits"])
        if args.results:
            with open(args.results, "w") as f:
                f.write(text)
                f.write("%016X\n" % out["checksum"])
        print(json.dumps({"start": lo, "end": hi, "ranks": world, "prp_count": out["prp_count"],
                          "checksum": "%016X" % out["checksum"], "hits": len(out["hits"]),
                          "prp_only_hits_dropped": dropped}))
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
