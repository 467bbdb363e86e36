"""Multi-rank host logic on CPU: two gloo ranks each search their piece of a
range with the CPU oracle (standing in for one GPU each) and the reduced
checksum, PRP count and hits equal the single-process result; checkpoint
state files survive corruption, truncation and mismatches."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import PKG, ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, lo, hi, out):
    import sys

    for p in (str(ROOT), str(PKG)):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    import shard
    from oracle.oracle import Oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    oracle = Oracle()

    def cpu_searcher(a, b):  # the oracle stands in for this rank's GPU
        summ, _, hits = oracle.scan_range(a, b, nthreads=2, hit_cap=100000)
        return summ["checksum"], summ["prp_count"], hits

    r = shard.search_range(lo, hi, cpu_searcher)
    out[rank] = (r["checksum"], r["prp_count"], r["hits"], r["piece"])
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("lo,hi", [(127, 3_000_000), (2**64 - 2**35, 2**64 - 2**35 + 1_000_000)])
def test_two_rank_split_equals_single(oracle, lo, hi):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, lo, hi, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    summ, _, hits = oracle.scan_range(lo, hi, hit_cap=100000)
    pieces = sorted(out[r][3] for r in range(world))
    assert pieces[0][0] == lo and pieces[-1][1] == hi and pieces[0][1] == pieces[1][0]
    for r in range(world):
        cks, cnt, allhits, _ = out[r]
        assert cks == summ["checksum"] and cnt == summ["prp_count"]
        assert sorted(allhits) == sorted(hits)


def test_split_units_balances_and_covers(ww):
    import shard

    units = ww.uneven_units(11, 300)
    world = 4
    owned = [shard.split_units(units, world, r) for r in range(world)]
    flat = sorted(i for o in owned for i in o)
    assert flat == list(range(len(units)))
    loads = [sum(units[i][1] - units[i][0] for i in o) for o in owned]
    assert max(loads) < 1.2 * min(loads)


def test_split_range_alignment():
    import shard

    for world in (1, 2, 3, 8):
        pieces = [shard.split_range(127, 10**12 + 7, world, r) for r in range(world)]
        assert pieces[0][0] == 127 and pieces[-1][1] == 10**12 + 7
        for (a, b), (c, d) in zip(pieces, pieces[1:]):
            assert b == c and c % 30 == 0


# ---------------------------------------------------------------- checkpoints

def test_state_alternates_and_newer_wins(ww, tmp_path):
    a, b = str(tmp_path / "stateA-WW.txt"), str(tmp_path / "stateB-WW.txt")
    nxt = True
    for cur in (1000, 2000, 3000):
        nxt = ww.state_write(a, b, 127, 10**6, cur, cur * 7, 1.5, 2, nxt)
    st, write_a_next = ww.state_read(a, b, 127, 10**6)
    assert st["current"] == 3000 and st["cksm"] == 21000
    # A got 1000 then 3000, B got 2000: A is newer, so B is written next
    assert write_a_next is False
    assert open(a).read().split()[:4] == ["127", "1000000", "3000", "21000"]


def test_state_torn_or_corrupt_file_falls_back(ww, tmp_path):
    a, b = str(tmp_path / "A"), str(tmp_path / "B")
    nxt = ww.state_write(a, b, 127, 10**6, 5000, 1, 0.0, 0, True)
    nxt = ww.state_write(a, b, 127, 10**6, 6000, 2, 0.0, 0, nxt)
    open(b, "w").write("127 1000000 60")  # torn write of the newer file
    st, _ = ww.state_read(a, b, 127, 10**6)
    assert st["current"] == 5000
    open(a, "w").write("garbage\n")
    assert ww.state_read(a, b, 127, 10**6) is None


def test_state_for_another_range_is_ignored(ww, tmp_path):
    a, b = str(tmp_path / "A"), str(tmp_path / "B")
    ww.state_write(a, b, 127, 10**6, 5000, 1, 0.0, 0, True)
    assert ww.state_read(a, b, 127, 2 * 10**6) is None
    assert ww.state_read(a, b, 128, 10**6) is None


def test_state_missing_files(ww, tmp_path):
    assert ww.state_read(str(tmp_path / "nope1"), str(tmp_path / "nope2"), 1, 2) is None
