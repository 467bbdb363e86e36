"""The 2^34-wide range below 2^64 - 2^34 ([2^64 - 2^35, 2^64 - 2^35 + 2^34),
about 3.9e8 PRPs) against the reference CPU code's own result for it
(tests/golden/ref_long.json, made by make_golden.py --long): the plain
per-segment path, the batched search over 2^30-wide units (the checkpoint
cadence of the reference program), and the same units split over two
simulated ranks and summed as the multi-GPU path does."""
from __future__ import annotations

import json
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

LONG = json.loads((Path(__file__).resolve().parent / "golden" / "ref_long.json").read_text())["config3"]


@pytest.fixture(scope="module")
def ctx(ww):
    c = ww.Context(0, max_prps=1 << 25, max_hits=15000)
    yield c
    c.close()


def _units(width: int) -> list[tuple[int, int]]:
    return [(a, min(a + width, LONG["hi"])) for a in range(LONG["lo"], LONG["hi"], width)]


def test_plain_path_matches_reference(ctx):
    r = ctx.run_range(LONG["lo"], LONG["hi"])
    assert r["overflow"] == 0
    assert r["total_prp_count"] == LONG["prp_count"]
    assert "%016X" % r["checksum"] == LONG["checksum"]
    assert r["result_count"] == LONG["cpu_results"] == 0


def test_batched_units_match_reference(ww, ctx):
    b = ww.Batch(ctx)
    got = b.run(_units(1 << 30))
    assert sum(u["prp_count"] for u in got) == LONG["prp_count"]
    assert "%016X" % (sum(u["checksum"] for u in got) % 2**64) == LONG["checksum"]
    assert sum(u["hits"] for u in got) == 0


def test_two_rank_split_sums_to_reference(ww, ctx):
    import shard

    units = _units(1 << 30)
    b = ww.Batch(ctx)
    total_c, total_n = 0, 0
    for rank in range(2):
        mine = [units[i] for i in shard.split_units(units, 2, rank)]
        got = b.run(mine)
        total_c += sum(u["checksum"] for u in got)
        total_n += sum(u["prp_count"] for u in got)
    assert total_n == LONG["prp_count"]
    assert "%016X" % (total_c % 2**64) == LONG["checksum"]


def test_kernel_shaped_loop_matches_reference(ww):
    """The reference program's own loop (main.cpp:1683-1795) through the
    drop-in launchers on caller-owned memory: clearresult once, then per
    2^30-number segment clearn, getsegprimes, wieferich, wallsunsun."""
    import torch

    L = ww.lib()
    dev = torch.device("cuda", 0)
    cap, nres = 1 << 25, 15000
    e = lambda n, dt: torch.empty(n, dtype=dt, device=dev)  # noqa: E731
    prime, inv, one = e(cap, torch.int64), e(cap, torch.int64), e(2 * cap, torch.int64)
    sp, rem, quot, res = e(nres, torch.int64), e(nres, torch.int32), e(nres, torch.int32), e(nres, torch.int32)
    cks, total, rc, pc = e(1, torch.int64), e(1, torch.int64), e(1, torch.int32), e(2, torch.int32)
    ovf = torch.zeros(1, dtype=torch.int32, device=dev)
    s = torch.cuda.Stream(dev)
    st = s.cuda_stream
    P = lambda t: t.data_ptr()  # noqa: E731
    torch.cuda.synchronize(dev)
    ww.check(L.ww_launch_clearresult(P(cks), P(rc), P(total), P(pc), st), "clearresult")
    for a, b in _units(1 << 30):
        start, idx = ww.find_wheel_offset(a)
        ww.check(L.ww_launch_clearn(P(pc), st), "clearn")
        ww.check(L.ww_launch_getsegprimes(start, b, idx, P(prime), P(inv), P(pc), cap, P(ovf), st), "gsp")
        ww.check(L.ww_launch_wieferich(P(pc), P(prime), P(inv), P(one), P(sp), P(rem), P(quot), P(res), P(cks),
                                       P(rc), P(total), cap, nres, P(ovf), st), "wieferich")
        ww.check(L.ww_launch_wallsunsun(P(pc), P(prime), P(inv), P(one), P(sp), P(rem), P(quot), P(res), P(cks),
                                        P(rc), cap, nres, P(ovf), st), "wallsunsun")
    s.synchronize()
    assert int(ovf.item()) == 0
    assert int(total.item()) == LONG["prp_count"]
    assert "%016X" % (int(cks.item()) % 2**64) == LONG["checksum"]
    assert int(rc.item()) == LONG["cpu_results"]


@pytest.mark.parametrize("case", [1, 2, 3])
def test_shard_entry_writes_reference_results(tests_txt, tmp_path, case):
    """shard.py's entry point (what torchrun starts on each GPU) on the
    reference's tests.txt vectors: the results file it writes -- prime hits,
    then the hex checksum -- equals the reference's."""
    import shard

    c = tests_txt[case]
    out = tmp_path / "results.txt"
    assert shard.main([c["start"], c["end"], "--results", str(out)]) == 0
    lines = out.read_text().splitlines()
    assert lines[-1] == c["checksum"]
    if c["hits"]:  # the [1, 6e10) vector lists its checksum only, not its small special instances
        assert lines[:-1] == c["hits"]
