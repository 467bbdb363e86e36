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
