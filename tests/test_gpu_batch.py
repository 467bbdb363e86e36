"""The batched persistent search: per-unit checksums, PRP counts and hits
bit-identical to running each unit alone, for every compiled configuration,
and against the oracle on small units."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(ww):
    c = ww.Context(0, max_prps=1 << 22, max_hits=15000)
    yield c
    c.close()


def _alone(ctx, lo, hi):
    r = ctx.run_range(lo, hi)
    return r["checksum"], r["total_prp_count"], r["result_count"]


def test_small_units_match_oracle(ww, ctx, oracle):
    units = [(127, 1_000_000), (4_294_000_000, 4_295_500_000), (2**64 - 2**35, 2**64 - 2**35 + 700_001),
             (2276306935816523 - 5000, 2276306935816523 + 5000), (1000, 1000), (2**64 - 1_000_001, 2**64 - 1),
             (2**63 - 500_001, 2**63 + 499_999), (2**62 - 300_000, 2**62 + 300_000)]
    b = ww.Batch(ctx)
    got = b.run(units)
    hits = b.hits()
    for i, (lo, hi) in enumerate(units):
        if hi > lo:
            want, _, whits = oracle.scan_range(lo, hi, hit_cap=100000)
        else:
            want, whits = dict(checksum=0, prp_count=0, gpu_results=0), []
        assert got[i]["checksum"] == want["checksum"], i
        assert got[i]["prp_count"] == want["prp_count"], i
        assert got[i]["hits"] == want["gpu_results"], i
        assert sorted(h[1:] for h in hits if h[0] == i) == sorted(whits), i


def test_every_config_matches_alone(ww, ctx):
    units = ww.uneven_units(11, 24, wmin=1e5, wmax=3e8)
    alone = [_alone(ctx, lo, hi) for lo, hi in units]
    b = ww.Batch(ctx)
    for cfg in ww.batch_configs():
        b.set_config(*cfg)
        got = b.run(units)
        for i, r in enumerate(got):
            assert (r["checksum"], r["prp_count"], r["hits"]) == alone[i], (cfg, i)


def test_tuner_picks_a_config(ww, ctx):
    b = ww.Batch(ctx)
    sample = ww.uneven_units(11, 64, wmin=1e6, wmax=1e9)
    cfg, ms = b.tune(sample)
    assert cfg in ww.batch_configs() and ms > 0
    assert b.config() == cfg


def test_config4_subsample_matches_alone(ww, ctx):
    """First 48 units of the seed-11 uneven mix (widths 1e6..1e10), batched
    versus one range per launch."""
    units = ww.uneven_units(11, 4096)[:48]
    b = ww.Batch(ctx)
    got = b.run(units)
    for i, (lo, hi) in enumerate(units):
        assert (got[i]["checksum"], got[i]["prp_count"], got[i]["hits"]) == _alone(ctx, lo, hi), i


def test_bad_unit_is_rejected(ww, ctx):
    b = ww.Batch(ctx)
    with pytest.raises(ww.WWError):
        b.run([(100, 1000)])


def test_one_and_two_number_ranges(ww, ctx, oracle):
    """Ranges one or two numbers wide on a Wieferich special instance, a WSS
    special instance, a base-2 strong pseudoprime (49141), the first allowed
    start, the largest 64-bit prime and the last numbers below 2^64: the
    batched engine, the plain path and the GPU count agree with the oracle,
    hits included."""
    units = [(2276306935816523, 2276306935816524), (338772621946054253, 338772621946054255),
             (49141, 49142), (127, 128), (127, 129), (2**64 - 59, 2**64 - 58), (2**64 - 3, 2**64 - 1),
             (2**64 - 2, 2**64 - 1), (1_000_003, 1_000_004), (1_000_004, 1_000_005)]
    b = ww.Batch(ctx)
    got = b.run(units)
    hits = b.hits()
    for i, (lo, hi) in enumerate(units):
        want, _, whits = oracle.scan_range(lo, hi, hit_cap=1000)
        assert got[i]["checksum"] == want["checksum"] and got[i]["prp_count"] == want["prp_count"], (lo, hi)
        assert sorted(h[1:] for h in hits if h[0] == i) == sorted(whits), (lo, hi)
        alone = ctx.run_range(lo, hi)
        assert alone["checksum"] == want["checksum"] and alone["total_prp_count"] == want["prp_count"], (lo, hi)
        assert sorted(alone["hits"]) == sorted(whits), (lo, hi)
        assert ctx.count_prps(lo, hi) == want["prp_count"], (lo, hi)
    assert got[0]["hits"] == 1 and got[1]["hits"] == 1 and got[2]["prp_count"] == 1 and got[5]["prp_count"] == 1
    # an empty batch, then a batch again
    assert b.run([]) == []
    assert b.run(units[:1])[0]["checksum"] == got[0]["checksum"]


def test_hit_overflow_keeps_results(ww, ctx, oracle):
    """More hits than the batch's hit buffer holds ([127, 2e6) has thousands
    of special instances): the overflow is reported, every range's checksum
    and PRP count is still right, and the records that fit are real hits."""
    units = [(127, 1_000_000), (1_000_000, 2_000_000)]
    with ww.Context(0, max_prps=1 << 20, max_hits=15000) as small:  # a fresh batch: its hit buffer only grows
        b = ww.Batch(small, max_hits=64)
        got = b.run(units)
        assert b.hit_overflow and b.hit_count > 64
        allhits = set()
        for i, (lo, hi) in enumerate(units):
            want, _, whits = oracle.scan_range(lo, hi, hit_cap=100000)
            assert got[i]["checksum"] == want["checksum"] and got[i]["prp_count"] == want["prp_count"]
            assert got[i]["hits"] == want["gpu_results"]
            allhits |= {(i, *h) for h in whits}
        kept = b.hits()
        assert len(kept) == 64 and all(h in allhits for h in kept)
        # a batch whose hits fit clears the flag
        b.run([(10**15, 10**15 + 10**6)])
        assert not b.hit_overflow
