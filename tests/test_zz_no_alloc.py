"""The allocation-free batched search (ww_batch_run_noalloc).

Some callers cannot allocate device memory -- a host that reserves the
whole card for its own memory pool, or a latency-bound loop that cannot
afford an allocation's device-wide synchronisation.  This entry point runs
the batched search with its scratch in a fixed array inside the library;
here it is called through the C ABI on buffers the test allocates, twice in
a row (the shared scratch keeps the previous call's contents), and each
call must give exactly what ww_batch_run gives.  The file sorts last so a
run that stops at the first failure has already run every other test."""
from __future__ import annotations

import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _noalloc(ww, units, hit_cap=4096, with_unit=True):
    """One call through the C ABI.  hit_cap = 0 passes hits = NULL;
    with_unit = False passes hit_unit = NULL (records then carry unit -1)."""
    import torch

    L = ww.lib()
    dev = torch.device("cuda", 0)
    n = len(units)
    out = torch.zeros(max(n, 1) * C.sizeof(ww.UnitResult), dtype=torch.uint8, device=dev)
    hits = torch.zeros(max(hit_cap, 1) * C.sizeof(ww.Hit), dtype=torch.uint8, device=dev)
    hit_unit = torch.full((max(hit_cap, 1),), -1, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    arr = (ww.Unit * max(n, 1))()
    for i, (a, b) in enumerate(units):
        arr[i].start, arr[i].end = a, b
    stream = torch.cuda.current_stream(dev).cuda_stream
    ww.check(L.ww_batch_run_noalloc(arr, n, out.data_ptr(), hits.data_ptr() if hit_cap else None,
                                    hit_unit.data_ptr() if with_unit else None, hit_cap, count.data_ptr(), stream),
             "ww_batch_run_noalloc")
    torch.cuda.synchronize(dev)
    res = (ww.UnitResult * max(n, 1)).from_buffer_copy(out.cpu().numpy().tobytes())[:n]
    nh = int(count.item())
    hh = (ww.Hit * max(hit_cap, 1)).from_buffer_copy(hits.cpu().numpy().tobytes())
    hu = hit_unit.cpu().numpy()
    results = [(r.checksum, r.prp_count, r.hits) for r in res]
    hit_list = sorted((int(hu[i]), hh[i].p, hh[i].result, hh[i].rem, hh[i].quot) for i in range(min(nh, hit_cap)))
    return results, hit_list, nh


def test_noalloc_matches_batch_twice(ww):
    units = ww.uneven_units(11, 48, wmin=1e5, wmax=2e8)
    units += [(127, 400_000), (2276306935816523 - 3000, 2276306935816523 + 3000), (5000, 5000)]
    with ww.Context(0, max_prps=1 << 20, max_hits=15000) as ctx:
        b = ww.Batch(ctx)
        b.set_config(8192, 256, 1)
        want = [(r["checksum"], r["prp_count"], r["hits"]) for r in b.run(units)]
        want_hits = sorted(b.hits())
    for _ in range(2):  # the second call starts from the first call's scratch contents
        got, hits, nh = _noalloc(ww, units)
        assert got == want
        assert nh == len(want_hits) and hits == want_hits


@pytest.mark.parametrize("hit_cap", [100, 4096])
def test_noalloc_reports_more_hits_than_records(ww, ref_ranges, hit_cap):
    """Two overlapping copies of [127, 5e7) find 2 x 3890 hits: more than
    the caller's records (100) or the scratch's (4096).  *hit_count still
    gives the total, each range its own count and the reference's
    checksum, and every record kept is one of the hits that ww_batch_run
    finds."""
    r = ref_ranges["config1_5e7"]
    units = [(r["lo"], r["hi"]), (r["lo"], r["hi"])]
    with ww.Context(0, max_prps=1 << 20, max_hits=15000) as ctx:
        b = ww.Batch(ctx)
        b.set_config(8192, 256, 1)
        b.run(units)
        want_hits = set(b.hits())
    got, hits, nh = _noalloc(ww, units, hit_cap=hit_cap)
    assert nh == 2 * r["cpu_results"]
    for checksum, prp_count, unit_hits in got:
        assert "%016X" % checksum == r["checksum"]
        assert prp_count == r["prp_count"] and unit_hits == r["cpu_results"]
    assert len(hits) == hit_cap and set(hits) <= want_hits


def _batch(ww, units):
    with ww.Context(0, max_prps=1 << 20, max_hits=15000) as ctx:
        b = ww.Batch(ctx)
        b.set_config(8192, 256, 1)
        want = [(r["checksum"], r["prp_count"], r["hits"]) for r in b.run(units)]
        return want, sorted(b.hits())


def test_noalloc_optional_outputs_and_empty_batch(ww):
    """hit_unit = NULL, and hits = NULL with hit_cap = 0, leave the per-range
    results and the hit count as they are; an empty batch reports nothing."""
    units = [(2276306935816523 - 3000, 2276306935816523 + 3000), (127, 200_000)]
    want, want_hits = _batch(ww, units)
    got, hits, nh = _noalloc(ww, units, with_unit=False)
    assert got == want and nh == len(want_hits)
    assert [h[1:] for h in hits] == sorted(h[1:] for h in want_hits)
    assert all(h[0] == -1 for h in hits)  # hit_unit untouched
    got, hits, nh = _noalloc(ww, units, hit_cap=0)
    assert got == want and nh == len(want_hits) and hits == []
    got, hits, nh = _noalloc(ww, [])
    assert got == [] and nh == 0 and hits == []


def test_noalloc_smaller_batch_after_larger(ww):
    """A call with fewer ranges than the one before ignores the scratch the
    earlier call left beyond its own ranges."""
    big = ww.uneven_units(11, 96, wmin=1e5, wmax=5e7) + [(127, 300_000)]
    small = [(10**13 + 30, 10**13 + 30 + 2_000_000), (2276306935816523 - 2000, 2276306935816523 + 2000)]
    want_big, want_big_hits = _batch(ww, big)
    want_small, want_small_hits = _batch(ww, small)
    got, hits, nh = _noalloc(ww, big)
    assert got == want_big and hits == want_big_hits
    got, hits, nh = _noalloc(ww, small)
    assert got == want_small and hits == want_small_hits and nh == len(want_small_hits)


def test_noalloc_rejects_too_many_ranges(ww):
    L = ww.lib()
    n = 4097
    arr = (ww.Unit * n)()
    for i in range(n):
        arr[i].start, arr[i].end = 10**12 + 1000 * i, 10**12 + 1000 * i + 500
    rc = L.ww_batch_run_noalloc(arr, n, None, None, None, 0, None, None)
    assert rc == -2
    assert b"4096" in L.ww_last_error()
