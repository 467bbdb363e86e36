"""The request server: continuous batching keeps every request's result
(checksum, PRP count, hits, PRP list) identical to running it alone, and
admission respects the PRP-buffer memory budget."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(ww):
    c = ww.Context(0, max_prps=1 << 22, max_hits=15000)
    yield c
    c.close()


def _requests(ww, n, seed=13):
    units = ww.uneven_units(seed, n, wmin=1e5, wmax=3e7, smin=10**12, smax=2**64 - 10**9)
    return [(1000 + i, a, b) for i, (a, b) in enumerate(units)]


def test_mix_equals_alone(ww, ctx):
    reqs = _requests(ww, 40)
    srv = ww.Server(ctx, prp_pool_bytes=1 << 30, max_active=16, epoch_tiles=64)
    srv.submit(reqs)
    mixed = {r["id"]: r for r in srv.drain()}
    hits_mixed = {rid: sorted(srv.hits(rid)) for rid, _, _ in reqs}
    srv.close()
    assert set(mixed) == {r[0] for r in reqs}
    for rid, a, b in reqs:
        srv1 = ww.Server(ctx, prp_pool_bytes=1 << 30, max_active=4, epoch_tiles=4096)
        srv1.submit([(rid, a, b)])
        alone = srv1.drain()
        assert len(alone) == 1
        al = alone[0]
        assert (mixed[rid]["checksum"], mixed[rid]["prp_count"], mixed[rid]["hits"]) == \
               (al["checksum"], al["prp_count"], al["hits"]), rid
        assert sorted(srv1.hits(rid)) == hits_mixed[rid]
        srv1.close()
        ref = ctx.run_range(a, b)
        assert (al["checksum"], al["prp_count"]) == (ref["checksum"], ref["total_prp_count"])


def test_results_match_oracle_and_prp_lists(ww, ctx, oracle):
    reqs = [(1, 2**64 - 2**35, 2**64 - 2**35 + 300_000), (2, 10**12, 10**12 + 400_000),
            (3, 2276306935816523 - 7000, 2276306935816523 + 7000), (4, 127, 200_000)]
    srv = ww.Server(ctx, prp_pool_bytes=1 << 26, max_active=8, epoch_tiles=16)
    srv.submit(reqs)
    got = {}
    for _ in range(1000):
        for r in srv.step():
            got[r["id"]] = (r, srv.prps(r["id"], r["prps_stored"]))
        q, a, _ = srv.status()
        if q == 0 and a == 0:
            break
    for rid, a, b in reqs:
        r, prps = got[rid]
        want, wprps, whits = oracle.scan_range(a, b, want_prps=True, prp_cap=(b - a) // 2 + 8, hit_cap=10000)
        assert r["status"] == 0
        assert (r["checksum"], r["prp_count"], r["hits"]) == (want["checksum"], want["prp_count"],
                                                             want["gpu_results"])
        assert np.array_equal(np.sort(prps), wprps)
        assert sorted(srv.hits(rid)) == sorted(whits)
    srv.close()


def test_admission_waits_for_memory(ww, ctx):
    # each request reserves ww_prp_count_bound * 8 bytes; a pool for about one
    # request at a time forces one-at-a-time admission and still finishes
    reqs = _requests(ww, 6, seed=5)
    need = max(ww.prp_count_bound(a, b) for _, a, b in reqs) * 8
    srv = ww.Server(ctx, prp_pool_bytes=need + 4096, max_active=8, epoch_tiles=32)
    srv.submit(reqs)
    seen_active = 0
    done = []
    for _ in range(100000):
        done += srv.step()
        q, a, used = srv.status()
        seen_active = max(seen_active, a)
        assert used <= need + 4096
        if q == 0 and a == 0:
            break
    assert len(done) == len(reqs) and seen_active <= 2
    # a request that could never fit the pool is refused at submission, with
    # the rest of its call, and the server goes on serving
    big = (99, 10**15, 10**15 + 10**9)
    with pytest.raises(ww.WWError) as err:
        srv.submit([reqs[0], big])
    assert err.value.status == -6
    assert srv.status()[0] == 0
    srv.submit([(100, reqs[0][1], reqs[0][2])])
    again = srv.drain()
    assert len(again) == 1 and again[0]["status"] == 0
    srv.close()


def test_hit_overflow_is_reported_per_request(ww, ctx):
    """A step whose hit records overflow loses records of the requests active
    in it: each such request reports WW_ERR_HIT_OVERFLOW when it finishes, in
    whatever later step that is, with its checksum and PRP count still right;
    a request whose hits all fit reports OK."""
    reqs = [(1, 127, 2_000_000), (2, 10**15, 10**15 + 10**6)]
    srv = ww.Server(ctx, prp_pool_bytes=1 << 28, max_active=4, epoch_tiles=2, max_hits=16)
    srv.submit(reqs)
    done = {r["id"]: r for r in srv.drain()}
    srv.close()
    assert done[1]["status"] == -4 and done[1]["hits"] > 16
    assert done[2]["status"] == 0
    for rid, a, b in reqs:
        ref = ctx.run_range(a, b)
        assert (done[rid]["checksum"], done[rid]["prp_count"]) == (ref["checksum"], ref["total_prp_count"])


def test_failed_open_leaves_no_server(ww, ctx):
    """A server whose PRP pool cannot be allocated is not left half open:
    the open reports WW_ERR_NOMEM, a submit then finds no server, and a
    server opened next on the same context serves a request to the plain
    path's result."""
    lo, hi = 10**12, 10**12 + 100_000
    with pytest.raises(ww.WWError) as e:
        ww.Server(ctx, prp_pool_bytes=1 << 50, max_active=4)
    assert e.value.status == -6
    req = (ww.Request * 1)(ww.Request(7, lo, hi))
    assert ww.lib().ww_server_submit(ctx.h, req, 1) == -8
    srv = ww.Server(ctx, prp_pool_bytes=1 << 26, max_active=4)
    srv.submit([(7, lo, hi)])
    (r,) = srv.drain()
    srv.close()
    ref = ctx.run_range(lo, hi)
    assert (r["checksum"], r["prp_count"]) == (ref["checksum"], ref["total_prp_count"])


def test_calls_out_of_order_are_refused(ww, ctx):
    """Without an open server every call reports WW_ERR_STATE; closing is
    idempotent; an empty submit is a no-op; a request's PRP list can be
    asked for once it is done, and not before or for an unknown id."""
    L = ww.lib()
    n = C.c_uint32(0)
    q, a, u = C.c_uint32(0), C.c_uint32(0), C.c_uint64(0)
    assert L.ww_server_close(ctx.h) == 0
    assert L.ww_server_step(ctx.h, None, 0, C.byref(n)) == -8
    assert L.ww_server_status(ctx.h, C.byref(q), C.byref(a), C.byref(u)) == -8
    assert L.ww_server_hits(ctx.h, 1, None, 0, C.byref(n)) == -8
    assert L.ww_server_close(ctx.h) == 0
    srv = ww.Server(ctx, prp_pool_bytes=1 << 26, max_active=4)
    srv.submit([])
    assert srv.status() == (0, 0, 0)
    assert L.ww_server_prps(ctx.h, 42, None, 0, C.byref(u)) == -8  # no such request
    srv.submit([(42, 10**12, 10**12 + 200_000)])
    (r,) = srv.drain()
    assert r["id"] == 42 and len(srv.prps(42, r["prps_stored"])) == r["prp_count"]
    srv.close()
    srv.close()


def test_requests_admitted_mid_flight_equal_alone_and_oracle(ww, ctx, oracle):
    """Continuous batching: requests are submitted between steps while
    others are on the device (widths across two decades, 2e5 to 2e7, plus
    the known Wieferich and WSS windows; two tiles of 2^20 numbers per step,
    so most requests take several steps).  Every finished request equals its
    run alone through the context API and the oracle: checksum, PRP count,
    hit records and PRP list."""
    units = ww.uneven_units(29, 30, wmin=2e5, wmax=2e7, smin=10**12, smax=2**64 - 10**8)
    reqs = [(5000 + i, a, b) for i, (a, b) in enumerate(units)]
    reqs.insert(7, (4998, 2276306935816523 - 5000, 2276306935816523 + 5000))
    reqs.insert(15, (4999, 338772621946054253 - 5000, 338772621946054253 + 5000))
    srv = ww.Server(ctx, prp_pool_bytes=1 << 28, max_active=8, epoch_tiles=2, store_prps=True)
    pending = list(reqs)
    srv.submit(pending[:5])
    pending = pending[5:]
    got, admitted_while_busy, steps = {}, 0, 0
    while len(got) < len(reqs) and steps < 20000:
        if pending and steps % 2 == 1:  # two more requests every other step, while others run
            q, active, _ = srv.status()
            admitted_while_busy += active > 0
            srv.submit(pending[:2])
            pending = pending[2:]
        for r in srv.step():
            got[r["id"]] = (r, srv.prps(r["id"], r["prps_stored"]), sorted(srv.hits(r["id"])))
        steps += 1
    srv.close()
    assert len(got) == len(reqs)
    assert admitted_while_busy >= 8  # the submissions really overlapped running requests
    for rid, a, b in reqs:
        r, prps, hits = got[rid]
        alone = ctx.run_range(a, b)
        want, wprps, whits = oracle.scan_range(a, b, want_prps=True, prp_cap=(b - a) // 2 + 8, hit_cap=10000)
        assert r["status"] == 0, rid
        assert (r["checksum"], r["prp_count"], r["hits"]) == \
               (alone["checksum"], alone["total_prp_count"], alone["result_count"]), rid
        assert (r["checksum"], r["prp_count"], r["hits"]) == \
               (want["checksum"], want["prp_count"], want["gpu_results"]), rid
        assert np.array_equal(np.sort(prps), wprps), rid
        assert hits == sorted(whits), rid
    assert got[4998][0]["hits"] >= 1 and got[4999][0]["hits"] >= 1
