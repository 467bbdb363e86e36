"""CUDA path against the oracle and the reference fixtures, through the C ABI.

Bit-exact everywhere: PRP sets (digests of the sorted list), per-prime
digits, checksums, hit records and counts."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import sample_names

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(ww):
    c = ww.Context(0, max_prps=1 << 22, max_hits=15000)
    yield c
    c.close()


def test_digits_kernel_matches_oracle(ww, oracle, ref_terms):
    for name in sample_names(ref_terms):
        ps = ref_terms[name + "_p"]
        d = ww.digits(ps)
        w, s = oracle.list_digits(ps)
        assert np.array_equal(d[:, 0:2], w), name
        assert np.array_equal(d[:, 2:4], s), name
        assert np.array_equal((d[:, 1] & 0xFFFFFFFF).astype(np.uint32), ref_terms[name + "_wterm"]), name
        assert np.array_equal((d[:, 3] & 0xFFFFFFFF).astype(np.uint32), ref_terms[name + "_sterm"]), name


def test_digits_kernel_random_list(ww, oracle):
    ps, _ = oracle.random_primes(7, 1 << 14)
    d = ww.digits(ps)
    w, s = oracle.list_digits(ps)
    assert np.array_equal(d[:, 0:2], w) and np.array_equal(d[:, 2:4], s)


def test_random_prime_list_matches_oracle(ww, oracle):
    got, used = ww.random_primes(7, 5000)
    want, used_o = oracle.random_primes(7, 5000)
    assert np.array_equal(got, want) and used == used_o


def _digest(arr):
    arr = np.sort(np.asarray(arr, dtype=np.uint64))
    return arr.size, int(arr.sum(dtype=np.uint64)), hashlib.sha256(arr.astype("<u8").tobytes()).hexdigest()


def test_sieve_prp_sets_match_reference(ctx, ref_prps):
    for name, r in ref_prps.items():
        ctx.clear_results()
        ctx.clear_segment()
        ctx.sieve_prp(r["lo"], r["hi"])
        ctx.sync()
        c = ctx.counters()
        assert c["overflow"] == 0, name
        lst = ctx.prps()
        assert _digest(lst) == (r["count"], r["sum_mod_2_64"], r["sha256"]), name


@pytest.mark.parametrize("lo,width", [(127, 1 << 28), (2**20 - 1001, 1 << 27), (2**32 - 2**26 + 1, 1 << 27),
                                      (2**63 - 2**26 + 7, (1 << 27) + 12345), (2**64 - 2**28 - 1, 1 << 28)])
def test_sieve_depth_keeps_the_prp_set(ww, lo, width):
    """The large deep primes (marked once per launch above 2^20) remove only
    composites that can never be base-2 pseudoprimes: the PRP list is the
    same at every depth -- over ranges that hold the deep primes themselves
    (127 .. 2^28), pseudoprimes with large factors, both sides of 2^32 and
    2^63, and the end of the domain.  Depth 20 is the path pinned to the
    reference's fixtures and random ranges."""
    hi = lo + width
    with ww.Context(0, max_prps=ww.prp_count_bound(lo, hi), max_hits=15000) as c:
        digests = {}
        for bits in (20, 24, 26, 28):
            c.set_sieve_depth(bits)
            assert c.sieve_depth() == bits
            c.clear_results()
            c.clear_segment()
            c.sieve_prp(lo, hi)
            c.sync()
            assert c.counters()["overflow"] == 0
            digests[bits] = _digest(c.prps())
        assert len(set(digests.values())) == 1, digests
        assert c.count_prps(lo, hi) == digests[20][0]  # the counting launch, at depth 28


def test_sieve_shapes_give_the_same_prp_set(ww, ref_prps):
    """Both segment shapes of the context's sieve (2^20 numbers for 512
    threads, 2^19 for 256) give the reference's PRP sets."""
    with ww.Context(0, max_prps=1 << 22, max_hits=15000) as c:
        for shape in (1, 2, 0):
            c.set_sieve_shape(shape)
            assert c.sieve_shape() == shape
            for name, r in ref_prps.items():
                c.clear_results()
                c.clear_segment()
                c.sieve_prp(r["lo"], r["hi"])
                c.sync()
                assert _digest(c.prps()) == (r["count"], r["sum_mod_2_64"], r["sha256"]), (shape, name)
        with pytest.raises(ww.WWError):
            c.set_sieve_shape(3)


def _order_of_two(r: int) -> int:
    m, fac, d = r - 1, [], 2
    x = m
    while d * d <= x:
        if x % d == 0:
            fac.append(d)
            while x % d == 0:
                x //= d
        d += 1
    if x > 1:
        fac.append(x)
    o = m
    for q in fac:
        while o % q == 0 and pow(2, o // q, r) == 1:
            o //= q
    return o


def test_large_prime_table_orders(ww):
    """The device's table of large deep primes (built by a sieve on the host
    and an order kernel) against an independent computation: the first and
    last 1500 rows at depth 26 are the primes there, with ord_r(2) exact --
    an order too large would let the sieve mark a pseudoprime -- and the
    table's length is the prime count of (2^20, 2^26)."""
    import itertools

    import sympy

    with ww.Context(0, max_prps=1 << 10, max_hits=1024) as c:
        r0, o0, total = c.deep_table(26, 0, 1500)
        assert total == sympy.primepi(2**26) - sympy.primepi(2**20)
        r1, o1, _ = c.deep_table(26, total - 1500, 1500)
    want0 = [int(p) for p in itertools.islice(sympy.primerange(2**20, 2**26), 1500)]
    assert [int(x) for x in r0] == want0
    assert [int(x) for x in r1] == [int(p) for p in sympy.primerange(2**26 - 60000, 2**26)][-1500:]
    for r, o in list(zip(r0, o0)) + list(zip(r1, o1)):
        assert int(o) == _order_of_two(int(r)), r
    # a large prime of small order: 616318177 divides 2^37 - 1 (depth 30)
    idx = int(sympy.primepi(616318177) - sympy.primepi(2**20)) - 1
    with ww.Context(0, max_prps=1 << 10, max_hits=1024) as c:
        r2, o2, _ = c.deep_table(30, idx, 1)
    assert (int(r2[0]), int(o2[0])) == (616318177, 37)


@pytest.mark.parametrize("tail", [12345, (1 << 19) + 777, (1 << 20) - 3])
def test_multi_round_launch_equals_single_round_pieces(ww, tail):
    """A launch of 396 whole 2^20-number segments plus a partial one of
    several lengths (more segments than the 296 resident CTAs take in one
    round, with the large deep primes' marks) gives the same PRP list as the
    range sieved in pieces of one round each."""
    lo = 2**63 + 2**40 + 1
    hi = lo + (396 << 20) + tail
    with ww.Context(0, max_prps=ww.prp_count_bound(lo, hi), max_hits=15000) as c:
        c.set_sieve_shape(1)
        c.clear_results()
        c.clear_segment()
        c.sieve_prp(lo, hi)
        c.sync()
        whole = _digest(c.prps())
        n_whole = c.count_prps(lo, hi)
        parts = []
        a = lo
        while a < hi:
            b = min(a + (200 << 20), hi)
            c.clear_segment()
            c.sieve_prp(a, b)
            c.sync()
            parts.append(c.prps())
            a = b
    assert whole == _digest(np.concatenate(parts))
    assert n_whole == whole[0]


def test_count_prps_depths_agree_to_2p32(ww):
    """[127, 2^32) holds every deep prime and many base-2 pseudoprimes with a
    factor above 2^20: its PRP count is the same at depths 20 and 30."""
    with ww.Context(0, max_prps=1 << 10, max_hits=1024) as c:
        c.set_sieve_depth(20)
        n20 = c.count_prps(127, 2**32)
        c.set_sieve_depth(30)
        assert c.count_prps(127, 2**32) == n20
        with pytest.raises(ww.WWError):
            c.set_sieve_depth(31)
        with pytest.raises(ww.WWError):
            c.set_sieve_depth(19)


def test_sieve_prp_list_inverse(ww):
    """g_invert holds p^-1 mod 2^64 for each listed p (getsegprimes.cl:291-296)."""
    import torch

    L = ww.lib()
    dev = torch.device("cuda", 0)
    cap = 1 << 16
    prime = torch.zeros(cap, dtype=torch.int64, device=dev)
    inv = torch.zeros(cap, dtype=torch.int64, device=dev)
    pc = torch.zeros(2, dtype=torch.int32, device=dev)
    ovf = torch.zeros(1, dtype=torch.int32, device=dev)
    lo, idx = ww.find_wheel_offset(2**64 - 10**6 - 1)
    st = torch.cuda.current_stream(dev).cuda_stream
    ww.check(L.ww_launch_getsegprimes(lo, 2**64 - 1, idx, prime.data_ptr(), inv.data_ptr(), pc.data_ptr(), cap,
                                      ovf.data_ptr(), st), "getsegprimes")
    torch.cuda.synchronize(dev)
    n = int(pc[0].item())
    assert n > 20000 and int(ovf.item()) == 0
    p = prime[:n].cpu().numpy().view(np.uint64)
    q = inv[:n].cpu().numpy().view(np.uint64)
    with np.errstate(over="ignore"):
        assert np.all(p * q == np.uint64(1))


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("name", ["small_3e6", "cross_2p32", "near_top_2e6", "wieferich_special_window",
                                  "wss_special_window", "mid_2p48", "config1_5e7", "top_1e8", "cross_2p62",
                                  "cross_2p63"])
def test_pipeline_matches_reference(ctx, ref_ranges, name, fused):
    r = ref_ranges[name]
    got = ctx.run_range(r["lo"], r["hi"], fused=fused)
    assert got["overflow"] == 0
    assert got["total_prp_count"] == r["prp_count"]
    assert "%016X" % got["checksum"] == r["checksum"]
    assert got["result_count"] == r["cpu_results"]


def test_segmented_run_equals_whole(ctx, ref_ranges):
    r = ref_ranges["small_3e6"]
    a = ctx.run_range(r["lo"], r["hi"], segment=123_457)
    assert "%016X" % a["checksum"] == r["checksum"]
    assert a["total_prp_count"] == r["prp_count"]
    assert a["max_prp_count"] < r["prp_count"]


def test_hits_match_oracle(ctx, oracle):
    lo, hi = 127, 2_000_000
    got = ctx.run_range(lo, hi)
    _, _, want = oracle.scan_range(lo, hi, hit_cap=100000)
    assert sorted(got["hits"]) == sorted(want)


def test_count_prps_matches_reference(ctx, ref_ranges):
    """ww_count_prps (the sieve kernel counting without a list) against the
    reference's PRP counts, including the 2^34-wide range, which is one full
    counting piece, and a range that ends at 2^64 - 1."""
    import json
    from pathlib import Path

    for name in ("small_3e6", "config1_5e7", "cross_2p32", "cross_2p63", "near_top_2e6", "top_1e8"):
        r = ref_ranges[name]
        assert ctx.count_prps(r["lo"], r["hi"]) == r["prp_count"], name
    long = json.loads((Path(__file__).resolve().parent / "golden" / "ref_long.json").read_text())["config3"]
    assert ctx.count_prps(long["lo"], long["hi"]) == long["prp_count"]
    # split at an odd point: the two counts add up
    r = ref_ranges["config1_5e7"]
    mid = 12_345_679
    assert ctx.count_prps(r["lo"], mid) + ctx.count_prps(mid, r["hi"]) == r["prp_count"]
    assert ctx.count_prps(2**64 - 3, 2**64 - 1) == 0


def test_host_list_pipeline_matches_loaded_list(ww, oracle, ref_terms):
    """ww_test_prps_host (chunked copy/test overlap) against ww_load_prps +
    ww_test_prps and the oracle: checksum, count and hits, over a list that
    spans several chunks of both buffer halves, including the known hits."""
    ps, _ = ww.random_primes(11, 3 * (1 << 20) + 12345)
    ps = np.concatenate([ps, ref_terms["known_hits_p"], ref_terms["small_p"]])
    with ww.Context(0, max_prps=1 << 21, max_hits=15000) as c:
        c.clear_results()
        c.test_prps_host(ps)
        got = c.counters()
        got_hits = sorted(c.hits())
    with ww.Context(0, max_prps=ps.size, max_hits=15000) as c:
        c.load_prps(ps)
        c.clear_results()
        c.test_prps()
        c.sync()
        want = c.counters()
        want_hits = sorted(c.hits())
    assert got["checksum"] == want["checksum"] and got["total_prp_count"] == ps.size == want["total_prp_count"]
    assert got["result_count"] == want["result_count"] > 0 and got_hits == want_hits
    summ, ohits = oracle.test_list(ps, hit_cap=15000)
    assert summ["checksum"] == got["checksum"] and sorted(ohits) == got_hits


def test_prp_overflow_is_reported(ww, oracle):
    with ww.Context(0, max_prps=1000, max_hits=100) as c:
        c.clear_results()
        c.clear_segment()
        c.sieve_prp(127, 1_000_000)
        c.sync()
        k = c.counters()
        summ, _, _ = oracle.scan_range(127, 1_000_000)
        assert k["overflow"] & 1 and k["seg_prp_count"] == summ["prp_count"]
        with pytest.raises(ww.WWError) as e:
            c.prps()
        assert e.value.status == -3


@pytest.mark.parametrize("slack", [0, -1])
def test_prp_buffer_exact_fit(ww, ref_prps, slack):
    """A PRP buffer of exactly the range's PRP count holds the whole list
    (the reference's set); one entry less sets the overflow flag, still
    counts every PRP, and keeps the list unreadable (the reference's
    check is count > mem_size, main.cpp:801-805)."""
    r = ref_prps["prp_top"]
    with ww.Context(0, max_prps=r["count"] + slack, max_hits=16) as c:
        c.clear_results()
        c.clear_segment()
        c.sieve_prp(r["lo"], r["hi"])
        c.sync()
        k = c.counters()
        assert k["seg_prp_count"] == r["count"]
        if slack == 0:
            assert k["overflow"] == 0
            assert _digest(c.prps()) == (r["count"], r["sum_mod_2_64"], r["sha256"])
        else:
            assert k["overflow"] & 1
            with pytest.raises(ww.WWError) as e:
                c.prps()
            assert e.value.status == -3


def test_hit_buffer_exact_fit(ww, ref_ranges):
    """A hit buffer of exactly the range's hit count keeps every hit with
    no overflow flag; one less overflows (the reference's check is
    count > numresults, main.cpp:811-814)."""
    r = ref_ranges["small_3e6"]
    for cap, over in ((r["cpu_results"], False), (r["cpu_results"] - 1, True)):
        with ww.Context(0, max_prps=1 << 19, max_hits=cap) as c:
            got = c.run_range(r["lo"], r["hi"])
            assert got["result_count"] == r["cpu_results"]
            assert "%016X" % got["checksum"] == r["checksum"]
            assert bool(got["overflow"] & 2) == over
            if not over:
                assert len(got["hits"]) == r["cpu_results"]


def test_hit_overflow_is_reported(ww):
    with ww.Context(0, max_prps=1 << 20, max_hits=10) as c:
        got = c.run_range(127, 1_000_000)
        assert got["overflow"] & 2 and got["result_count"] > 10
        with pytest.raises(ww.WWError) as e:
            c.hits()
        assert e.value.status == -4


class _KernelSequence:
    """The reference kernel sequence clearresult, clearn, getsegprimes,
    wieferich, wallsunsun over one range, on caller-owned device memory."""

    def __init__(self, ww, r, cap=1 << 18, nres=15000):
        import torch

        dev = torch.device("cuda", 0)
        self.ww, self.L, self.r, self.cap, self.nres = ww, ww.lib(), r, cap, nres
        e = lambda n, dt: torch.empty(n, dtype=dt, device=dev)  # noqa: E731
        self.prime, self.inv, self.one = e(cap, torch.int64), e(cap, torch.int64), e(2 * cap, torch.int64)
        self.sp, self.rem, self.quot, self.res = (e(nres, torch.int64), e(nres, torch.int32), e(nres, torch.int32),
                                                  e(nres, torch.int32))
        self.cks, self.total = e(1, torch.int64), e(1, torch.int64)
        self.rc, self.pc, self.ovf = e(1, torch.int32), e(2, torch.int32), torch.zeros(1, dtype=torch.int32,
                                                                                         device=dev)

    def launch(self, st, fused=False):
        ww, L, r, cap, nres = self.ww, self.L, self.r, self.cap, self.nres
        P = lambda t: t.data_ptr()  # noqa: E731
        start, idx = ww.find_wheel_offset(r["lo"])
        ww.check(L.ww_launch_clearresult(P(self.cks), P(self.rc), P(self.total), P(self.pc), st), "clearresult")
        ww.check(L.ww_launch_clearn(P(self.pc), st), "clearn")
        ww.check(L.ww_launch_getsegprimes(start, r["hi"], idx, P(self.prime), P(self.inv), P(self.pc), cap,
                                          P(self.ovf), st), "gsp")
        if fused:  # both tests in one launch
            ww.check(L.ww_launch_test_prps(P(self.pc), P(self.prime), P(self.inv), P(self.sp), P(self.rem),
                                           P(self.quot), P(self.res), P(self.cks), P(self.rc), P(self.total), cap,
                                           nres, P(self.ovf), st), "test_prps")
            return
        ww.check(L.ww_launch_wieferich(P(self.pc), P(self.prime), P(self.inv), P(self.one), P(self.sp), P(self.rem),
                                       P(self.quot), P(self.res), P(self.cks), P(self.rc), P(self.total), cap, nres,
                                       P(self.ovf), st), "wieferich")
        ww.check(L.ww_launch_wallsunsun(P(self.pc), P(self.prime), P(self.inv), P(self.one), P(self.sp),
                                        P(self.rem), P(self.quot), P(self.res), P(self.cks), P(self.rc), cap, nres,
                                        P(self.ovf), st), "wallsunsun")

    def check(self, label=""):
        r = self.r
        assert int(self.ovf.item()) == 0, label
        assert int(self.total.item()) == r["prp_count"], label
        assert "%016X" % (int(self.cks.item()) % 2**64) == r["checksum"], label
        assert int(self.rc.item()) == r["cpu_results"], label


def test_kernel_shaped_launchers_on_torch_memory(ww, ref_ranges):
    """The reference kernel sequence on caller-owned device memory and stream."""
    import torch

    seq = _KernelSequence(ww, ref_ranges["cross_2p32"])
    s = torch.cuda.Stream(torch.device("cuda", 0))
    seq.launch(s.cuda_stream)
    s.synchronize()
    seq.check()


@pytest.mark.parametrize("name", ["small_3e6", "wieferich_special_window", "wss_special_window", "cross_2p63"])
def test_fused_kernel_shaped_launcher(ww, ref_ranges, name):
    """ww_launch_test_prps in place of the wieferich + wallsunsun pair: the
    same checksum, counts and hit records as the reference."""
    import torch

    seq = _KernelSequence(ww, ref_ranges[name], cap=1 << 18, nres=15000)
    s = torch.cuda.Stream(torch.device("cuda", 0))
    seq.launch(s.cuda_stream, fused=True)
    s.synchronize()
    seq.check(name)


def test_kernel_shaped_launchers_on_many_streams(ww, ref_ranges):
    """The kernel-shaped launchers lend each stream a work cursor from a
    fixed pool of 64 per device.  96 distinct streams, all queued before any
    finishes: streams that find no free slot take the static split, the
    second round reuses slots whose work has completed, and every stream's
    results equal the reference's.  The default stream runs one too."""
    import torch

    cudart = pytest.importorskip("cuda.bindings.runtime")
    dev = torch.device("cuda", 0)
    names = ["cross_2p32", "wieferich_special_window", "near_top_2e6", "cross_2p63", "wss_special_window"]
    handles = []
    try:
        for _ in range(96):
            err, h = cudart.cudaStreamCreateWithFlags(cudart.cudaStreamNonBlocking)
            assert err == cudart.cudaError_t.cudaSuccess
            handles.append(h)
        seqs = [_KernelSequence(ww, ref_ranges[names[i % len(names)]], cap=1 << 17, nres=64)
                for i in range(len(handles))]
        default = _KernelSequence(ww, ref_ranges["mid_2p48"], cap=1 << 17, nres=64)
        torch.cuda.synchronize(dev)
        for rnd in range(2):
            for h, q in zip(handles, seqs):
                q.launch(int(h))
            default.launch(0)
            torch.cuda.synchronize(dev)
            for i, q in enumerate(seqs):
                q.check("round %d stream %d" % (rnd, i))
            default.check("default stream")
    finally:
        torch.cuda.synchronize(dev)
        for h in handles:
            cudart.cudaStreamDestroy(h)


def test_kernel_shaped_launchers_from_host_threads(ww, ref_ranges):
    """Four host threads, each with its own stream and buffers, queue the
    reference kernel sequence five times each at the same time (the foreign
    calls release the interpreter lock): every stream's results equal the
    reference's."""
    import threading

    import torch

    dev = torch.device("cuda", 0)
    names = ["cross_2p32", "wieferich_special_window", "near_top_2e6", "wss_special_window"]
    streams = [torch.cuda.Stream(dev, priority=-1 if i % 2 else 0) for i in range(4)]
    seqs = [_KernelSequence(ww, ref_ranges[n], cap=1 << 17, nres=64) for n in names]
    torch.cuda.synchronize(dev)
    errors = []

    def work(k):
        try:
            torch.cuda.set_device(dev)
            for _ in range(5):
                seqs[k].launch(streams[k].cuda_stream)
        except Exception as e:  # noqa: BLE001 -- reported below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    torch.cuda.synchronize(dev)
    assert not errors, errors
    for k, q in enumerate(seqs):
        q.check("thread %d" % k)


def test_kernel_shaped_launchers_under_graph_capture(ww, ref_ranges):
    """Launches captured into a CUDA graph (no cursor there) replay to the
    reference's results, twice."""
    import torch

    seq = _KernelSequence(ww, ref_ranges["wieferich_special_window"], cap=1 << 17, nres=64)
    s = torch.cuda.Stream(torch.device("cuda", 0))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
        seq.launch(s.cuda_stream)
    for _ in range(2):
        seq.ovf.zero_()
        g.replay()
        torch.cuda.synchronize()
        seq.check()


def test_context_buffers_drive_the_kernel_shaped_launchers(ww, ref_ranges):
    """ww_get_buffers hands out the context's own device buffers and stream:
    the kernel-shaped sequence run on them leaves counters and hits that
    the context's read-backs return, equal to the reference's."""
    r = ref_ranges["wss_special_window"]
    L = ww.lib()
    with ww.Context(0, max_prps=1 << 18, max_hits=64) as c:
        b = c.buffers()
        assert b.prp_capacity == 1 << 18 and b.hit_capacity == 64
        start, idx = ww.find_wheel_offset(r["lo"])
        ww.check(L.ww_launch_clearresult(b.checksum, b.result_count, b.total_prp_count, b.primecount, b.stream),
                 "clearresult")
        ww.check(L.ww_launch_clearn(b.primecount, b.stream), "clearn")
        ww.check(L.ww_launch_getsegprimes(start, r["hi"], idx, b.prime, b.invert, b.primecount, b.prp_capacity,
                                          b.overflow, b.stream), "gsp")
        ww.check(L.ww_launch_wieferich(b.primecount, b.prime, b.invert, b.one, b.special_prime, b.rem, b.quot,
                                       b.result, b.checksum, b.result_count, b.total_prp_count, b.prp_capacity,
                                       b.hit_capacity, b.overflow, b.stream), "wieferich")
        ww.check(L.ww_launch_wallsunsun(b.primecount, b.prime, b.invert, b.one, b.special_prime, b.rem, b.quot,
                                        b.result, b.checksum, b.result_count, b.prp_capacity, b.hit_capacity,
                                        b.overflow, b.stream), "wallsunsun")
        c.sync()
        k = c.counters()
        assert k["overflow"] == 0 and k["total_prp_count"] == r["prp_count"]
        assert "%016X" % k["checksum"] == r["checksum"]
        assert k["result_count"] == r["cpu_results"] == len(c.hits())
        assert sorted(c.hits()) == sorted(_range_hits(ww, r))


def _range_hits(ww, r):
    with ww.Context(0, max_prps=1 << 18, max_hits=64) as c:
        return c.run_range(r["lo"], r["hi"])["hits"]


def test_bad_arguments_are_rejected(ww):
    with ww.Context(0, max_prps=1024, max_hits=16) as c:
        L = ww.lib()
        # wheel index that does not belong to the start
        assert L.ww_sieve_prp(c.h, 127, 1000, 3) == -2
        # start below 127 (main.cpp:1265-1269 clamps; the kernel refuses)
        assert L.ww_sieve_prp(c.h, 121, 1000, 7) == -2
        # empty range
        assert L.ww_sieve_prp(c.h, 127, 127, 0) == -2
        c.sync()
        assert c.counters()["seg_prp_count"] == 0


def test_failed_reserve_leaves_context_usable(ww, ref_ranges):
    """A PRP buffer that cannot be allocated leaves none: the reserve reports
    WW_ERR_NOMEM, the sieve then refuses with WW_ERR_STATE, and a reserve
    that fits makes the context run a range to the reference's result."""
    r = ref_ranges["cross_2p32"]
    with ww.Context(0, max_prps=1 << 18, max_hits=64) as c:
        with pytest.raises(ww.WWError) as e:
            c.reserve(1 << 40, 64)
        assert e.value.status == -6
        start, idx = ww.find_wheel_offset(r["lo"])
        assert ww.lib().ww_sieve_prp(c.h, start, r["hi"], idx) == -8
        c.reserve(1 << 18, 64)
        got = c.run_range(r["lo"], r["hi"])
        assert got["total_prp_count"] == r["prp_count"]
        assert "%016X" % got["checksum"] == r["checksum"]


def test_sync_and_marker_time_out_then_complete(ww):
    """ww_sync and ww_wait_marker give up with WW_ERR_TIMEOUT while work is
    still running (main.cpp:329-446 poll the same way), the context stays
    usable, and a later wait completes: the counters then hold three passes
    of the tests over one sieved list."""
    lo = 2**64 - 2**35
    hi = lo + 2**32
    L = ww.lib()
    with ww.Context(0, max_prps=1 << 27, max_hits=64) as c:
        one = c.run_range(lo, hi)
        c.clear_results()
        c.clear_segment()
        c.sieve_prp(lo, hi)
        for _ in range(3):  # about 0.3 s of queued work
            c.test_prps()
        c.marker(0)
        assert L.ww_wait_marker(c.h, 0, 1) == -5
        assert L.ww_sync(c.h, 1) == -5
        c.sync()
        assert L.ww_wait_marker(c.h, 0, 1) == 0
        k = c.counters()
        assert k["overflow"] == 0
        assert k["total_prp_count"] == 3 * one["total_prp_count"]
        assert k["checksum"] == (3 * one["checksum"]) % 2**64


def test_pipe_bench_runs(ww):
    for mode in range(6):
        ops, ms = ww.pipe_bench(mode)
        assert ops > 1e11 and ms > 0
