"""libwwcuda.so without a GPU: the library loads, exports every entry point
include/wwcuda.h declares, and its host side (the reference's main.cpp
helpers and the host instantiation of the kernels' arithmetic) agrees with
the oracle and the reference fixtures."""
from __future__ import annotations

import ctypes as C
import subprocess

import numpy as np
import pytest

from conftest import PKG, sample_names


def test_library_exports_header_symbols(ww):
    declared = ww.header_symbols()
    assert len(declared) >= 35
    out = subprocess.run(["nm", "-D", "--defined-only", str(ww.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for s in declared:  # and they resolve through the dynamic loader
        getattr(ww.lib(), s)
    assert ww.lib().ww_abi_version() == 1


def test_binding_covers_header(ww):
    assert set(ww.header_symbols()) == set(ww.exported_symbols())


def test_no_device_is_reported_not_faked(ww):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ww.WWError) as e:
        ww.Context(0)
    assert e.value.status in (-9, -1)


def test_host_twin_digits_match_oracle_and_reference(ww, oracle, ref_terms):
    for name in sample_names(ref_terms):
        ps = ref_terms[name + "_p"]
        d = ww.selftest_digits(ps)
        w, s = oracle.list_digits(ps)
        assert np.array_equal(d[:, 0:2], w), name
        assert np.array_equal(d[:, 2:4], s), name
        assert np.array_equal((d[:, 1] & 0xFFFFFFFF).astype(np.uint32), ref_terms[name + "_wterm"]), name
        assert np.array_equal((d[:, 3] & 0xFFFFFFFF).astype(np.uint32), ref_terms[name + "_sterm"]), name


def test_host_twin_random_primes(ww, oracle):
    ps, _ = oracle.random_primes(7, 3000)
    d = ww.selftest_digits(ps)
    w, s = oracle.list_digits(ps)
    assert np.array_equal(d[:, 0:2], w) and np.array_equal(d[:, 2:4], s)
    assert np.all(d[:, 2] == 0)  # F_{p-(p|5)} = 0 mod p for primes


@pytest.mark.parametrize("name", ["small_3e6", "cross_2p32", "near_top_2e6", "wss_special_window"])
def test_host_twin_range(ww, ref_ranges, name):
    r = ref_ranges[name]
    got = ww.selftest_range(r["lo"], r["hi"])
    assert got["prp_count"] == r["prp_count"]
    assert "%016X" % got["checksum"] == r["checksum"]
    assert got["result_count"] == r["cpu_results"]


def test_wheel_offset_matches_reference_walk(ww, oracle):
    rng = np.random.default_rng(1)
    starts = [127, 128, 129, 133, 2**32 - 1, 2**63, 2**64 - 100, 2**64 - 60]
    starts += [int(x) for x in rng.integers(127, 2**63, 2000, dtype=np.uint64)]
    starts += list(range(127, 127 + 90))
    for s in starts:
        assert ww.find_wheel_offset(s) == oracle.wheel_offset(s), s
    with pytest.raises(ww.WWError):
        ww.find_wheel_offset(2**64 - 2)  # nothing prime to 30 left below 2^64


def test_primality_helpers(ww, oracle):
    rng = np.random.default_rng(2)
    xs = [int(x) | 1 for x in rng.integers(3, 2**64 - 1, 4000, dtype=np.uint64)]
    xs += [42799, 49141, 88357, 3825123056546413051, 2**64 - 59, 2**64 - 1, 127, 131]
    for x in xs:
        assert ww.is_prime(x) == oracle.is_prime(x), x
        assert ww.is_prp(x) == oracle.is_prp(x), x


def test_parse_number_matches_reference(ww, oracle):
    # (a hex mantissa that swallows the 'e', like "0x10e2", makes the reference
    # read past the string's end, main.cpp:1200-1201; it is not a valid input)
    for text in ["127", "6e10", "227630e10", "18446744073709551615", "338772621946054253", "1e7", "3e1"]:
        rc, val = oracle.parse_number(text)
        assert rc == 0
        assert ww.parse_number(text) == val, text
    for text in ["1e0", "2e19", "0e5"]:
        assert oracle.parse_number(text)[0] != 0
        with pytest.raises(ww.WWError):
            ww.parse_number(text)


def test_format_hits_matches_oracle(ww, oracle):
    hits = [(338772621946054253, 2, 0, 91), (2276306935816523, 1093, -1, -3), (1093, 1093, 1, 0),
            (3511, 1093, 1, 0), (42799, 1093, 1, 5), (1093, 2, 0, -7), (127, 1, 0, 0)]
    text, dropped = ww.format_hits(list(hits))
    rc, otext, odrop = oracle.format_results(list(hits))
    assert rc >= 0 and text == otext and dropped == odrop == 1
    assert text.splitlines()[0] == "127 is a WallSunSun prime"
    assert text.splitlines()[1] == "1093 is a Wieferich prime"
    assert text.splitlines()[2] == "1093 is a WallSunSun special instance (+0 -7 p)"
    with pytest.raises(ww.WWError):
        ww.format_hits([(127 * 131, 1093, 1, 0)])


def test_prp_bound_covers_fixtures(ww, ref_ranges):
    for r in ref_ranges.values():
        assert ww.prp_count_bound(r["lo"], r["hi"]) >= r["prp_count"]


def _m2_exact(op, p, x0, x1, y0, y1):
    n = p * p
    rinv = pow(2**64, -1, n)
    x, y = x0 + p * x1, y0 + p * y1
    z = (x * y if op == 0 else x * x if op == 1 else x) * rinv % n
    return z % p, z // p


def test_m2_arithmetic_edge_cases(ww):
    """The 32-bit carry-chain products (the instruction sequence the kernels
    run) against exact integer arithmetic, operand by operand, including
    the digits 0, 1, p-1 and moduli at the 2^32, 2^63 and 2^64 edges."""
    rng = np.random.default_rng(3)
    mods = [127, 131, 65521, 2**31 - 1, 4294967291, 4294967311, 2**32 + 15, 2**61 - 1, 2**62 + 135,
            9223372036854775783, 2**63 + 29, 2**64 - 59, 2**64 - 1, 2**64 - 3, 12297829382473034411]
    for p in mods:
        special = sorted({0, 1, 2, p - 1, p - 2, p // 2, (p + 1) // 2, 2**32 % p, (2**32 - 1) % p, p - 2**31 % p}
                         | {int(v) % p for v in rng.integers(0, 2**63, 6, dtype=np.uint64)})
        cases = [(a, b, c, d) for a in special for b in special[:6] for c in special[:6] for d in special]
        xy = np.array(cases, dtype=np.uint64)
        for op in (0, 1, 2):
            want = [_m2_exact(op, p, *c) for c in cases]
            for impl in (0, 1, 2, 3):
                got = ww.selftest_m2(op | impl << 4, p, xy)
                assert [tuple(map(int, g)) for g in got] == want, (p, op, impl)


def test_m2_arithmetic_random(ww):
    rng = np.random.default_rng(4)
    for _ in range(40):
        p = int(rng.integers(2**40, 2**64 - 1, dtype=np.uint64)) | 1
        cases = [tuple(int(v) % p for v in rng.integers(0, 2**64 - 1, 4, dtype=np.uint64)) for _ in range(500)]
        xy = np.array(cases, dtype=np.uint64)
        for op in (0, 1, 2):
            want = [_m2_exact(op, p, *c) for c in cases]
            for impl in (0, 1, 2, 3):
                got = ww.selftest_m2(op | impl << 4, p, xy)
                assert [tuple(map(int, g)) for g in got] == want, (p, op, impl)


@pytest.mark.parametrize("lo,hi", [(127, 2_000_000), (1_373_553, 4_373_653), (2**32 - 10**6, 2**32 + 10**6),
                                   (2**64 - 2 * 10**6 - 1, 2**64 - 1), (10**15, 10**15 + 3_000_000)])
def test_deep_sieve_keeps_every_prp(ww, oracle, lo, hi):
    """The deep sieve (primes to 2^20), which spares every multiple r*k with
    k = 1 (mod ord_r(2)), keeps every PRP of the reference's definition, and
    only numbers with no factor <= 113 reach the PRP test."""
    cand, spared = ww.selftest_candidates(lo, hi)
    summ, prps, _ = oracle.scan_range(lo, hi, want_prps=True, prp_cap=(hi - lo) // 2 + 8)
    assert np.unique(cand).size == cand.size, "a candidate would be tested twice"
    assert np.all(np.isin(prps, cand)), "a PRP was sieved out"
    assert not np.any(np.isin(cand, np.array([1], np.uint64)))
    sample = cand[:: max(1, cand.size // 2000)]
    assert all(not oracle.small_factor(int(x)) for x in sample)
    # about 0.05 candidates per integer at large n (Mertens), against 0.119
    # after 113; at small n the primes themselves are denser than that
    assert cand.size < 0.062 * (hi - lo) + 1.1 * prps.size
    spsp = [int(p) for p in prps if not oracle.is_prime(int(p))]
    for n in spsp:
        assert n in set(cand.tolist())


def test_deep_sieve_spares_pseudoprimes_with_deep_factors(ww, oracle):
    # 49141 = 157 * 313 and 88357 = 149 * 593 are base-2 strong pseudoprimes
    # whose factors are deep-sieve primes: only the cofactor rule keeps them
    for n in (49141, 88357, 104653):
        assert oracle.is_prp(n) and not oracle.is_prime(n)
        cand, spared = ww.selftest_candidates(n - 2000, n + 2000)
        assert cand.tolist().count(n) == 1 and spared >= 1
    # 49141 is spared by both of its factors; it must reach the PRP test once
    cand, spared = ww.selftest_candidates(49141 - 10, 49141 + 10)
    assert spared >= 2 and cand.tolist().count(49141) == 1


def test_deep_table_rows_are_exact():
    """Every row of the generated deep-sieve table: r prime (113 < r), o the
    exact multiplicative order of 2 mod r, r^-1 mod 2^64, floor(2^64 / r),
    floor(2^64 / o); rows ascending; the band counts add up."""
    import re

    from conftest import PKG

    text = (PKG / "csrc" / "ww_deep_table.h").read_text()
    counts = {int(b): int(n) for b, n in re.findall(r"#define WW_DEEP_COUNT_(\d+) (\d+)", text)}
    rows = [tuple(int(v, 0) for v in m) for m in
            re.findall(r"X\((\d+)u, (\d+)u, (0x[0-9a-f]+)ull, (0x[0-9a-f]+)ull, (0x[0-9a-f]+)ull\)", text)]
    assert len(rows) == max(counts.values())
    for b, n in counts.items():
        assert sum(1 for r in rows if r[0] < (1 << b)) == n, b
    limit = 1 << max(counts)
    sieve = bytearray([1]) * limit
    sieve[0:2] = b"\0\0"
    for i in range(2, int(limit ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = bytearray(len(range(i * i, limit, i)))
    assert [r[0] for r in rows] == [p for p in range(114, limit) if sieve[p]]
    M = 1 << 64
    for r, o, rinv, mr, mo in rows:
        assert (r * rinv) % M == 1 and mr == M // r and mo == M // o, r
        assert (r - 1) % o == 0 and pow(2, o, r) == 1, r
        # o is the order: no proper divisor o/q with q prime works
        x, q = o, 2
        while q * q <= x:
            if x % q == 0:
                assert pow(2, o // q, r) != 1, r
                while x % q == 0:
                    x //= q
            q += 1
        if x > 1:
            assert pow(2, o // x, r) != 1, r


def test_checkpoint_files_alternate_and_resume_from_newest(ww, tmp_path):
    """write_state / read_state (main.cpp:103-209): the files alternate A, B,
    A ...; the text is "start stop current cksm psum pcnt" with psum as %lf;
    a read takes the valid file with the larger current (B on a tie) and
    names the other file as the one to write next."""
    fa, fb = str(tmp_path / "stateA-WW.txt"), str(tmp_path / "stateB-WW.txt")
    start, stop = 10**12, 10**12 + 6 * 10**10
    assert ww.state_read(fa, fb, start, stop) is None  # no files yet
    nxt = True
    for i, cur in enumerate((start + 10**10, start + 2 * 10**10, start + 3 * 10**10)):
        nxt = ww.state_write(fa, fb, start, stop, cur, 0xABC0 + i, 1.5 * i, i, nxt)
    # three writes: A, B, A -> B is due next
    assert nxt is False
    assert open(fa).read() == "%d %d %d %d %f %d\n" % (start, stop, start + 3 * 10**10, 0xABC2, 3.0, 2)
    assert open(fb).read() == "%d %d %d %d %f %d\n" % (start, stop, start + 2 * 10**10, 0xABC1, 1.5, 1)
    st, write_a = ww.state_read(fa, fb, start, stop)
    assert st["current"] == start + 3 * 10**10 and st["cksm"] == 0xABC2 and st["pcnt"] == 2
    assert write_a is False  # A was read, so B is overwritten next
    # equal positions: B wins, A is written next
    open(fb, "w").write(open(fa).read())
    st, write_a = ww.state_read(fa, fb, start, stop)
    assert write_a is True


def test_checkpoint_files_that_do_not_belong_are_ignored(ww, tmp_path):
    """A file that does not parse, or that was written for another start or
    stop, is not used (main.cpp:147-175); the other file still is.  A
    position outside [start, stop] is refused too (the reference would
    resume from it)."""
    fa, fb = str(tmp_path / "a.txt"), str(tmp_path / "b.txt")
    start, stop = 10**9, 2 * 10**9
    ww.state_write(fa, fb, start, stop, start + 5, 7, 0.0, 0, True)  # A
    open(fb, "w").write("garbage\n")
    st, write_a = ww.state_read(fa, fb, start, stop)
    assert st["current"] == start + 5 and write_a is False
    ww.state_write(fa, fb, start, stop + 1, start + 9, 8, 0.0, 0, False)  # B, for another range
    st, _ = ww.state_read(fa, fb, start, stop)
    assert st["current"] == start + 5
    assert ww.state_read(fa, fb, start, stop + 1)[0]["current"] == start + 9
    open(fa, "w").write("%d %d %d 0 0.000000 0\n" % (start, stop, stop + 1))  # past the end
    assert ww.state_read(fa, fb, start, stop) is None


def test_status_strings(ww):
    """Every status code of the header has its own message."""
    L = ww.lib()
    seen = {code: L.ww_status_string(code).decode() for code in range(-9, 1)}
    assert seen[0] == "ok" and len(set(seen.values())) == len(seen)
    assert L.ww_status_string(-100).decode() == "unknown status"


def test_cli_host_range_split(tmp_path):
    """The CLI's host side splits a range over host threads
    (host/wwhost.hpp): the pieces tile [lo, hi) exactly, and the CPU prime
    list built from them equals one built in a single pass, near 2^64 and
    at the ranges' smallest start."""
    src = tmp_path / "split.cpp"
    src.write_text(r'''
#include <stdio.h>
#include <mutex>
#include "wwhost.hpp"
using namespace wwhost;
static std::vector<uint64_t> single(uint64_t lo, uint64_t hi) {
    std::vector<uint64_t> out;
    for (uint64_t n = lo | 1; n < hi && n >= lo; n += 2) {
        bool small = false;
        for (uint32_t r = 3; r <= 113 && !small; r += 2) small = (n % r == 0) && n != r;
        if (!small && n > 113 && ww_is_prime(n)) out.push_back(n);
        if (n > UINT64_MAX - 2) break;
    }
    return out;
}
int main() {
    const uint64_t cases[][2] = {{127, 300000}, {18446744073708551615ull - 2000000, 18446744073709551615ull},
                                 {1000000007, 1000000008}, {5000, 5000 + 65536 * 3 + 1}};
    for (auto &c : cases) {
        std::mutex m;
        std::vector<std::pair<uint64_t, uint64_t>> pieces;
        parallel_pieces(c[0], c[1], [&](uint64_t a, uint64_t b, unsigned) {
            std::lock_guard<std::mutex> g(m);
            pieces.push_back({a, b});
        });
        std::sort(pieces.begin(), pieces.end());
        uint64_t at = c[0];
        for (auto &p : pieces) {
            if (p.first != at || p.second <= p.first) return printf("bad piece\n"), 1;
            at = p.second;
        }
        if (at != c[1]) return printf("gap at the end\n"), 1;
        if (cpu_primes(c[0], c[1]) != single(c[0], c[1])) return printf("prime list differs\n"), 1;
    }
    printf("ok\n");
    return 0;
}
''')
    exe = tmp_path / "split"
    inc = PKG / "host"
    cuda_inc = "/usr/local/cuda/include"
    b = subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", f"-I{inc}", f"-I{PKG.parent / 'include'}",
                        f"-I{cuda_inc}", str(src), "-o", str(exe), f"-L{PKG / 'lib'}", "-lwwcuda",
                        f"-Wl,-rpath,{PKG / 'lib'}"], capture_output=True, text=True)
    assert b.returncode == 0, b.stderr[-2000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def _primes_near(oracle, x: int, count: int, up: bool = True) -> list[int]:
    out, n = [], x | 1
    while len(out) < count and 127 <= n < 2**64:
        if oracle.is_prime(n):
            out.append(n)
        n += 2 if up else -2
    return out


def test_host_twin_ladder_start_edges(ww, oracle):
    """The ladders start from the top bits of their exponents (a Lucas number
    or a power of two times the Montgomery one, reduced with a double-precision
    quotient estimate).  Primes where that start is least ordinary: every
    prime below 20000, the Mersenne primes whose p + 1 is a power of two
    (the Lucas index then has two bits more than (p-1)/2), and primes on both
    sides of each power of two from 2^7 to 2^64."""
    ps = [n for n in range(127, 20000, 2) if oracle.is_prime(n)]
    ps += [2**7 - 1, 2**13 - 1, 2**17 - 1, 2**19 - 1, 2**31 - 1, 2**61 - 1]
    for b in range(8, 65):
        ps += _primes_near(oracle, 2**b - 1, 6, up=False)
        if b < 64:
            ps += _primes_near(oracle, 2**b + 1, 6, up=True)
    ps = np.array(sorted(set(ps)), dtype=np.uint64)
    d = ww.selftest_digits(ps)
    w, s = oracle.list_digits(ps)
    assert np.array_equal(d[:, 0:2], w)
    assert np.array_equal(d[:, 2:4], s)


@pytest.mark.parametrize("lo,hi", [(127, 40000), (2**13 - 200, 2**13 + 200), (2**19 - 300, 2**19 + 300),
                                   (2**31 - 400, 2**31 + 400), (2**32 - 20000, 2**32 + 20000),
                                   (2**61 - 30000, 2**61 + 30000), (2**62 - 20000, 2**62 + 20000),
                                   (2**63 - 20000, 2**63 + 20000)])
def test_host_twin_range_at_boundaries(ww, oracle, lo, hi):
    """The SPRP test starts after the top five bits of n-1 when its 2-adic
    valuation lies below them (the pseudoprime 2^32 + 1, whose n-1 is a power
    of two, takes the other start), the separate Wieferich and Wall-Sun-Sun
    ladders from their top bits: PRP count, checksum and hits of ranges across
    powers of two (and Mersenne primes) equal the oracle's."""
    got = ww.selftest_range(lo, hi)
    want, _, _ = oracle.scan_range(lo, hi)
    assert got["prp_count"] == want["prp_count"]
    assert got["checksum"] == want["checksum"]
    assert got["result_count"] == want["gpu_results"]


def test_devtest_m2_rejects_bad_arguments(ww):
    """The device arithmetic check refuses an even or too small modulus and an
    unknown operation before it touches a device, and does nothing for zero
    cases."""
    xy = np.zeros(4, dtype=np.uint64)
    for op, p in [(0, 2**64 - 2), (0, 1), (9, 2**64 - 59), (-1, 2**64 - 59)]:
        with pytest.raises(ww.WWError) as e:
            ww.devtest_m2(op, p, xy)
        assert e.value.status == -2
    assert ww.devtest_m2(1, 2**64 - 59, np.zeros(0, dtype=np.uint64)).shape == (0, 2)
