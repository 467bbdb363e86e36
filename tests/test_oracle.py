"""The CPU oracle pinned against the reference: its own test vectors
(tests.txt), and fixtures produced by the reference's own CPU code
(tests/golden/make_golden.py over oracle/_ref)."""
from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from conftest import GOLDEN, sample_names


def test_known_answer_wieferich(oracle):
    # tests.txt:15-17: 2276306935816523 is a Wieferich special instance (-1 -3 p)
    p = 2276306935816523
    s0, s1 = oracle.wieferich_digits(p)
    assert s0 == p - 1 and s1 == p - 4
    rc, text, dropped = oracle.format_results([(p, 1093, -1, s1 + 1 - p)])
    assert text == "2276306935816523 is a Wieferich special instance (-1 -3 p)\n"


def test_known_answer_wss(oracle):
    # tests.txt:22-24: 338772621946054253 is a WallSunSun special instance (+0 +91 p)
    p = 338772621946054253
    c0, c1 = oracle.wss_digits(p)
    assert c0 == 0 and c1 == 91
    rc, text, _ = oracle.format_results([(p, 2, 0, 91)])
    assert text == "338772621946054253 is a WallSunSun special instance (+0 +91 p)\n"


def test_tests_txt_hits_in_windows(oracle, tests_txt):
    # every hit line tests.txt lists is reproduced from a window around it
    for case in tests_txt:
        for line in case["hits"]:
            p = int(line.split()[0])
            summ, _, hits = oracle.scan_range(p - 1000, p + 1000, nthreads=1)
            rc, text, _ = oracle.format_results(hits)
            assert rc >= 0
            assert text == line + "\n"


@pytest.mark.parametrize("name", ["small_3e6", "cross_2p32", "near_top_2e6", "wieferich_special_window",
                                  "wss_special_window", "mid_2p48", "config1_5e7", "top_1e8", "cross_2p62",
                                  "cross_2p63"])
def test_oracle_ranges_match_reference(oracle, ref_ranges, name):
    r = ref_ranges[name]
    summ, _, _ = oracle.scan_range(r["lo"], r["hi"])
    assert summ["prp_count"] == r["prp_count"]
    assert "%016X" % summ["checksum"] == r["checksum"]
    assert summ["cpu_results"] == r["cpu_results"]
    # the kernels' hit classification agrees with wwcpu.cpp's count
    assert summ["gpu_results"] == summ["cpu_results"]


def test_oracle_terms_match_reference(oracle, ref_terms):
    for name in sample_names(ref_terms):
        ps = ref_terms[name + "_p"]
        w, s = oracle.list_digits(ps)
        assert np.array_equal((w[:, 1] & 0xFFFFFFFF).astype(np.uint32), ref_terms[name + "_wterm"]), name
        assert np.array_equal((s[:, 1] & 0xFFFFFFFF).astype(np.uint32), ref_terms[name + "_sterm"]), name


def test_oracle_hit_flags_match_reference(oracle, ref_terms):
    import ctypes as C
    from oracle.oracle import WoDigits

    L = oracle.L
    L.wo_wieferich_cpu_hit.argtypes = [C.c_uint64, WoDigits]
    L.wo_wss_cpu_hit.argtypes = [C.c_uint64, WoDigits]
    for name in sample_names(ref_terms):
        ps = ref_terms[name + "_p"]
        w, s = oracle.list_digits(ps)
        wh = [L.wo_wieferich_cpu_hit(int(p), WoDigits(int(a), int(b))) for p, (a, b) in zip(ps, w)]
        sh = [L.wo_wss_cpu_hit(int(p), WoDigits(int(a), int(b))) for p, (a, b) in zip(ps, s)]
        assert np.array_equal(np.array(wh, np.int8), ref_terms[name + "_whit"]), name
        assert np.array_equal(np.array(sh, np.int8), ref_terms[name + "_shit"]), name


def test_oracle_prp_lists_match_reference(oracle, ref_prps):
    for name, r in ref_prps.items():
        cap = (r["hi"] - r["lo"]) // 2 + 16
        summ, prps, _ = oracle.scan_range(r["lo"], r["hi"], want_prps=True, prp_cap=cap)
        assert prps.size == r["count"], name
        assert int(prps.sum(dtype=np.uint64)) == r["sum_mod_2_64"], name
        assert hashlib.sha256(np.sort(prps).astype("<u8").tobytes()).hexdigest() == r["sha256"], name


def test_spsp_are_tested_and_dropped(oracle):
    # base-2 strong pseudoprimes with no factor <= 113 are PRPs: they add to
    # the checksum (main.cpp:689-693) but never reach the results file
    # (main.cpp:907-911).
    spsp = [n for n in range(127, 400_000, 2) if oracle.is_prp(n) and not oracle.is_prime(n)]
    assert spsp[:3] == [42799, 49141, 88357]
    hits = []
    for n in spsp:
        s = oracle.wieferich_digits(n)
        hits.append((n, 1093, 1, 5))  # forced hit record for a pseudoprime
        assert s[0] in (1, n - 1)  # Euler's criterion holds for strong pseudoprimes
    rc, text, dropped = oracle.format_results(hits)
    assert rc == 0 and text == "" and dropped == len(spsp)


def test_composite_hit_is_refused(oracle):
    rc, _, _ = oracle.format_results([(127 * 131, 1093, 1, 0)])
    assert rc == -2


def test_parse_number(oracle):
    cases = {"127": (0, 127), "6e10": (0, 60_000_000_000), "227630e10": (0, 2276300000000000),
             "1e0": (-1, 0), "18446744073709551615": (0, 18446744073709551615), "2e19": (-2, 0)}
    for text, (rc, val) in cases.items():
        got_rc, got = oracle.parse_number(text)
        assert got_rc == rc, text
        if rc == 0:
            assert got == val, text


def test_wheel_offset(oracle):
    for start in [127, 128, 129, 130, 131, 150, 10**12 + 1, 2**64 - 60]:
        n, idx = oracle.wheel_offset(start)
        assert n >= start and n - start < 7
        assert n % 2 and n % 3 and n % 5
        assert [7, 11, 13, 17, 19, 23, 29, 1][idx] == n % 30


def test_random_prime_stream(oracle):
    ps, used = oracle.random_primes(7, 2000)
    assert ps.size == 2000 and np.all(ps >= np.uint64(2**62)) and np.all(ps & np.uint64(1))
    assert all(oracle.is_prime(int(p)) for p in ps[:200])
    # stream order: re-derive the first primes position by position
    i, k = 0, 0
    while k < 50:
        c = oracle.splitmix64(7, i) | 1
        if c >= 2**62 and oracle.is_prime(c):
            assert c == int(ps[k])
            k += 1
        i += 1


def test_oracle_matches_reference_code_on_random_ranges(oracle):
    """The C restatement against the reference's own CPU code (oracle/_ref,
    wwcpu.cpp + prime.h compiled in place) on seeded random ranges:
    magnitudes log-uniform over [127, 2^64), widths from one number to 2e5."""
    import math
    import random

    from oracle.oracle import RefCPU

    if not RefCPU.available():
        pytest.skip("oracle/_ref not built")
    ref = RefCPU()
    rng = random.Random(2027)
    for _ in range(400):
        lo = int(math.exp(rng.uniform(math.log(127), math.log(2**64 - 2))))
        hi = min(lo + int(math.exp(rng.uniform(0, math.log(2e5)))), 2**64 - 1)
        mine, _, _ = oracle.scan_range(lo, hi)
        theirs = ref.scan_range(lo, hi)
        assert (mine["prp_count"], mine["checksum"], mine["cpu_results"]) == \
               (theirs["prp_count"], theirs["checksum"], theirs["cpu_results"]), (lo, hi)


def test_oracle_results_file_config1_matches_reference_digest(oracle):
    """The oracle's restatement of getResults over its own hits of
    [127, 5e7) gives the results file whose digest make_golden.py --results
    computed after checking the hit set against the reference's own CPU hit
    flags (wieferichCPU / wallsunsunCPU over every PRP of the range)."""
    g = json.loads((GOLDEN / "results_127_5e7.json").read_text())
    summ, _, hits = oracle.scan_range(g["lo"], g["hi"], hit_cap=16384)
    assert summ["prp_count"] == g["prp_count"] and len(hits) == g["hit_records"]
    rc, text, dropped = oracle.format_results(hits)
    text += "%016X\n" % summ["checksum"]
    assert rc >= 0 and dropped == g["dropped_prp_only"]
    assert hashlib.sha256(text.encode()).hexdigest() == g["sha256"]
    lines = text.splitlines()
    assert lines[:6] == g["head"] and lines[-6:] == g["tail"]
