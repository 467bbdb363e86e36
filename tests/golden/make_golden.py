"""Regenerate the golden fixtures in this folder from the reference's own CPU
code (oracle/_ref/libwwref.so, compiled in place from the reference tree by
oracle/Makefile).  Run from the repository root, naming the reference
source tree (its tests.txt gives the end-to-end vectors):

    make -C oracle REF_DIR=<tree> && python tests/golden/make_golden.py <tree>

    python tests/golden/make_golden.py <tree> --long     # config 3's range, minutes
    python tests/golden/make_golden.py <tree> --results  # config 1's results file

Outputs (small, committed):
  ref_ranges.json  per-range PRP count, checksum and CPU result count
  ref_terms.npz    per-prime low 32 bits of the Wieferich and WSS checksum
                   terms and the wwcpu.cpp hit flags for fixed prime samples
  ref_prps.json    PRP-list digests (count, sum, sha256 of the sorted list)
  ref_long.json    config 3's full range (with --long)
  results_127_5e7.json  the expected results file of `WWocl 127 5e7` (with
                   --results): line count, sha256, first and last lines
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import Oracle, RefCPU  # noqa: E402

OUT = Path(__file__).resolve().parent
TOP = 2**64

RANGES = [
    ("small_3e6", 127, 3_000_000),
    ("config1_5e7", 127, 50_000_000),
    ("cross_2p32", 4_294_000_000, 4_295_500_000),
    ("near_top_2e6", TOP - 2**35, TOP - 2**35 + 2_000_000),
    ("top_1e8", 18446744073609551615, 18446744073709551615),
    ("wieferich_special_window", 2276306935816523 - 1_000_000, 2276306935816523 + 1_000_000),
    ("wss_special_window", 338772621946054253, 338772621946054253 + 2_000_000),
    ("mid_2p48", 2**48, 2**48 + 3_000_000),
    ("cross_2p62", 2**62 - 1_000_000, 2**62 + 1_000_000),
    ("cross_2p63", 2**63 - 1_000_000, 2**63 + 1_000_000),
]

PRP_RANGES = [
    ("prp_small", 127, 2_000_000),
    ("prp_2p32", 2**32 - 1_000_000, 2**32 + 1_000_000),
    ("prp_2p63", 2**63 - 500_000, 2**63 + 500_000),
    ("prp_top", TOP - 1_000_001, TOP - 1),
    ("prp_spsp", 1_373_653 - 100, 1_373_653 + 3_000_000),
]


def digest(arr: np.ndarray) -> dict:
    arr = np.sort(np.asarray(arr, dtype=np.uint64))
    return {
        "count": int(arr.size),
        "sum_mod_2_64": int(arr.sum(dtype=np.uint64)),
        "sha256": hashlib.sha256(arr.astype("<u8").tobytes()).hexdigest(),
    }


def prime_samples(o: Oracle) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(20201226)
    out = {}
    out["small"] = np.array([p for p in range(127, 20000, 2) if o.is_prp(p)], dtype=np.uint64)
    near32 = []
    n = 2**32 - 20001
    while len(near32) < 2000:
        if o.is_prp(n):
            near32.append(n)
        n += 2
    out["near_2p32"] = np.array(near32, dtype=np.uint64)
    below32 = []
    n = 2**32 - 1
    while len(below32) < 500:
        if o.is_prp(n):
            below32.append(n)
        n -= 2
    out["below_2p32"] = np.array(below32, dtype=np.uint64)
    top = []
    n = TOP - 1
    while len(top) < 2000:
        if o.is_prp(n):
            top.append(n)
        n -= 2
    out["near_2p64"] = np.array(top, dtype=np.uint64)
    for name, centre in (("near_2p63", 2**63), ("near_2p62", 2**62)):
        side = []
        n = centre - 1
        while len(side) < 800:
            if o.is_prp(n):
                side.append(n)
            n -= 2
        n = centre + 1
        while len(side) < 1600:
            if o.is_prp(n):
                side.append(n)
            n += 2
        out[name] = np.array(side, dtype=np.uint64)
    rnd = []
    while len(rnd) < 4000:
        c = int(rng.integers(0, 2**63, dtype=np.uint64)) * 2 + 1
        if c > 113 and o.is_prp(c):
            rnd.append(c)
    out["random64"] = np.array(rnd, dtype=np.uint64)
    spsp = [p for p in range(127, 3_000_000, 2) if o.is_prp(p) and not o.is_prime(p)]
    out["spsp"] = np.array(spsp, dtype=np.uint64)
    out["known_hits"] = np.array([2276306935816523, 338772621946054253], dtype=np.uint64)
    return out


def parse_tests_txt(path: Path) -> list[dict]:
    """The reference's end-to-end vectors (tests.txt): 'START END', optional
    hit lines, then the final 16-hex-digit checksum, blocks split by dashes."""
    blocks, cur = [], []
    for ln in path.read_text().splitlines():
        ln = ln.strip()
        if ln and set(ln) == {"-"}:
            blocks.append(cur)
            cur = []
        elif ln and not ln.startswith("test cases"):
            cur.append(ln)
    blocks.append(cur)
    cases = []
    for lines in blocks:
        if len(lines) < 2:
            continue
        start, end = lines[0].split()
        cases.append({"start": start, "end": end, "hits": lines[1:-1], "checksum": lines[-1]})
    return cases


def long_ranges(ref: RefCPU) -> None:
    """Config 3's range [2^64-2^35, 2^64-2^35+2^34): about 3.9e8 PRPs, several
    minutes on 8 cores (only with --long)."""
    lo = 2**64 - 2**35
    hi = lo + 2**34
    r = ref.scan_range(lo, hi, nthreads=8)
    out = {"config3": {"lo": lo, "hi": hi, "prp_count": r["prp_count"], "checksum": "%016X" % r["checksum"],
                       "cpu_results": r["cpu_results"]}}
    (OUT / "ref_long.json").write_text(json.dumps(out, indent=1) + "\n")
    print(out, flush=True)


def results_file(ref: RefCPU, o: Oracle) -> None:
    """The results file the reference program writes for `WWocl 127 5e7`
    (config 1): one flush at the range's end (main.cpp:1743-1760), hits
    sorted by p with the Wieferich kernel's hit first for equal p
    (main.cpp:843-854, a stable sort of the Wieferich-then-WSS hit list),
    PRP-only hits dropped (isPrime, main.cpp:869-911), then the checksum line
    (main.cpp:1759-1766).  Which primes hit is pinned to the reference's own
    wieferichCPU / wallsunsunCPU flags over every PRP of the range; the hit
    records' rem/quot and the line formats come from the oracle's
    restatement (the formats are pinned by tests.txt)."""
    lo, hi = 127, 50_000_000
    prps = ref.prp_list(lo, hi, cap=4_000_000)
    _, _, w_hit, s_hit = ref.list_terms(prps)
    summ, _, hits = o.scan_range(lo, hi, hit_cap=16384)
    assert summ["gpu_results"] == len(hits)
    assert {p for p, r, _, _ in hits if r == 1093} == {int(p) for p, h in zip(prps, w_hit) if h}
    assert {p for p, r, _, _ in hits if r in (1, 2)} == {int(p) for p, h in zip(prps, s_hit) if h}
    rc, text, dropped = o.format_results(hits)
    assert rc >= 0
    text += "%016X\n" % summ["checksum"]
    lines = text.splitlines()
    out = {"start": "127", "end": "5e7", "lo": lo, "hi": hi, "prp_count": int(prps.size),
           "hit_records": len(hits), "dropped_prp_only": dropped, "lines": len(lines),
           "wieferich_lines": sum(" Wieferich " in ln for ln in lines),
           "wallsunsun_lines": sum(" WallSunSun " in ln for ln in lines),
           "sha256": hashlib.sha256(text.encode()).hexdigest(), "head": lines[:6], "tail": lines[-6:]}
    (OUT / "results_127_5e7.json").write_text(json.dumps(out, indent=1) + "\n")
    print({k: v for k, v in out.items() if k not in ("head", "tail")}, flush=True)


def main() -> None:
    ref = RefCPU()
    o = Oracle()
    if "--long" in sys.argv:
        long_ranges(ref)
        return
    if "--results" in sys.argv:
        results_file(ref, o)
        return
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not args or not (Path(args[0]) / "tests.txt").exists():
        raise SystemExit("usage: make_golden.py <reference source tree> [--long | --results]")
    ref_tree = Path(args[0])
    cases = parse_tests_txt(ref_tree / "tests.txt")
    (OUT / "tests_txt.json").write_text(json.dumps(cases, indent=1) + "\n")
    print(cases, flush=True)
    ranges = {}
    for name, lo, hi in RANGES:
        r = ref.scan_range(lo, hi)
        ranges[name] = {"lo": lo, "hi": hi, "prp_count": r["prp_count"],
                        "checksum": "%016X" % r["checksum"], "cpu_results": r["cpu_results"]}
        print(name, ranges[name], flush=True)
    (OUT / "ref_ranges.json").write_text(json.dumps(ranges, indent=1) + "\n")

    prps = {}
    for name, lo, hi in PRP_RANGES:
        lst = ref.prp_list(lo, hi, cap=(hi - lo) // 2 + 16)
        prps[name] = {"lo": lo, "hi": hi, **digest(lst)}
        print(name, prps[name], flush=True)
    (OUT / "ref_prps.json").write_text(json.dumps(prps, indent=1) + "\n")

    samples = prime_samples(o)
    arrays = {}
    for name, ps in samples.items():
        wt, st, wh, sh = ref.list_terms(ps)
        arrays[f"{name}_p"] = ps
        arrays[f"{name}_wterm"] = wt
        arrays[f"{name}_sterm"] = st
        arrays[f"{name}_whit"] = wh.astype(np.int8)
        arrays[f"{name}_shit"] = sh.astype(np.int8)
        print(name, ps.size, flush=True)
    np.savez_compressed(OUT / "ref_terms.npz", **arrays)


if __name__ == "__main__":
    main()
