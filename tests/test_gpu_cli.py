"""The wwocl program end to end: the reference's own regression vectors
(tests.txt) -- START/END parsing, the segment loop, checkpoints and the
results file with its final checksum -- and checkpoint/resume behaviour."""
from __future__ import annotations

import os
import subprocess

import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu
WWOCL = PKG / "bin" / "wwocl"


def run(args, cwd, timeout=900):
    return subprocess.run([str(WWOCL), *args], cwd=cwd, capture_output=True, text=True, timeout=timeout)


@pytest.mark.parametrize("case", range(4))
def test_tests_txt_vector(tests_txt, tmp_path, case):
    c = tests_txt[case]
    r = run([c["start"], c["end"], "-compute"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = (tmp_path / "results-WW.txt").read_text().splitlines()
    assert lines[-1] == c["checksum"]
    if c["hits"] or case == 0:
        assert lines[:-1] == c["hits"]
    assert f"Checksum: {c['checksum']}" in r.stdout


def test_results_file_config1_byte_for_byte(oracle, tmp_path):
    """`WWocl 127 5e7` (config 1) writes the reference's results file byte
    for byte: 3890 hit lines sorted by p (the Wieferich line first where one
    prime has both), then the checksum.  The file is compared with the
    oracle's restatement of getResults over the oracle's hits and with the
    committed digest of the file generated from the reference's own CPU hit
    flags (tests/golden/results_127_5e7.json).  No range below 2e9 has a hit
    on a pseudoprime, so the dropped count is 0 here; the drop rule itself is
    tested on the host (test_format_hits_matches_oracle)."""
    import hashlib
    import json

    from conftest import GOLDEN

    g = json.loads((GOLDEN / "results_127_5e7.json").read_text())
    r = run([g["start"], g["end"], "-debug"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    got = (tmp_path / "results-WW.txt").read_bytes()
    summ, _, hits = oracle.scan_range(g["lo"], g["hi"], hit_cap=16384)
    rc, text, dropped = oracle.format_results(hits)
    want = (text + "%016X\n" % summ["checksum"]).encode()
    assert got == want
    assert hashlib.sha256(got).hexdigest() == g["sha256"]
    lines = got.decode().splitlines()
    assert len(lines) == g["lines"] and lines[:6] == g["head"] and lines[-6:] == g["tail"]
    assert f"Number of results:                 {g['hit_records']}" in r.stdout
    assert f"PRPs removed from results:         {g['dropped_prp_only']}" in r.stdout


def test_separate_kernels_and_ckpt_cadence(tests_txt, tmp_path):
    c = tests_txt[2]  # the Wieferich special instance window
    r = run([c["start"], c["end"], "-separate", "-ckpt", "2e9", "-results", "results-WWocl.txt"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = (tmp_path / "results-WWocl.txt").read_text().splitlines()
    assert lines == c["hits"] + [c["checksum"]]
    assert r.stdout.count("Checkpoint, current:") == 30  # 6e10 numbers / 2e9
    # the autotune picked a sieve shape and depth on the device (in place of profileGPU)
    assert "Sieve shape" in r.stderr and "depth" in r.stderr


def test_resume_from_checkpoint(tests_txt, tmp_path):
    """Kill-free resume: a state file written at a segment boundary makes a
    second run finish with the same checksum and results."""
    c = tests_txt[3]
    r = run([c["start"], c["end"], "-ckpt", "1e10"], tmp_path)
    assert r.returncode == 0
    full = (tmp_path / "results-WW.txt").read_text()
    # rewind: keep a mid-way state file (A/B alternate; take the older one)
    a = (tmp_path / "stateA-WW.txt").read_text().split()
    b = (tmp_path / "stateB-WW.txt").read_text().split()
    older = min((a, b), key=lambda s: int(s[2]))
    assert int(older[2]) < int(c["end"])
    (tmp_path / "stateA-WW.txt").write_text(" ".join(older) + "\n")
    (tmp_path / "stateB-WW.txt").write_text("garbage\n")
    # results written after that checkpoint are lost with the crash
    kept = [ln for ln in full.splitlines() if ln != c["checksum"]]
    p_hit = int(c["hits"][0].split()[0])
    if p_hit >= int(older[2]):
        kept = [ln for ln in kept if int(ln.split()[0]) < int(older[2])]
    (tmp_path / "results-WW.txt").write_text("".join(ln + "\n" for ln in kept))
    r2 = run([c["start"], c["end"], "-ckpt", "1e10"], tmp_path)
    assert r2.returncode == 0, r2.stdout + r2.stderr
    assert "Resuming search from checkpoint" in r2.stdout
    assert (tmp_path / "results-WW.txt").read_text() == full


def test_finished_workunit_exits_early(tmp_path):
    r = run(["1e6", "2e6"], tmp_path)
    assert r.returncode == 0
    r2 = run(["1e6", "2e6"], tmp_path)
    assert r2.returncode == 0 and "Workunit complete." in r2.stdout


def test_bad_range_is_an_error(tmp_path):
    r = run(["2e6", "1e6"], tmp_path)
    assert r.returncode != 0 and "END must be > START" in r.stdout


def test_debug_prints_kernel_profile_and_counters(tests_txt, tmp_path):
    """-debug (main.cpp:1632-1661, 932-939): the per-kernel time shares of one
    segment and the checkpoint counters; the search result is unchanged."""
    c = tests_txt[2]
    r = run([c["start"], c["end"], "-debug"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout
    assert "Profiling kernels..." in out and "Percent of time spent in each kernel:" in out
    for name in ("Prime Generator:", "Wieferich Test:", "WallSunSun Test:"):
        assert name in out
    assert "PRPs tested since last checkpoint:" in out
    lines = (tmp_path / "results-WW.txt").read_text().splitlines()
    assert lines == c["hits"] + [c["checksum"]]


def test_testprimes_checks_every_segment(ref_ranges, tmp_path):
    """-testprimes (main.cpp:1177-1183,1732-1735): every segment's GPU PRP
    list, pseudoprimes set aside, equals the CPU prime list; the range
    [127, 3e6) holds base-2 strong pseudoprimes (1373653 = 829 * 1657 among
    them), and the run still ends with the reference checksum."""
    r = ref_ranges["small_3e6"]
    out = run([str(r["lo"]), str(r["hi"]), "-testprimes", "-ckpt", "1e6"], tmp_path)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count("GPU primes match CPU") >= 3
    lines = (tmp_path / "results-WW.txt").read_text().splitlines()
    assert lines[-1] == r["checksum"]


@pytest.mark.parametrize("name", ["config1_5e7", "wss_special_window", "long"])
def test_dropin_example_matches_reference(ref_ranges, tmp_path, name):
    """bin/dropin_example, the reference program's device loop rewired onto
    the kernel-shaped launchers in C++ (host/dropin_example.cpp), prints the
    reference's PRP count, result count and checksum."""
    import json

    if name == "long":
        r = json.loads((PKG.parent / "tests" / "golden" / "ref_long.json").read_text())["config3"]
    else:
        r = ref_ranges[name]
    p = subprocess.run([str(PKG / "bin" / "dropin_example"), str(r["lo"]), str(r["hi"])], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    assert p.stdout.split() == ["prps", str(r["prp_count"]), "results", str(r["cpu_results"]),
                                "checksum", r["checksum"]]
