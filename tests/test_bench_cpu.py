"""bench.py's reference arm runs on the host (the reference's own CPU code,
oracle/_ref): its JSON line keeps the benchmark contract."""
from __future__ import annotations

import json
import subprocess
import sys

import pytest

from conftest import ROOT


def test_reference_arm_json_line():
    from oracle.oracle import RefCPU

    if not RefCPU.available():
        pytest.skip("oracle/_ref not built")
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "1",
                        "--cpu-sample", "20000"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_under_torchrun_prints_one_line():
    """Launched as the scaling run launches it (torchrun, two ranks): rank 0
    alone runs the reference and prints the line; the other rank exits 0."""
    import socket

    from oracle.oracle import RefCPU

    if not RefCPU.available():
        pytest.skip("oracle/_ref not built")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    p = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--cpu-sample", "20000"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def test_summary_is_short_and_carries_every_leg():
    """The JSON line ends with a summary of every leg that fits in the last
    1500 characters of the output."""
    import importlib

    sys.path.insert(0, str(ROOT))
    bench = importlib.import_module("bench")
    line = {"value": 1.1e9, "e2e": {"value": 1.0e9},
            "roofline": {"frac": 0.93, "executed": {"frac": 0.64}, "mad_lo_only": {"frac": 0.62, "frac_executed": 0.43}},
            "cpu_baseline": {"value": 5.8e6, "checksum_match": True}}
    seg = {"sieve_ms": 7.7, "test_ms": 22.0}
    extra = {"range_pipeline": {"primes_per_s": 8.1e8, "numbers_per_s": 3.6e10, "segment_2p30": seg,
                                "checksum": "1715455BAC8C55C2", "reference_checksum_equal": True},
             "batched_vs_plain": {"units": 4096, "batched_primes_per_s": 8.0e8, "plain_primes_per_s": 7.7e8,
                                  "speedup_batched_vs_plain": 1.04, "target_1p5x_met": False,
                                  "per_unit_bit_identical": True, "narrow_units": {"speedup_batched_vs_plain": 2.6},
                                  "per_run": {"speedup_batched_vs_per_run": 60.0},
                                  "tuned_config": {"seg_words": 16384, "threads": 512, "primes_per_thread": 1,
                                                   "joint_test_loop": 0}},
             "serving": {"requests": 24008, "p50_ms": 15.9, "p99_ms": 168.0, "max_ms": 394.0, "primes_per_s": 5.1e8,
                         "all_ok": True, "cpu_checksum_equal_on_smallest": True}}
    s = bench.summarize(line, extra)
    text = json.dumps({"summary": s})
    assert len(text) < 1400, len(text)
    assert set(s) == {"config2_fixed_list", "config3_plain_range", "config4_batched_vs_plain", "config5_serving"}
    assert s["config4_batched_vs_plain"]["target_1p5x_met"] is False
    assert s["config5_serving"]["p99_ms"] == 168.0
