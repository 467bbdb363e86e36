"""Benchmark of the WWocl search path on B200: primes tested (Wieferich +
Wall-Sun-Sun) per second on the fixed-list workload -- 2^26 primes in
[2^62, 2^64) drawn from the SplitMix64 stream of seed 7 and kept when they
pass deterministic Miller-Rabin.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one fused Wieferich + Wall-Sun-Sun launch over the whole list
(`value`: list resident in HBM; `e2e`: the same step through the C ABI with
the list copied from pinned host memory and the counters read back, every
step).  Under torchrun each rank tests its own list (seed 7 + rank): weak
scaling, no data-path collective.  Rank 0 prints one JSON line, which at
N = 1 also carries: `roofline` (the test kernel against the measured
integer-multiply chain peak), `cpu_baseline` (the reference's own CPU code on
the host cores), `range_pipeline` (the plain path over the 2^34-wide range
below 2^64, checksum against the reference), `batched_vs_plain` (all 4096
units of the uneven mix: batched engine vs one launch sequence per range in
the same process; one program run per range as a deployment note) and
`serving` (the 120-s Poisson request stream, p50/p99 latency), and last a
short `summary` of every leg.  The default run takes about eight minutes;
--batch-units / --serve-seconds / --range-width shorten or skip the legs.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "wwocl-boinc_b200"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(PKG))

METRIC = "primes/s tested (W+WSS), fixed prime list"
UNIT = "primes/s"
SEED = 7
N_PRIMES = 1 << 26
PEAKS = ROOT / "MEASURED_PEAKS.json"
PROFILE = ROOT / "profiles" / "test_prps_fixed_list.md"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n-primes", type=int, default=N_PRIMES)
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="primes in the bounded CPU sample (0: sized to --cpu-seconds)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="target wall time of the CPU-baseline sample (reference arm: per step / 8)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--range-width", type=float, default=float(1 << 34),
                    help="width of the plain-path range leg starting at 2^64-2^35 (0: skip)")
    ap.add_argument("--batch-config", default="",
                    help="force the batched configuration SEG_WORDS/THREADS/PPT[/JOINT] instead of the autotuner's choice")
    ap.add_argument("--batch-units", type=int, default=4096,
                    help="units of the seed-11 uneven mix for the batched-vs-plain leg (4096: the whole mix; 0: skip)")
    ap.add_argument("--serve-seconds", type=float, default=120.0,
                    help="length of the Poisson request stream (120: the whole stream; 0: skip)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def config(args, world):
    return {"workload": "fixed prime list: 2^26 primes in [2^62, 2^64), SplitMix64 seed 7, deterministic MR",
            "n_primes_per_gpu": args.n_primes, "global_primes": args.n_primes * world,
            "parallelism": f"weak x{world} (independent lists, seed 7+rank)",
            "l2": "inputs larger than L2 (8 B x 2^26 = 512 MiB list per step)"}


def algorithmic_imad_per_prime(primes: np.ndarray) -> tuple[float, float]:
    """32-bit multiply instructions per prime, counted with fixed costs: a
    64x64->128 product = 8, a low 64-bit product = 4, a high 64-bit product =
    8, so a two-digit square mod p^2 = 40 and a product = 48 (38 for the
    square k_test_prps runs, whose low digit is squared from three 32x32
    products instead of four).  k = bitlength(p).

    Returns (reference_count, executed_count):
      reference_count: the reference kernels' algorithm -- Wieferich k-3
        squarings (wieferich.cl:196-328), the Lucas ladder k-1 steps of two
        squarings and one product (wallsunsun.cl:221-354): 40(k-3) + 128(k-1).
      executed_count: what k_test_prps runs -- both ladders start from the
        top bits of their exponents (three small numbers turned into
        Montgomery form, 40 each), then Wieferich k-6 squarings and the Lucas
        ladder k-6 steps of two squarings (38 each), two conversions out of
        Montgomery form (24 each): 114(k-6) + 120 + 48."""
    bits = np.floor(np.log2(primes.astype(np.float64))) + 1  # exact away from powers of two
    ref = 40.0 * (bits - 3) + 128.0 * (bits - 1)
    run = 114.0 * (bits - 6) + 168.0
    return float(ref.mean()), float(run.mean())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = [r.split(",") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def profile_traffic():
    """Per-launch DRAM bytes of the fused test kernel from the committed ncu
    summary (line 'traffic_bytes_per_launch: N'), or None."""
    if not PROFILE.exists():
        return None
    for line in PROFILE.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return int(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def cpu_reference_rate(primes: np.ndarray, threads: int):
    """The reference's own wieferichCPU + wallsunsunCPU (oracle/_ref) over the
    sample on `threads` host threads.  Returns (primes/s, checksum, seconds)."""
    from oracle.oracle import RefCPU

    ref = RefCPU()
    t0 = time.perf_counter()
    r = ref.test_list(primes, nthreads=threads)
    dt = time.perf_counter() - t0
    return primes.size / dt, r["checksum"], dt


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle.oracle import Oracle, RefCPU

    if not RefCPU.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libwwref.so was not built "
                          "(needs the reference sources at build time)"}))
        return 0
    threads = os.cpu_count() or 1
    sample_n = args.cpu_sample
    if sample_n <= 0:  # each step about --cpu-seconds / 8 of CPU time
        probe, _ = Oracle().random_primes(SEED, 1 << 18, threads)
        r0, _, _ = cpu_reference_rate(probe, threads)
        sample_n = max(1 << 20, int(r0 * args.cpu_seconds / 8))
    primes, _ = Oracle().random_primes(SEED, sample_n, threads)
    rates, times = [], []
    for i in range(args.warmup + args.steps):
        rate, cks, dt = cpu_reference_rate(primes, threads)
        if i >= args.warmup:
            rates.append(rate)
            times.append(dt)
    value = primes.size * len(times) / sum(times)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "impl": "reference", "config": config(args, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"first {sample_n} primes of the seed-7 list, wwcpu.cpp "
                                       "wieferichCPU+wallsunsunCPU over std::thread workers",
                             "checksum": "%016X" % cks},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_range_pipeline(ww, local: int, width: int, ckpt: int = 1 << 30, chain_peak: float | None = None) -> dict:
    """The plain one-range path over [2^64-2^35, 2^64-2^35+width): per 2^30
    numbers (the checkpoint cadence) clear, sieve + SPRP, both tests, sync and
    read the counters back, as the reference program's loop does.  With the
    default width 2^34 this is the whole range of tests/golden/ref_long.json,
    whose reference checksum the result is compared with."""
    lo = 2**64 - 2**35
    hi = lo + width
    ctx = ww.Context(local, max_prps=ww.prp_count_bound(0, ckpt), max_hits=15000)
    depth = ctx.sieve_depth()  # deep primes below 2^depth (large ones marked once per launch)
    ctx.run_range(lo, min(hi, lo + ckpt))  # warm

    # sieve and test kernel times of one full checkpoint segment
    ctx.clear_results()
    ctx.clear_segment()
    ctx.marker(0)
    ctx.sieve_prp(lo, min(hi, lo + ckpt))
    ctx.marker(1)
    ctx.test_prps()
    ctx.marker(2)
    ctx.sync()
    seg_prps = ctx.counters()["total_prp_count"]
    sieve_ms, test_ms = ctx.elapsed_ms(0, 1), ctx.elapsed_ms(1, 2)

    cks, cnt, res = 0, 0, 0
    ctx.marker(3)
    t0 = time.perf_counter()
    start = lo
    while start < hi:
        stop = min(start + ckpt, hi)
        ctx.clear_results()
        ctx.clear_segment()
        ctx.sieve_prp(start, stop)
        ctx.test_prps()
        k = ctx.counters()  # sync + read-back at every checkpoint
        if k["overflow"]:
            raise SystemExit(f"range leg overflow flag {k['overflow']}")
        cks, cnt, res = (cks + k["checksum"]) % 2**64, cnt + k["total_prp_count"], res + k["result_count"]
        start = stop
    wall = time.perf_counter() - t0
    ctx.marker(4)
    ctx.sync()
    dev_ms = ctx.elapsed_ms(3, 4)
    ctx.close()
    out = {"workload": f"plain path over [2^64-2^35, 2^64-2^35+{width}), checkpoint every 2^30 numbers",
           "numbers": width, "prps": cnt, "device_ms": dev_ms, "wall_s": wall,
           "primes_per_s": cnt / wall, "numbers_per_s": width / wall,
           "segment_2p30": {"prps": seg_prps, "sieve_ms": sieve_ms, "test_ms": test_ms,
                            "sieve_numbers_per_s": min(width, ckpt) / (sieve_ms * 1e-3),
                            "test_primes_per_s": seg_prps / (test_ms * 1e-3)},
           "checksum": "%016X" % cks, "results": res, "sieve_depth": depth}
    if chain_peak:
        # end to end over sieve + tests, in the same 32-bit multiply units as
        # the test kernel's roofline (k = 64 here): the reference's SPRP of a
        # candidate is 20(k-1) and its sieve hands ~5.3 candidates per PRP to
        # it; here the SPRP starts after the top five bits of n-1 (20(k-5)
        # plus a 12-multiply start) and the deep sieve to 2^depth leaves
        # 0.5615 / ln 2^depth candidates per integer, against the PRP density
        # 1 / ln 2^64
        k = 64
        ref_ops = 40.0 * (k - 3) + 128.0 * (k - 1) + 5.3 * 20.0 * (k - 1)
        cand = (0.5615 / np.log(2.0**depth)) * np.log(2.0**64)
        run_ops = 114.0 * (k - 6) + 168.0 + cand * (20.0 * (k - 5) + 12.0)
        rate = out["primes_per_s"]
        out["roofline_end_to_end"] = {
            "peak_tops": chain_peak / 1e12,
            "reference_ops_per_prime": ref_ops, "frac_reference_ops": rate * ref_ops / chain_peak,
            "executed_ops_per_prime": run_ops, "frac_executed_ops": rate * run_ops / chain_peak,
            "note": "reference ops count the reference algorithm's work (more SPRP candidates, a longer "
                    "Lucas ladder); above 1.0 means less work than the reference needs, not above peak"}
        # the sieve kernel alone over one 2^30-number segment: its multiplies
        # are the SPRP tests of the candidates it leaves (estimated from the
        # depth as above; the sieving itself is shifts, ORs and atomics)
        seg = out["segment_2p30"]
        cand_per_number = cand / np.log(2.0**64)
        sieve_ops = cand_per_number * (20.0 * (k - 5) + 12.0) * min(width, ckpt)
        out["sieve_roofline"] = {"executed_ops_per_number": cand_per_number * (20.0 * (k - 5) + 12.0),
                                 "achieved_tops": sieve_ops / (seg["sieve_ms"] * 1e-3) / 1e12,
                                 "frac_chain_peak": sieve_ops / (seg["sieve_ms"] * 1e-3) / chain_peak,
                                 "note": "candidates per number estimated as 0.5615 / ln 2^depth (Mertens)"}
    golden = ROOT / "tests" / "golden" / "ref_long.json"
    if golden.exists():
        g = json.loads(golden.read_text())["config3"]
        if g["lo"] == lo and g["hi"] == hi:
            out["reference_checksum_equal"] = bool(out["checksum"] == g["checksum"] and cnt == g["prp_count"])
    return out


def compare_batched_plain(ww, local: int, units: list, workload: str, tune_units: int = 32,
                          force_cfg: tuple | None = None, fused_units: int | None = None) -> dict:
    """Plain = one range per launch sequence (clear, sieve, test, read)
    through the context API; batched = one persistent CUDA-graph launch over
    the tile queue after the autotuner picked the configuration.  Per-unit
    checksums, PRP counts and hit counts must agree.  The batched launch is
    warmed on a subset of the units (the autotuner has already run every
    configuration), so at the mix's full size each path runs once.
    fused_units: how many of the units also run one launch sequence per range
    with the fused test kernel (None: all)."""
    ctx = ww.Context(local, max_prps=ww.prp_count_bound(0, 1 << 30), max_hits=15000)
    b = ww.Batch(ctx)
    if force_cfg:
        b.set_config(*force_cfg)
        cfg = b.config()
    else:
        cfg, _ = b.tune(units[:tune_units])
    b.run(units[:64])  # warm: graph capture of the batched launch
    ctx.marker(0)
    res = b.run(units)
    ctx.marker(1)
    ctx.sync()
    batch_ms = ctx.elapsed_ms(0, 1)
    prps = sum(r["prp_count"] for r in res)
    # plain, the reference program's flow: per range, sieve -> Wieferich ->
    # WSS kernels with a checkpoint (sync, counters and hits read back,
    # clear) every 2^30 numbers and at the range's end
    ckpt = 1 << 30
    # warm the plain path as the batched one was: its first launch wide
    # enough for the large deep primes builds their table and mark bitmap
    wa = units[0][0]
    ctx.clear_results()
    ctx.clear_segment()
    ctx.sieve_prp(wa, wa + (1 << 27))
    ctx.wieferich()
    ctx.wallsunsun()
    ctx.sync()
    ctx.clear_results()
    t0 = time.perf_counter()
    plain = []
    for a, z in units:
        cks, cnt, hits = 0, 0, 0
        start = a
        ctx.clear_results()
        while start < z:
            stop = min(start + ckpt, z)
            ctx.clear_segment()
            ctx.sieve_prp(start, stop)
            ctx.wieferich()
            ctx.wallsunsun()
            ctx.sync()
            k = ctx.counters()
            if k["result_count"]:
                ctx.hits()
            cks, cnt, hits = (cks + k["checksum"]) % 2**64, cnt + k["total_prp_count"], hits + k["result_count"]
            ctx.clear_results()
            start = stop
        plain.append((cks, cnt, hits))
    plain_s = time.perf_counter() - t0
    equal = all((r["checksum"], r["prp_count"], r["hits"]) == p for r, p in zip(res, plain))
    # the same ranges one per launch sequence with the fused test kernel
    nf = len(units) if fused_units is None else min(fused_units, len(units))
    t0 = time.perf_counter()
    alone = [ctx.run_range(a, z) for a, z in units[:nf]]
    fused_s = time.perf_counter() - t0
    equal_fused = all(r["checksum"] == a["checksum"] and r["prp_count"] == a["total_prp_count"] and
                      r["hits"] == a["result_count"] for r, a in zip(res, alone))
    ctx.close()
    numbers = sum(z - a for a, z in units)
    fused_prps = sum(r["prp_count"] for r in res[:nf])
    ratio = plain_s / (batch_ms * 1e-3)
    return {"workload": workload, "units": len(units),
            "numbers": numbers, "prps": prps, "batched_primes_per_s": prps / (batch_ms * 1e-3),
            "plain_primes_per_s": prps / plain_s, "batched_numbers_per_s": numbers / (batch_ms * 1e-3),
            "speedup_batched_vs_plain": ratio, "target_1p5x_met": bool(ratio >= 1.5),
            "plain_definition": "per range: sieve, Wieferich, WSS kernels; checkpoint sync + read-back "
                                "every 2^30 numbers (the reference program's loop), in the same process",
            "per_unit_bit_identical": bool(equal and equal_fused),
            "plain_fused": {"units": nf, "primes_per_s": fused_prps / fused_s if nf else None,
                            "definition": "per range: sieve, fused Wieferich+WSS kernel, read-back"},
            "tuned_config": {"seg_words": cfg[0], "seg_bytes": 4 * cfg[0], "threads": cfg[1],
                             "primes_per_thread": cfg[2], "joint_test_loop": cfg[3]}}


def compare_batched_per_run(ww, local: int, units: list, workload: str) -> dict:
    """The reference's deployment: one program run per range (a BOINC work
    unit), each with its own device set-up, work-size profiling and start-up
    self-test (main.cpp:959-1107, 590-738), here bin/wwocl started once per
    range; against one batched launch over the same ranges.  Each run's
    final checksum (results file) must equal the batched per-range one."""
    import tempfile

    exe = ROOT / "wwocl-boinc_b200" / "bin" / "wwocl"
    if not exe.exists():
        return {"workload": workload, "unavailable": "bin/wwocl not built"}
    ctx = ww.Context(local, max_prps=1 << 20, max_hits=15000)
    b = ww.Batch(ctx)
    b.run(units)  # warm
    ctx.marker(0)
    res = b.run(units)
    ctx.marker(1)
    ctx.sync()
    batch_ms = ctx.elapsed_ms(0, 1)
    ctx.close()
    equal = True
    t0 = time.perf_counter()
    for (a, z), r in zip(units, res):
        with tempfile.TemporaryDirectory() as d:
            p = subprocess.run([str(exe), str(a), str(z), "-device", str(local)], cwd=d, capture_output=True,
                               text=True, timeout=600)
            lines = (Path(d) / "results-WW.txt").read_text().splitlines() if p.returncode == 0 else []
        equal &= bool(lines) and lines[-1] == "%016X" % r["checksum"]
    per_run_s = time.perf_counter() - t0
    prps = sum(r["prp_count"] for r in res)
    return {"workload": workload, "units": len(units), "prps": prps,
            "batched_primes_per_s": prps / (batch_ms * 1e-3), "per_run_primes_per_s": prps / per_run_s,
            "speedup_batched_vs_per_run": per_run_s / (batch_ms * 1e-3),
            "per_run_definition": "bin/wwocl START END once per range: device set-up, work-size profiling, "
                                  "start-up self-test, the range, results file",
            "checksums_equal": bool(equal)}


def run_batched_vs_plain(ww, local: int, n_units: int, force_cfg: tuple | None = None) -> dict:
    """The seed-11 uneven mix (4096 units, widths log-uniform in [1e6, 1e10],
    starts uniform in [1e15, 2^64-1e10], multiples of 30): its first n_units
    units (all 4096 by default), and separately its first 256 units narrower
    than 1e8 (where one launch sequence per range leaves most of the GPU
    idle).  The per-process comparison (one program run per range) is a
    deployment note on 8 units, not the batching result."""
    mix = ww.uneven_units(11, 4096)
    what = "all 4096 units" if n_units >= 4096 else f"first {n_units} units"
    out = compare_batched_plain(ww, local, mix[:n_units], f"{what} of the seed-11 uneven mix", force_cfg=force_cfg,
                                fused_units=min(n_units, 128))
    narrow = [u for u in mix if u[1] - u[0] < 10**8][:256]
    out["narrow_units"] = compare_batched_plain(
        ww, local, narrow, f"first {len(narrow)} units of the same mix narrower than 1e8", force_cfg=force_cfg)
    out["per_run"] = compare_batched_per_run(ww, local, mix[:8], "first 8 units of the same mix, one program "
                                             "run per range (deployment note, not the batching target)")
    return out


def run_serving(ww, local: int, seconds: float, rate: float = 200.0, seed: int = 13, check_cpu: int = 12):
    """Config 5: Poisson arrivals at `rate` req/s for `seconds` (120 s in full),
    widths log-uniform in [1e5, 1e9], starts uniform in [1e12, 2^64-1e9].
    Latency = completion time - arrival time on the host monotonic clock."""
    rng = np.random.default_rng(seed)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        arrivals.append(t)
    widths = np.exp(rng.uniform(np.log(1e5), np.log(1e9), len(arrivals)))
    starts = rng.integers(10**12, 2**64 - 10**9, len(arrivals), dtype=np.uint64)
    reqs = [(i, int(s), int(s) + int(w)) for i, (s, w) in enumerate(zip(starts, widths))]
    ctx = ww.Context(local, max_prps=1 << 20, max_hits=15000)
    srv = ww.Server(ctx, prp_pool_bytes=24 << 30, max_active=256, epoch_tiles=0, store_prps=True)  # one wave of resident CTAs per step
    srv.submit([(10**9, 10**12, 10**12 + 10**6)])  # warm-up request
    srv.drain()
    done = {}
    i = 0
    t0 = time.monotonic()
    while len(done) < len(reqs):
        now = time.monotonic() - t0
        batch = []
        while i < len(reqs) and arrivals[i] <= now:
            batch.append(reqs[i])
            i += 1
        if batch:
            srv.submit(batch)
        q, a, _ = srv.status()
        if q == 0 and a == 0:
            if i < len(reqs):
                time.sleep(max(0.0, min(arrivals[i] - now, 0.01)))
            continue
        for r in srv.step():
            done[r["id"]] = r
    wall = time.monotonic() - t0
    lat = np.array([done[k]["t_done"] - (t0 + arrivals[k]) for k in range(len(reqs))]) * 1e3
    prps = sum(r["prp_count"] for r in done.values())
    numbers = sum(b - a for _, a, b in reqs)
    ok_status = all(r["status"] == 0 for r in done.values())
    cpu_equal = None
    try:
        from oracle.oracle import RefCPU

        if RefCPU.available():
            ref = RefCPU()
            small = sorted(reqs, key=lambda r: r[2] - r[1])[:check_cpu]
            cpu_equal = all(ref.scan_range(a, b)["checksum"] == done[k]["checksum"] for k, a, b in small)
    except OSError:
        cpu_equal = None
    srv.close()
    ctx.close()
    return {"workload": f"Poisson {rate:g} req/s for {seconds:g} s (config 5, seed 13), widths 1e5..1e9",
            "requests": len(reqs), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()), "primes_per_s": prps / wall, "numbers_per_s": numbers / wall,
            "offered_numbers_per_s": numbers / seconds, "all_ok": bool(ok_status),
            "cpu_checksum_equal_on_smallest": cpu_equal}


def summarize(line: dict, extra: dict) -> dict:
    """Short figures of every leg, for the end of the JSON line."""
    def r(x, d=3):
        return None if x is None else float(f"{x:.{d}g}")

    rl = line["roofline"]
    cpu = line.get("cpu_baseline") or {}
    out = {"config2_fixed_list": {"primes_per_s": r(line["value"], 4), "e2e_primes_per_s": r(line["e2e"]["value"], 4),
                                  "frac_chain_peak_ref_ops": r(rl["frac"]),
                                  "frac_chain_peak_executed": r(rl["executed"]["frac"]),
                                  "frac_madlo_peak_ref_ops": r(rl["mad_lo_only"]["frac"]),
                                  "frac_madlo_peak_executed": r(rl["mad_lo_only"]["frac_executed"]),
                                  "cpu_primes_per_s": r(cpu.get("value"), 4),
                                  "cpu_checksum_match": cpu.get("checksum_match")}}
    if "range_pipeline" in extra:
        g = extra["range_pipeline"]
        out["config3_plain_range"] = {"primes_per_s": r(g["primes_per_s"], 4), "numbers_per_s": r(g["numbers_per_s"], 4),
                                      "sieve_ms_2p30": r(g["segment_2p30"]["sieve_ms"]),
                                      "test_ms_2p30": r(g["segment_2p30"]["test_ms"]),
                                      "sieve_frac_chain_peak": r((g.get("sieve_roofline") or {}).get("frac_chain_peak")),
                                      "checksum": g["checksum"],
                                      "checksum_equal_reference": g.get("reference_checksum_equal")}
    if "batched_vs_plain" in extra:
        g = extra["batched_vs_plain"]
        out["config4_batched_vs_plain"] = {
            "units": g["units"], "batched_primes_per_s": r(g["batched_primes_per_s"], 4),
            "plain_primes_per_s": r(g["plain_primes_per_s"], 4), "ratio": r(g["speedup_batched_vs_plain"]),
            "target_1p5x_met": g["target_1p5x_met"], "per_unit_bit_identical": g["per_unit_bit_identical"],
            "narrow_ratio": r(g["narrow_units"]["speedup_batched_vs_plain"]),
            "per_process_ratio_note": r(g["per_run"].get("speedup_batched_vs_per_run")),
            "tuned": "%d/%d/%d/%d" % tuple(g["tuned_config"][k] for k in ("seg_words", "threads", "primes_per_thread",
                                                                           "joint_test_loop"))}
    if "serving" in extra:
        g = extra["serving"]
        out["config5_serving"] = {"requests": g["requests"], "p50_ms": r(g["p50_ms"]), "p99_ms": r(g["p99_ms"]),
                                  "max_ms": r(g["max_ms"]), "primes_per_s": r(g["primes_per_s"], 4),
                                  "all_ok": g["all_ok"], "cpu_checksum_equal": g["cpu_checksum_equal_on_smallest"]}
    return out


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (no CPU fallback)")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                              device_id=torch.device("cuda", local))

    import wwcuda as ww

    n = args.n_primes
    t0 = time.perf_counter()
    primes, _ = ww.random_primes(SEED + rank, n, device=local)
    gen_s = time.perf_counter() - t0
    host = torch.from_numpy(primes.view(np.int64)).pin_memory()
    host_ptr = host.data_ptr()

    ctx = ww.Context(local, max_prps=n, max_hits=15000)
    ctx.load_prps_ptr(host_ptr, n)
    ctx.sync()

    # integer-multiply peaks on this device, at this moment (roofline
    # denominators): the 64x64->128 mad.lo/mad.hi carry chain the op count is
    # made of (8 multiply instructions per product), and mad.lo alone
    chain_peak, _ = ww.pipe_bench(3, device=local)
    madlo_peak, _ = ww.pipe_bench(0, device=local)

    def step():
        ctx.clear_results()
        ctx.test_prps()

    for _ in range(args.warmup):
        step()
    ctx.sync()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing
    barrier()
    with ClockSampler(local) as clocks:
        ctx.marker(0)
        for _ in range(args.steps):
            step()
        ctx.marker(1)
        ctx.sync()
    dev_ms = ctx.elapsed_ms(0, 1)
    c = ctx.counters()
    if c["overflow"]:
        raise SystemExit(f"overflow flag {c['overflow']}")
    checksum = c["checksum"]
    t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(t.item())
    value = n * world * args.steps / (ms_max * 1e-3)

    # ---- end to end through the C ABI: H2D list, test, D2H counters
    hit_bytes = 24
    barrier()
    t_e0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.clear_results()
        ctx.test_prps_host_ptr(host_ptr, n)  # H2D copy of each chunk overlaps the test of the previous one
        k = ctx.counters()
        if k["result_count"]:
            ctx.hits()
    barrier()
    e2e_s = time.perf_counter() - t_e0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
    e2e_value = n * world * args.steps / float(te.item())
    hits_per_step = k["result_count"]
    e2e_checksum = k["checksum"]

    if world > 1:
        torch.distributed.barrier()
    if rank != 0:
        ctx.close()
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    # ---- roofline (IMAD pipe) and CPU baseline on rank 0
    per_prime, per_prime_run = algorithmic_imad_per_prime(primes)
    launch_ms = dev_ms / args.steps
    achieved = per_prime * n / (launch_ms * 1e-3)
    achieved_run = per_prime_run * n / (launch_ms * 1e-3)
    roofline = {"bound": "imad", "achieved": achieved / 1e12, "peak": chain_peak / 1e12, "unit": "Tops/s",
                "frac": achieved / chain_peak, "traffic": profile_traffic(),
                "peak_source": "measured live: 64x64->128 mad.lo.cc/madc.hi carry chains on every SM, per "
                               "multiply instruction (ww_pipe_bench mode 3)",
                "ops_per_prime": per_prime,
                "ops_source": "reference kernels' algorithm: 40(k-3) + 128(k-1) 32-bit multiplies per prime",
                "frac_note": "frac counts the reference algorithm's multiplies, more than this kernel executes, so "
                             "it can pass 1.0; executed.frac is the pipe-occupancy view",
                "executed": {"ops_per_prime": per_prime_run, "achieved": achieved_run / 1e12,
                             "frac": achieved_run / chain_peak,
                             "note": "multiplies k_test_prps itself runs: 114(k-6) + 168 (ladders started from their top bits, three-product squares of the low digit)"},
                "mad_lo_only": {"peak": madlo_peak / 1e12, "frac": achieved / madlo_peak,
                                "frac_executed": achieved_run / madlo_peak},
                "hbm": {"bytes_per_launch": 16 * n, "GBps": 16 * n / (launch_ms * 1e-3) / 1e9,
                        "peak_GBps": json.loads(PEAKS.read_text())["hbm_gbs"] if PEAKS.exists() else 6650.0,
                        "peak_source": "measured copy bandwidth" if PEAKS.exists()
                        else "fallback 6.65 TB/s (no measured peaks file)"}}

    cpu = None
    if not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            take = args.cpu_sample
            if take <= 0:  # calibrate on 2^18 primes, then size the sample to --cpu-seconds
                r0, _, _ = cpu_reference_rate(primes[: 1 << 18], threads)
                take = max(1 << 20, int(r0 * args.cpu_seconds))
            sample = primes[: min(take, n)]
            rate, cks_cpu, dt = cpu_reference_rate(sample, threads)
            ctx2 = ww.Context(local, max_prps=sample.size, max_hits=15000)
            ctx2.load_prps(sample)
            ctx2.clear_results()
            ctx2.test_prps()
            ctx2.sync()
            gpu_cks = ctx2.counters()["checksum"]
            ctx2.close()
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"first {sample.size} primes of the list, wwcpu.cpp on {threads} threads, {dt:.1f} s",
                   "checksum_match": bool(gpu_cks == cks_cpu)}
        except (FileNotFoundError, OSError) as e:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    extra = {}
    if world > 1:  # the single-GPU legs below are measured at N = 1; a scaling run keeps its GPUs short
        args.range_width = args.batch_units = args.serve_seconds = 0
    if args.range_width:
        extra["range_pipeline"] = run_range_pipeline(ww, local, int(args.range_width), chain_peak=chain_peak)
    if args.batch_units:
        force = tuple(int(x) for x in args.batch_config.split("/")) if args.batch_config else None
        extra["batched_vs_plain"] = run_batched_vs_plain(ww, local, args.batch_units, force)
    if args.serve_seconds:
        extra["serving"] = run_serving(ww, local, args.serve_seconds)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": config(args, world), **extra,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": 32 + hit_bytes * hits_per_step,
                    "call": "ww_test_prps_host (pinned list, copy of chunk k+1 overlapping the test of chunk k) "
                            "+ ww_read_counters", "checksum_equal": bool(e2e_checksum == checksum)},
            "gpu_launches": args.steps, "roofline": roofline, "cpu_baseline": cpu,
            "clocks": clocks.summary(), "checksum": "%016X" % checksum, "list_gen_s": gen_s}
    # last key: every leg's results in a few hundred bytes (kept by a reader
    # that keeps only the end of the output)
    line["summary"] = summarize(line, extra)
    print(json.dumps(line))
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
