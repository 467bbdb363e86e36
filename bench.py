"""Benchmark of the WWocl search path on B200: primes tested (Wieferich +
Wall-Sun-Sun) per second on the fixed-list workload -- 2^26 primes in
[2^62, 2^64) drawn from the SplitMix64 stream of seed 7 and kept when they
pass deterministic Miller-Rabin.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one fused Wieferich + Wall-Sun-Sun launch over the whole list
(`value`: list resident in HBM; `e2e`: the same step through the C ABI with
the list copied from pinned host memory and the counters read back, every
step).  Under torchrun each rank tests its own list (seed 7 + rank): weak
scaling, no data-path collective.  Rank 0 prints one JSON line.
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
    ap.add_argument("--cpu-sample", type=int, default=1 << 20,
                    help="primes in the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-units", type=int, default=128,
                    help="units of the uneven mix for the batched-vs-plain line (0: skip)")
    ap.add_argument("--serve-seconds", type=float, default=10.0,
                    help="length of the Poisson request stream (0: skip)")
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


def algorithmic_imad_per_prime(primes: np.ndarray) -> float:
    """32-bit multiply-adds one prime needs in the algorithm the kernel runs,
    counted with the survey's fixed costs: a 64x64->128 product = 8, a low
    64-bit product = 4, a high 64-bit product = 8; so a two-digit square
    mod p^2 = 40 and a product = 48.  With k = bitlength(p): Wieferich does
    k-2 squarings, the Lucas ladder k-1 (square + product), plus two
    conversions out of Montgomery form (24 each)."""
    bits = np.floor(np.log2(primes.astype(np.float64))) + 1  # exact away from powers of two
    per = 40.0 * (bits - 2) + 88.0 * (bits - 1) + 48.0
    return float(per.mean())


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


def run_batched_vs_plain(ww, local: int, n_units: int, tune_units: int = 32):
    """Config 4 subsample: the first n_units of the seed-11 uneven mix (widths
    log-uniform in [1e6, 1e10], starts uniform in [1e15, 2^64-1e10], multiples
    of 30).  Plain = one range per launch sequence (clear, sieve, test, read)
    through the context API; batched = one persistent CUDA-graph launch over
    the tile queue after the autotuner picked the configuration.  Per-unit
    checksums and PRP counts must agree."""
    units = ww.uneven_units(11, 4096)[:n_units]
    ctx = ww.Context(local, max_prps=ww.prp_count_bound(0, 1 << 30), max_hits=15000)
    b = ww.Batch(ctx)
    cfg, _ = b.tune(units[:tune_units])
    b.run(units)  # warm
    ctx.marker(0)
    res = b.run(units)
    ctx.marker(1)
    ctx.sync()
    batch_ms = ctx.elapsed_ms(0, 1)
    prps = sum(r["prp_count"] for r in res)
    # plain, config 3's definition: per range, sieve -> Wieferich -> WSS kernels
    # with a checkpoint (sync, counters and hits read back, clear) every 2^30
    # numbers and at the range's end
    ckpt = 1 << 30
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
    # the same ranges one per launch sequence with the fused test kernel
    t0 = time.perf_counter()
    alone = [ctx.run_range(a, z) for a, z in units]
    fused_s = time.perf_counter() - t0
    equal = all(r["checksum"] == a["checksum"] and r["prp_count"] == a["total_prp_count"] and
                r["hits"] == a["result_count"] and (r["checksum"], r["prp_count"], r["hits"]) == p
                for r, a, p in zip(res, alone, plain))
    ctx.close()
    numbers = sum(z - a for a, z in units)
    return {"workload": f"first {n_units} units of the seed-11 uneven mix (config 4)", "units": n_units,
            "numbers": numbers, "prps": prps, "batched_primes_per_s": prps / (batch_ms * 1e-3),
            "plain_primes_per_s": prps / plain_s, "plain_fused_primes_per_s": prps / fused_s,
            "batched_numbers_per_s": numbers / (batch_ms * 1e-3),
            "speedup_batched_vs_plain": plain_s / (batch_ms * 1e-3),
            "speedup_batched_vs_plain_fused": fused_s / (batch_ms * 1e-3),
            "plain_definition": "per range: sieve, Wieferich, WSS kernels; checkpoint sync + read-back "
                                "every 2^30 numbers (config 3)",
            "per_unit_bit_identical": bool(equal),
            "tuned_config": {"seg_words": cfg[0], "seg_bytes": 4 * cfg[0], "threads": cfg[1],
                             "primes_per_thread": cfg[2]}}


def run_serving(ww, local: int, seconds: float, rate: float = 200.0, seed: int = 13, check_cpu: int = 12):
    """Config 5, shortened: Poisson arrivals at `rate` req/s for `seconds`,
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
    srv = ww.Server(ctx, prp_pool_bytes=24 << 30, max_active=256, epoch_tiles=1024, store_prps=True)
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

    # IMAD pipe peak on this device, at this moment (roofline denominator)
    imad_peak, _ = ww.pipe_bench(0, device=local)

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
        ctx.load_prps_ptr(host_ptr, n)
        step()
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

    if world > 1:
        torch.distributed.barrier()
    if rank != 0:
        ctx.close()
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    # ---- roofline (IMAD pipe) and CPU baseline on rank 0
    per_prime = algorithmic_imad_per_prime(primes)
    launch_ms = dev_ms / args.steps
    achieved = per_prime * n / (launch_ms * 1e-3)
    roofline = {"bound": "imad", "achieved": achieved / 1e12, "peak": imad_peak / 1e12, "unit": "Tops/s",
                "frac": achieved / imad_peak, "traffic": profile_traffic(),
                "peak_source": "measured live: mad.lo.u32 chains on every SM (ww_pipe_bench mode 0)",
                "ops_per_prime": per_prime,
                "hbm": {"bytes_per_launch": 16 * n, "GBps": 16 * n / (launch_ms * 1e-3) / 1e9,
                        "peak_GBps": json.loads(PEAKS.read_text())["hbm_gbs"] if PEAKS.exists() else 6650.0}}

    cpu = None
    if not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            sample = primes[: min(args.cpu_sample, n)]
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
    if args.batch_units:
        extra["batched_vs_plain"] = run_batched_vs_plain(ww, local, args.batch_units)
    if args.serve_seconds:
        extra["serving"] = run_serving(ww, local, args.serve_seconds)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": config(args, world), **extra,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": 32 + hit_bytes * hits_per_step},
            "gpu_launches": args.steps, "roofline": roofline, "cpu_baseline": cpu,
            "clocks": clocks.summary(), "checksum": "%016X" % checksum, "list_gen_s": gen_s}
    print(json.dumps(line))
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
