"""Offline model of the request server's scheduling (ww_server_step) on the
200 req/s stream of the serving benchmark: Poisson arrivals for 120 s (seed
13), widths log-uniform in [1e5, 1e9], tiles of 2^20 numbers, 296 resident
CTAs taking one tile each per step, and a step time set by the measured
batched throughput (33.8e9 numbers/s).  It compares the p50 / p99 / max
latency (ms) of three ways of handing out a step's tiles: equal round-robin
shares, oldest request first, and earliest deadline first with deadline =
arrival + 2 x the request's tiles on the whole GPU (the server's policy).

    python wwocl-boinc_b200/serve_sim.py
"""
import numpy as np
rng = np.random.default_rng(13)
arr, t = [], 0.0
while True:
    t += rng.exponential(1 / 200.0)
    if t > 120.0: break
    arr.append(t)
n = len(arr)
widths = np.exp(rng.uniform(np.log(1e5), np.log(1e9), n))
tiles = np.ceil(widths / (1 << 20)).astype(int)
SLOTS, WAVE = 296, 296 * (1 << 20) / 33.8e9
def run(keyf):
    now, i, active, lat, done = 0.0, 0, [], np.zeros(n), 0
    while done < n:
        while i < n and arr[i] <= now and len(active) < 256:
            active.append([arr[i], tiles[i], i]); i += 1
        if not active:
            now = arr[i]; continue
        alloc, rem = {}, SLOTS
        if keyf is None:  # equal round-robin shares
            act = sorted(active, key=lambda a: a[2])
            while rem > 0 and any(a[1] - alloc.get(a[2], 0) > 0 for a in act):
                for a in act:
                    if rem and a[1] - alloc.get(a[2], 0) > 0:
                        alloc[a[2]] = alloc.get(a[2], 0) + 1; rem -= 1
        else:
            for a in sorted(active, key=keyf):
                take = min(a[1], rem); alloc[a[2]] = take; rem -= take
                if rem == 0: break
        now += WAVE + 3e-4
        nxt = []
        for a in active:
            a[1] -= alloc.get(a[2], 0)
            if a[1] <= 0: lat[a[2]] = now - a[0]; done += 1
            else: nxt.append(a)
        active = nxt
    return [round(float(x) * 1e3, 1) for x in (np.percentile(lat, 50), np.percentile(lat, 99), lat.max())]
print("load", round(widths.sum() / 120 / 33.8e9, 3))
print("round-robin", run(None))
print("oldest first", run(lambda a: a[0]))
print("EDF k=2", run(lambda a: a[0] + 2 * tiles[a[2]] * WAVE / SLOTS))
