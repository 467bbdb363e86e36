"""Seeded random ranges against the oracle: magnitudes log-uniform over
[127, 2^64), widths from one number to 2e5, so starts fall on every wheel
residue and segments end at arbitrary bits.  Three device paths must agree
with the oracle bit for bit: the context path, the drop-in launchers, and
the batched engine with all ranges as units of one launch."""
from __future__ import annotations

import math
import random

import pytest

pytestmark = pytest.mark.gpu


def _ranges(seed=2026, n=200):
    rng = random.Random(seed)
    out = []
    for _ in range(n):
        lo = int(math.exp(rng.uniform(math.log(127), math.log(2**64 - 2))))
        w = int(math.exp(rng.uniform(0, math.log(2e5))))
        out.append((lo, min(lo + w, 2**64 - 1)))
    out += [(127, 128), (2**64 - 3, 2**64 - 1), (2**32 - 7, 2**32 + 7), (2**63 - 101, 2**63 + 99)]
    return out


@pytest.fixture(scope="module")
def want(oracle):
    return [oracle.scan_range(a, b, hit_cap=10000) for a, b in _ranges()]


def test_context_path(ww, want):
    with ww.Context(0, max_prps=1 << 18, max_hits=10000) as c:
        for (a, b), (summ, _, hits) in zip(_ranges(), want):
            got = c.run_range(a, b)
            assert got["overflow"] == 0
            assert (got["total_prp_count"], got["checksum"]) == (summ["prp_count"], summ["checksum"]), (a, b)
            assert sorted(got["hits"]) == sorted(hits), (a, b)


def test_batched_units(ww, want):
    units = _ranges()
    with ww.Context(0, max_prps=1 << 18, max_hits=10000) as c:
        b = ww.Batch(c)
        got = b.run(units)
        all_hits = b.hits()
    for i, ((a, bb), (summ, _, hits)) in enumerate(zip(units, want)):
        assert (got[i]["prp_count"], got[i]["checksum"], got[i]["hits"]) == \
               (summ["prp_count"], summ["checksum"], len(hits)), (a, bb)
        assert sorted(h[1:] for h in all_hits if h[0] == i) == sorted(hits), (a, bb)


def test_drop_in_launchers(ww, want):
    from test_gpu_parity import _KernelSequence

    import torch

    s = torch.cuda.Stream(torch.device("cuda", 0))
    for (a, b), (summ, _, hits) in zip(_ranges(), want):
        try:
            start, _ = ww.find_wheel_offset(a)
        except ww.WWError:
            start = b  # nothing prime to 30 from a on
        if start >= b:
            assert summ["prp_count"] == 0
            continue
        r = {"lo": a, "hi": b, "prp_count": summ["prp_count"], "checksum": "%016X" % summ["checksum"],
             "cpu_results": len(hits)}
        seq = _KernelSequence(ww, r, cap=1 << 17, nres=10000)
        seq.launch(s.cuda_stream)
        s.synchronize()
        seq.check((a, b))
