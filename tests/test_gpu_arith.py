"""Operand-level parity of the device arithmetic: every operation the test and
sieve kernels are built from (two-digit products, squares, the exit from
Montgomery form, sums and differences mod p^2, and the mod-p Montgomery
product, sum and reduction of the PRP test), run on the GPU through the same
inline-PTX sequences the kernels execute, against exact integer arithmetic,
including the digits 0, 1, p-1 and moduli at the 2^32, 2^62, 2^63 and 2^64
edges."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODS = [127, 131, 65521, 2**31 - 1, 4294967291, 4294967311, 2**32 + 15, 2**61 - 1, 2**62 - 57, 2**62 + 135,
        9223372036854775783, 2**63 + 29, 2**64 - 59, 2**64 - 1, 2**64 - 3, 12297829382473034411,
        0xFFFFFFFF00000001, 0x80000000FFFFFFFF]


def _exact(op, p, x0, x1, y0, y1):
    n = p * p
    x, y = x0 + p * x1, y0 + p * y1
    if op <= 2:
        rinv = pow(2**64, -1, n)
        z = (x * y if op == 0 else x * x if op == 1 else x) * rinv % n
    elif op == 3:
        z = (x + y) % n
    elif op == 4:
        z = (x - y) % n
    elif op == 5:
        z = 2 * x % n
    else:
        rinv = pow(2**64, -1, p)
        z = (x0 * y0 if op == 6 else x0 + y0 if op == 7 else x0 + (x1 << 64)) * (rinv if op != 7 else 1) % p
        return z, 0
    return z % p, z // p


def _check(ww, p, cases):
    xy = np.array(cases, dtype=np.uint64)
    for op in range(9):
        got = ww.devtest_m2(op, p, xy)
        want = [_exact(op, p, *c) for c in cases]
        bad = [i for i, g in enumerate(got) if (int(g[0]), int(g[1])) != want[i]]
        assert not bad, (hex(p), op, [cases[i] for i in bad[:3]], [tuple(map(int, got[i])) for i in bad[:3]],
                         [want[i] for i in bad[:3]])


@pytest.mark.parametrize("p", MODS)
def test_device_arithmetic_edge_operands(ww, p):
    rng = np.random.default_rng(p % 1000)
    special = sorted({0, 1, 2, p - 1, p - 2, p // 2, (p + 1) // 2, 2**32 % p, (2**32 - 1) % p, p - 2**31 % p,
                      (2**63) % p, (2**64 - 1) % p}
                     | {int(v) % p for v in rng.integers(0, 2**63, 4, dtype=np.uint64)})
    cases = [(a, b, c, d) for a in special for b in special[:6] for c in special[:6] for d in special]
    _check(ww, p, cases)


def test_device_arithmetic_random(ww):
    rng = np.random.default_rng(5)
    for _ in range(24):
        lo = int(rng.choice([2**40, 2**62, 2**63]))
        p = int(rng.integers(lo, 2**64 - 1, dtype=np.uint64)) | 1
        cases = [tuple(int(v) % p for v in rng.integers(0, 2**64 - 1, 4, dtype=np.uint64)) for _ in range(2000)]
        _check(ww, p, cases)
