"""Generate ww_deep_table.h: the primes 127 < r < 2^16 whose multiplicative
order of 2 is at least 32, with o = ord_r(2), m = r*o and the constants
2^32 mod r, 2^32 mod m used for 32-bit modular reductions on the device.

Run from the repository root:  python wwocl-boinc_b200/csrc/gen_deep_table.py
"""
from pathlib import Path

LIMIT = 1 << 16
MIN_ORDER = 32


def primes_below(n):
    s = bytearray([1]) * n
    s[0:2] = b"\0\0"
    for i in range(2, int(n ** 0.5) + 1):
        if s[i]:
            s[i * i::i] = bytearray(len(range(i * i, n, i)))
    return [i for i in range(n) if s[i]]


def order_of_two(r):
    m = r - 1
    fac, x, d = [], m, 2
    while d * d <= x:
        if x % d == 0:
            fac.append(d)
            while x % d == 0:
                x //= d
        d += 1
    if x > 1:
        fac.append(x)
    o = m
    for q in fac:
        while o % q == 0 and pow(2, o // q, r) == 1:
            o //= q
    return o


def main():
    rows = []
    for r in primes_below(LIMIT):
        if r <= 113:
            continue
        o = order_of_two(r)
        if o < MIN_ORDER:
            continue
        m = r * o
        assert m < 2**32
        rows.append((r, m, (2**32) % r, (2**32) % m))
    out = Path(__file__).resolve().parent / "ww_deep_table.h"
    lines = ["// Generated by gen_deep_table.py -- do not edit.",
             "// Deep-sieve primes 127 < r < 2^16 with ord_r(2) >= %d, one row each:" % MIN_ORDER,
             "// X(r, m = r * ord_r(2), 2^32 mod r, 2^32 mod m)",
             "#pragma once",
             "#define WW_DEEP_COUNT %d" % len(rows),
             "#define WW_DEEP_ROWS(X) \\"]
    for i in range(0, len(rows), 4):
        lines.append("    " + " ".join("X(%du, %du, %du, %du)" % row for row in rows[i:i + 4]) + " \\")
    lines.append("")
    out.write_text("\n".join(lines) + "\n")
    print(len(rows), "primes;", "excluded (small order):",
          [r for r in primes_below(LIMIT) if r > 113 and order_of_two(r) < MIN_ORDER])


if __name__ == "__main__":
    main()
