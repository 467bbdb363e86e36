"""Generate ww_deep_table.h: the deep-sieve primes 113 < r < 2^20, one row
each with o = ord_r(2) and the constants the device uses to start a
prime's marking in a segment without divisions:

    rinv = r^-1 mod 2^64          (exact quotient n / r of a multiple n)
    mr   = floor(2^64 / r)        (Barrett reduction of a 64-bit number mod r)
    mo   = floor(2^64 / o)        (the same mod o)

The rows come in bands: WW_DEEP_ROWS_<b>(X) holds the primes with
2^(b-1) <= r < 2^b (b = 16 for all r < 2^16), and WW_DEEP_COUNT_<b> counts
the rows below 2^b, so a build that sieves to 2^B compiles only the bands up
to B.

The build (wwocl-boinc_b200/Makefile) runs it; the header is not committed.
"""
from pathlib import Path

LIMIT_BITS = 20


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
    for r in primes_below(1 << LIMIT_BITS):
        if r <= 113:
            continue
        o = order_of_two(r)
        assert o >= 3
        rows.append((r, o, pow(r, -1, 2**64), 2**64 // r, 2**64 // o))
    out = Path(__file__).resolve().parent / "ww_deep_table.h"
    lines = ["// Generated by gen_deep_table.py -- do not edit.",
             "// Deep-sieve primes 113 < r < 2^%d in bands by bit length, one row each:" % LIMIT_BITS,
             "// X(r, o = ord_r(2), r^-1 mod 2^64, floor(2^64 / r), floor(2^64 / o))",
             "#pragma once"]
    for b in range(16, LIMIT_BITS + 1):
        lines.append("#define WW_DEEP_COUNT_%d %d" % (b, sum(1 for row in rows if row[0] < (1 << b))))
    for b in range(16, LIMIT_BITS + 1):
        band = [row for row in rows if row[0] < (1 << b) and (b == 16 or row[0] >= (1 << (b - 1)))]
        lines.append("#define WW_DEEP_ROWS_%d(X) \\" % b)
        for i in range(0, len(band), 2):
            lines.append("    " + " ".join("X(%du, %du, 0x%016xull, 0x%016xull, 0x%016xull)" % row
                                           for row in band[i:i + 2]) + " \\")
        lines.append("")
    out.write_text("\n".join(lines) + "\n")
    print(len(rows), "rows")


if __name__ == "__main__":
    main()
