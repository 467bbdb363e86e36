// ww_deep.cuh -- deep-sieve table and index helpers (host and device).
#pragma once

#include "ww_arith.cuh"
#include "ww_deep_table.h"

namespace ww {

// After the small primes 3..113, each segment is sieved by the primes
// 113 < r < 2^WW_DEEP_BITS of ww_deep_table.h.
//
// The PRP set is "no factor <= 113 and a base-2 strong probable prime", so a
// multiple n = r*k of a deep prime r may only be marked when it can never be
// a base-2 (strong) pseudoprime.  With o = ord_r(2): 2^(n-1) = 1 (mod r)
// needs o | n - 1, and since o | r - 1, n = r*k = k (mod o).  So n is marked
// exactly when k != 1 (mod o).  The multiples with k = 1 (mod o) -- r itself
// and every possible pseudoprime with the factor r -- stay candidates and
// meet the PRP test.  The marking loop carries k mod o along (k grows by 2
// per odd multiple), so the candidate set is the reference's PRP set plus a
// few composites the PRP test rejects, for any sieve depth.

#ifndef WW_DEEP_BITS
#define WW_DEEP_BITS 20
#endif
// the table in use: the bands of primes below 2^WW_DEEP_BITS
#if WW_DEEP_BITS == 16
#define WW_DEEP_ROWS(X) WW_DEEP_ROWS_16(X)
#elif WW_DEEP_BITS == 17
#define WW_DEEP_ROWS(X) WW_DEEP_ROWS_16(X) WW_DEEP_ROWS_17(X)
#elif WW_DEEP_BITS == 18
#define WW_DEEP_ROWS(X) WW_DEEP_ROWS_16(X) WW_DEEP_ROWS_17(X) WW_DEEP_ROWS_18(X)
#elif WW_DEEP_BITS == 19
#define WW_DEEP_ROWS(X) WW_DEEP_ROWS_16(X) WW_DEEP_ROWS_17(X) WW_DEEP_ROWS_18(X) WW_DEEP_ROWS_19(X)
#elif WW_DEEP_BITS == 20
#define WW_DEEP_ROWS(X) \
    WW_DEEP_ROWS_16(X) WW_DEEP_ROWS_17(X) WW_DEEP_ROWS_18(X) WW_DEEP_ROWS_19(X) WW_DEEP_ROWS_20(X)
#else
#error "WW_DEEP_BITS must be 16..20"
#endif
#define WW_DEEP_CAT2(a, b) a##b
#define WW_DEEP_CAT(a, b) WW_DEEP_CAT2(a, b)
#define WW_DEEP_COUNT WW_DEEP_CAT(WW_DEEP_COUNT_, WW_DEEP_BITS)
constexpr int kDeepUse = WW_DEEP_COUNT;

struct DeepRow {
    u32 r, o;  // prime, order of 2 mod r
    u64 rinv;  // r^-1 mod 2^64
    u64 mr;    // floor(2^64 / r)
    u64 mo;    // floor(2^64 / o)
};

// x mod d for d < 2^63 with m = floor(2^64 / d): the quotient estimate is
// short by at most one.
WW_HD u64 barrett_mod(u64 x, u64 d, u64 m) {
    const u64 r = x - mul_hi(x, m) * d;
    return r >= d ? r - d : r;
}

// Where a deep prime starts in a segment whose bit j is the odd number
// first + 2j (first odd): j0, the bit of the first odd multiple n0 >= first,
// and n0 / r mod o.  When n0 would pass 2^64 the segment ends before it
// (j0 >= the segment's valid bits), so its km0 is never used.
WW_HD void deep_start(u64 first, const DeepRow &e, u32 &j0, u32 &km0) {
    const u64 res = barrett_mod(first, e.r, e.mr);
    u64 t = res ? e.r - res : 0;  // first + t = 0 (mod r)
    if (t & 1) t += e.r;          // first is odd: the next odd multiple is an even step away
    j0 = (u32)(t >> 1);
    const u64 k0 = (first + t) * e.rinv;  // exact quotient of a multiple of r
    km0 = (u32)barrett_mod(k0, e.o, e.mo);
}

// bit index (j) of the first odd multiple of r at or after `first` (odd):
// first + 2j = 0 (mod r); t32r = 2^32 mod r (the small primes of the host
// twin of the sieve)
WW_HD u32 deep_first_multiple(u64 first, u32 r, u32 t32r) {
    const u32 res = ((u32)(first >> 32) % r * t32r + (u32)first % r) % r;
    return ((r - res) % r) * ((r + 1) >> 1) % r;
}

}  // namespace ww
