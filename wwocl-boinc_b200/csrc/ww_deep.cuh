// ww_deep.cuh -- deep-sieve table and index helpers (host and device).
#pragma once

#include "ww_arith.cuh"
#include "ww_deep_table.h"

namespace ww {

// After the small primes 3..113, each segment is sieved by the primes
// 127 < r < 2^16 of ww_deep_table.h.  A multiple n of r can only be a base-2
// (strong) pseudoprime when ord_r(2) | n - 1, i.e. n = r (mod r * ord_r(2));
// those multiples are put on a rescue list before the marking, so the
// candidate set (unmarked bits plus the rescue list) still contains every
// number with no factor <= 113 that passes the base-2 strong PRP test --
// the reference's PRP set exactly -- while about 2.35x fewer candidates
// reach the PRP test.  Primes with ord_r(2) < 32 are left out of the table
// so their rescue classes stay sparse.

constexpr int kRescueCap = 2048;

// bit index (j) of the first odd multiple of r at or after `first` (odd):
// first + 2j = 0 (mod r)
WW_HD u32 deep_first_multiple(u64 first, u32 r, u32 t32r) {
    const u32 res = ((u32)(first >> 32) % r * t32r + (u32)first % r) % r;
    return ((r - res) % r) * ((r + 1) >> 1) % r;
}

// offset (even, in integers) from `first` to the first n = r (mod m), n odd, n >= first
WW_HD u64 deep_first_rescue(u64 first, u32 r, u32 m, u32 t32m) {
    const u64 res = ((u64)((u32)(first >> 32) % m) * t32m + (u32)first % m) % m;
    u64 d = ((u64)r + m - res) % m;
    if (d & 1) d += m;  // only for odd m: first is odd, so an even offset keeps n odd
    return d;
}

// distance between consecutive odd members of the class r (mod m): with m
// even every member is odd (r is), with m odd every other one is
WW_HD u64 deep_rescue_step(u32 m) { return (m & 1) ? 2ull * m : (u64)m; }


}  // namespace ww
