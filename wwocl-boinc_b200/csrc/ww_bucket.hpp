// ww_bucket.hpp -- the deep sieve's large primes, marked once per launch
// (ww_bucket.cu).
#pragma once

#include <cuda_runtime.h>

#include "ww_deep.cuh"

namespace ww {

// Deepest table: primes below 2^30 (the rows keep r in 32 bits).
constexpr int kDeepLargeMaxBits = 30;

// One large deep prime: r, o = ord_r(2) and floor(2^64 / o).  The other
// constants of its start (r^-1 mod 2^64, floor(2^64 / r)) are recomputed at
// every launch: 16 bytes a row instead of 32 keep the table's stream from
// evicting the mark bitmap from L2.  floor(2^64 / o) stays in the row: for
// small orders (o = 37 for r = 616318177, a factor of 2^37 - 1) the quotient
// is beyond a double-precision estimate's reach.
struct __align__(16) DeepPrime {
    u32 r, o;
    u64 mo;
};

// Rows of the primes 2^WW_DEEP_BITS < r < 2^bits on one device, in
// ascending order.
struct DeepLarge {
    const DeepPrime *rows;
    u32 n;
};

// The table for `bits` on the current device, built on first use (a host
// sieve and one kernel; cached until the process exits).
int deep_large_device(int bits, DeepLarge *out);

// Rows first .. first+n-1 of the table of `bits` on the current device
// (r and ord_r(2)), and the table's length, for checking the table.
int read_deep_large(int bits, uint64_t first, uint64_t n, uint32_t *r, uint32_t *o, uint64_t *total);

// Zero bits[0, nwords) and mark, for the odd numbers first + 2j (j < nodd),
// the multiples of the table's primes that the cofactor rule marks.
int launch_deep_fill(u64 first, u64 nodd, const DeepLarge &t, u32 *bits, u64 nwords, cudaStream_t stream);

}  // namespace ww
