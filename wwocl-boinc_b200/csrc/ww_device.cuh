// ww_device.cuh -- device helpers shared by the kernels of the WWocl search
// path on sm_100a (the kernels themselves are in ww_kernels.cuh and
// ww_batch.cuh).

#pragma once

#include <cuda_runtime.h>

#include "ww_deep.cuh"
#include "ww_tests.cuh"

namespace ww {

// A warp queue holds the < 32 candidates carried over plus one chunk of 32
// words (1024 odd numbers).  Among any 1024 consecutive odd numbers at most
// 378 have no factor 3..17 (the maximum over the full period 3*5*...*17), so
// 31 + 378 entries always suffice.
constexpr int kQueueCap = 416;

// A segment shape of k_sieve_prp: W bitmap words (32 W odd numbers) for T
// threads; its dynamic shared memory is the bitmap, then one queue per warp.
template <int W, int T>
struct SieveGeom {
    static constexpr int kWords = W;
    static constexpr int kThreads = T;
    static constexpr int kOdd = W * 32;
    static constexpr int kWarps = T / 32;
    static constexpr int kWordsPerThread = W / T;
    static constexpr size_t kSmem = (size_t)W * 4 + (size_t)(T / 32) * kQueueCap * 4;
    static_assert(W % T == 0 && W % 32 == 0 && T % 32 == 0, "sieve geometry");
};
// 2^20 numbers per segment for 512 threads, two CTAs and 32 warps per SM.
// Each doubling of the segment halves the deep primes' per-segment start-up
// work: on 4e9 numbers below 2^64 in one launch, 2^19 numbers for 256
// threads took 29.0 ms, 2^20 for 512 threads 28.6 ms, 2^21 for 1024
// threads 28.1 ms.  But a 2^30-number launch (the checkpoint cadence) has
// only 512 segments of 2^21 for 148 one-CTA SMs, and the plain range
// pipeline fell from 775 M to 754 M primes/s with them.
#ifndef WW_SIEVE_WIDE_WORDS
#define WW_SIEVE_WIDE_WORDS 16384
#define WW_SIEVE_WIDE_THREADS 512
#endif
typedef SieveGeom<WW_SIEVE_WIDE_WORDS, WW_SIEVE_WIDE_THREADS> SieveWide;
// 2^19 numbers for 256 threads: twice the segments, for ranges that would
// not give every resident CTA of the wide shape a segment.
typedef SieveGeom<8192, 256> SieveNarrow;

#ifndef WW_TEST_THREADS
#define WW_TEST_THREADS 256
#endif
constexpr int kTestThreads = WW_TEST_THREADS;
#ifndef WW_TEST_MINB
#define WW_TEST_MINB 1  // minimum resident CTAs per SM asked of the test kernels
#endif

struct HitOut {
    u64 *prime;
    int *rem, *quot, *result;
    u32 *count;
    u32 capacity;
    u32 *overflow;
};

__device__ __forceinline__ void emit_hit(const HitOut &h, u64 p, int result, int rem, int quot) {
    const u32 ix = atomicAdd(h.count, 1u);
    if (ix < h.capacity) {
        h.prime[ix] = p;
        h.result[ix] = result;
        h.rem[ix] = rem;
        h.quot[ix] = quot;
    } else {
        atomicOr(h.overflow, 2u);
    }
}

__device__ __forceinline__ u64 warp_sum(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------ sieve

// Composite mask of one prime r for a word whose first bit is at j0 (bit j
// of the word is the odd number n_w + 2j; r divides n_w + 2 j0).
template <u32 R>
__device__ __forceinline__ u32 prime_mask(u32 j0) {
    if (R < 32) {
        u32 pat = 0;
#pragma unroll
        for (u32 k = 0; k < 32; k += R) pat |= 1u << k;
        return pat << j0;
    }
    return j0 < 32 ? (1u << (j0 & 31)) : 0u;
}

template <u32 R>
__device__ __forceinline__ u32 first_hit(u64 n) {
    // smallest j >= 0 with R | n + 2j
    const u32 res = (u32)(n % R);
    const u32 inv2 = (R + 1) / 2;
    return ((R - res) % R) * inv2 % R;
}

template <u32 R>
__device__ __forceinline__ void step_hit(u32 &j0) {
    // next word: the index moves down by 32 (mod R)
    const u32 d = 32 % R;
    j0 = (j0 >= d) ? j0 - d : j0 + R - d;
}

#define WW_FOR_SMALL_PRIMES(X) \
    X(3) X(5) X(7) X(11) X(13) X(17) X(19) X(23) X(29) X(31) X(37) X(41) X(43) X(47) X(53) \
    X(59) X(61) X(67) X(71) X(73) X(79) X(83) X(89) X(97) X(101) X(103) X(107) X(109) X(113)

// ------------------------------------------------------------- deep sieve
// (the scheme is described in ww_deep.cuh)

// The deep-sieve table lives once in device memory (ww_capi.cu); kernels
// get its address as an argument.  Host code asks for it per device.
const DeepRow *deep_rows_device();

// Mark the odd multiples n = r*k of the deep primes in the segment, except
// those with k = 1 (mod ord_r(2)) (ww_deep.cuh says why).  The smallest
// primes have the most multiples: each of the first kDeepWarpPrimes primes
// is marked by a whole warp (lane l takes the multiples l, l + 32, ...; k
// then grows by 64 per step), the rest one prime per thread, so no thread
// holds the others at the next barrier.
constexpr int kDeepWarpPrimes = 512;

__device__ __forceinline__ void deep_mark(u64 first, u32 nvalid, u32 *bitmap, int tid, int nthreads,
                                          const DeepRow *__restrict__ deep) {
    const int lane = tid & 31, warp = tid >> 5, nwarps = nthreads >> 5;
    for (int i = warp; i < kDeepWarpPrimes && i < kDeepUse; i += nwarps) {
        const DeepRow e = deep[i];
        u32 j0, km0;
        deep_start(first, e, j0, km0);
        u32 km = (km0 + 2u * (u32)lane) % e.o;
        const u32 step = 64u % e.o;
        for (u32 j = j0 + (u32)lane * e.r; j < nvalid; j += 32u * e.r) {
            if (km != 1u) atomicOr(&bitmap[j >> 5], 1u << (j & 31));
            km += step;
            if (km >= e.o) km -= e.o;
        }
    }
    for (int i = kDeepWarpPrimes + tid; i < kDeepUse; i += nthreads) {
        const DeepRow e = deep[i];
        u32 j, km;
        deep_start(first, e, j, km);
        for (; j < nvalid; j += e.r) {
            if (km != 1u) atomicOr(&bitmap[j >> 5], 1u << (j & 31));
            km += 2u;
            if (km >= e.o) km -= e.o;
        }
    }
}

struct PrpOut {
    u64 *prime, *inv;
    u32 *count;
    u64 capacity;
    u32 *overflow;
};

__device__ __forceinline__ void sprp_emit(const PrpOut &out, u64 n, bool active) {
    u64 q = 0;
    const bool pass = prp_test_warp(n, active, q);
    const u32 ballot = __ballot_sync(0xffffffffu, pass);
    if (ballot == 0) return;
    const int lane = threadIdx.x & 31;
    u32 base = 0;
    if (lane == 0) base = atomicAdd(out.count, (u32)__popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (pass && out.prime) {  // no list: count only
        const u64 ix = (u64)base + (u64)__popc(ballot & ((1u << lane) - 1u));
        if (ix < out.capacity) {
            out.prime[ix] = n;
            out.inv[ix] = q;
        } else {
            atomicOr(out.overflow, 1u);
        }
    }
}

}  // namespace ww
