// ww_kernels.cuh -- kernels of the WWocl search path on sm_100a.
//
//   k_sieve_prp   getsegprimes (getsegprimes.cl:228-301): a CTA sieves one
//                 segment of 2*G::kOdd integers at a time (taken from a cursor,
//                 or by grid stride).  The odd numbers of the segment form a
//                 shared-memory bitmap; each thread ORs the composite patterns
//                 of 3..113 into its words (the reference's 27 constant tables,
//                 getsegprimes.cl:169-225, become per-prime bit offsets kept
//                 incrementally), the deep sieve marks the multiples of the
//                 primes up to 2^WW_DEEP_BITS that cannot be pseudoprimes
//                 (ww_deep.cuh), then each warp compacts the survivors with
//                 ballot/popc into a warp queue and runs the base-2 strong
//                 PRP test 32 candidates at a time, one atomic per warp for the
//                 output slots.
//   k_wieferich / k_wallsunsun   the two reference test kernels.
//   k_test_prps   both tests in one pass over the PRP list (warps pull work
//                 from a cursor, or stride).
//   k_digits      per-prime canonical digits (verification only).
#pragma once

#include "ww_device.cuh"

namespace ww {

// Threads per SM the sieve's launch bounds ask for: 1024 holds it to 64
// registers (2 CTAs of 512, or 4 of 256, per SM).  Uncapped it takes 128;
// at 512 or 768 (1 CTA of 512 per SM, 128 registers) the sieve measured
// 7.19 against 5.90 ms per 2^30 numbers on a B200.
#ifndef WW_SIEVE_MINB_THREADS
#define WW_SIEVE_MINB_THREADS 1024
#endif

// Sieve + SPRP over [lo, hi) in segments of shape G (SieveGeom).  b0 = lo & ~1;
// segment s holds the odd numbers b0 + 2(s*G::kOdd + j) + 1, j < G::kOdd.
// With a segment cursor (zeroed before the launch) the CTAs take segments
// one at a time from it; without one (a launch captured into a graph, or
// one that found every cursor of the library's pool busy) they stride over
// the segments.  marks (optional): the large deep primes' marks of the whole
// launch, bit j of word w = odd number b0 + 2(32 w + j) + 1 (ww_bucket.cu),
// ORed into each segment's bitmap.
template <class G>
__global__ void __launch_bounds__(G::kThreads, WW_SIEVE_MINB_THREADS / G::kThreads) k_sieve_prp(u64 lo, u64 hi, u64 nseg, PrpOut out,
                                                                              u64 *cursor, const DeepRow *deep,
                                                                              const u32 *__restrict__ marks) {
    extern __shared__ u32 sieve_smem[];  // G::kSmem bytes
    u32 *bitmap = sieve_smem;
    u32(*queue)[kQueueCap] = reinterpret_cast<u32(*)[kQueueCap]>(sieve_smem + G::kWords);
    __shared__ u32 s_chunk;
    __shared__ u64 s_seg;
    const u64 b0 = lo & ~1ull;
    const u64 span = hi - b0;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;

    u64 seg = blockIdx.x;
    if (cursor) {
        if (threadIdx.x == 0) s_seg = atomicAdd((unsigned long long *)cursor, 1ull);
        __syncthreads();
        seg = s_seg;
    }
    while (seg < nseg) {
        const u64 seg_off = seg * (u64)(2 * G::kOdd);
        const u64 rem_span = span - seg_off;  // > 0
        const u64 nvalid = (rem_span / 2 < (u64)G::kOdd) ? rem_span / 2 : (u64)G::kOdd;

        // ---- pre-sieve 3..113 on this thread's contiguous words
        {
            const int w0 = threadIdx.x * G::kWordsPerThread;
            const u64 n0 = b0 + seg_off + 64ull * (u64)w0 + 1;  // may wrap past 2^64 beyond hi
            const u32 *seg_marks = marks ? marks + seg * (u64)G::kWords : nullptr;
#define WW_J0(R) u32 j##R = first_hit<R>(n0);
            WW_FOR_SMALL_PRIMES(WW_J0)
#undef WW_J0
#pragma unroll 4
            for (int w = w0; w < w0 + G::kWordsPerThread; ++w) {
                u32 m = seg_marks ? seg_marks[w] : 0u;
#define WW_MASK(R) m |= prime_mask<R>(j##R); step_hit<R>(j##R);
                WW_FOR_SMALL_PRIMES(WW_MASK)
#undef WW_MASK
                // bits past the end of the range are not candidates
                const u64 first = (u64)w * 32;
                if (first + 32 > nvalid) {
                    const u64 keep = nvalid > first ? nvalid - first : 0;  // < 32
                    m |= ~((1u << keep) - 1u);
                }
                bitmap[w] = m;
            }
        }
        if (threadIdx.x == 0) s_chunk = 0;
        __syncthreads();

        // ---- deep sieve 113 < r < 2^WW_DEEP_BITS, sparing possible pseudoprimes
        const u64 nbase = b0 + seg_off + 1;
        deep_mark(nbase, (u32)nvalid, bitmap, threadIdx.x, G::kThreads, deep);
        __syncthreads();

        // ---- warps take 32-word chunks dynamically (so they reach the next
        // barrier together), compact the survivors with ballot/popc into a
        // warp queue and PRP-test them 32 at a time
        u32 *q = queue[warp];
        int qn = 0;
        for (;;) {
            u32 chunk = 0;
            if (lane == 0) chunk = atomicAdd(&s_chunk, 1u);
            chunk = __shfl_sync(0xffffffffu, chunk, 0);
            const bool more = chunk < (u32)(G::kWords / 32);
            if (more) {
                const int w = chunk * 32 + lane;
                u32 cand = ~bitmap[w];
                const int cnt = __popc(cand);
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                int pos = qn + incl - cnt;
                while (cand) {
                    const int b = __ffs(cand) - 1;
                    q[pos++] = (u32)(w * 32 + b);
                    cand &= cand - 1;
                }
                qn += total;
                __syncwarp();
            }
            while (qn >= 32 || (!more && qn > 0)) {
                const int take = qn >= 32 ? 32 : qn;
                qn -= take;
                const bool act = lane < take;
                const u32 j = act ? q[qn + lane] : 0u;
                __syncwarp();
                sprp_emit(out, nbase + 2ull * j, act);
            }
            if (!more) break;
        }
        __syncthreads();  // bitmap reused by the next segment
        if (cursor) {
            if (threadIdx.x == 0) s_seg = atomicAdd((unsigned long long *)cursor, 1ull);
            __syncthreads();
            seg = s_seg;
        } else {
            seg += gridDim.x;
        }
    }
}

// ------------------------------------------------------------------ tests

__device__ __forceinline__ void count_update(u32 *primecount, u64 *totalprimecount) {
    // wieferich.cl:317-326: accumulate the launch's PRP count, keep the max
    const u32 pc = primecount[0];
    *totalprimecount += pc;
    if (pc > primecount[1]) primecount[1] = pc;
}

// Primes a warp takes per fetch from the work cursor: one per lane, so a
// short list still spreads over every warp and the last fetch of a launch
// is one prime per lane.
constexpr u64 kWarpFetch = 32;

// Runs f(i) for every list index i < n.  With a work cursor (zeroed before
// the launch) each warp pulls kWarpFetch indices at a time, so warps that run
// ahead take more of the list and all finish together; without one (a
// launch captured into a graph, or one that found every cursor of the
// library's pool busy) the grid strides.
template <class F>
__device__ __forceinline__ void for_each_prime(u64 n, u64 *cursor, F &&f) {
    if (cursor) {
        const int lane = threadIdx.x & 31;
        for (;;) {
            u64 base = 0;
            if (lane == 0) base = atomicAdd((unsigned long long *)cursor, (unsigned long long)kWarpFetch);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= n) break;
            const u64 end = min(base + kWarpFetch, n);
            for (u64 i = base + lane; i < end; i += 32) f(i);
        }
    } else {
        for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) f(i);
    }
}

__global__ void __launch_bounds__(kTestThreads, WW_TEST_MINB) k_wieferich(u32 *primecount, const u64 *prime,
                                                             const u64 *inv, u64 *g_one, HitOut hits,
                                                             u64 *checksum, u64 *totalprimecount,
                                                             u64 capacity, u64 *cursor) {
    const u64 n = min((u64)primecount[0], capacity);
    u64 sum = 0;
    for_each_prime(n, cursor, [&](u64 i) {
        const u64 p = prime[i];
        const u64 q = inv ? inv[i] : inv64(p);
        const D2 one = m2_one(p);
        if (g_one) {
            g_one[2 * i] = one.d0;
            g_one[2 * i + 1] = one.d1;
        }
        const D2 s = wieferich_digits(p, q, one);
        sum += s.d1 & 0xffffffffull;
        int rem, quot;
        if (wieferich_classify(p, s, rem, quot)) emit_hit(hits, p, 1093, rem, quot);
    });
    sum = warp_sum(sum);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(checksum, sum);
    if (blockIdx.x == 0 && threadIdx.x == 0) count_update(primecount, totalprimecount);
}

__global__ void __launch_bounds__(kTestThreads, WW_TEST_MINB) k_wallsunsun(const u32 *primecount, const u64 *prime,
                                                              const u64 *inv, const u64 *g_one,
                                                              HitOut hits, u64 *checksum, u64 capacity,
                                                              u64 *cursor) {
    const u64 n = min((u64)primecount[0], capacity);
    u64 sum = 0;
    for_each_prime(n, cursor, [&](u64 i) {
        const u64 p = prime[i];
        const u64 q = inv ? inv[i] : inv64(p);
        D2 one;
        if (g_one) {
            one.d0 = g_one[2 * i];
            one.d1 = g_one[2 * i + 1];
        } else {
            one = m2_one(p);
        }
        const D2 c = wss_digits(p, q, one);
        sum += c.d1 & 0xffffffffull;
        int res, quot;
        if (wss_classify(p, c, res, quot)) emit_hit(hits, p, res, 0, quot);
    });
    sum = warp_sum(sum);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(checksum, sum);
}

// Both tests over the list in one pass.
__global__ void __launch_bounds__(kTestThreads, WW_TEST_MINB) k_test_prps(u32 *primecount, const u64 *prime,
                                                             const u64 *inv, HitOut hits, u64 *checksum,
                                                             u64 *totalprimecount, u64 capacity,
                                                             u64 *cursor) {
    const u64 n = min((u64)primecount[0], capacity);
    u64 sum = 0;
    for_each_prime(n, cursor, [&](u64 i) {
        const u64 p = prime[i];
        const u64 q = inv ? inv[i] : inv64(p);
        const D2 one = m2_one(p);
        D2 s, c;
        both_digits(p, q, one, s, c);
        sum += (s.d1 & 0xffffffffull) + (c.d1 & 0xffffffffull);
        int rem, quot, res;
        if (wieferich_classify(p, s, rem, quot)) emit_hit(hits, p, 1093, rem, quot);
        if (wss_classify(p, c, res, quot)) emit_hit(hits, p, res, 0, quot);
    });
    sum = warp_sum(sum);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(checksum, sum);
    if (blockIdx.x == 0 && threadIdx.x == 0) count_update(primecount, totalprimecount);
}

__global__ void k_digits(const u64 *primes, u64 n, u64 *out) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 p = primes[i];
        const u64 q = inv64(p);
        const D2 one = m2_one(p);
        D2 s, c;
        both_digits(p, q, one, s, c);
        out[4 * i] = s.d0;
        out[4 * i + 1] = s.d1;
        out[4 * i + 2] = c.d0;
        out[4 * i + 3] = c.d1;
    }
}

// q = p^-1 mod 2^64 for a loaded list; sets the segment count.
__global__ void k_fill_inverse(const u64 *prime, u64 *inv, u64 n) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        inv[i] = inv64(prime[i]);
}

}  // namespace ww
