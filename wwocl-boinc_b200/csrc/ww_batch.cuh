// ww_batch.cuh -- the tile engine of the batched search and of the request
// server: many ranges of uneven width in one persistent launch that pulls
// (range, segment) tiles from a device queue.
//
// One CTA takes one tile at a time (an atomic on the tile counter), sieves
// it in a shared-memory bitmap, and runs the whole path on it without a PRP
// list in global memory: warps take 32-word chunks of the bitmap from a
// shared counter (so the warps of a CTA finish a tile together), compact
// the survivors into a warp queue, run the base-2 strong PRP test 32 at a
// time, and push the PRPs into a second warp queue that feeds the
// Wieferich and Wall-Sun-Sun tests 32 (or 64 with two primes per thread) at
// a time.  Checksums and PRP counts go to the tile's unit with one atomic
// per warp per batch; the sums are order-free, so every unit's checksum is
// bit-identical to a run of that unit alone.
#pragma once

#include "ww_device.cuh"

namespace ww {

// Device state of one range (a unit of a batch or a served request).
struct UnitState {
    u64 start, end;          // [start, end), start >= 127 unless empty
    u64 n_tiles;             // ceil((end - start) / tile)
    u64 next_tile;           // sieve cursor: next tile to hand out (serving)
    u64 checksum;            // sum of both checksum terms
    u64 prp_count;           // PRPs tested
    u64 *prp_out;            // optional PRP buffer of the range (nullptr: none)
    u64 prp_cap;
    u64 prp_written;         // PRPs found (may exceed prp_cap: overflow)
    u32 hits, tiles_done;
    u32 active, pad;
};

struct BatchArgs {
    UnitState *units;
    u32 n_units;
    // static tile table (batch): tile_first[k] = first tile of unit k, n_units + 1 entries
    const u64 *tile_first;
    u64 n_tiles;
    u64 *next_tile;          // queue head
    // serving: at most `budget` tiles this launch, handed out in the order of
    // `order` (slot indices, earliest deadline first; n_order entries)
    u32 *epoch_tiles;
    u32 budget;
    const u32 *order;
    u32 n_order;
    // hits: p, result, rem, quot, unit
    u64 *hit_p;
    int *hit_result, *hit_rem, *hit_quot;
    u32 *hit_unit;
    u32 *hit_count;
    u32 hit_capacity;
    u32 *overflow;           // bit 1: hit list overflow, bit 0: a PRP buffer overflowed
    const DeepRow *deep;     // the deep-sieve table (deep_rows_device())
};

// A tile configuration: SEG_WORDS bitmap words, THREADS per CTA, PPT batches
// of 32 PRPs a warp collects before testing them, and JOINT = 1 for the
// Wieferich and WSS tests of a prime in one loop (the list kernel's form)
// instead of one after the other.
template <int SEG_WORDS, int THREADS, int PPT, int JOINT = 0>
struct BatchCfg {
    static constexpr int kWords = SEG_WORDS;
    static constexpr int kThreads = THREADS;
    static constexpr int kWarps = THREADS / 32;
    static constexpr int kPpt = PPT;
    static constexpr bool kJoint = JOINT != 0;
    // resident threads per SM the registers must allow: 1024 (64 registers,
    // 32 warps) with one or two batches of PRPs per warp -- left to the
    // compiler, the 512-thread tiles took 128 registers (16 warps per SM)
    // and ran 7 % slower; four or eight batches keep the compiler's choice
    // (142 and 146 registers at 256 threads), which measured faster than
    // 78 and 80 registers at three CTAs per SM (they spill 128 and 256 bytes
    // at 64)
    static constexpr int kSmThreads = PPT >= 4 ? THREADS : 1024;
    static constexpr int kMinBlocks = kSmThreads / THREADS > 0 ? kSmThreads / THREADS : 1;
    static constexpr int kChunks = SEG_WORDS / 32;
    static constexpr u64 kTileNumbers = 64ull * SEG_WORDS;  // integers per tile
    static constexpr int kCandCap = 416;  // as kQueueCap: 31 carried + at most 378 per 32-word chunk
    static constexpr int kPrpCap = 32 * PPT + 32;
    static_assert(SEG_WORDS % THREADS == 0, "words per thread");
};

struct WarpAcc {
    u64 checksum;
    u32 count;
};

__device__ __forceinline__ void emit_batch_hit(const BatchArgs &a, u32 unit, u64 p, int result, int rem, int quot) {
    const u32 ix = atomicAdd(a.hit_count, 1u);
    if (ix < a.hit_capacity) {
        a.hit_p[ix] = p;
        a.hit_result[ix] = result;
        a.hit_rem[ix] = rem;
        a.hit_quot[ix] = quot;
        a.hit_unit[ix] = unit;
    } else {
        atomicOr(a.overflow, 2u);
    }
    atomicAdd(&a.units[unit].hits, 1u);
}

// Wieferich + WSS on the warp's PRP queue entries [base, base + 32*PPT);
// `valid` lanes only.  Adds to the warp's accumulator (lane 0 holds it).
template <int PPT, bool JOINT>
__device__ __forceinline__ void test_batch(const u64 *qp, int n_valid, u32 unit, const BatchArgs &a,
                                           WarpAcc &acc) {
    const int lane = threadIdx.x & 31;
    u64 sum = 0;
    u32 cnt = 0;
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int idx = k * 32 + lane;
        const bool act = idx < n_valid;
        const u64 p = act ? qp[idx] : 0xFFFFFFFFFFFFFFC5ull;  // 2^64-59, a harmless prime
        const u64 q = inv64(p);
        const D2 one = m2_one(p);
        // one after the other: fewer registers live at once, so the
        // 512-thread tiles fit 64 registers (two CTAs, 32 warps per SM);
        // the joint loop has three independent squarings per step
        D2 s, c;
        if (JOINT) {
            both_digits(p, q, one, s, c);
        } else {
            s = wieferich_digits(p, q, one);
            c = wss_digits(p, q, one);
        }
        if (act) {
            sum += (s.d1 & 0xffffffffull) + (c.d1 & 0xffffffffull);
            ++cnt;
            int rem, quot_w, res, quot_s;
            const bool hw = wieferich_classify(p, s, rem, quot_w);
            const bool hs = wss_classify(p, c, res, quot_s);
            if (hw) emit_batch_hit(a, unit, p, 1093, rem, quot_w);  // as the wieferich kernel would
            if (hs) emit_batch_hit(a, unit, p, res, 0, quot_s);     // as the wallsunsun kernel would
        }
    }
    sum = warp_sum(sum);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if (lane == 0) {
        acc.checksum += sum;
        acc.count += cnt;
    }
}

template <class Cfg>
constexpr size_t batch_smem_bytes() {
    return (size_t)Cfg::kWarps * Cfg::kPrpCap * 8 + (size_t)Cfg::kWords * 4 +
           (size_t)Cfg::kWarps * Cfg::kCandCap * 4;
}

// Hand out the next tile.  Batch: the global queue head over the static
// tile table.  Serving: the first unit in the host's priority order that
// has tiles left, through that unit's own cursor, at most `budget` tiles per
// launch; the loop is bounded by the number of units, so an exhausted queue
// ends the kernel instead of spinning.
template <bool SERVE>
__device__ __forceinline__ bool next_tile(const BatchArgs &a, u32 &unit, u64 &tile) {
    if (!SERVE) {
        const u64 t = atomicAdd((unsigned long long *)a.next_tile, 1ull);
        if (t >= a.n_tiles) return false;
        u32 lo = 0, hi = a.n_units;  // last k with tile_first[k] <= t
        while (hi - lo > 1) {
            const u32 mid = (lo + hi) >> 1;
            if (a.tile_first[mid] <= t) lo = mid; else hi = mid;
        }
        unit = lo;
        tile = t - a.tile_first[lo];
        return true;
    }
    if (atomicAdd(a.epoch_tiles, 1u) >= a.budget) return false;
    for (u32 i = 0; i < a.n_order; ++i) {
        const u32 k = a.order[i];
        UnitState &u = a.units[k];
        // the cursor is read past L1 (other CTAs move it); a stale value
        // only costs an atomic that finds the unit exhausted
        if (!u.active || *(volatile u64 *)&u.next_tile >= u.n_tiles) continue;
        const u64 t = atomicAdd((unsigned long long *)&u.next_tile, 1ull);
        if (t < u.n_tiles) {
            unit = k;
            tile = t;
            return true;
        }
    }
    return false;
}

template <class Cfg, bool SERVE>
__global__ void __launch_bounds__(Cfg::kThreads, Cfg::kMinBlocks) k_tiles(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    u64(*prpq)[Cfg::kPrpCap] = reinterpret_cast<u64(*)[Cfg::kPrpCap]>(smem);
    u32 *bitmap = reinterpret_cast<u32 *>(smem + (size_t)Cfg::kWarps * Cfg::kPrpCap * 8);
    u32(*candq)[Cfg::kCandCap] =
        reinterpret_cast<u32(*)[Cfg::kCandCap]>(smem + (size_t)Cfg::kWarps * Cfg::kPrpCap * 8 + Cfg::kWords * 4);
    __shared__ u64 s_lo, s_hi;
    __shared__ u32 s_unit, s_chunk, s_ok;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;

    for (;;) {
        if (threadIdx.x == 0) {
            u32 k = 0;
            u64 t = 0;
            s_chunk = 0;
            s_ok = next_tile<SERVE>(a, k, t) ? 1u : 0u;
            if (s_ok) {
                const UnitState &u = a.units[k];
                const u64 tlo = u.start + t * Cfg::kTileNumbers;
                const u64 room = u.end - tlo;
                s_unit = k;
                s_lo = tlo;
                s_hi = room > Cfg::kTileNumbers ? tlo + Cfg::kTileNumbers : u.end;
            }
        }
        __syncthreads();
        if (!s_ok) return;
        const u64 lo = s_lo, hi = s_hi;
        const u32 unit = s_unit;

        // ---- pre-sieve 3..113 over [lo, hi): bit j of the tile is b0 + 2j + 1
        const u64 b0 = lo & ~1ull;
        const u64 span = hi - b0;
        const u64 nvalid = span / 2 < (u64)(Cfg::kWords * 32) ? span / 2 : (u64)(Cfg::kWords * 32);
        {
            constexpr int kWpt = Cfg::kWords / Cfg::kThreads;
            const int w0 = threadIdx.x * kWpt;
            const u64 n0 = b0 + 64ull * (u64)w0 + 1;
#define WW_J0(R) u32 j##R = first_hit<R>(n0);
            WW_FOR_SMALL_PRIMES(WW_J0)
#undef WW_J0
#pragma unroll 2
            for (int w = w0; w < w0 + kWpt; ++w) {
                u32 m = 0;
#define WW_MASK(R) m |= prime_mask<R>(j##R); step_hit<R>(j##R);
                WW_FOR_SMALL_PRIMES(WW_MASK)
#undef WW_MASK
                const u64 first = (u64)w * 32;
                if (first + 32 > nvalid) {
                    const u64 keep = nvalid > first ? nvalid - first : 0;
                    m |= ~((1u << keep) - 1u);
                }
                bitmap[w] = m;
            }
        }
        __syncthreads();

        // ---- deep sieve 113 < r < 2^WW_DEEP_BITS, sparing possible pseudoprimes
        const u64 nbase = b0 + 1;
        deep_mark(nbase, (u32)nvalid, bitmap, threadIdx.x, Cfg::kThreads, a.deep);
        __syncthreads();

        // ---- chunks of 32 words, taken dynamically by the warps
        u32 *cq = candq[warp];
        u64 *pq = prpq[warp];
        int cn = 0, pn = 0;
        WarpAcc acc = {0, 0};
        // one PRP test per lane; passing numbers go to the warp's PRP queue,
        // which feeds the Wieferich + WSS batches
        auto sprp_step = [&](u32 j, bool act) {
            const u64 n = nbase + 2ull * j;
            u64 q = 0;
            const bool pass = prp_test_warp(n, act, q);
            const u32 ballot = __ballot_sync(0xffffffffu, pass);
            const u32 rank = __popc(ballot & ((1u << lane) - 1u));
            if (pass) pq[pn + rank] = n;
            if (a.units[unit].prp_out && ballot) {  // the range's PRP buffer (serving)
                u64 base = 0;
                if (lane == 0)
                    base = atomicAdd((unsigned long long *)&a.units[unit].prp_written,
                                     (unsigned long long)__popc(ballot));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (pass) {
                    if (base + rank < a.units[unit].prp_cap) a.units[unit].prp_out[base + rank] = n;
                    else atomicOr(a.overflow, 1u);
                }
            }
            pn += __popc(ballot);
            __syncwarp();
            while (pn >= 32 * Cfg::kPpt) {
                pn -= 32 * Cfg::kPpt;
                test_batch<Cfg::kPpt, Cfg::kJoint>(pq + pn, 32 * Cfg::kPpt, unit, a, acc);
                __syncwarp();
            }
        };
        for (;;) {
            u32 chunk = 0;
            if (lane == 0) chunk = atomicAdd(&s_chunk, 1u);
            chunk = __shfl_sync(0xffffffffu, chunk, 0);
            const bool more = chunk < (u32)Cfg::kChunks;
            if (more) {
                const int w = chunk * 32 + lane;
                u32 cand = ~bitmap[w];
                const int c = __popc(cand);
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                int pos = cn + incl - c;
                while (cand) {
                    const int b = __ffs(cand) - 1;
                    cq[pos++] = (u32)(w * 32 + b);
                    cand &= cand - 1;
                }
                cn += total;
                __syncwarp();
            }
            // SPRP 32 candidates at a time; the last partial batch once the bitmap is done
            while (cn >= 32 || (!more && cn > 0)) {
                const int take = cn >= 32 ? 32 : cn;
                cn -= take;
                const bool act = lane < take;
                const u32 j = act ? cq[cn + lane] : 0u;
                __syncwarp();
                sprp_step(j, act);
            }
            if (!more) break;
        }
        if (pn > 0) {
            test_batch<Cfg::kPpt, Cfg::kJoint>(pq, pn, unit, a, acc);
            pn = 0;
        }
        if (lane == 0 && acc.count) {
            atomicAdd((unsigned long long *)&a.units[unit].checksum, (unsigned long long)acc.checksum);
            atomicAdd((unsigned long long *)&a.units[unit].prp_count, (unsigned long long)acc.count);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&a.units[unit].tiles_done, 1u);
        }
    }
}

}  // namespace ww
