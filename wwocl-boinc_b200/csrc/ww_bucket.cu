// ww_bucket.cu -- the deep sieve's large primes, marked once per launch.
//
// The sieve kernel marks the multiples of the deep primes below 2^WW_DEEP_BITS
// segment by segment: each prime's start in a segment costs two Barrett
// reductions, which pays only while the prime has several multiples per
// segment.  The primes 2^WW_DEEP_BITS < r < 2^B have one multiple per
// segment or fewer, so here one thread per prime starts once per launch and
// walks its odd multiples over the whole launch, setting a bit in a global
// bitmap of the launch's odd numbers (one atomic OR each); the sieve kernel
// then ORs its segment's words of that bitmap into its shared-memory bitmap.
// The cofactor rule is the one of ww_deep.cuh: a multiple n = r*k is marked
// only when k != 1 (mod ord_r(2)), so every possible base-2 pseudoprime --
// and r itself -- stays a candidate and the PRP set does not change.
//
// The table of large primes (r, ord_r(2) and floor(2^64 / ord_r(2))) is
// built once per device and depth: the primes come from a segmented sieve on
// the host, the orders from a kernel that factors r - 1 by trial division.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/wwcuda.h"
#include "ww_bucket.hpp"
#include "ww_device.cuh"

namespace ww {
void set_err(const char *fmt, ...);  // ww_capi.cu
}

using namespace ww;

namespace {

// Odd primes below 2^15: enough to factor any r - 1 < 2^30.
std::vector<u32> small_odd_primes() {
    std::vector<u32> out;
    std::vector<uint8_t> comp(1u << 15, 0);
    for (u32 i = 3; i < (1u << 15); i += 2) {
        if (comp[i]) continue;
        out.push_back(i);
        for (u32 j = i * i; j < (1u << 15); j += 2 * i) comp[j] = 1;
    }
    return out;
}

// Primes lo <= r < hi (lo odd, hi <= 2^30) by a segmented odd-only sieve.
std::vector<u32> primes_between(u32 lo, u32 hi, const std::vector<u32> &small) {
    std::vector<u32> out;
    constexpr u32 kSeg = 1u << 22;  // odd numbers per piece
    std::vector<uint8_t> comp(kSeg);
    for (u64 a = lo; a < hi; a += 2ull * kSeg) {
        const u64 b = a + 2ull * kSeg < hi ? a + 2ull * kSeg : hi;  // odd numbers a, a+2, ... < b
        const u64 n = (b - a + 1) / 2;
        std::fill(comp.begin(), comp.begin() + n, 0);
        for (u32 p : small) {
            const u64 pp = (u64)p * p;
            if (pp >= b) break;
            u64 m = pp >= a ? pp : ((a + p - 1) / p) * p;
            if (!(m & 1)) m += p;  // odd multiples only
            for (; m < b; m += 2ull * p) comp[(m - a) / 2] = 1;
        }
        for (u64 i = 0; i < n; ++i)
            if (!comp[i]) out.push_back((u32)(a + 2 * i));
    }
    return out;
}

__device__ u32 pow2_mod(u32 e, u32 r) {  // 2^e mod r for e >= 1, r < 2^30
    u64 x = 1;
    for (int i = 31 - __clz(e); i >= 0; --i) {
        x = (x * x) % r;
        if ((e >> i) & 1) x = (2 * x) % r;
    }
    return (u32)x;
}

// One table row per prime: o = ord_r(2) from the prime factors of r - 1
// (trial division by the odd primes below 2^15; r - 1 < 2^30 has at most
// nine distinct prime factors).
__global__ void k_deep_orders(const u32 *primes, u32 n, const u32 *small, u32 nsmall, DeepPrime *rows) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 r = primes[i];
    u32 fac[10];
    int nf = 0;
    fac[nf++] = 2;
    u32 m = (r - 1) >> (__ffs((int)(r - 1)) - 1);
    for (u32 k = 0; k < nsmall; ++k) {
        const u32 q = small[k];
        if (q * q > m) break;
        if (m % q == 0) {
            fac[nf++] = q;
            do m /= q;
            while (m % q == 0);
        }
    }
    if (m > 1) fac[nf++] = m;
    u32 o = r - 1;
    for (int f = 0; f < nf; ++f)
        while (o % fac[f] == 0 && pow2_mod(o / fac[f], r) == 1) o /= fac[f];
    // floor(2^64 / o), exact (a power of two divides 2^64)
    rows[i] = DeepPrime{r, o, (o & (o - 1)) ? ~0ull / o : (1ull << (65 - __ffs((int)o)))};
}

// floor(2^64 / d) for odd 2^11 < d < 2^32: the quotient is below 2^53, so a
// double-precision estimate is within one of it, and one exact correction
// finishes.
__device__ __forceinline__ u64 floor_2p64_div(u64 d) {
    u64 q = (u64)(18446744073709551616.0 / (double)d);
    if (mul_hi(q, d) != 0) --q;  // q d > 2^64 - 1
    if (0 - q * d >= d) ++q;     // 2^64 - q d >= d
    return q;
}

// Cofactors k of a multiple n = r k that have a factor 3, 5, 7 or 11 (bit
// k mod 1155 of a constant mask, copied into each CTA's shared memory): the
// pre-sieve by 3..113 marks those n in every segment, so the fill skips them
// -- 58 % of the atomics.
constexpr u32 kCofWheel = 1155;                       // 3 * 5 * 7 * 11
constexpr u64 kCofWheelM = 0x38bdba67495d50ull;       // floor(2^64 / 1155)
constexpr u32 kCofWords = (kCofWheel + 31) / 32;
struct CofMask {
    u32 w[kCofWords];
};
constexpr CofMask make_cof_mask() {
    CofMask m{};
    for (u32 k = 0; k < kCofWheel; ++k)
        if (k % 3 == 0 || k % 5 == 0 || k % 7 == 0 || k % 11 == 0) m.w[k >> 5] |= 1u << (k & 31);
    return m;
}
__device__ const CofMask g_cof_mask = make_cof_mask();

// One thread per large prime: its odd multiples first + 2j, j < nodd, that
// the cofactor rule marks.  The rows are streamed with evict-first loads so
// that the bitmap the atomics hit stays in L2.
__global__ void k_deep_fill(u64 first, u64 nodd, const DeepPrime *__restrict__ rows, u32 n, u32 *bits) {
    __shared__ u32 s_small[kCofWords];
    for (u32 w = threadIdx.x; w < kCofWords; w += blockDim.x) s_small[w] = g_cof_mask.w[w];
    __syncthreads();
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 row = __ldcs(reinterpret_cast<const uint4 *>(rows) + i);
    const u32 r = row.x, o = row.y;
    const u64 mo = ((u64)row.w << 32) | row.z;
    // the first odd multiple first + t of r, t even, and its cofactor k0
    // (deep_start, with k0 kept for the small-factor wheel)
    const u64 res = barrett_mod(first, r, floor_2p64_div(r));
    u64 t = res ? r - res : 0;
    if (t & 1) t += r;
    const u64 k0 = (first + t) * inv64(r);  // exact quotient; unused when first + t passes 2^64 (then 2j0 >= 2 nodd)
    u32 km = (u32)barrett_mod(k0, o, mo);
    u32 kw = (u32)barrett_mod(k0, kCofWheel, kCofWheelM);
    for (u64 j = t >> 1; j < nodd; j += r) {
        const bool small = (s_small[kw >> 5] >> (kw & 31)) & 1u;
        if ((km != 1u) & !small) atomicOr(&bits[j >> 5], 1u << (j & 31));
        km += 2u;
        if (km >= o) km -= o;
        kw += 2u;
        if (kw >= kCofWheel) kw -= kCofWheel;
    }
}

struct TableKey {
    int dev, bits;
    bool operator<(const TableKey &o) const { return dev != o.dev ? dev < o.dev : bits < o.bits; }
};
std::mutex g_table_mutex;
std::map<TableKey, DeepLarge> g_tables;  // device memory held until the process exits

}  // namespace

namespace ww {

int deep_large_device(int bits, DeepLarge *out) {
    if (bits <= WW_DEEP_BITS || bits > kDeepLargeMaxBits) {
        set_err("deep-sieve depth %d outside (%d, %d]", bits, WW_DEEP_BITS, kDeepLargeMaxBits);
        return WW_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_err("no usable current device");
        return WW_ERR_NODEV;
    }
    std::lock_guard<std::mutex> lock(g_table_mutex);
    auto it = g_tables.find({dev, bits});
    if (it != g_tables.end()) {
        *out = it->second;
        return WW_OK;
    }
    const std::vector<u32> small = small_odd_primes();
    const std::vector<u32> primes = primes_between((1u << WW_DEEP_BITS) + 1, 1u << bits, small);
    u32 *d_primes = nullptr, *d_small = nullptr;
    DeepPrime *d_rows = nullptr;
    cudaError_t e = cudaMalloc(&d_primes, primes.size() * sizeof(u32));
    if (e == cudaSuccess) e = cudaMalloc(&d_small, small.size() * sizeof(u32));
    if (e == cudaSuccess) e = cudaMalloc(&d_rows, primes.size() * sizeof(DeepPrime));
    if (e == cudaSuccess)
        e = cudaMemcpy(d_primes, primes.data(), primes.size() * sizeof(u32), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_small, small.data(), small.size() * sizeof(u32), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const u32 n = (u32)primes.size();
        k_deep_orders<<<(n + 255) / 256, 256>>>(d_primes, n, d_small, (u32)small.size(), d_rows);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(d_primes);
    cudaFree(d_small);
    if (e != cudaSuccess) {
        cudaFree(d_rows);
        cudaGetLastError();
        set_err("deep-sieve table (depth %d): %s", bits, cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? WW_ERR_NOMEM : WW_ERR_CUDA;
    }
    DeepLarge t{d_rows, (u32)primes.size()};
    g_tables[{dev, bits}] = t;
    *out = t;
    return WW_OK;
}

int read_deep_large(int bits, uint64_t first, uint64_t n, uint32_t *r, uint32_t *o, uint64_t *total) {
    DeepLarge t{nullptr, 0};
    const int rc = deep_large_device(bits, &t);
    if (rc) return rc;
    *total = t.n;
    if (first >= t.n) return WW_OK;
    if (n > t.n - first) n = t.n - first;
    std::vector<DeepPrime> rows(n);
    const cudaError_t e = cudaMemcpy(rows.data(), t.rows + first, n * sizeof(DeepPrime), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_err("deep-sieve table read: %s", cudaGetErrorString(e));
        return WW_ERR_CUDA;
    }
    for (uint64_t i = 0; i < n; ++i) {
        r[i] = rows[i].r;
        o[i] = rows[i].o;
    }
    return WW_OK;
}

int launch_deep_fill(u64 first, u64 nodd, const DeepLarge &t, u32 *bits, u64 nwords, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(bits, 0, nwords * sizeof(u32), stream);
    if (e == cudaSuccess && t.n) {
        k_deep_fill<<<(t.n + 255) / 256, 256, 0, stream>>>(first, nodd, t.rows, t.n, bits);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_err("deep-sieve marks: %s", cudaGetErrorString(e));
        return WW_ERR_CUDA;
    }
    return WW_OK;
}

}  // namespace ww
