// ww_util.cu -- measurement utilities of libwwcuda.so (no reference
// counterpart): the seeded random prime list used by the fixed-list
// benchmark, and the integer/FP64 pipe microbenchmark that measures the
// roofline denominator on the device at hand.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/wwcuda.h"
#include "ww_arith.cuh"
#include "ww_tests.cuh"

using namespace ww;

namespace {

WW_HD u64 splitmix64(u64 seed, u64 i) {
    u64 z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Strong probable-prime test to an arbitrary base (prime.h:65-114).
__device__ bool sprp_base(u64 n, u64 q, u64 one, u64 r2, u64 base) {
    const u64 nm1 = n - 1;
    const int t = __ffsll((long long)nm1) - 1;
    const u64 d = nm1 >> t;
    const u64 mb = mont_mul(base % n, r2, n, q);
    u64 a = mb;
    for (int i = 62 - __clzll((long long)d); i >= 0; --i) {
        a = mont_mul(a, a, n, q);
        if ((d >> i) & 1) a = mont_mul(a, mb, n, q);
    }
    const u64 mone = n - one;
    if (a == one || a == mone) return true;
    for (int s = 1; s < t; ++s) {
        a = mont_mul(a, a, n, q);
        if (a == mone) return true;
    }
    return false;
}

// isPrime (main.cpp:301-324) for odd n > 113.
__device__ bool is_prime_dev(u64 n) {
    const u64 q = inv64(n);
    const u64 one = r_mod(n);
    u64 r2 = add_mod(one, one, n);
    r2 = add_mod(r2, r2, n);
#pragma unroll 1
    for (int i = 0; i < 5; ++i) r2 = mont_mul(r2, r2, n, q);
    const int nb = n < 3825123056546413051ull ? 9 : 12;
    const u64 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
#pragma unroll 1
    for (int i = 0; i < nb; ++i)
        if (!sprp_base(n, q, one, r2, bases[i])) return false;
    return true;
}

__device__ bool small_factor(u64 n) {
    const u32 ps[29] = {3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
                        59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113};
#pragma unroll
    for (int i = 0; i < 29; ++i)
        if (n % ps[i] == 0) return true;
    return false;
}

// One bit per stream position i0 + k: candidate kept and prime.
__global__ void k_rand_bits(u64 seed, u64 i0, u64 nwords, u32 *bits) {
    const int lane = threadIdx.x & 31;
    const u64 warp = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
    for (u64 w = warp; w < nwords; w += nwarps) {
        const u64 i = i0 + w * 32 + lane;
        const u64 c = splitmix64(seed, i) | 1;
        const bool ok = (c >> 62) != 0 && !small_factor(c) && is_prime_dev(c);
        const u32 b = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) bits[w] = b;
    }
}

template <int MODE>
__global__ void k_pipe(int iters, u32 seed, u32 *sink) {
    u32 x[8];
    unsigned long long X[8];
    double f[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = threadIdx.x * 17u + (u32)k + seed;
        X[k] = ((unsigned long long)x[k] << 32) | (x[k] ^ 0x9e3779b9u);
        f[k] = (double)x[k] * 1e-9;
    }
    const u32 y = seed | 1u, z = seed ^ 0x1234u;
    const double fy = 1.0000001, fz = 1e-7;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (MODE == 0) {
                asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[k]) : "r"(y), "r"(z));
            } else if (MODE == 1) {
                asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(x[k]) : "r"(y), "r"(z));
            } else if (MODE == 2) {
                asm volatile(
                    "{\n\t.reg .u32 lo, hi;\n\tmov.b64 {lo, hi}, %0;\n\t"
                    "mad.wide.u32 %0, lo, %1, %0;\n\t}"
                    : "+l"(X[k])
                    : "r"(y));
            } else if (MODE == 3) {
                // 64x64 -> 128 product as 8 multiply-adds with carries (the
                // partial products of mul_wide): X[k] = lo, x[k] = folded hi
                asm volatile(
                    "{\n\t.reg .u32 a0, a1, b0, b1, r0, r1, r2, r3;\n\t"
                    "mov.b64 {a0, a1}, %0;\n\t"
                    "mov.b32 b0, %2;\n\tmov.b32 b1, %3;\n\t"
                    "mul.lo.u32 r0, a0, b0;\n\t"
                    "mul.hi.u32 r1, a0, b0;\n\t"
                    "mad.lo.cc.u32 r1, a0, b1, r1;\n\t"
                    "madc.hi.u32 r2, a0, b1, 0;\n\t"
                    "mad.lo.cc.u32 r2, a1, b1, r2;\n\t"
                    "madc.hi.u32 r3, a1, b1, 0;\n\t"
                    "mad.lo.cc.u32 r1, a1, b0, r1;\n\t"
                    "madc.hi.cc.u32 r2, a1, b0, r2;\n\t"
                    "addc.u32 r3, r3, 0;\n\t"
                    "xor.b32 r0, r0, r2;\n\txor.b32 r1, r1, r3;\n\t"
                    "mov.b64 %0, {r0, r1};\n\t"
                    "add.u32 %1, %1, r3;\n\t}"
                    : "+l"(X[k]), "+r"(x[k])
                    : "r"(y), "r"(z));
            } else if (MODE == 4) {
                asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(f[k]) : "d"(fy), "d"(fz));
            } else {
                asm volatile("add.u32 %0, %0, %1;" : "+r"(x[k]) : "r"(y));
            }
        }
    }
    u32 acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc ^= x[k] ^ (u32)X[k] ^ (u32)(X[k] >> 32) ^ (u32)(long long)f[k];
    if (acc == 0x7fffffffu) sink[threadIdx.x] = acc;  // keeps the chains live
}

// One operation of the device arithmetic per case (the instruction sequences
// the kernels run), for checking it operand by operand: ops 0-2 as
// ww_selftest_m2, 3 X+Y, 4 X-Y, 5 2X (mod p^2), 6 x0*y0/2^64, 7 x0+y0,
// 8 (x1:x0)/2^64 (mod p).
__global__ void k_m2_cases(int op, u64 p, const u64 *xy, u64 n, u64 *out) {
    const u64 q = inv64(p);
    const WW_ARITH ar(p, q);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const D2 x = {xy[4 * i], xy[4 * i + 1]};
        const D2 y = {xy[4 * i + 2], xy[4 * i + 3]};
        D2 z = {0, 0};
        switch (op) {
            case 0: z = ar.mul(x, y); break;
            case 1: z = ar.sqr(x); break;
            case 2: z = ar.redc(x); break;
            case 3: z = m2_add(x, y, p); break;
            case 4: z = m2_sub(x, y, p); break;
            case 5: z = m2_dbl(x, p); break;
            case 6: z.d0 = mont_mul(x.d0, y.d0, p, q); break;
            case 7: z.d0 = add_mod(x.d0, y.d0, p); break;
            default: z.d0 = redc(x.d0, x.d1, p, q); break;
        }
        out[2 * i] = z.d0;
        out[2 * i + 1] = z.d1;
    }
}

}  // namespace

extern "C" {

int ww_random_primes(int device, uint64_t seed, uint64_t n, uint64_t *out, uint64_t *consumed) {
    if (!out && n) return WW_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return WW_ERR_NODEV;
    const u64 chunk_words = 1ull << 21;  // 2^26 stream positions per launch
    u32 *dbits = nullptr;
    if (cudaMalloc(&dbits, chunk_words * 4) != cudaSuccess) return WW_ERR_NOMEM;
    std::vector<u32> hbits(chunk_words);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    u64 have = 0, pos = 0, used = 0;
    int rc = WW_OK;
    while (have < n) {
        k_rand_bits<<<sms * 8, 256>>>(seed, pos, chunk_words, dbits);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(hbits.data(), dbits, chunk_words * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = WW_ERR_CUDA;
            break;
        }
        for (u64 w = 0; w < chunk_words && have < n; ++w) {
            u32 b = hbits[w];
            while (b && have < n) {
                const int k = __builtin_ctz(b);
                const u64 i = pos + w * 32 + (u64)k;
                out[have++] = splitmix64(seed, i) | 1;
                used = i + 1;
                b &= b - 1;
            }
        }
        pos += chunk_words * 32;
    }
    cudaFree(dbits);
    if (consumed) *consumed = used;
    return rc;
}

int ww_devtest_m2(int device, int op, uint64_t p, const uint64_t *xy, uint64_t n, uint64_t *out) {
    if ((p & 1) == 0 || p < 3 || ((!xy || !out) && n) || op < 0 || op > 8) return WW_ERR_ARG;
    if (n == 0) return WW_OK;
    if (cudaSetDevice(device) != cudaSuccess) return WW_ERR_NODEV;
    u64 *d = nullptr;
    if (cudaMalloc(&d, n * 48) != cudaSuccess) return WW_ERR_NOMEM;
    int rc = WW_OK;
    if (cudaMemcpy(d, xy, n * 32, cudaMemcpyHostToDevice) != cudaSuccess) rc = WW_ERR_CUDA;
    if (rc == WW_OK) {
        const u64 blocks = (n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184;
        k_m2_cases<<<(unsigned)blocks, 256>>>(op, p, d, n, d + 4 * n);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(out, d + 4 * n, n * 16, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = WW_ERR_CUDA;
    }
    cudaFree(d);
    return rc;
}

int ww_pipe_bench(int device, int mode, double *ops_per_s, double *ms_out) {
    if (mode < 0 || mode > 5 || !ops_per_s) return WW_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return WW_ERR_NODEV;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    u32 *sink = nullptr;
    if (cudaMalloc(&sink, 1024 * 4) != cudaSuccess) return WW_ERR_NOMEM;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 8, threads = 256;
    auto launch = [&](int iters) {
        switch (mode) {
            case 0: k_pipe<0><<<blocks, threads>>>(iters, 7u, sink); break;
            case 1: k_pipe<1><<<blocks, threads>>>(iters, 7u, sink); break;
            case 2: k_pipe<2><<<blocks, threads>>>(iters, 7u, sink); break;
            case 3: k_pipe<3><<<blocks, threads>>>(iters, 7u, sink); break;
            case 4: k_pipe<4><<<blocks, threads>>>(iters, 7u, sink); break;
            default: k_pipe<5><<<blocks, threads>>>(iters, 7u, sink); break;
        }
    };
    int iters = 1024;
    launch(iters);  // warm-up
    cudaDeviceSynchronize();
    float ms = 0;
    for (;;) {
        cudaEventRecord(a);
        launch(iters);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        if (ms > 20.0f || iters >= (1 << 22)) break;
        iters *= 4;
    }
    const int rc = cudaGetLastError() == cudaSuccess ? WW_OK : WW_ERR_CUDA;
    // instructions of the measured kind per chain step: 8 for mode 3 (the
    // multiply-adds of one 64x64->128 product), 1 otherwise
    const double per = mode == 3 ? 8.0 : 1.0;
    *ops_per_s = (double)blocks * threads * 8.0 * iters * per / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    return rc;
}

}  // extern "C"
