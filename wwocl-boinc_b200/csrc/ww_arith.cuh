// ww_arith.cuh -- exact modular arithmetic for the WWocl search path.
//
// Compiles for the device (sm_100a) and for the host, so the same algorithm
// runs in the GPU kernels and in the host self-test.
//
//  mod n   : Montgomery, R = 2^64, with q = n^-1 mod 2^64 (the value the
//            reference's getsegprimes stores in g_invert, getsegprimes.cl:70-75)
//  mod p^2 : residues X = x0 + p*x1 (0 <= x0, x1 < p) in Montgomery form with
//            R = 2^64, the "two-digit" representation of Dorais and Klyve
//            (J. Integer Sequences 14, 2011) that the reference kernels use
//            (wieferich.cl:111-193).  Products reduce the low digit by one
//            REDC modulo p and the carry digit by a second one.
//
// The 64x64 products come from `mul_wide`/`mul_hi` (__umul64hi on the
// device, which lowers to 32-bit multiply-adds on the integer pipe).
#pragma once

#include <stdint.h>

// On the device the modular corrections (REDC's final subtraction, the
// two-digit sum and difference, the finish of a two-digit product) are PTX
// borrow chains: each turns its borrow into a mask m (0 or 2^32 - 1) and
// adds m & p back, instead of a compare and a select.  -DWW_NO_PTX_CC selects
// the C forms (measured 3 % slower on the fused test kernel).
#if !defined(WW_NO_PTX_CC) && !defined(WW_PTX_CC)
#define WW_PTX_CC 1
#endif
//
// With every correction on the integer ALU, that pipe was the busier of the
// two integer pipes in the test loops (73 % against 71 %: adds, borrows,
// selects and shifts outnumber the multiplies), so the "& p" of a correction
// runs as two 32-bit multiplies by the mask on the multiply pipe instead
// (add_masked, form 2), which leaves the multiply pipe the busier one.  WW_MAD_SITES picks where:
// bit 0 the mod-n REDC and sum of the PRP test, bit 1 the finish of a
// two-digit product, bit 2 two-digit differences, bit 3 two-digit sums; the
// places left out keep the ALU form.  Measured on a B200 (fused test kernel,
// 2^26 primes, before the three-product square): sites 1-3 in form 2,
// 1 318 M primes/s; sites 1-2, 1 340 M (with the square); sites 1 and 3 or
// 2 and 3, 1 283 and 1 216 M; the ALU mask form everywhere, 1 233 M; the
// compare/select sums and and+add masks before it, 1 148 M; form 1 (one wide
// multiply-add) at sites 1-3, 1 117 M; mad.lo.cc/madc.lo (the add fused into
// the multiply with a carry), 1 279 M against 1 364 M; the same two
// multiplies written in C, 1 221 M, or as asm on 32-bit halves, 1 349 M.
// Bit 0 slows the sieve (6.07 against 5.88 ms per 2^30 numbers), so it is off.
#ifndef WW_MAD_SITES
#define WW_MAD_SITES 14
#endif
#ifndef WW_MAD_FORM
#define WW_MAD_FORM 2
#endif
#define WW_FIX(site) ((WW_MAD_SITES >> (site)) & 1 ? WW_MAD_FORM : 0)

#if defined(__CUDACC__)
#define WW_HD __host__ __device__ __forceinline__
#else
#define WW_HD inline
#endif

namespace ww {

typedef unsigned long long u64;
typedef unsigned int u32;

struct D2 {
    u64 d0, d1;  // value = d0 + p * d1
};

// ------------------------------------------------------------ 64-bit products

WW_HD u64 mul_hi(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (u64)(((unsigned __int128)a * b) >> 64);
#endif
}

WW_HD void mul_wide(u64 a, u64 b, u64 &lo, u64 &hi) {
    lo = a * b;
    hi = mul_hi(a, b);
}

// a^2 as (hi:lo) from three 32x32 products (a0^2, a1^2 and a0 a1 once):
// a^2 = a0^2 + 2^33 a0 a1 + 2^64 a1^2.  Used for the low digit of a
// two-digit square, where it measured 3.5 % faster on the fused test kernel
// than the four-product mul_wide; in the PRP test's squaring and as the
// high word of a REDC's u*p (three products, with the carry of the known
// low word) it measured slower.
WW_HD void sqr_wide(u64 a, u64 &lo, u64 &hi) {
    const u32 a0 = (u32)a, a1 = (u32)(a >> 32);
    const u64 m = (u64)a0 * a1;
    const u64 t = m << 33;
    lo = (u64)a0 * a0 + t;
    hi = (u64)a1 * a1 + (m >> 31) + (u64)(lo < t);
}

#if defined(__CUDA_ARCH__) && defined(WW_PTX_CC)
// r + (m ? p : 0) mod 2^64 for a borrow mask m (0 or 2^32 - 1).
//   F = 0: r + (p & m:m), an and and an add on the integer ALU;
//   F = 1: two multiply-adds: with pa = -p_lo and pb = ~p_lo - p_hi (mod 2^32),
//          m pa + 2^32 (m pb) = p (mod 2^64) for m = 2^32 - 1, since
//          (2^32 - 1)(pa + 2^32 pb) = 2^32 (pa - pb) - pa = p_lo + 2^32 p_hi;
//   F = 2: the and as two multiplies (m (-p_lo) = p_lo, m (-p_hi) = p_hi
//          mod 2^32 for m = 2^32 - 1), then the add with carry.
// The constants depend on p alone, so loops hoist them.
template <int F>
__device__ __forceinline__ u64 add_masked(u64 r, u32 m, u64 p) {
    u64 t;
    if (F == 1) {
        const u32 pa = 0u - (u32)p;
        const u32 pb = ~(u32)p - (u32)(p >> 32);
        asm("{\n\t.reg .u32 lo, hi;\n\t"
            "mad.wide.u32 %0, %1, %2, %3;\n\t"
            "mov.b64 {lo, hi}, %0;\n\t"
            "mad.lo.u32 hi, %1, %4, hi;\n\t"
            "mov.b64 %0, {lo, hi};\n\t}"
            : "=l"(t) : "r"(m), "r"(pa), "l"(r), "r"(pb));
    } else if (F == 2) {
        const u32 pa = 0u - (u32)p;
        const u32 pc = 0u - (u32)(p >> 32);
        asm("{\n\t.reg .u32 a0, a1, r0, r1;\n\t"
            "mul.lo.u32 a0, %1, %2;\n\t"
            "mul.lo.u32 a1, %1, %3;\n\t"
            "mov.b64 {r0, r1}, %4;\n\t"
            "add.cc.u32 r0, r0, a0;\n\t"
            "addc.u32 r1, r1, a1;\n\t"
            "mov.b64 %0, {r0, r1};\n\t}"
            : "=l"(t) : "r"(m), "r"(pa), "r"(pc), "l"(r));
    } else {
        asm("{\n\t.reg .u64 mm;\n\t"
            "mov.b64 mm, {%1, %1};\n\t"
            "and.b64 mm, mm, %2;\n\t"
            "add.u64 %0, %3, mm;\n\t}"
            : "=l"(t) : "r"(m), "l"(p), "l"(r));
    }
    return t;
}

// a + b - n mod 2^64 for a + b < 2n, and in m the sign of the exact value:
// (c:s) = a + b, then m = c - borrow of s - n (0, or -1 when a + b < n).
// Flags set by an add are read by adds and flags set by a subtraction by
// subtractions only: ptxas does not carry the PTX meaning of the flag from
// an add.cc into a subc (measured on sm_100a: after an add.cc without carry,
// subc subtracted one).
__device__ __forceinline__ u64 sum_minus(u64 a, u64 b, u64 n, u32 &m) {
    u64 t;
    asm("{\n\t.reg .u32 c;\n\t"
        "add.cc.u64 %0, %2, %3;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "sub.cc.u64 %0, %0, %4;\n\t"
        "subc.u32 %1, c, 0;\n\t}"
        : "=&l"(t), "=r"(m) : "l"(a), "l"(b), "l"(n));
    return t;
}
#endif

// n^-1 mod 2^64 (Newton; n*n = 1 mod 8 seeds 3 correct bits).
WW_HD u64 inv64(u64 n) {
    u64 x = n;
    x *= 2 - n * x;
    x *= 2 - n * x;
    x *= 2 - n * x;
    x *= 2 - n * x;
    x *= 2 - n * x;
    return x;
}

// ------------------------------------------------------------------- mod n

WW_HD u64 add_mod(u64 a, u64 b, u64 n) {  // a <= n, b < n
#if defined(__CUDA_ARCH__) && defined(WW_PTX_CC) && (WW_MAD_SITES & 1)
    u32 m;
    const u64 t = sum_minus(a, b, n, m);
    return add_masked<WW_FIX(0)>(t, m, n);
#else
    u64 s = a + b;
    return (s < a || s >= n) ? s - n : s;
#endif
}

WW_HD u64 sub_mod(u64 a, u64 b, u64 n) {  // a < n, b <= n
    return a >= b ? a - b : a - b + n;
}

// (hi:lo) * 2^-64 mod n for (hi:lo) < n * 2^64, q = n^-1 mod 2^64.
WW_HD u64 redc(u64 lo, u64 hi, u64 n, u64 q) {
    u64 u = lo * q;
    u64 v = mul_hi(u, n);
#if defined(__CUDA_ARCH__) && defined(WW_PTX_CC) && (WW_MAD_SITES & 1)
    u64 r;
    u32 m;
    asm("sub.cc.u64 %0, %2, %3;\n\t"  // hi - v, borrow-out
        "subc.u32 %1, 0, 0;"          // -borrow
        : "=&l"(r), "=r"(m) : "l"(hi), "l"(v));
    return add_masked<WW_FIX(0)>(r, m, n);
#elif defined(__CUDA_ARCH__) && defined(WW_PTX_CC)
    u64 r;
    asm("{\n\t.reg .u64 m;\n\t"
        "sub.cc.u64 %0, %1, %2;\n\t"  // hi - v, borrow-out
        "subc.u64 m, 0, 0;\n\t"       // -borrow
        "and.b64 m, m, %3;\n\t"
        "add.u64 %0, %0, m;\n\t}"
        : "=&l"(r) : "l"(hi), "l"(v), "l"(n));
    return r;
#else
    return hi >= v ? hi - v : hi - v + n;
#endif
}

WW_HD u64 mont_mul(u64 a, u64 b, u64 n, u64 q) {
    u64 lo, hi;
    mul_wide(a, b, lo, hi);
    return redc(lo, hi, n, q);
}


// For odd n in [2^32, 2^63): q = floor(2^64 / n) and 2^64 - q n.  On the
// device the quotient comes from a double-precision estimate (off by at most
// one) corrected exactly, instead of the 64-bit division subroutine, which
// would also split the lanes of a warp.
WW_HD u64 div_r64(u64 n, u64 &q_out) {
#if defined(__CUDA_ARCH__)
    u64 q = (u64)(18446744073709551616.0 / (double)n);
    if (mul_hi(q, n) != 0) --q;  // q n >= 2^64 (never equal: n is odd and > 1)
    u64 rem = 0 - q * n;         // 2^64 - q n, in [0, 2n)
    if (rem >= n) {
        rem -= n;
        ++q;
    }
    q_out = q;
    return rem;
#else
    q_out = (0 - n) / n + 1;
    return (0 - n) % n;
#endif
}

// 2^64 mod n for odd n > 1.
WW_HD u64 r_mod(u64 n) {
    if (n >> 63) return 0 - n;  // 2^64 - n < n
    if (n >> 62) {              // 2^64 - 2n <= 2^63 < 2n
        const u64 r = 0 - 2 * n;
        return r >= n ? r - n : r;
    }
    if (n >> 32) {
        u64 q;
        return div_r64(n, q);
    }
    return (0 - n) % n;
}

// T mod n and floor(T / n) for T = h 2^64 + l < 2^46 n, n odd and > 1, with
// rn = 1.0 / (double)n.  The quotient (below 2^46) is estimated in double
// precision: T and rn each carry a relative rounding error of at most 2^-52
// and the product one more rounding, so the estimate is within 2^-4 of T / n
// and its truncation is the quotient or one off it; T - qe n then lies in
// [-n, 2n) and one exact correction finishes.  Host and device run the same
// steps.  This is how the ladders start from their top bits (a small power
// or Lucas number times the Montgomery one) without a division loop.
WW_HD u64 mod_est(u64 h, u64 l, u64 n, double rn, u64 &quot) {
    const double t = (double)h * 18446744073709551616.0 + (double)l;
    u64 qe = (u64)(t * rn);
    const u64 ql = qe * n;
    u64 lo = l - ql;
    const u64 hi = h - mul_hi(qe, n) - (u64)(l < ql);  // (hi:lo) = T - qe n
    if ((long long)hi < 0) {
        lo += n;
        --qe;
    } else if (hi != 0 || lo >= n) {
        lo -= n;
        ++qe;
    }
    quot = qe;
    return lo;
}

// Where the base-2 powering of the SPRP test starts: after the top five bits
// v of n-1 (2^v R mod n from one exact reduction, mod_est) when the 2-adic
// valuation t of n-1 lies below them, which saves the first four squarings;
// otherwise after the leading bit.  Returns s, the loop then takes the bits
// s-1 .. 1 of n-1; a receives the start value.
WW_HD int sprp2_start(u64 n, u64 one, int top, int t, u64 &a) {
    const int s = (top - 4 > t) ? top - 4 : top;
    const u32 v = (u32)((n - 1) >> s);  // in [16, 32), or 1
    u64 qd;
    a = mod_est(one >> (64 - v), one << v, n, 1.0 / (double)n, qd);
    return s;
}

// Base-2 strong probable-prime test (prime.h:65-114, getsegprimes.cl:118-164)
// written as one uniform loop over the bits of n-1 so that a warp's lanes
// stay converged whatever the 2-adic valuation t of n-1 is: the trailing t
// zero bits square without doubling; the loop keeps a^d (the value at bit t)
// and whether a^(d 2^s) = -1 below it, and the checks run once at the end.
// The powering starts from the top bits of n-1 (sprp2_start).  Returns the
// result and n^-1 mod 2^64.
WW_HD bool sprp2(u64 n, u64 &q_out) {
    const u64 q = inv64(n);
    q_out = q;
    const u64 one = r_mod(n);
    const u64 mone = n - one;
    const u64 nm1 = n - 1;
#if defined(__CUDA_ARCH__)
    const int t = __ffsll((long long)nm1) - 1;
    const int top = 63 - __clzll((long long)nm1);
#else
    const int t = __builtin_ctzll(nm1);
    const int top = 63 - __builtin_clzll(nm1);
#endif
    u64 a;
    const int s = sprp2_start(n, one, top, t, a);
    u64 at_t = 0;                  // 2^d, the value at bit t
    bool m1 = false;               // 2^(d 2^s) = -1 for some 0 < s < t
    for (int i = s - 1; i >= 1; --i) {
        a = mont_mul(a, a, n, q);
        const u64 d = add_mod(a, a, n);
        a = ((nm1 >> i) & 1) ? d : a;
        at_t = (i == t) ? a : at_t;
        m1 |= (i < t) & (a == mone);
    }
    bool ok = (at_t == one) | (at_t == mone) | m1;
    if (t == 0) ok = false;  // even n is never a candidate
    // t == top (n-1 a power of two, as for the pseudoprime 2^32+1): the value
    // at bit t is 2, never +-1, and m1 covers every s < t
    return ok;
}

#if defined(__CUDACC__)
// sprp2 for a whole warp: all 32 lanes call it, and lanes with act false test
// the first active lane's number and return false.  The squarings above
// every lane's bit t touch neither the value at bit t nor the -1 check, so
// they run in a first loop without that bookkeeping; the second loop is
// sprp2's own, from the warp's largest t down.
__device__ __forceinline__ bool sprp2_warp(u64 n, bool act, u64 &q_out) {
    const u32 live = __ballot_sync(0xffffffffu, act);
    if (live == 0) {
        q_out = 0;
        return false;
    }
    const u64 src = __shfl_sync(0xffffffffu, n, __ffs((int)live) - 1);
    n = act ? n : src;
    const u64 q = inv64(n);
    q_out = q;
    const u64 one = r_mod(n);
    const u64 mone = n - one;
    const u64 nm1 = n - 1;
    const int t = __ffsll((long long)nm1) - 1;  // >= 1: n is odd
    const int top = 63 - __clzll((long long)nm1);
    const int tw = (int)__reduce_max_sync(0xffffffffu, (unsigned)t);
    u64 a;
    const int s = sprp2_start(n, one, top, t, a);
    u64 ebits = nm1 << (64 - s);  // bit s-1 of n-1 at bit 63
    int i = s - 1;
    for (; i > tw; --i) {
        a = mont_mul(a, a, n, q);
        const u64 d = add_mod(a, a, n);
        a = ((long long)ebits < 0) ? d : a;
        ebits <<= 1;
    }
    u64 at_t = 0;
    bool m1 = false;
    for (; i >= 1; --i) {
        a = mont_mul(a, a, n, q);
        const u64 d = add_mod(a, a, n);
        a = ((long long)ebits < 0) ? d : a;
        ebits <<= 1;
        at_t = (i == t) ? a : at_t;
        m1 |= (i < t) & (a == mone);
    }
    const bool ok = (at_t == one) | (at_t == mone) | m1;
    return act && ok;
}
#endif

// ----------------------------------------------------------------- mod p^2
// ----------------------------------------------------------------- mod p^2

struct ModP2 {
    u64 p, q;  // q = p^-1 mod 2^64
};

WW_HD D2 m2_add(D2 x, D2 y, u64 p) {
    D2 r;
#if defined(__CUDA_ARCH__) && defined(WW_PTX_CC) && (WW_MAD_SITES & 8)
    // low digit: (c:s) = x0 + y0 - p with m0 = c - borrow (0 or -1); the
    // high digit x1 + (1 + m0) + y1 - p the same way (x1 + 1 + m0 <= p)
    u32 m0, m1;
    const u64 t0 = sum_minus(x.d0, y.d0, p, m0);
    const u64 t1 = sum_minus(x.d1 + (u64)(m0 + 1u), y.d1, p, m1);
    r.d0 = add_masked<WW_FIX(3)>(t0, m0, p);
    r.d1 = add_masked<WW_FIX(3)>(t1, m1, p);
#else
    u64 s = x.d0 + y.d0;
    bool c = (s < x.d0) | (s >= p);
    r.d0 = c ? s - p : s;
    u64 h = x.d1 + (u64)c;  // <= p
    u64 t = h + y.d1;
    r.d1 = ((t < h) | (t >= p)) ? t - p : t;
#endif
    return r;
}

WW_HD D2 m2_sub(D2 x, D2 y, u64 p) {
    D2 r;
#if defined(__CUDA_ARCH__) && defined(WW_PTX_CC) && (WW_MAD_SITES & 4)
    // one borrow chain through both digits; each digit's borrow-out becomes a
    // mask (subc without .cc leaves the flag for the next digit)
    u64 t0, t1;
    u32 m0, m1;
    asm("sub.cc.u64 %0, %4, %6;\n\t"
        "subc.u32 %2, 0, 0;\n\t"
        "subc.cc.u64 %1, %5, %7;\n\t"  // x1 - y1 - borrow
        "subc.u32 %3, 0, 0;"
        : "=&l"(t0), "=&l"(t1), "=&r"(m0), "=&r"(m1)
        : "l"(x.d0), "l"(x.d1), "l"(y.d0), "l"(y.d1));
    r.d0 = add_masked<WW_FIX(2)>(t0, m0, p);
    r.d1 = add_masked<WW_FIX(2)>(t1, m1, p);
    return r;
#elif defined(__CUDA_ARCH__) && defined(WW_PTX_CC)
    // one borrow chain through both digits; each digit adds p back on its
    // own borrow-out
    asm("{\n\t.reg .u64 m0, m1;\n\t"
        "sub.cc.u64 %0, %2, %4;\n\t"
        "subc.u64 m0, 0, 0;\n\t"       // reads the low borrow, keeps it
        "subc.cc.u64 %1, %3, %5;\n\t"  // x1 - y1 - borrow
        "subc.u64 m1, 0, 0;\n\t"
        "and.b64 m0, m0, %6;\n\t"
        "and.b64 m1, m1, %6;\n\t"
        "add.u64 %0, %0, m0;\n\t"
        "add.u64 %1, %1, m1;\n\t}"
        : "=&l"(r.d0), "=&l"(r.d1)
        : "l"(x.d0), "l"(x.d1), "l"(y.d0), "l"(y.d1), "l"(p));
    return r;
#else
    bool b = x.d0 < y.d0;
    r.d0 = b ? x.d0 - y.d0 + p : x.d0 - y.d0;
    u64 t = y.d1 + (u64)b;  // <= p
    r.d1 = x.d1 >= t ? x.d1 - t : x.d1 - t + p;
    return r;
#endif
}

WW_HD D2 m2_dbl(D2 x, u64 p) { return m2_add(x, x, p); }

// Finish a product: A = (alo, ahi) is x0*y0, (clo, chi, ctop) the cross sum
// x0*y1 + x1*y0 (129 bits).  Montgomery: X*Y*2^-64 = (A - u p)/2^64
// + p * ((C + u) * 2^-64 mod p), u = alo * q.
WW_HD D2 m2_finish(u64 alo, u64 ahi, u64 clo, u64 chi, u64 ctop, u64 p, u64 q) {
    const u64 u = alo * q;
    const u64 v = mul_hi(u, p);
    D2 r;
#if defined(__CUDA_ARCH__) && defined(WW_PTX_CC) && (WW_MAD_SITES & 2)
    u64 t0, s, t1, t2;
    u32 mb, mh, md;
    // low digit ahi - v, plus p on borrow (mb = -borrow)
    asm("sub.cc.u64 %0, %2, %3;\n\t"
        "subc.u32 %1, 0, 0;"
        : "=&l"(t0), "=r"(mb) : "l"(ahi), "l"(v));
    r.d0 = add_masked<WW_FIX(1)>(t0, mb, p);
    // (k:h) = (C + u) >> 64 < 2p and s its low word; then (k:h) - p with
    // mh = k - borrow, which is -1 exactly when (k:h) < p
    asm("{\n\t.reg .u32 k;\n\t.reg .u64 h;\n\t"
        "add.cc.u64 %0, %3, %4;\n\t"
        "addc.cc.u64 h, %5, 0;\n\t"
        "addc.u32 k, %6, 0;\n\t"
        "sub.cc.u64 %1, h, %7;\n\t"
        "subc.u32 %2, k, 0;\n\t}"
        : "=&l"(s), "=&l"(t1), "=&r"(mh)
        : "l"(clo), "l"(u), "l"(chi), "r"((u32)ctop), "l"(p));
    const u64 h2 = add_masked<WW_FIX(1)>(t1, mh, p);
    const u64 v2 = mul_hi(s * q, p);
    // high digit h2 - v2 - borrow of the low digit (the flag set again from
    // mb: 0 - mb borrows exactly when mb = -1), plus p on borrow.  Every flag
    // here is set by a subtraction and read by one: ptxas does not carry the
    // PTX meaning of the flag from an add.cc into a subc (measured on sm_100a:
    // after an add.cc without carry, subc subtracted one).
    asm("{\n\t.reg .u32 z;\n\t"
        "sub.cc.u32 z, 0, %2;\n\t"
        "subc.cc.u64 %0, %3, %4;\n\t"
        "subc.u32 %1, 0, 0;\n\t}"
        : "=&l"(t2), "=r"(md) : "r"(mb), "l"(h2), "l"(v2));
    r.d1 = add_masked<WW_FIX(1)>(t2, md, p);
    return r;
#elif defined(__CUDA_ARCH__) && defined(WW_PTX_CC)
    u64 mb, s, h, k, h2;
    // low digit ahi - v, plus p on borrow; mb = -borrow
    asm("{\n\t.reg .u64 t;\n\t"
        "sub.cc.u64 %0, %2, %3;\n\t"
        "subc.u64 %1, 0, 0;\n\t"
        "and.b64 t, %1, %4;\n\t"
        "add.u64 %0, %0, t;\n\t}"
        : "=&l"(r.d0), "=&l"(mb) : "l"(ahi), "l"(v), "l"(p));
    // (k:h) = (C + u) >> 64 < 2p, s = low word of C + u
    asm("add.cc.u64 %0, %3, %4;\n\t"
        "addc.cc.u64 %1, %5, 0;\n\t"
        "addc.u64 %2, %6, 0;"
        : "=&l"(s), "=&l"(h), "=&l"(k) : "l"(clo), "l"(u), "l"(chi), "l"(ctop));
    // h2 = (k:h) mod p: subtract p; the high word k - borrow is -1 exactly
    // when (k:h) < p, and then p is added back
    asm("{\n\t.reg .u64 m;\n\t"
        "sub.cc.u64 %0, %1, %2;\n\t"
        "subc.u64 m, %3, 0;\n\t"
        "shr.s64 m, m, 1;\n\t"
        "and.b64 m, m, %2;\n\t"
        "add.u64 %0, %0, m;\n\t}"
        : "=&l"(h2) : "l"(h), "l"(p), "l"(k));
    const u64 v2 = mul_hi(s * q, p);
    const u64 t = v2 - mb;  // v2 + borrow <= p
    asm("{\n\t.reg .u64 m;\n\t"
        "sub.cc.u64 %0, %1, %2;\n\t"
        "subc.u64 m, 0, 0;\n\t"
        "and.b64 m, m, %3;\n\t"
        "add.u64 %0, %0, m;\n\t}"
        : "=&l"(r.d1) : "l"(h2), "l"(t), "l"(p));
    return r;
#else
    const bool b = ahi < v;
    r.d0 = b ? ahi - v + p : ahi - v;
    // C + u
    u64 s = clo + u;
    u64 c = s < clo;
    u64 h = chi + c;
    ctop += (h < c);
    // high part < 2p: reduce once
    if (ctop | (h >= p)) h -= p;
    const u64 u2 = s * q;
    const u64 v2 = mul_hi(u2, p);
    const u64 t = v2 + (u64)b;  // <= p
    r.d1 = h >= t ? h - t : h - t + p;
    return r;
#endif
}

WW_HD D2 m2_mul(D2 x, D2 y, u64 p, u64 q) {
    u64 alo, ahi, l1, h1, l2, h2;
    mul_wide(x.d0, y.d0, alo, ahi);
    mul_wide(x.d0, y.d1, l1, h1);
    mul_wide(x.d1, y.d0, l2, h2);
    u64 clo = l1 + l2;
    u64 c = clo < l1;
    u64 chi = h1 + h2;
    u64 ctop = chi < h1;
    chi += c;
    ctop += chi < c;
    return m2_finish(alo, ahi, clo, chi, ctop, p, q);
}

WW_HD D2 m2_sqr(D2 x, u64 p, u64 q) {
    u64 alo, ahi, l, h;
    sqr_wide(x.d0, alo, ahi);
    mul_wide(x.d0, x.d1, l, h);
    const u64 ctop = h >> 63;
    const u64 chi = (h << 1) | (l >> 63);
    const u64 clo = l << 1;
    return m2_finish(alo, ahi, clo, chi, ctop, p, q);
}

// Leave Montgomery form: canonical digits of X * 2^-64 mod p^2.
WW_HD D2 m2_redc(D2 x, u64 p, u64 q) { return m2_finish(x.d0, 0, x.d1, 0, 0, p, q); }

// 2^64 mod p^2 as digits: the Montgomery form of 1 (wieferich.cl:116-126).
WW_HD D2 m2_one(u64 p) {
    D2 r;
    if ((p >> 32) == 0) {
        const u64 p2 = p * p;
        const u64 rr = (0 - p2) % p2;
        r.d0 = rr % p;
        r.d1 = rr / p;
        return r;
    }
    if (p >> 63) {  // 2^64 = (2^64 - p) + 1 * p
        r.d0 = 0 - p;
        r.d1 = 1;
        return r;
    }
    if (p >> 62) {  // 2^64 = 2p + (2^64 - 2p), and 2^64 - 2p <= 2^63 < 2p
        r.d0 = 0 - 2 * p;
        r.d1 = 2;
        if (r.d0 >= p) {
            r.d0 -= p;
            r.d1 = 3;
        }
        return r;
    }
    // 2^32 <= p < 2^62: 2^64 = q p + rem with q < p
    u64 q;
    r.d0 = div_r64(p, q);
    r.d1 = q;
    return r;
}

// L R mod p^2 as canonical digits for L < 2^45, from the Montgomery one
// (R mod p^2 = o0 + p o1): L o0 = d0 + p q0 with d0 < p, then d1 = (q0 + L o1)
// mod p.  Both reductions see a number below 2^46 p (mod_est); rp = 1/(double)p.
WW_HD D2 m2_small(u64 L, D2 one, u64 p, double rp) {
    u64 l, h, q0, q1;
    D2 r;
    mul_wide(L, one.d0, l, h);
    r.d0 = mod_est(h, l, p, rp, q0);
    mul_wide(L, one.d1, l, h);
    l += q0;
    h += (u64)(l < q0);
    r.d1 = mod_est(h, l, p, rp, q1);
    return r;
}

// X 2^v mod p^2 for v < 16 (a plain multiple, so Montgomery form is kept):
// x0 2^v = d0 + p q0, then d1 = (x1 2^v + q0) mod p, both below 2^16 p.
WW_HD D2 m2_mul_pow2(D2 x, u32 v, u64 p, double rp) {
    u64 q0, q1;
    D2 r;
    const u64 h0 = v ? x.d0 >> (64 - v) : 0;
    r.d0 = mod_est(h0, x.d0 << v, p, rp, q0);
    u64 h1 = v ? x.d1 >> (64 - v) : 0;
    const u64 l1 = (x.d1 << v) + q0;
    h1 += (u64)(l1 < q0);
    r.d1 = mod_est(h1, l1, p, rp, q1);
    return r;
}

// x / 5 mod p for 0 <= x < p, p prime to 5; also returns j with 5y = x + j p.
WW_HD u64 div5_mod(u64 x, u64 p, u32 pm5, u32 &j) {
    // inverse of p mod 5 for residues 1..4: 1, 3, 2, 4
    const u32 inv = (0x42310u >> (4 * pm5)) & 0xF;  // nibbles 0..4: 0, 1, 3, 2, 4
    const u32 xm5 = (u32)(x % 5);
    j = ((5 - xm5) * inv) % 5;
    return (x + (u64)j * p) * 0xCCCCCCCCCCCCCCCDull;  // exact division by 5 mod 2^64
}

// Canonical digits t -> digits of t / 5 mod p^2.
WW_HD D2 m2_div5(D2 t, u64 p) {
    const u32 pm5 = (u32)(p % 5);
    u32 j0, j1;
    D2 y;
    y.d0 = div5_mod(t.d0, p, pm5, j0);
    y.d1 = div5_mod(sub_mod(t.d1, (u64)j0, p), p, pm5, j1);
    return y;
}

}  // namespace ww
