// ww_chain.cuh -- 32-bit multiply-add carry chains and the two-digit mod p^2
// arithmetic built on them.
//
// On the device every Chain method is one PTX instruction (add.cc, madc.hi,
// ...), so each 32x32 partial product is a single IMAD on the integer pipe
// and the carries ride the condition-code flag.  On the host the same calls
// run against an emulated carry flag, which lets the CPU tests exercise the
// exact instruction sequence the kernels execute.
//
// Reduction is Montgomery's REDC in two 32-bit steps (m_i = t_i * (-p^-1)
// mod 2^32): 4 low and 4 high partial products per reduction, where a
// 64-bit q = p^-1 reduction needs 7 low and 5 high ones.  The low partial
// product m_i * p0 is never formed: it cancels t_i exactly, and its carry
// into the next limb is (t_i != 0).
#pragma once

#include "ww_arith.cuh"

namespace ww {

struct Chain {
#if !defined(__CUDA_ARCH__)
    u32 cf = 0;
#endif

#if defined(__CUDA_ARCH__)
#define WW_ASM2(op, r, a, b) asm volatile(op " %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b))
#define WW_ASM3(op, r, a, b, c) asm volatile(op " %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c))
    __device__ __forceinline__ u32 add_cc(u32 a, u32 b) { u32 r; WW_ASM2("add.cc.u32", r, a, b); return r; }
    __device__ __forceinline__ u32 addc_cc(u32 a, u32 b) { u32 r; WW_ASM2("addc.cc.u32", r, a, b); return r; }
    __device__ __forceinline__ u32 addc(u32 a, u32 b) { u32 r; WW_ASM2("addc.u32", r, a, b); return r; }
    __device__ __forceinline__ u32 mad_lo_cc(u32 a, u32 b, u32 c) { u32 r; WW_ASM3("mad.lo.cc.u32", r, a, b, c); return r; }
    __device__ __forceinline__ u32 madc_lo_cc(u32 a, u32 b, u32 c) { u32 r; WW_ASM3("madc.lo.cc.u32", r, a, b, c); return r; }
    __device__ __forceinline__ u32 mad_hi_cc(u32 a, u32 b, u32 c) { u32 r; WW_ASM3("mad.hi.cc.u32", r, a, b, c); return r; }
    __device__ __forceinline__ u32 madc_hi_cc(u32 a, u32 b, u32 c) { u32 r; WW_ASM3("madc.hi.cc.u32", r, a, b, c); return r; }
    __device__ __forceinline__ u32 madc_hi(u32 a, u32 b, u32 c) { u32 r; WW_ASM3("madc.hi.u32", r, a, b, c); return r; }
#undef WW_ASM2
#undef WW_ASM3
#else
    u32 add_cc(u32 a, u32 b) { u64 s = (u64)a + b; cf = (u32)(s >> 32); return (u32)s; }
    u32 addc_cc(u32 a, u32 b) { u64 s = (u64)a + b + cf; cf = (u32)(s >> 32); return (u32)s; }
    u32 addc(u32 a, u32 b) { return a + b + cf; }
    u32 mad_lo_cc(u32 a, u32 b, u32 c) { u64 s = (u64)(u32)(a * b) + c; cf = (u32)(s >> 32); return (u32)s; }
    u32 madc_lo_cc(u32 a, u32 b, u32 c) { u64 s = (u64)(u32)(a * b) + c + cf; cf = (u32)(s >> 32); return (u32)s; }
    static u32 hi(u32 a, u32 b) { return (u32)(((u64)a * b) >> 32); }
    u32 mad_hi_cc(u32 a, u32 b, u32 c) { u64 s = (u64)hi(a, b) + c; cf = (u32)(s >> 32); return (u32)s; }
    u32 madc_hi_cc(u32 a, u32 b, u32 c) { u64 s = (u64)hi(a, b) + c + cf; cf = (u32)(s >> 32); return (u32)s; }
    u32 madc_hi(u32 a, u32 b, u32 c) { return hi(a, b) + c + cf; }
#endif
};

WW_HD u32 lo32(u64 x) { return (u32)x; }
WW_HD u32 hi32(u64 x) { return (u32)(x >> 32); }
WW_HD u64 join(u32 lo, u32 hi) { return ((u64)hi << 32) | lo; }

// Per-modulus constants of the 32-bit arithmetic.
struct P32 {
    u64 p;
    u32 p0, p1;
    u32 np;  // -p^-1 mod 2^32
};

WW_HD P32 make_p32(u64 p, u64 q /* p^-1 mod 2^64 */) {
    P32 r;
    r.p = p;
    r.p0 = lo32(p);
    r.p1 = hi32(p);
    r.np = 0u - lo32(q);
    return r;
}

// 64x64 -> 128: r0..r3 (8 partial products).
WW_HD void mul64(u64 a, u64 b, u32 &r0, u32 &r1, u32 &r2, u32 &r3) {
    const u32 a0 = lo32(a), a1 = hi32(a), b0 = lo32(b), b1 = hi32(b);
    Chain c;
    r0 = a0 * b0;
    r1 = c.mad_hi_cc(a0, b0, 0);  // cannot carry
    r1 = c.mad_lo_cc(a0, b1, r1);
    r2 = c.madc_hi_cc(a0, b1, 0);  // cannot carry
    r1 = c.mad_lo_cc(a1, b0, r1);
    r2 = c.madc_hi_cc(a1, b0, r2);
    r3 = c.addc(0, 0);
    r2 = c.mad_lo_cc(a1, b1, r2);
    r3 = c.madc_hi(a1, b1, r3);
}

// a^2 -> 128 (6 partial products, the cross term added twice).
WW_HD void sqr64(u64 a, u32 &r0, u32 &r1, u32 &r2, u32 &r3) {
    const u32 a0 = lo32(a), a1 = hi32(a);
    Chain c;
    r0 = a0 * a0;
    r1 = c.mad_hi_cc(a0, a0, 0);
    r2 = a1 * a1;
    r3 = c.mad_hi_cc(a1, a1, 0);
    const u32 k0 = a0 * a1;
    const u32 k1 = c.mad_hi_cc(a0, a1, 0);
    r1 = c.add_cc(r1, k0);
    r2 = c.addc_cc(r2, k1);
    r3 = c.addc(r3, 0);
    r1 = c.add_cc(r1, k0);
    r2 = c.addc_cc(r2, k1);
    r3 = c.addc(r3, 0);
}

// Montgomery reduction of t0..t3 (+ t4) by 2^64 in two 32-bit steps:
// w = (T + m p) / 2^64 with m = m0 + 2^32 m1, T + m p = 0 mod 2^64.
WW_HD void redc32(u32 t0, u32 t1, u32 t2, u32 t3, u32 t4, const P32 &P, u64 &w, u32 &wtop, u64 &m) {
    Chain c;
    const u32 m0 = t0 * P.np;
    c.add_cc(t0, 0xffffffffu);  // carry of t0 + lo(m0 p0) = (t0 != 0)
    t1 = c.madc_hi_cc(m0, P.p0, t1);
    t2 = c.madc_hi_cc(m0, P.p1, t2);
    t3 = c.addc_cc(t3, 0);
    t4 = c.addc(t4, 0);
    t1 = c.mad_lo_cc(m0, P.p1, t1);
    t2 = c.addc_cc(t2, 0);
    t3 = c.addc_cc(t3, 0);
    t4 = c.addc(t4, 0);
    const u32 m1 = t1 * P.np;
    c.add_cc(t1, 0xffffffffu);
    t2 = c.madc_hi_cc(m1, P.p0, t2);
    t3 = c.madc_hi_cc(m1, P.p1, t3);
    t4 = c.addc(t4, 0);
    t2 = c.mad_lo_cc(m1, P.p1, t2);
    t3 = c.addc_cc(t3, 0);
    t4 = c.addc(t4, 0);
    w = join(t2, t3);
    wtop = t4;
    m = join(m0, m1);
}

// a^2 * 2^-64 mod n for a < n (Montgomery squaring modulo a 64-bit n).
WW_HD u64 mont_sqr32(u64 a, const P32 &P) {
    u32 r0, r1, r2, r3;
    sqr64(a, r0, r1, r2, r3);
    u64 w, m;
    u32 wtop;
    redc32(r0, r1, r2, r3, 0, P, w, wtop, m);
    return ((wtop != 0) | (w >= P.p)) ? w - P.p : w;  // w < 2n
}

// Base-2 strong probable-prime test (prime.h:65-114, getsegprimes.cl:118-164)
// as one uniform loop over the bits of n-1, so that a warp's lanes stay
// converged whatever the 2-adic valuation t of n-1: the trailing t zero
// bits square without doubling, and the checks fire at bit t (a^d = +-1)
// and below it (a^(d 2^s) = -1).  Also returns q = n^-1 mod 2^64, the
// value the reference stores in g_invert.
WW_HD bool sprp2_32(u64 n, u64 &q_out) {
    const u64 q = inv64(n);
    q_out = q;
    const P32 P = make_p32(n, q);
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
    u64 a = add_mod(one, one, n);  // 2 for the leading bit
    bool ok = false;
    for (int i = top - 1; i >= 1; --i) {
        a = mont_sqr32(a, P);
        const u64 d = add_mod(a, a, n);
        a = ((nm1 >> i) & 1) ? d : a;
        ok |= (i == t) & ((a == one) | (a == mone));
        ok |= (i < t) & (a == mone);
    }
    return ok & (t > 0);
}

// Shared tail of a product: A = x0*y0 in a0..a3, C = cross sum + u (built
// by the caller after the first reduction gave m) in c0..c4.
WW_HD D2 m2_tail(u64 w, u32 wtop, u64 m, u32 c0, u32 c1, u32 c2, u32 c3, u32 c4, const P32 &P) {
    const u64 p = P.p;
    D2 r;
    // low digit: w in [0, 2p)
    const bool ge = (wtop != 0) | (w >= p);
    r.d0 = ge ? w - p : w;
    // borrow into the high digit: (A - u p)/2^64 = w - p when m != 0, = w when m == 0
    const u64 b = (!ge & (m != 0)) ? 1 : 0;
    // high part of C + u is < 2p: bring it below p
    u64 eh = join(c2, c3);
    if ((c4 != 0) | (eh >= p)) eh -= p;
    u64 w2, m2;
    u32 wtop2;
    redc32(c0, c1, lo32(eh), hi32(eh), 0, P, w2, wtop2, m2);
    // z1 = w2 - b mod p, w2 in [0, 2p)
    const u64 t = w2 - b;
    const bool neg = (w2 < b) & (wtop2 == 0);
    const bool big = (wtop2 != 0) | (!neg & (t >= p));
    r.d1 = neg ? p - 1 : (big ? t - p : t);
    return r;
}

WW_HD D2 m2_mul32(D2 x, D2 y, const P32 &P) {
    u32 a0, a1, a2, a3;
    mul64(x.d0, y.d0, a0, a1, a2, a3);
    u64 w, m;
    u32 wtop;
    redc32(a0, a1, a2, a3, 0, P, w, wtop, m);
    const u64 u = 0 - m;  // A * p^-1 mod 2^64
    // C = x0*y1 + x1*y0 + u
    const u32 x00 = lo32(x.d0), x01 = hi32(x.d0), x10 = lo32(x.d1), x11 = hi32(x.d1);
    const u32 y00 = lo32(y.d0), y01 = hi32(y.d0), y10 = lo32(y.d1), y11 = hi32(y.d1);
    Chain c;
    u32 c0 = c.mad_lo_cc(x00, y10, lo32(u));
    u32 c1 = c.madc_hi_cc(x00, y10, hi32(u));
    u32 c2 = c.addc(0, 0);
    c1 = c.mad_lo_cc(x00, y11, c1);
    c2 = c.madc_hi_cc(x00, y11, c2);
    u32 c3 = c.addc(0, 0);
    c1 = c.mad_lo_cc(x01, y10, c1);
    c2 = c.madc_hi_cc(x01, y10, c2);
    c3 = c.addc(c3, 0);
    c2 = c.mad_lo_cc(x01, y11, c2);
    c3 = c.madc_hi(x01, y11, c3);
    c0 = c.mad_lo_cc(x10, y00, c0);
    c1 = c.madc_hi_cc(x10, y00, c1);
    c2 = c.addc_cc(c2, 0);
    c3 = c.addc_cc(c3, 0);
    u32 c4 = c.addc(0, 0);
    c1 = c.mad_lo_cc(x10, y01, c1);
    c2 = c.madc_hi_cc(x10, y01, c2);
    c3 = c.addc_cc(c3, 0);
    c4 = c.addc(c4, 0);
    c1 = c.mad_lo_cc(x11, y00, c1);
    c2 = c.madc_hi_cc(x11, y00, c2);
    c3 = c.addc_cc(c3, 0);
    c4 = c.addc(c4, 0);
    c2 = c.mad_lo_cc(x11, y01, c2);
    c3 = c.madc_hi_cc(x11, y01, c3);
    c4 = c.addc(c4, 0);
    return m2_tail(w, wtop, m, c0, c1, c2, c3, c4, P);
}

WW_HD D2 m2_sqr32(D2 x, const P32 &P) {
    u32 a0, a1, a2, a3;
    sqr64(x.d0, a0, a1, a2, a3);
    u64 w, m;
    u32 wtop;
    redc32(a0, a1, a2, a3, 0, P, w, wtop, m);
    const u64 u = 0 - m;
    // C = 2 x0 x1 + u
    u32 k0, k1, k2, k3;
    mul64(x.d0, x.d1, k0, k1, k2, k3);
    Chain c;
    u32 c0 = c.add_cc(k0, k0);
    u32 c1 = c.addc_cc(k1, k1);
    u32 c2 = c.addc_cc(k2, k2);
    u32 c3 = c.addc_cc(k3, k3);
    u32 c4 = c.addc(0, 0);
    c0 = c.add_cc(c0, lo32(u));
    c1 = c.addc_cc(c1, hi32(u));
    c2 = c.addc_cc(c2, 0);
    c3 = c.addc_cc(c3, 0);
    c4 = c.addc(c4, 0);
    return m2_tail(w, wtop, m, c0, c1, c2, c3, c4, P);
}

// Canonical digits of X * 2^-64 mod p^2 (leave Montgomery form).
WW_HD D2 m2_redc32(D2 x, const P32 &P) {
    u64 w, m;
    u32 wtop;
    redc32(lo32(x.d0), hi32(x.d0), 0, 0, 0, P, w, wtop, m);
    const u64 u = 0 - m;
    Chain c;
    const u32 c0 = c.add_cc(lo32(x.d1), lo32(u));
    const u32 c1 = c.addc_cc(hi32(x.d1), hi32(u));
    const u32 c2 = c.addc(0, 0);
    return m2_tail(w, wtop, m, c0, c1, c2, 0, 0, P);
}

}  // namespace ww

namespace ww {

// ---------------------------------------------------------------------------
// The same two-digit arithmetic written for IMAD.WIDE.U32: every 32x32
// partial product is formed as (u64)a * b + c with a 64-bit addend, which
// cannot overflow when c is the sum of at most two 32-bit words
// ((2^32-1)^2 + 2(2^32-1) = 2^64-1), so the carries ride inside the wide
// products instead of separate add-with-carry instructions.

WW_HD void mul64w(u64 a, u64 b, u64 &lo, u64 &hi) {
    const u32 a0 = lo32(a), a1 = hi32(a), b0 = lo32(b), b1 = hi32(b);
    const u64 t0 = (u64)a0 * b0;
    const u64 t1 = (u64)a0 * b1 + (t0 >> 32);
    const u64 t2 = (u64)a1 * b0 + (u32)t1;
    hi = (u64)a1 * b1 + (t1 >> 32) + (t2 >> 32);
    lo = (t2 << 32) | (u32)t0;
}

WW_HD u64 mulhi64w(u64 a, u64 b) {
    u64 lo, hi;
    mul64w(a, b, lo, hi);
    return hi;
}

// Finish of a product with 64-bit q = p^-1 reductions (the formulation of
// m2_finish, wide products).
WW_HD D2 m2_finish_w(u64 alo, u64 ahi, u64 clo, u64 chi, u64 ctop, u64 p, u64 q) {
    const u64 u = alo * q;
    const u64 v = mulhi64w(u, p);
    D2 r;
    const bool b = ahi < v;
    r.d0 = ahi - v + (b ? p : 0);
    u64 s = clo + u;
    const u64 c = s < clo;
    u64 h = chi + c;
    ctop += (h < c);
    if (ctop | (h >= p)) h -= p;
    const u64 v2 = mulhi64w(s * q, p);
    const u64 t = v2 + (u64)b;
    r.d1 = h - t + (h < t ? p : 0);
    return r;
}

WW_HD D2 m2_mul_w(D2 x, D2 y, u64 p, u64 q) {
    u64 alo, ahi, l1, h1, l2, h2;
    mul64w(x.d0, y.d0, alo, ahi);
    mul64w(x.d0, y.d1, l1, h1);
    mul64w(x.d1, y.d0, l2, h2);
    const u64 clo = l1 + l2;
    const u64 c = clo < l1;
    u64 chi = h1 + h2;
    u64 ctop = chi < h1;
    chi += c;
    ctop += chi < c;
    return m2_finish_w(alo, ahi, clo, chi, ctop, p, q);
}

WW_HD D2 m2_sqr_w(D2 x, u64 p, u64 q) {
    u64 alo, ahi, l, h;
    mul64w(x.d0, x.d0, alo, ahi);
    mul64w(x.d0, x.d1, l, h);
    return m2_finish_w(alo, ahi, l << 1, (h << 1) | (l >> 63), h >> 63, p, q);
}

WW_HD D2 m2_redc_w(D2 x, u64 p, u64 q) { return m2_finish_w(x.d0, 0, x.d1, 0, 0, p, q); }

}  // namespace ww
