// ww_tests.cuh -- the Wieferich and Wall-Sun-Sun tests of one prime, and the
// reference's hit classification.
//
// The mod p^2 arithmetic is a policy: Arith64 uses 64-bit C products
// (ww_arith.cuh), Arith32 explicit 32-bit PTX carry chains and ArithWide
// 32x32+64 wide products (ww_chain.cuh).  All produce the same canonical
// digits; kernels and the host self-test use WW_ARITH.
#pragma once

#include "ww_arith.cuh"
#include "ww_chain.cuh"

namespace ww {

struct Arith64 {
    u64 p, q;
    WW_HD Arith64(u64 p_, u64 q_) : p(p_), q(q_) {}
    WW_HD D2 mul(D2 x, D2 y) const { return m2_mul(x, y, p, q); }
    WW_HD D2 sqr(D2 x) const { return m2_sqr(x, p, q); }
    WW_HD D2 redc(D2 x) const { return m2_redc(x, p, q); }
};

struct Arith32 {
    P32 P;
    WW_HD Arith32(u64 p, u64 q) : P(make_p32(p, q)) {}
    WW_HD D2 mul(D2 x, D2 y) const { return m2_mul32(x, y, P); }
    WW_HD D2 sqr(D2 x) const { return m2_sqr32(x, P); }
    WW_HD D2 redc(D2 x) const { return m2_redc32(x, P); }
};

struct ArithWide {
    u64 p, q;
    WW_HD ArithWide(u64 p_, u64 q_) : p(p_), q(q_) {}
    WW_HD D2 mul(D2 x, D2 y) const { return m2_mul_w(x, y, p, q); }
    WW_HD D2 sqr(D2 x) const { return m2_sqr_w(x, p, q); }
    WW_HD D2 redc(D2 x) const { return m2_redc_w(x, p, q); }
};

// WW_ARITH_VERSION: 1 = 64-bit C products (default), 2 = PTX carry chains,
// 3 = wide 32x32+64 products.  All three give identical digits.
#if defined(WW_ARITH_VERSION) && WW_ARITH_VERSION == 2
typedef Arith32 WW_ARITH;
WW_HD bool prp_test(u64 n, u64 &q) { return sprp2_32(n, q); }
#elif defined(WW_ARITH_VERSION) && WW_ARITH_VERSION == 3
typedef ArithWide WW_ARITH;
WW_HD bool prp_test(u64 n, u64 &q) { return sprp2(n, q); }
#else
typedef Arith64 WW_ARITH;
WW_HD bool prp_test(u64 n, u64 &q) { return sprp2(n, q); }
#endif

#if defined(__CUDACC__)
// prp_test for a whole warp (all lanes call it; act false gives false)
__device__ __forceinline__ bool prp_test_warp(u64 n, bool act, u64 &q) {
#if defined(WW_ARITH_VERSION) && WW_ARITH_VERSION == 2
    return act && sprp2_32(n, q);
#else
    return sprp2_warp(n, act, q);
#endif
}
#endif

WW_HD int top_bit(u64 x) {
#if defined(__CUDA_ARCH__)
    return 63 - __clzll((long long)x);
#else
    return 63 - __builtin_clzll(x);
#endif
}

WW_HD D2 sel(bool c, D2 a, D2 b) {
    D2 r;
    r.d0 = c ? a.d0 : b.d0;
    r.d1 = c ? a.d1 : b.d1;
    return r;
}

// Lucas numbers V_k (P = 1, Q = -1: V_0 = 2, V_1 = 1) for 32 <= k <= 64, all
// below 2^45: the Lucas ladder's state after the top six bits of its index.
#define WW_LUCAS_32_64                                                                                \
    4870847ull, 7881196ull, 12752043ull, 20633239ull, 33385282ull, 54018521ull, 87403803ull,        \
        141422324ull, 228826127ull, 370248451ull, 599074578ull, 969323029ull, 1568397607ull,        \
        2537720636ull, 4106118243ull, 6643838879ull, 10749957122ull, 17393796001ull, 28143753123ull, \
        45537549124ull, 73681302247ull, 119218851371ull, 192900153618ull, 312119004989ull,          \
        505019158607ull, 817138163596ull, 1322157322203ull, 2139295485799ull, 3461452808002ull,     \
        5600748293801ull, 9062201101803ull, 14662949395604ull, 23725150497407ull
#if defined(__CUDACC__)
static __device__ const u64 g_lucas_32_64[33] = {WW_LUCAS_32_64};
#endif
static const u64 h_lucas_32_64[33] = {WW_LUCAS_32_64};

WW_HD u64 lucas_small(u32 k) {  // 32 <= k <= 64
#if defined(__CUDA_ARCH__)
    return __ldg(&g_lucas_32_64[k - 32]);
#else
    return h_lucas_32_64[k - 32];
#endif
}

// Where the ladders start.  Each takes the bits of its exponent below its
// start bit in the loop and begins from the value of the bits above it:
//   Lucas: i0 = top_bit(n) - 6 for n = p - (p|5); k0 = n >> (i0 + 1) is the
//          top six bits of n (32 <= k0 < 64), so the pair (V_k0, V_k0+1)
//          comes from lucas_small;
//   Wieferich: iw = top_bit(e) - 5 for e = (p-1)/2; e0 = e >> (iw + 1) is the
//          top five bits of e (16 <= e0 < 32), so the start is 2^e0.
// e has one bit fewer than n, so iw = i0 (two fewer when p + 1 is a power of
// two, and then the first loop step is the Lucas ladder's alone).  m2_small
// turns each start into Montgomery form with two exact reductions: six
// reductions of about 25 instructions replace the first five ladder steps
// (ten squarings) and four Wieferich squarings.
struct LadderStart {
    int i0, iw;
    bool odd;  // parity of the Lucas index k0
    D2 a, b, w;
    double rp;  // 1 / (double)p
};

WW_HD LadderStart ladder_start(u64 p, u64 n, D2 one) {
    LadderStart st;
    const u64 e = p >> 1;
    st.i0 = top_bit(n) - 6;
    st.iw = top_bit(e) - 5;
    const u32 k0 = (u32)(n >> (st.i0 + 1));
    const u32 e0 = (u32)(e >> (st.iw + 1));
    const double rp = 1.0 / (double)p;
    st.rp = rp;
    st.odd = k0 & 1u;
    st.a = m2_small(lucas_small(k0), one, p, rp);
    st.b = m2_small(lucas_small(k0 + 1), one, p, rp);
    st.w = m2_small(1ull << e0, one, p, rp);
    return st;
}

// 2^((p-1)/2) mod p^2 as canonical digits: left-to-right powering of 2, a
// squaring per exponent bit and a doubling where the bit is set
// (wieferich.cl:219-245), from 2^e0 for the top five bits e0 of the exponent.
template <class A>
WW_HD D2 wieferich_digits_t(u64 p, u64 q, D2 one) {
    const A ar(p, q);
    const u64 e = p >> 1;
    const int i0 = top_bit(e) - 5;
    const double rp = 1.0 / (double)p;
    D2 a = m2_small(1ull << (u32)(e >> (i0 + 1)), one, p, rp);
    u64 eb = e << (63 - i0);  // bit i of e at bit 63 in step i
    for (int i = i0; i >= 0; --i) {
        a = ar.sqr(a);
#if defined(WW_W_WINDOW)
        if (((i0 - i) & 3) == 3) a = m2_mul_pow2(a, (u32)(e >> i) & 15u, p, rp);
#else
        a = sel((long long)eb < 0, m2_dbl(a, p), a);
#endif
        eb <<= 1;
    }
#if defined(WW_W_WINDOW)
    const int rest = (i0 + 1) & 3;
    if (rest) a = m2_mul_pow2(a, (u32)e & ((1u << rest) - 1u), p, rp);
#endif
    return ar.redc(a);
}

// One step of the Lucas ladder kept as (e, o): for the pair of indices
// (k, k+1), e is V at the even one and o is V at the odd one up to sign.
// Since V_2m = V_m^2 - 2(-1)^m, x = e^2 - 2 and y = o^2 + 2 are V at twice
// the even and twice the odd index, whatever the parity of k, and their
// difference is V_2k+1 up to sign (y - x = +V_2k+1 for k even, -V_2k+1 for k
// odd), which the next squaring does not see.  The new pair is (2k, 2k+1)
// for bit 0 and (2k+1, 2k+2) for bit 1; its even index is 2k or 2k+2, so e
// becomes x or y by the bit and the parity of k.  Against a ladder on
// (V_k, V_k+1) this saves the selection of the constant -2(-1)^k and one of
// the two pair selections.  two and mtwo: 2 and -2 in Montgomery form.
template <class A>
WW_HD void eo_step(const A &ar, D2 &e, D2 &o, bool &kodd, bool bit, D2 two, D2 mtwo, u64 p) {
    const D2 x = m2_sub(ar.sqr(e), two, p);   // V_2k (k even) or V_2k+2 (k odd)
    const D2 y = m2_sub(ar.sqr(o), mtwo, p);  // the other of the two
    o = m2_sub(y, x, p);
    e = sel(bit != kodd, y, x);
    kodd = bit;
}

// 2 V_n+1 - V_n for the ladder's final (e, o) at k = n, n even (n = p +- 1):
// e = V_n, and o = y - x of the last step, from k = n/2, is +V_n+1 when n/2
// is even (bit 1 of n clear) and -V_n+1 when it is odd.
WW_HD D2 eo_finish(D2 e, D2 o, u64 n, u64 p) {
    const D2 zero = {0, 0};
    const D2 t = m2_dbl(o, p);
    return m2_sub(((n >> 1) & 1) ? m2_sub(zero, t, p) : t, e, p);
}

// F_{p-(p|5)} mod p^2 as canonical digits.  The reference walks the
// (F_k, F_{k-1}) doubling ladder, two squarings and a product per bit
// (wallsunsun.cl:242-300).  Here the Lucas numbers V_k = L_k run a ladder
// on (V_k, V_{k+1}) with two squarings per bit:
//   V_2k = V_k^2 - 2(-1)^k,  V_2k+2 = V_k+1^2 + 2(-1)^k,  V_2k+1 = V_2k+2 - V_2k,
// and F_n = (2 V_{n+1} - V_n) / 5 gives the same residue exactly (5 is a
// unit mod p^2 since p has no factor below 127).  The ladder starts from
// the top six bits of n (ladder_start) and keeps its pair as (V at the even
// index, V at the odd index up to sign), eo_step; -DWW_NO_EO_LADDER keeps
// (V_k, V_k+1) instead.
template <class A>
WW_HD D2 wss_digits_t(u64 p, u64 q, D2 one) {
    const A ar(p, q);
    const u32 pm5 = (u32)(p % 5);
    const u64 n = (pm5 == 2 || pm5 == 3) ? p + 1 : p - 1;  // p - (p|5)
    const D2 zero = {0, 0};
    const D2 two = m2_dbl(one, p);
    const D2 mtwo = m2_sub(zero, two, p);
    const int i0 = top_bit(n) - 6;
    const u32 k0 = (u32)(n >> (i0 + 1));
    const double rp = 1.0 / (double)p;
    const D2 a = m2_small(lucas_small(k0), one, p, rp);      // V_k0
    const D2 b = m2_small(lucas_small(k0 + 1), one, p, rp);  // V_k0+1
    bool odd = k0 & 1u;      // parity of the ladder index k
    u64 nb = n << (63 - i0);  // bit i of n at bit 63 in step i
#if !defined(WW_NO_EO_LADDER)
    D2 e = sel(odd, b, a), o = sel(odd, a, b);
    for (int i = i0; i >= 0; --i) {
        const bool bit = (long long)nb < 0;
        nb <<= 1;
        eo_step(ar, e, o, odd, bit, two, mtwo, p);
    }
    const D2 t = ar.redc(eo_finish(e, o, n, p));
#else
    D2 va = a, vb = b;
    for (int i = i0; i >= 0; --i) {
        const bool bit = (long long)nb < 0;
        nb <<= 1;
        const D2 c = sel(odd, two, mtwo);  // -2(-1)^k
        const D2 v2k = m2_add(ar.sqr(va), c, p);
        const D2 v2k2 = m2_sub(ar.sqr(vb), c, p);
        const D2 v2k1 = m2_sub(v2k2, v2k, p);
        va = sel(bit, v2k1, v2k);
        vb = sel(bit, v2k2, v2k1);
        odd = bit;
    }
    const D2 t = ar.redc(m2_sub(m2_dbl(vb, p), va, p));
#endif
    return m2_div5(t, p);
}

// Both tests in one loop: each iteration advances the Lucas ladder by one
// bit of p - (p|5) and the Wieferich powering by one bit of (p-1)/2.  The
// ladder step uses two squarings instead of a squaring and a product:
//   V_2k = V_k^2 - 2(-1)^k,  V_2k+2 = V_k+1^2 + 2(-1)^k,
//   V_2k+1 = V_2k+2 - V_2k   (the recurrence V_m+1 = V_m + V_m-1),
// so the three products of an iteration are squarings, independent of each
// other, and no operand has to be selected before multiplying.  Both start
// from their top bits (ladder_start), the Wieferich powering at most one
// bit after the ladder; the Lucas pair is kept as eo_step's (e, o).
template <class A>
WW_HD void both_digits_t(u64 p, u64 q, D2 one, D2 &s_out, D2 &c_out) {
    const A ar(p, q);
    const u32 pm5 = (u32)(p % 5);
    const u64 n = (pm5 == 2 || pm5 == 3) ? p + 1 : p - 1;
    const u64 e = p >> 1;
    const D2 zero = {0, 0};
    const D2 two = m2_dbl(one, p);
    const D2 mtwo = m2_sub(zero, two, p);
    const LadderStart st = ladder_start(p, n, one);
    D2 w = st.w;
    bool odd = st.odd;
    // bit i of n and of e at bit 63 in step i (shifts by one instead of by i)
    u64 nb = n << (63 - st.i0);
    u64 eb = e << (63 - st.i0);
#if !defined(WW_NO_EO_LADDER)
    D2 le = sel(odd, st.b, st.a), lo = sel(odd, st.a, st.b);
    for (int i = st.i0; i >= 0; --i) {
        const bool bit = (long long)nb < 0;
        const bool ebit = (long long)eb < 0;
        nb <<= 1;
        eb <<= 1;
        eo_step(ar, le, lo, odd, bit, two, mtwo, p);
        if (i <= st.iw) {
            w = ar.sqr(w);
#if defined(WW_W_WINDOW)
            if (((st.iw - i) & 3) == 3) w = m2_mul_pow2(w, (u32)(e >> i) & 15u, p, st.rp);
#else
            w = sel(ebit, m2_dbl(w, p), w);
#endif
        }
    }
#if defined(WW_W_WINDOW)
    const int rest = (st.iw + 1) & 3;
    if (rest) w = m2_mul_pow2(w, (u32)e & ((1u << rest) - 1u), p, st.rp);
#endif
    s_out = ar.redc(w);
    c_out = m2_div5(ar.redc(eo_finish(le, lo, n, p)), p);
#else
    D2 a = st.a, b = st.b;
    for (int i = st.i0; i >= 0; --i) {
        const bool bit = (long long)nb < 0;
        const bool ebit = (long long)eb < 0;
        nb <<= 1;
        eb <<= 1;
        const D2 a2 = ar.sqr(a);
        const D2 b2 = ar.sqr(b);
        if (i <= st.iw) {
            w = ar.sqr(w);
#if defined(WW_W_WINDOW)
            // every fourth bit from iw down: w *= 2^v for the group's four bits
            if (((st.iw - i) & 3) == 3) w = m2_mul_pow2(w, (u32)(e >> i) & 15u, p, st.rp);
#else
            w = sel(ebit, m2_dbl(w, p), w);
#endif
        }
        const D2 c = sel(odd, two, mtwo);     // -2(-1)^k
        const D2 v2k = m2_add(a2, c, p);      // V_2k
        const D2 v2k2 = m2_sub(b2, c, p);     // V_2k+2
        const D2 v2k1 = m2_sub(v2k2, v2k, p); // V_2k+1
        a = sel(bit, v2k1, v2k);
        b = sel(bit, v2k2, v2k1);
        odd = bit;
    }
#if defined(WW_W_WINDOW)
    const int rest = (st.iw + 1) & 3;  // the last, partial group of bits
    if (rest) w = m2_mul_pow2(w, (u32)e & ((1u << rest) - 1u), p, st.rp);
#endif
    s_out = ar.redc(w);
    c_out = m2_div5(ar.redc(m2_sub(m2_dbl(b, p), a, p)), p);
#endif
}

WW_HD D2 wieferich_digits(u64 p, u64 q, D2 one) { return wieferich_digits_t<WW_ARITH>(p, q, one); }
WW_HD void both_digits(u64 p, u64 q, D2 one, D2 &s, D2 &c) { both_digits_t<WW_ARITH>(p, q, one, s, c); }
WW_HD D2 wss_digits(u64 p, u64 q, D2 one) { return wss_digits_t<WW_ARITH>(p, q, one); }

// ------------------------------------------------------------ classification

constexpr u64 kThreshold = 1000;  // WW.h:8 SPECIAL_THRESHOLD

// wieferich.cl:248-293.  Returns true and fills rem/quot for a hit.
WW_HD bool wieferich_classify(u64 p, D2 s, int &rem, int &quot) {
    if (((s.d1 == 0) & (s.d0 == 1)) | ((s.d1 == p - 1) & (s.d0 == p - 1))) {
        rem = 1;
        quot = 0;
        return true;
    }
    if (s.d1 <= kThreshold) {
        if (s.d0 == 1) { rem = 1; quot = (int)s.d1; return true; }
        if (s.d0 == p - 1) { rem = -1; quot = (int)(s.d1 + 1); return true; }
        return false;
    }
    if (s.d1 >= p - kThreshold) {
        if (s.d0 == 1) { rem = 1; quot = (int)(s.d1 - p); return true; }
        if (s.d0 == p - 1) { rem = -1; quot = (int)(s.d1 + 1 - p); return true; }
    }
    return false;
}

// wallsunsun.cl:325-349.  result 1 = WSS prime, 2 = special instance.
WW_HD bool wss_classify(u64 p, D2 c, int &result, int &quot) {
    if (c.d1 == 0) { result = 1; quot = 0; return true; }
    if (c.d1 <= kThreshold) { result = 2; quot = (int)c.d1; return true; }
    if (c.d1 >= p - kThreshold) { result = 2; quot = (int)(c.d1 - p); return true; }
    return false;
}

}  // namespace ww
