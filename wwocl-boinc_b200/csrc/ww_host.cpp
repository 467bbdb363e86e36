// ww_host.cpp -- host-side helpers of the reference program (main.cpp)
// exported through the C ABI: wheel offset, primality checks of reported
// hits, START/END parsing, result-line formatting and PRP-buffer sizing.
#include <inttypes.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <vector>

#include "../../include/wwcuda.h"
#include "ww_tests.cuh"

using namespace ww;

namespace ww {
void set_err(const char *fmt, ...);  // ww_capi.cu
}

namespace {

bool sprp_base_host(u64 n, u64 base) {
    const u64 q = inv64(n);
    const u64 one = r_mod(n);
    u64 r2 = add_mod(one, one, n);
    r2 = add_mod(r2, r2, n);
    for (int i = 0; i < 5; ++i) r2 = mont_mul(r2, r2, n, q);  // (4R)^(2^5) = R^2
    const u64 nm1 = n - 1;
    const int t = __builtin_ctzll(nm1);
    const u64 d = nm1 >> t;
    const u64 mb = mont_mul(base % n, r2, n, q);
    u64 a = mb;
    for (int i = 62 - __builtin_clzll(d); i >= 0; --i) {
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

bool hit_before(const ww_hit &a, const ww_hit &b) {
    if (a.p != b.p) return a.p < b.p;
    return a.result == 1093 && b.result != 1093;  // the Wieferich kernel runs first
}

}  // namespace

extern "C" {

int ww_find_wheel_offset(uint64_t *start, int32_t *index) {
    if (!start || !index) return WW_ERR_ARG;
    // first n >= start prime to 30, and its position in the gap table
    // {4,2,4,2,4,6,2,6} that starts at residue 7 (main.cpp:528-587)
    static const int8_t pos_of[30] = {-1, 7, -1, -1, -1, -1, -1, 0, -1, -1, -1, 1, -1, 2, -1,
                                      -1, -1, 3, -1, 4, -1, -1, -1, 5, -1, -1, -1, -1, -1, 6};
    uint64_t n = *start;
    for (int k = 0; k < 7; ++k) {
        const int i = pos_of[n % 30];
        if (i >= 0) {
            *start = n;
            *index = i;
            return WW_OK;
        }
        if (n == UINT64_MAX) break;
        ++n;
    }
    set_err("no number >= %" PRIu64 " below 2^64 is prime to 30", *start);
    return WW_ERR_ARG;
}

int ww_is_prime(uint64_t n) {
    static const u64 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    if (n < 4) return 1;
    if ((n & 1) == 0) return 0;
    const int nb = n < 3825123056546413051ull ? 9 : 12;  // main.cpp:312-321
    for (int i = 0; i < nb; ++i) {
        if (n == bases[i]) return 1;
        if (n % bases[i] == 0) return 0;
    }
    for (int i = 0; i < nb; ++i)
        if (!sprp_base_host(n, bases[i])) return 0;
    return 1;
}

int ww_is_prp(uint64_t n) {
    static const uint32_t small[29] = {3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
                                       59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113};
    if ((n & 1) == 0) return 0;  // main.cpp:247-280
    for (uint32_t r : small)
        if (n % r == 0) return 0;
    return sprp_base_host(n, 2) ? 1 : 0;
}

int ww_parse_number(const char *s, uint64_t *out) {
    if (!s || !out) return WW_ERR_ARG;
    const char *e = strchr(s, 'e');
    if (e) {  // main.cpp:1194-1221: strtoull mantissa (base 0) times 10^exp
        char *end = nullptr;
        uint64_t num = strtoull(s, &end, 0);
        long exp = (end && *end) ? (long)strtoul(end + 1, nullptr, 0) : 0;
        if (num == 0 || exp == 0) return set_err("unable to parse '%s'", s), WW_ERR_ARG;
        for (long i = 0; i < exp; ++i) {
            if (num > UINT64_MAX / 10) return set_err("'%s' is out of range", s), WW_ERR_ARG;
            num *= 10;
        }
        *out = num;
        return WW_OK;
    }
    uint64_t v = 0;
    if (sscanf(s, "%" SCNu64, &v) != 1) return set_err("unable to parse '%s'", s), WW_ERR_ARG;
    *out = v;
    return WW_OK;
}

int ww_format_hits(ww_hit *hits, uint32_t n, char *buf, size_t cap, uint32_t *dropped) {
    if ((!hits && n) || !buf || cap == 0) return WW_ERR_ARG;
    std::stable_sort(hits, hits + n, hit_before);  // main.cpp:843-854
    size_t off = 0;
    uint32_t drop = 0;
    buf[0] = '\0';
    for (uint32_t i = 0; i < n; ++i) {
        const ww_hit &h = hits[i];
        char line[256];
        if (ww_is_prime(h.p)) {  // main.cpp:869-906
            if (h.result == 1093) {
                if (h.rem == 1 && h.quot == 0)
                    snprintf(line, sizeof line, "%" PRIu64 " is a Wieferich prime\n", h.p);
                else
                    snprintf(line, sizeof line, "%" PRIu64 " is a Wieferich special instance (%+d %+d p)\n", h.p,
                             h.rem, h.quot);
            } else if (h.result == 1) {
                snprintf(line, sizeof line, "%" PRIu64 " is a WallSunSun prime\n", h.p);
            } else if (h.result == 2) {
                snprintf(line, sizeof line, "%" PRIu64 " is a WallSunSun special instance (+0 %+d p)\n", h.p,
                         h.quot);
            } else {
                return WW_ERR_ARG;
            }
            const size_t len = strlen(line);
            if (off + len + 1 > cap) return WW_ERR_ARG;
            memcpy(buf + off, line, len + 1);
            off += len;
        } else if (ww_is_prp(h.p)) {
            ++drop;  // PRP-only hit (main.cpp:907-911)
        } else {
            set_err("computation error, composite result %" PRIu64, h.p);
            return WW_ERR_COMPOSITE;  // main.cpp:912-916
        }
    }
    if (dropped) *dropped = drop;
    return (int)off;
}

// Montgomery-Vaughan: pi(x+y) - pi(x) < 2y / ln y for y > 1, plus room for
// base-2 strong pseudoprimes (very rare, and counted past the buffer end by
// the kernels so an overflow is always detected).
uint64_t ww_prp_count_bound(uint64_t lo, uint64_t hi) {
    if (hi <= lo) return 0;
    const double y = (double)(hi - lo);
    if (y < 64) return (uint64_t)y;
    const double b = 2.0 * y / log(y);
    return (uint64_t)b + 1024;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Startup self-test twin (testKernels, main.cpp:590-738): the same exact
// arithmetic as the kernels, instantiated on the host, over a short range.
// Used only to cross-check the GPU at start-up; results are never taken
// from it.

extern "C" {

int ww_selftest_digits(const uint64_t *primes, uint64_t n, uint64_t *out) {
    if ((!primes || !out) && n) return WW_ERR_ARG;
    for (uint64_t i = 0; i < n; ++i) {
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
    return WW_OK;
}

int ww_selftest_range(uint64_t lo, uint64_t hi, uint64_t *prp_count, uint64_t *checksum,
                      uint32_t *result_count) {
    if (!prp_count || !checksum || !result_count) return WW_ERR_ARG;
    *prp_count = 0;
    *checksum = 0;
    *result_count = 0;
    if (hi <= lo) return WW_OK;
    uint64_t n = lo | 1;  // main.cpp:649-651
    for (; n < hi && n >= lo; n += 2) {
        bool small = false;
        for (uint32_t r : {3u, 5u, 7u, 11u, 13u, 17u, 19u, 23u, 29u, 31u, 37u, 41u, 43u, 47u, 53u,
                           59u, 61u, 67u, 71u, 73u, 79u, 83u, 89u, 97u, 101u, 103u, 107u, 109u, 113u})
            small |= (n % r == 0);
        u64 q = 0;
        if (small || !prp_test(n, q)) continue;  // the kernels' SPRP loop
        const D2 one = m2_one(n);
        const D2 s = wieferich_digits(n, q, one);
        const D2 c = wss_digits(n, q, one);
        ++*prp_count;
        *checksum += (s.d1 & 0xffffffffull) + (c.d1 & 0xffffffffull);
        int rem, quot, res;
        *result_count += wieferich_classify(n, s, rem, quot) ? 1u : 0u;
        *result_count += wss_classify(n, c, res, quot) ? 1u : 0u;
        if (n > UINT64_MAX - 2) break;
    }
    return WW_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Operation-level check of the two-digit arithmetic the kernels run (host
// instantiation of the same source): op 0 product, 1 square, 2 leave
// Montgomery form.  xy holds (x0, x1, y0, y1) per case, out (z0, z1).

namespace {
template <class A>
void m2_cases(int op, uint64_t p, const uint64_t *xy, uint64_t n, uint64_t *out) {
    const A ar(p, inv64(p));
    for (uint64_t i = 0; i < n; ++i) {
        const D2 x = {xy[4 * i], xy[4 * i + 1]};
        const D2 y = {xy[4 * i + 2], xy[4 * i + 3]};
        const D2 z = op == 0 ? ar.mul(x, y) : op == 1 ? ar.sqr(x) : ar.redc(x);
        out[2 * i] = z.d0;
        out[2 * i + 1] = z.d1;
    }
}
}  // namespace

// impl (op >> 4): 0 = the kernels' policy, 1 = 64-bit C, 2 = PTX chains, 3 = wide.
extern "C" int ww_selftest_m2(int op, uint64_t p, const uint64_t *xy, uint64_t n, uint64_t *out) {
    const int impl = op >> 4;
    op &= 15;
    if ((p & 1) == 0 || p < 3 || ((!xy || !out) && n) || op < 0 || op > 2 || impl > 3) return WW_ERR_ARG;
    switch (impl) {
        case 1: m2_cases<Arith64>(op, p, xy, n, out); break;
        case 2: m2_cases<Arith32>(op, p, xy, n, out); break;
        case 3: m2_cases<ArithWide>(op, p, xy, n, out); break;
        default: m2_cases<WW_ARITH>(op, p, xy, n, out); break;
    }
    return WW_OK;
}

// ---------------------------------------------------------------------------
// Host emulation of the kernels' candidate generation (small primes 3..113,
// then the deep sieve that spares multiples r*k with k = 1 (mod ord_r(2))),
// one segment over [lo, hi), for checking that the candidate set keeps every
// PRP.

#include "ww_deep.cuh"

namespace {
#define WW_DEEP_ROWH(r, o, rinv, mr, mo) {r, o, rinv, mr, mo},
const DeepRow kDeepHost[WW_DEEP_COUNT] = {WW_DEEP_ROWS(WW_DEEP_ROWH)};
#undef WW_DEEP_ROWH
}  // namespace

extern "C" int ww_selftest_candidates(uint64_t lo, uint64_t hi, uint64_t *out, uint64_t cap, uint64_t *n,
                                      uint64_t *spared_out) {
    if (!n || (!out && cap) || hi <= lo || lo < 127 || hi - lo > (1ull << 32)) return WW_ERR_ARG;
    const u64 b0 = lo & ~1ull, first = b0 + 1;
    const u64 nvalid = (hi - b0) / 2;
    std::vector<u32> bitmap((nvalid + 31) / 32, 0);
    auto mark = [&](u64 j) { bitmap[j >> 5] |= 1u << (j & 31); };
    static const u32 small[29] = {3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
                                  59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113};
    for (u32 r : small)
        for (u64 j = deep_first_multiple(first, r, (u32)((1ull << 32) % r)); j < nvalid; j += r) mark(j);
    u64 spared = 0;  // multiples of deep primes left unmarked (k = 1 mod o)
    for (int i = 0; i < kDeepUse; ++i) {
        const DeepRow &e = kDeepHost[i];
        u32 j0, km;
        deep_start(first, e, j0, km);
        for (u64 j = j0; j < nvalid; j += e.r) {
            if (km != 1u) mark(j);
            else ++spared;
            km += 2u;
            if (km >= e.o) km -= e.o;
        }
    }
    std::vector<u64> cand;
    for (u64 j = 0; j < nvalid; ++j)
        if (!((bitmap[j >> 5] >> (j & 31)) & 1u)) cand.push_back(first + 2 * j);
    *n = cand.size();
    if (spared_out) *spared_out = spared;
    for (u64 i = 0; i < cap && i < cand.size(); ++i) out[i] = cand[i];
    return WW_OK;
}

// ---------------------------------------------------------------------------
// Checkpoint files (main.cpp:103-209).

namespace {

bool read_state_file(const char *name, uint64_t start, uint64_t stop, ww_state &st) {
    FILE *in = fopen(name, "r");
    if (!in) return false;
    uint64_t a = 0, b = 0;
    ww_state t{};
    const int n = fscanf(in, "%" SCNu64 " %" SCNu64 " %" SCNu64 " %" SCNu64 " %lf %d", &a, &b, &t.current, &t.cksm,
                         &t.psum, &t.pcnt);
    fclose(in);
    if (n != 6) {
        fprintf(stderr, "Cannot parse %s !!!\n", name);
        return false;
    }
    if (a != start || b != stop) return false;  // main.cpp:157,173
    if (t.current < start || t.current > stop) return false;
    st = t;
    return true;
}

}  // namespace

extern "C" int ww_state_write(const char *file_a, const char *file_b, uint64_t start, uint64_t stop,
                              const ww_state *st, int *write_a_next) {
    if (!file_a || !file_b || !st || !write_a_next) return WW_ERR_ARG;
    const char *name = *write_a_next ? file_a : file_b;
    FILE *out = fopen(name, "w");
    if (!out) {
        set_err("cannot open %s", name);
        return WW_ERR_ARG;
    }
    if (fprintf(out, "%" PRIu64 " %" PRIu64 " %" PRIu64 " %" PRIu64 " %lf %d\n", start, stop, st->current, st->cksm,
                st->psum, st->pcnt) < 0) {
        fclose(out);
        set_err("cannot write %s", name);
        return WW_ERR_ARG;
    }
    fflush(out);
    fsync(fileno(out));
    if (fclose(out) == 0) *write_a_next = !*write_a_next;  // main.cpp:124-129
    return WW_OK;
}

extern "C" int ww_state_read(const char *file_a, const char *file_b, uint64_t start, uint64_t stop, ww_state *st,
                             int *write_a_next) {
    if (!file_a || !file_b || !st || !write_a_next) return WW_ERR_ARG;
    ww_state a{}, b{};
    bool ga = read_state_file(file_a, start, stop, a);
    bool gb = read_state_file(file_b, start, stop, b);
    if (ga && gb) {  // main.cpp:179-185
        if (a.current > b.current) gb = false;
        else ga = false;
    }
    if (ga) {
        *st = a;
        *write_a_next = 0;
        return 1;
    }
    if (gb) {
        *st = b;
        *write_a_next = 1;
        return 1;
    }
    return 0;
}
