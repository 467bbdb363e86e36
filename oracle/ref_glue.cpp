/*
 * ref_glue.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Thin C entry points around the reference's own CPU code, which is compiled
 * in place from the reference tree (wwcpu.cpp as its own translation unit,
 * prime.h included here) by oracle/Makefile into oracle/_ref/.  Nothing from
 * the reference is copied into this repository.
 *
 * main.cpp itself cannot be compiled without BOINC and OpenCL, so the two
 * pieces of it that the CPU path needs are restated here:
 *   isPRP            main.cpp:245-291 (trial division 3..113, then SPRP(2))
 *   the test loop    main.cpp:649-697 (odd numbers of [start, stop))
 * The loop is split over std::thread workers on contiguous sub-ranges; the
 * checksum is a sum, so the split does not change it.
 */
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "prime.h" /* montInit, strong_prp (reference) */
#include "WW.h"    /* wieferichCPU, wallsunsunCPU (reference, wwcpu.cpp) */

namespace {

int ref_isprp(uint64_t n) {
    static const uint32_t small[29] = {3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
                                       59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113};
    if (n % 2 == 0) return 0;
    for (uint32_t r : small)
        if (n % r == 0) return 0;
    uint64_t q, one, r2, nmo;
    montInit(n, &q, &one, &nmo, &r2);
    return strong_prp(2, n, q, one, nmo, r2);
}

struct Part {
    uint64_t prps = 0, cksm = 0, results = 0;
};

void scan(uint64_t lo, uint64_t hi, Part *out) {
    Part r;
    uint64_t n = lo;
    if (n % 2 == 0) ++n;
    for (; n < hi && n >= lo; n += 2) {
        if (ref_isprp(n)) {
            ++r.prps;
            if (wieferichCPU(n, r.cksm)) ++r.results;
            if (wallsunsunCPU(n, r.cksm)) ++r.results;
        }
        if (n > UINT64_MAX - 2) break;
    }
    *out = r;
}

void list(const uint64_t *p, uint64_t n, Part *out) {
    Part r;
    for (uint64_t i = 0; i < n; ++i) {
        ++r.prps;
        if (wieferichCPU(p[i], r.cksm)) ++r.results;
        if (wallsunsunCPU(p[i], r.cksm)) ++r.results;
    }
    *out = r;
}

}  // namespace

extern "C" {

int ref_wieferich(uint64_t p, uint64_t *cksm) { return wieferichCPU(p, *cksm); }
int ref_wallsunsun(uint64_t p, uint64_t *cksm) { return wallsunsunCPU(p, *cksm); }
int ref_is_prp(uint64_t n) { return ref_isprp(n); }

/* Per-prime low 32 bits of the two checksum terms (s1, c21), read back from
   the checksum deltas the reference functions add. */
void ref_list_terms(const uint64_t *p, uint64_t n, uint32_t *w_term, uint32_t *s_term, int32_t *w_hit,
                    int32_t *s_hit) {
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t a = 0, b = 0;
        w_hit[i] = wieferichCPU(p[i], a);
        s_hit[i] = wallsunsunCPU(p[i], b);
        w_term[i] = (uint32_t)a;
        s_term[i] = (uint32_t)b;
    }
}

/* The PRP list of [lo, hi) by the reference's test loop (single thread). */
uint64_t ref_prp_list(uint64_t lo, uint64_t hi, uint64_t *out, uint64_t cap) {
    uint64_t k = 0;
    uint64_t n = lo;
    if (n % 2 == 0) ++n;
    for (; n < hi && n >= lo; n += 2) {
        if (ref_isprp(n)) {
            if (k < cap) out[k] = n;
            ++k;
        }
        if (n > UINT64_MAX - 2) break;
    }
    return k;
}

int ref_scan_range(uint64_t lo, uint64_t hi, int nthreads, uint64_t *prps, uint64_t *cksm, uint64_t *results) {
    if (nthreads < 1) nthreads = 1;
    *prps = *cksm = *results = 0;
    if (hi <= lo) return 0;
    uint64_t width = hi - lo;
    if (width < (uint64_t)nthreads * 64) nthreads = 1;
    uint64_t step = (width / (uint64_t)nthreads) & ~(uint64_t)1;
    std::vector<Part> parts((size_t)nthreads);
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) {
        uint64_t a = lo + step * (uint64_t)i;
        uint64_t b = (i == nthreads - 1) ? hi : lo + step * (uint64_t)(i + 1);
        th.emplace_back(scan, a, b, &parts[(size_t)i]);
    }
    for (auto &t : th) t.join();
    for (auto &p : parts) {
        *prps += p.prps;
        *cksm += p.cksm;
        *results += p.results;
    }
    return 0;
}

int ref_test_list(const uint64_t *primes, uint64_t n, int nthreads, uint64_t *cksm, uint64_t *results) {
    if (nthreads < 1) nthreads = 1;
    if ((uint64_t)nthreads > n) nthreads = n ? (int)n : 1;
    *cksm = *results = 0;
    uint64_t per = n / (uint64_t)nthreads;
    std::vector<Part> parts((size_t)nthreads);
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) {
        uint64_t off = per * (uint64_t)i;
        uint64_t cnt = (i == nthreads - 1) ? n - off : per;
        th.emplace_back(list, primes + off, cnt, &parts[(size_t)i]);
    }
    for (auto &t : th) t.join();
    for (auto &p : parts) {
        *cksm += p.cksm;
        *results += p.results;
    }
    return 0;
}

}  // extern "C"
