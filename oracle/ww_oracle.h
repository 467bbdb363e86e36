/*
 * ww_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the WWocl search path (candidate filter -> base-2 strong
 * probable-prime test -> Wieferich test -> Wall-Sun-Sun test -> checksum and
 * hits).  It is the checker for the CUDA library: only the tests, the smoke
 * check and the CPU-baseline leg of the benchmark may load it.  The product
 * never links it.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths relative to the WWocl-boinc source tree).  Exact integer arithmetic
 * makes the canonical residues unique, so the mod p^2 arithmetic here is a
 * plain 128-bit Montgomery form (R = 2^128) rather than the reference's
 * two-digit form: an independent route to the same digits.
 */
#ifndef WW_ORACLE_H
#define WW_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Canonical digits of a residue v mod p^2: v = d0 + p * d1, 0 <= d0, d1 < p. */
typedef struct { uint64_t d0, d1; } wo_digits;

/* One hit as the reference kernels record it (wieferich.cl:248-293,
 * wallsunsun.cl:325-349): result 1093 = Wieferich, 1 = WSS prime,
 * 2 = WSS special instance. */
typedef struct { uint64_t p; int32_t result, rem, quot, pad; } wo_hit;

typedef struct {
    uint64_t prp_count;     /* numbers that passed the filter + SPRP(2)      */
    uint64_t checksum;      /* sum of (s1 mod 2^32) + (c21 mod 2^32)         */
    uint64_t cpu_results;   /* wieferichCPU + wallsunsunCPU return count      */
    uint64_t gpu_results;   /* hits recorded with the kernel classification   */
} wo_summary;

uint64_t wo_inv64(uint64_t p);
int      wo_small_factor(uint64_t n);
int      wo_sprp2(uint64_t n);
int      wo_is_prp(uint64_t n);
int      wo_is_prime(uint64_t n);

wo_digits wo_wieferich_digits(uint64_t p);
wo_digits wo_wss_digits(uint64_t p);

/* Classification; return 1 when the kernel would record a hit. */
int wo_wieferich_classify(uint64_t p, wo_digits s, wo_hit *out);
int wo_wss_classify(uint64_t p, wo_digits c, wo_hit *out);
/* wwcpu.cpp return-value semantics (counts only). */
int wo_wieferich_cpu_hit(uint64_t p, wo_digits s);
int wo_wss_cpu_hit(uint64_t p, wo_digits c);

/* Full per-prime test: adds both checksum terms, appends up to two hits.
 * Returns the number of hits appended. */
int wo_test_prime(uint64_t p, uint64_t *checksum, wo_hit *hits, uint64_t *cpu_results);

void wo_find_wheel_offset(uint64_t *start, int32_t *index);

/* Scan odd n in [lo, hi) like main.cpp:649-697.  prps/hits may be NULL; their
 * capacities bound what is written, the summary counts everything.
 * nthreads <= 1 runs on the calling thread. */
int wo_scan_range(uint64_t lo, uint64_t hi, int nthreads, wo_summary *sum,
                  uint64_t *prps, uint64_t prp_cap,
                  wo_hit *hits, uint64_t hit_cap);

/* W+WSS over an explicit list (checksum, counts, hits). */
int wo_test_list(const uint64_t *primes, uint64_t n, int nthreads, wo_summary *sum,
                 wo_hit *hits, uint64_t hit_cap);

/* Per-prime digits for a list (W digits into w, WSS digits into s). */
void wo_list_digits(const uint64_t *primes, uint64_t n, int nthreads,
                    wo_digits *w, wo_digits *s);

/* Sort hits by p (stable, Wieferich before WSS for equal p) and format the
 * lines the results file receives (main.cpp:843-916).  Returns bytes
 * written (excluding NUL), -1 on overflow of buf, -2 when a hit is
 * composite (the reference aborts).  *dropped receives the PRP-only count. */
int wo_format_results(wo_hit *hits, uint64_t n, char *buf, size_t cap, uint32_t *dropped);

/* main.cpp:1193-1262: START/END parsing with the e-notation branch.
 * Returns 0 on success, -1 on parse error, -2 on overflow. */
int wo_parse_number(const char *s, uint64_t *out);

/* Counter-based candidate stream for the fixed prime list workload:
 * SplitMix64 output i for the seed, kept when >= 2^62, forced odd. */
uint64_t wo_splitmix64(uint64_t seed, uint64_t i);
/* First n numbers of that stream that pass the deterministic MR test, in
 * stream order.  Returns how many stream positions were consumed. */
uint64_t wo_random_primes(uint64_t seed, uint64_t n, uint64_t *out, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
