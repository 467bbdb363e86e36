/*
 * ww_oracle.c -- TEST INFRASTRUCTURE ONLY (see ww_oracle.h).
 *
 * CPU restatement of the WWocl search path, used as the parity checker of the
 * CUDA library.  Citations are reference file:line (WWocl-boinc tree).
 *
 * Arithmetic choices (all exact, so the digits are unique):
 *   mod n   : 64-bit Montgomery, R = 2^64, unsigned __int128 products.
 *   mod p^2 : 128-bit Montgomery, R = 2^128, two 64-bit limbs.  The
 *             reference's kernels use a two-digit x0 + p*x1 form instead;
 *             both give the same canonical residue.
 */
#include "ww_oracle.h"

#include <inttypes.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

#define WO_THRESHOLD 1000u /* WW.h:8 SPECIAL_THRESHOLD */

static const uint32_t kSmallPrimes[29] = {3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
                                          59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113};

/* ------------------------------------------------------------------ mod n */

/* p^-1 mod 2^64 by Newton iteration (prime.h:7-12, wwcpu.cpp:65-70). */
uint64_t wo_inv64(uint64_t p) {
    uint64_t x = p; /* correct to 3 bits for odd p */
    for (int i = 0; i < 5; ++i) x *= 2 - p * x;
    return x;
}

/* a*b*2^-64 mod n, a,b < n; q = n^-1 mod 2^64 (prime.h:15-30). */
static inline uint64_t mont64(uint64_t a, uint64_t b, uint64_t n, uint64_t q) {
    u128 t = (u128)a * b;
    uint64_t lo = (uint64_t)t, hi = (uint64_t)(t >> 64);
    uint64_t m = lo * q;
    uint64_t mh = (uint64_t)(((u128)m * n) >> 64);
    return hi >= mh ? hi - mh : hi - mh + n;
}

static inline uint64_t addmod64(uint64_t a, uint64_t b, uint64_t n) {
    return (a >= n - b) ? a + b - n : a + b; /* prime.h:33-43 */
}

/* Strong probable-prime test to base `base` (prime.h:65-114). */
static int sprp_base(uint64_t n, uint64_t base) {
    uint64_t q = wo_inv64(n);
    uint64_t one = (0 - n) % n; /* 2^64 mod n */
    uint64_t mone = n - one;
    /* 2^128 mod n: square 2^64 twice-over via four doublings then squarings,
       as montInit does (prime.h:46-59): 4 = 2^2 in Montgomery form, ^(2^5). */
    uint64_t r2 = addmod64(one, one, n);
    r2 = addmod64(r2, r2, n);
    for (int i = 0; i < 5; ++i) r2 = mont64(r2, r2, n, q);
    uint64_t nm1 = n - 1;
    int t = __builtin_ctzll(nm1);
    uint64_t d = nm1 >> t;
    uint64_t mb = mont64(base % n, r2, n, q);
    uint64_t a = mb;
    for (int bit = 62 - __builtin_clzll(d); bit >= 0; --bit) {
        a = mont64(a, a, n, q);
        if ((d >> bit) & 1) a = mont64(a, mb, n, q);
    }
    if (a == one || a == mone) return 1;
    for (int s = 1; s < t; ++s) {
        a = mont64(a, a, n, q);
        if (a == mone) return 1;
    }
    return 0;
}

int wo_sprp2(uint64_t n) { return sprp_base(n, 2); }

/* Trial division by 2 and the odd primes 3..113 (main.cpp:247-280). */
int wo_small_factor(uint64_t n) {
    if ((n & 1) == 0) return 1;
    for (int i = 0; i < 29; ++i)
        if (n % kSmallPrimes[i] == 0) return 1;
    return 0;
}

/* isPRP (main.cpp:245-291). */
int wo_is_prp(uint64_t n) { return !wo_small_factor(n) && wo_sprp2(n); }

/* isPrime (main.cpp:301-324): deterministic Miller-Rabin, 9 or 12 bases. */
int wo_is_prime(uint64_t n) {
    static const uint64_t bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if ((n & 1) == 0) return 0;
    int nb = (n < 3825123056546413051ULL) ? 9 : 12;
    for (int i = 0; i < nb; ++i)
        if (!sprp_base(n, bases[i])) return 0;
    return 1;
}

/* -------------------------------------------------------------- mod p^2 */

typedef struct {
    u128 N;        /* p^2 */
    uint64_t ninv; /* -N^-1 mod 2^64 */
    u128 one;      /* 2^128 mod N (Montgomery form of 1) */
} modsq;

static void modsq_init(modsq *m, uint64_t p) {
    m->N = (u128)p * p;
    m->ninv = 0 - wo_inv64((uint64_t)m->N);
    m->one = ((u128)0 - m->N) % m->N; /* (2^128 - N) mod N = 2^128 mod N */
}

static inline u128 modsq_add(const modsq *m, u128 a, u128 b) {
    u128 s = a + b;
    if (s < a || s >= m->N) s -= m->N; /* wraps correctly when the add carried */
    return s;
}

static inline u128 modsq_sub(const modsq *m, u128 a, u128 b) {
    return a >= b ? a - b : a - b + m->N;
}

/* a*b*2^-128 mod N with two 64-bit limbs (schoolbook + 2-step REDC). */
static u128 modsq_mul(const modsq *m, u128 a, u128 b) {
    uint64_t a0 = (uint64_t)a, a1 = (uint64_t)(a >> 64);
    uint64_t b0 = (uint64_t)b, b1 = (uint64_t)(b >> 64);
    uint64_t n0 = (uint64_t)m->N, n1 = (uint64_t)(m->N >> 64);
    uint64_t t[5] = {0, 0, 0, 0, 0};
    /* t = a*b */
    u128 c;
    c = (u128)a0 * b0;
    t[0] = (uint64_t)c;
    c = (c >> 64) + (u128)a0 * b1;
    t[1] = (uint64_t)c;
    t[2] = (uint64_t)(c >> 64);
    c = (u128)a1 * b0 + t[1];
    t[1] = (uint64_t)c;
    c = (c >> 64) + (u128)a1 * b1 + t[2];
    t[2] = (uint64_t)c;
    t[3] = (uint64_t)(c >> 64);
    /* two reduction steps */
    for (int i = 0; i < 2; ++i) {
        uint64_t q = t[i] * m->ninv;
        c = (u128)q * n0 + t[i];
        c = (c >> 64) + (u128)q * n1 + t[i + 1];
        t[i + 1] = (uint64_t)c;
        c = (c >> 64) + t[i + 2];
        t[i + 2] = (uint64_t)c;
        for (int k = i + 3; k < 5 && (c >> 64); ++k) {
            c = (c >> 64) + t[k];
            t[k] = (uint64_t)c;
        }
    }
    u128 r = ((u128)t[3] << 64) | t[2];
    if (t[4] || r >= m->N) r -= m->N;
    return r;
}

static inline wo_digits modsq_digits(const modsq *m, uint64_t p, u128 xm) {
    u128 v = modsq_mul(m, xm, 1); /* leave Montgomery form */
    wo_digits d;
    d.d0 = (uint64_t)(v % p);
    d.d1 = (uint64_t)(v / p);
    return d;
}

/* 2^((p-1)/2) mod p^2 by left-to-right binary powering of 2
   (wieferich.cl:219-245, wwcpu.cpp:258-284). */
wo_digits wo_wieferich_digits(uint64_t p) {
    modsq m;
    modsq_init(&m, p);
    uint64_t e = p >> 1;
    u128 a = modsq_add(&m, m.one, m.one); /* 2 */
    for (int bit = 62 - __builtin_clzll(e); bit >= 0; --bit) {
        a = modsq_mul(&m, a, a);
        if ((e >> bit) & 1) a = modsq_add(&m, a, a);
    }
    return modsq_digits(&m, p, a);
}

/* F_{p-(p|5)} mod p^2 by the (F_n, F_{n-1}) doubling ladder
   (wallsunsun.cl:242-300, wwcpu.cpp:311-372). */
wo_digits wo_wss_digits(uint64_t p) {
    modsq m;
    modsq_init(&m, p);
    int pm5 = (int)(p % 5);
    int kro = (pm5 == 2 || pm5 == 3) ? -1 : 1;
    uint64_t e = p - (uint64_t)(int64_t)kro - 1;
    u128 b = m.one, c = 0; /* F_1, F_0 */
    for (int bit = 62 - __builtin_clzll(e); bit >= 0; --bit) {
        u128 b2 = modsq_mul(&m, b, b);
        u128 c2 = modsq_mul(&m, c, c);
        u128 a = modsq_add(&m, b, c);
        b = modsq_mul(&m, b, modsq_add(&m, a, c)); /* F_2n = F_n (F_n+1 + F_n-1) */
        c = modsq_add(&m, b2, c2);                 /* F_2n-1 = F_n^2 + F_n-1^2 */
        if ((e >> bit) & 1) {
            u128 t = modsq_add(&m, b, c);
            c = b;
            b = t;
        }
    }
    return modsq_digits(&m, p, modsq_add(&m, b, c)); /* F_{e+1} */
}

/* ----------------------------------------------------------- classification */

/* wieferich.cl:248-293 */
int wo_wieferich_classify(uint64_t p, wo_digits s, wo_hit *out) {
    int rem = 0, quot = 0, hit = 0;
    if ((s.d1 == 0 && s.d0 == 1) || (s.d1 == p - 1 && s.d0 == p - 1)) {
        hit = 1; rem = 1; quot = 0;
    } else if (s.d1 <= WO_THRESHOLD) {
        if (s.d0 == 1) { hit = 1; rem = 1; quot = (int32_t)s.d1; }
        else if (s.d0 == p - 1) { hit = 1; rem = -1; quot = (int32_t)(s.d1 + 1); }
    } else if (s.d1 >= p - WO_THRESHOLD) {
        if (s.d0 == 1) { hit = 1; rem = 1; quot = (int32_t)(s.d1 - p); }
        else if (s.d0 == p - 1) { hit = 1; rem = -1; quot = (int32_t)(s.d1 + 1 - p); }
    }
    if (hit && out) { out->p = p; out->result = 1093; out->rem = rem; out->quot = quot; out->pad = 0; }
    return hit;
}

/* wallsunsun.cl:325-349 */
int wo_wss_classify(uint64_t p, wo_digits c, wo_hit *out) {
    int hit = 0, result = 0, quot = 0;
    if (c.d1 == 0) { hit = 1; result = 1; quot = 0; }
    else if (c.d1 <= WO_THRESHOLD) { hit = 1; result = 2; quot = (int32_t)c.d1; }
    else if (c.d1 >= p - WO_THRESHOLD) { hit = 1; result = 2; quot = (int32_t)(c.d1 - p); }
    if (hit && out) { out->p = p; out->result = result; out->rem = 0; out->quot = quot; out->pad = 0; }
    return hit;
}

/* wwcpu.cpp:290-303 */
int wo_wieferich_cpu_hit(uint64_t p, wo_digits s) {
    return ((s.d1 == 0 && s.d0 == 1) || (s.d1 == p - 1 && s.d0 == p - 1)) ||
           s.d1 <= WO_THRESHOLD || s.d1 >= p - WO_THRESHOLD;
}

/* wwcpu.cpp:382-395 */
int wo_wss_cpu_hit(uint64_t p, wo_digits c) {
    return c.d1 == 0 || c.d1 <= WO_THRESHOLD || c.d1 >= p - WO_THRESHOLD;
}

int wo_test_prime(uint64_t p, uint64_t *checksum, wo_hit *hits, uint64_t *cpu_results) {
    wo_digits s = wo_wieferich_digits(p);
    wo_digits c = wo_wss_digits(p);
    *checksum += (s.d1 & 0xffffffffu) + (c.d1 & 0xffffffffu); /* wieferich.cl:315, wallsunsun.cl:352 */
    if (cpu_results) *cpu_results += (uint64_t)wo_wieferich_cpu_hit(p, s) + (uint64_t)wo_wss_cpu_hit(p, c);
    int n = 0;
    n += wo_wieferich_classify(p, s, hits ? &hits[n] : NULL);
    n += wo_wss_classify(p, c, hits ? &hits[n] : NULL);
    return n;
}

/* ------------------------------------------------------------------ wheel */

/* findWheelOffset (main.cpp:528-587): first n >= start prime to 30 and the
   index of n mod 30 in the gap table {4,2,4,2,4,6,2,6}, which starts at
   residue 7.  Restated by walking the mod 6 wheel as the reference does. */
void wo_find_wheel_offset(uint64_t *start, int32_t *index) {
    static const int32_t wheel[8] = {4, 2, 4, 2, 4, 6, 2, 6};
    uint64_t s = *start;
    uint64_t n = (s / 6) * 6 - 1;
    int plus2 = 1;
    while (n < s || n % 5 == 0) {
        n += plus2 ? 2 : 4;
        plus2 = !plus2;
    }
    uint64_t first = n;
    int32_t idx = -1;
    while (idx < 0) {
        if (plus2) {
            n += 2; plus2 = 0;
            if (n % 5 == 0) { n -= 2; idx = 5; }
        } else {
            n += 4; plus2 = 1;
            if (n % 5 == 0) { n -= 4; idx = 7; }
        }
    }
    while (n != first) {
        if (--idx < 0) idx = 7;
        n -= (uint64_t)wheel[idx];
    }
    *start = first;
    *index = idx;
}

/* ------------------------------------------------------------- range scan */

typedef struct {
    uint64_t lo, hi;
    wo_summary sum;
    uint64_t *prps; uint64_t prp_cap, prp_n;
    wo_hit *hits; uint64_t hit_cap, hit_n;
    const uint64_t *list; uint64_t list_n;
    wo_digits *wd, *sd;
} scan_job;

static void scan_one(scan_job *j, uint64_t n) {
    j->sum.prp_count++;
    if (j->prps) {
        if (j->prp_n < j->prp_cap) j->prps[j->prp_n] = n;
        j->prp_n++;
    }
    wo_hit h[2];
    int k = wo_test_prime(n, &j->sum.checksum, h, &j->sum.cpu_results);
    j->sum.gpu_results += (uint64_t)k;
    for (int i = 0; i < k; ++i) {
        if (j->hits && j->hit_n < j->hit_cap) j->hits[j->hit_n] = h[i];
        j->hit_n++;
    }
}

/* main.cpp:649-697: odd numbers, trial division 3..113, then SPRP(2). */
static void *scan_worker(void *arg) {
    scan_job *j = (scan_job *)arg;
    if (j->lo >= j->hi) return NULL;
    uint64_t n = j->lo | 1;
    while (n < j->hi && n >= j->lo) {
        if (!wo_small_factor(n) && wo_sprp2(n)) scan_one(j, n);
        if (n > UINT64_MAX - 2) break;
        n += 2;
    }
    return NULL;
}

static void *list_worker(void *arg) {
    scan_job *j = (scan_job *)arg;
    for (uint64_t i = 0; i < j->list_n; ++i) {
        if (j->wd) {
            j->wd[i] = wo_wieferich_digits(j->list[i]);
            j->sd[i] = wo_wss_digits(j->list[i]);
        } else {
            wo_hit h[2];
            int k = wo_test_prime(j->list[i], &j->sum.checksum, h, &j->sum.cpu_results);
            j->sum.prp_count++;
            j->sum.gpu_results += (uint64_t)k;
            for (int t = 0; t < k; ++t) {
                if (j->hits && j->hit_n < j->hit_cap) j->hits[j->hit_n] = h[t];
                j->hit_n++;
            }
        }
    }
    return NULL;
}

static int run_jobs(scan_job *jobs, int nt, void *(*fn)(void *)) {
    if (nt <= 1) {
        fn(&jobs[0]);
        return 0;
    }
    pthread_t *th = (pthread_t *)calloc((size_t)nt, sizeof(pthread_t));
    if (!th) return -1;
    for (int i = 0; i < nt; ++i) pthread_create(&th[i], NULL, fn, &jobs[i]);
    for (int i = 0; i < nt; ++i) pthread_join(th[i], NULL);
    free(th);
    return 0;
}

static void merge_jobs(scan_job *jobs, int nt, wo_summary *sum, uint64_t *prps, uint64_t prp_cap,
                       wo_hit *hits, uint64_t hit_cap) {
    memset(sum, 0, sizeof(*sum));
    uint64_t pn = 0, hn = 0;
    for (int i = 0; i < nt; ++i) {
        sum->prp_count += jobs[i].sum.prp_count;
        sum->checksum += jobs[i].sum.checksum;
        sum->cpu_results += jobs[i].sum.cpu_results;
        sum->gpu_results += jobs[i].sum.gpu_results;
        if (prps) {
            uint64_t k = jobs[i].prp_n < jobs[i].prp_cap ? jobs[i].prp_n : jobs[i].prp_cap;
            for (uint64_t t = 0; t < k && pn < prp_cap; ++t) prps[pn++] = jobs[i].prps[t];
        }
        if (hits) {
            uint64_t k = jobs[i].hit_n < jobs[i].hit_cap ? jobs[i].hit_n : jobs[i].hit_cap;
            for (uint64_t t = 0; t < k && hn < hit_cap; ++t) hits[hn++] = jobs[i].hits[t];
        }
    }
}

int wo_scan_range(uint64_t lo, uint64_t hi, int nthreads, wo_summary *sum, uint64_t *prps,
                  uint64_t prp_cap, wo_hit *hits, uint64_t hit_cap) {
    if (nthreads < 1) nthreads = 1;
    if (hi <= lo) {
        memset(sum, 0, sizeof(*sum));
        return 0;
    }
    uint64_t width = hi - lo;
    if (width < (uint64_t)nthreads * 64) nthreads = 1;
    scan_job *jobs = (scan_job *)calloc((size_t)nthreads, sizeof(scan_job));
    if (!jobs) return -1;
    uint64_t step = (width / (uint64_t)nthreads) & ~(uint64_t)1;
    for (int i = 0; i < nthreads; ++i) {
        jobs[i].lo = lo + step * (uint64_t)i;
        jobs[i].hi = (i == nthreads - 1) ? hi : lo + step * (uint64_t)(i + 1);
        if (prps) {
            jobs[i].prp_cap = prp_cap;
            jobs[i].prps = (uint64_t *)malloc(prp_cap * sizeof(uint64_t) + 8);
        }
        if (hits) {
            jobs[i].hit_cap = hit_cap;
            jobs[i].hits = (wo_hit *)malloc(hit_cap * sizeof(wo_hit) + sizeof(wo_hit));
        }
    }
    /* each sub-range must start on the same parity as the reference loop (odd) */
    run_jobs(jobs, nthreads, scan_worker);
    merge_jobs(jobs, nthreads, sum, prps, prp_cap, hits, hit_cap);
    for (int i = 0; i < nthreads; ++i) {
        free(jobs[i].prps);
        free(jobs[i].hits);
    }
    free(jobs);
    return 0;
}

int wo_test_list(const uint64_t *primes, uint64_t n, int nthreads, wo_summary *sum, wo_hit *hits,
                 uint64_t hit_cap) {
    if (nthreads < 1) nthreads = 1;
    if ((uint64_t)nthreads > n) nthreads = n ? (int)n : 1;
    scan_job *jobs = (scan_job *)calloc((size_t)nthreads, sizeof(scan_job));
    if (!jobs) return -1;
    uint64_t per = n / (uint64_t)nthreads;
    for (int i = 0; i < nthreads; ++i) {
        jobs[i].list = primes + per * (uint64_t)i;
        jobs[i].list_n = (i == nthreads - 1) ? n - per * (uint64_t)i : per;
        if (hits) {
            jobs[i].hit_cap = hit_cap;
            jobs[i].hits = (wo_hit *)malloc(hit_cap * sizeof(wo_hit) + sizeof(wo_hit));
        }
    }
    run_jobs(jobs, nthreads, list_worker);
    merge_jobs(jobs, nthreads, sum, NULL, 0, hits, hit_cap);
    for (int i = 0; i < nthreads; ++i) free(jobs[i].hits);
    free(jobs);
    return 0;
}

void wo_list_digits(const uint64_t *primes, uint64_t n, int nthreads, wo_digits *w, wo_digits *s) {
    if (nthreads < 1) nthreads = 1;
    if ((uint64_t)nthreads > n) nthreads = n ? (int)n : 1;
    scan_job *jobs = (scan_job *)calloc((size_t)nthreads, sizeof(scan_job));
    if (!jobs) return;
    uint64_t per = n / (uint64_t)nthreads;
    for (int i = 0; i < nthreads; ++i) {
        uint64_t off = per * (uint64_t)i;
        jobs[i].list = primes + off;
        jobs[i].list_n = (i == nthreads - 1) ? n - off : per;
        jobs[i].wd = w + off;
        jobs[i].sd = s + off;
    }
    run_jobs(jobs, nthreads, list_worker);
    free(jobs);
}

/* ---------------------------------------------------------------- results */

static int hit_less(const wo_hit *a, const wo_hit *b) {
    if (a->p != b->p) return a->p < b->p;
    return (a->result == 1093) && (b->result != 1093);
}

/* getResults (main.cpp:843-916): sort by p, keep prime hits, drop PRP-only
   hits, refuse composites; the line formats of main.cpp:873-901. */
int wo_format_results(wo_hit *hits, uint64_t n, char *buf, size_t cap, uint32_t *dropped) {
    /* insertion sort: stable, fine for the few hits a range produces */
    for (uint64_t i = 1; i < n; ++i) {
        wo_hit h = hits[i];
        uint64_t j = i;
        while (j > 0 && hit_less(&h, &hits[j - 1])) {
            hits[j] = hits[j - 1];
            --j;
        }
        hits[j] = h;
    }
    size_t off = 0;
    uint32_t drop = 0;
    if (cap) buf[0] = '\0';
    for (uint64_t i = 0; i < n; ++i) {
        char line[256];
        const wo_hit *h = &hits[i];
        if (wo_is_prime(h->p)) {
            if (h->result == 1093) {
                if (h->rem == 1 && h->quot == 0)
                    snprintf(line, sizeof line, "%" PRIu64 " is a Wieferich prime\n", h->p);
                else
                    snprintf(line, sizeof line, "%" PRIu64 " is a Wieferich special instance (%+d %+d p)\n",
                             h->p, h->rem, h->quot);
            } else if (h->result == 1) {
                snprintf(line, sizeof line, "%" PRIu64 " is a WallSunSun prime\n", h->p);
            } else if (h->result == 2) {
                snprintf(line, sizeof line, "%" PRIu64 " is a WallSunSun special instance (+0 %+d p)\n", h->p,
                         h->quot);
            } else {
                return -2;
            }
            size_t len = strlen(line);
            if (off + len + 1 > cap) return -1;
            memcpy(buf + off, line, len + 1);
            off += len;
        } else if (wo_is_prp(h->p)) {
            ++drop;
        } else {
            return -2;
        }
    }
    if (dropped) *dropped = drop;
    return (int)off;
}

/* ---------------------------------------------------------------- parsing */

/* main.cpp:1193-1226: a string containing 'e' is mantissa (strtoull base 0)
   times 10^exp with an overflow check; anything else is %llu. */
int wo_parse_number(const char *s, uint64_t *out) {
    const char *e = strchr(s, 'e');
    if (e) {
        char *end = NULL;
        uint64_t num = strtoull(s, &end, 0);
        long exp = (long)strtoul(end + 1, NULL, 0);
        if (num == 0 || exp == 0) return -1;
        for (long i = 0; i < exp; ++i) {
            if (num > UINT64_MAX / 10) return -2;
            num *= 10;
        }
        *out = num;
        return 0;
    }
    uint64_t v = 0;
    if (sscanf(s, "%" SCNu64, &v) != 1) v = 0; /* the reference leaves it unset */
    *out = v;
    return 0;
}

/* ------------------------------------------------------ fixed prime list */

uint64_t wo_splitmix64(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

typedef struct {
    uint64_t seed, i0, i1;
    uint64_t *buf, *pos;
    uint64_t n;
} gen_job;

static void *gen_worker(void *arg) {
    gen_job *g = (gen_job *)arg;
    g->n = 0;
    for (uint64_t i = g->i0; i < g->i1; ++i) {
        uint64_t c = wo_splitmix64(g->seed, i) | 1;
        if (c < (1ULL << 62)) continue;
        if (wo_small_factor(c) || !wo_is_prime(c)) continue;
        g->buf[g->n] = c;
        g->pos[g->n] = i;
        g->n++;
    }
    return NULL;
}

uint64_t wo_random_primes(uint64_t seed, uint64_t n, uint64_t *out, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    const uint64_t chunk = 1ULL << 16; /* positions per thread per round */
    gen_job *jobs = (gen_job *)calloc((size_t)nthreads, sizeof(gen_job));
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    for (int t = 0; t < nthreads; ++t) {
        jobs[t].buf = (uint64_t *)malloc(chunk * sizeof(uint64_t));
        jobs[t].pos = (uint64_t *)malloc(chunk * sizeof(uint64_t));
        jobs[t].seed = seed;
    }
    uint64_t have = 0, next = 0, consumed = 0;
    while (have < n) {
        for (int t = 0; t < nthreads; ++t) {
            jobs[t].i0 = next + chunk * (uint64_t)t;
            jobs[t].i1 = jobs[t].i0 + chunk;
        }
        if (nthreads == 1) gen_worker(&jobs[0]);
        else {
            for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, gen_worker, &jobs[t]);
            for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
        }
        for (int t = 0; t < nthreads && have < n; ++t)
            for (uint64_t k = 0; k < jobs[t].n && have < n; ++k) {
                out[have++] = jobs[t].buf[k];
                consumed = jobs[t].pos[k] + 1;
            }
        next += chunk * (uint64_t)nthreads;
    }
    for (int t = 0; t < nthreads; ++t) {
        free(jobs[t].buf);
        free(jobs[t].pos);
    }
    free(jobs);
    free(th);
    return consumed;
}
