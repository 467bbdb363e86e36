/*
 * wwcuda.h -- C ABI of libwwcuda.so, the B200 (sm_100a) implementation of the
 * WWocl search path: segmented wheel sieve + base-2 strong PRP test,
 * Wieferich test 2^((p-1)/2) mod p^2 and Wall-Sun-Sun test F_{p-(p|5)} mod p^2,
 * with the reference's checksum and hit records.
 *
 * It replaces the reference's device layer (simpleCL.h:63-140 / simpleCL.c)
 * and its five OpenCL kernels.  Two levels:
 *
 *  1. Kernel-shaped entry points (ww_launch_*) that take the same arguments
 *     as the reference kernels, as plain device pointers plus the buffer
 *     capacities the reference left implicit and a cudaStream_t passed as
 *     void*.  They allocate nothing and never synchronise.
 *  2. A context (ww_ctx) that owns the stream, the device buffers and the
 *     pinned read-back area -- the reference's progData (main.cpp:51-66)
 *     plus its sclRead/sclFinish calls -- used by the wwocl host program.
 *
 * Conventions: every function returns an int status (WW_OK = 0, negative on
 * error, see WW_ERR_*); ww_last_error() gives a message for the calling
 * thread.  No function calls exit().  One host thread per ww_ctx.  All
 * context calls are ordered on the context's stream.
 */
#ifndef WWCUDA_H
#define WWCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WW_ABI_VERSION 1

/* status codes */
#define WW_OK 0
#define WW_ERR_CUDA (-1)          /* a CUDA runtime call failed             */
#define WW_ERR_ARG (-2)           /* bad argument (range, size, pointer)    */
#define WW_ERR_PRP_OVERFLOW (-3)  /* PRP list longer than its buffer        */
#define WW_ERR_HIT_OVERFLOW (-4)  /* more hits than the hit buffer holds    */
#define WW_ERR_TIMEOUT (-5)       /* ww_sync gave up waiting                */
#define WW_ERR_NOMEM (-6)         /* device or pinned allocation failed     */
#define WW_ERR_COMPOSITE (-7)     /* a reported hit is composite            */
#define WW_ERR_STATE (-8)         /* call out of order / no buffers         */
#define WW_ERR_NODEV (-9)         /* no usable CUDA device                  */

/* Hit record: the fields of gpuSpecialPrime / gpuResult / gpuRem / gpuQuot
 * (main.cpp:52-56).  result 1093 = Wieferich, 1 = WSS prime, 2 = WSS
 * special instance (wieferich.cl:248-293, wallsunsun.cl:325-349). */
typedef struct {
    uint64_t p;
    int32_t result;
    int32_t rem;
    int32_t quot;
    int32_t pad;
} ww_hit;

/* Device counters (main.cpp:1446-1493): checksum, result count, PRP count
 * of the current launch (primecount[0]), largest launch PRP count
 * (primecount[1]), PRPs tested since the last clear (totalprimecount). */
typedef struct {
    uint64_t checksum;
    uint64_t total_prp_count;
    uint32_t result_count;
    uint32_t seg_prp_count;
    uint32_t max_prp_count;
    uint32_t overflow; /* bit 0: PRP list overflow, bit 1: hit overflow */
} ww_counters;

const char *ww_last_error(void);
const char *ww_status_string(int status);
int ww_abi_version(void);

/* ---------------------------------------------------------------------------
 * 1. Kernel-shaped entry points.  Device pointers; stream is a cudaStream_t
 *    (NULL = legacy default stream).  Capacities bound every device write;
 *    counters keep counting past them so the host can detect overflow.
 * ------------------------------------------------------------------------- */

/* clearn (clearn.cl:12-21): primecount[0] = 0. */
int ww_launch_clearn(uint32_t *primecount, void *stream);

/* clearresult (clearresult.cl:12-26): checksum, resultcount,
 * totalprimecount and primecount[1] = 0. */
int ww_launch_clearresult(uint64_t *checksum, uint32_t *resultcount, uint64_t *totalprimecount,
                          uint32_t *primecount, void *stream);

/* The four launchers below take work from a cursor that the library lends
 * to the calling stream (a pool of 64 per device). A stream being captured
 * into a CUDA graph, or a launch that finds every cursor busy, splits the
 * work statically instead, with the same results. */

/* getsegprimes (getsegprimes.cl:228-301): every base-2 strong probable prime
 * in [low, high) with no prime factor <= 113 is appended to g_prime, with
 * q = p^-1 mod 2^64 in g_invert, counted in primecount[0].  low must be the
 * wheel-aligned start and wheelidx its index from ww_find_wheel_offset
 * (main.cpp:1716-1721); 127 <= low, high <= 2^64-1.  List order is
 * unspecified.  *overflow |= 1 when more than capacity PRPs were found. */
int ww_launch_getsegprimes(uint64_t low, uint64_t high, int32_t wheelidx, uint64_t *g_prime,
                           uint64_t *g_invert, uint32_t *primecount, uint64_t capacity,
                           uint32_t *overflow, void *stream);

/* wieferich (wieferich.cl:196-328): for each of the primecount[0] PRPs,
 * 2^((p-1)/2) mod p^2; hits appended to the SoA hit arrays (capacity
 * numresults), checksum += high digit mod 2^32, totalprimecount +=
 * primecount[0], primecount[1] = max(primecount[1], primecount[0]).
 * g_invert and g_one may be NULL (computed in the kernel); when g_one is
 * non-NULL the Montgomery one (2 words per PRP) is stored for wallsunsun. */
int ww_launch_wieferich(uint32_t *primecount, const uint64_t *g_prime, const uint64_t *g_invert,
                        uint64_t *g_one, uint64_t *special_prime, int32_t *rem, int32_t *quot,
                        int32_t *result, uint64_t *checksum, uint32_t *resultcount,
                        uint64_t *totalprimecount, uint64_t capacity, uint32_t numresults,
                        uint32_t *overflow, void *stream);

/* wallsunsun (wallsunsun.cl:221-354): F_{p-(p|5)} mod p^2 for each PRP;
 * hits and checksum as above.  g_invert / g_one may be NULL. */
int ww_launch_wallsunsun(const uint32_t *primecount, const uint64_t *g_prime,
                         const uint64_t *g_invert, const uint64_t *g_one, uint64_t *special_prime,
                         int32_t *rem, int32_t *quot, int32_t *result, uint64_t *checksum,
                         uint32_t *resultcount, uint64_t capacity, uint32_t numresults,
                         uint32_t *overflow, void *stream);

/* Both tests in one kernel (no reference counterpart; replaces the
 * wieferich + wallsunsun pair of main.cpp:1738-1741 with one launch).
 * Same effect on checksum, hits and counters as the pair. */
int ww_launch_test_prps(uint32_t *primecount, const uint64_t *g_prime, const uint64_t *g_invert,
                        uint64_t *special_prime, int32_t *rem, int32_t *quot, int32_t *result,
                        uint64_t *checksum, uint32_t *resultcount, uint64_t *totalprimecount,
                        uint64_t capacity, uint32_t numresults, uint32_t *overflow, void *stream);

/* Per-prime canonical digits for verification (no reference counterpart):
 * out[4i..4i+3] = (s0, s1, c20, c21) with 2^((p-1)/2) = s0 + p s1 and
 * F_{p-(p|5)} = c20 + p c21 mod p^2. */
int ww_launch_digits(const uint64_t *primes, uint64_t n, uint64_t *out, void *stream);

/* ---------------------------------------------------------------------------
 * 2. Context API (progData + simpleCL replacement).
 * ------------------------------------------------------------------------- */

typedef struct ww_ctx ww_ctx;

/* Open device `device` (cudaSetDevice) and create the stream and counters. */
int ww_open(int device, ww_ctx **out);
void ww_close(ww_ctx *ctx);

/* (Re)allocate the PRP buffers (prime, invert, one) for max_prps entries and
 * the hit arrays for max_hits (numresults, main.cpp:1119). */
int ww_reserve(ww_ctx *ctx, uint64_t max_prps, uint32_t max_hits);

int ww_clear_results(ww_ctx *ctx); /* clearresult */
int ww_clear_segment(ww_ctx *ctx); /* clearn */

/* getsegprimes over [kernel_start, stop) into the context's PRP buffers. */
int ww_sieve_prp(ww_ctx *ctx, uint64_t kernel_start, uint64_t stop, int32_t wheel_idx);

/* Sieve depth of the context's sieve launches (ww_sieve_prp, ww_count_prps).
 * No reference counterpart: getsegprimes sieves by 3..113 only
 * (getsegprimes.cl:169-225).  After 3..113 every launch sieves by the primes
 * below 2^20 segment by segment; at depth bits > 20, a launch of 2^26
 * numbers or more also marks the multiples of the primes below 2^bits, once
 * per launch (bits <= 30; the first use of a depth on a device builds its
 * prime table, which allocates device memory and synchronises the device,
 * so it belongs before any stream capture; each context also allocates a
 * 64 MiB mark bitmap on its first such launch).  Only composites that can
 * never be base-2 pseudoprimes are marked, so the PRP list is the same at
 * every depth.  A new context sieves at depth 28; depth 20 turns the large
 * primes off.  The kernel-shaped ww_launch_getsegprimes, which gets no
 * scratch, always sieves at depth 20. */
int ww_set_sieve_depth(ww_ctx *ctx, int bits);
int ww_get_sieve_depth(ww_ctx *ctx, int *bits);
/* Rows first .. first+n-1 of the device's prime table of that depth (the
 * primes 2^20 < r < 2^bits in ascending order, with ord_r(2)) and its
 * length in *total, for checking the table against an independent
 * computation.  Builds the table when it does not exist yet. */
int ww_selftest_deep_table(ww_ctx *ctx, int bits, uint64_t first, uint64_t n, uint32_t *r, uint32_t *order,
                           uint64_t *total);

/* Segment shape of the context's sieve launches (no reference counterpart;
 * with the depth, what the program's autotune picks in place of the
 * reference's work-size profiling, main.cpp:959-1107): 1 = segments of 2^20
 * numbers for 512-thread CTAs, 2 = 2^19 numbers for 256-thread CTAs, 0 (the
 * default) = the wide shape when the launch gives each resident CTA a
 * segment, else the narrow one.  Results do not depend on the shape. */
int ww_set_sieve_shape(ww_ctx *ctx, int shape);
int ww_get_sieve_shape(ww_ctx *ctx, int *shape);
int ww_wieferich(ww_ctx *ctx);
int ww_wallsunsun(ww_ctx *ctx);
int ww_test_prps(ww_ctx *ctx); /* fused wieferich + wallsunsun */

/* Copy a host list of PRPs into the context's PRP buffer (sets the segment
 * count, q computed on the device).  For fixed-list workloads. */
int ww_load_prps(ww_ctx *ctx, const uint64_t *host_primes, uint64_t n);

/* Both tests over a host list of PRPs, accumulating into the context's
 * checksum, PRP count and hit list like ww_load_prps + ww_test_prps.  The
 * list moves in chunks through the two halves of the PRP buffer on a second
 * stream, so the copy of one chunk overlaps the test of the previous one
 * (pinned host memory is needed for the overlap).  Returns when the work is
 * queued; read the counters after ww_sync.  No counterpart in the reference,
 * whose lists come from getsegprimes on the device. */
int ww_test_prps_host(ww_ctx *ctx, const uint64_t *host_primes, uint64_t n);

/* Record an event after the work queued so far; ww_wait_marker blocks until
 * the event `slot` (0..7) completed or timeout_ms passed (the reference's
 * launchEvent / waitOnEvent, main.cpp:329-377). */
int ww_marker(ww_ctx *ctx, int slot);
int ww_wait_marker(ww_ctx *ctx, int slot, uint32_t timeout_ms);

/* Wait for all queued work (sclFinish / sleepCPU, main.cpp:381-446). */
int ww_sync(ww_ctx *ctx, uint32_t timeout_ms);

/* Blocking read-backs (sclRead of main.cpp:793-840). */
int ww_read_counters(ww_ctx *ctx, ww_counters *out);
int ww_read_hits(ww_ctx *ctx, ww_hit *out, uint32_t cap, uint32_t *n);
int ww_read_prps(ww_ctx *ctx, uint64_t *out, uint64_t cap, uint64_t *n);

/* Elapsed device milliseconds between two markers (ProfilesclEnqueueKernel,
 * simpleCL.c:511-534). */
int ww_marker_elapsed(ww_ctx *ctx, int slot_a, int slot_b, float *ms);

/* Device pointers owned by the context (for the kernel-shaped calls). */
typedef struct {
    uint64_t *prime, *invert, *one;
    uint64_t *special_prime;
    int32_t *rem, *quot, *result;
    uint64_t *checksum, *total_prp_count;
    uint32_t *result_count, *primecount, *overflow;
    uint64_t prp_capacity;
    uint32_t hit_capacity;
    void *stream;
} ww_buffers;
int ww_get_buffers(ww_ctx *ctx, ww_buffers *out);

/* ---------------------------------------------------------------------------
 * Batched search (no reference counterpart; replaces running the reference
 * program once per range).  Many ranges of uneven width run in one
 * persistent, CUDA-graph-captured launch: the kernel pulls (range, segment)
 * tiles from a device queue and runs sieve, PRP test and both tests on each
 * tile inside one CTA.  Per-unit checksums equal those of running each
 * range alone.  Hits carry the unit index.
 * ------------------------------------------------------------------------- */

typedef struct {
    uint64_t start, end; /* [start, end), 127 <= start, or start == end */
} ww_unit;

typedef struct {
    uint64_t checksum;  /* sum of both checksum terms over the unit's PRPs */
    uint64_t prp_count; /* PRPs tested */
    uint32_t hits;      /* hit records of the unit */
    uint32_t tiles_done;
} ww_unit_result;

/* seg_words: 32-bit words of a tile's bitmap (64 integers per word);
 * threads: per CTA; ppt: primes per thread in the test phase (batches of 32
 * PRPs a warp collects before testing); joint: 1 = the Wieferich and WSS
 * tests of a prime in one loop, 0 = one after the other. */
typedef struct {
    uint32_t seg_words, threads, ppt, joint;
} ww_batch_cfg;

int ww_batch_configs(ww_batch_cfg *out, uint32_t cap, uint32_t *n);
int ww_batch_set_config(ww_ctx *ctx, const ww_batch_cfg *cfg);
int ww_batch_get_config(ww_ctx *ctx, ww_batch_cfg *cfg);
int ww_batch_reserve_hits(ww_ctx *ctx, uint32_t max_hits);
/* Queue the units (async on the context stream); collect waits and reads
 * the per-unit results. */
int ww_batch_submit(ww_ctx *ctx, const ww_unit *units, uint32_t n);
int ww_batch_collect(ww_ctx *ctx, ww_unit_result *out, uint32_t n, uint32_t *hit_count);
int ww_batch_run(ww_ctx *ctx, const ww_unit *units, uint32_t n, ww_unit_result *out);
int ww_batch_hits(ww_ctx *ctx, ww_hit *out, uint32_t *unit_of_hit, uint32_t cap, uint32_t *n);
/* Autotuner (replaces profileGPU, main.cpp:959-1107): times every compiled
 * configuration on the sample and keeps the fastest in the context. */
int ww_batch_tune(ww_ctx *ctx, const ww_unit *sample, uint32_t n, ww_batch_cfg *best, float *best_ms);

/* The batched search for callers that cannot allocate device memory (no
 * counterpart in the reference).  Hosts that reserve all of the GPU's
 * memory up front and forbid later allocations, or latency-bound loops
 * that cannot afford an allocation's device-wide synchronisation, get the
 * same per-range results as ww_batch_run without any allocation: the
 * scratch lives in one fixed __device__ array of the library (480 KiB per
 * device, kept until exit).  units: host array, n <= 4096 ranges;
 * out[n], hits[hit_cap] (at most 4096 records), hit_unit[hit_cap] (may be
 * NULL) and *hit_count are device memory; work is queued on `stream` (a
 * cudaStream_t) and the call does not wait for it.  Calls share the array:
 * each clears it, and calls whose GPU work overlaps race, so keep them on
 * one stream.  The first call on a device does a one-time set-up (it looks
 * up the array's address with cudaGetSymbolAddress); make that first call
 * before any stream capture.  *hit_count receives the number of hits found.  When that exceeds
 * min(hit_cap, 4096), the records hold that many of them, in no set
 * order, and out[i].hits still counts every hit of range i.
 * Returns WW_ERR_ARG for more than 4096 ranges. */
int ww_batch_run_noalloc(const ww_unit *units, uint32_t n, ww_unit_result *out, ww_hit *hits,
                         uint32_t *hit_unit, uint32_t hit_cap, uint32_t *hit_count, void *stream);

/* ---------------------------------------------------------------------------
 * Request server (no reference counterpart; the reference runs one range
 * per process).  Continuous batching: requests wait in a host queue and are
 * admitted into device slots while slots and PRP-buffer memory last (each
 * request reserves ww_prp_count_bound(start, end) * 8 bytes); every
 * ww_server_step runs one bounded launch of the tile engine over all
 * admitted requests (round-robin, each request's sieve cursor, checksum,
 * counters and PRP buffer resident on the device) and returns the requests
 * that finished.  A request's results equal those of running it alone.
 * ------------------------------------------------------------------------- */

typedef struct {
    uint64_t id, start, end; /* [start, end), 127 <= start */
} ww_request;

typedef struct {
    uint64_t id;
    uint64_t checksum, prp_count;
    uint64_t prps_stored;   /* PRPs written to the request's buffer */
    uint32_t hits;          /* hit records (read them with ww_server_hits) */
    int32_t status;         /* WW_OK, or WW_ERR_PRP_OVERFLOW / WW_ERR_HIT_OVERFLOW */
    double t_submit, t_admit, t_done; /* host monotonic seconds */
} ww_request_result;

typedef struct {
    uint64_t prp_pool_bytes; /* device memory for per-request PRP buffers */
    uint32_t max_active;     /* device slots */
    uint32_t epoch_tiles;    /* tiles one step launches (rounded to whole
                                waves of resident CTAs when above one wave;
                                0: one wave) */
    uint32_t max_hits;       /* hit records per step */
    uint32_t store_prps;     /* 1: keep each request's PRP list on the device */
} ww_server_cfg;

int ww_server_open(ww_ctx *ctx, const ww_server_cfg *cfg);
int ww_server_close(ww_ctx *ctx);
/* Queue requests (host side, any time).  All or none: WW_ERR_ARG for a bad
 * range, WW_ERR_NOMEM for a request whose PRP list could never fit the pool
 * (store_prps), and then no request of the call is queued. */
int ww_server_submit(ww_ctx *ctx, const ww_request *reqs, uint32_t n);
/* Admit, run one epoch, collect finished requests into done[0..*ndone). */
int ww_server_step(ww_ctx *ctx, ww_request_result *done, uint32_t cap, uint32_t *ndone);
int ww_server_status(ww_ctx *ctx, uint32_t *queued, uint32_t *active, uint64_t *pool_used);
/* Hits of a finished request (kept until the next ww_server_hits call for
 * that id). */
int ww_server_hits(ww_ctx *ctx, uint64_t id, ww_hit *out, uint32_t cap, uint32_t *n);
/* PRP list of a finished request with store_prps (read before its slot is
 * reused: valid until the next ww_server_step). */
int ww_server_prps(ww_ctx *ctx, uint64_t id, uint64_t *out, uint64_t cap, uint64_t *n);

/* ---------------------------------------------------------------------------
 * 3. Host helpers of the reference program (main.cpp), exported so every
 *    caller shares one implementation.
 * ------------------------------------------------------------------------- */

/* findWheelOffset (main.cpp:528-587).  Returns WW_ERR_ARG when no number
 * >= start below 2^64 is prime to 30. */
int ww_find_wheel_offset(uint64_t *start, int32_t *index);

/* isPrime (main.cpp:301-324) and isPRP (main.cpp:245-291), on the host. */
int ww_is_prime(uint64_t n);
int ww_is_prp(uint64_t n);

/* START/END parsing (main.cpp:1193-1262): e-notation or decimal. */
int ww_parse_number(const char *text, uint64_t *out);

/* getResults formatting (main.cpp:843-916): sorts hits by p, writes the
 * result lines of prime hits into buf, counts PRP-only hits in *dropped.
 * Returns bytes written, WW_ERR_COMPOSITE for a composite hit, WW_ERR_ARG
 * when buf is too small. */
int ww_format_hits(ww_hit *hits, uint32_t n, char *buf, size_t cap, uint32_t *dropped);

/* Checkpoint state (write_state / read_state, main.cpp:103-209): two files
 * written alternately, each one line "start stop current cksm psum pcnt".
 * ww_state_write writes the file due next (A when *write_a_next) and flips
 * *write_a_next only when the file was closed successfully.
 * ww_state_read returns 1 and the newer valid state (larger current; B on a
 * tie) of the files whose start/stop match, 0 when neither is usable. */
typedef struct {
    uint64_t current, cksm;
    double psum;
    int32_t pcnt, pad;
} ww_state;
int ww_state_write(const char *file_a, const char *file_b, uint64_t start, uint64_t stop,
                   const ww_state *st, int *write_a_next);
int ww_state_read(const char *file_a, const char *file_b, uint64_t start, uint64_t stop, ww_state *st,
                  int *write_a_next);

/* Upper bound on the number of base-2 strong PRPs in [lo, hi) used to size
 * PRP buffers (replaces primesieve_count_primes, main.cpp:1087-1091). */
uint64_t ww_prp_count_bound(uint64_t lo, uint64_t hi);

/* Exact number of base-2 strong PRPs with no factor <= 113 in [lo, hi),
 * lo >= 127, counted on the GPU by the sieve kernel without listing them
 * (the count primesieve_count_primes gave the reference for sizing,
 * main.cpp:1000,1087, with its pseudoprimes included).  Synchronises. */
int ww_count_prps(ww_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t *count);

/* Host twin of the kernels for the start-up self-test (testKernels,
 * main.cpp:590-738): digits of a list (same layout as ww_launch_digits) and
 * the PRP count, checksum and hit count of [lo, hi).  Never used to produce
 * results, only to check the GPU against. */
int ww_selftest_digits(const uint64_t *primes, uint64_t n, uint64_t *out);
int ww_selftest_range(uint64_t lo, uint64_t hi, uint64_t *prp_count, uint64_t *checksum,
                      uint32_t *result_count);
/* One operation of the kernels' mod p^2 arithmetic on the host, for
 * checking it operand by operand: op & 15 = 0 X*Y/2^64, 1 X^2/2^64,
 * 2 X/2^64 (mod p^2); op >> 4 picks the formulation (0 the kernels' own,
 * 1 64-bit products, 2 PTX carry chains, 3 wide 32x32+64 products).
 * Inputs and outputs are digit pairs x0 + p x1; xy = (x0, x1, y0, y1) per
 * case, out = (z0, z1). */
int ww_selftest_m2(int op, uint64_t p, const uint64_t *xy, uint64_t n, uint64_t *out);
/* The same check on the device, through the instruction sequences the
 * kernels run (borrow masks, multiply-pipe corrections): op 0-2 as above,
 * 3 X+Y, 4 X-Y, 5 2X (mod p^2), and on the low digits alone 6 x0*y0/2^64,
 * 7 x0+y0, 8 (x1 2^64 + x0)/2^64 (mod p).  Host arrays; synchronises and
 * allocates its own device copy (no reference counterpart: a test hook). */
int ww_devtest_m2(int device, int op, uint64_t p, const uint64_t *xy, uint64_t n, uint64_t *out);
/* The kernels' PRP-test candidates of [lo, hi) computed on the host
 * (small primes 3..113, then the deep sieve, which leaves unmarked every
 * multiple r*k with k = 1 (mod ord_r(2)): r itself and every possible
 * base-2 pseudoprime with the factor r), sorted; *spared = the number of
 * deep-prime multiples left unmarked that way. */
int ww_selftest_candidates(uint64_t lo, uint64_t hi, uint64_t *out, uint64_t cap, uint64_t *n,
                           uint64_t *spared);

/* ---------------------------------------------------------------------------
 * 4. Measurement utilities (no reference counterpart).
 * ------------------------------------------------------------------------- */

/* First n numbers of the SplitMix64 stream for `seed` (each output forced
 * odd, kept when >= 2^62) that pass deterministic Miller-Rabin, in stream
 * order, into the host array out (the GPU runs the primality tests).
 * *consumed receives the stream positions used.  Allocates its own scratch. */
int ww_random_primes(int device, uint64_t seed, uint64_t n, uint64_t *out, uint64_t *consumed);

/* Integer-pipe microbenchmark: mode 0 mad.lo.u32, 1 mad.hi.u32,
 * 2 mad.wide.u32, 3 64x64->128 multiply (carry chain), 4 fma.rn.f64,
 * 5 add.u32 chains.  Returns operations per second in *ops_per_s
 * (one op = one PTX instruction of that kind per thread). */
int ww_pipe_bench(int device, int mode, double *ops_per_s, double *ms);

#ifdef __cplusplus
}
#endif
#endif /* WWCUDA_H */
