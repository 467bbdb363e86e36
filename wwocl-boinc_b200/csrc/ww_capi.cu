// ww_capi.cu -- the C ABI of libwwcuda.so (include/wwcuda.h): kernel-shaped
// launchers and the ww_ctx context that replaces the reference's progData +
// simpleCL layer (main.cpp:51-90, simpleCL.c:352-719).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <thread>

#include "../../include/wwcuda.h"
#include "ww_bucket.hpp"
#include "ww_kernels.cuh"
#include "ww_trace.hpp"

using namespace ww;

namespace {
thread_local char g_err[512] = "";
}  // namespace

namespace ww {
// Message for ww_last_error(), per calling thread (shared with ww_host.cpp).
void set_err(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}
}  // namespace ww

namespace {

// A failed call leaves WW_ERR_NOMEM for an allocation, WW_ERR_CUDA otherwise,
// and clears a non-sticky error so that the next launch check does not see it.
#define WW_CU(call)                                                                             \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            cudaGetLastError();                                                                 \
            return e_ == cudaErrorMemoryAllocation ? WW_ERR_NOMEM : WW_ERR_CUDA;                \
        }                                                                                       \
    } while (0)

#define WW_CHECK_LAUNCH() WW_CU(cudaGetLastError())

int sm_count() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

int wheel_index_of(uint64_t n) {
    switch (n % 30) {
        case 7: return 0;
        case 11: return 1;
        case 13: return 2;
        case 17: return 3;
        case 19: return 4;
        case 23: return 5;
        case 29: return 6;
        case 1: return 7;
        default: return -1;
    }
}

// One full wave of resident CTAs: the test kernels take work from a cursor
// (or, without one, split the list evenly over the grid), so a grid above
// the resident count would only add CTAs that wait for a free slot.
template <class Kernel>
int resident_grid(Kernel k, int threads) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return sm_count() * per_sm;
}

int test_grid() {
    static const int g = resident_grid(k_test_prps, kTestThreads);
    return g;
}
int wieferich_grid() {
    static const int g = resident_grid(k_wieferich, kTestThreads);
    return g;
}
int wallsunsun_grid() {
    static const int g = resident_grid(k_wallsunsun, kTestThreads);
    return g;
}

}  // namespace

// The deep-sieve table: the one device copy in the library (every kernel
// that sieves gets its address).
#define WW_DEEP_ROWD(r, o, rinv, mr, mo) {r, o, rinv, mr, mo},
__device__ const DeepRow g_deep_rows[kDeepUse] = {WW_DEEP_ROWS(WW_DEEP_ROWD)};
#undef WW_DEEP_ROWD

namespace ww {
// Device address of g_deep_rows on the current device (looked up once per
// device), or nullptr with the error set.
const DeepRow *deep_rows_device() {
    constexpr int kMaxDevices = 64;
    static std::mutex mutex;
    static const DeepRow *addr[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_err("no usable current device");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mutex);
    if (!addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_deep_rows);
        if (e != cudaSuccess) {
            set_err("deep-sieve table: %s", cudaGetErrorString(e));
            return nullptr;
        }
        addr[dev] = static_cast<const DeepRow *>(p);
    }
    return addr[dev];
}
}  // namespace ww

// Work cursors for the kernel-shaped launchers, whose callers pass no scratch:
// a pool per device, each slot (one 128-byte line, so the slots' atomics do
// not share a line) lent to one stream at a time.
constexpr int kLaunchCursorSlots = 64;
constexpr int kLaunchCursorStride = 16;
__device__ u64 g_launch_cursors[kLaunchCursorSlots * kLaunchCursorStride];

namespace {

// The host side of g_launch_cursors, one per device, shared by every
// launcher (one lock, one owner table).
struct CursorPool {
    enum State : unsigned char { kFree, kLent, kRetired };
    u64 *base = nullptr;
    State state[kLaunchCursorSlots] = {};
    unsigned long long owner[kLaunchCursorSlots] = {};  // stream id
    cudaEvent_t done[kLaunchCursorSlots] = {};         // behind the owner's last launch
};
constexpr int kCursorPoolDevices = 64;
std::mutex g_cursor_mutex;
CursorPool g_cursor_pools[kCursorPoolDevices];

// Runs launch(cursor) with a cursor lent to `stream`; launch zeroes it on the
// stream before its kernel.  The lookup, the launch and an event recorded
// behind it happen under one lock, so the launches that share a slot -- all
// on its stream, hence in order -- each find it zeroed.  A slot passes to
// another stream only once its event has completed.  A stream being captured
// into a graph, or a launch that finds every slot busy, runs launch(nullptr):
// the kernels' static grid-stride split, with the same results.
template <class Launch>
int with_stream_cursor(void *stream, Launch launch) {
    using Pool = CursorPool;
    const cudaStream_t s = as_stream(stream);
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    int dev = 0;
    unsigned long long id = 0;
    if (cudaStreamIsCapturing(s, &capture) != cudaSuccess || capture != cudaStreamCaptureStatusNone ||
        cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kCursorPoolDevices ||
        cudaStreamGetId(s, &id) != cudaSuccess) {
        cudaGetLastError();
        return launch(nullptr);
    }
    std::lock_guard<std::mutex> lock(g_cursor_mutex);
    Pool &p = g_cursor_pools[dev];
    if (!p.base) {
        void *a = nullptr;
        if (cudaGetSymbolAddress(&a, g_launch_cursors) != cudaSuccess) {
            cudaGetLastError();
            return launch(nullptr);
        }
        p.base = static_cast<u64 *>(a);
    }
    int slot = -1;
    for (int i = 0; i < kLaunchCursorSlots && slot < 0; ++i)
        if (p.state[i] == Pool::kLent && p.owner[i] == id) slot = i;
    for (int i = 0; i < kLaunchCursorSlots && slot < 0; ++i) {
        if (p.state[i] == Pool::kFree) {
            if (cudaEventCreateWithFlags(&p.done[i], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                break;
            }
            slot = i;
        } else if (p.state[i] == Pool::kLent && cudaEventQuery(p.done[i]) == cudaSuccess) {
            slot = i;
        }
    }
    if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();  // from the busy slots' queries
    if (slot < 0) return launch(nullptr);
    p.state[slot] = Pool::kLent;
    p.owner[slot] = id;
    const int rc = launch(p.base + (size_t)slot * kLaunchCursorStride);
    // recorded whatever launch returned: its zeroing of the slot may be queued
    if (cudaEventRecord(p.done[slot], s) != cudaSuccess) {
        cudaGetLastError();
        p.state[slot] = Pool::kRetired;  // its event no longer covers its work
    }
    return rc;
}

}  // namespace

struct LargeMarks;
int launch_sieve(uint64_t low, uint64_t high, int32_t wheelidx, uint64_t *g_prime, uint64_t *g_invert,
                 uint32_t *primecount, uint64_t capacity, uint32_t *overflow, void *stream, u64 *cursor,
                 LargeMarks *large = nullptr, int shape = 0);

extern "C" {

const char *ww_last_error(void) { return g_err; }

const char *ww_status_string(int s) {
    switch (s) {
        case WW_OK: return "ok";
        case WW_ERR_CUDA: return "CUDA error";
        case WW_ERR_ARG: return "bad argument";
        case WW_ERR_PRP_OVERFLOW: return "PRP buffer overflow";
        case WW_ERR_HIT_OVERFLOW: return "hit buffer overflow";
        case WW_ERR_TIMEOUT: return "timeout";
        case WW_ERR_NOMEM: return "out of memory";
        case WW_ERR_COMPOSITE: return "composite hit";
        case WW_ERR_STATE: return "bad state";
        case WW_ERR_NODEV: return "no CUDA device";
        default: return "unknown status";
    }
}

int ww_abi_version(void) { return WW_ABI_VERSION; }

// ------------------------------------------------------------------ launchers

int ww_launch_clearn(uint32_t *primecount, void *stream) {
    if (!primecount) return set_err("null primecount"), WW_ERR_ARG;
    WW_CU(cudaMemsetAsync(primecount, 0, sizeof(uint32_t), as_stream(stream)));
    return WW_OK;
}

int ww_launch_clearresult(uint64_t *checksum, uint32_t *resultcount, uint64_t *totalprimecount,
                          uint32_t *primecount, void *stream) {
    if (!checksum || !resultcount || !totalprimecount || !primecount)
        return set_err("null counter pointer"), WW_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    WW_CU(cudaMemsetAsync(checksum, 0, sizeof(uint64_t), s));
    WW_CU(cudaMemsetAsync(resultcount, 0, sizeof(uint32_t), s));
    WW_CU(cudaMemsetAsync(totalprimecount, 0, sizeof(uint64_t), s));
    WW_CU(cudaMemsetAsync(primecount + 1, 0, sizeof(uint32_t), s));
    return WW_OK;
}

int ww_launch_getsegprimes(uint64_t low, uint64_t high, int32_t wheelidx, uint64_t *g_prime,
                           uint64_t *g_invert, uint32_t *primecount, uint64_t capacity,
                           uint32_t *overflow, void *stream) {
    if (!g_prime || !g_invert) return set_err("null pointer"), WW_ERR_ARG;
    return with_stream_cursor(stream, [&](u64 *cursor) -> int {
        return launch_sieve(low, high, wheelidx, g_prime, g_invert, primecount, capacity, overflow, stream, cursor);
    });
}

}  // extern "C"

namespace {

// Resident CTAs of k_sieve_prp<G> on the current device (the dynamic
// shared memory limit is raised first).
template <class G>
cudaError_t sieve_slots(int *slots) {
    cudaError_t e = cudaFuncSetAttribute(k_sieve_prp<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::kSmem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sieve_prp<G>, G::kThreads, G::kSmem);
    if (e != cudaSuccess) return e;
    *slots = sm_count() * (per_sm < 1 ? 1 : per_sm);
    return cudaSuccess;
}

template <class G>
int launch_sieve_shape(uint64_t low, uint64_t high, uint64_t span, const PrpOut &out, u64 *cursor,
                       const DeepRow *deep, cudaStream_t stream, const u32 *marks) {
    const uint64_t per = 2ull * G::kOdd;
    const uint64_t nseg = span / per + (span % per ? 1 : 0);
    int slots = 0;
    WW_CU(sieve_slots<G>(&slots));
    const uint64_t grid = nseg < (uint64_t)slots ? nseg : (uint64_t)slots;
    if (cursor) WW_CU(cudaMemsetAsync(cursor, 0, sizeof(u64), stream));
    k_sieve_prp<G><<<(unsigned)grid, G::kThreads, G::kSmem, stream>>>(low, high, nseg, out, cursor, deep, marks);
    WW_CHECK_LAUNCH();
    return WW_OK;
}

// One sieve launch over [low, high).  shape 1: the wide segments, 2: the
// narrow ones, 0: the wide shape once the range gives each of its resident
// CTAs a segment, below that the narrow one, which has twice the segments.
int launch_sieve_range(uint64_t low, uint64_t high, const PrpOut &out, u64 *cursor, const DeepRow *deep,
                       cudaStream_t stream, const u32 *marks, int shape) {
    const uint64_t span = high - (low & ~1ull);
    int wide_slots = 0;
    WW_CU(sieve_slots<SieveWide>(&wide_slots));
    const uint64_t wide_segs = span / (2ull * SieveWide::kOdd) + 1;
    if (shape == 1 || (shape == 0 && wide_segs >= (uint64_t)wide_slots))
        return launch_sieve_shape<SieveWide>(low, high, span, out, cursor, deep, stream, marks);
    return launch_sieve_shape<SieveNarrow>(low, high, span, out, cursor, deep, stream, marks);
}

}  // namespace

// The large deep primes of a context's sieve launches (ww_bucket.cu): the
// table of the context's depth and the mark bitmap the context owns.
struct LargeMarks {
    DeepLarge table;
    u32 *bits;
    u64 words;  // capacity of bits
};

// Launches of at most this many numbers each get one mark bitmap (64 MiB);
// wider ranges are sieved in pieces of this width.
constexpr u64 kLargeMarksPiece = 1ull << 30;
// Below this width a launch sieves with the per-segment deep primes only.
constexpr u64 kLargeMarksMinSpan = 1ull << 26;

// The sieve launch; with a segment cursor (zeroed here, on the stream) the
// CTAs take segments dynamically instead of striding.  With large (a
// context's table and bitmap) a launch of kLargeMarksMinSpan numbers or
// more also marks the multiples of the table's primes: in pieces of
// kLargeMarksPiece numbers, each a fill kernel and a sieve launch.
int launch_sieve(uint64_t low, uint64_t high, int32_t wheelidx, uint64_t *g_prime, uint64_t *g_invert,
                 uint32_t *primecount, uint64_t capacity, uint32_t *overflow, void *stream, u64 *cursor,
                 LargeMarks *large, int shape) {
    // g_prime == nullptr: count the PRPs without listing them
    if ((!g_prime && capacity) || !primecount || !overflow) return set_err("null pointer"), WW_ERR_ARG;
    if (low < 127 || high <= low) return set_err("bad range [%llu, %llu)", (unsigned long long)low,
                                                  (unsigned long long)high), WW_ERR_ARG;
    if (wheel_index_of(low) != wheelidx)
        return set_err("wheel index %d does not match start %llu", wheelidx, (unsigned long long)low),
               WW_ERR_ARG;
    if (ww_prp_count_bound(low, high) >= 0xffffffffull)
        return set_err("range too wide for a 32-bit PRP counter"), WW_ERR_ARG;
    const uint64_t b0 = low & ~1ull;
    PrpOut out{(u64 *)g_prime, (u64 *)g_invert, primecount, capacity, overflow};
    const DeepRow *deep = deep_rows_device();
    if (!deep) return WW_ERR_CUDA;
    cudaStream_t st = as_stream(stream);
    if (!large || !large->table.n || high - b0 < kLargeMarksMinSpan)
        return launch_sieve_range(low, high, out, cursor, deep, st, nullptr, shape);
    for (u64 a = b0; a < high;) {
        const u64 b = high - a > kLargeMarksPiece ? a + kLargeMarksPiece : high;
        const u64 lo = a == b0 ? low : a;  // pieces after the first start on an even number
        const u64 nodd = (b - a) / 2;
        // whole segments of the wide shape (2^19 odd numbers) cover either shape's reads
        const u64 words = ((nodd + SieveWide::kOdd - 1) / SieveWide::kOdd) * (u64)SieveWide::kWords;
        if (words > large->words) return set_err("mark bitmap too small"), WW_ERR_STATE;
        int rc = launch_deep_fill(a + 1, nodd, large->table, large->bits, words, st);
        if (rc) return rc;
        rc = launch_sieve_range(lo, b, out, cursor, deep, st, large->bits, shape);
        if (rc) return rc;
        a = b;
    }
    return WW_OK;
}

extern "C" {

int ww_launch_wieferich(uint32_t *primecount, const uint64_t *g_prime, const uint64_t *g_invert,
                        uint64_t *g_one, uint64_t *special_prime, int32_t *rem, int32_t *quot,
                        int32_t *result, uint64_t *checksum, uint32_t *resultcount,
                        uint64_t *totalprimecount, uint64_t capacity, uint32_t numresults,
                        uint32_t *overflow, void *stream) {
    if (!primecount || !g_prime || !special_prime || !rem || !quot || !result || !checksum ||
        !resultcount || !totalprimecount || !overflow)
        return set_err("null pointer"), WW_ERR_ARG;
    HitOut h{(u64 *)special_prime, rem, quot, result, resultcount, numresults, overflow};
    return with_stream_cursor(stream, [&](u64 *cursor) -> int {
        if (cursor) WW_CU(cudaMemsetAsync(cursor, 0, sizeof(u64), as_stream(stream)));
        k_wieferich<<<wieferich_grid(), kTestThreads, 0, as_stream(stream)>>>(
            primecount, (const u64 *)g_prime, (const u64 *)g_invert, (u64 *)g_one, h, (u64 *)checksum,
            (u64 *)totalprimecount, capacity, cursor);
        WW_CHECK_LAUNCH();
        return WW_OK;
    });
}

int ww_launch_wallsunsun(const uint32_t *primecount, const uint64_t *g_prime,
                         const uint64_t *g_invert, const uint64_t *g_one, uint64_t *special_prime,
                         int32_t *rem, int32_t *quot, int32_t *result, uint64_t *checksum,
                         uint32_t *resultcount, uint64_t capacity, uint32_t numresults,
                         uint32_t *overflow, void *stream) {
    if (!primecount || !g_prime || !special_prime || !rem || !quot || !result || !checksum ||
        !resultcount || !overflow)
        return set_err("null pointer"), WW_ERR_ARG;
    HitOut h{(u64 *)special_prime, rem, quot, result, resultcount, numresults, overflow};
    return with_stream_cursor(stream, [&](u64 *cursor) -> int {
        if (cursor) WW_CU(cudaMemsetAsync(cursor, 0, sizeof(u64), as_stream(stream)));
        k_wallsunsun<<<wallsunsun_grid(), kTestThreads, 0, as_stream(stream)>>>(
            primecount, (const u64 *)g_prime, (const u64 *)g_invert, (const u64 *)g_one, h,
            (u64 *)checksum, capacity, cursor);
        WW_CHECK_LAUNCH();
        return WW_OK;
    });
}

int ww_launch_test_prps(uint32_t *primecount, const uint64_t *g_prime, const uint64_t *g_invert,
                        uint64_t *special_prime, int32_t *rem, int32_t *quot, int32_t *result,
                        uint64_t *checksum, uint32_t *resultcount, uint64_t *totalprimecount,
                        uint64_t capacity, uint32_t numresults, uint32_t *overflow, void *stream) {
    if (!primecount || !g_prime || !special_prime || !rem || !quot || !result || !checksum ||
        !resultcount || !totalprimecount || !overflow)
        return set_err("null pointer"), WW_ERR_ARG;
    HitOut h{(u64 *)special_prime, rem, quot, result, resultcount, numresults, overflow};
    return with_stream_cursor(stream, [&](u64 *cursor) -> int {
        if (cursor) WW_CU(cudaMemsetAsync(cursor, 0, sizeof(u64), as_stream(stream)));
        k_test_prps<<<test_grid(), kTestThreads, 0, as_stream(stream)>>>(
            primecount, (const u64 *)g_prime, (const u64 *)g_invert, h, (u64 *)checksum,
            (u64 *)totalprimecount, capacity, cursor);
        WW_CHECK_LAUNCH();
        return WW_OK;
    });
}

int ww_launch_digits(const uint64_t *primes, uint64_t n, uint64_t *out, void *stream) {
    if (!primes || !out) return set_err("null pointer"), WW_ERR_ARG;
    if (n == 0) return WW_OK;
    uint64_t blocks = (n + kTestThreads - 1) / kTestThreads;
    if (blocks > (uint64_t)test_grid() * 8) blocks = (uint64_t)test_grid() * 8;
    k_digits<<<(unsigned)blocks, kTestThreads, 0, as_stream(stream)>>>((const u64 *)primes, n, (u64 *)out);
    WW_CHECK_LAUNCH();
    return WW_OK;
}

}  // extern "C"


// ------------------------------------------------------------------ context

namespace {

struct DevCounters {
    unsigned long long checksum;
    unsigned long long total;
    unsigned int resultcount;
    unsigned int primecount[2];
    unsigned int overflow;
};

__global__ void k_set_count(unsigned int *pc, unsigned int v) { pc[0] = v; }

}  // namespace

namespace ww {
struct BatchState;
struct ServerState;
void destroy_batch_state(BatchState *s);
void destroy_server_state(ServerState *s);
}  // namespace ww

// Sieve depth of a new context: the deep primes below 2^kDefaultSieveDepth
// (ww_set_sieve_depth).
#ifndef WW_SIEVE_DEPTH
#define WW_SIEVE_DEPTH 28
#endif
constexpr int kDefaultSieveDepth = WW_SIEVE_DEPTH;

struct ww_ctx {
    ww::BatchState *batch = nullptr;
    ww::ServerState *server = nullptr;
    int device = 0;
    cudaStream_t stream = nullptr;
    DevCounters *dc = nullptr;
    DevCounters *hc = nullptr;  // pinned
    u64 *prime = nullptr, *inv = nullptr, *one = nullptr;
    u64 cap = 0;
    u64 *hprime = nullptr;
    int *hrem = nullptr, *hquot = nullptr, *hres = nullptr;
    u32 hcap = 0;
    cudaEvent_t ev[8] = {};
    // ww_test_prps_host: copy stream, per-half events, per-chunk counts
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copied[2] = {}, consumed[2] = {};
    u32 *d_chunk = nullptr, *h_chunk = nullptr;  // [2 * kHostChunksMax]: count, max
    u32 *d_count = nullptr;   // ww_count_prps: count, max, overflow
    u64 *d_cursor = nullptr;  // work cursors: [0] ww_test_prps, [1] ww_sieve_prp, [2] ww_wieferich,
                              // [3] ww_wallsunsun, [4] ww_count_prps, [5 + i] host chunk i
    // the large deep primes of ww_sieve_prp / ww_count_prps (ww_set_sieve_depth)
    int sieve_depth = kDefaultSieveDepth;
    int sieve_shape = 0;  // ww_set_sieve_shape
    LargeMarks large{{nullptr, 0}, nullptr, 0};
};

namespace {
constexpr u64 kHostChunksMax = 1024;

// The context's large deep primes for a sieve launch over [lo, hi): nullptr
// at depth WW_DEEP_BITS or for a launch too narrow to use them; otherwise
// the table of its depth and the context's mark bitmap (allocated on first
// use, one piece wide).
int context_large_marks(ww_ctx *c, u64 lo, u64 hi, LargeMarks **out) {
    *out = nullptr;
    if (c->sieve_depth <= WW_DEEP_BITS || hi <= lo || hi - (lo & ~1ull) < kLargeMarksMinSpan) return WW_OK;
    DeepLarge t{nullptr, 0};
    const int rc = deep_large_device(c->sieve_depth, &t);
    if (rc) return rc;
    c->large.table = t;
    if (!c->large.bits) {
        const u64 words = (kLargeMarksPiece / 2 / SieveWide::kOdd) * (u64)SieveWide::kWords;
        const cudaError_t e = cudaMalloc(&c->large.bits, words * sizeof(u32));
        if (e != cudaSuccess) {
            cudaGetLastError();
            c->large.bits = nullptr;
            return set_err("mark bitmap: %s", cudaGetErrorString(e)), WW_ERR_NOMEM;
        }
        c->large.words = words;
    }
    *out = &c->large;
    return WW_OK;
}
}

extern "C" {

int ww_open(int device, ww_ctx **out) {
    if (!out) return set_err("null out"), WW_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0)
        return set_err("no CUDA device %d (count %d)", device, ndev), WW_ERR_NODEV;
    WW_CU(cudaSetDevice(device));
    ww_ctx *c = new (std::nothrow) ww_ctx;
    if (!c) return set_err("host allocation failed"), WW_ERR_NOMEM;
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->dc, sizeof(DevCounters));
    if (e == cudaSuccess) e = cudaMallocHost(&c->hc, sizeof(DevCounters));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_cursor, (5 + kHostChunksMax) * sizeof(u64));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_count, 4 * sizeof(u32));
    for (int i = 0; i < 8 && e == cudaSuccess; ++i) e = cudaEventCreate(&c->ev[i]);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->dc, 0, sizeof(DevCounters), c->stream);
    if (e != cudaSuccess) {
        set_err("ww_open: %s", cudaGetErrorString(e));
        ww_close(c);
        return WW_ERR_CUDA;
    }
    *out = c;
    return WW_OK;
}

void ww_close(ww_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    ww::destroy_server_state(c->server);
    ww::destroy_batch_state(c->batch);
    cudaFree(c->prime);
    cudaFree(c->inv);
    cudaFree(c->one);
    cudaFree(c->hprime);
    cudaFree(c->hrem);
    cudaFree(c->hquot);
    cudaFree(c->hres);
    cudaFree(c->dc);
    cudaFree(c->d_cursor);
    cudaFree(c->d_count);
    cudaFree(c->large.bits);
    if (c->hc) cudaFreeHost(c->hc);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    cudaFree(c->d_chunk);
    if (c->h_chunk) cudaFreeHost(c->h_chunk);
    for (int i = 0; i < 2; ++i) {
        if (c->copied[i]) cudaEventDestroy(c->copied[i]);
        if (c->consumed[i]) cudaEventDestroy(c->consumed[i]);
    }
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    for (int i = 0; i < 8; ++i)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int ww_reserve(ww_ctx *c, uint64_t max_prps, uint32_t max_hits) {
    if (!c || max_prps == 0 || max_hits == 0) return set_err("bad reserve arguments"), WW_ERR_ARG;
    WW_CU(cudaSetDevice(c->device));
    WW_CU(cudaStreamSynchronize(c->stream));
    if (max_prps != c->cap) {
        cudaFree(c->prime);
        cudaFree(c->inv);
        cudaFree(c->one);
        c->prime = c->inv = c->one = nullptr;
        c->cap = 0;
        if (cudaMalloc(&c->prime, max_prps * 8) != cudaSuccess ||
            cudaMalloc(&c->inv, max_prps * 8) != cudaSuccess ||
            cudaMalloc(&c->one, max_prps * 16) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(c->prime);
            cudaFree(c->inv);
            cudaFree(c->one);
            c->prime = c->inv = c->one = nullptr;
            return set_err("cannot allocate PRP buffers for %llu entries", (unsigned long long)max_prps),
                   WW_ERR_NOMEM;
        }
        c->cap = max_prps;
    }
    if (max_hits != c->hcap) {
        cudaFree(c->hprime);
        cudaFree(c->hrem);
        cudaFree(c->hquot);
        cudaFree(c->hres);
        c->hprime = nullptr;
        c->hrem = c->hquot = c->hres = nullptr;
        c->hcap = 0;
        if (cudaMalloc(&c->hprime, (size_t)max_hits * 8) != cudaSuccess ||
            cudaMalloc(&c->hrem, (size_t)max_hits * 4) != cudaSuccess ||
            cudaMalloc(&c->hquot, (size_t)max_hits * 4) != cudaSuccess ||
            cudaMalloc(&c->hres, (size_t)max_hits * 4) != cudaSuccess) {
            cudaGetLastError();
            // none or all: the launches check hprime alone
            cudaFree(c->hprime);
            cudaFree(c->hrem);
            cudaFree(c->hquot);
            cudaFree(c->hres);
            c->hprime = nullptr;
            c->hrem = c->hquot = c->hres = nullptr;
            return set_err("cannot allocate hit buffers for %u entries", max_hits), WW_ERR_NOMEM;
        }
        c->hcap = max_hits;
    }
    return WW_OK;
}

int ww_get_buffers(ww_ctx *c, ww_buffers *b) {
    if (!c || !b) return set_err("null argument"), WW_ERR_ARG;
    b->prime = (uint64_t *)c->prime;
    b->invert = (uint64_t *)c->inv;
    b->one = (uint64_t *)c->one;
    b->special_prime = (uint64_t *)c->hprime;
    b->rem = c->hrem;
    b->quot = c->hquot;
    b->result = c->hres;
    b->checksum = (uint64_t *)&c->dc->checksum;
    b->total_prp_count = (uint64_t *)&c->dc->total;
    b->result_count = &c->dc->resultcount;
    b->primecount = c->dc->primecount;
    b->overflow = &c->dc->overflow;
    b->prp_capacity = c->cap;
    b->hit_capacity = c->hcap;
    b->stream = c->stream;
    return WW_OK;
}

int ww_clear_results(ww_ctx *c) {
    if (!c) return set_err("null ctx"), WW_ERR_ARG;
    int rc = ww_launch_clearresult((uint64_t *)&c->dc->checksum, &c->dc->resultcount, (uint64_t *)&c->dc->total,
                                   c->dc->primecount, c->stream);
    if (rc) return rc;
    WW_CU(cudaMemsetAsync(&c->dc->overflow, 0, sizeof(unsigned int), c->stream));
    return WW_OK;
}

int ww_clear_segment(ww_ctx *c) {
    if (!c) return set_err("null ctx"), WW_ERR_ARG;
    return ww_launch_clearn(c->dc->primecount, c->stream);
}

#define WW_NEED_BUFFERS(c)                                                        \
    do {                                                                          \
        if (!(c)) return set_err("null ctx"), WW_ERR_ARG;                         \
        if (!(c)->prime || !(c)->hprime) return set_err("ww_reserve first"), WW_ERR_STATE; \
    } while (0)

int ww_sieve_prp(ww_ctx *c, uint64_t kernel_start, uint64_t stop, int32_t wheel_idx) {
    ww::TraceRange trace("ww_sieve_prp");
    WW_NEED_BUFFERS(c);
    LargeMarks *large = nullptr;
    const int rc = context_large_marks(c, kernel_start, stop, &large);
    if (rc) return rc;
    return launch_sieve(kernel_start, stop, wheel_idx, (uint64_t *)c->prime, (uint64_t *)c->inv, c->dc->primecount,
                        c->cap, &c->dc->overflow, c->stream, c->d_cursor + 1, large, c->sieve_shape);
}

int ww_set_sieve_shape(ww_ctx *c, int shape) {
    if (!c) return set_err("null context"), WW_ERR_ARG;
    if (shape < 0 || shape > 2) return set_err("sieve shape %d: 0 (by width), 1 (wide) or 2 (narrow)", shape), WW_ERR_ARG;
    c->sieve_shape = shape;
    return WW_OK;
}

int ww_get_sieve_shape(ww_ctx *c, int *shape) {
    if (!c || !shape) return set_err("null argument"), WW_ERR_ARG;
    *shape = c->sieve_shape;
    return WW_OK;
}

int ww_set_sieve_depth(ww_ctx *c, int bits) {
    if (!c) return set_err("null context"), WW_ERR_ARG;
    if (bits != WW_DEEP_BITS && (bits <= WW_DEEP_BITS || bits > kDeepLargeMaxBits))
        return set_err("sieve depth %d: %d (no large primes) or %d..%d", bits, WW_DEEP_BITS, WW_DEEP_BITS + 1,
                       kDeepLargeMaxBits), WW_ERR_ARG;
    c->sieve_depth = bits;
    return WW_OK;
}

int ww_selftest_deep_table(ww_ctx *c, int bits, uint64_t first, uint64_t n, uint32_t *r, uint32_t *order,
                           uint64_t *total) {
    if (!c || !total || ((!r || !order) && n)) return set_err("null argument"), WW_ERR_ARG;
    WW_CU(cudaSetDevice(c->device));
    return read_deep_large(bits, first, n, r, order, total);
}

int ww_get_sieve_depth(ww_ctx *c, int *bits) {
    if (!c || !bits) return set_err("null argument"), WW_ERR_ARG;
    *bits = c->sieve_depth;
    return WW_OK;
}

int ww_wieferich(ww_ctx *c) {
    ww::TraceRange trace("ww_wieferich");
    WW_NEED_BUFFERS(c);
    WW_CU(cudaMemsetAsync(c->d_cursor + 2, 0, sizeof(u64), c->stream));
    HitOut h{c->hprime, c->hrem, c->hquot, c->hres, &c->dc->resultcount, c->hcap, &c->dc->overflow};
    k_wieferich<<<wieferich_grid(), kTestThreads, 0, c->stream>>>(c->dc->primecount, c->prime, c->inv, c->one, h,
                                                                  (u64 *)&c->dc->checksum, (u64 *)&c->dc->total,
                                                                  c->cap, c->d_cursor + 2);
    WW_CHECK_LAUNCH();
    return WW_OK;
}

int ww_wallsunsun(ww_ctx *c) {
    ww::TraceRange trace("ww_wallsunsun");
    WW_NEED_BUFFERS(c);
    WW_CU(cudaMemsetAsync(c->d_cursor + 3, 0, sizeof(u64), c->stream));
    HitOut h{c->hprime, c->hrem, c->hquot, c->hres, &c->dc->resultcount, c->hcap, &c->dc->overflow};
    k_wallsunsun<<<wallsunsun_grid(), kTestThreads, 0, c->stream>>>(c->dc->primecount, c->prime, c->inv, c->one, h,
                                                                    (u64 *)&c->dc->checksum, c->cap,
                                                                    c->d_cursor + 3);
    WW_CHECK_LAUNCH();
    return WW_OK;
}

int ww_test_prps(ww_ctx *c) {
    ww::TraceRange trace("ww_test_prps");
    WW_NEED_BUFFERS(c);
    WW_CU(cudaMemsetAsync(c->d_cursor, 0, sizeof(u64), c->stream));
    HitOut h{c->hprime, c->hrem, c->hquot, c->hres, &c->dc->resultcount, c->hcap, &c->dc->overflow};
    k_test_prps<<<test_grid(), kTestThreads, 0, c->stream>>>(c->dc->primecount, c->prime, c->inv, h,
                                                             (u64 *)&c->dc->checksum, (u64 *)&c->dc->total,
                                                             c->cap, c->d_cursor);
    WW_CHECK_LAUNCH();
    return WW_OK;
}

int ww_load_prps(ww_ctx *c, const uint64_t *host_primes, uint64_t n) {
    WW_NEED_BUFFERS(c);
    if (n > c->cap || n > 0xffffffffull || (!host_primes && n))
        return set_err("list of %llu PRPs does not fit (capacity %llu)", (unsigned long long)n,
                       (unsigned long long)c->cap), WW_ERR_ARG;
    if (n) WW_CU(cudaMemcpyAsync(c->prime, host_primes, n * 8, cudaMemcpyHostToDevice, c->stream));
    k_set_count<<<1, 1, 0, c->stream>>>(c->dc->primecount, (unsigned)n);
    WW_CHECK_LAUNCH();
    if (n) {
        uint64_t blocks = (n + 255) / 256;
        if (blocks > (uint64_t)sm_count() * 8) blocks = (uint64_t)sm_count() * 8;
        k_fill_inverse<<<(unsigned)blocks, 256, 0, c->stream>>>(c->prime, c->inv, n);
        WW_CHECK_LAUNCH();
    }
    return WW_OK;
}

int ww_test_prps_host(ww_ctx *c, const uint64_t *host_primes, uint64_t n) {
    ww::TraceRange trace("ww_test_prps_host");
    WW_NEED_BUFFERS(c);
    if (!host_primes && n) return set_err("null list"), WW_ERR_ARG;
    if (n == 0) return WW_OK;
    if (c->cap < 2) return set_err("PRP buffer too small for double buffering"), WW_ERR_ARG;
    WW_CU(cudaSetDevice(c->device));
    // each resource on its own, so a call after a failed one creates what is missing
    if (!c->copy_stream) WW_CU(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
        if (!c->copied[i]) WW_CU(cudaEventCreateWithFlags(&c->copied[i], cudaEventDisableTiming));
        if (!c->consumed[i]) WW_CU(cudaEventCreateWithFlags(&c->consumed[i], cudaEventDisableTiming));
    }
    if (!c->d_chunk) WW_CU(cudaMalloc(&c->d_chunk, 2 * kHostChunksMax * sizeof(u32)));
    if (!c->h_chunk) WW_CU(cudaMallocHost(&c->h_chunk, 2 * kHostChunksMax * sizeof(u32)));
    // Chunks grow from 2^19 PRPs by doubling up to half the buffer, so the
    // one copy that nothing overlaps (the first) is short and every later
    // copy hides behind the test of the chunk before it.
    const u64 maxc = std::min<u64>(c->cap / 2, 0xffffffffull);
    // the previous call's copy of the count table may still read h_chunk
    WW_CU(cudaStreamSynchronize(c->stream));
    u64 nchunks = 0;
    for (u64 done = 0, len = std::min<u64>(1ull << 19, maxc); done < n; len = std::min<u64>(2 * len, maxc)) {
        if (nchunks == kHostChunksMax)
            return set_err("list of %llu PRPs needs a larger PRP buffer (capacity %llu)", (unsigned long long)n,
                           (unsigned long long)c->cap), WW_ERR_ARG;
        const u64 take = std::min<u64>(len, n - done);
        c->h_chunk[2 * nchunks] = (u32)take;
        c->h_chunk[2 * nchunks + 1] = 0;
        ++nchunks;
        done += take;
    }
    WW_CU(cudaMemcpyAsync(c->d_chunk, c->h_chunk, 2 * nchunks * sizeof(u32), cudaMemcpyHostToDevice, c->stream));
    WW_CU(cudaMemsetAsync(c->d_cursor + 5, 0, nchunks * sizeof(u64), c->stream));
    // the copy stream must not overwrite a half that earlier test work still reads
    WW_CU(cudaEventRecord(c->consumed[0], c->stream));
    WW_CU(cudaEventRecord(c->consumed[1], c->stream));
    HitOut h{c->hprime, c->hrem, c->hquot, c->hres, &c->dc->resultcount, c->hcap, &c->dc->overflow};
    u64 offset = 0;
    for (u64 i = 0; i < nchunks; ++i) {
        const int half = (int)(i & 1);
        u64 *dst = c->prime + (u64)half * maxc;
        const u64 len = c->h_chunk[2 * i];
        WW_CU(cudaStreamWaitEvent(c->copy_stream, c->consumed[half], 0));
        WW_CU(cudaMemcpyAsync(dst, host_primes + offset, len * 8, cudaMemcpyHostToDevice, c->copy_stream));
        WW_CU(cudaEventRecord(c->copied[half], c->copy_stream));
        WW_CU(cudaStreamWaitEvent(c->stream, c->copied[half], 0));
        k_test_prps<<<test_grid(), kTestThreads, 0, c->stream>>>(c->d_chunk + 2 * i, dst, nullptr, h,
                                                                 (u64 *)&c->dc->checksum, (u64 *)&c->dc->total,
                                                                 len, c->d_cursor + 5 + i);
        WW_CHECK_LAUNCH();
        WW_CU(cudaEventRecord(c->consumed[half], c->stream));
        offset += len;
    }
    return WW_OK;
}

int ww_count_prps(ww_ctx *c, uint64_t lo, uint64_t hi, uint64_t *count) {
    ww::TraceRange trace("ww_count_prps");
    if (!c || !count) return set_err("null argument"), WW_ERR_ARG;
    if (lo < 127 || hi < lo) return set_err("bad range [%llu, %llu)", (unsigned long long)lo,
                                            (unsigned long long)hi), WW_ERR_ARG;
    WW_CU(cudaSetDevice(c->device));
    *count = 0;
    // pieces of 2^34 numbers keep every piece's count inside the 32-bit counter
    constexpr u64 kPiece = 1ull << 34;
    for (u64 a = lo; a < hi;) {
        const u64 b = hi - a > kPiece ? a + kPiece : hi;
        uint64_t ks = a;
        int32_t idx = 0;
        if (ww_find_wheel_offset(&ks, &idx) != WW_OK) break;  // nothing prime to 30 is left below 2^64
        if (ks < b) {
            WW_CU(cudaMemsetAsync(c->d_count, 0, 4 * sizeof(u32), c->stream));
            LargeMarks *large = nullptr;
            int rc = context_large_marks(c, ks, b, &large);
            if (rc) return rc;
            rc = launch_sieve(ks, b, idx, nullptr, nullptr, c->d_count, 0, c->d_count + 2, c->stream,
                              c->d_cursor + 4, large, c->sieve_shape);
            if (rc) return rc;
            u32 n = 0;
            WW_CU(cudaMemcpyAsync(&n, c->d_count, sizeof(u32), cudaMemcpyDeviceToHost, c->stream));
            WW_CU(cudaStreamSynchronize(c->stream));
            *count += n;
        }
        a = b;
    }
    return WW_OK;
}

int ww_marker(ww_ctx *c, int slot) {
    if (!c || slot < 0 || slot >= 8) return set_err("bad marker slot"), WW_ERR_ARG;
    WW_CU(cudaEventRecord(c->ev[slot], c->stream));
    return WW_OK;
}

static int wait_event(cudaEvent_t ev, uint32_t timeout_ms) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return WW_OK;
        if (e != cudaErrorNotReady) {
            set_err("cudaEventQuery: %s", cudaGetErrorString(e));
            return WW_ERR_CUDA;
        }
        const auto dt = std::chrono::steady_clock::now() - t0;
        if (timeout_ms && std::chrono::duration_cast<std::chrono::milliseconds>(dt).count() >= timeout_ms)
            return set_err("timed out after %u ms", timeout_ms), WW_ERR_TIMEOUT;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
}

int ww_wait_marker(ww_ctx *c, int slot, uint32_t timeout_ms) {
    if (!c || slot < 0 || slot >= 8) return set_err("bad marker slot"), WW_ERR_ARG;
    return wait_event(c->ev[slot], timeout_ms);
}

int ww_marker_elapsed(ww_ctx *c, int a, int b, float *ms) {
    if (!c || a < 0 || a >= 8 || b < 0 || b >= 8 || !ms) return set_err("bad marker slot"), WW_ERR_ARG;
    WW_CU(cudaEventElapsedTime(ms, c->ev[a], c->ev[b]));
    return WW_OK;
}

int ww_sync(ww_ctx *c, uint32_t timeout_ms) {
    if (!c) return set_err("null ctx"), WW_ERR_ARG;
    WW_CU(cudaEventRecord(c->ev[7], c->stream));
    return wait_event(c->ev[7], timeout_ms);
}

int ww_read_counters(ww_ctx *c, ww_counters *out) {
    if (!c || !out) return set_err("null argument"), WW_ERR_ARG;
    WW_CU(cudaMemcpyAsync(c->hc, c->dc, sizeof(DevCounters), cudaMemcpyDeviceToHost, c->stream));
    WW_CU(cudaStreamSynchronize(c->stream));
    out->checksum = c->hc->checksum;
    out->total_prp_count = c->hc->total;
    out->result_count = c->hc->resultcount;
    out->seg_prp_count = c->hc->primecount[0];
    out->max_prp_count = c->hc->primecount[1];
    out->overflow = c->hc->overflow;
    return WW_OK;
}

int ww_read_hits(ww_ctx *c, ww_hit *out, uint32_t cap, uint32_t *n) {
    if (!c || !n || (!out && cap)) return set_err("null argument"), WW_ERR_ARG;
    ww_counters k;
    int rc = ww_read_counters(c, &k);
    if (rc) return rc;
    *n = k.result_count;
    uint32_t m = k.result_count < c->hcap ? k.result_count : c->hcap;
    if (m > cap) m = cap;
    if (m) {
        u64 *p = new (std::nothrow) u64[m];
        int *a = new (std::nothrow) int[3 * (size_t)m];
        if (!p || !a) {
            delete[] p;
            delete[] a;
            return set_err("host allocation failed"), WW_ERR_NOMEM;
        }
        cudaError_t e = cudaMemcpy(p, c->hprime, (size_t)m * 8, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(a, c->hres, (size_t)m * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(a + m, c->hrem, (size_t)m * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(a + 2 * (size_t)m, c->hquot, (size_t)m * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            delete[] p;
            delete[] a;
            return set_err("hit read-back: %s", cudaGetErrorString(e)), WW_ERR_CUDA;
        }
        for (uint32_t i = 0; i < m; ++i) {
            out[i].p = p[i];
            out[i].result = a[i];
            out[i].rem = a[m + i];
            out[i].quot = a[2 * (size_t)m + i];
            out[i].pad = 0;
        }
        delete[] p;
        delete[] a;
    }
    if (k.result_count > c->hcap) return set_err("%u hits, buffer holds %u", k.result_count, c->hcap),
                                          WW_ERR_HIT_OVERFLOW;
    return WW_OK;
}

int ww_read_prps(ww_ctx *c, uint64_t *out, uint64_t cap, uint64_t *n) {
    if (!c || !n || (!out && cap)) return set_err("null argument"), WW_ERR_ARG;
    ww_counters k;
    int rc = ww_read_counters(c, &k);
    if (rc) return rc;
    *n = k.seg_prp_count;
    uint64_t m = k.seg_prp_count < c->cap ? k.seg_prp_count : c->cap;
    if (m > cap) m = cap;
    if (m) WW_CU(cudaMemcpy(out, c->prime, m * 8, cudaMemcpyDeviceToHost));
    if (k.seg_prp_count > c->cap) return set_err("%u PRPs, buffer holds %llu", k.seg_prp_count,
                                                 (unsigned long long)c->cap), WW_ERR_PRP_OVERFLOW;
    return WW_OK;
}

}  // extern "C"

namespace ww {
int ctx_device(ww_ctx *c) { return c->device; }
void *ctx_stream(ww_ctx *c) { return c->stream; }
BatchState *&ctx_batch(ww_ctx *c) { return c->batch; }
ServerState *&ctx_server(ww_ctx *c) { return c->server; }
}  // namespace ww
