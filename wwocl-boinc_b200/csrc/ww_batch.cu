// ww_batch.cu -- host side of the batched search (include/wwcuda.h section 5):
// the compiled configurations, the tile table, the CUDA-graph-captured
// persistent launch and the autotuner that picks segment size, threads per
// CTA, primes per thread and the test loop by timing them on a sample of
// the workload.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <deque>
#include <map>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "../../include/wwcuda.h"
#include "ww_trace.hpp"
#include "ww_batch.cuh"

using namespace ww;

namespace ww {
void set_err(const char *fmt, ...);  // ww_capi.cu
int ctx_device(ww_ctx *c);
void *ctx_stream(ww_ctx *c);
struct BatchState;
BatchState *&ctx_batch(ww_ctx *c);
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

typedef void (*TileKernel)(BatchArgs);

struct CfgEntry {
    int seg_words, threads, ppt, joint;
    TileKernel kernel;        // static tile table (batch)
    TileKernel serve_kernel;  // request slots in deadline order (serving)
    size_t smem;
};

template <int W, int T, int P, int J = 0>
CfgEntry entry() {
    typedef BatchCfg<W, T, P, J> C;
    return CfgEntry{W, T, P, J, &k_tiles<C, false>, &k_tiles<C, true>, batch_smem_bytes<C>()};
}

// Segment bitmaps of 16-128 KB: the whole segment sits in one CTA's shared
// memory (at most 227 KB per CTA on the B200, so a 256 KB segment cannot be
// a tile), beside the warps' queues.  128-1024 threads.  1-8 batches of 32
// PRPs per warp before testing: 4 and 8 only at 256 threads, with the
// registers the compiler picks (BatchCfg::kMinBlocks).  The joint test loop
// (both tests in one loop, 72 registers in the list kernel) at 256 and 512
// threads, held to 64 registers.
const std::vector<CfgEntry> &configs() {
    static const std::vector<CfgEntry> table = {
        entry<4096, 128, 1>(),     entry<4096, 256, 1>(),     entry<4096, 512, 1>(),    entry<4096, 256, 2>(),
        entry<8192, 256, 1>(),     entry<8192, 512, 1>(),     entry<8192, 1024, 1>(),   entry<8192, 256, 2>(),
        entry<8192, 256, 4>(),     entry<8192, 256, 8>(),     entry<16384, 256, 1>(),   entry<16384, 512, 1>(),
        entry<16384, 1024, 1>(),   entry<16384, 512, 2>(),    entry<32768, 256, 1>(),   entry<32768, 512, 1>(),
        entry<8192, 256, 1, 1>(),  entry<16384, 256, 1, 1>(), entry<16384, 512, 1, 1>(),
    };
    return table;
}

const CfgEntry *find_cfg(const ww_batch_cfg &c) {
    for (const CfgEntry &e : configs())
        if (e.seg_words == (int)c.seg_words && e.threads == (int)c.threads && e.ppt == (int)c.ppt &&
            e.joint == (int)c.joint)
            return &e;
    return nullptr;
}

// the configuration the autotuner picks on the uneven mix: 64 KB tiles, 512
// threads, two CTAs per SM at 64 registers, the tests one after the other
// (841 M primes/s on its first 128 units, against 774 M for the joint test
// loop, which needs the same 64 registers with more live state)
ww_batch_cfg default_cfg() { return ww_batch_cfg{16384, 512, 1, 0}; }

// the request server's unless the caller chose one for the context: the same
// tile, with one CTA per SM per step (server_init)
ww_batch_cfg default_serve_cfg() { return default_cfg(); }

}  // namespace

namespace ww {

struct BatchState {
    UnitState *d_units = nullptr;
    u64 *d_first = nullptr;
    u64 *d_next = nullptr;
    u32 *d_epoch = nullptr;
    u32 *d_hit_count = nullptr, *d_overflow = nullptr, *d_hit_unit = nullptr;
    u64 *d_hit_p = nullptr;
    int *d_hit_res = nullptr, *d_hit_rem = nullptr, *d_hit_quot = nullptr;
    u32 unit_cap = 0, hit_cap = 0;
    UnitState *h_units = nullptr;  // pinned mirror of d_units
    u64 *h_first = nullptr;        // pinned tile table
    u32 n_units = 0;
    cudaGraphExec_t exec = nullptr;
    bool tuned = false;
    ww_batch_cfg cfg = default_cfg();

    ~BatchState() {
        cudaFree(d_units);
        cudaFree(d_first);
        cudaFree(d_next);
        cudaFree(d_epoch);
        cudaFree(d_hit_count);
        cudaFree(d_overflow);
        cudaFree(d_hit_unit);
        cudaFree(d_hit_p);
        cudaFree(d_hit_res);
        cudaFree(d_hit_rem);
        cudaFree(d_hit_quot);
        if (h_units) cudaFreeHost(h_units);
        if (h_first) cudaFreeHost(h_first);
        if (exec) cudaGraphExecDestroy(exec);
    }
};

void destroy_batch_state(BatchState *s) { delete s; }

}  // namespace ww

namespace {

int ensure_capacity(BatchState &b, u32 n_units, u32 hit_cap) {
    if (n_units > b.unit_cap) {
        cudaFree(b.d_units);
        cudaFree(b.d_first);
        if (b.h_units) cudaFreeHost(b.h_units);
        if (b.h_first) cudaFreeHost(b.h_first);
        b.d_units = nullptr;
        b.d_first = nullptr;
        b.h_units = nullptr;
        b.h_first = nullptr;
        b.unit_cap = 0;
        WW_CU(cudaMalloc(&b.d_units, (size_t)n_units * sizeof(UnitState)));
        WW_CU(cudaMalloc(&b.d_first, ((size_t)n_units + 1) * sizeof(u64)));
        WW_CU(cudaMallocHost(&b.h_units, (size_t)n_units * sizeof(UnitState)));
        WW_CU(cudaMallocHost(&b.h_first, ((size_t)n_units + 1) * sizeof(u64)));
        b.unit_cap = n_units;
    }
    // each on its own, so a call after a failed one allocates what is missing
    if (!b.d_next) WW_CU(cudaMalloc(&b.d_next, sizeof(u64)));
    if (!b.d_epoch) WW_CU(cudaMalloc(&b.d_epoch, sizeof(u32)));
    if (!b.d_hit_count) WW_CU(cudaMalloc(&b.d_hit_count, sizeof(u32)));
    if (!b.d_overflow) WW_CU(cudaMalloc(&b.d_overflow, sizeof(u32)));
    if (hit_cap > b.hit_cap) {
        cudaFree(b.d_hit_unit);
        cudaFree(b.d_hit_p);
        cudaFree(b.d_hit_res);
        cudaFree(b.d_hit_rem);
        cudaFree(b.d_hit_quot);
        b.hit_cap = 0;
        WW_CU(cudaMalloc(&b.d_hit_unit, (size_t)hit_cap * 4));
        WW_CU(cudaMalloc(&b.d_hit_p, (size_t)hit_cap * 8));
        WW_CU(cudaMalloc(&b.d_hit_res, (size_t)hit_cap * 4));
        WW_CU(cudaMalloc(&b.d_hit_rem, (size_t)hit_cap * 4));
        WW_CU(cudaMalloc(&b.d_hit_quot, (size_t)hit_cap * 4));
        b.hit_cap = hit_cap;
    }
    return WW_OK;
}

BatchArgs make_args(BatchState &b, u32 n, u64 n_tiles) {
    BatchArgs a;
    a.units = b.d_units;
    a.n_units = n;
    a.tile_first = b.d_first;
    a.n_tiles = n_tiles;
    a.next_tile = b.d_next;
    a.epoch_tiles = b.d_epoch;
    a.budget = 0;
    a.hit_p = b.d_hit_p;
    a.hit_result = b.d_hit_res;
    a.hit_rem = b.d_hit_rem;
    a.hit_quot = b.d_hit_quot;
    a.hit_unit = b.d_hit_unit;
    a.hit_count = b.d_hit_count;
    a.hit_capacity = b.hit_cap;
    a.overflow = b.d_overflow;
    a.deep = deep_rows_device();  // callers check it before launching
    return a;
}

int launch_grid(const CfgEntry &e, int device, int *grid) {
    int optin = 0;
    WW_CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    if ((int)e.smem > optin) return set_err("batch config needs %zu bytes of shared memory", e.smem), WW_ERR_ARG;
    WW_CU(cudaFuncSetAttribute(e.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem));
    int per_sm = 0, sms = 0;
    WW_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, e.kernel, e.threads, e.smem));
    WW_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (per_sm < 1) return set_err("batch config does not fit on an SM"), WW_ERR_ARG;
    *grid = per_sm * sms;
    return WW_OK;
}

// Upload the units (their device state doubles as the cleared result
// block) and the tile table, then record clear + persistent launch as a
// CUDA graph on the stream and run it.
int run_batch(ww_ctx *ctx, BatchState &b, const ww_unit *units, uint32_t n, const CfgEntry &e,
              u64 *n_tiles_out) {
    const int dev = ctx_device(ctx);
    cudaStream_t st = (cudaStream_t)ctx_stream(ctx);
    const u64 tile = 64ull * (u64)e.seg_words;
    int rc = ensure_capacity(b, n ? n : 1, b.hit_cap ? b.hit_cap : 1u << 16);
    if (rc) return rc;
    WW_CU(cudaStreamSynchronize(st));  // the pinned mirror may still feed a previous launch
    u64 acc = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (units[i].end < units[i].start || (units[i].end > units[i].start && units[i].start < 127))
            return set_err("unit %u: bad range [%llu, %llu)", i, (unsigned long long)units[i].start,
                           (unsigned long long)units[i].end), WW_ERR_ARG;
        UnitState &u = b.h_units[i];
        memset(&u, 0, sizeof u);
        u.start = units[i].start;
        u.end = units[i].end;
        const u64 w = units[i].end - units[i].start;
        u.n_tiles = w / tile + (w % tile ? 1 : 0);
        u.active = 1;
        b.h_first[i] = acc;
        acc += u.n_tiles;
    }
    b.h_first[n] = acc;
    b.n_units = n;
    *n_tiles_out = acc;
    int grid = 0;
    rc = launch_grid(e, dev, &grid);
    if (rc) return rc;
    const BatchArgs a = make_args(b, n, acc);
    if (!a.deep) return WW_ERR_CUDA;

    cudaGraph_t g = nullptr;
    WW_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(b.d_units, b.h_units, (size_t)n * sizeof(UnitState), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b.d_first, b.h_first, ((size_t)n + 1) * sizeof(u64), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(b.d_next, 0, sizeof(u64), st);
    cudaMemsetAsync(b.d_hit_count, 0, sizeof(u32), st);
    cudaMemsetAsync(b.d_overflow, 0, sizeof(u32), st);
    if (acc) e.kernel<<<grid, e.threads, e.smem, st>>>(a);
    cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (ce != cudaSuccess) return set_err("graph capture: %s", cudaGetErrorString(ce)), WW_ERR_CUDA;
    bool updated = false;
    if (b.exec) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(b.exec, g, &info) == cudaSuccess;
        if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(b.exec);
            b.exec = nullptr;
        }
    }
    if (!updated) {
        ce = cudaGraphInstantiate(&b.exec, g, 0);
        if (ce != cudaSuccess) {
            cudaGraphDestroy(g);
            return set_err("graph instantiate: %s", cudaGetErrorString(ce)), WW_ERR_CUDA;
        }
    }
    cudaGraphDestroy(g);
    WW_CU(cudaGraphLaunch(b.exec, st));
    return WW_OK;
}

}  // namespace

extern "C" {

int ww_batch_configs(ww_batch_cfg *out, uint32_t cap, uint32_t *n) {
    if (!n || (!out && cap)) return WW_ERR_ARG;
    const auto &t = configs();
    *n = (uint32_t)t.size();
    for (uint32_t i = 0; i < cap && i < t.size(); ++i)
        out[i] = ww_batch_cfg{(uint32_t)t[i].seg_words, (uint32_t)t[i].threads, (uint32_t)t[i].ppt,
                              (uint32_t)t[i].joint};
    return WW_OK;
}

int ww_batch_set_config(ww_ctx *ctx, const ww_batch_cfg *cfg) {
    if (!ctx || !cfg) return set_err("null argument"), WW_ERR_ARG;
    if (!find_cfg(*cfg))
        return set_err("config %u/%u/%u/%u is not compiled", cfg->seg_words, cfg->threads, cfg->ppt, cfg->joint),
               WW_ERR_ARG;
    BatchState *&bs = ctx_batch(ctx);
    if (!bs) bs = new (std::nothrow) BatchState;
    if (!bs) return set_err("host allocation failed"), WW_ERR_NOMEM;
    bs->cfg = *cfg;
    bs->tuned = true;
    return WW_OK;
}

int ww_batch_get_config(ww_ctx *ctx, ww_batch_cfg *cfg) {
    if (!ctx || !cfg) return set_err("null argument"), WW_ERR_ARG;
    BatchState *bs = ctx_batch(ctx);
    *cfg = bs ? bs->cfg : default_cfg();
    return WW_OK;
}

int ww_batch_reserve_hits(ww_ctx *ctx, uint32_t max_hits) {
    if (!ctx || max_hits == 0) return set_err("bad argument"), WW_ERR_ARG;
    BatchState *&bs = ctx_batch(ctx);
    if (!bs) bs = new (std::nothrow) BatchState;
    if (!bs) return set_err("host allocation failed"), WW_ERR_NOMEM;
    cudaSetDevice(ctx_device(ctx));
    return ensure_capacity(*bs, 1, max_hits);
}

int ww_batch_submit(ww_ctx *ctx, const ww_unit *units, uint32_t n) {
    ww::TraceRange trace("ww_batch_submit");
    if (!ctx || (!units && n)) return set_err("null argument"), WW_ERR_ARG;
    BatchState *&bs = ctx_batch(ctx);
    if (!bs) bs = new (std::nothrow) BatchState;
    if (!bs) return set_err("host allocation failed"), WW_ERR_NOMEM;
    WW_CU(cudaSetDevice(ctx_device(ctx)));
    const CfgEntry *e = find_cfg(bs->cfg);
    if (!e) return set_err("no batch config"), WW_ERR_STATE;
    u64 tiles = 0;
    return run_batch(ctx, *bs, units, n, *e, &tiles);
}

int ww_batch_collect(ww_ctx *ctx, ww_unit_result *out, uint32_t n, uint32_t *hit_count) {
    ww::TraceRange trace("ww_batch_collect");
    if (!ctx || (!out && n)) return set_err("null argument"), WW_ERR_ARG;
    BatchState *bs = ctx_batch(ctx);
    if (!bs || n > bs->n_units) return set_err("no batch of %u units submitted", n), WW_ERR_STATE;
    cudaStream_t st = (cudaStream_t)ctx_stream(ctx);
    u32 hc[2] = {0, 0};
    if (n) WW_CU(cudaMemcpyAsync(bs->h_units, bs->d_units, (size_t)n * sizeof(UnitState), cudaMemcpyDeviceToHost, st));
    WW_CU(cudaMemcpyAsync(&hc[0], bs->d_hit_count, 4, cudaMemcpyDeviceToHost, st));
    WW_CU(cudaMemcpyAsync(&hc[1], bs->d_overflow, 4, cudaMemcpyDeviceToHost, st));
    WW_CU(cudaStreamSynchronize(st));
    for (uint32_t i = 0; i < n; ++i) {
        out[i].checksum = bs->h_units[i].checksum;
        out[i].prp_count = bs->h_units[i].prp_count;
        out[i].hits = bs->h_units[i].hits;
        out[i].tiles_done = bs->h_units[i].tiles_done;
    }
    if (hit_count) *hit_count = hc[0];
    if (hc[1] & 2) return set_err("%u hits, buffer holds %u", hc[0], bs->hit_cap), WW_ERR_HIT_OVERFLOW;
    return WW_OK;
}

int ww_batch_run(ww_ctx *ctx, const ww_unit *units, uint32_t n, ww_unit_result *out) {
    int rc = ww_batch_submit(ctx, units, n);
    if (rc) return rc;
    uint32_t hits = 0;
    return ww_batch_collect(ctx, out, n, &hits);
}

int ww_batch_hits(ww_ctx *ctx, ww_hit *out, uint32_t *unit_of_hit, uint32_t cap, uint32_t *n) {
    if (!ctx || !n || (!out && cap)) return set_err("null argument"), WW_ERR_ARG;
    BatchState *bs = ctx_batch(ctx);
    if (!bs || !bs->d_hit_count) return set_err("no batch submitted"), WW_ERR_STATE;
    u32 cnt = 0;
    WW_CU(cudaMemcpy(&cnt, bs->d_hit_count, 4, cudaMemcpyDeviceToHost));
    *n = cnt;
    u32 m = std::min(std::min(cnt, bs->hit_cap), cap);
    if (m) {
        std::vector<u64> p(m);
        std::vector<int> r(m), rem(m), q(m);
        std::vector<u32> u(m);
        WW_CU(cudaMemcpy(p.data(), bs->d_hit_p, (size_t)m * 8, cudaMemcpyDeviceToHost));
        WW_CU(cudaMemcpy(r.data(), bs->d_hit_res, (size_t)m * 4, cudaMemcpyDeviceToHost));
        WW_CU(cudaMemcpy(rem.data(), bs->d_hit_rem, (size_t)m * 4, cudaMemcpyDeviceToHost));
        WW_CU(cudaMemcpy(q.data(), bs->d_hit_quot, (size_t)m * 4, cudaMemcpyDeviceToHost));
        WW_CU(cudaMemcpy(u.data(), bs->d_hit_unit, (size_t)m * 4, cudaMemcpyDeviceToHost));
        for (u32 i = 0; i < m; ++i) {
            out[i] = ww_hit{p[i], r[i], rem[i], q[i], 0};
            if (unit_of_hit) unit_of_hit[i] = u[i];
        }
    }
    if (cnt > bs->hit_cap) return set_err("%u hits, buffer holds %u", cnt, bs->hit_cap), WW_ERR_HIT_OVERFLOW;
    return WW_OK;
}

// Time every compiled configuration on the sample (after one warm-up run
// each) and keep the fastest in the context.
int ww_batch_tune(ww_ctx *ctx, const ww_unit *sample, uint32_t n, ww_batch_cfg *best, float *best_ms) {
    ww::TraceRange trace("ww_batch_tune");
    if (!ctx || !sample || n == 0) return set_err("bad argument"), WW_ERR_ARG;
    BatchState *&bs = ctx_batch(ctx);
    if (!bs) bs = new (std::nothrow) BatchState;
    if (!bs) return set_err("host allocation failed"), WW_ERR_NOMEM;
    WW_CU(cudaSetDevice(ctx_device(ctx)));
    cudaStream_t st = (cudaStream_t)ctx_stream(ctx);
    cudaEvent_t a, b;
    WW_CU(cudaEventCreate(&a));
    WW_CU(cudaEventCreate(&b));
    float bestv = 1e30f;
    ww_batch_cfg bestc = default_cfg();
    for (const CfgEntry &e : configs()) {
        u64 tiles = 0;
        int rc = run_batch(ctx, *bs, sample, n, e, &tiles);  // warm-up (also instantiates)
        if (rc == WW_ERR_ARG) continue;                      // does not fit
        if (rc) return rc;
        cudaEventRecord(a, st);
        rc = run_batch(ctx, *bs, sample, n, e, &tiles);
        if (rc) return rc;
        cudaEventRecord(b, st);
        WW_CU(cudaEventSynchronize(b));
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < bestv) {
            bestv = ms;
            bestc = ww_batch_cfg{(uint32_t)e.seg_words, (uint32_t)e.threads, (uint32_t)e.ppt, (uint32_t)e.joint};
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    bs->cfg = bestc;
    bs->tuned = true;
    if (best) *best = bestc;
    if (best_ms) *best_ms = bestv;
    return WW_OK;
}

}  // extern "C"

// ===========================================================================
// Request server: continuous batching over device slots.

namespace ww {
struct ServerState;
ServerState *&ctx_server(ww_ctx *c);
}

namespace ww {

struct ServerReq {
    ww_request r;
    double t_submit;
};

struct ServerSlot {
    bool busy = false;
    ww_request r{};
    double t_submit = 0, t_admit = 0;
    u64 pool_off = 0, pool_len = 0;  // bytes
};

struct ServerState {
    ww_server_cfg cfg{};
    const CfgEntry *e = nullptr;
    int grid = 0;
    UnitState *d_slots = nullptr, *h_slots = nullptr;
    u64 *pool = nullptr;
    u32 *d_epoch = nullptr, *d_hit_count = nullptr, *d_overflow = nullptr;
    u32 *d_order = nullptr, *h_order = nullptr;  // slots in deadline order (pinned mirror)
    double tile_s = 0;                           // EMA of a step's seconds per wave of tiles
    u32 *d_hit_unit = nullptr, *h_hit_unit = nullptr;
    u64 *d_hit_p = nullptr, *h_hit_p = nullptr;
    int *d_hit_res = nullptr, *d_hit_rem = nullptr, *d_hit_quot = nullptr;
    int *h_hit_res = nullptr, *h_hit_rem = nullptr, *h_hit_quot = nullptr;
    u32 *h_counts = nullptr;  // pinned: hit count, overflow
    std::vector<ServerSlot> slots;
    std::deque<ServerReq> queue;
    std::map<u64, u64> free_blocks;  // offset -> length (bytes), coalesced
    u64 pool_used = 0;
    std::map<u64, std::vector<ww_hit>> hits;       // per request id, finished + running
    std::map<u64, std::pair<u64, u64>> done_prps;  // id -> (pool offset, count) until next step

    ~ServerState() {
        cudaFree(d_slots);
        cudaFree(pool);
        cudaFree(d_epoch);
        cudaFree(d_order);
        cudaFree(d_hit_count);
        cudaFree(d_overflow);
        cudaFree(d_hit_unit);
        cudaFree(d_hit_p);
        cudaFree(d_hit_res);
        cudaFree(d_hit_rem);
        cudaFree(d_hit_quot);
        if (h_slots) cudaFreeHost(h_slots);
        if (h_hit_unit) cudaFreeHost(h_hit_unit);
        if (h_hit_p) cudaFreeHost(h_hit_p);
        if (h_hit_res) cudaFreeHost(h_hit_res);
        if (h_hit_rem) cudaFreeHost(h_hit_rem);
        if (h_hit_quot) cudaFreeHost(h_hit_quot);
        if (h_counts) cudaFreeHost(h_counts);
        if (h_order) cudaFreeHost(h_order);
    }

    // first fit over the coalesced free list
    bool alloc(u64 len, u64 &off) {
        if (len == 0) {
            off = 0;
            return true;
        }
        for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it) {
            if (it->second >= len) {
                off = it->first;
                const u64 rest = it->second - len;
                const u64 roff = it->first + len;
                free_blocks.erase(it);
                if (rest) free_blocks[roff] = rest;
                pool_used += len;
                return true;
            }
        }
        return false;
    }
    void release(u64 off, u64 len) {
        if (len == 0) return;
        pool_used -= len;
        auto it = free_blocks.emplace(off, len).first;
        auto nx = std::next(it);
        if (nx != free_blocks.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_blocks.erase(nx);
        }
        if (it != free_blocks.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_blocks.erase(it);
            }
        }
    }
};

void destroy_server_state(ServerState *s) { delete s; }

}  // namespace ww

namespace {

double mono_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int server_init(ServerState &s, ww_ctx *ctx, const ww_server_cfg *cfg);

}  // namespace

extern "C" {

int ww_server_open(ww_ctx *ctx, const ww_server_cfg *cfg) {
    if (!ctx || !cfg || cfg->max_active == 0 || cfg->max_hits == 0)
        return set_err("bad server configuration"), WW_ERR_ARG;
    WW_CU(cudaSetDevice(ctx_device(ctx)));
    ServerState *&sv = ctx_server(ctx);
    if (sv) {
        cudaStreamSynchronize((cudaStream_t)ctx_stream(ctx));
        delete sv;
        sv = nullptr;
    }
    // built aside and registered only when complete: a failed open leaves
    // no server behind, and the destructor frees what was allocated
    std::unique_ptr<ServerState> own(new (std::nothrow) ServerState);
    if (!own) return set_err("host allocation failed"), WW_ERR_NOMEM;
    const int rc = server_init(*own, ctx, cfg);
    if (rc == WW_OK) sv = own.release();
    return rc;
}

}  // extern "C"

namespace {

int server_init(ServerState &s, ww_ctx *ctx, const ww_server_cfg *cfg) {
    s.cfg = *cfg;
    ww_batch_cfg bc = default_serve_cfg();
    BatchState *bs = ctx_batch(ctx);
    if (bs && bs->tuned) bc = bs->cfg;  // the configuration the caller set or tuned
    s.e = find_cfg(bc);
    if (!s.e) return set_err("no tile configuration"), WW_ERR_STATE;
    WW_CU(cudaFuncSetAttribute(s.e->serve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.e->smem));
    int per_sm = 0, sms = 0;
    WW_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, s.e->serve_kernel, s.e->threads, s.e->smem));
    WW_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx_device(ctx)));
    // a step hands out one tile per CTA, and small requests wait about one
    // step: with 512 threads' worth of CTAs per SM (one 512-thread tile) the
    // step is half as long as with the two an SM can hold, for 7 % less
    // throughput, which the server's load leaves room for
    const int step_per_sm = std::max(1, std::min(per_sm, 512 / s.e->threads));
    s.grid = step_per_sm * sms;
    const u32 n = cfg->max_active, h = cfg->max_hits;
    WW_CU(cudaMalloc(&s.d_slots, (size_t)n * sizeof(UnitState)));
    WW_CU(cudaMallocHost(&s.h_slots, (size_t)n * sizeof(UnitState)));
    memset(s.h_slots, 0, (size_t)n * sizeof(UnitState));
    WW_CU(cudaMemcpy(s.d_slots, s.h_slots, (size_t)n * sizeof(UnitState), cudaMemcpyHostToDevice));
    if (cfg->prp_pool_bytes) {
        WW_CU(cudaMalloc(&s.pool, cfg->prp_pool_bytes));
        s.free_blocks[0] = cfg->prp_pool_bytes & ~7ull;
    }
    WW_CU(cudaMalloc(&s.d_order, (size_t)n * 4));
    WW_CU(cudaMallocHost(&s.h_order, (size_t)n * 4));
    WW_CU(cudaMalloc(&s.d_epoch, 4));
    WW_CU(cudaMalloc(&s.d_hit_count, 4));
    WW_CU(cudaMalloc(&s.d_overflow, 4));
    WW_CU(cudaMalloc(&s.d_hit_unit, (size_t)h * 4));
    WW_CU(cudaMalloc(&s.d_hit_p, (size_t)h * 8));
    WW_CU(cudaMalloc(&s.d_hit_res, (size_t)h * 4));
    WW_CU(cudaMalloc(&s.d_hit_rem, (size_t)h * 4));
    WW_CU(cudaMalloc(&s.d_hit_quot, (size_t)h * 4));
    WW_CU(cudaMallocHost(&s.h_hit_unit, (size_t)h * 4));
    WW_CU(cudaMallocHost(&s.h_hit_p, (size_t)h * 8));
    WW_CU(cudaMallocHost(&s.h_hit_res, (size_t)h * 4));
    WW_CU(cudaMallocHost(&s.h_hit_rem, (size_t)h * 4));
    WW_CU(cudaMallocHost(&s.h_hit_quot, (size_t)h * 4));
    WW_CU(cudaMallocHost(&s.h_counts, 8));
    s.slots.assign(n, ServerSlot());
    return WW_OK;
}

}  // namespace

extern "C" {

int ww_server_close(ww_ctx *ctx) {
    if (!ctx) return set_err("null ctx"), WW_ERR_ARG;
    ServerState *&sv = ctx_server(ctx);
    if (sv) cudaStreamSynchronize((cudaStream_t)ctx_stream(ctx));
    delete sv;
    sv = nullptr;
    return WW_OK;
}

int ww_server_submit(ww_ctx *ctx, const ww_request *reqs, uint32_t n) {
    ServerState *sv = ctx ? ctx_server(ctx) : nullptr;
    if (!sv) return set_err("server not open"), WW_ERR_STATE;
    if (!reqs && n) return set_err("null requests"), WW_ERR_ARG;
    // check every request first, so a refused call queues none of them
    for (uint32_t i = 0; i < n; ++i) {
        if (reqs[i].end <= reqs[i].start || reqs[i].start < 127)
            return set_err("request %llu: bad range", (unsigned long long)reqs[i].id), WW_ERR_ARG;
        // a PRP list that could never fit the pool would wait at the head of
        // the queue for ever
        if (sv->cfg.store_prps && ww_prp_count_bound(reqs[i].start, reqs[i].end) * 8 > sv->cfg.prp_pool_bytes)
            return set_err("request %llu needs %llu bytes of PRP pool, the pool has %llu",
                           (unsigned long long)reqs[i].id,
                           (unsigned long long)(ww_prp_count_bound(reqs[i].start, reqs[i].end) * 8),
                           (unsigned long long)sv->cfg.prp_pool_bytes), WW_ERR_NOMEM;
    }
    const double t = mono_s();
    for (uint32_t i = 0; i < n; ++i) sv->queue.push_back(ServerReq{reqs[i], t});
    return WW_OK;
}

int ww_server_status(ww_ctx *ctx, uint32_t *queued, uint32_t *active, uint64_t *pool_used) {
    ServerState *sv = ctx ? ctx_server(ctx) : nullptr;
    if (!sv) return set_err("server not open"), WW_ERR_STATE;
    uint32_t a = 0;
    for (const ServerSlot &s : sv->slots) a += s.busy ? 1 : 0;
    if (queued) *queued = (uint32_t)sv->queue.size();
    if (active) *active = a;
    if (pool_used) *pool_used = sv->pool_used;
    return WW_OK;
}

int ww_server_step(ww_ctx *ctx, ww_request_result *done, uint32_t cap, uint32_t *ndone) {
    ww::TraceRange trace("ww_server_step");
    ServerState *sv = ctx ? ctx_server(ctx) : nullptr;
    if (!sv) return set_err("server not open"), WW_ERR_STATE;
    if (!ndone || (!done && cap)) return set_err("null argument"), WW_ERR_ARG;
    *ndone = 0;
    ServerState &s = *sv;
    cudaStream_t st = (cudaStream_t)ctx_stream(ctx);
    const u64 tile = 64ull * (u64)s.e->seg_words;
    s.done_prps.clear();

    // ---- admission: FIFO while a slot and PRP-buffer memory are free
    const u32 n = s.cfg.max_active;
    bool changed = false;
    for (u32 k = 0; k < n && !s.queue.empty(); ++k) {
        if (s.slots[k].busy) continue;
        const ServerReq &q = s.queue.front();
        const u64 bound = ww_prp_count_bound(q.r.start, q.r.end);
        const u64 len = s.cfg.store_prps ? bound * 8 : 0;
        u64 off = 0;
        if (len > s.cfg.prp_pool_bytes && s.cfg.store_prps)
            return set_err("request %llu needs %llu bytes, pool has %llu", (unsigned long long)q.r.id,
                           (unsigned long long)len, (unsigned long long)s.cfg.prp_pool_bytes), WW_ERR_NOMEM;
        if (!s.alloc(len, off)) break;  // wait for memory
        ServerSlot &sl = s.slots[k];
        sl.busy = true;
        sl.r = q.r;
        sl.t_submit = q.t_submit;
        sl.t_admit = mono_s();
        sl.pool_off = off;
        sl.pool_len = len;
        UnitState &u = s.h_slots[k];
        memset(&u, 0, sizeof u);
        u.start = q.r.start;
        u.end = q.r.end;
        const u64 w = q.r.end - q.r.start;
        u.n_tiles = w / tile + (w % tile ? 1 : 0);
        u.active = 1;
        if (s.cfg.store_prps) {
            u.prp_out = s.pool + off / 8;
            u.prp_cap = bound;
        }
        s.queue.pop_front();
        changed = true;
    }
    u32 active = 0;
    for (const ServerSlot &sl : s.slots) active += sl.busy ? 1 : 0;
    if (active == 0) return WW_OK;

    // ---- one epoch over every admitted request, tiles handed out earliest
    // deadline first: a request's deadline is its submission time plus twice
    // the time its tiles take on the whole GPU (a bounded slowdown for every
    // size).  In a model of the 200 req/s stream (serve_sim.py) this took the p99
    // latency from 134 ms (equal round-robin shares) to 93 ms at the same
    // p50.  Until a step has been timed, the order is that of submission.
    const double wave_s = s.tile_s > 0 ? s.tile_s : 1e-6;
    const double grid_slots = (double)std::max(1, s.grid);
    u32 n_order = 0;
    std::vector<std::pair<double, u32>> by_deadline;
    by_deadline.reserve(active);
    for (u32 k = 0; k < n; ++k)
        if (s.slots[k].busy)
            by_deadline.emplace_back(s.slots[k].t_submit + 2.0 * (double)s.h_slots[k].n_tiles / grid_slots * wave_s, k);
    std::sort(by_deadline.begin(), by_deadline.end());
    for (const auto &d : by_deadline) s.h_order[n_order++] = d.second;
    if (changed)
        WW_CU(cudaMemcpyAsync(s.d_slots, s.h_slots, (size_t)n * sizeof(UnitState), cudaMemcpyHostToDevice, st));
    WW_CU(cudaMemcpyAsync(s.d_order, s.h_order, (size_t)n_order * 4, cudaMemcpyHostToDevice, st));
    WW_CU(cudaMemsetAsync(s.d_epoch, 0, 4, st));
    WW_CU(cudaMemsetAsync(s.d_hit_count, 0, 4, st));
    WW_CU(cudaMemsetAsync(s.d_overflow, 0, 4, st));
    BatchArgs a;
    memset(&a, 0, sizeof a);
    a.units = s.d_slots;
    a.n_units = n;
    a.order = s.d_order;
    a.n_order = n_order;
    a.epoch_tiles = s.d_epoch;
    // whole waves of the resident CTAs: a partial last wave would leave most
    // SMs idle while its few tiles finish
    const u32 g = (u32)s.grid;
    if (s.cfg.epoch_tiles == 0) a.budget = g;  // one wave
    else a.budget = s.cfg.epoch_tiles < g ? s.cfg.epoch_tiles : std::max(1u, (s.cfg.epoch_tiles + g / 2) / g) * g;
    a.hit_p = s.d_hit_p;
    a.hit_result = s.d_hit_res;
    a.hit_rem = s.d_hit_rem;
    a.hit_quot = s.d_hit_quot;
    a.hit_unit = s.d_hit_unit;
    a.hit_count = s.d_hit_count;
    a.hit_capacity = s.cfg.max_hits;
    a.overflow = s.d_overflow;
    a.deep = deep_rows_device();
    if (!a.deep) return WW_ERR_CUDA;
    const int grid = std::min<int>(s.grid, (int)a.budget);
    u64 tiles_before = 0;
    for (u32 k = 0; k < n; ++k)
        if (s.slots[k].busy) tiles_before += std::min(s.h_slots[k].next_tile, s.h_slots[k].n_tiles);
    const double t_launch = mono_s();
    s.e->serve_kernel<<<grid, s.e->threads, s.e->smem, st>>>(a);
    WW_CU(cudaGetLastError());
    WW_CU(cudaMemcpyAsync(s.h_slots, s.d_slots, (size_t)n * sizeof(UnitState), cudaMemcpyDeviceToHost, st));
    WW_CU(cudaMemcpyAsync(s.h_counts, s.d_hit_count, 4, cudaMemcpyDeviceToHost, st));
    WW_CU(cudaMemcpyAsync(s.h_counts + 1, s.d_overflow, 4, cudaMemcpyDeviceToHost, st));
    WW_CU(cudaStreamSynchronize(st));
    {  // seconds per wave of tiles, from this step's tiles and time
        u64 tiles_after = 0;
        for (u32 k = 0; k < n; ++k)
            if (s.slots[k].busy) tiles_after += std::min(s.h_slots[k].next_tile, s.h_slots[k].n_tiles);
        const u64 ran = tiles_after - tiles_before;
        if (ran) {
            const double per = (mono_s() - t_launch) / std::ceil((double)ran / grid_slots);
            s.tile_s = s.tile_s > 0 ? 0.8 * s.tile_s + 0.2 * per : per;
        }
    }
    const u32 nh = std::min(s.h_counts[0], s.cfg.max_hits);
    if (nh) {
        WW_CU(cudaMemcpy(s.h_hit_unit, s.d_hit_unit, (size_t)nh * 4, cudaMemcpyDeviceToHost));
        WW_CU(cudaMemcpy(s.h_hit_p, s.d_hit_p, (size_t)nh * 8, cudaMemcpyDeviceToHost));
        WW_CU(cudaMemcpy(s.h_hit_res, s.d_hit_res, (size_t)nh * 4, cudaMemcpyDeviceToHost));
        WW_CU(cudaMemcpy(s.h_hit_rem, s.d_hit_rem, (size_t)nh * 4, cudaMemcpyDeviceToHost));
        WW_CU(cudaMemcpy(s.h_hit_quot, s.d_hit_quot, (size_t)nh * 4, cudaMemcpyDeviceToHost));
        for (u32 i = 0; i < nh; ++i) {
            const u32 k = s.h_hit_unit[i];
            if (k < n && s.slots[k].busy)
                s.hits[s.slots[k].r.id].push_back(
                    ww_hit{s.h_hit_p[i], s.h_hit_res[i], s.h_hit_rem[i], s.h_hit_quot[i], 0});
        }
    }

    // ---- finished requests
    const double t = mono_s();
    bool freed = false;
    for (u32 k = 0; k < n; ++k) {
        ServerSlot &sl = s.slots[k];
        UnitState &u = s.h_slots[k];
        if (!sl.busy || u.tiles_done < u.n_tiles) continue;
        if (*ndone < cap) {
            ww_request_result &r = done[*ndone];
            r.id = sl.r.id;
            r.checksum = u.checksum;
            r.prp_count = u.prp_count;
            r.prps_stored = u.prp_out ? std::min(u.prp_written, u.prp_cap) : 0;
            r.hits = u.hits;
            // a step whose hit records overflowed loses records of every
            // request active in it: compare the request's own count of hits
            // with the records it got, over all of its steps
            const auto it = s.hits.find(sl.r.id);
            const size_t kept = it == s.hits.end() ? 0 : it->second.size();
            r.status = kept < u.hits ? WW_ERR_HIT_OVERFLOW
                                     : (u.prp_written > u.prp_cap && u.prp_out ? WW_ERR_PRP_OVERFLOW : WW_OK);
            r.t_submit = sl.t_submit;
            r.t_admit = sl.t_admit;
            r.t_done = t;
            ++*ndone;
        } else {
            continue;  // reported at the next step
        }
        if (u.prp_out) s.done_prps[sl.r.id] = std::make_pair(sl.pool_off, std::min(u.prp_written, u.prp_cap));
        s.release(sl.pool_off, sl.pool_len);
        sl.busy = false;
        memset(&u, 0, sizeof u);
        freed = true;
    }
    if (freed)
        WW_CU(cudaMemcpyAsync(s.d_slots, s.h_slots, (size_t)n * sizeof(UnitState), cudaMemcpyHostToDevice, st));
    return WW_OK;
}

int ww_server_hits(ww_ctx *ctx, uint64_t id, ww_hit *out, uint32_t cap, uint32_t *n) {
    ServerState *sv = ctx ? ctx_server(ctx) : nullptr;
    if (!sv) return set_err("server not open"), WW_ERR_STATE;
    if (!n || (!out && cap)) return set_err("null argument"), WW_ERR_ARG;
    auto it = sv->hits.find(id);
    *n = 0;
    if (it == sv->hits.end()) return WW_OK;
    *n = (uint32_t)it->second.size();
    for (uint32_t i = 0; i < cap && i < it->second.size(); ++i) out[i] = it->second[i];
    sv->hits.erase(it);
    return WW_OK;
}

int ww_server_prps(ww_ctx *ctx, uint64_t id, uint64_t *out, uint64_t cap, uint64_t *n) {
    ServerState *sv = ctx ? ctx_server(ctx) : nullptr;
    if (!sv) return set_err("server not open"), WW_ERR_STATE;
    if (!n || (!out && cap)) return set_err("null argument"), WW_ERR_ARG;
    auto it = sv->done_prps.find(id);
    if (it == sv->done_prps.end()) return set_err("no stored PRP list for request %llu", (unsigned long long)id),
                                          WW_ERR_STATE;
    *n = it->second.second;
    const u64 m = std::min<u64>(cap, it->second.second);
    if (m) WW_CU(cudaMemcpy(out, sv->pool + it->second.first / 8, m * 8, cudaMemcpyDeviceToHost));
    return WW_OK;
}

}  // extern "C"
