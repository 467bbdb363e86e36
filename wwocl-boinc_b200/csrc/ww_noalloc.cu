// ww_noalloc.cu -- the batched search for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc: a host that reserves all of the
// GPU's memory for its own pool when it starts (a volunteer-computing
// client sharing the card with other work, say) and forbids any later
// allocation, or a latency-bound service loop in which an allocation --
// which may synchronise the whole device -- is not acceptable.  For them
// ww_batch_run_noalloc runs the batched search with all of its scratch
// (per-range device state, the tile table, the tile-queue head, the hit
// staging area) in one file-scope __device__ array of fixed size, so the
// call itself allocates nothing; the caller still passes the ranges and the
// output buffers.
//
// Limits and sharing: at most kNoAllocMaxUnits ranges and kNoAllocMaxHits
// hit records per call.  Every call on a device shares the one array and it
// keeps the previous call's contents, so each call clears what must start
// at zero, and calls whose GPU work overlaps (on different streams, or from
// different host threads) race on it -- order them on one stream.  The
// first call on each device does a one-time set-up (the device addresses of
// the array and of the library's deep-sieve table, and the kernel's
// shared-memory attribute); that first call should come before any stream
// capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/wwcuda.h"
#include "ww_batch.cuh"

using namespace ww;

namespace ww {
void set_err(const char *fmt, ...);  // ww_capi.cu
}

namespace {

constexpr uint32_t kNoAllocMaxUnits = 4096;
constexpr uint32_t kNoAllocMaxHits = 4096;
constexpr int kNoAllocMaxDevices = 64;
typedef BatchCfg<8192, 256, 1> NoAllocCfg;

struct NoAllocScratch {
    UnitState units[kNoAllocMaxUnits];
    u64 tile_first[kNoAllocMaxUnits + 1];
    u64 next_tile;
    u32 reserved, epoch, hit_count, overflow;
    u64 hit_p[kNoAllocMaxHits];
    int hit_result[kNoAllocMaxHits], hit_rem[kNoAllocMaxHits], hit_quot[kNoAllocMaxHits];
    u32 hit_unit[kNoAllocMaxHits];
};

// The scratch of every call on a device: 491 552 bytes (480 KiB) per device
// that loads the library, held until the process exits.
static_assert(sizeof(NoAllocScratch) == 491552, "the documented scratch size");
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

struct DeviceSetup {
    bool done = false;
    NoAllocScratch *scratch = nullptr;  // device address of g_noalloc_scratch
    int grid = 0;
};

DeviceSetup g_setup[kNoAllocMaxDevices];
std::mutex g_mutex;  // guards g_setup and the host staging below

// Host staging of the per-range state and tile table (copied into the
// device array on the caller's stream).  These are pageable: a host-to-device
// cudaMemcpyAsync from pageable memory returns only once the source has been
// staged, so the next call may refill them as soon as the mutex is free.
UnitState g_h_units[kNoAllocMaxUnits];
u64 g_h_first[kNoAllocMaxUnits + 1];

__global__ void k_noalloc_finish(const NoAllocScratch *s, uint32_t n, ww_unit_result *out, ww_hit *hits,
                                 uint32_t *hit_unit, uint32_t hit_cap, uint32_t *hit_count) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t i = tid; i < n; i += gridDim.x * blockDim.x) {
        out[i].checksum = s->units[i].checksum;
        out[i].prp_count = s->units[i].prp_count;
        out[i].hits = s->units[i].hits;
        out[i].tiles_done = s->units[i].tiles_done;
    }
    const uint32_t nh = s->hit_count < kNoAllocMaxHits ? s->hit_count : kNoAllocMaxHits;
    for (uint32_t i = tid; i < nh && i < hit_cap; i += gridDim.x * blockDim.x) {
        hits[i].p = s->hit_p[i];
        hits[i].result = s->hit_result[i];
        hits[i].rem = s->hit_rem[i];
        hits[i].quot = s->hit_quot[i];
        hits[i].pad = 0;
        if (hit_unit) hit_unit[i] = s->hit_unit[i];
    }
    if (tid == 0) *hit_count = s->hit_count;
}

int setup_device(int dev, DeviceSetup &d) {
    if (d.done) return WW_OK;
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) {
        set_err("cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return WW_ERR_CUDA;
    }
    constexpr size_t smem = batch_smem_bytes<NoAllocCfg>();
    e = cudaFuncSetAttribute(k_tiles<NoAllocCfg, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tiles<NoAllocCfg, false>, NoAllocCfg::kThreads,
                                                          smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        set_err("device set-up: %s", cudaGetErrorString(e));
        return WW_ERR_CUDA;
    }
    d.scratch = static_cast<NoAllocScratch *>(addr);
    d.grid = (per_sm > 0 ? per_sm : 1) * sms;
    d.done = true;
    return WW_OK;
}

}  // namespace

extern "C" int ww_batch_run_noalloc(const ww_unit *units, uint32_t n, ww_unit_result *out, ww_hit *hits,
                                    uint32_t *hit_unit, uint32_t hit_cap, uint32_t *hit_count, void *stream) {
    if (n > kNoAllocMaxUnits) {
        set_err("%u ranges: the allocation-free batch takes at most %u", n, kNoAllocMaxUnits);
        return WW_ERR_ARG;
    }
    if ((!units && n) || (!out && n) || !hit_count || (!hits && hit_cap)) {
        set_err("null argument");
        return WW_ERR_ARG;
    }
    if (hit_cap > kNoAllocMaxHits) hit_cap = kNoAllocMaxHits;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
        set_err("no usable current device");
        return WW_ERR_NODEV;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceSetup &d = g_setup[dev];
    int rc = setup_device(dev, d);
    if (rc) return rc;

    const u64 tile = NoAllocCfg::kTileNumbers;
    u64 acc = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (units[i].end < units[i].start || (units[i].end > units[i].start && units[i].start < 127)) {
            set_err("range %u: bad range [%llu, %llu)", i, (unsigned long long)units[i].start,
                    (unsigned long long)units[i].end);
            return WW_ERR_ARG;
        }
        UnitState &u = g_h_units[i];
        memset(&u, 0, sizeof u);
        u.start = units[i].start;
        u.end = units[i].end;
        const u64 w = units[i].end - units[i].start;
        u.n_tiles = w / tile + (w % tile ? 1 : 0);
        u.active = 1;
        g_h_first[i] = acc;
        acc += u.n_tiles;
    }
    g_h_first[n] = acc;

    NoAllocScratch *s = d.scratch;
    // the per-range state doubles as the cleared result block; counters restart at zero
    cudaError_t e = cudaSuccess;
    if (n) e = cudaMemcpyAsync(s->units, g_h_units, (size_t)n * sizeof(UnitState), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->tile_first, g_h_first, ((size_t)n + 1) * sizeof(u64), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(&s->next_tile, 0, sizeof(u64) + 4 * sizeof(u32), st);  // next_tile..overflow
    if (e != cudaSuccess) {
        set_err("staging copy: %s", cudaGetErrorString(e));
        return WW_ERR_CUDA;
    }
    BatchArgs a;
    memset(&a, 0, sizeof a);
    a.units = s->units;
    a.n_units = n;
    a.tile_first = s->tile_first;
    a.n_tiles = acc;
    a.next_tile = &s->next_tile;
    a.epoch_tiles = &s->epoch;
    a.hit_p = s->hit_p;
    a.hit_result = s->hit_result;
    a.hit_rem = s->hit_rem;
    a.hit_quot = s->hit_quot;
    a.hit_unit = s->hit_unit;
    a.hit_count = &s->hit_count;
    a.hit_capacity = kNoAllocMaxHits;
    a.overflow = &s->overflow;
    a.deep = deep_rows_device();  // the library's constant table, no allocation
    if (!a.deep) return WW_ERR_CUDA;
    if (acc)
        k_tiles<NoAllocCfg, false><<<d.grid, NoAllocCfg::kThreads, batch_smem_bytes<NoAllocCfg>(), st>>>(a);
    k_noalloc_finish<<<32, 256, 0, st>>>(s, n, out, hits, hit_unit, hit_cap, hit_count);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_err("launch: %s", cudaGetErrorString(e));
        return WW_ERR_CUDA;
    }
    return WW_OK;
}
