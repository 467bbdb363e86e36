// wwocl.cpp -- the WWocl search program on the B200 kernels.
//
//   wwocl START END [-testprimes] [-compute] [-debug] [-ws N] [-separate]
//                   [-ckpt NUMBERS] [-results FILE] [-device D]
//
// Keeps the reference program's interface and behaviour (main.cpp:1110-1803):
// START/END parsing with e-notation, START clamped to 127, A/B checkpoint
// files, the results file with one line per prime hit and the final 16-digit
// hex checksum, the start-up self-test and the segment loop with a queue at
// most three segments deep.  The device work goes through libwwcuda.so.
//
// Extra flags: -separate runs the reference's two test kernels instead of
// the fused one; -ckpt N also checkpoints every N numbers; -results FILE
// names the results file (default results-WW.txt, the reference code's
// name; the reference README calls it results-WWocl.txt); -device D picks
// the CUDA device.
#include <inttypes.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../host/wwhost.hpp"
#include "wwcuda.h"

using namespace wwhost;

namespace {

const uint32_t kNumResults = 15000;             // main.cpp:1119
const uint64_t kMaxRange = 4000000000ull;       // segment width cap (PRP buffer <= ~12 GB)

[[noreturn]] void fail(const char *what, int rc) {
    fprintf(stderr, "ERROR: %s: %s (%s)\n", what, ww_status_string(rc), ww_last_error());
    printf("ERROR: %s: %s\n", what, ww_status_string(rc));
    exit(EXIT_FAILURE);
}

void must(int rc, const char *what) {
    if (rc != WW_OK) fail(what, rc);
}

struct Options {
    uint64_t bottom = 0, top = 0;
    bool testprimes = false, compute = false, debug = false, separate = false;
    int ws = 0;
    uint64_t ckpt_numbers = 0;
    int device = 0;
    Files files;
};

void usage(const char *prog) {
    printf("Usage: %s START END -testprimes -compute -debug -ws #\nWhere 127 <= START < END < 2^64\n", prog);
    printf("-testprimes compares every GPU PRP list with a CPU prime list (slow)\n");
    printf("-compute sizes segments for a fully loaded GPU (100 ms per segment)\n");
    printf("-debug prints counters at each checkpoint\n");
    printf("-ws # sets the segment time target in ms (1..100, default 10)\n");
    printf("-separate runs the Wieferich and WallSunSun kernels one after the other\n");
    printf("-ckpt N also checkpoints every N numbers; -results FILE; -device D\n");
    printf("Example format: %s 10000000 20000000\n            Or: %s 1e7 2e7\n", prog, prog);
}

Options parse(int argc, char **argv) {
    Options o;
    if (argc < 3) {
        usage(argv[0]);
        exit(EXIT_FAILURE);
    }
    for (int w = 3; w < argc; ++w) {  // main.cpp:1171-1190, 1427-1443
        if (!strcmp(argv[w], "-compute")) {
            o.compute = true;
            fprintf(stderr, "Compute mode enabled.\n");
            printf("Compute mode enabled.\n");
        } else if (!strcmp(argv[w], "-testprimes")) {
            o.testprimes = true;
            fprintf(stderr, "Comparing all GPU generated primes with CPU generated primes.\n");
            printf("Comparing all GPU generated primes with CPU generated primes.\n");
        } else if (!strcmp(argv[w], "-debug")) {
            o.debug = true;
            printf("Debug info enabled.\n");
        } else if (!strcmp(argv[w], "-separate")) {
            o.separate = true;
        } else if (!strcmp(argv[w], "-ws") && w + 1 < argc) {
            o.ws = atoi(argv[++w]);
            if (o.ws < 1 || o.ws > 100) o.ws = 0;
        } else if (!strcmp(argv[w], "-ckpt") && w + 1 < argc) {
            if (ww_parse_number(argv[++w], &o.ckpt_numbers) != WW_OK) o.ckpt_numbers = 0;
        } else if (!strcmp(argv[w], "-results") && w + 1 < argc) {
            o.files.results = argv[++w];
        } else if (!strcmp(argv[w], "-device") && w + 1 < argc) {
            o.device = atoi(argv[++w]);
        }
    }
    if (ww_parse_number(argv[1], &o.bottom) != WW_OK) {
        printf("ERROR: unable to parse START\n");
        fprintf(stderr, "ERROR: unable to parse START\n");
        exit(EXIT_FAILURE);
    }
    if (ww_parse_number(argv[2], &o.top) != WW_OK) {
        printf("ERROR: unable to parse END\n");
        fprintf(stderr, "ERROR: unable to parse END\n");
        exit(EXIT_FAILURE);
    }
    if (o.bottom < 127) {  // main.cpp:1265-1274
        printf("START below minimum. Starting search at 127\n");
        fprintf(stderr, "START below minimum. Starting search at 127\n");
        o.bottom = 127;
    }
    if (o.top <= o.bottom) {
        printf("ERROR: END must be > START\n");
        fprintf(stderr, "ERROR: END must be > START\n");
        exit(EXIT_FAILURE);
    }
    return o;
}

// One segment: clearn, getsegprimes, then the tests.
void enqueue_segment(ww_ctx *ctx, uint64_t start, uint64_t stop, bool separate) {
    must(ww_clear_segment(ctx), "clearn");
    uint64_t ks = start;
    int32_t idx = 0;
    if (ww_find_wheel_offset(&ks, &idx) != WW_OK || ks >= stop) return;  // nothing prime to 30 left
    must(ww_sieve_prp(ctx, ks, stop, idx), "getsegprimes");
    if (separate) {
        must(ww_wieferich(ctx), "wieferich");
        must(ww_wallsunsun(ctx), "wallsunsun");
    } else {
        must(ww_test_prps(ctx), "test_prps");
    }
}

// -debug's kernel profile (main.cpp:1632-1661): one segment's sieve,
// Wieferich and WallSunSun kernels timed with events, as shares of the sum.
void profile_kernels(ww_ctx *ctx, uint64_t start, uint64_t stop) {
    printf("Profiling kernels...\n");
    uint64_t ks = start;
    int32_t idx = 0;
    if (ww_find_wheel_offset(&ks, &idx) != WW_OK || ks >= stop) return;
    must(ww_clear_results(ctx), "clearresult");
    must(ww_clear_segment(ctx), "clearn");
    must(ww_marker(ctx, 1), "marker");
    must(ww_sieve_prp(ctx, ks, stop, idx), "getsegprimes");
    must(ww_marker(ctx, 2), "marker");
    must(ww_wieferich(ctx), "wieferich");
    must(ww_marker(ctx, 3), "marker");
    must(ww_wallsunsun(ctx), "wallsunsun");
    must(ww_marker(ctx, 4), "marker");
    must(ww_sync(ctx, 600000), "sync");
    float prime_ms = 0, wie_ms = 0, wall_ms = 0;
    must(ww_marker_elapsed(ctx, 1, 2, &prime_ms), "elapsed");
    must(ww_marker_elapsed(ctx, 2, 3, &wie_ms), "elapsed");
    must(ww_marker_elapsed(ctx, 3, 4, &wall_ms), "elapsed");
    const double total = (double)prime_ms + wie_ms + wall_ms;
    const int prime_pct = (int)(prime_ms / total * 100.0), wie_pct = (int)(wie_ms / total * 100.0),
              wall_pct = (int)(wall_ms / total * 100.0);
    printf("Percent of time spent in each kernel:\n");
    printf("\tPrime Generator:\t%d %%\t(%0.1f ms)\n\tWieferich Test:\t\t%d %%\t(%0.1f ms)\n"
           "\tWallSunSun Test:\t%d %%\t(%0.1f ms)\n",
           prime_pct, prime_ms, wie_pct, wie_ms, wall_pct, wall_ms);
    must(ww_clear_results(ctx), "clearresult");
}

// checkPRPS (main.cpp:451-523): the GPU PRP list minus base-2 pseudoprimes
// must equal the CPU prime list of [start, stop).
uint32_t check_prps(ww_ctx *ctx, uint64_t start, uint64_t stop, uint64_t cap) {
    ww_counters k;
    must(ww_read_counters(ctx, &k), "read counters");
    if (k.seg_prp_count > cap) {
        fprintf(stderr, "Error: prime array overflow!\n");
        exit(EXIT_FAILURE);
    }
    std::vector<uint64_t> gpu(k.seg_prp_count);
    uint64_t n = 0;
    must(ww_read_prps(ctx, gpu.data(), gpu.size(), &n), "read PRP list");
    gpu.resize(n);
    const uint32_t prpcount = (uint32_t)n;
    std::vector<uint64_t> primes;
    primes.reserve(n);
    for (uint64_t p : gpu) {
        if (ww_is_prime(p)) primes.push_back(p);
        else if (!ww_is_prp(p)) {
            fprintf(stderr, "Computation error, GPU found a composite: %" PRIu64 "\n", p);
            exit(EXIT_FAILURE);
        }
    }
    std::sort(primes.begin(), primes.end());
    const std::vector<uint64_t> cpu = cpu_primes(start, stop);
    if (primes.size() != cpu.size()) {
        fprintf(stderr, "ERROR: gpu prime count: %zu does not match cpu: %zu\n", primes.size(), cpu.size());
        printf("ERROR: gpu prime count: %zu does not match cpu: %zu\n", primes.size(), cpu.size());
        exit(EXIT_FAILURE);
    }
    for (size_t i = 0; i < cpu.size(); ++i)
        if (cpu[i] != primes[i]) {
            fprintf(stderr, "ERROR: gpu/cpu prime mismatch %" PRIu64 " vs %" PRIu64 "\n", primes[i], cpu[i]);
            printf("ERROR: gpu/cpu prime mismatch %" PRIu64 " vs %" PRIu64 "\n", primes[i], cpu[i]);
            exit(EXIT_FAILURE);
        }
    return prpcount;
}

// testKernels (main.cpp:590-738): GPU against the host twin and the CPU
// prime list over min(2e6, calc_range) numbers from start.
void self_test(ww_ctx *ctx, uint64_t start, uint64_t top, uint64_t calc_range, uint64_t cap, bool debug,
               bool separate) {
    uint64_t stop = start + std::min<uint64_t>(2000000, calc_range);
    if (stop < start || stop > top) stop = top;
    fprintf(stderr, "Verifying GPU kernels using range %" PRIu64 " to %" PRIu64 "...\n", start, stop);
    if (debug) printf("Verifying GPU kernels using range %" PRIu64 " to %" PRIu64 "...\n", start, stop);
    must(ww_clear_results(ctx), "clearresult");
    enqueue_segment(ctx, start, stop, separate);
    // the host twin on every host thread while the GPU works; the sums do
    // not depend on how the range is split
    uint64_t prp = 0, cks = 0;
    uint32_t res = 0;
    uint64_t part_prp[16] = {}, part_cks[16] = {};
    uint32_t part_res[16] = {};
    int part_rc[16] = {};
    const unsigned parts = parallel_pieces(start, stop, [&](uint64_t a, uint64_t b, unsigned i) {
        part_rc[i] = ww_selftest_range(a, b, &part_prp[i], &part_cks[i], &part_res[i]);
    });
    for (unsigned i = 0; i < parts; ++i) {
        must(part_rc[i], "host self-test");
        prp += part_prp[i];
        cks += part_cks[i];
        res += part_res[i];
    }
    must(ww_sync(ctx, 600000), "sync");
    const uint32_t gpuprimecount = check_prps(ctx, start, stop, cap);
    if (gpuprimecount != prp) {
        fprintf(stderr, "ERROR: gpu / cpu prp count mismatch %u / %" PRIu64 "\n", gpuprimecount, prp);
        printf("ERROR: gpu / cpu prp count mismatch %u / %" PRIu64 "\n", gpuprimecount, prp);
        exit(EXIT_FAILURE);
    }
    fprintf(stderr, "GPU prime generator kernel test passed. (%" PRIu64 " PRPs)\n", prp);
    if (debug) printf("GPU prime generator kernel test passed. (%" PRIu64 " PRPs)\n", prp);
    ww_counters k;
    must(ww_read_counters(ctx, &k), "read counters");
    if (k.checksum != cks) {
        fprintf(stderr, "ERROR: gpu / cpu checksum mismatch %" PRIu64 " / %" PRIu64 "\n", k.checksum, cks);
        printf("ERROR: gpu / cpu checksum mismatch %" PRIu64 " / %" PRIu64 "\n", k.checksum, cks);
        exit(EXIT_FAILURE);
    }
    if (k.result_count != res) {
        fprintf(stderr, "ERROR: gpu / cpu result count mismatch %u / %u\n", k.result_count, res);
        printf("ERROR: gpu / cpu result count mismatch %u / %u\n", k.result_count, res);
        exit(EXIT_FAILURE);
    }
    fprintf(stderr, "GPU Wieferich/WallSunSun kernel tests passed. (%" PRIu64 " checksum, %u results)\n", cks, res);
    if (debug) printf("GPU Wieferich/WallSunSun kernel tests passed. (%" PRIu64 " checksum, %u results)\n", cks, res);
}

// getResults (main.cpp:768-956).
void get_results(ww_ctx *ctx, const Options &o, double ckpt_secs, State &st, uint64_t mem_size) {
    ww_counters k;
    must(ww_read_counters(ctx, &k), "read counters");
    st.cksm += k.checksum;  // main.cpp:799
    if (k.max_prp_count > mem_size || (k.overflow & 1)) {
        fprintf(stderr, "Error: prime array overflow!\n");
        exit(EXIT_FAILURE);
    }
    uint32_t dropped = 0;
    if (k.result_count > 0) {
        if (k.result_count > kNumResults || (k.overflow & 2)) {
            fprintf(stderr, "Error: number of results (%u) overflowed array.\n", k.result_count);
            exit(EXIT_FAILURE);
        }
        std::vector<ww_hit> hits(k.result_count);
        uint32_t n = 0;
        must(ww_read_hits(ctx, hits.data(), k.result_count, &n), "read hits");
        std::vector<char> buf((size_t)n * 256 + 1);
        const int rc = ww_format_hits(hits.data(), n, buf.data(), buf.size(), &dropped);
        if (rc == WW_ERR_COMPOSITE) {
            fprintf(stderr, "Computation error, GPU found a composite result: %s\n", ww_last_error());
            exit(EXIT_FAILURE);
        }
        if (rc < 0) fail("format results", rc);
        if (!report_solution(o.files, std::string(buf.data(), (size_t)rc))) exit(EXIT_FAILURE);
    }
    if (o.debug) {
        printf("PRPs tested since last checkpoint: %" PRIu64 "\n", k.total_prp_count);
        printf("Max number of results:             %u\n", kNumResults);
        printf("Number of results:                 %u\n", k.result_count);
        printf("PRPs removed from results:         %u\n", dropped);
        printf("Largest kernel PRP count:          %u\n", k.max_prp_count);
        printf("Max kernel PRP count for malloc:   %" PRIu64 "\n", mem_size);
    }
    if (ckpt_secs <= 0) ckpt_secs = 1e-3;
    st.psum += (double)k.total_prp_count / ckpt_secs / 1e6;  // main.cpp:946-949
    ++st.pcnt;
}

// profileGPU (main.cpp:959-1107), re-done as a measurement of one sieve +
// test segment: grow the width until a segment takes the target time.
uint64_t autotune(ww_ctx *ctx, uint64_t current, uint64_t top, double target_ms, bool separate, bool debug) {
    uint64_t width = 1ull << 26;
    uint64_t start = current;
    if (top - start < width) return std::max<uint64_t>(top - start, 1);
    double ms = 0;
    for (int it = 0; it < 6; ++it) {
        if (width > kMaxRange) width = kMaxRange;
        const uint64_t need = ww_prp_count_bound(start, start + width);
        must(ww_reserve(ctx, need, kNumResults), "reserve (autotune)");
        must(ww_clear_results(ctx), "clearresult");
        uint64_t stop = start + width;
        if (stop < start || stop > top) stop = top;
        enqueue_segment(ctx, start, stop, separate);  // warm
        must(ww_marker(ctx, 5), "marker");
        enqueue_segment(ctx, start, stop, separate);
        must(ww_marker(ctx, 6), "marker");
        must(ww_sync(ctx, 600000), "sync");
        float m = 0;
        must(ww_marker_elapsed(ctx, 5, 6, &m), "elapsed");
        ms = m;
        if (ms <= 0) ms = 1e-3;
        const double scale = target_ms / ms;
        if (scale < 1.25 && scale > 0.8) break;
        const double nw = (double)width * std::min(scale, 8.0);
        width = (uint64_t)std::min(nw, (double)kMaxRange);
        if (stop == top) break;
    }
    // then the sieve's segment shape and depth: one segment of the chosen
    // width timed for each, the fastest kept in the context (results do not
    // depend on either)
    uint64_t stop = start + std::min<uint64_t>(width, top - start);
    if (stop < start) stop = top;
    const int shapes[2] = {1, 2}, depths[4] = {20, 24, 26, 28};
    int best_shape = 0, best_depth = 20;
    float best = 0;
    for (int sh : shapes) {
        for (int d : depths) {
            must(ww_set_sieve_shape(ctx, sh), "sieve shape");
            must(ww_set_sieve_depth(ctx, d), "sieve depth");
            must(ww_clear_results(ctx), "clearresult");
            enqueue_segment(ctx, start, stop, separate);  // warm (and builds the depth's table)
            must(ww_marker(ctx, 5), "marker");
            enqueue_segment(ctx, start, stop, separate);
            must(ww_marker(ctx, 6), "marker");
            must(ww_sync(ctx, 600000), "sync");
            float m = 0;
            must(ww_marker_elapsed(ctx, 5, 6, &m), "elapsed");
            if (best == 0 || m < best) {
                best = m;
                best_shape = sh;
                best_depth = d;
            }
        }
    }
    must(ww_set_sieve_shape(ctx, best_shape), "sieve shape");
    must(ww_set_sieve_depth(ctx, best_depth), "sieve depth");
    must(ww_clear_results(ctx), "clearresult");
    fprintf(stderr, "Kernel profile: %0.3f ms. Worksize: %" PRIu64 ". Sieve shape %d, depth %d: %0.3f ms\n", ms, width,
            best_shape, best_depth, best);
    if (debug)
        printf("Kernel profile: %0.3f ms. Worksize: %" PRIu64 ". Sieve shape %d, depth %d: %0.3f ms\n", ms, width,
               best_shape, best_depth, best);
    return std::max<uint64_t>(width, 1ull << 20);
}

}  // namespace

int main(int argc, char **argv) {
    fprintf(stderr, "\nwwocl (B200 CUDA) -- a Wieferich and WallSunSun prime search program\n");
    printf("wwocl (B200 CUDA) -- a Wieferich and WallSunSun prime search program\n");
    fprintf(stderr, "Command line: ");
    for (int i = 0; i < argc; i++) fprintf(stderr, "%s ", argv[i]);
    fprintf(stderr, "\n");

    Options o = parse(argc, argv);
    const uint64_t bottom = o.bottom, top = o.top;
    fprintf(stderr, "Starting search at: %" PRIu64 "\nStopping search at: %" PRIu64 "\n", bottom, top);
    printf("Starting search at: %" PRIu64 "\nStopping search at: %" PRIu64 "\n", bottom, top);

    ww_ctx *ctx = nullptr;
    must(ww_open(o.device, &ctx), "open device");

    State st;
    bool write_a_next = true;
    if (read_state(o.files, bottom, top, st, write_a_next)) {  // main.cpp:1518-1541
        printf("Resuming search from checkpoint. Current: %" PRIu64 "\n", st.current);
        fprintf(stderr, "Resuming search from checkpoint. Current: %" PRIu64 "\n", st.current);
    } else {
        printf("Beginning a new search with parameters from the command line\n");
        st = State();
        st.current = bottom;
        write_a_next = true;
        if (!truncate_results(o.files)) {
            fprintf(stderr, "Cannot open %s !!!\n", o.files.results.c_str());
            exit(EXIT_FAILURE);
        }
    }
    if (st.current == top) {  // main.cpp:1544-1551
        printf("Workunit complete.\n");
        fprintf(stderr, "Workunit complete.\n");
        ww_close(ctx);
        boinc::finish(0);
    }

    const double target_ms = o.compute ? 100.0 : (o.ws ? (double)o.ws : 10.0);
    uint64_t calc_range = autotune(ctx, st.current, top, target_ms, o.separate, o.debug);
    if (o.ckpt_numbers) calc_range = std::min(calc_range, o.ckpt_numbers);
    const uint64_t mem_size = ww_prp_count_bound(0, calc_range);
    must(ww_reserve(ctx, mem_size, kNumResults), "reserve");
    if (o.debug) printf("segment width %" PRIu64 ", PRP buffer %" PRIu64 "\n", calc_range, mem_size);

    if (o.debug) {
        uint64_t k_stop = st.current + calc_range;
        if (k_stop > top || k_stop < st.current) k_stop = top;
        profile_kernels(ctx, st.current, k_stop);
    }
    self_test(ctx, st.current, top, calc_range, mem_size, o.debug, o.separate);

    fprintf(stderr, "Starting search...\n");
    printf("Starting search...\n");

    double last_progress = now_s(), last_ckpt = now_s();
    uint64_t since_ckpt = 0;
    must(ww_clear_results(ctx), "clearresult");
    int iter = 0;
    uint64_t stop = 0;
    for (uint64_t start = st.current; start < top; start = stop) {
        if (iter == 3) {  // keep at most three segments queued (main.cpp:1685-1691)
            must(ww_wait_marker(ctx, 0, 0), "wait");
            iter = 0;
        }
        stop = start + calc_range;
        if (stop > top || stop < start) stop = top;  // main.cpp:1693-1697
        if (o.ckpt_numbers) {
            const uint64_t room = o.ckpt_numbers - since_ckpt;
            if (stop - start > room) stop = start + room;
        }
        const double t = now_s();
        if (t - last_progress > 1.0) {  // main.cpp:1699-1708
            const double fd = (double)(start - bottom) / (double)(top - bottom);
            boinc::fraction_done(fd);
            if (boinc::is_standalone()) printf("Tests done: %.4f%%\n", fd * 100.0);
            last_progress = t;
        }
        nvtxRangePushA("segment");
        enqueue_segment(ctx, start, stop, o.separate);
        nvtxRangePop();
        if (iter == 0) must(ww_marker(ctx, 0), "marker");
        ++iter;
        since_ckpt += stop - start;
        if (o.testprimes) {
            must(ww_sync(ctx, 0), "sync");
            const uint32_t prpcnt = check_prps(ctx, start, stop, mem_size);
            printf("GPU primes match CPU (%u PRPs)\n", prpcnt);
        }
        const double ckpt_secs = now_s() - last_ckpt;
        const bool by_count = o.ckpt_numbers && since_ckpt >= o.ckpt_numbers;
        if (ckpt_secs > 60.0 || stop == top || by_count) {  // main.cpp:1743-1792
            must(ww_sync(ctx, 0), "sync");
            iter = 0;
            nvtxRangePushA("checkpoint");
            boinc::begin_critical_section();
            get_results(ctx, o, now_s() - last_ckpt, st, mem_size);
            if (stop == top) {
                char buffer[64];
                snprintf(buffer, sizeof buffer, "%016" PRIX64 "\n", st.cksm);
                if (!report_solution(o.files, buffer)) exit(EXIT_FAILURE);
                const double p_avg = st.pcnt ? st.psum / st.pcnt : 0.0;
                printf("Workunit complete. Average speed: %.2f Million primes per second.\n", p_avg);
                fprintf(stderr, "Workunit complete. Average speed: %.2f Million primes per second.\n", p_avg);
                printf("Checksum: %016" PRIX64 "\n", st.cksm);
                boinc::fraction_done(1.0);
            }
            st.current = stop;
            write_state(o.files, bottom, top, st, write_a_next);  // checkpoint(), main.cpp:212-221
            if (boinc::is_standalone()) printf("Checkpoint, current: %" PRIu64 "\n", stop);
            boinc::checkpoint_completed();
            boinc::end_critical_section();
            nvtxRangePop();
            last_ckpt = now_s();
            since_ckpt = 0;
            must(ww_clear_results(ctx), "clearresult");
        }
    }
    ww_close(ctx);
    boinc::finish(0);
}
