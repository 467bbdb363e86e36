// dropin_example.cpp -- the reference program's device loop rewired onto the
// kernel-shaped launchers of libwwcuda.so, the way a maintainer would change
// main.cpp: caller-owned device buffers in place of progData's cl_mem
// buffers (main.cpp:51-66, 1446-1493), one CUDA stream in place of the
// command queue, and one launcher call per sclSetKernelArg/sclEnqueueKernel
// pair (main.cpp:1704-1745).  Checkpoints, the results file and the CLI
// options stay with bin/wwocl; this program keeps only what the launchers
// replace, and prints the range's totals:
//
//   dropin_example START END [SEGMENT]
//   -> "prps N results N checksum %016llX"
//
// The checksum is the reference's: the per-segment device sums added up
// (main.cpp:799), printed as its results file's last line (main.cpp:1761).
#include <cuda_runtime.h>
#include <inttypes.h>
#include <stdio.h>
#include <stdlib.h>

#include "wwcuda.h"

namespace {

void must_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        exit(EXIT_FAILURE);
    }
}

void must(int rc, const char *what) {
    if (rc != WW_OK) {
        fprintf(stderr, "%s: %s (%s)\n", what, ww_status_string(rc), ww_last_error());
        exit(EXIT_FAILURE);
    }
}

// progData's device buffers (main.cpp:51-66)
struct DeviceBuffers {
    uint64_t *prime = nullptr, *invert = nullptr, *one = nullptr;
    uint64_t *special_prime = nullptr;
    int32_t *rem = nullptr, *quot = nullptr, *result = nullptr;
    uint64_t *checksum = nullptr, *total = nullptr;
    uint32_t *result_count = nullptr, *primecount = nullptr, *overflow = nullptr;
};

}  // namespace

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s START END [SEGMENT]\n", argv[0]);
        return EXIT_FAILURE;
    }
    uint64_t start = 0, top = 0, segment = 1ull << 30;
    must(ww_parse_number(argv[1], &start), "START");
    must(ww_parse_number(argv[2], &top), "END");
    if (argc > 3) must(ww_parse_number(argv[3], &segment), "SEGMENT");
    if (start < 127 || top <= start || segment == 0) {
        fprintf(stderr, "need 127 <= START < END and SEGMENT > 0\n");
        return EXIT_FAILURE;
    }
    const uint32_t numresults = 15000;                             // main.cpp:1119
    const uint64_t mem_size = ww_prp_count_bound(0, segment);     // the PRP buffer, as mem_size
    DeviceBuffers d;
    must_cuda(cudaMalloc(&d.prime, mem_size * 8), "prime buffer");
    must_cuda(cudaMalloc(&d.invert, mem_size * 8), "invert buffer");
    must_cuda(cudaMalloc(&d.one, mem_size * 16), "one buffer");
    must_cuda(cudaMalloc(&d.special_prime, numresults * 8), "hit buffer");
    must_cuda(cudaMalloc(&d.rem, numresults * 4), "hit buffer");
    must_cuda(cudaMalloc(&d.quot, numresults * 4), "hit buffer");
    must_cuda(cudaMalloc(&d.result, numresults * 4), "hit buffer");
    must_cuda(cudaMalloc(&d.checksum, 8), "counter");
    must_cuda(cudaMalloc(&d.total, 8), "counter");
    must_cuda(cudaMalloc(&d.result_count, 4), "counter");
    must_cuda(cudaMalloc(&d.primecount, 8), "counter");
    must_cuda(cudaMalloc(&d.overflow, 4), "counter");
    must_cuda(cudaMemset(d.overflow, 0, 4), "counter");
    cudaStream_t stream;
    must_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");

    // clearresult once per checkpoint interval (main.cpp:1791); here, once
    must(ww_launch_clearresult(d.checksum, d.result_count, d.total, d.primecount, stream), "clearresult");
    for (uint64_t current = start; current < top;) {
        uint64_t stop = current + segment;
        if (stop > top || stop < current) stop = top;
        uint64_t ks = current;
        int32_t wheelidx = 0;
        // findWheelOffset (main.cpp:1716); nothing prime to 30 is left below 2^64
        if (ww_find_wheel_offset(&ks, &wheelidx) != WW_OK) break;
        if (ks < stop) {
            must(ww_launch_clearn(d.primecount, stream), "clearn");                      // main.cpp:1711
            must(ww_launch_getsegprimes(ks, stop, wheelidx, d.prime, d.invert, d.primecount, mem_size,
                                        d.overflow, stream),
                 "getsegprimes");                                                         // main.cpp:1719-1727
            must(ww_launch_wieferich(d.primecount, d.prime, d.invert, d.one, d.special_prime, d.rem, d.quot,
                                     d.result, d.checksum, d.result_count, d.total, mem_size, numresults,
                                     d.overflow, stream),
                 "wieferich");                                                            // main.cpp:1738
            must(ww_launch_wallsunsun(d.primecount, d.prime, d.invert, d.one, d.special_prime, d.rem, d.quot,
                                      d.result, d.checksum, d.result_count, mem_size, numresults, d.overflow,
                                      stream),
                 "wallsunsun");                                                           // main.cpp:1741
        }
        current = stop;
    }
    uint64_t checksum = 0, total = 0;
    uint32_t results = 0, overflow = 0;
    must_cuda(cudaMemcpyAsync(&checksum, d.checksum, 8, cudaMemcpyDeviceToHost, stream), "read back");
    must_cuda(cudaMemcpyAsync(&total, d.total, 8, cudaMemcpyDeviceToHost, stream), "read back");
    must_cuda(cudaMemcpyAsync(&results, d.result_count, 4, cudaMemcpyDeviceToHost, stream), "read back");
    must_cuda(cudaMemcpyAsync(&overflow, d.overflow, 4, cudaMemcpyDeviceToHost, stream), "read back");
    must_cuda(cudaStreamSynchronize(stream), "sync");
    if (overflow) {  // main.cpp:802-814 stop the program on either overflow
        fprintf(stderr, "buffer overflow (flags %u)\n", overflow);
        return EXIT_FAILURE;
    }
    printf("prps %" PRIu64 " results %u checksum %016" PRIX64 "\n", total, results, checksum);

    cudaStreamDestroy(stream);
    cudaFree(d.prime);
    cudaFree(d.invert);
    cudaFree(d.one);
    cudaFree(d.special_prime);
    cudaFree(d.rem);
    cudaFree(d.quot);
    cudaFree(d.result);
    cudaFree(d.checksum);
    cudaFree(d.total);
    cudaFree(d.result_count);
    cudaFree(d.primecount);
    cudaFree(d.overflow);
    return EXIT_SUCCESS;
}
