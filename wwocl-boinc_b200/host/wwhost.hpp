// wwhost.hpp -- host services of the wwocl program: A/B checkpoint files,
// the results file, the CPU prime list used to check the GPU PRP list, the
// split of a range over host threads, and a monotonic clock.  Behaviour follows the reference's main.cpp; every
// function cites the lines it mirrors.
#pragma once

#include <inttypes.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include "boinc_shim.hpp"
#include "wwcuda.h"

namespace wwhost {

struct Files {
    std::string results = "results-WW.txt";  // main.cpp:40
    std::string state_a = "stateA-WW.txt";   // main.cpp:41
    std::string state_b = "stateB-WW.txt";   // main.cpp:42
};

struct State {
    uint64_t current = 0, cksm = 0;
    double psum = 0.0;
    int pcnt = 0;
};

// write_state / read_state (main.cpp:103-209) live in the library
// (ww_state_write / ww_state_read) so the CPU tests can exercise them.
inline void write_state(const Files &f, uint64_t start, uint64_t stop, const State &s, bool &write_a_next) {
    ww_state st{s.current, s.cksm, s.psum, s.pcnt, 0};
    int a = write_a_next ? 1 : 0;
    const std::string fa = boinc::resolve_filename(f.state_a), fb = boinc::resolve_filename(f.state_b);
    if (ww_state_write(fa.c_str(), fb.c_str(), start, stop, &st, &a) != WW_OK)
        fprintf(stderr, "Cannot write state !!! Continuing... (%s)\n", ww_last_error());
    write_a_next = a != 0;
}

inline bool read_state(const Files &f, uint64_t start, uint64_t stop, State &s, bool &write_a_next) {
    ww_state st{};
    int a = 1;
    const std::string fa = boinc::resolve_filename(f.state_a), fb = boinc::resolve_filename(f.state_b);
    if (ww_state_read(fa.c_str(), fb.c_str(), start, stop, &st, &a) != 1) return false;
    s.current = st.current;
    s.cksm = st.cksm;
    s.psum = st.psum;
    s.pcnt = st.pcnt;
    write_a_next = a != 0;
    return true;
}

// report_solution (main.cpp:741-765): append and fsync.  Returns false on
// failure (the caller exits, as the reference does).
inline bool report_solution(const Files &f, const std::string &text) {
    FILE *r = boinc::fopen_resolved(f.results, "a");
    if (!r) {
        fprintf(stderr, "Cannot open %s !!!\n", f.results.c_str());
        return false;
    }
    if (fprintf(r, "%s", text.c_str()) < 0) {
        fprintf(stderr, "Cannot write to %s !!!\n", f.results.c_str());
        fclose(r);
        return false;
    }
    fflush(r);
    fsync(fileno(r));
    fclose(r);
    return true;
}

inline bool truncate_results(const Files &f) {
    FILE *r = boinc::fopen_resolved(f.results, "w");  // main.cpp:1535-1540
    if (!r) return false;
    fclose(r);
    return true;
}

// The primes of [lo, hi) for lo >= 127, the list primesieve produced in the
// reference's PRP check (main.cpp:498): numbers with no prime factor <= 113
// that pass the deterministic Miller-Rabin test.
// Splits [lo, hi) into contiguous pieces, one per host thread (at most 16,
// none shorter than 2^16 numbers), and runs f(a, b, i) on piece i = [a, b)
// in its own thread.  Returns the number of pieces.
template <class F>
inline unsigned parallel_pieces(uint64_t lo, uint64_t hi, F f) {
    if (hi <= lo) return 0;
    unsigned t = std::thread::hardware_concurrency();
    t = t < 1 ? 1 : (t > 16 ? 16 : t);
    const uint64_t span = hi - lo;
    const uint64_t by_size = span / 65536 + 1;
    const unsigned parts = (unsigned)(by_size < t ? by_size : t);
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < parts; ++i) {
        const uint64_t a = lo + span / parts * i;
        const uint64_t b = i + 1 == parts ? hi : lo + span / parts * (i + 1);
        pool.emplace_back([=, &f] { f(a, b, i); });
    }
    for (std::thread &th : pool) th.join();
    return parts;
}

// The primes of [lo, hi) with no factor up to 113 (the CPU side of
// checkPRPS, main.cpp:451-523), in increasing order; the pieces of the
// range are tested on all host threads.
inline std::vector<uint64_t> cpu_primes(uint64_t lo, uint64_t hi) {
    static const uint32_t small[29] = {3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53,
                                       59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113};
    std::vector<std::vector<uint64_t>> part(16);
    const unsigned parts = parallel_pieces(lo, hi, [&](uint64_t a, uint64_t b, unsigned i) {
        for (uint64_t n = a | 1; n < b && n >= a; n += 2) {
            bool sf = false;
            for (uint32_t r : small)
                if (n % r == 0) {
                    sf = true;
                    break;
                }
            if (!sf && ww_is_prime(n)) part[i].push_back(n);
            if (n > UINT64_MAX - 2) break;
        }
    });
    std::vector<uint64_t> out;
    for (unsigned i = 0; i < parts; ++i) out.insert(out.end(), part[i].begin(), part[i].end());
    return out;
}

inline double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace wwhost
