// host_threads.h -- splitting host-side loops (validation, packing) over the host's threads.
#pragma once

#include <stdint.h>

#include <algorithm>
#include <thread>
#include <vector>

namespace hy {

// Runs f(begin, end) over [0, n) split across the host's threads.
template <class F>
inline void parallel_for(uint64_t n, uint64_t min_chunk, F f) {
    unsigned t = std::max(1u, std::thread::hardware_concurrency());
    t = (unsigned)std::min<uint64_t>(t, std::max<uint64_t>(1, n / std::max<uint64_t>(min_chunk, 1)));
    if (t <= 1) {
        f(0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    const uint64_t per = (n + t - 1) / t;
    for (unsigned i = 0; i < t; ++i) {
        const uint64_t a = i * per, e = std::min(n, a + per);
        if (a >= e) break;
        th.emplace_back(f, a, e, i);
    }
    for (auto &x : th) x.join();
}

inline unsigned host_threads(uint64_t n, uint64_t min_chunk) {
    unsigned t = std::max(1u, std::thread::hardware_concurrency());
    return (unsigned)std::min<uint64_t>(t, std::max<uint64_t>(1, n / std::max<uint64_t>(min_chunk, 1)));
}

// The first symbol of seq[0 .. len) that is >= alphabet_len, or -1: a branch-free maximum over
// the bytes (which the compiler vectorizes) and a scan for the offender only when there is one.
inline int first_bad_symbol(const uint8_t *seq, uint64_t len, uint64_t alphabet_len) {
    if (alphabet_len > 255) return -1;
    uint8_t mx = 0;
    for (uint64_t i = 0; i < len; ++i) mx = seq[i] > mx ? seq[i] : mx;
    if (mx < alphabet_len) return -1;
    for (uint64_t i = 0; i < len; ++i)
        if (seq[i] >= alphabet_len) return seq[i];
    return -1;
}

}  // namespace hy
