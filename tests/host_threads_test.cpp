// Host-side checks of hyalite_b200/csrc/host_threads.h, built and run by tests/test_host_threads.py:
// parallel_for covers every index exactly once (the worker pool repeatedly, from several threads
// at once, and nested); AsyncCopy copies two ranges laid end to end and widens int16 to int32,
// across many jobs, and in a child process made by fork() after its threads started.
#include <sys/wait.h>

#include <atomic>
#include <cstdio>
#include <random>
#include <thread>
#include <vector>

#include "host_threads.h"

using namespace hy;

static int failures = 0;
#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
            ++failures;                                            \
        }                                                          \
    } while (0)

static void cover(uint64_t n, uint64_t min_chunk) {
    std::vector<std::atomic<int>> hits(n);
    for (auto &h : hits) h.store(0);
    parallel_for(n, min_chunk, [&](uint64_t a, uint64_t e, unsigned) {
        for (uint64_t i = a; i < e; ++i) hits[i].fetch_add(1);
    });
    for (uint64_t i = 0; i < n; ++i) CHECK(hits[i].load() == 1);
}

int main() {
    for (int r = 0; r < 200; ++r) cover(1 + (uint64_t)r * 977, 1 + r % 7);
    {
        std::vector<std::thread> th;
        for (int t = 0; t < 6; ++t)
            th.emplace_back([t] {
                for (int r = 0; r < 50; ++r) cover(10000 + t * 31 + r, 64);
            });
        for (auto &x : th) x.join();
    }
    // A parallel loop inside a pool task runs on threads of its own.
    parallel_for(64, 1, [&](uint64_t a, uint64_t e, unsigned) {
        for (uint64_t i = a; i < e; ++i) cover(300 + i, 16);
    });

    std::mt19937_64 rng(7);
    AsyncCopy copier(3);
    for (int r = 0; r < 100; ++r) {
        const uint64_t n0 = rng() % (3u << 20), n1 = rng() % (3u << 20);
        std::vector<uint8_t> s0(n0 + 1), s1(n1 + 1), d0(n0 + 1, 0), d1(n1 + 1, 0);
        for (auto &x : s0) x = (uint8_t)rng();
        for (auto &x : s1) x = (uint8_t)rng();
        copier.start(d0.data(), s0.data(), n0, d1.data(), s1.data(), n1);
        copier.wait();
        CHECK(std::equal(s0.begin(), s0.begin() + n0, d0.begin()));
        CHECK(std::equal(s1.begin(), s1.begin() + n1, d1.begin()));
        CHECK(d0[n0] == 0 && d1[n1] == 0);  // nothing past the ranges
    }
    for (int r = 0; r < 20; ++r) {
        const uint64_t n = rng() % (2u << 20);
        std::vector<int16_t> src(n);
        std::vector<int32_t> dst(n + 1, 77);
        for (auto &x : src) x = (int16_t)rng();
        copier.start_widen(dst.data(), src.data(), n);
        copier.wait();
        for (uint64_t i = 0; i < n; ++i) CHECK(dst[i] == (int32_t)src[i]);
        CHECK(dst[n] == 77);
    }
    const pid_t child = fork();
    if (child == 0) {
        std::vector<uint8_t> s(5 << 20, 3), d(5 << 20, 0);
        copier.start(d.data(), s.data(), s.size() / 2, d.data() + s.size() / 2, s.data() + s.size() / 2,
                     s.size() / 2);
        copier.wait();
        bool ok = d == s;
        cover(100000, 128);
        std::_Exit(ok && failures == 0 ? 0 : 3);
    }
    int status = 0;
    waitpid(child, &status, 0);
    CHECK(WIFEXITED(status) && WEXITSTATUS(status) == 0);
    std::printf("%s\n", failures ? "FAIL" : "OK");
    return failures ? 1 : 0;
}
