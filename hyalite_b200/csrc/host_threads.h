// host_threads.h -- splitting host-side loops (validation, packing) over the host's threads.
#pragma once

#include <stdint.h>

#include <pthread.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

namespace hy {

// A pool of host worker threads (one fewer than the host's hardware threads; the caller is the
// last), created on first use and kept for the process, so a parallel loop costs a wake-up rather
// than thread creation. One loop runs on the pool at a time; a loop issued while the pool is busy
// (another caller thread, or a loop inside a pool task) runs on threads of its own. A child made
// by fork() starts a new pool.
class HostPool {
  public:
    static HostPool *get() {
        static std::once_flag once;
        std::call_once(once, [] { pthread_atfork(nullptr, nullptr, [] { instance() = nullptr; }); });
        HostPool *&p = instance();
        static std::mutex make;
        std::lock_guard<std::mutex> lk(make);
        if (!p) p = new HostPool();  // kept for the process: workers wait on a condition at exit
        return p;
    }
    unsigned size() const { return (unsigned)workers_.size() + 1; }
    // Runs task(i) for i in [0, n_tasks) on the pool and the calling thread; false (nothing run)
    // when the pool is busy.
    template <class T>
    bool run(unsigned n_tasks, T &task) {
        if (in_task() || !busy_.try_lock()) return false;
        Job job;
        {
            std::lock_guard<std::mutex> lk(m_);
            job.call = [](void *ctx, unsigned i) { (*static_cast<T *>(ctx))(i); };
            job.ctx = &task;
            job.n = n_tasks;
            job.gen = ++gen_;
            job_ = job;
            left_.store(n_tasks);
            // Task indices are claimed from `next_`, whose high half names the job, so a worker
            // still holding an earlier job claims nothing from this one.
            next_.store(job.gen << 32);
        }
        cv_.notify_all();
        work(job);
        {
            std::unique_lock<std::mutex> lk(m_);
            done_.wait(lk, [&] { return left_.load() == 0; });
        }
        busy_.unlock();
        return true;
    }

  private:
    struct Job {
        void (*call)(void *, unsigned) = nullptr;
        void *ctx = nullptr;
        unsigned n = 0;
        uint64_t gen = 0;
    };
    HostPool() {
        const unsigned t = std::max(1u, std::thread::hardware_concurrency());
        for (unsigned i = 1; i < t; ++i)
            workers_.emplace_back([this] {
                in_task() = true;
                uint64_t seen = 0;
                for (;;) {
                    Job job;
                    {
                        std::unique_lock<std::mutex> lk(m_);
                        cv_.wait(lk, [&] { return gen_ != seen; });
                        seen = gen_;
                        job = job_;
                    }
                    work(job);
                }
            });
        for (auto &w : workers_) w.detach();
    }
    static HostPool *&instance() {
        static HostPool *p = nullptr;
        return p;
    }
    static bool &in_task() {
        static thread_local bool t = false;
        return t;
    }
    void work(const Job &job) {
        const bool was = in_task();
        in_task() = true;
        uint64_t cur = next_.load();
        for (;;) {
            if ((cur >> 32) != (job.gen & 0xffffffffu)) break;
            const unsigned i = (unsigned)cur;
            if (i >= job.n) break;
            if (!next_.compare_exchange_weak(cur, cur + 1)) continue;
            job.call(job.ctx, i);
            if (left_.fetch_sub(1) == 1) {
                std::lock_guard<std::mutex> lk(m_);
                done_.notify_all();
            }
            cur = next_.load();
        }
        in_task() = was;
    }
    std::vector<std::thread> workers_;
    std::mutex busy_, m_;
    std::condition_variable cv_, done_;
    Job job_;
    uint64_t gen_ = 0;
    std::atomic<uint64_t> next_{0};
    std::atomic<unsigned> left_{0};
};

// Copies up to two byte ranges on threads of its own while the caller goes on, one job at a time:
// start() hands the ranges over and returns, wait() returns once they are copied (start_widen():
// one range of int16 values widened to int32). In a process made by fork() after the threads
// started, both work synchronously (the threads are not there).
class AsyncCopy {
  public:
    explicit AsyncCopy(unsigned threads) : pid_(getpid()) {
        for (unsigned i = 0; i < std::max(1u, threads); ++i) workers_.emplace_back([this] { loop(); });
    }
    ~AsyncCopy() {
        if (getpid() != pid_) {
            for (auto &w : workers_) w.detach();
            return;
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &w : workers_) w.join();
    }
    void start(uint8_t *d0, const uint8_t *s0, uint64_t n0, uint8_t *d1, const uint8_t *s1, uint64_t n1) {
        if (getpid() != pid_) {
            if (n0) memcpy(d0, s0, n0);
            if (n1) memcpy(d1, s1, n1);
            return;
        }
        submit(Job{d0, s0, n0, d1, s1, n1, 0, 0, false});
    }
    void start_widen(int32_t *d, const int16_t *src, uint64_t n) {
        if (getpid() != pid_) {
            widen(d, src, n);
            return;
        }
        submit(Job{(uint8_t *)d, (const uint8_t *)src, 2 * n, nullptr, nullptr, 0, 0, 0, true});
    }
    void wait() {
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return left_.load() == 0; });
    }

  private:
    static constexpr uint64_t PIECE = 1 << 20;
    struct Job {
        uint8_t *d0;
        const uint8_t *s0;
        uint64_t n0;  // bytes (of the int16 source when widening)
        uint8_t *d1;
        const uint8_t *s1;
        uint64_t n1;
        uint64_t pieces;
        uint64_t gen;
        bool widen;
    };
    static void widen(int32_t *d, const int16_t *src, uint64_t n) {
        for (uint64_t i = 0; i < n; ++i) d[i] = src[i];
    }
    void submit(Job j) {
        j.pieces = (j.n0 + j.n1 + PIECE - 1) / PIECE;
        {
            std::lock_guard<std::mutex> lk(m_);
            j.gen = ++gen_;
            job_ = j;
            left_.store(j.pieces);
            next_.store(j.gen << 32);
        }
        if (j.pieces) cv_.notify_all();
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                j = job_;
            }
            uint64_t cur = next_.load();
            for (;;) {
                if ((cur >> 32) != (j.gen & 0xffffffffu)) break;
                const uint64_t i = cur & 0xffffffffu;
                if (i >= j.pieces) break;
                if (!next_.compare_exchange_weak(cur, cur + 1)) continue;
                // Piece i of the two ranges laid end to end (whole int16 values when widening).
                const uint64_t a = i * PIECE, e = std::min(j.n0 + j.n1, a + PIECE);
                if (j.widen)
                    widen((int32_t *)j.d0 + a / 2, (const int16_t *)j.s0 + a / 2, (e - a) / 2);
                else if (a < j.n0)
                    memcpy(j.d0 + a, j.s0 + a, std::min(e, j.n0) - a);
                if (!j.widen && e > j.n0) {
                    const uint64_t b = std::max(a, j.n0) - j.n0;
                    memcpy(j.d1 + b, j.s1 + b, e - j.n0 - b);
                }
                if (left_.fetch_sub(1) == 1) {
                    std::lock_guard<std::mutex> lk(m_);
                    done_.notify_all();
                }
                cur = next_.load();
            }
        }
    }
    const pid_t pid_;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    Job job_{};
    uint64_t gen_ = 0;
    bool stop_ = false;
    std::atomic<uint64_t> next_{0}, left_{0};
};

// Runs f(begin, end, part) over [0, n) split across the host's threads (at most one part per
// min_chunk elements).
template <class F>
inline void parallel_for(uint64_t n, uint64_t min_chunk, F f) {
    unsigned t = std::max(1u, std::thread::hardware_concurrency());
    t = (unsigned)std::min<uint64_t>(t, std::max<uint64_t>(1, n / std::max<uint64_t>(min_chunk, 1)));
    if (t <= 1) {
        f(0, n, 0);
        return;
    }
    const uint64_t per = (n + t - 1) / t;
    auto task = [&](unsigned i) {
        const uint64_t a = i * per, e = std::min(n, a + per);
        if (a < e) f(a, e, i);
    };
    if (HostPool::get()->run(t, task)) return;
    std::vector<std::thread> th;
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
