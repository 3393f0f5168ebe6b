// pairs.cu -- align_pairs (src/kernel.rs:429-452) on the device.
//
// Every pair has its own query and target. The reference validates pairs in input order exactly
// like align_pair_with (src/kernel.rs:354-415): symbols of the query then the target, then the
// width proof on the pair's own lengths; the first failure ends the batch. Here the host checks
// what depends on lengths only (the width proof and the routing) over all pairs, and the device
// checks the symbols while it packs; the first failure in input order is then re-derived for the
// one pair where it lies, so the error, its details and the prefix of results are the reference's.
//
// The accepted pairs run in chunks of input order. For each chunk the host sorts the pairs by
// (query length, target length), groups two pairs of EQUAL query length per int16x2 item (both
// halves share one row structure) and copies the chunk's raw residues and offsets into a pinned
// staging slot; a copy stream moves them to the device while the compute stream packs and aligns
// the previous chunk. Results do not depend on the order, only the speed does. Rows per lane are
// chosen per query length so that a pass (8 lanes x rows) wastes the fewest padded rows; items of
// one choice run in one launch.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

#include "db_internal.h"
#include "host_common.h"
#include "scan_kernel.cuh"
#include "traceback_internal.h"
#include "host_threads.h"

using namespace hy;

namespace hy {

constexpr int PAIR_G = 8;
constexpr int PAIR_R32 = 16;
constexpr size_t PAIR_SMEM_LIMIT = 200 * 1024;
// Largest global scratch for group profiles that do not fit in shared memory, per launch.
constexpr size_t PAIR_GPROF_BYTES = 256ull << 20;
// Chunks of input pairs the pipeline runs in: up to PAIR_MAX_CHUNKS of at least PAIR_CHUNK_MIN
// pairs each, and more when that would put over PAIR_CHUNK_BYTES of residues in one chunk (the
// pinned staging holds three chunks).
constexpr uint64_t PAIR_MAX_CHUNKS = 16;
constexpr uint64_t PAIR_CHUNK_MIN = 1 << 16;
constexpr uint64_t PAIR_CHUNK_BYTES = 512ull << 20;
// The chunk boundaries of pairs [0, L): cut at equal shares of the residues (query plus target
// bytes), so that no chunk holds much more than PAIR_CHUNK_BYTES whatever the order of long and
// short pairs (one pair is never split); every chunk gets at least one pair.
static std::vector<uint64_t> plan_pair_chunks(const uint64_t *q_off, const uint64_t *t_off, uint64_t L) {
    auto residues = [&](uint64_t a) { return (q_off[a] - q_off[0]) + (t_off[a] - t_off[0]); };
    const uint64_t total = residues(L);
    const uint64_t n_chunks = std::min<uint64_t>(
        L, std::max<uint64_t>({1, std::min<uint64_t>(PAIR_MAX_CHUNKS, L / PAIR_CHUNK_MIN),
                               (total + PAIR_CHUNK_BYTES - 1) / PAIR_CHUNK_BYTES}));
    std::vector<uint64_t> b(n_chunks + 1, 0);
    b[n_chunks] = L;
    for (uint64_t c = 1; c < n_chunks; ++c) {
        const uint64_t target = (uint64_t)((unsigned __int128)total * c / n_chunks);
        uint64_t lo = 0, hi = L;  // first a with residues(a) >= target
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (residues(mid) >= target) hi = mid; else lo = mid + 1;
        }
        b[c] = std::min(std::max(lo, b[c - 1] + 1), L - (n_chunks - c));
    }
    return b;
}

// Pinned staging slots the chunks rotate through.
constexpr int PAIR_SLOTS = 3;
// Most warps (128-row stripes) the long pairs of one call may take on the stripe kernel.
constexpr uint64_t LONG_PAIR_MAX_STRIPES = 2048;
// Rows per lane the int16x2 pair kernel is compiled for.
constexpr int PAIR_ROWS[] = {8, 12, 16, 20, 24, 32};

// Per-pair routing from the lengths pass.
constexpr uint8_t PAIR_I32 = 1;   // the width proof needs int32 lanes
constexpr uint8_t PAIR_LONG = 2;  // a long single pair (the stripe kernel, if the call takes it)

// Grow-only host array (no zeroing: every element read is written first in the same call).
template <class T>
struct HostArr {
    std::unique_ptr<T[]> p;
    size_t n = 0;
    T *get(size_t want) {
        want = std::max<size_t>(want, 1);
        if (n < want) {
            p.reset(new T[want]);
            n = want;
        }
        return p.get();
    }
};

// Device buffer slots of a PairsContext.
enum PairSlot {
    PS_Q = 0,    // raw query residues at their q_off positions
    PS_T,        // raw target residues at their t_off positions
    PS_QOFF,     // q_off[0 .. n] of the accepted pairs
    PS_TOFF,     // t_off[0 .. n]
    PS_META16,   // int16x2 items of the whole call (ItemMeta), then their query lengths and offsets
    PS_QLEN16,
    PS_IQOFF16,
    PS_RES16,    // one chunk's packed target columns
    PS_BND16,    // one chunk's boundary rows (queries longer than one pass)
    PS_META32,   // the same for int32 items
    PS_QLEN32,
    PS_IQOFF32,
    PS_RES32,
    PS_BND32,
    PS_MATRIX,
    PS_OUT,      // scores, query ends, target ends per pair, the first bad-symbol pair, score2 pairs
    PS_GPROF,    // group profiles in global memory (large alphabets)
    PS_ITOFF16,  // position maxima: items' target offsets per half
    PS_ITOFF32,
    PS_COLMAX,   // position maxima: column maxima at the targets' offsets
    PS_CM16,     // position maxima: one chunk's column maxima narrowed for the copy back
    PS_COUNT
};

// Grow-only device, pinned and host buffers of the calling thread, reused across its calls.
struct PairsContext {
    int device = -1;
    cudaStream_t stream = nullptr;       // packing kernels, pair kernels, results
    cudaStream_t copy_stream = nullptr;  // host-to-device copies of the chunks
    cudaStream_t d2h_stream = nullptr;   // position maxima: each chunk's column maxima back
    std::vector<cudaEvent_t> ev;         // around each chunk's device work, then its copy back
    cudaEvent_t slot_ev[PAIR_SLOTS] = {};
    struct Buf {
        void *p = nullptr;
        size_t n = 0;
    };
    Buf b[PS_COUNT];
    Buf pinned[PAIR_SLOTS + 2];  // the staging ring, the results, the column maxima
    double kernel_ms = 0.0, call_ms = 0.0;  // the last call: device time of its kernels, whole call
    // The last call's phases (ms): the lengths pass and routing, host sort and item packing, host
    // staging copies, the chunk pipeline (wall time to the device's end), results, host waits for
    // a staging slot, host copies of the column maxima into the caller's array (position maxima).
    double phase_ms[7] = {0, 0, 0, 0, 0, 0, 0};
    ~PairsContext() {
        for (auto &x : b) hy::dev_free(x.p);
        for (auto &x : pinned) cudaFreeHost(x.p);
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        for (cudaEvent_t e : slot_ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (d2h_stream) cudaStreamDestroy(d2h_stream);
    }
    cudaError_t get_pinned(int slot, size_t bytes, void **out) {
        bytes = std::max<size_t>(bytes, 16);
        if (pinned[slot].n < bytes) {
            cudaFreeHost(pinned[slot].p);
            pinned[slot].p = nullptr;
            pinned[slot].n = 0;
            cudaError_t e = cudaMallocHost(&pinned[slot].p, bytes);
            if (e != cudaSuccess) return e;
            pinned[slot].n = bytes;
        }
        *out = pinned[slot].p;
        return cudaSuccess;
    }
    // Device buffer of at least `bytes`. Growing a buffer the compute stream may still be reading
    // first waits for that stream.
    cudaError_t get(int slot, size_t bytes, void **out) {
        bytes = std::max<size_t>(bytes, 16);
        if (b[slot].n < bytes) {
            if (stream) {
                cudaError_t e = cudaStreamSynchronize(stream);
                if (e != cudaSuccess) return e;
            }
            hy::dev_free(b[slot].p);
            b[slot].p = nullptr;
            b[slot].n = 0;
            cudaError_t e = hy::dev_malloc(&b[slot].p, bytes);
            if (e != cudaSuccess) return e;
            b[slot].n = bytes;
        }
        *out = b[slot].p;
        return cudaSuccess;
    }
};

static thread_local PairsContext g_ctx;

// Grow-only host arrays of the calling thread: per-pair routes, a chunk's sort and item arrays.
struct PairsHost {
    HostArr<uint8_t> route;
    HostArr<uint32_t> ord[2], ord_tmp, start, qlen[4];  // qlen: two chunks x two arithmetics
    HostArr<uint64_t> keys[2], keys_tmp;
    std::vector<std::vector<uint64_t>> count;  // radix histograms, one per host thread
    // Copies a chunk's residues into its staging slot while the next chunk is sorted and packed;
    // the second copies column maxima back into the caller's array.
    std::unique_ptr<AsyncCopy> copier, cm_copier;
};

// Position maxima into a pageable caller array over several chunks: a thread of its own waits for
// each issued chunk's column maxima to reach the pinned copy and moves them into the caller's
// array while the calling thread prepares and issues later chunks.
class ColmaxDrainer {
  public:
    ColmaxDrainer(int device, uint64_t n_chunks, AsyncCopy &cp, const std::vector<cudaEvent_t> &ev,
                  uint64_t ev_base, std::function<void(uint64_t, uint64_t *, uint64_t *)> range,
                  int32_t *dst, const int32_t *src, const std::vector<char> &narrow)
        : n_(n_chunks), cp_(cp) {
        th_ = std::thread([=, &ev, &narrow] {
            cudaSetDevice(device);
            for (uint64_t c = 0; c < n_; ++c) {
                {
                    std::unique_lock<std::mutex> lk(m_);
                    cv_.wait(lk, [&] { return stop_ || issued_ > (int64_t)c; });
                    if (stop_ && issued_ <= (int64_t)c) return;
                }
                if (cudaEventSynchronize(ev[ev_base + c]) != cudaSuccess) {
                    cudaGetLastError();
                    failed_ = true;
                    return;
                }
                const auto t0 = std::chrono::steady_clock::now();
                uint64_t x0, x1;
                range(c, &x0, &x1);
                // A narrowed chunk's int16 maxima sit at the start of its region of the pinned copy.
                if (narrow[c])
                    cp_.start_widen(dst + x0, (const int16_t *)(src + x0), x1 - x0);
                else
                    cp_.start((uint8_t *)(dst + x0), (const uint8_t *)(src + x0), 4 * (x1 - x0), nullptr, nullptr, 0);
                cp_.wait();
                ms_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            }
        });
    }
    // Chunk c's copy back is enqueued (its event recorded).
    void issued(uint64_t c) {
        {
            std::lock_guard<std::mutex> lk(m_);
            issued_ = (int64_t)c + 1;
        }
        cv_.notify_one();
    }
    // Waits for the thread (after every chunk, or, on an early return, after the issued ones).
    double join(bool *ok) {
        if (th_.joinable()) {
            {
                std::lock_guard<std::mutex> lk(m_);
                stop_ = true;
            }
            cv_.notify_one();
            th_.join();
        }
        if (ok) *ok = !failed_;
        return ms_;
    }
    ~ColmaxDrainer() { join(nullptr); }

  private:
    const uint64_t n_;
    AsyncCopy &cp_;
    std::thread th_;
    std::mutex m_;
    std::condition_variable cv_;
    int64_t issued_ = 0;
    bool stop_ = false;
    std::atomic<bool> failed_{false};
    double ms_ = 0.0;
};

// One chunk of pairs between its host preparation and its issue to the device.
struct ChunkState {
    uint64_t c, a, b, n, qb, tb;
    int s;  // staging slot
    uint8_t *slot;
    uint64_t *s_qoff, *s_toff;
    ItemMeta *s_meta[2];
    size_t n_items[2];
    uint64_t cols[2];
    uint32_t *qlen[2];
    bool narrow;  // position maxima: the chunk's column maxima go back as int16
};

static thread_local PairsHost g_host;

#define HY_CK(call)                                                                                \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            cudaGetLastError();                                                                    \
            return fail(e_ == cudaErrorMemoryAllocation ? HY_ERR_OUT_OF_MEMORY : HY_ERR_CUDA, e_); \
        }                                                                                          \
    } while (0)

template <class A, int G, int R, int MODE, bool ENDS, bool GPROF, bool COLMAX = false>
static cudaError_t launch_pairs_mode(const PairParams &p, int blocks, int threads, size_t smem,
                                     cudaStream_t st) {
    auto kern = pairs_kernel<A, G, R, MODE, ENDS, GPROF, COLMAX>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        // All shared memory: the blocks' group profiles decide how many fit on an SM.
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
    }
    kern<<<blocks, threads, smem, st>>>(p);
    return cudaGetLastError();
}

// The form with group profiles in global memory (p.gprof set): only the smallest row shape of
// each lane arithmetic, which is what a large alphabet runs. p.colmax set: the column-maxima form
// (local mode, score only).
template <class A, int G, int R>
static cudaError_t launch_pairs_gprof(int mode, bool ends, const PairParams &p, int blocks,
                                      int threads, cudaStream_t st) {
    if constexpr ((A::NH == 2 && R == 8) || (A::NH == 1 && R == PAIR_R32)) {
        if (p.colmax) return launch_pairs_mode<A, G, R, MODE_SW, false, true, true>(p, blocks, threads, 0, st);
#define HY_MODE_CASE(M)                                                                     \
    case M:                                                                                 \
        return ends ? launch_pairs_mode<A, G, R, M, true, true>(p, blocks, threads, 0, st)  \
                    : launch_pairs_mode<A, G, R, M, false, true>(p, blocks, threads, 0, st);
        switch (mode) {
            HY_MODE_CASE(MODE_SW)
            HY_MODE_CASE(MODE_NW)
            HY_MODE_CASE(MODE_HW)
            HY_MODE_CASE(MODE_OV)
            HY_MODE_CASE(MODE_SHW)
        }
#undef HY_MODE_CASE
    }
    return cudaErrorInvalidValue;
}

template <class A, int G, int R>
static cudaError_t launch_pairs(int mode, bool ends, const PairParams &p, int blocks, int threads,
                                size_t smem, cudaStream_t st) {
    if (p.gprof) return launch_pairs_gprof<A, G, R>(mode, ends, p, blocks, threads, st);
    if (p.colmax) return launch_pairs_mode<A, G, R, MODE_SW, false, false, true>(p, blocks, threads, smem, st);
#define HY_MODE_CASE(M)                                                                        \
    case M:                                                                                    \
        return ends ? launch_pairs_mode<A, G, R, M, true, false>(p, blocks, threads, smem, st) \
                    : launch_pairs_mode<A, G, R, M, false, false>(p, blocks, threads, smem, st);
    switch (mode) {
        HY_MODE_CASE(MODE_SW)
        HY_MODE_CASE(MODE_NW)
        HY_MODE_CASE(MODE_HW)
        HY_MODE_CASE(MODE_OV)
        HY_MODE_CASE(MODE_SHW)
    }
#undef HY_MODE_CASE
    return cudaErrorInvalidValue;
}

template <class A, int G>
static cudaError_t launch_pairs_rows(int rows, int mode, bool ends, const PairParams &p, int blocks,
                                     int threads, size_t smem, cudaStream_t st) {
    if constexpr (A::NH == 2) {
        switch (rows) {
        case 8: return launch_pairs<A, G, 8>(mode, ends, p, blocks, threads, smem, st);
        case 12: return launch_pairs<A, G, 12>(mode, ends, p, blocks, threads, smem, st);
        case 16: return launch_pairs<A, G, 16>(mode, ends, p, blocks, threads, smem, st);
        case 20: return launch_pairs<A, G, 20>(mode, ends, p, blocks, threads, smem, st);
        case 24: return launch_pairs<A, G, 24>(mode, ends, p, blocks, threads, smem, st);
        case 32: return launch_pairs<A, G, 32>(mode, ends, p, blocks, threads, smem, st);
        }
        return cudaErrorInvalidValue;
    } else {
        (void)rows;
        return launch_pairs<A, G, PAIR_R32>(mode, ends, p, blocks, threads, smem, st);
    }
}

// Shared memory of an SM (B200), and what each resident block reserves of it.
constexpr size_t SM_SMEM = 228 * 1024, BLOCK_SMEM_RESERVE = 1024;

// Groups per block of the pair kernel for group profiles of gb bytes: up to 256 threads, whole
// warps, within PAIR_SMEM_LIMIT; 0 when not one warp of groups fits (the global-profile form).
static int pair_groups_per_block(size_t gb, int G) {
    int g = (int)std::min<size_t>(256 / G, PAIR_SMEM_LIMIT / gb);
    return g / (32 / G) * (32 / G);
}

// Warps of pair-kernel groups one SM holds with group profiles of gb bytes: as many blocks as its
// shared memory and registers (at most 128 a thread) allow.
static double pair_resident_warps(size_t gb, int G) {
    const int gpb = pair_groups_per_block(gb, G);
    if (gpb == 0) return 0.0;
    const size_t by_smem = SM_SMEM / ((size_t)gpb * gb + BLOCK_SMEM_RESERVE);
    const size_t by_regs = 65536 / ((size_t)gpb * G * 128);
    return (double)std::min(by_smem, by_regs) * gpb * G / 32.0;
}

// Rows per lane for an int16x2 item of query length q: the least estimated time over the pass
// shapes, counting the padded rows of the last pass, the per-step work shared by a lane's rows,
// and the warps an SM holds (each group keeps its own query profile in shared memory, so more rows
// per lane means fewer resident warps; about 12 warps keep the pipes busy). Ties go to more rows.
static int pair_rows(uint64_t q, int32_t al) {
    int best = 8;
    double best_cost = 1e300;
    for (int r : PAIR_ROWS) {
        const size_t gb = (size_t)(al + 1) * PAIR_G * r * profile_row_bytes<Pair16H>();
        const double w = pair_resident_warps(gb, PAIR_G);
        if (w <= 0.0) continue;
        const uint64_t rpp = (uint64_t)PAIR_G * r;
        const double pad = (double)((q + rpp - 1) / rpp * rpp);
        const double cost = pad * (r + 6.0) / r / std::min(1.0, w / 12.0);
        if (cost <= best_cost) {
            best_cost = cost;
            best = r;
        }
    }
    return best;
}

// Packs the target columns of the int16x2 or int32 items [i0, i1) of one chunk (item columns run
// from meta.col_off to the next item's col_off, the last item's to col_end): an int16x2 item keeps
// pair 0 in the low byte and pair 1 in the high byte, the shorter padded with symbol `al`; an
// int32 item one byte a column, padded with 0. Writes each item's query length and query offsets
// (and, for column maxima, target offsets), and checks every residue of the items' queries and targets against the alphabet: a symbol
// >= al records its pair in *bad (the smallest such pair wins) and is replaced by a valid code, so
// no kernel indexes a profile or the matrix with it. Such pairs are at or past the batch's first
// failure, and their results are never returned. One warp an item.
template <class A>
__global__ void __launch_bounds__(256) pack_items_kernel(const ItemMeta *meta, uint32_t i0, uint32_t i1,
                                                         uint64_t col_end, const uint64_t *q_off,
                                                         const uint64_t *t_off, uint8_t *q_res,
                                                         const uint8_t *t_res, typename A::RES *res,
                                                         uint32_t *qlen, uint64_t *iqoff, uint64_t *itoff,
                                                         uint32_t al, uint32_t *bad) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t it = i0 + (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); it < i1; it += n_warps) {
        const ItemMeta m = meta[it];
        const uint64_t end = it + 1 < i1 ? meta[it + 1].col_off : col_end;
        const bool two = A::NH == 2 && m.idx[1] != NO_INDEX;
        const uint8_t *t0 = t_res + t_off[m.idx[0]];
        const uint8_t *t1 = two ? t_res + t_off[m.idx[1]] : t0;
        typename A::RES *out = res + m.col_off;
        bool bad0 = false, bad1 = false;
        for (uint64_t j = lane; j < end - m.col_off; j += 32) {
            if constexpr (A::NH == 2) {
                uint32_t lo = al, hi = al;
                if (j < m.n[0]) {
                    lo = t0[j];
                    if (lo >= al) bad0 = true, lo = al;
                }
                if (two && j < m.n[1]) {
                    hi = t1[j];
                    if (hi >= al) bad1 = true, hi = al;
                }
                out[j] = (typename A::RES)(lo | (hi << 8));
            } else {
                uint32_t v = 0;
                if (j < m.n[0]) {
                    v = t0[j];
                    if (v >= al) bad0 = true, v = 0;
                }
                out[j] = (typename A::RES)v;
            }
        }
        for (int h = 0; h < (two ? 2 : 1); ++h) {
            const uint64_t qa = q_off[m.idx[h]], ql = q_off[m.idx[h] + 1] - qa;
            bool bq = false;
            for (uint64_t i = lane; i < ql; i += 32)
                if (q_res[qa + i] >= al) bq = true, q_res[qa + i] = 0;
            (h == 0 ? bad0 : bad1) |= bq;
        }
        bad0 = __any_sync(0xffffffffu, bad0);
        bad1 = __any_sync(0xffffffffu, bad1);
        if (lane == 0) {
            const uint64_t qa = q_off[m.idx[0]];
            qlen[it] = (uint32_t)(q_off[m.idx[0] + 1] - qa);
            iqoff[2 * it] = qa;
            iqoff[2 * it + 1] = two ? q_off[m.idx[1]] : qa;
            if (itoff) {
                itoff[2 * it] = t_off[m.idx[0]];
                itoff[2 * it + 1] = two ? t_off[m.idx[1]] : t_off[m.idx[0]];
            }
            if (bad0) atomicMin(bad, m.idx[0]);
            if (bad1) atomicMin(bad, m.idx[1]);
        }
    }
}

// Sort keys: complemented query length above complemented target length, so ascending keys are
// query length desc, then target length desc.
static inline uint64_t shape_key(uint64_t ql, uint64_t tl) {
    return ((uint64_t)~(uint32_t)ql << 32) | ~(uint32_t)tl;
}
static inline uint32_t key_qlen(uint64_t k) { return ~(uint32_t)(k >> 32); }
static inline uint32_t key_tlen(uint64_t k) { return ~(uint32_t)k; }

// Sorts n pair indices (ascending on entry) with their keys: a stable LSD radix sort on 8-bit
// digits, skipping digits every key shares (lengths of one workload differ in a few low bits); histograms and scatters on all host threads
// (per-thread ranges in order keep it stable). o / keys end up pointing at the sorted arrays
// (either the given ones or the scratch ones, which are swapped with them).
static void sort_by_shape(PairsHost &hs, uint32_t *&o, uint64_t *&keys, uint32_t *&o_tmp,
                          uint64_t *&k_tmp, size_t n) {
    if (n < 2) return;
    const unsigned nt = host_threads(n, 1 << 14);
    const uint64_t per = (n + nt - 1) / nt;
    if (hs.count.size() < nt) hs.count.resize(nt);
    for (unsigned t = 0; t < nt; ++t) hs.count[t].resize(256);
    // Bits in which some key differs from the first: digits without any are skipped.
    std::vector<uint64_t> diff(nt, 0);
    parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
        for (uint64_t t = ta; t < te; ++t) {
            uint64_t acc = 0;
            for (uint64_t i = t * per; i < std::min<uint64_t>(n, (t + 1) * per); ++i) acc |= keys[i] ^ keys[0];
            diff[t] = acc;
        }
    });
    uint64_t varies = 0;
    for (uint64_t x : diff) varies |= x;
    for (int shift = 0; shift < 64; shift += 8) {
        if (((varies >> shift) & 0xff) == 0) continue;
        parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
            for (uint64_t t = ta; t < te; ++t) {
                std::vector<uint64_t> &c = hs.count[t];
                std::fill(c.begin(), c.end(), 0);
                for (uint64_t i = t * per; i < std::min<uint64_t>(n, (t + 1) * per); ++i)
                    ++c[(keys[i] >> shift) & 0xff];
            }
        });
        uint64_t sum = 0;
        for (size_t d = 0; d < 256; ++d)
            for (unsigned t = 0; t < nt; ++t) {
                const uint64_t c = hs.count[t][d];
                hs.count[t][d] = sum;
                sum += c;
            }
        parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
            for (uint64_t t = ta; t < te; ++t) {
                std::vector<uint64_t> &c = hs.count[t];
                for (uint64_t i = t * per; i < std::min<uint64_t>(n, (t + 1) * per); ++i) {
                    const uint64_t dst = c[(keys[i] >> shift) & 0xff]++;
                    o_tmp[dst] = o[i];
                    k_tmp[dst] = keys[i];
                }
            }
        });
        std::swap(o, o_tmp);
        std::swap(keys, k_tmp);
    }
}

// Groups n sorted pairs into items (an int16x2 item takes two consecutive pairs of equal query
// length) and writes their ItemMeta (columns from 0 within the chunk, each item's padded to
// `align`) and query lengths; returns the item count and sets *cols. Boundaries come from one
// sequential pass over the keys; the items are filled, and their column offsets prefix-summed, on
// all host threads.
static size_t pack_items(PairsHost &hs, const uint32_t *order, const uint64_t *keys, size_t n,
                         bool two, ItemMeta *meta, uint32_t *qlen, uint64_t *cols) {
    const uint64_t align = two ? 8 : 16;
    uint32_t *start = hs.start.get(n + 1);
    size_t n_items = 0;
    for (size_t i = 0; i < n;) {
        start[n_items++] = (uint32_t)i;
        i += (two && i + 1 < n && key_qlen(keys[i + 1]) == key_qlen(keys[i])) ? 2 : 1;
    }
    start[n_items] = (uint32_t)n;
    const unsigned nt = host_threads(n_items, 1 << 14);
    const uint64_t per = (n_items + nt - 1) / nt;
    std::vector<uint64_t> part(nt + 1, 0);
    parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
        for (uint64_t t = ta; t < te; ++t) {
            uint64_t c = 0;
            for (uint64_t it = t * per; it < std::min<uint64_t>(n_items, (t + 1) * per); ++it) {
                const size_t i = start[it];
                const bool pair = start[it + 1] - i == 2;
                ItemMeta &m = meta[it];
                m.pad_ = 0;
                m.idx[0] = order[i];
                m.n[0] = key_tlen(keys[i]);
                m.idx[1] = pair ? order[i + 1] : NO_INDEX;
                m.n[1] = pair ? key_tlen(keys[i + 1]) : 0;
                m.w = std::max(m.n[0], m.n[1]);
                m.col_off = c;  // within this thread's range; shifted below
                c += (m.w + align - 1) / align * align;
                qlen[it] = key_qlen(keys[i]);
            }
            part[t + 1] = c;
        }
    });
    for (unsigned t = 0; t < nt; ++t) part[t + 1] += part[t];
    parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
        for (uint64_t t = ta; t < te; ++t)
            for (uint64_t it = t * per; it < std::min<uint64_t>(n_items, (t + 1) * per); ++it)
                meta[it].col_off += part[t];
    });
    *cols = part[nt];
    return n_items;
}

// Packs and aligns one chunk's items of one lane arithmetic: the packing kernel, then one launch
// per run of items with the same rows per lane (items are sorted by query length). Items
// [ib, ib + n_items) of the call; qlen (host) their query lengths; cols the chunk's columns.
template <class A, int G>
static hy_status run_items(PairsContext &ctx, PairParams p, int res_slot, int bnd_slot,
                           const uint32_t *qlen, size_t ib, size_t n_items, uint64_t cols,
                           const uint64_t *d_qoff, const uint64_t *d_toff, uint8_t *d_q,
                           const uint8_t *d_t, uint32_t *d_bad, int mode, bool ends) {
    if (n_items == 0) return fail(HY_OK);
    constexpr bool two = A::NH == 2;
    void *d_res;
    HY_CK(ctx.get(res_slot, cols * sizeof(typename A::RES), &d_res));
    {
        const int blocks = (int)std::min<uint64_t>((n_items + 7) / 8, 148 * 16);
        pack_items_kernel<A><<<blocks, 256, 0, ctx.stream>>>(
            p.meta, (uint32_t)ib, (uint32_t)(ib + n_items), cols, d_qoff, d_toff, d_q, d_t,
            (typename A::RES *)d_res, const_cast<uint32_t *>(p.qlen), const_cast<uint64_t *>(p.qoff),
            const_cast<uint64_t *>(p.toff), (uint32_t)p.al, d_bad);
        HY_CK(cudaGetLastError());
    }
    // Rows per lane of each run of equal query lengths.
    auto rows_of = [&](uint32_t q) { return two ? pair_rows(q, p.al) : PAIR_R32; };
    bool multipass = false;
    for (size_t i = 0; i < n_items;) {
        size_t j = i;
        while (j < n_items && qlen[j] == qlen[i]) ++j;
        multipass = multipass || qlen[i] > (uint32_t)(G * rows_of(qlen[i]));
        i = j;
    }
    void *d_bnd = nullptr;
    if (multipass) HY_CK(ctx.get(bnd_slot, 2 * sizeof(typename A::V) * cols, &d_bnd));
    p.res = d_res;
    p.boundary = d_bnd;
    p.gprof = nullptr;
    for (size_t i0 = 0; i0 < n_items;) {
        const int r = rows_of(qlen[i0]);
        size_t i1 = i0;
        while (i1 < n_items && (qlen[i1] == qlen[i0] || rows_of(qlen[i1]) == r)) ++i1;
        const size_t group_bytes = (size_t)(p.al + 1) * G * r * profile_row_bytes<A>();
        int gpb = pair_groups_per_block(group_bytes, G);
        p.group_bytes = (uint32_t)group_bytes;
        if (gpb == 0) {
            // Not one warp of group profiles fits in shared memory (a large alphabet): the groups
            // keep their profiles in a global scratch region, in launches of bounded size.
            gpb = 256 / G;
            const size_t per_block = (size_t)gpb * group_bytes;
            const size_t max_blocks = std::max<size_t>(1, PAIR_GPROF_BYTES / per_block);
            const size_t need_blocks = (i1 - i0 + gpb - 1) / gpb;
            void *d_gprof;
            HY_CK(ctx.get(PS_GPROF, std::min(max_blocks, need_blocks) * per_block, &d_gprof));
            p.gprof = (uint8_t *)d_gprof;
            for (size_t j0 = i0; j0 < i1; j0 += max_blocks * gpb) {
                const size_t j1 = std::min(i1, j0 + max_blocks * gpb);
                p.item_base = (uint32_t)(ib + j0);
                p.n_items = (uint32_t)(ib + j1);
                const int blocks = (int)((j1 - j0 + gpb - 1) / gpb);
                HY_CK((launch_pairs_rows<A, G>(r, mode, ends, p, blocks, gpb * G, 0, ctx.stream)));
            }
            p.gprof = nullptr;
        } else {
            p.item_base = (uint32_t)(ib + i0);
            p.n_items = (uint32_t)(ib + i1);
            const int blocks = (int)((i1 - i0 + gpb - 1) / gpb);
            HY_CK((launch_pairs_rows<A, G>(r, mode, ends, p, blocks, gpb * G, gpb * group_bytes, ctx.stream)));
        }
        i0 = i1;
    }
    return fail(HY_OK);
}

// One chunk's column maxima narrowed to int16 for the copy back: every pair of the chunk proved
// int16 lanes, so every maximum (at most 32767 - gap_open) fits.
__global__ void narrow_colmax_kernel(const int32_t *src, int16_t *dst, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = (int16_t)src[i];
}

// align_pair_position_max's BestHit and score2 for pairs [0, n) from their column maxima at
// colmax + t_off[k] (position_hits). One thread per pair.
__global__ void pos_hits_kernel(uint64_t n, const uint64_t *t_off, const int32_t *colmax, int32_t *scores,
                                int32_t *tend, int32_t matrix_max, int32_t min_score, int32_t *s2) {
    const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    position_hits(colmax + t_off[k], (uint32_t)(t_off[k + 1] - t_off[k]), matrix_max, min_score, scores + k,
                  tend + k, s2 ? s2 + 2 * k : nullptr);
}

// Whether p lies in page-locked host memory the device can copy from or to directly (memory from
// cudaMallocHost / cudaHostAlloc / cudaHostRegister, such as a pinned tensor's).
static bool host_pinned(const void *p) {
    if (!p) return false;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost;
}

// What a call computes besides align_pairs' hits: align_pair_position_max (posmax: SW, score only,
// the column maxima, each pair's BestHit from them and, with score2, its score2).
struct PairsCall {
    bool posmax = false;
    int32_t *colmax = nullptr;  // host, at t_off[k] - t_off[0] (null: not copied)
    int32_t min_score = 0;
    int32_t *score2 = nullptr;  // host, {score, position} per pair (null: not computed)
};

struct PosTiming {
    double kernel_ms = 0.0, call_ms = 0.0, cells = 0.0;
};
static thread_local PosTiming g_pos_timing;

// The pairs' routing from their lengths alone, chunked over the host threads: each pair's width
// proof (int16x2 or int32 lanes) and whether it is a long single pair for the stripe kernel, into
// route[k]. Each chunk stops at its own first failure, and the batch's first length failure is
// that of the first chunk that has one. A few long pairs (the single-pair path) take the
// score-only stripe kernel, every 128 query rows on their own warp; many keep the packed pair
// kernels, whose throughput is higher once the whole GPU is busy. The host checks the long pairs'
// symbols (the device checks the others while packing them).
struct LengthsPlan {
    uint64_t n_len = 0;          // pairs before the first length failure
    hy_status len_st = HY_OK;    // that failure's error and detail
    int64_t len_d0 = 0;
    uint64_t n_part[2] = {0, 0};  // packed pairs of each lane arithmetic (long pairs apart)
    bool use_long = false;       // the long pairs take the stripe kernel
    std::vector<uint32_t> run_long;  // the long pairs it runs: those before the first bad one
    uint64_t n_long_bad = 0;     // the first long pair with a symbol out of range (n_pairs: none)
};

static LengthsPlan plan_lengths(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                                const uint64_t *t_off, uint64_t n_pairs, int mode, int32_t min_e,
                                int32_t max_e, int32_t gap_open, int32_t gap_ext, uint64_t alphabet_len,
                                uint8_t *route) {
    LengthsPlan lp;
    const unsigned nt = host_threads(n_pairs, 1 << 15);
    struct LenPart {
        uint64_t first_bad = ~0ull;
        hy_status st = HY_OK;
        int64_t d0 = 0;
        uint64_t n[2] = {0, 0};
        std::vector<uint32_t> longs;
    };
    std::vector<LenPart> parts(nt);
    const uint64_t per = (n_pairs + nt - 1) / nt;
    parallel_for(nt, 1, [&](uint64_t ca, uint64_t ce, unsigned) {
        for (uint64_t c = ca; c < ce; ++c) {
            LenPart &pt = parts[c];
            const uint64_t a = c * per, e = std::min(n_pairs, a + per);
            for (uint64_t k = a; k < e; ++k) {
                const uint64_t ql = q_off[k + 1] - q_off[k], tl = t_off[k + 1] - t_off[k];
                const int64_t b = magnitude_bound(mode, min_e, max_e, gap_open, gap_ext, ql, tl);
                if (narrowest_width(b) < 0 || ql >= (1u << 30) || tl >= (1u << 31)) {
                    pt.st = narrowest_width(b) < 0 ? HY_ERR_SCORE_RANGE_TOO_WIDE : HY_ERR_UNSUPPORTED;
                    pt.d0 = narrowest_width(b) < 0 ? b : 0;
                    pt.first_bad = k;
                    break;
                }
                uint8_t r = device_fits_i16(b, gap_open) ? 0 : PAIR_I32;
                if (tb_long_pair(ql, tl)) {
                    r |= PAIR_LONG;
                    pt.longs.push_back((uint32_t)k);
                }
                route[k] = r;
                ++pt.n[r & PAIR_I32];
            }
        }
    });
    lp.n_len = n_pairs;
    std::vector<uint32_t> olong;
    for (LenPart &pt : parts) {
        olong.insert(olong.end(), pt.longs.begin(), pt.longs.end());
        lp.n_part[0] += pt.n[0];
        lp.n_part[1] += pt.n[1];
        if (pt.st != HY_OK) {
            lp.n_len = pt.first_bad;
            lp.len_st = pt.st;
            lp.len_d0 = pt.d0;
            break;
        }
    }
    lp.n_long_bad = n_pairs;
    uint64_t stripes = 0;
    for (uint32_t k : olong) stripes += tb_long_pair_stripes(q_off[k + 1] - q_off[k]);
    if (stripes > LONG_PAIR_MAX_STRIPES) olong.clear();
    for (uint32_t k : olong) {
        if (first_bad_symbol(q_res + q_off[k], q_off[k + 1] - q_off[k], alphabet_len) >= 0 ||
            first_bad_symbol(t_res + t_off[k], t_off[k + 1] - t_off[k], alphabet_len) >= 0) {
            lp.n_long_bad = k;
            break;
        }
        lp.run_long.push_back(k);
    }
    lp.use_long = !olong.empty();
    if (lp.use_long)
        for (uint32_t k : olong) --lp.n_part[route[k] & PAIR_I32];
    return lp;
}

static hy_status pairs_run(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                           const uint64_t *t_off, uint64_t n_pairs, const int32_t *matrix,
                           uint64_t alphabet_len, int32_t gap_open, int32_t gap_ext, hy_mode mode,
                           hy_search_type search_type, hy_hit *out, uint64_t *failed_pair,
                           const PairsCall &pc) {
    using clock = std::chrono::steady_clock;
    auto since = [](clock::time_point t) {
        return std::chrono::duration<double, std::milli>(clock::now() - t).count();
    };
    const auto t_call = clock::now();
    PairsContext &ctx = g_ctx;
    PairsHost &hs = g_host;
    ctx.kernel_ms = 0.0;
    ctx.call_ms = 0.0;
    for (double &x : ctx.phase_ms) x = 0.0;
    if (failed_pair) *failed_pair = n_pairs;
    if ((int)mode < 0 || (int)mode > 4) return fail(HY_ERR_INVALID_ARGUMENT);
    if ((int)search_type < HY_SEARCH_SCORE || (int)search_type > HY_SEARCH_ALIGNMENT)
        return fail(HY_ERR_UNSUPPORTED);
    hy_status st = validate_scoring(alphabet_len, matrix, alphabet_len * alphabet_len, gap_open, gap_ext);
    if (st != HY_OK) return st;
    if (n_pairs == 0) return fail(HY_OK);
    if (!q_off || !t_off || !out) return fail(HY_ERR_INVALID_ARGUMENT);
    if (alphabet_len > 255 || n_pairs >= (uint64_t)NO_INDEX) return fail(HY_ERR_UNSUPPORTED);
    const int32_t min_e = *std::min_element(matrix, matrix + alphabet_len * alphabet_len);
    const int32_t max_e = *std::max_element(matrix, matrix + alphabet_len * alphabet_len);

    LengthsPlan lp = plan_lengths(q_res, q_off, t_res, t_off, n_pairs, mode, min_e, max_e, gap_open, gap_ext,
                                  alphabet_len, hs.route.get(n_pairs));
    const uint8_t *route = hs.route.get(n_pairs);
    const uint64_t n_len = lp.n_len, n_long_bad = lp.n_long_bad;
    const bool use_long = lp.use_long;
    const uint64_t *n_part = lp.n_part;
    const std::vector<uint32_t> &run_long = lp.run_long;
    ctx.phase_ms[0] = since(t_call);
    // One long pair whose band passes fit one round (align_pair's single-pair path): straight to the
    // band kernel with one copy in and one copy out, without the chunk pipeline.
    if (n_pairs == 1 && !pc.posmax && n_len == 1 && n_long_bad == 1 && run_long.size() == 1 &&
        band_long_pair_fits(q_off[1] - q_off[0], alphabet_len)) {
        int32_t r[3];
        st = band_single_pair(q_res + q_off[0], q_off[1] - q_off[0], t_res + t_off[0], t_off[1] - t_off[0], matrix,
                              alphabet_len, gap_open, gap_ext, (int)mode, r, &ctx.kernel_ms);
        if (st != HY_OK) return st;
        const bool with_ends = search_type != HY_SEARCH_SCORE;
        out[0].score = r[0];
        out[0].reserved = 0;
        out[0].db_index = 0;
        out[0].query_end = with_ends ? (int64_t)r[1] : -1;
        out[0].target_end = with_ends ? (int64_t)r[2] : -1;
        ctx.call_ms = since(t_call);
        return fail(HY_OK);
    }

    uint32_t dev_bad = NO_INDEX;  // the first pair whose symbols the device found out of range
    const bool ends = !pc.posmax && search_type != HY_SEARCH_SCORE;
    const bool posmax = pc.posmax;
    const int32_t *h_out = nullptr;
    int32_t *h_cm = nullptr;  // posmax: pinned column maxima, from t_off[0]
    bool cm_direct = false;   // h_cm is the caller's own (pinned) array
    const auto t_pipe = clock::now();
    if (n_len > 0) {
        int dev = 0;
        HY_CK(cudaGetDevice(&dev));
        if (ctx.device != dev) {
            ctx.~PairsContext();
            new (&ctx) PairsContext();
            ctx.device = dev;
            HY_CK(cudaStreamCreateWithFlags(&ctx.stream, cudaStreamNonBlocking));
            HY_CK(cudaStreamCreateWithFlags(&ctx.copy_stream, cudaStreamNonBlocking));
            HY_CK(cudaStreamCreateWithFlags(&ctx.d2h_stream, cudaStreamNonBlocking));
            for (cudaEvent_t &e : ctx.slot_ev) HY_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        const uint64_t L = n_len;
        const std::vector<uint64_t> bounds = plan_pair_chunks(q_off, t_off, L);
        const uint64_t n_chunks = bounds.size() - 1;
        auto chunk_at = [&](uint64_t c) { return bounds[c]; };
        while (ctx.ev.size() < 3 * n_chunks + 2) {
            cudaEvent_t e;
            HY_CK(cudaEventCreate(&e));
            ctx.ev.push_back(e);
        }
        // Buffers of the whole call, and the largest chunk's staging and packed columns.
        uint64_t slot_bytes = 0, res_cols = 0;
        for (uint64_t c = 0; c < n_chunks; ++c) {
            const uint64_t a = chunk_at(c), b = chunk_at(c + 1);
            const uint64_t qb = q_off[b] - q_off[a], tb = t_off[b] - t_off[a];
            slot_bytes = std::max(slot_bytes, (qb + tb + 7) / 8 * 8 + 16 * (b - a + 1) + sizeof(ItemMeta) * (b - a));
            res_cols = std::max(res_cols, tb + 16 * (b - a));
        }
        void *d_q, *d_t, *d_qoff, *d_toff, *d_matrix, *d_out, *scratch;
        HY_CK(ctx.get(PS_Q, q_off[L], &d_q));
        HY_CK(ctx.get(PS_T, t_off[L], &d_t));
        HY_CK(ctx.get(PS_QOFF, sizeof(uint64_t) * (L + 1), &d_qoff));
        HY_CK(ctx.get(PS_TOFF, sizeof(uint64_t) * (L + 1), &d_toff));
        HY_CK(ctx.get(PS_MATRIX, sizeof(int32_t) * alphabet_len * alphabet_len, &d_matrix));
        // Scores, query ends, target ends, the first bad pair, then (posmax) score2 pairs.
        const uint64_t out_words = posmax ? 5 * L + 2 : 3 * L + 1;
        HY_CK(ctx.get(PS_OUT, sizeof(int32_t) * out_words, &d_out));
        int32_t *d_scores = (int32_t *)d_out, *d_qend = d_scores + L, *d_tend = d_qend + L;
        uint32_t *d_bad = (uint32_t *)(d_tend + L);
        int32_t *d_s2 = d_tend + L + 2;
        int32_t *d_colmax = nullptr;
        if (posmax) {
            void *cmv;
            HY_CK(ctx.get(PS_COLMAX, sizeof(int32_t) * t_off[L], &cmv));
            d_colmax = (int32_t *)cmv;
            if (pc.colmax && t_off[L] > t_off[0]) {
                // A pinned caller array takes the column maxima straight from the device.
                cm_direct = host_pinned(pc.colmax);
                void *hv = pc.colmax;
                if (!cm_direct) HY_CK(ctx.get_pinned(PAIR_SLOTS + 1, sizeof(int32_t) * (t_off[L] - t_off[0]), &hv));
                h_cm = (int32_t *)hv;
            }
        }
        PairParams pp[2];
        const int meta_slot[2] = {PS_META16, PS_META32}, qlen_slot[2] = {PS_QLEN16, PS_QLEN32};
        const int iqoff_slot[2] = {PS_IQOFF16, PS_IQOFF32}, res_slot[2] = {PS_RES16, PS_RES32};
        const int itoff_slot[2] = {PS_ITOFF16, PS_ITOFF32};
        for (int h = 0; h < 2; ++h) {
            PairParams &p = pp[h];
            p = PairParams{};
            if (n_part[h] == 0) continue;
            void *m, *ql, *qo;
            HY_CK(ctx.get(meta_slot[h], sizeof(ItemMeta) * n_part[h], &m));
            HY_CK(ctx.get(qlen_slot[h], sizeof(uint32_t) * n_part[h], &ql));
            HY_CK(ctx.get(iqoff_slot[h], 2 * sizeof(uint64_t) * n_part[h], &qo));
            HY_CK(ctx.get(res_slot[h], res_cols * (h == 0 ? sizeof(Pair16H::RES) : sizeof(Single32::RES)), &scratch));
            p.meta = (const ItemMeta *)m;
            p.qlen = (const uint32_t *)ql;
            p.qoff = (const uint64_t *)qo;
            p.q_res = (const uint8_t *)d_q;
            p.matrix = (const int32_t *)d_matrix;
            p.al = (int32_t)alphabet_len;
            p.lim = h == 0 ? 32767 - gap_open : 536870911;
            p.go = gap_open;
            p.ge = gap_ext;
            p.sentinel = h == 0 ? -32768 + gap_ext : INT32_MIN / 4;
            p.top_free = ((int)mode == MODE_SW || (int)mode == MODE_HW || (int)mode == MODE_OV) ? 1 : 0;
            p.scores = d_scores;
            p.qend = d_qend;
            p.tend = d_tend;
            if (posmax) {
                void *to;
                HY_CK(ctx.get(itoff_slot[h], 2 * sizeof(uint64_t) * n_part[h], &to));
                p.toff = (const uint64_t *)to;
                p.colmax = d_colmax;
            }
        }
        // Residues already in pinned memory are copied to the device from where they are; others go
        // through the staging slots.
        const bool q_pinned = host_pinned(q_res), t_pinned = host_pinned(t_res);
        void *slots[PAIR_SLOTS];
        for (int s = 0; s < PAIR_SLOTS && s < (int)n_chunks; ++s) HY_CK(ctx.get_pinned(s, slot_bytes, &slots[s]));
        HY_CK(cudaMemsetAsync(d_bad, 0xff, sizeof(uint32_t), ctx.stream));
        HY_CK(cudaMemcpyAsync(d_matrix, matrix, sizeof(int32_t) * alphabet_len * alphabet_len,
                              cudaMemcpyHostToDevice, ctx.stream));
        uint64_t ib[2] = {0, 0};
        // Declared before the drainer, whose thread reads it: locals are destroyed in reverse
        // order, so the thread is joined (on any early return) before this vector goes away.
        std::vector<char> chunk_narrow(n_chunks, 0);
        std::unique_ptr<ColmaxDrainer> drainer;
        int16_t *d_cm16 = nullptr;
        if (h_cm && !cm_direct && n_chunks > 1) {
            uint64_t max_tb = 0;
            for (uint64_t c = 0; c < n_chunks; ++c)
                max_tb = std::max(max_tb, t_off[chunk_at(c + 1)] - t_off[chunk_at(c)]);
            void *p16;
            HY_CK(ctx.get(PS_CM16, sizeof(int16_t) * max_tb, &p16));
            d_cm16 = (int16_t *)p16;
            if (!hs.cm_copier) hs.cm_copier.reset(new AsyncCopy(std::max(2u, std::thread::hardware_concurrency() / 2)));
            drainer.reset(new ColmaxDrainer(
                dev, n_chunks, *hs.cm_copier, ctx.ev, 2 * n_chunks,
                [&](uint64_t c, uint64_t *x0, uint64_t *x1) {
                    *x0 = t_off[chunk_at(c)] - t_off[0];
                    *x1 = t_off[chunk_at(c + 1)] - t_off[0];
                },
                pc.colmax, h_cm, chunk_narrow));
        }
        // Host side of chunk c: its pairs partitioned, sorted and packed into items, written with
        // its offsets to its staging slot (the residues follow on the copier).
        auto prep = [&](uint64_t c, ChunkState &cs) -> hy_status {
            const uint64_t a = chunk_at(c), b = chunk_at(c + 1), n = b - a;
            auto t0 = clock::now();
            // This chunk's packed pairs of each lane arithmetic, in input order, with their keys.
            uint32_t *o[2], *o_tmp[2];
            uint64_t *k[2], *k_tmp[2];
            for (int h = 0; h < 2; ++h) {
                o[h] = hs.ord[h].get(n);
                k[h] = hs.keys[h].get(n);
            }
            o_tmp[0] = hs.ord_tmp.get(n);
            k_tmp[0] = hs.keys_tmp.get(n);
            size_t cnt[2] = {0, 0};
            {
                const unsigned pt = host_threads(n, 1 << 14);
                const uint64_t per = (n + pt - 1) / pt;
                std::vector<uint64_t> at(2 * (pt + 1), 0);
                parallel_for(pt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
                    for (uint64_t t = ta; t < te; ++t)
                        for (uint64_t x = a + t * per; x < std::min<uint64_t>(b, a + (t + 1) * per); ++x)
                            if (!(use_long && (route[x] & PAIR_LONG))) ++at[2 * (t + 1) + (route[x] & PAIR_I32)];
                });
                for (unsigned t = 0; t < pt; ++t) {
                    at[2 * (t + 1)] += at[2 * t];
                    at[2 * (t + 1) + 1] += at[2 * t + 1];
                }
                cnt[0] = at[2 * pt];
                cnt[1] = at[2 * pt + 1];
                parallel_for(pt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
                    for (uint64_t t = ta; t < te; ++t) {
                        uint64_t pos[2] = {at[2 * t], at[2 * t + 1]};
                        for (uint64_t x = a + t * per; x < std::min<uint64_t>(b, a + (t + 1) * per); ++x) {
                            if (use_long && (route[x] & PAIR_LONG)) continue;
                            const int h = route[x] & PAIR_I32;
                            o[h][pos[h]] = (uint32_t)x;
                            k[h][pos[h]++] = shape_key(q_off[x + 1] - q_off[x], t_off[x + 1] - t_off[x]);
                        }
                    }
                });
            }
            for (int h = 0; h < 2; ++h) {
                o_tmp[h] = o_tmp[0];
                k_tmp[h] = k_tmp[0];
            }
            // The staging slot: [query residues][target residues][q_off, t_off slices][items]. It was
            // last used by chunk c - 3, already issued.
            const int s = (int)(c % PAIR_SLOTS);
            auto tw = clock::now();
            if (c >= (uint64_t)PAIR_SLOTS) HY_CK(cudaEventSynchronize(ctx.slot_ev[s]));
            ctx.phase_ms[5] += since(tw);
            cs.c = c;
            cs.a = a;
            cs.b = b;
            cs.n = n;
            cs.s = s;
            cs.slot = (uint8_t *)slots[s];
            cs.qb = q_off[b] - q_off[a];
            cs.tb = t_off[b] - t_off[a];
            cs.s_qoff = (uint64_t *)(cs.slot + (cs.qb + cs.tb + 7) / 8 * 8);
            cs.s_toff = cs.s_qoff + (n + 1);
            cs.s_meta[0] = (ItemMeta *)(cs.s_toff + (n + 1));
            // Every pair int16 and none on the stripe kernel: the maxima fit int16.
            cs.narrow = d_cm16 != nullptr && cnt[1] == 0 && cnt[0] == n;
            for (int h = 0; h < 2; ++h) {
                cs.n_items[h] = 0;
                cs.cols[h] = 0;
                if (h == 1) cs.s_meta[1] = cs.s_meta[0] + cs.n_items[0];
                cs.qlen[h] = hs.qlen[2 * (c & 1) + h].get(cnt[h]);
                if (cnt[h] == 0) continue;
                // One scratch pair serves both arithmetics: sort and pack the first before the second.
                sort_by_shape(hs, o[h], k[h], o_tmp[h], k_tmp[h], cnt[h]);
                cs.n_items[h] = pack_items(hs, o[h], k[h], cnt[h], h == 0, cs.s_meta[h], cs.qlen[h], &cs.cols[h]);
            }
            parallel_for(2 * (n + 1), 1 << 18, [&](uint64_t x0, uint64_t x1, unsigned) {
                for (uint64_t x = x0; x < x1; ++x)
                    (x <= n ? cs.s_qoff[x] : cs.s_toff[x - n - 1]) = x <= n ? q_off[a + x] : t_off[a + x - n - 1];
            });
            ctx.phase_ms[1] += since(t0);
            return fail(HY_OK);
        };
        // Device side of a prepared chunk whose residues are staged: its copies on the copy stream,
        // then its packing and pair kernels on the compute stream.
        auto issue = [&](const ChunkState &cs) -> hy_status {
            const uint64_t c = cs.c, a = cs.a, n = cs.n, qb = cs.qb, tb = cs.tb;
            cudaStream_t cp = ctx.copy_stream;
            if (qb)
                HY_CK(cudaMemcpyAsync((uint8_t *)d_q + q_off[a], q_pinned ? q_res + q_off[a] : cs.slot, qb,
                                      cudaMemcpyHostToDevice, cp));
            if (tb)
                HY_CK(cudaMemcpyAsync((uint8_t *)d_t + t_off[a], t_pinned ? t_res + t_off[a] : cs.slot + qb, tb,
                                      cudaMemcpyHostToDevice, cp));
            HY_CK(cudaMemcpyAsync((uint64_t *)d_qoff + a, cs.s_qoff, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, cp));
            HY_CK(cudaMemcpyAsync((uint64_t *)d_toff + a, cs.s_toff, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, cp));
            for (int h = 0; h < 2; ++h)
                if (cs.n_items[h])
                    HY_CK(cudaMemcpyAsync(const_cast<ItemMeta *>(pp[h].meta) + ib[h], cs.s_meta[h],
                                          sizeof(ItemMeta) * cs.n_items[h], cudaMemcpyHostToDevice, cp));
            HY_CK(cudaEventRecord(ctx.slot_ev[cs.s], cp));
            HY_CK(cudaStreamWaitEvent(ctx.stream, ctx.slot_ev[cs.s], 0));
            if (posmax && tb) HY_CK(cudaMemsetAsync(d_colmax + t_off[a], 0, sizeof(int32_t) * tb, ctx.stream));
            HY_CK(cudaEventRecord(ctx.ev[2 * c], ctx.stream));
            hy_status s2 = run_items<Pair16H, PAIR_G>(ctx, pp[0], PS_RES16, PS_BND16, cs.qlen[0], ib[0], cs.n_items[0],
                                                      cs.cols[0], (const uint64_t *)d_qoff, (const uint64_t *)d_toff,
                                                      (uint8_t *)d_q, (const uint8_t *)d_t, d_bad, mode, ends);
            if (s2 != HY_OK) return s2;
            s2 = run_items<Single32, PAIR_G>(ctx, pp[1], PS_RES32, PS_BND32, cs.qlen[1], ib[1], cs.n_items[1],
                                             cs.cols[1], (const uint64_t *)d_qoff, (const uint64_t *)d_toff,
                                             (uint8_t *)d_q, (const uint8_t *)d_t, d_bad, mode, ends);
            if (s2 != HY_OK) return s2;
            HY_CK(cudaEventRecord(ctx.ev[2 * c + 1], ctx.stream));
            if (h_cm && tb) {
                // This chunk's column maxima back while the next chunks run (a long pair's are
                // copied again once the stripe kernel has written them), narrowed when they fit.
                HY_CK(cudaStreamWaitEvent(ctx.d2h_stream, ctx.ev[2 * c + 1], 0));
                if (cs.narrow) {
                    const int blocks = (int)std::min<uint64_t>((tb + 255) / 256, 148 * 8);
                    narrow_colmax_kernel<<<blocks, 256, 0, ctx.d2h_stream>>>(d_colmax + t_off[a], d_cm16, tb);
                    HY_CK(cudaGetLastError());
                    HY_CK(cudaMemcpyAsync(h_cm + (t_off[a] - t_off[0]), d_cm16, sizeof(int16_t) * tb,
                                          cudaMemcpyDeviceToHost, ctx.d2h_stream));
                } else {
                    HY_CK(cudaMemcpyAsync(h_cm + (t_off[a] - t_off[0]), d_colmax + t_off[a], sizeof(int32_t) * tb,
                                          cudaMemcpyDeviceToHost, ctx.d2h_stream));
                }
            }
            HY_CK(cudaEventRecord(ctx.ev[2 * n_chunks + c], ctx.d2h_stream));
            chunk_narrow[c] = cs.narrow ? 1 : 0;
            if (drainer) drainer->issued(c);
            ib[0] += cs.n_items[0];
            ib[1] += cs.n_items[1];
            return fail(HY_OK);
        };
        // Chunk c is sorted and packed on the host threads while the copier stages chunk c - 1's
        // residues; chunk c - 1 then goes to the device and chunk c's staging starts.
        if (!hs.copier) hs.copier.reset(new AsyncCopy(std::max(2u, std::thread::hardware_concurrency() / 2)));
        AsyncCopy &copier = *hs.copier;
        struct CopierWait {  // no return leaves a copy running into a staging slot
            AsyncCopy &cp;
            ~CopierWait() { cp.wait(); }
        } copier_wait{copier};
        ChunkState cur{}, pend{};
        bool have_pend = false;
        auto flush = [&]() -> hy_status {
            const auto tw = clock::now();
            copier.wait();
            ctx.phase_ms[2] += since(tw);
            return issue(pend);
        };
        for (uint64_t c = 0; c < n_chunks; ++c) {
            if ((st = prep(c, cur)) != HY_OK) return st;
            if (have_pend && (st = flush()) != HY_OK) return st;
            copier.start(cur.slot, q_res + q_off[cur.a], q_pinned ? 0 : cur.qb, cur.slot + cur.qb,
                         t_res + t_off[cur.a], t_pinned ? 0 : cur.tb);
            pend = cur;
            have_pend = true;
        }
        if (have_pend && (st = flush()) != HY_OK) return st;
        // The long pairs, once every chunk's queries are on the device (the compute stream has
        // waited for each chunk's copies).
        if (run_long.size() == 1 && !posmax &&
            band_long_pair_fits(q_off[run_long[0] + 1] - q_off[run_long[0]], alphabet_len)) {
            // One long pair (align_pair's single-pair path) whose passes fit one round: the band
            // kernel, its passes on the warps of one block or of a cluster, ends tracked in the
            // same sweep (measured 2000 x 2000 0.55 ms, 5000 x 5000 1.6 ms against the stripe
            // kernel's 0.97 and 2.5 ms; at 20,000 query rows, two rounds, the stripes are faster).
            const uint32_t k = run_long[0];
            st = band_long_pair((const uint8_t *)d_q + q_off[k], q_off[k + 1] - q_off[k], t_res + t_off[k],
                                t_off[k + 1] - t_off[k], (const int32_t *)d_matrix, alphabet_len, gap_open,
                                gap_ext, mode, ctx.stream, k, d_scores, d_qend, d_tend, &ctx.kernel_ms);
            if (st != HY_OK) return st;
        } else if (!run_long.empty()) {
            const TbColmaxOut cmx{d_colmax, pc.score2 ? d_s2 : nullptr, max_e, pc.min_score};
            st = tb_long_pair_scores(q_res, q_off, t_res, t_off, run_long, (const uint8_t *)d_q,
                                     (const int32_t *)d_matrix, alphabet_len, gap_open, gap_ext, mode,
                                     ctx.stream, d_scores, d_qend, d_tend, &ctx.kernel_ms,
                                     posmax ? &cmx : nullptr);
            if (st != HY_OK) return st;
        }
        if (posmax) {
            // Every pair's BestHit (and score2) from its column maxima.
            HY_CK(cudaEventRecord(ctx.ev[3 * n_chunks], ctx.stream));
            pos_hits_kernel<<<(unsigned)((L + 127) / 128), 128, 0, ctx.stream>>>(
                L, (const uint64_t *)d_toff, d_colmax, d_scores, d_tend, max_e, pc.min_score,
                pc.score2 ? d_s2 : nullptr);
            HY_CK(cudaGetLastError());
            HY_CK(cudaEventRecord(ctx.ev[3 * n_chunks + 1], ctx.stream));
            if (h_cm && !run_long.empty()) {
                // The long pairs' maxima over the zeros their chunks copied back.
                HY_CK(cudaStreamWaitEvent(ctx.stream, ctx.ev[2 * n_chunks + n_chunks - 1], 0));
                for (uint32_t k : run_long)
                    if (t_off[k + 1] > t_off[k])
                        HY_CK(cudaMemcpyAsync(h_cm + (t_off[k] - t_off[0]), d_colmax + t_off[k],
                                              sizeof(int32_t) * (t_off[k + 1] - t_off[k]),
                                              cudaMemcpyDeviceToHost, ctx.stream));
            }
        }
        void *h_stage = nullptr;
        HY_CK(ctx.get_pinned(PAIR_SLOTS, sizeof(int32_t) * out_words, &h_stage));
        HY_CK(cudaMemcpyAsync(h_stage, d_out, sizeof(int32_t) * out_words, cudaMemcpyDeviceToHost, ctx.stream));
        if (h_cm && cm_direct) HY_CK(cudaStreamSynchronize(ctx.d2h_stream));
        if (drainer) {
            bool ok = true;
            ctx.phase_ms[6] += drainer->join(&ok);
            drainer.reset();
            if (!ok) return fail(HY_ERR_CUDA);
        } else if (h_cm && !cm_direct) {
            // The chunk's column maxima into the caller's array.
            for (uint64_t c = 0; c < n_chunks; ++c) {
                HY_CK(cudaEventSynchronize(ctx.ev[2 * n_chunks + c]));
                const auto tc = clock::now();
                const uint64_t x0 = t_off[chunk_at(c)] - t_off[0], x1 = t_off[chunk_at(c + 1)] - t_off[0];
                parallel_for(x1 - x0, 1 << 18, [&](uint64_t e0, uint64_t e1, unsigned) {
                    memcpy(pc.colmax + x0 + e0, h_cm + x0 + e0, sizeof(int32_t) * (e1 - e0));
                });
                ctx.phase_ms[6] += since(tc);
            }
        }
        HY_CK(cudaStreamSynchronize(ctx.stream));
        if (h_cm && !cm_direct)
            for (uint32_t k : run_long)
                memcpy(pc.colmax + (t_off[k] - t_off[0]), h_cm + (t_off[k] - t_off[0]),
                       sizeof(int32_t) * (t_off[k + 1] - t_off[k]));
        for (uint64_t c = 0; c < n_chunks; ++c) {
            float ms = 0.0f;
            HY_CK(cudaEventElapsedTime(&ms, ctx.ev[2 * c], ctx.ev[2 * c + 1]));
            ctx.kernel_ms += ms;
        }
        if (posmax) {
            float ms = 0.0f;
            HY_CK(cudaEventElapsedTime(&ms, ctx.ev[3 * n_chunks], ctx.ev[3 * n_chunks + 1]));
            ctx.kernel_ms += ms;
        }
        h_out = (const int32_t *)h_stage;
        memcpy(&dev_bad, h_out + 3 * L, sizeof(uint32_t));
    }
    ctx.phase_ms[3] = since(t_pipe);
    const auto t_res_fill = clock::now();
    // The batch's first failure in input order, and its details from that pair alone: symbols of
    // the query, then of the target, then the width proof.
    const uint64_t n_ok = std::min<uint64_t>({n_len, n_long_bad, (uint64_t)dev_bad});
    hy_status first = HY_OK;
    int64_t d[3] = {0, 0, 0};
    if (n_ok < n_pairs) {
        const uint64_t kk = n_ok;
        const int bq = first_bad_symbol(q_res + q_off[kk], q_off[kk + 1] - q_off[kk], alphabet_len);
        const int bt = bq >= 0 ? -1 : first_bad_symbol(t_res + t_off[kk], t_off[kk + 1] - t_off[kk], alphabet_len);
        if (bq >= 0 || bt >= 0) {
            first = HY_ERR_SYMBOL_OUT_OF_RANGE;
            d[0] = bq >= 0 ? bq : bt;
            d[1] = (int64_t)alphabet_len;
        } else {
            first = lp.len_st;
            d[0] = lp.len_d0;
        }
        if (failed_pair) *failed_pair = n_ok;
    }
    if (n_ok > 0) {
        const uint64_t L = n_len;
        const int32_t *h = h_out;
        parallel_for(n_ok, 1 << 16, [&](uint64_t a, uint64_t e, unsigned) {
            for (uint64_t k = a; k < e; ++k) {
                out[k].score = h[k];
                out[k].reserved = 0;
                out[k].db_index = k;
                out[k].query_end = ends ? (int64_t)h[L + k] : -1;
                out[k].target_end = (ends || posmax) ? (int64_t)h[2 * L + k] : -1;
                if (posmax && pc.score2) {
                    pc.score2[2 * k] = h[3 * L + 2 + 2 * k];
                    pc.score2[2 * k + 1] = h[3 * L + 2 + 2 * k + 1];
                }
            }
        });
    }
    // Positions of the pairs from the failing one on are left at 0.
    if (h_cm && n_ok < n_len)
        memset(pc.colmax + (t_off[n_ok] - t_off[0]), 0, sizeof(int32_t) * (t_off[n_len] - t_off[n_ok]));
    ctx.phase_ms[4] = since(t_res_fill);
    ctx.call_ms = since(t_call);
    if (posmax) {
        g_pos_timing.kernel_ms = ctx.kernel_ms;
        g_pos_timing.call_ms = ctx.call_ms;
        double cells = 0.0;
        for (uint64_t k = 0; k < n_ok; ++k)
            cells += (double)(q_off[k + 1] - q_off[k]) * (double)(t_off[k + 1] - t_off[k]);
        g_pos_timing.cells = cells;
    }
    return fail(first, d[0], d[1], d[2]);
}

}  // namespace hy

extern "C" hy_status hy_align_pairs(const uint8_t *q_res, const uint64_t *q_off,
                                    const uint8_t *t_res, const uint64_t *t_off, uint64_t n_pairs,
                                    const int32_t *matrix, uint64_t alphabet_len, int32_t gap_open,
                                    int32_t gap_ext, hy_mode mode, hy_search_type search_type,
                                    hy_hit *out, uint64_t *failed_pair) {
    return pairs_run(q_res, q_off, t_res, t_off, n_pairs, matrix, alphabet_len, gap_open, gap_ext, mode,
                     search_type, out, failed_pair, PairsCall{});
}

extern "C" hy_status hy_align_pairs_position_max(const uint8_t *q_res, const uint64_t *q_off,
                                                 const uint8_t *t_res, const uint64_t *t_off,
                                                 uint64_t n_pairs, const int32_t *matrix,
                                                 uint64_t alphabet_len, int32_t gap_open, int32_t gap_ext,
                                                 int32_t *colmax, hy_hit *out, int32_t min_score,
                                                 int32_t *score2, uint64_t *failed_pair) {
    g_pos_timing = PosTiming{};
    PairsCall pc;
    pc.posmax = true;
    pc.colmax = colmax;
    pc.min_score = min_score;
    pc.score2 = score2;
    return pairs_run(q_res, q_off, t_res, t_off, n_pairs, matrix, alphabet_len, gap_open, gap_ext, HY_MODE_SW,
                     HY_SEARCH_SCORE, out, failed_pair, pc);
}

extern "C" hy_status hy_position_max_timing(double out[3]) {
    if (!out) return fail(HY_ERR_INVALID_ARGUMENT);
    out[0] = g_pos_timing.kernel_ms;
    out[1] = g_pos_timing.call_ms;
    out[2] = g_pos_timing.cells;
    return fail(HY_OK);
}

extern "C" hy_status hy_align_pairs_timing(double *kernel_ms, double *call_ms) {
    if (kernel_ms) *kernel_ms = g_ctx.kernel_ms;
    if (call_ms) *call_ms = g_ctx.call_ms;
    return fail(HY_OK);
}

extern "C" hy_status hy_align_pairs_phases(double *ms, uint32_t n) {
    if (!ms && n) return fail(HY_ERR_INVALID_ARGUMENT);
    for (uint32_t i = 0; i < n && i < 7; ++i) ms[i] = g_ctx.phase_ms[i];
    return fail(HY_OK);
}

// The chunk boundaries hy_align_pairs would use for these offsets (introspection for tests):
// writes up to `cap` boundaries and returns the number of chunks.
extern "C" uint64_t hy_debug_pair_chunks(const uint64_t *q_off, const uint64_t *t_off, uint64_t n_pairs,
                                         uint64_t *bounds, uint64_t cap) {
    if (!q_off || !t_off || n_pairs == 0) return 0;
    const std::vector<uint64_t> b = plan_pair_chunks(q_off, t_off, n_pairs);
    for (uint64_t i = 0; i < b.size() && i < cap; ++i) bounds[i] = b[i];
    return b.size() - 1;
}
