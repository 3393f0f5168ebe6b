// pairs.cu -- align_pairs (src/kernel.rs:429-452) on the device.
//
// Every pair has its own query and target. Pairs are validated in input order exactly like
// align_pair_with (src/kernel.rs:354-415): symbols of the query then the target, then the width
// proof on the pair's own lengths; the first failure ends the batch. The accepted prefix is
// partitioned by the device width rule, sorted by (query length, target length), and packed two
// pairs of EQUAL query length per int16x2 item so both halves share one row structure. Rows per
// lane are chosen per query length so that a pass (8 lanes x rows) wastes the fewest padded
// rows; items of one choice run in one launch. Validation and packing run on all host threads.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

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
// Chunks of items the residue packing is split into, so host packing overlaps the device's copies
// and kernels (each chunk at least 65,536 items).
constexpr size_t PAIR_PACK_CHUNKS = 8;
// Most warps (128-row stripes) the long pairs of one call may take on the stripe kernel.
constexpr uint64_t LONG_PAIR_MAX_STRIPES = 2048;
// Rows per lane the int16x2 pair kernel is compiled for.
constexpr int PAIR_ROWS[] = {8, 12, 16, 20, 24, 32};

// Grow-only device and pinned buffers of the calling thread (align_pairs keeps one PairScratch
// per call in the reference; here the device buffers survive across calls of the same thread).
struct PairsContext {
    int device = -1;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> ev;  // around each chunk's kernels
    struct Buf {
        void *p = nullptr;
        size_t n = 0;
    };
    Buf b[14];
    // Grow-only pinned host staging: the packed target residues (one per partition), then the
    // queries going in and the results coming back (in that stream order).
    Buf pinned[3];
    double kernel_ms = 0.0, call_ms = 0.0;  // the last call: pair kernels' device time, whole call
    ~PairsContext() {
        for (auto &x : b) cudaFree(x.p);
        for (auto &x : pinned) cudaFreeHost(x.p);
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
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
    cudaError_t get(int slot, size_t bytes, void **out) {
        bytes = std::max<size_t>(bytes, 16);
        if (b[slot].n < bytes) {
            cudaFree(b[slot].p);
            b[slot].p = nullptr;
            b[slot].n = 0;
            cudaError_t e = cudaMalloc(&b[slot].p, bytes);
            if (e != cudaSuccess) return e;
            b[slot].n = bytes;
        }
        *out = b[slot].p;
        return cudaSuccess;
    }
};

static thread_local PairsContext g_ctx;

#define HY_CK(call)                                                                                \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            cudaGetLastError();                                                                    \
            return fail(e_ == cudaErrorMemoryAllocation ? HY_ERR_OUT_OF_MEMORY : HY_ERR_CUDA, e_); \
        }                                                                                          \
    } while (0)

template <class A, int G, int R, int MODE, bool ENDS, bool GPROF>
static cudaError_t launch_pairs_mode(const PairParams &p, int blocks, int threads, size_t smem,
                                     cudaStream_t st) {
    auto kern = pairs_kernel<A, G, R, MODE, ENDS, GPROF>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<blocks, threads, smem, st>>>(p);
    return cudaGetLastError();
}

// The form with group profiles in global memory (p.gprof set): only the smallest row shape of
// each lane arithmetic, which is what a large alphabet runs.
template <class A, int G, int R>
static cudaError_t launch_pairs_gprof(int mode, bool ends, const PairParams &p, int blocks,
                                      int threads, cudaStream_t st) {
    if constexpr ((A::NH == 2 && R == 8) || (A::NH == 1 && R == PAIR_R32)) {
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

// Rows per lane for an int16x2 item of query length q: the fewest padded rows over the pass
// shapes whose per-group profile keeps at least two warps of groups per block; ties go to more
// rows (fewer passes).
static int pair_rows(uint64_t q, int32_t al) {
    int best = 8;
    uint64_t best_pad = ~0ull;
    for (int r : PAIR_ROWS) {
        const size_t group_bytes = (size_t)(al + 1) * PAIR_G * r * profile_row_bytes<Pair16>();
        if (r > 8 && group_bytes * 8 > PAIR_SMEM_LIMIT) continue;
        const uint64_t rpp = (uint64_t)PAIR_G * r;
        const uint64_t pad = (q + rpp - 1) / rpp * rpp;
        if (pad <= best_pad) {
            best_pad = pad;
            best = r;
        }
    }
    return best;
}

// Sorts pair indices (given in ascending order) by (query length desc, target length desc), index
// asc for equal lengths: a stable LSD radix sort of 64-bit keys (complemented query length above
// complemented target length) on 16-bit digits, skipping digits every pair shares. The keys are
// built once from the offsets in input order and travel with the indices, so no pass reads the
// offsets at random; histograms and scatters run on all host threads (per-thread ranges in order,
// which keeps the sort stable). `keys` receives the sorted keys.
static inline uint32_t key_qlen(uint64_t k) { return ~(uint32_t)(k >> 32); }
static inline uint32_t key_tlen(uint64_t k) { return ~(uint32_t)k; }

static void sort_by_shape(std::vector<uint32_t> &o, const uint64_t *q_off, const uint64_t *t_off,
                          std::vector<uint64_t> &keys) {
    const size_t n = o.size();
    keys.resize(n);
    parallel_for(n, 1 << 16, [&](uint64_t a, uint64_t e, unsigned) {
        for (uint64_t i = a; i < e; ++i) {
            const uint32_t k = o[i];
            keys[i] = ((uint64_t)~(uint32_t)(q_off[k + 1] - q_off[k]) << 32) | ~(uint32_t)(t_off[k + 1] - t_off[k]);
        }
    });
    if (n < 2) return;
    std::vector<uint32_t> tmp(n);
    std::vector<uint64_t> key_tmp(n);
    const unsigned nt = host_threads(n, 1 << 16);
    const uint64_t per = (n + nt - 1) / nt;
    std::vector<std::vector<size_t>> count(nt, std::vector<size_t>(1 << 16));
    for (int shift = 0; shift < 64; shift += 16) {
        parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
            for (uint64_t t = ta; t < te; ++t) {
                std::fill(count[t].begin(), count[t].end(), 0);
                for (uint64_t i = t * per; i < std::min<uint64_t>(n, (t + 1) * per); ++i)
                    ++count[t][(keys[i] >> shift) & 0xffff];
            }
        });
        const size_t d0 = (keys[0] >> shift) & 0xffff;
        size_t total0 = 0;
        for (unsigned t = 0; t < nt; ++t) total0 += count[t][d0];
        if (total0 == n) continue;  // one digit value: nothing to do
        size_t sum = 0;
        for (size_t d = 0; d < (1u << 16); ++d)
            for (unsigned t = 0; t < nt; ++t) {
                const size_t c = count[t][d];
                count[t][d] = sum;
                sum += c;
            }
        parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
            for (uint64_t t = ta; t < te; ++t)
                for (uint64_t i = t * per; i < std::min<uint64_t>(n, (t + 1) * per); ++i) {
                    const size_t dst = count[t][(keys[i] >> shift) & 0xffff]++;
                    tmp[dst] = o[i];
                    key_tmp[dst] = keys[i];
                }
        });
        o.swap(tmp);
        keys.swap(key_tmp);
    }
}

struct PairPart {
    std::vector<ItemMeta> meta;
    std::vector<uint32_t> qlen;
    std::vector<uint64_t> qoff;
    uint64_t cols = 0;
};

// Packs the pairs listed in `order` (already sorted by query length, then target length, both
// descending; `keys` their sort keys). Pair16 items take two consecutive pairs when their query
// lengths are equal. Item boundaries come from one sequential pass over the keys; the items are
// then filled, and their column offsets prefix-summed, on all host threads.
static void pack_pairs(const std::vector<uint32_t> &order, const std::vector<uint64_t> &keys,
                       const uint64_t *q_off, bool two, PairPart &pp) {
    const uint64_t align = two ? 8 : 16;
    std::vector<uint32_t> start;
    start.reserve(two ? order.size() / 2 + 1 : order.size());
    for (size_t i = 0; i < order.size();) {
        start.push_back((uint32_t)i);
        i += (two && i + 1 < order.size() && key_qlen(keys[i + 1]) == key_qlen(keys[i])) ? 2 : 1;
    }
    const size_t n_items = start.size();
    pp.meta.resize(n_items);
    pp.qlen.resize(n_items);
    pp.qoff.resize(2 * n_items);
    const unsigned nt = host_threads(n_items, 1 << 15);
    const uint64_t per = (n_items + nt - 1) / nt;
    std::vector<uint64_t> part(nt + 1, 0);
    parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
        for (uint64_t t = ta; t < te; ++t) {
            uint64_t cols = 0;
            for (uint64_t it = t * per; it < std::min<uint64_t>(n_items, (t + 1) * per); ++it) {
                const size_t i = start[it];
                const bool pair = it + 1 < n_items ? start[it + 1] - i == 2 : order.size() - i == 2;
                ItemMeta &m = pp.meta[it];
                m.pad_ = 0;
                m.idx[0] = order[i];
                m.n[0] = key_tlen(keys[i]);
                m.idx[1] = pair ? order[i + 1] : NO_INDEX;
                m.n[1] = pair ? key_tlen(keys[i + 1]) : 0;
                m.w = std::max(m.n[0], m.n[1]);
                m.col_off = cols;  // within this thread's range; shifted below
                cols += (m.w + align - 1) / align * align;
                pp.qlen[it] = key_qlen(keys[i]);
                pp.qoff[2 * it] = q_off[m.idx[0]];
                pp.qoff[2 * it + 1] = pair ? q_off[m.idx[1]] : q_off[m.idx[0]];
            }
            part[t + 1] = cols;
        }
    });
    for (unsigned t = 0; t < nt; ++t) part[t + 1] += part[t];
    parallel_for(nt, 1, [&](uint64_t ta, uint64_t te, unsigned) {
        for (uint64_t t = ta; t < te; ++t)
            for (uint64_t it = t * per; it < std::min<uint64_t>(n_items, (t + 1) * per); ++it)
                pp.meta[it].col_off += part[t];
    });
    pp.cols = part[nt];
}

template <class A, int G>
static hy_status run_part(PairsContext &ctx, int slot0, const PairPart &pp, const uint8_t *t_res,
                          const uint64_t *t_off, const uint8_t *d_q, const int32_t *d_matrix,
                          int32_t al, int32_t go, int32_t ge, int mode, bool ends, int32_t *d_scores,
                          int32_t *d_qend, int32_t *d_tend) {
    if (pp.meta.empty()) return fail(HY_OK);
    const bool two = A::NH == 2;
    const size_t n_items = pp.meta.size();
    void *d_meta, *d_qlen, *d_qoff, *d_res, *d_bnd;
    HY_CK(ctx.get(slot0 + 0, sizeof(ItemMeta) * n_items, &d_meta));
    HY_CK(ctx.get(slot0 + 1, sizeof(uint32_t) * n_items, &d_qlen));
    HY_CK(ctx.get(slot0 + 2, sizeof(uint64_t) * 2 * n_items, &d_qoff));
    const size_t res_bytes = pp.cols * sizeof(typename A::RES);
    HY_CK(ctx.get(slot0 + 3, res_bytes, &d_res));
    // Rows per lane of each item (a function of its query length; items are sorted by it).
    std::vector<int> rows(n_items);
    bool multipass = false;
    for (size_t i = 0; i < n_items; ++i) {
        rows[i] = two ? pair_rows(pp.qlen[i], al) : PAIR_R32;
        multipass = multipass || pp.qlen[i] > (uint32_t)(G * rows[i]);
    }
    HY_CK(ctx.get(slot0 + 4, multipass ? 2 * sizeof(typename A::V) * pp.cols : 16, &d_bnd));
    // Target residues (the shorter half of a pair item padded with symbol `al`) are packed
    // straight into pinned staging (every column, padding included, is written), in chunks of
    // items: while the device copies and aligns chunk c, the host threads pack chunk c + 1.
    void *h_res = nullptr;
    HY_CK(ctx.get_pinned(slot0 == 0 ? 0 : 1, res_bytes, &h_res));
    typename A::RES *res = static_cast<typename A::RES *>(h_res);
    HY_CK(cudaMemcpyAsync(d_meta, pp.meta.data(), sizeof(ItemMeta) * n_items, cudaMemcpyHostToDevice, ctx.stream));
    HY_CK(cudaMemcpyAsync(d_qlen, pp.qlen.data(), sizeof(uint32_t) * n_items, cudaMemcpyHostToDevice, ctx.stream));
    HY_CK(cudaMemcpyAsync(d_qoff, pp.qoff.data(), sizeof(uint64_t) * 2 * n_items, cudaMemcpyHostToDevice, ctx.stream));
    PairParams p{};
    p.meta = (const ItemMeta *)d_meta;
    p.qlen = (const uint32_t *)d_qlen;
    p.qoff = (const uint64_t *)d_qoff;
    p.q_res = d_q;
    p.res = d_res;
    p.matrix = d_matrix;
    p.al = al;
    p.lim = two ? 32767 - go : 536870911;
    p.go = go;
    p.ge = ge;
    p.sentinel = two ? -32768 + ge : INT32_MIN / 4;
    p.top_free = (mode == MODE_SW || mode == MODE_HW || mode == MODE_OV) ? 1 : 0;
    p.boundary = d_bnd;
    p.scores = d_scores;
    p.qend = d_qend;
    p.tend = d_tend;
    p.gprof = nullptr;
    // Kernels of items [a, b), split where the rows per lane change.
    auto launch_range = [&](size_t a, size_t b) -> hy_status {
        for (size_t i0 = a; i0 < b;) {
            size_t i1 = i0;
            while (i1 < b && rows[i1] == rows[i0]) ++i1;
            const int r = rows[i0];
            const size_t group_bytes = (size_t)(al + 1) * G * r * profile_row_bytes<A>();
            int gpb = (int)std::min<size_t>(256 / G, PAIR_SMEM_LIMIT / group_bytes);
            gpb = gpb / (32 / G) * (32 / G);  // whole warps
            p.group_bytes = (uint32_t)group_bytes;
            if (gpb == 0) {
                // Not one warp of group profiles fits in shared memory (a large alphabet): the
                // groups keep their profiles in a global scratch region, in launches of bounded size.
                gpb = 256 / G;
                const size_t per_block = (size_t)gpb * group_bytes;
                const size_t max_blocks = std::max<size_t>(1, PAIR_GPROF_BYTES / per_block);
                const size_t need_blocks = (i1 - i0 + gpb - 1) / gpb;
                void *d_gprof;
                HY_CK(ctx.get(13, std::min(max_blocks, need_blocks) * per_block, &d_gprof));
                p.gprof = (uint8_t *)d_gprof;
                for (size_t j0 = i0; j0 < i1; j0 += max_blocks * gpb) {
                    const size_t j1 = std::min(i1, j0 + max_blocks * gpb);
                    p.item_base = (uint32_t)j0;
                    p.n_items = (uint32_t)j1;
                    const int blocks = (int)((j1 - j0 + gpb - 1) / gpb);
                    HY_CK((launch_pairs_rows<A, G>(r, mode, ends, p, blocks, gpb * G, 0, ctx.stream)));
                }
                p.gprof = nullptr;
            } else {
                p.item_base = (uint32_t)i0;
                p.n_items = (uint32_t)i1;
                const int blocks = (int)((i1 - i0 + gpb - 1) / gpb);
                HY_CK((launch_pairs_rows<A, G>(r, mode, ends, p, blocks, gpb * G, gpb * group_bytes, ctx.stream)));
            }
            i0 = i1;
        }
        return fail(HY_OK);
    };
    const size_t n_chunks = std::max<size_t>(1, std::min<size_t>(PAIR_PACK_CHUNKS, n_items / (1 << 16)));
    while (ctx.ev.size() < 2 * n_chunks) {
        cudaEvent_t e;
        HY_CK(cudaEventCreate(&e));
        ctx.ev.push_back(e);
    }
    for (size_t c = 0; c < n_chunks; ++c) {
        const size_t a = n_items * c / n_chunks, b = n_items * (c + 1) / n_chunks;
        parallel_for(b - a, 1 << 14, [&](uint64_t x0, uint64_t x1, unsigned) {
            for (uint64_t it = a + x0; it < a + x1; ++it) {
                const ItemMeta &m = pp.meta[it];
                const uint64_t end = it + 1 < n_items ? pp.meta[it + 1].col_off : pp.cols;
                const uint8_t *t0 = t_res + t_off[m.idx[0]];
                const uint8_t *t1 = m.idx[1] == NO_INDEX ? nullptr : t_res + t_off[m.idx[1]];
                for (uint64_t j = 0; j < end - m.col_off; ++j) {
                    if (two) {
                        uint32_t lo = j < m.n[0] ? t0[j] : (uint32_t)al;
                        uint32_t hi = (t1 && j < m.n[1]) ? t1[j] : (uint32_t)al;
                        res[m.col_off + j] = (typename A::RES)(lo | (hi << 8));
                    } else {
                        res[m.col_off + j] = (typename A::RES)(j < m.n[0] ? t0[j] : 0);
                    }
                }
            }
        });
        const uint64_t c0 = pp.meta[a].col_off, c1 = b < n_items ? pp.meta[b].col_off : pp.cols;
        HY_CK(cudaMemcpyAsync((typename A::RES *)d_res + c0, res + c0, (c1 - c0) * sizeof(typename A::RES),
                              cudaMemcpyHostToDevice, ctx.stream));
        HY_CK(cudaEventRecord(ctx.ev[2 * c], ctx.stream));
        hy_status st = launch_range(a, b);
        if (st != HY_OK) return st;
        HY_CK(cudaEventRecord(ctx.ev[2 * c + 1], ctx.stream));
    }
    // The host staging (the item vectors and the pinned residues) must outlive the async copies.
    HY_CK(cudaStreamSynchronize(ctx.stream));
    for (size_t c = 0; c < n_chunks; ++c) {
        float ms = 0.0f;
        HY_CK(cudaEventElapsedTime(&ms, ctx.ev[2 * c], ctx.ev[2 * c + 1]));
        ctx.kernel_ms += ms;
    }
    return fail(HY_OK);
}

}  // namespace hy

extern "C" hy_status hy_align_pairs(const uint8_t *q_res, const uint64_t *q_off,
                                    const uint8_t *t_res, const uint64_t *t_off, uint64_t n_pairs,
                                    const int32_t *matrix, uint64_t alphabet_len, int32_t gap_open,
                                    int32_t gap_ext, hy_mode mode, hy_search_type search_type,
                                    hy_hit *out, uint64_t *failed_pair) {
    const auto t_call = std::chrono::steady_clock::now();
    PairsContext &ctx = g_ctx;
    ctx.kernel_ms = 0.0;
    ctx.call_ms = 0.0;
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

    // Validate in input order, chunked over the host threads: each chunk stops at its own first
    // failure, and the batch's first failure is that of the first chunk that has one. The pairs
    // before it are partitioned by the device width rule in input order.
    const unsigned nt = host_threads(n_pairs, 1 << 15);
    struct Chunk {
        uint64_t first_bad = ~0ull;
        hy_status st = HY_OK;
        int64_t d[3] = {0, 0, 0};
        std::vector<uint32_t> o16, o32;
    };
    std::vector<Chunk> chunks(nt);
    const uint64_t per = (n_pairs + nt - 1) / nt;
    parallel_for(nt, 1, [&](uint64_t ca, uint64_t ce, unsigned) {
        for (uint64_t c = ca; c < ce; ++c) {
            Chunk &ch = chunks[c];
            const uint64_t a = c * per, e = std::min(n_pairs, a + per);
            for (uint64_t k = a; k < e && ch.st == HY_OK; ++k) {
                const uint64_t ql = q_off[k + 1] - q_off[k], tl = t_off[k + 1] - t_off[k];
                for (int s = 0; s < 2 && ch.st == HY_OK; ++s) {
                    const uint8_t *seq = s == 0 ? q_res + q_off[k] : t_res + t_off[k];
                    const uint64_t len = s == 0 ? ql : tl;
                    const int bad = first_bad_symbol(seq, len, alphabet_len);
                    if (bad >= 0) {
                        ch.st = HY_ERR_SYMBOL_OUT_OF_RANGE;
                        ch.d[0] = bad;
                        ch.d[1] = (int64_t)alphabet_len;
                    }
                }
                if (ch.st == HY_OK) {
                    const int64_t b = magnitude_bound(mode, min_e, max_e, gap_open, gap_ext, ql, tl);
                    if (narrowest_width(b) < 0) {
                        ch.st = HY_ERR_SCORE_RANGE_TOO_WIDE;
                        ch.d[0] = b;
                    } else if (ql >= (1u << 30) || tl >= (1u << 31)) {
                        ch.st = HY_ERR_UNSUPPORTED;
                    } else {
                        (device_fits_i16(b, gap_open) ? ch.o16 : ch.o32).push_back((uint32_t)k);
                    }
                }
                if (ch.st != HY_OK) ch.first_bad = k;
            }
        }
    });
    uint64_t n_ok = n_pairs;
    hy_status first = HY_OK;
    int64_t d[3] = {0, 0, 0};
    std::vector<uint32_t> o16, o32;
    for (Chunk &ch : chunks) {
        o16.insert(o16.end(), ch.o16.begin(), ch.o16.end());
        o32.insert(o32.end(), ch.o32.begin(), ch.o32.end());
        if (ch.st != HY_OK) {
            first = ch.st;
            n_ok = ch.first_bad;
            memcpy(d, ch.d, sizeof(d));
            break;
        }
    }
    if (failed_pair && first != HY_OK) *failed_pair = n_ok;
    // A few long pairs (the single-pair path) take the score-only stripe kernel: every 128 query
    // rows on their own warp. Many long pairs keep the packed pair kernels, whose throughput is
    // higher once the whole GPU is busy.
    std::vector<uint32_t> olong;
    {
        uint64_t stripes = 0;
        for (const std::vector<uint32_t> *v : {&o16, &o32})
            for (uint32_t k : *v) {
                const uint64_t ql = q_off[k + 1] - q_off[k], tl = t_off[k + 1] - t_off[k];
                if (tb_long_pair(ql, tl)) {
                    olong.push_back(k);
                    stripes += tb_long_pair_stripes(ql);
                }
            }
        if (stripes > LONG_PAIR_MAX_STRIPES) {
            olong.clear();
        } else if (!olong.empty()) {
            std::vector<char> is_long(n_ok, 0);
            for (uint32_t k : olong) is_long[k] = 1;
            for (std::vector<uint32_t> *v : {&o16, &o32})
                v->erase(std::remove_if(v->begin(), v->end(), [&](uint32_t k) { return is_long[k] != 0; }),
                         v->end());
        }
    }
    if (n_ok > 0) {
        int dev = 0;
        HY_CK(cudaGetDevice(&dev));
        if (ctx.device != dev) {
            ctx.~PairsContext();
            new (&ctx) PairsContext();
            ctx.device = dev;
            HY_CK(cudaStreamCreateWithFlags(&ctx.stream, cudaStreamNonBlocking));
        }
        // Sort by (query length desc, target length desc, index asc) through 64-bit keys.
        std::vector<uint64_t> k16, k32;
        sort_by_shape(o16, q_off, t_off, k16);
        sort_by_shape(o32, q_off, t_off, k32);
        PairPart p16, p32;
        pack_pairs(o16, k16, q_off, true, p16);
        pack_pairs(o32, k32, q_off, false, p32);

        void *d_q, *d_matrix, *d_out;
        const uint64_t qbytes = q_off[n_ok] - q_off[0];
        HY_CK(ctx.get(10, q_off[n_ok], &d_q));
        HY_CK(ctx.get(11, sizeof(int32_t) * alphabet_len * alphabet_len, &d_matrix));
        HY_CK(ctx.get(12, 3 * sizeof(int32_t) * n_ok, &d_out));
        void *h_stage = nullptr;
        HY_CK(ctx.get_pinned(2, std::max<uint64_t>(qbytes, 3 * sizeof(int32_t) * n_ok), &h_stage));
        if (qbytes) {
            parallel_for(qbytes, 1 << 24, [&](uint64_t a, uint64_t e, unsigned) {
                memcpy((uint8_t *)h_stage + a, q_res + q_off[0] + a, e - a);
            });
            HY_CK(cudaMemcpyAsync((uint8_t *)d_q + q_off[0], h_stage, qbytes, cudaMemcpyHostToDevice, ctx.stream));
        }
        HY_CK(cudaMemcpyAsync(d_matrix, matrix, sizeof(int32_t) * alphabet_len * alphabet_len,
                              cudaMemcpyHostToDevice, ctx.stream));
        int32_t *d_scores = (int32_t *)d_out, *d_qend = d_scores + n_ok, *d_tend = d_qend + n_ok;
        const bool ends = search_type != HY_SEARCH_SCORE;
        if (!olong.empty()) {
            st = tb_long_pair_scores(q_res, q_off, t_res, t_off, olong, (const uint8_t *)d_q,
                                     (const int32_t *)d_matrix, alphabet_len, gap_open, gap_ext, mode,
                                     ctx.stream, d_scores, d_qend, d_tend, &ctx.kernel_ms);
            if (st != HY_OK) return st;
        }
        st = run_part<Pair16, PAIR_G>(ctx, 0, p16, t_res, t_off, (const uint8_t *)d_q,
                                      (const int32_t *)d_matrix, (int32_t)alphabet_len, gap_open,
                                      gap_ext, mode, ends, d_scores, d_qend, d_tend);
        if (st != HY_OK) return st;
        st = run_part<Single32, PAIR_G>(ctx, 5, p32, t_res, t_off, (const uint8_t *)d_q,
                                        (const int32_t *)d_matrix, (int32_t)alphabet_len, gap_open,
                                        gap_ext, mode, ends, d_scores, d_qend, d_tend);
        if (st != HY_OK) return st;
        // Stream order: the query copy out of the staging buffer is done before this copy into it.
        const int32_t *h = (const int32_t *)h_stage;
        HY_CK(cudaMemcpyAsync(h_stage, d_out, 3 * sizeof(int32_t) * n_ok, cudaMemcpyDeviceToHost, ctx.stream));
        HY_CK(cudaStreamSynchronize(ctx.stream));
        parallel_for(n_ok, 1 << 16, [&](uint64_t a, uint64_t e, unsigned) {
            for (uint64_t k = a; k < e; ++k) {
                out[k].score = h[k];
                out[k].reserved = 0;
                out[k].db_index = k;
                out[k].query_end = ends ? (int64_t)h[n_ok + k] : -1;
                out[k].target_end = ends ? (int64_t)h[2 * n_ok + k] : -1;
            }
        });
    }
    ctx.call_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_call).count();
    return fail(first, d[0], d[1], d[2]);
}

extern "C" hy_status hy_align_pairs_timing(double *kernel_ms, double *call_ms) {
    if (kernel_ms) *kernel_ms = g_ctx.kernel_ms;
    if (call_ms) *call_ms = g_ctx.call_ms;
    return fail(HY_OK);
}
