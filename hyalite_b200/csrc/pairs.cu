// pairs.cu -- align_pairs (src/kernel.rs:429-452) on the device.
//
// Every pair has its own query and target. Pairs are validated in input order exactly like
// align_pair_with (src/kernel.rs:354-415): symbols of the query then the target, then the width
// proof on the pair's own lengths; the first failure ends the batch. The accepted prefix is
// partitioned by the device width rule, sorted by (query length, target length), and packed two
// pairs of EQUAL query length per int16x2 item so both halves share one row structure.
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "host_common.h"
#include "scan_kernel.cuh"

using namespace hy;

namespace hy {

constexpr int PAIR_G = 8;
constexpr int PAIR_R16 = 16;
constexpr int PAIR_R32 = 16;
constexpr size_t PAIR_SMEM_LIMIT = 200 * 1024;

// Grow-only device and pinned buffers of the calling thread (align_pairs keeps one PairScratch
// per call in the reference; here the device buffers survive across calls of the same thread).
struct PairsContext {
    int device = -1;
    cudaStream_t stream = nullptr;
    struct Buf {
        void *p = nullptr;
        size_t n = 0;
    };
    Buf b[13];
    ~PairsContext() {
        for (auto &x : b) cudaFree(x.p);
        if (stream) cudaStreamDestroy(stream);
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

template <class A, int G, int R, int MODE, bool ENDS>
static cudaError_t launch_pairs_mode(const PairParams &p, int blocks, int threads, size_t smem,
                                     cudaStream_t st) {
    auto kern = pairs_kernel<A, G, R, MODE, ENDS>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<blocks, threads, smem, st>>>(p);
    return cudaGetLastError();
}

template <class A, int G, int R>
static cudaError_t launch_pairs(int mode, bool ends, const PairParams &p, int blocks, int threads,
                                size_t smem, cudaStream_t st) {
#define HY_MODE_CASE(M)                                                                 \
    case M:                                                                             \
        return ends ? launch_pairs_mode<A, G, R, M, true>(p, blocks, threads, smem, st) \
                    : launch_pairs_mode<A, G, R, M, false>(p, blocks, threads, smem, st);
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

struct PairPart {
    std::vector<ItemMeta> meta;
    std::vector<uint32_t> qlen;
    std::vector<uint64_t> qoff;
    uint64_t cols = 0;
};

// Packs the pairs listed in `order` (already sorted by query length, then target length, both
// descending). Pair16 items take two consecutive pairs when their query lengths are equal.
static void pack_pairs(const std::vector<uint32_t> &order, const uint64_t *q_off,
                       const uint64_t *t_off, bool two, PairPart &pp) {
    const uint64_t align = two ? 8 : 16;
    size_t i = 0;
    while (i < order.size()) {
        ItemMeta m;
        m.pad_ = 0;
        m.col_off = pp.cols;
        const uint32_t a = order[i];
        const uint64_t qa = q_off[a + 1] - q_off[a];
        m.idx[0] = a;
        m.n[0] = (uint32_t)(t_off[a + 1] - t_off[a]);
        m.idx[1] = NO_INDEX;
        m.n[1] = 0;
        uint64_t qb_off = q_off[a];
        ++i;
        if (two && i < order.size()) {
            const uint32_t b = order[i];
            if (q_off[b + 1] - q_off[b] == qa) {
                m.idx[1] = b;
                m.n[1] = (uint32_t)(t_off[b + 1] - t_off[b]);
                qb_off = q_off[b];
                ++i;
            }
        }
        m.w = std::max(m.n[0], m.n[1]);
        pp.cols += (m.w + align - 1) / align * align;
        pp.meta.push_back(m);
        pp.qlen.push_back((uint32_t)qa);
        pp.qoff.push_back(q_off[a]);
        pp.qoff.push_back(qb_off);
    }
}

template <class A, int G, int R>
static hy_status run_part(PairsContext &ctx, int slot0, const PairPart &pp, const uint8_t *t_res,
                          const uint64_t *t_off, const uint8_t *d_q, const int32_t *d_matrix,
                          int32_t al, int32_t go, int32_t ge, int mode, bool ends, int32_t *d_scores,
                          int32_t *d_qend, int32_t *d_tend) {
    if (pp.meta.empty()) return fail(HY_OK);
    const bool two = A::NH == 2;
    const size_t group_bytes = (size_t)(al + 1) * G * R * profile_row_bytes<A>();
    int gpb = (int)std::min<size_t>(256 / G, PAIR_SMEM_LIMIT / group_bytes);
    gpb = gpb / (32 / G) * (32 / G);  // whole warps
    if (gpb == 0) return fail(HY_ERR_UNSUPPORTED);
    const size_t n_items = pp.meta.size();
    void *d_meta, *d_qlen, *d_qoff, *d_res, *d_bnd;
    HY_CK(ctx.get(slot0 + 0, sizeof(ItemMeta) * n_items, &d_meta));
    HY_CK(ctx.get(slot0 + 1, sizeof(uint32_t) * n_items, &d_qlen));
    HY_CK(ctx.get(slot0 + 2, sizeof(uint64_t) * 2 * n_items, &d_qoff));
    const size_t res_bytes = pp.cols * sizeof(typename A::RES);
    HY_CK(ctx.get(slot0 + 3, res_bytes, &d_res));
    size_t max_q = 0;
    for (uint32_t q : pp.qlen) max_q = std::max<size_t>(max_q, q);
    const bool multipass = max_q > (size_t)(G * R);
    HY_CK(ctx.get(slot0 + 4, multipass ? 2 * sizeof(typename A::V) * pp.cols : 16, &d_bnd));
    // Pack target residues (the shorter half of a pair item padded with symbol `al`).
    std::vector<typename A::RES> res(std::max<size_t>(pp.cols, 1), (typename A::RES)(two ? (al | (al << 8)) : 0));
    for (const ItemMeta &m : pp.meta) {
        const uint8_t *t0 = t_res + t_off[m.idx[0]];
        const uint8_t *t1 = m.idx[1] == NO_INDEX ? nullptr : t_res + t_off[m.idx[1]];
        for (uint32_t j = 0; j < m.w; ++j) {
            if (two) {
                uint32_t lo = j < m.n[0] ? t0[j] : (uint32_t)al;
                uint32_t hi = (t1 && j < m.n[1]) ? t1[j] : (uint32_t)al;
                res[m.col_off + j] = (typename A::RES)(lo | (hi << 8));
            } else {
                res[m.col_off + j] = (typename A::RES)t0[j];
            }
        }
    }
    HY_CK(cudaMemcpyAsync(d_meta, pp.meta.data(), sizeof(ItemMeta) * n_items, cudaMemcpyHostToDevice, ctx.stream));
    HY_CK(cudaMemcpyAsync(d_qlen, pp.qlen.data(), sizeof(uint32_t) * n_items, cudaMemcpyHostToDevice, ctx.stream));
    HY_CK(cudaMemcpyAsync(d_qoff, pp.qoff.data(), sizeof(uint64_t) * 2 * n_items, cudaMemcpyHostToDevice, ctx.stream));
    HY_CK(cudaMemcpyAsync(d_res, res.data(), res_bytes, cudaMemcpyHostToDevice, ctx.stream));
    PairParams p;
    p.meta = (const ItemMeta *)d_meta;
    p.qlen = (const uint32_t *)d_qlen;
    p.qoff = (const uint64_t *)d_qoff;
    p.n_items = (uint32_t)n_items;
    p.q_res = d_q;
    p.res = d_res;
    p.matrix = d_matrix;
    p.al = al;
    p.lim = two ? 32767 - go : 536870911;
    p.go = go;
    p.ge = ge;
    p.sentinel = two ? -32768 + ge : INT32_MIN / 4;
    p.top_free = (mode == MODE_SW || mode == MODE_HW || mode == MODE_OV) ? 1 : 0;
    p.group_bytes = (uint32_t)group_bytes;
    p.boundary = d_bnd;
    p.scores = d_scores;
    p.qend = d_qend;
    p.tend = d_tend;
    const int blocks = (int)((n_items + gpb - 1) / gpb);
    HY_CK((launch_pairs<A, G, R>(mode, ends, p, blocks, gpb * G, gpb * group_bytes, ctx.stream)));
    // The host staging vector must outlive the async copy.
    HY_CK(cudaStreamSynchronize(ctx.stream));
    return fail(HY_OK);
}

}  // namespace hy

extern "C" hy_status hy_align_pairs(const uint8_t *q_res, const uint64_t *q_off,
                                    const uint8_t *t_res, const uint64_t *t_off, uint64_t n_pairs,
                                    const int32_t *matrix, uint64_t alphabet_len, int32_t gap_open,
                                    int32_t gap_ext, hy_mode mode, hy_search_type search_type,
                                    hy_hit *out, uint64_t *failed_pair) {
    if (failed_pair) *failed_pair = n_pairs;
    if ((int)mode < 0 || (int)mode > 4) return fail(HY_ERR_INVALID_ARGUMENT);
    if ((int)search_type != HY_SEARCH_SCORE && (int)search_type != HY_SEARCH_SCORE_END)
        return fail(HY_ERR_UNSUPPORTED);
    hy_status st = validate_scoring(alphabet_len, matrix, alphabet_len * alphabet_len, gap_open, gap_ext);
    if (st != HY_OK) return st;
    if (n_pairs == 0) return fail(HY_OK);
    if (!q_off || !t_off || !out) return fail(HY_ERR_INVALID_ARGUMENT);
    if (alphabet_len > 255 || n_pairs >= (uint64_t)NO_INDEX) return fail(HY_ERR_UNSUPPORTED);
    const int32_t min_e = *std::min_element(matrix, matrix + alphabet_len * alphabet_len);
    const int32_t max_e = *std::max_element(matrix, matrix + alphabet_len * alphabet_len);

    // Validate in input order; remember the first failure.
    uint64_t n_ok = n_pairs;
    hy_status first = HY_OK;
    int64_t d[3] = {0, 0, 0};
    std::vector<uint32_t> o16, o32;
    for (uint64_t k = 0; k < n_pairs && first == HY_OK; ++k) {
        const uint64_t ql = q_off[k + 1] - q_off[k], tl = t_off[k + 1] - t_off[k];
        for (int s = 0; s < 2 && first == HY_OK; ++s) {
            const uint8_t *seq = s == 0 ? q_res + q_off[k] : t_res + t_off[k];
            const uint64_t len = s == 0 ? ql : tl;
            for (uint64_t i = 0; i < len; ++i)
                if (seq[i] >= alphabet_len) {
                    first = HY_ERR_SYMBOL_OUT_OF_RANGE;
                    d[0] = seq[i];
                    d[1] = (int64_t)alphabet_len;
                    break;
                }
        }
        if (first == HY_OK) {
            const int64_t b = magnitude_bound(mode, min_e, max_e, gap_open, gap_ext, ql, tl);
            if (narrowest_width(b) < 0) {
                first = HY_ERR_SCORE_RANGE_TOO_WIDE;
                d[0] = b;
            } else if (ql >= (1u << 30) || tl >= (1u << 31)) {
                first = HY_ERR_UNSUPPORTED;
            } else {
                (device_fits_i16(b, gap_open) ? o16 : o32).push_back((uint32_t)k);
            }
        }
        if (first != HY_OK) n_ok = k;
    }
    if (failed_pair && first != HY_OK) *failed_pair = n_ok;
    if (n_ok > 0) {
        PairsContext &ctx = g_ctx;
        int dev = 0;
        HY_CK(cudaGetDevice(&dev));
        if (ctx.device != dev) {
            ctx.~PairsContext();
            new (&ctx) PairsContext();
            ctx.device = dev;
            HY_CK(cudaStreamCreateWithFlags(&ctx.stream, cudaStreamNonBlocking));
        }
        auto shape = [&](uint32_t a, uint32_t b) {
            const uint64_t qa = q_off[a + 1] - q_off[a], qb = q_off[b + 1] - q_off[b];
            if (qa != qb) return qa > qb;
            const uint64_t ta = t_off[a + 1] - t_off[a], tb = t_off[b + 1] - t_off[b];
            return ta != tb ? ta > tb : a < b;
        };
        std::sort(o16.begin(), o16.end(), shape);
        std::sort(o32.begin(), o32.end(), shape);
        PairPart p16, p32;
        pack_pairs(o16, q_off, t_off, true, p16);
        pack_pairs(o32, q_off, t_off, false, p32);

        void *d_q, *d_matrix, *d_out;
        const uint64_t qbytes = q_off[n_ok] - q_off[0];
        HY_CK(ctx.get(10, q_off[n_ok], &d_q));
        HY_CK(ctx.get(11, sizeof(int32_t) * alphabet_len * alphabet_len, &d_matrix));
        HY_CK(ctx.get(12, 3 * sizeof(int32_t) * n_ok, &d_out));
        if (qbytes)
            HY_CK(cudaMemcpyAsync((uint8_t *)d_q + q_off[0], q_res + q_off[0], qbytes,
                                  cudaMemcpyHostToDevice, ctx.stream));
        HY_CK(cudaMemcpyAsync(d_matrix, matrix, sizeof(int32_t) * alphabet_len * alphabet_len,
                              cudaMemcpyHostToDevice, ctx.stream));
        int32_t *d_scores = (int32_t *)d_out, *d_qend = d_scores + n_ok, *d_tend = d_qend + n_ok;
        const bool ends = search_type == HY_SEARCH_SCORE_END;
        st = run_part<Pair16, PAIR_G, PAIR_R16>(ctx, 0, p16, t_res, t_off, (const uint8_t *)d_q,
                                                (const int32_t *)d_matrix, (int32_t)alphabet_len,
                                                gap_open, gap_ext, mode, ends, d_scores, d_qend, d_tend);
        if (st != HY_OK) return st;
        st = run_part<Single32, PAIR_G, PAIR_R32>(ctx, 5, p32, t_res, t_off, (const uint8_t *)d_q,
                                                  (const int32_t *)d_matrix, (int32_t)alphabet_len,
                                                  gap_open, gap_ext, mode, ends, d_scores, d_qend, d_tend);
        if (st != HY_OK) return st;
        std::vector<int32_t> h(3 * n_ok);
        HY_CK(cudaMemcpyAsync(h.data(), d_out, 3 * sizeof(int32_t) * n_ok, cudaMemcpyDeviceToHost, ctx.stream));
        HY_CK(cudaStreamSynchronize(ctx.stream));
        for (uint64_t k = 0; k < n_ok; ++k) {
            out[k].score = h[k];
            out[k].reserved = 0;
            out[k].db_index = k;
            out[k].query_end = ends ? (int64_t)h[n_ok + k] : -1;
            out[k].target_end = ends ? (int64_t)h[2 * n_ok + k] : -1;
        }
    }
    return fail(first, d[0], d[1], d[2]);
}
