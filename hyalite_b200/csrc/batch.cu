// batch.cu -- the batched form of the database scan.
//
// Many queries, each against its own Database (any mode and search type; all databases on one
// device), run in persistent kernels that pull (query, item chunk) units from a device work queue.
// The queue is walked chunk-major: chunk 0 (the longest targets, the databases being length
// sorted) for every query, longest query first, then chunk 1, and so on, so the largest units go
// first and the queue drains with a short tail; all queries reading the same chunk at about the
// same time also share its residues in L2. Each class of launch shape (int16x2 pairs with 8, 16 or
// 32 rows per lane; pairs wider than the long-pair split, one warp each; int32 items) has its own
// persistent kernel and queue. The winners' end positions are recovered by one block per query.
//
// All device work of a batch is captured once into a CUDA graph: the kernels read the batch from
// device descriptors (BatchQuery, BatchCtl) that each call rewrites with a few copies before
// replaying the graph. An autotuner times candidate launch configurations (rows per lane by query
// length, the long-pair width split) on a sampled part of a batch and keeps the fastest per batch
// shape. Results are bit-identical to hy_scan per query: the same per-cell kernels, reduction keys
// and winner-ends recovery.
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "batch_internal.h"

using namespace hy;

namespace hy {

static constexpr int LCG = LONG_G, LCR = LONG_R;      // long pairs and the int16x2 band
static constexpr int ICG = MAIN_G32, ICR = MAIN_R32;  // int32 items
static constexpr uint32_t LONG_W_MAX = 4096;          // largest long-pair split allowed

struct ClassLaunch {
    const BatchQuery *queries;
    const uint32_t *order;  // this class's query slots, longest query first
    BatchCtl *ctl;
    int cls;
    uint8_t *bnd;           // block-private boundary regions
    size_t bnd_stride;
};

struct BandLaunch {
    const BatchQuery *queries;
    const BatchCtl *ctl;
    uint8_t *bnd;           // one boundary region per query slot
    size_t bnd_stride;
    int32_t *ends;          // {score, query end, target end} per query slot
};

__device__ __forceinline__ void class_range(const BatchQuery &bq, int cls, uint32_t &lo, uint32_t &hi) {
    if (cls == BC_LONG || cls == BC_TLONG) {
        lo = bq.k0;
        hi = bq.kl;
    } else if (cls == BC_I32) {
        lo = 0;
        hi = bq.n_i32;
    } else {
        lo = bq.kl;
        hi = bq.n16;
    }
}

// One persistent kernel per launch class: blocks take units off the class queue until it is empty.
// Shared memory: the two profile mbarriers, then two pass slices of the largest pass of the batch.
// SW_ONLY: the SW classes, compiled for the SW sweep alone (the two-column form's register budget).
template <class A, int G, int R, int PK, bool SW_ONLY = false>
__global__ void __launch_bounds__(256, (scan_min_blocks<A, G, R, SW_ONLY && two_col_form<A, R, MODE_SW, false, false>()>()))
    batch_scan_kernel(const ClassLaunch L) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint32_t s_unit;
    constexpr uint32_t IPU = 256 / G;  // items per unit: one per group of the block
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    uint8_t *bufs = smem + 128;
    const uint32_t nq = L.ctl->count[L.cls];
    const uint32_t stride = L.ctl->chunk_stride;
    const uint32_t n_chunks = (L.ctl->n_chunks[L.cls] + stride - 1) / stride;
    const uint32_t n_units = n_chunks * nq;
    if (n_units == 0) return;
    init_profile_bars(bars);
    __syncthreads();
    uint32_t phase = 0;
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(&L.ctl->head[L.cls], 1u);
        __syncthreads();
        const uint32_t u = s_unit;
        __syncthreads();  // every thread has read s_unit before thread 0 takes the next unit
        if (u >= n_units) break;
        const uint32_t chunk = (u / nq) * stride;
        const uint32_t slot = L.order[u % nq];
        const BatchQuery &bq = L.queries[slot];
        uint32_t lo, hi;
        class_range(bq, L.cls, lo, hi);
        const uint32_t first = max(lo, chunk * IPU), end = min(hi, (chunk + 1) * IPU);
        if (first >= end) continue;
        ScanParams p = bq.sp[PK];
        p.boundary = L.bnd + (size_t)blockIdx.x * L.bnd_stride;
        p.bnd_col0 = p.meta[first].col_off;
        p.bnd_cols = L.bnd_stride / (2 * sizeof(typename A::V));
        bool ok = true;
        if constexpr (SW_ONLY) {
            ok = scan_unit<A, G, R, MODE_SW, false>(p, first, end, bufs, bars, phase);
        } else {
            switch (bq.mode) {
            case MODE_SW: ok = scan_unit<A, G, R, MODE_SW, false>(p, first, end, bufs, bars, phase); break;
            case MODE_NW: ok = scan_unit<A, G, R, MODE_NW, false>(p, first, end, bufs, bars, phase); break;
            case MODE_HW: ok = scan_unit<A, G, R, MODE_HW, false>(p, first, end, bufs, bars, phase); break;
            case MODE_OV: ok = scan_unit<A, G, R, MODE_OV, false>(p, first, end, bufs, bars, phase); break;
            default: ok = scan_unit<A, G, R, MODE_SHW, false>(p, first, end, bufs, bars, phase); break;
            }
        }
        if (!ok) return;
    }
}

// Query profiles of every (query slot, profile kind) the batch needs: blockIdx.y names the job.
__global__ void batch_profile_kernel(const BatchQuery *queries, const BatchCtl *ctl) {
    const uint32_t slot = blockIdx.y / PK_N;
    const int kind = (int)(blockIdx.y % PK_N);
    if (slot >= ctl->n_queries) return;
    const BatchQuery &bq = queries[slot];
    const ScanParams &sp = bq.sp[kind];
    if (sp.profile == nullptr || sp.n_passes == 0) return;
    const int64_t first = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    uint8_t *out = const_cast<uint8_t *>(sp.profile);
    const int32_t lim32 = 536870911;
    switch (kind) {
    case PK_BULK:
        if (bq.tab) {
            if (bq.bulk_rows == 8)
                build_profile_words<PairTab16, MAIN_G, 8>(bq.q, bq.matrix, bq.al, sp.go, bq.lim16, bq.top_free,
                                                          sp.vrow0, sp.n_passes, (uint32_t *)out, first, stride);
            else if (bq.bulk_rows == 16)
                build_profile_words<PairTab16, MAIN_G, 16>(bq.q, bq.matrix, bq.al, sp.go, bq.lim16, bq.top_free,
                                                           sp.vrow0, sp.n_passes, (uint32_t *)out, first, stride);
            else
                build_profile_words<PairTab16, MAIN_G, 32>(bq.q, bq.matrix, bq.al, sp.go, bq.lim16, bq.top_free,
                                                           sp.vrow0, sp.n_passes, (uint32_t *)out, first, stride);
        } else if (bq.bulk_rows == 8)
            build_profile_words<Pair16, MAIN_G, 8>(bq.q, bq.matrix, bq.al, sp.go, bq.lim16, bq.top_free,
                                                   sp.vrow0, sp.n_passes, (uint32_t *)out, first, stride);
        else if (bq.bulk_rows == 16)
            build_profile_words<Pair16, MAIN_G, 16>(bq.q, bq.matrix, bq.al, sp.go, bq.lim16, bq.top_free,
                                                    sp.vrow0, sp.n_passes, (uint32_t *)out, first, stride);
        else
            build_profile_words<Pair16, MAIN_G, 32>(bq.q, bq.matrix, bq.al, sp.go, bq.lim16, bq.top_free,
                                                    sp.vrow0, sp.n_passes, (uint32_t *)out, first, stride);
        break;
    case PK_W16:
        if (bq.tab)
            build_profile_words<PairTab16, LCG, LCR>(bq.q, bq.matrix, bq.al, sp.go, bq.lim16, bq.top_free,
                                                     sp.vrow0, sp.n_passes, (uint32_t *)out, first, stride);
        else
            build_profile_words<Pair16, LCG, LCR>(bq.q, bq.matrix, bq.al, sp.go, bq.lim16, bq.top_free,
                                                  sp.vrow0, sp.n_passes, (uint32_t *)out, first, stride);
        break;
    case PK_I32:
        build_profile_words<Single32, ICG, ICR>(bq.q, bq.matrix, bq.al, sp.go, lim32, bq.top_free,
                                                sp.vrow0, sp.n_passes, (int32_t *)out, first, stride);
        break;
    default:
        build_profile_words<Single32, WIN_G, WIN_R>(bq.q, bq.matrix, bq.al, sp.go, lim32, bq.top_free,
                                                    sp.vrow0, sp.n_passes, (int32_t *)out, first, stride);
        break;
    }
}

// End positions of each ScoreEnd query's winner: block `slot` reruns the winner's item with
// position tracking when the winner lives in this kernel's partition (int16x2 pair or int32 item).
template <class A, int PK>
__global__ void __launch_bounds__(1024) batch_band_kernel(const BandLaunch L) {
    extern __shared__ __align__(128) uint8_t smem[];
    const uint32_t slot = blockIdx.x;
    if (slot >= L.ctl->n_queries) return;
    const BatchQuery &bq = L.queries[slot];
    if (!bq.ends) return;
    const ScanParams &sp0 = bq.sp[PK];
    const unsigned long long key = *sp0.best_key;
    if (key == 0) return;
    const uint32_t idx = ~(uint32_t)(key & 0xffffffffu);
    const uint32_t r = bq.rank[idx];
    const bool packed = r / 2 >= bq.k0;
    uint32_t item;
    if (A::NH == 2) {
        if (!packed || (bq.tab != 0) != A::PAIRTAB) return;
        item = r / 2;
    } else {
        if (packed) return;
        item = r;
    }
    ScanParams p = sp0;
    p.boundary = L.bnd + (size_t)slot * L.bnd_stride;
    p.bnd_col0 = p.meta[item].col_off;
    p.bnd_cols = L.bnd_stride / (2 * sizeof(typename A::V));
    p.ends_out = L.ends + 3 * (size_t)slot;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    switch (bq.mode) {
    case MODE_SW: band_item<A, WIN_R, MODE_SW>(p, item, smem + 128, bar, phase); break;
    case MODE_NW: band_item<A, WIN_R, MODE_NW>(p, item, smem + 128, bar, phase); break;
    case MODE_HW: band_item<A, WIN_R, MODE_HW>(p, item, smem + 128, bar, phase); break;
    case MODE_OV: band_item<A, WIN_R, MODE_OV>(p, item, smem + 128, bar, phase); break;
    default: band_item<A, WIN_R, MODE_SHW>(p, item, smem + 128, bar, phase); break;
    }
}

__global__ void batch_finalize_kernel(const BatchQuery *queries, const BatchCtl *ctl,
                                      const int32_t *ends, hy_hit *out) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= ctl->n_queries) return;
    const BatchQuery &bq = queries[slot];
    const unsigned long long k = *bq.sp[PK_BULK].best_key;
    hy_hit h;
    h.score = (int32_t)((uint32_t)(k >> 32) ^ 0x80000000u);
    h.reserved = 0;
    h.db_index = ~(uint32_t)(k & 0xffffffffu);
    h.query_end = bq.ends ? (int64_t)ends[3 * (size_t)slot + 1] : -1;
    h.target_end = bq.ends ? (int64_t)ends[3 * (size_t)slot + 2] : -1;
    out[slot] = h;
}

// ---- host side ------------------------------------------------------------------------------

#define HB_CK(call)                                                                  \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            cudaGetLastError();                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? HY_ERR_OUT_OF_MEMORY : HY_ERR_CUDA, e_); \
        }                                                                            \
    } while (0)

static size_t align128(size_t x) { return (x + 127) / 128 * 128; }

static size_t pass_bytes_of(int32_t al, int rpp, size_t row_bytes) {
    return (size_t)(al + 1) * rpp * row_bytes;
}

// Which profiles one query needs and their shapes.
struct QueryKinds {
    QuerySplit split;
    int rows = 8;
    bool need[PK_N] = {false, false, false, false};
    QueryPlan qp[PK_N];
    uint64_t bytes = 0;  // device bytes of all needed profiles (128-byte aligned each)
};

static void plan_kinds(const hy_db *db, uint64_t qlen, bool ends, const BatchConfig &cfg, QueryKinds &k) {
    const bool tab = db->layout == HY_LAYOUT_PRECOMPUTED;
    k.split = split_for_query(db, qlen, cfg.long_w);
    // SW scores (the bulk classes never record ends) take the plain scan's two-column shapes; the
    // other modes the tuned thresholds.
    if (db->mode == MODE_SW)
        k.rows = bulk_rows(qlen, true);
    else
        k.rows = (int64_t)qlen <= cfg.rows8_max ? 8 : (int64_t)qlen <= cfg.rows16_max ? 16 : 32;
    const QuerySplit &sp = k.split;
    k.need[PK_BULK] = sp.kl < db->p16.n_items;
    k.need[PK_W16] = sp.kl > sp.k0 || ends;
    k.need[PK_I32] = sp.n_i32 > 0;
    k.need[PK_W32] = ends && sp.n_i32 > 0;
    const int rpp[PK_N] = {MAIN_G * k.rows, LCG * LCR, ICG * ICR, WIN_G * WIN_R};
    k.bytes = 0;
    for (int i = 0; i < PK_N; ++i) {
        const bool i16 = i == PK_BULK || i == PK_W16;
        k.qp[i] = !i16 ? plan_for<Single32>(qlen, rpp[i], db->al)
                  : tab ? plan_for<PairTab16>(qlen, rpp[i], db->al)
                        : plan_for<Pair16>(qlen, rpp[i], db->al);
        if (k.need[i]) k.bytes += align128((size_t)k.qp[i].pass_bytes * k.qp[i].n_passes);
    }
}

template <class A, int G, int R, int PK, bool SW_ONLY = false>
static cudaError_t prepare_class(hy_batch *b, int cls, size_t smem, int n_sm) {
    auto kern = batch_scan_kernel<A, G, R, PK, SW_ONLY>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem);
    if (e != cudaSuccess) return e;
    b->grid[cls] = std::max(1, per_sm) * n_sm;
    b->smem[cls] = smem;
    return cudaSuccess;
}

template <class A, int G, int R, int PK, bool SW_ONLY = false>
static void launch_class(hy_batch *b, int cls, uint8_t *bnd, size_t stride, cudaStream_t st) {
    ClassLaunch L;
    L.queries = b->d_queries;
    L.order = b->d_order + (size_t)cls * b->max_queries;
    L.ctl = b->d_ctl;
    L.cls = cls;
    L.bnd = bnd;
    L.bnd_stride = stride;
    batch_scan_kernel<A, G, R, PK, SW_ONLY><<<b->grid[cls], 256, b->smem[cls], st>>>(L);
}

// Records the batch's device work on b->stream (under stream capture).
static hy_status record_graph_body(hy_batch *b) {
    HB_CK(cudaMemsetAsync(&b->d_ctl->head[0], 0, sizeof(uint32_t) * BC_N, b->stream));
    HB_CK(cudaMemsetAsync(b->d_keys, 0, sizeof(unsigned long long) * b->max_queries, b->stream));
    batch_profile_kernel<<<dim3(32, b->max_queries * PK_N), 256, 0, b->stream>>>(b->d_queries, b->d_ctl);
    HB_CK(cudaGetLastError());
    HB_CK(cudaEventRecord(b->ev_fork, b->stream));
    HB_CK(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
    launch_class<Pair16, LCG, LCR, PK_W16>(b, BC_LONG, b->d_bnd_side, b->stride_side, b->side);
    launch_class<PairTab16, LCG, LCR, PK_W16>(b, BC_TLONG, b->d_bnd_side, b->stride_side, b->side);
    launch_class<Single32, ICG, ICR, PK_I32>(b, BC_I32, b->d_bnd_side, b->stride_side, b->side);
    HB_CK(cudaGetLastError());
    HB_CK(cudaEventRecord(b->ev_join, b->side));
    launch_class<Pair16, MAIN_G, 32, PK_BULK>(b, BC_BULK32, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<Pair16, MAIN_G, 16, PK_BULK>(b, BC_BULK16, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<Pair16, MAIN_G, 8, PK_BULK>(b, BC_BULK8, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<PairTab16, MAIN_G, 32, PK_BULK>(b, BC_TBULK32, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<PairTab16, MAIN_G, 16, PK_BULK>(b, BC_TBULK16, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<PairTab16, MAIN_G, 8, PK_BULK>(b, BC_TBULK8, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<Pair16, MAIN_G, 16, PK_BULK, true>(b, BC_SW16, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<Pair16, MAIN_G, 8, PK_BULK, true>(b, BC_SW8, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<PairTab16, MAIN_G, 16, PK_BULK, true>(b, BC_TSW16, b->d_bnd_bulk, b->stride_bulk, b->stream);
    launch_class<PairTab16, MAIN_G, 8, PK_BULK, true>(b, BC_TSW8, b->d_bnd_bulk, b->stride_bulk, b->stream);
    HB_CK(cudaGetLastError());
    HB_CK(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
    BandLaunch bl;
    bl.queries = b->d_queries;
    bl.ctl = b->d_ctl;
    bl.bnd = b->d_bnd_band;
    bl.bnd_stride = b->stride_band;
    bl.ends = b->d_ends;
    batch_band_kernel<Pair16, PK_W16><<<b->max_queries, b->band_threads, b->band_smem, b->stream>>>(bl);
    batch_band_kernel<PairTab16, PK_W16><<<b->max_queries, b->band_threads, b->band_smem, b->stream>>>(bl);
    batch_band_kernel<Single32, PK_W32><<<b->max_queries, b->band_threads, b->band_smem, b->stream>>>(bl);
    batch_finalize_kernel<<<(b->max_queries + 127) / 128, 128, 0, b->stream>>>(b->d_queries, b->d_ctl,
                                                                               b->d_ends, b->d_hits);
    HB_CK(cudaGetLastError());
    b->kernels_per_run = 19;
    return fail(HY_OK);
}

void batch_free(hy_batch *b) {
    if (!b) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    void *dev[] = {b->d_queries, b->d_ctl, b->d_order, b->d_qres, b->d_prof, b->d_bnd_bulk,
                   b->d_bnd_side, b->d_bnd_band, b->d_keys, b->d_ends, b->d_hits, b->d_err};
    for (void *p : dev)
        if (p) hy::dev_free(p);
    void *host[] = {b->h_queries, b->h_ctl, b->h_order, b->h_qres, b->h_hits, b->h_err};
    for (void *p : host)
        if (p) cudaFreeHost(p);
    cudaEvent_t evs[] = {b->ev_fork, b->ev_join, b->ev_t0, b->ev_t1};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->side) cudaStreamDestroy(b->side);
    cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    delete b;
}

struct BatchDeviceGuard {
    int prev = -1;
    explicit BatchDeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
        cudaGetLastError();
    }
    ~BatchDeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
        cudaGetLastError();
    }
};

uint64_t batch_profile_bytes(const hy_batch *b, const hy_db *db, uint64_t qlen, bool ends) {
    QueryKinds k;
    plan_kinds(db, qlen, ends && db->search_type != HY_SEARCH_SCORE, b->cfg, k);
    return k.bytes;
}

hy_status batch_stage(hy_batch *b, const BatchItem *items, uint32_t n, const BatchConfig &cfg,
                      uint32_t chunk_stride, uint32_t *failed) {
    if (n > b->max_queries) return fail(HY_ERR_INVALID_ARGUMENT, n, b->max_queries);
    if (n > 0 && !items) return fail(HY_ERR_INVALID_ARGUMENT);
    uint64_t total_res = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (failed) *failed = i;
        const BatchItem &it = items[i];
        if (it.db >= b->dbs.size()) return fail(HY_ERR_INVALID_ARGUMENT, it.db, (int64_t)b->dbs.size());
        const hy_db *db = b->dbs[it.db];
        if (it.qlen > db->mql) return fail(HY_ERR_QUERY_TOO_LONG, (int64_t)it.qlen, (int64_t)db->mql);
        if (it.qlen && !it.q) return fail(HY_ERR_INVALID_ARGUMENT);
        for (uint64_t k = 0; k < it.qlen; ++k)
            if (it.q[k] >= db->al) return fail(HY_ERR_SYMBOL_OUT_OF_RANGE, it.q[k], (int64_t)db->al);
        total_res += it.qlen;
    }
    if (failed) *failed = n;
    if (total_res > b->max_q_res) return fail(HY_ERR_INVALID_ARGUMENT, (int64_t)total_res, (int64_t)b->max_q_res);
    BatchCtl &ctl = *b->h_ctl;
    memset(&ctl, 0, sizeof(ctl));
    ctl.n_queries = n;
    ctl.chunk_stride = std::max<uint32_t>(1, chunk_stride);
    std::vector<std::vector<uint32_t>> lists(BC_N);
    uint64_t prof_off = 0, q_off = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const BatchItem &it = items[i];
        const hy_db *db = b->dbs[it.db];
        const uint64_t qlen = it.qlen;
        if (qlen) memcpy(b->h_qres + q_off, it.q, qlen);
        BatchQuery &bq = b->h_queries[i];
        memset(&bq, 0, sizeof(bq));
        const bool ends = it.ends && db->search_type != HY_SEARCH_SCORE;
        QueryKinds k;
        plan_kinds(db, qlen, ends, cfg, k);
        if (prof_off + k.bytes > b->prof_cap) {
            if (failed) *failed = i;
            return fail(HY_ERR_REJECTED, (int64_t)(prof_off + k.bytes), (int64_t)b->prof_cap);
        }
        const QuerySplit &sp = k.split;
        bq.matrix = db->d_matrix;
        bq.q = b->d_qres + q_off;
        bq.rank = db->d_rank;
        bq.qlen = (int32_t)qlen;
        bq.mode = db->mode;
        bq.ends = ends ? 1 : 0;
        bq.bulk_rows = k.rows;
        bq.top_free = (db->mode == MODE_SW || db->mode == MODE_HW || db->mode == MODE_OV) ? 1 : 0;
        bq.al = (int32_t)db->al;
        bq.lim16 = 32767 - db->go;
        bq.tab = db->layout == HY_LAYOUT_PRECOMPUTED ? 1 : 0;
        bq.k0 = sp.k0;
        bq.kl = sp.kl;
        bq.n_i32 = sp.n_i32;
        bq.n16 = db->p16.n_items;
        for (int kk = 0; kk < PK_N; ++kk) {
            ScanParams &p = bq.sp[kk];
            const bool i16 = kk == PK_BULK || kk == PK_W16;
            const Partition &part = i16 ? db->p16 : db->p32;
            p.meta = part.d_meta;
            p.n_items = part.n_items;
            p.res = part.d_res;
            p.qlen = (int32_t)qlen;
            p.go = db->go;
            p.ge = db->ge;
            p.sentinel = i16 ? (-32768 + db->ge) : (INT32_MIN / 4);
            p.scores = it.d_scores;
            p.best_key = b->d_keys + i;
            p.err = b->d_err;
            p.wait_polls = wait_polls();
            if (i16)
                set_extents<Pair16>(p, db, part, 0);
            else
                set_extents<Single32>(p, db, part, 0);
            if (i16 && bq.tab) p.letters = (uint32_t)PairTab16::letters((int64_t)db->al);
            if (!k.need[kk]) continue;
            p.pass_bytes = k.qp[kk].pass_bytes;
            p.n_passes = k.qp[kk].n_passes;
            p.vrow0 = k.qp[kk].vrow0;
            p.profile = b->d_prof + prof_off;
            prof_off += align128((size_t)p.pass_bytes * p.n_passes);
        }
        q_off += qlen;
        const int bulk_cls = db->mode == MODE_SW
                                 ? (k.rows == 8 ? BC_SW8 : BC_SW16) + (bq.tab ? BC_TSW8 - BC_SW8 : 0)
                                 : (k.rows == 8 ? BC_BULK8 : k.rows == 16 ? BC_BULK16 : BC_BULK32) +
                                       (bq.tab ? BC_TBULK8 - BC_BULK8 : 0);
        const int long_cls = bq.tab ? BC_TLONG : BC_LONG;
        if (sp.kl < db->p16.n_items) {
            lists[bulk_cls].push_back(i);
            ctl.n_chunks[bulk_cls] = std::max<uint32_t>(ctl.n_chunks[bulk_cls], (db->p16.n_items + 31) / 32);
        }
        if (sp.kl > sp.k0) {
            lists[long_cls].push_back(i);
            ctl.n_chunks[long_cls] = std::max<uint32_t>(ctl.n_chunks[long_cls], (sp.kl + 7) / 8);
        }
        if (sp.n_i32 > 0) {
            lists[BC_I32].push_back(i);
            ctl.n_chunks[BC_I32] = std::max<uint32_t>(ctl.n_chunks[BC_I32], (sp.n_i32 + 7) / 8);
        }
    }
    for (int c = 0; c < BC_N; ++c) {
        std::vector<uint32_t> &l = lists[c];
        std::stable_sort(l.begin(), l.end(), [&](uint32_t x, uint32_t y) {
            return b->h_queries[x].qlen > b->h_queries[y].qlen;
        });
        ctl.count[c] = (uint32_t)l.size();
        std::copy(l.begin(), l.end(), b->h_order + (size_t)c * b->max_queries);
    }
    return fail(HY_OK);
}

hy_status batch_launch(hy_batch *b, uint32_t n) {
    uint64_t total_res = 0;
    for (uint32_t i = 0; i < n; ++i) total_res += (uint64_t)b->h_queries[i].qlen;
    if (total_res) HB_CK(cudaMemcpyAsync(b->d_qres, b->h_qres, total_res, cudaMemcpyHostToDevice, b->stream));
    if (n) HB_CK(cudaMemcpyAsync(b->d_queries, b->h_queries, sizeof(BatchQuery) * n, cudaMemcpyHostToDevice, b->stream));
    HB_CK(cudaMemcpyAsync(b->d_order, b->h_order, sizeof(uint32_t) * BC_N * b->max_queries,
                          cudaMemcpyHostToDevice, b->stream));
    HB_CK(cudaMemcpyAsync(b->d_ctl, b->h_ctl, sizeof(BatchCtl), cudaMemcpyHostToDevice, b->stream));
    HB_CK(cudaGraphLaunch(b->exec, b->stream));
    if (n) HB_CK(cudaMemcpyAsync(b->h_hits, b->d_hits, sizeof(hy_hit) * n, cudaMemcpyDeviceToHost, b->stream));
    HB_CK(cudaMemcpyAsync(b->h_err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    ++b->runs;
    return fail(HY_OK);
}

hy_status batch_collect(hy_batch *b, uint32_t n, hy_hit *out) {
    if (const int w = *b->h_err) {
        *b->h_err = 0;
        HB_CK(cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream));
        HB_CK(cudaStreamSynchronize(b->stream));
        return fail(device_error(w));
    }
    if (n && out) memcpy(out, b->h_hits, sizeof(hy_hit) * n);
    return fail(HY_OK);
}

static hy_status run_sync(hy_batch *b, uint32_t n, hy_hit *out) {
    hy_status st = batch_launch(b, n);
    if (st != HY_OK) return st;
    HB_CK(cudaStreamSynchronize(b->stream));
    return batch_collect(b, n, out);
}

// Shape signature of a batch: the share of queries in each (mode, log2 length) bucket, in
// eighths, plus the databases used.
static uint64_t batch_signature(const hy_batch *b, const BatchItem *items, uint32_t n) {
    std::vector<uint32_t> hist(5 * 24, 0);
    std::vector<char> used(b->dbs.size(), 0);
    for (uint32_t i = 0; i < n; ++i) {
        int lg = 0;
        while (lg < 23 && (1ull << (lg + 1)) <= items[i].qlen + 1) ++lg;
        ++hist[b->dbs[items[i].db]->mode * 24 + lg];
        used[items[i].db] = 1;
    }
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
    for (uint32_t c : hist) mix(n ? (uint64_t)std::lround(8.0 * c / n) : 0);
    for (char u : used) mix((uint64_t)u);
    return h;
}

// Times one configuration on a sampled part of the batch (every `stride`-th item chunk).
static hy_status time_config(hy_batch *b, const BatchItem *items, uint32_t n, const BatchConfig &cfg,
                             uint32_t stride, float *ms) {
    hy_status st = batch_stage(b, items, n, cfg, stride, nullptr);
    if (st != HY_OK) return st;
    HB_CK(cudaEventRecord(b->ev_t0, b->stream));
    st = batch_launch(b, n);
    if (st != HY_OK) return st;
    HB_CK(cudaEventRecord(b->ev_t1, b->stream));
    HB_CK(cudaStreamSynchronize(b->stream));
    st = batch_collect(b, 0, nullptr);
    if (st != HY_OK) return st;
    HB_CK(cudaEventElapsedTime(ms, b->ev_t0, b->ev_t1));
    return fail(HY_OK);
}

// Coordinate search: the rows-per-lane thresholds first (at the default split), then the split.
static hy_status tune(hy_batch *b, const BatchItem *items, uint32_t n, uint32_t stride,
                      BatchConfig *best_cfg, double *best_ms) {
    static const int32_t rows_c[][2] = {{64, 192}, {0, 256}, {128, 512}, {0, 0}, {64, 64}, {32, 128}};
    static const uint32_t long_c[] = {1024, 2048, 4096};
    BatchConfig best = b->cfg;
    float best_t = 1e30f;
    for (const auto &rc : rows_c) {
        BatchConfig c;
        c.rows8_max = rc[0];
        c.rows16_max = rc[1];
        c.long_w = LONG_W;
        float t = 0;
        hy_status st = time_config(b, items, n, c, stride, &t);
        if (st != HY_OK) return st;
        if (t < best_t) {
            best_t = t;
            best = c;
        }
    }
    for (uint32_t lw : long_c) {
        if (lw == LONG_W) continue;
        BatchConfig c = best;
        c.long_w = lw;
        float t = 0;
        hy_status st = time_config(b, items, n, c, stride, &t);
        if (st != HY_OK) return st;
        if (t < best_t) {
            best_t = t;
            best = c;
        }
    }
    *best_cfg = best;
    if (best_ms) *best_ms = best_t;
    return fail(HY_OK);
}

// The sampling stride that leaves about 256 bulk chunks per query in a tuning run.
static uint32_t sample_stride(const hy_batch *b) {
    uint32_t n16 = 0;
    for (const hy_db *db : b->dbs) n16 = std::max(n16, db->p16.n_items);
    return std::max<uint32_t>(1, (n16 + 31) / 32 / 256);
}

static hy_status items_from_arrays(const hy_batch *b, uint32_t n, const uint32_t *dbq,
                                   const uint8_t *q_res, const uint64_t *q_off,
                                   std::vector<BatchItem> &items) {
    if (n > 0 && (!dbq || !q_off)) return fail(HY_ERR_INVALID_ARGUMENT);
    items.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        if (q_off[i + 1] < q_off[i]) return fail(HY_ERR_INVALID_ARGUMENT);
        items[i].db = dbq[i];
        items[i].qlen = q_off[i + 1] - q_off[i];
        items[i].q = items[i].qlen ? q_res + (q_off[i] - q_off[0]) : nullptr;
        items[i].d_scores = nullptr;
        items[i].ends = true;
        if (items[i].qlen && !q_res) return fail(HY_ERR_INVALID_ARGUMENT);
    }
    (void)b;
    return fail(HY_OK);
}

hy_status batch_create(const hy_db *const *dbs, uint32_t n_dbs, uint32_t max_queries,
                       uint64_t prof_cap, bool autotune, hy_batch **out) {
    if (!dbs || n_dbs == 0 || max_queries == 0 || !out) return fail(HY_ERR_INVALID_ARGUMENT);
    *out = nullptr;
    for (uint32_t i = 0; i < n_dbs; ++i) {
        if (!dbs[i]) return fail(HY_ERR_INVALID_ARGUMENT);
        if (dbs[i]->device != dbs[0]->device) return fail(HY_ERR_INVALID_ARGUMENT, i);
    }
    if (max_queries > 16000) return fail(HY_ERR_INVALID_ARGUMENT, max_queries, 16000);
    hy_batch *b = new hy_batch();
    b->device = dbs[0]->device;
    b->dbs.assign(dbs, dbs + n_dbs);
    b->max_queries = max_queries;
    b->autotune = autotune;
    for (const hy_db *db : b->dbs) {
        b->al_max = std::max<int32_t>(b->al_max, (int32_t)db->al);
        b->mql_max = std::max(b->mql_max, db->mql);
        b->max_t = std::max(b->max_t, db->max_t);
    }
    b->max_q_res = std::max<uint64_t>(1, (uint64_t)max_queries * b->mql_max);
    BatchDeviceGuard guard(b->device);
    hy_status st = HY_OK;
    auto ck = [&](cudaError_t e) {
        if (st == HY_OK && e != cudaSuccess) {
            cudaGetLastError();
            st = fail(e == cudaErrorMemoryAllocation ? HY_ERR_OUT_OF_MEMORY : HY_ERR_CUDA, e);
        }
    };
    int n_sm = 0, smem_optin = 0;
    ck(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, b->device));
    ck(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device));
    const int32_t al = b->al_max;
    const size_t pb16 = profile_row_bytes<Pair16>(), pb32 = profile_row_bytes<Single32>();
    const size_t sm_bulk32 = 128 + 2 * pass_bytes_of(al, MAIN_G * 32, pb16);
    const size_t sm_bulk16 = 128 + 2 * pass_bytes_of(al, MAIN_G * 16, pb16);
    const size_t sm_bulk8 = 128 + 2 * pass_bytes_of(al, MAIN_G * 8, pb16);
    const size_t sm_long = 128 + 2 * pass_bytes_of(al, LCG * LCR, pb16);
    const size_t sm_i32 = 128 + 2 * pass_bytes_of(al, ICG * ICR, pb32);
    // The Precomputed classes size their pair tables by the largest alphabet among the
    // Precomputed databases (0 letters when there is none: those classes then never run).
    int32_t al_tab = -1;
    for (const hy_db *db : b->dbs)
        if (db->layout == HY_LAYOUT_PRECOMPUTED) al_tab = std::max<int32_t>(al_tab, (int32_t)db->al);
    const size_t tab_row = al_tab < 0 ? 0 : profile_slice_row_bytes<PairTab16>(al_tab);
    const size_t sm_tbulk32 = 128 + 2 * tab_row * MAIN_G * 32;
    const size_t sm_tbulk16 = 128 + 2 * tab_row * MAIN_G * 16;
    const size_t sm_tbulk8 = 128 + 2 * tab_row * MAIN_G * 8;
    const size_t sm_tlong = 128 + 2 * tab_row * LCG * LCR;
    const size_t band_pass = std::max({pass_bytes_of(al, WIN_G * WIN_R, pb16), pass_bytes_of(al, WIN_G * WIN_R, pb32),
                                       tab_row * WIN_G * WIN_R});
    if (st == HY_OK && (std::max({sm_bulk32, sm_long, sm_i32, sm_tbulk32, sm_tlong}) > (size_t)smem_optin ||
                        128 + band_pass > (size_t)smem_optin)) {
        st = fail(HY_ERR_UNSUPPORTED, al, smem_optin);
    }
    if (st == HY_OK) {
        ck(prepare_class<Pair16, MAIN_G, 8, PK_BULK>(b, BC_BULK8, sm_bulk8, n_sm));
        ck(prepare_class<Pair16, MAIN_G, 16, PK_BULK>(b, BC_BULK16, sm_bulk16, n_sm));
        ck(prepare_class<Pair16, MAIN_G, 32, PK_BULK>(b, BC_BULK32, sm_bulk32, n_sm));
        ck(prepare_class<Pair16, LCG, LCR, PK_W16>(b, BC_LONG, sm_long, n_sm));
        ck(prepare_class<Single32, ICG, ICR, PK_I32>(b, BC_I32, sm_i32, n_sm));
        ck(prepare_class<PairTab16, MAIN_G, 8, PK_BULK>(b, BC_TBULK8, sm_tbulk8, n_sm));
        ck(prepare_class<PairTab16, MAIN_G, 16, PK_BULK>(b, BC_TBULK16, sm_tbulk16, n_sm));
        ck(prepare_class<PairTab16, MAIN_G, 32, PK_BULK>(b, BC_TBULK32, sm_tbulk32, n_sm));
        ck(prepare_class<PairTab16, LCG, LCR, PK_W16>(b, BC_TLONG, sm_tlong, n_sm));
        ck(prepare_class<Pair16, MAIN_G, 8, PK_BULK, true>(b, BC_SW8, sm_bulk8, n_sm));
        ck(prepare_class<Pair16, MAIN_G, 16, PK_BULK, true>(b, BC_SW16, sm_bulk16, n_sm));
        ck(prepare_class<PairTab16, MAIN_G, 8, PK_BULK, true>(b, BC_TSW8, sm_tbulk8, n_sm));
        ck(prepare_class<PairTab16, MAIN_G, 16, PK_BULK, true>(b, BC_TSW16, sm_tbulk16, n_sm));
        int warps = (int)std::min<size_t>(32, BAND_SMEM_BUDGET / std::max<size_t>(band_pass, 1));
        warps = std::max(1, warps);
        b->band_threads = 32 * warps;
        b->band_smem = 128 + (size_t)warps * band_pass;
        ck(cudaFuncSetAttribute(batch_band_kernel<Pair16, PK_W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->band_smem));
        ck(cudaFuncSetAttribute(batch_band_kernel<Single32, PK_W32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->band_smem));
        ck(cudaFuncSetAttribute(batch_band_kernel<PairTab16, PK_W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->band_smem));
    }
    // Boundary regions: a block's unit spans at most IPU items of the class's widest width.
    const bool multipass = b->mql_max > (uint64_t)MAIN_G * 8;
    const uint64_t w_bulk = std::min<uint64_t>(b->max_t, LONG_W_MAX) + 16;
    b->stride_bulk = multipass ? align128(32 * w_bulk * 2 * sizeof(uint32_t)) : 128;
    b->stride_side = multipass ? align128(8 * (b->max_t + 16) * 2 * sizeof(uint32_t)) : 128;
    b->stride_band = align128((b->max_t + 16) * 2 * sizeof(uint32_t));
    const int side_grid = std::max({b->grid[BC_LONG], b->grid[BC_I32], b->grid[BC_TLONG]});
    const int bulk_grid = std::max({b->grid[BC_BULK8], b->grid[BC_BULK16], b->grid[BC_BULK32],
                                    b->grid[BC_TBULK8], b->grid[BC_TBULK16], b->grid[BC_TBULK32],
                                    b->grid[BC_SW8], b->grid[BC_SW16], b->grid[BC_TSW8], b->grid[BC_TSW16]});
    const uint64_t mq = b->mql_max;
    const uint64_t pair_row = std::max<uint64_t>(pass_bytes_of(al, 1, pb16), tab_row);
    const uint64_t per_query = align128(pair_row * (mq + 255)) +                   // bulk, any rows
                               align128(pair_row * (mq + 255)) +                   // long / band int16x2
                               align128(pass_bytes_of(al, 1, pb32) * (mq + 511)) +  // int32
                               align128(pass_bytes_of(al, 1, pb32) * (mq + 255));   // band int32
    b->prof_cap = prof_cap ? prof_cap : per_query * max_queries;
    if (st == HY_OK) {
        ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        ck(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
        ck(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
        ck(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
        ck(cudaEventCreate(&b->ev_t0));
        ck(cudaEventCreate(&b->ev_t1));
        auto dalloc = [&](void **p, size_t bytes) {
            ck(hy::dev_malloc(p, std::max<size_t>(bytes, 16)));
            if (st == HY_OK) b->device_bytes += bytes;
        };
        dalloc((void **)&b->d_queries, sizeof(BatchQuery) * max_queries);
        dalloc((void **)&b->d_ctl, sizeof(BatchCtl));
        dalloc((void **)&b->d_order, sizeof(uint32_t) * BC_N * max_queries);
        dalloc((void **)&b->d_qres, b->max_q_res);
        dalloc((void **)&b->d_prof, b->prof_cap);
        dalloc((void **)&b->d_bnd_bulk, b->stride_bulk * bulk_grid);
        dalloc((void **)&b->d_bnd_side, b->stride_side * side_grid);
        dalloc((void **)&b->d_bnd_band, b->stride_band * max_queries);
        dalloc((void **)&b->d_keys, sizeof(unsigned long long) * max_queries);
        dalloc((void **)&b->d_ends, 3 * sizeof(int32_t) * max_queries);
        dalloc((void **)&b->d_hits, sizeof(hy_hit) * max_queries);
        dalloc((void **)&b->d_err, 64);
        ck(cudaMallocHost((void **)&b->h_queries, sizeof(BatchQuery) * max_queries));
        ck(cudaMallocHost((void **)&b->h_ctl, sizeof(BatchCtl)));
        ck(cudaMallocHost((void **)&b->h_order, sizeof(uint32_t) * BC_N * max_queries));
        ck(cudaMallocHost((void **)&b->h_qres, b->max_q_res));
        ck(cudaMallocHost((void **)&b->h_hits, sizeof(hy_hit) * max_queries));
        ck(cudaMallocHost((void **)&b->h_err, sizeof(int)));
    }
    if (st == HY_OK) {
        ck(cudaMemset(b->d_err, 0, 64));
        ck(cudaMemset(b->d_ctl, 0, sizeof(BatchCtl)));
        *b->h_err = 0;
    }
    if (st == HY_OK) {
        cudaGraph_t graph = nullptr;
        ck(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        if (st == HY_OK) {
            hy_status rs = record_graph_body(b);
            cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
            if (rs != HY_OK && st == HY_OK) st = rs;
            ck(e);
        }
        if (st == HY_OK) ck(cudaGraphInstantiate(&b->exec, graph, 0));
        if (graph) cudaGraphDestroy(graph);
    }
    if (st != HY_OK) {
        int64_t d[3];
        hy_last_error_detail(d);
        batch_free(b);
        return fail(st, d[0], d[1], d[2]);
    }
    *out = b;
    return fail(HY_OK);
}

}  // namespace hy

extern "C" {

hy_status hy_batch_create(const hy_db *const *dbs, uint32_t n_dbs, uint32_t max_queries,
                          int autotune, hy_batch **out) {
    return batch_create(dbs, n_dbs, max_queries, 0, autotune != 0, out);
}

void hy_batch_destroy(hy_batch *b) { batch_free(b); }

uint64_t hy_batch_device_bytes(const hy_batch *b) { return b ? b->device_bytes : 0; }

void *hy_batch_stream(hy_batch *b) { return b ? (void *)b->stream : nullptr; }

hy_status hy_batch_get_config(const hy_batch *b, int32_t cfg[3]) {
    if (!b || !cfg) return fail(HY_ERR_INVALID_ARGUMENT);
    cfg[0] = b->cfg.rows8_max;
    cfg[1] = b->cfg.rows16_max;
    cfg[2] = (int32_t)b->cfg.long_w;
    return fail(HY_OK);
}

hy_status hy_batch_set_config(hy_batch *b, const int32_t cfg[3]) {
    if (!b || !cfg || cfg[2] < 1 || (uint32_t)cfg[2] > LONG_W_MAX) return fail(HY_ERR_INVALID_ARGUMENT);
    b->cfg.rows8_max = cfg[0];
    b->cfg.rows16_max = cfg[1];
    b->cfg.long_w = (uint32_t)cfg[2];
    b->autotune = false;
    return fail(HY_OK);
}

hy_status hy_batch_tune(hy_batch *b, uint32_t n_queries, const uint32_t *db_of_query,
                        const uint8_t *q_res, const uint64_t *q_off, uint32_t stride, double *best_ms) {
    if (!b) return fail(HY_ERR_INVALID_ARGUMENT);
    BatchDeviceGuard guard(b->device);
    std::vector<BatchItem> items;
    hy_status st = items_from_arrays(b, n_queries, db_of_query, q_res, q_off, items);
    if (st != HY_OK) return st;
    if (stride == 0) stride = sample_stride(b);
    BatchConfig best;
    st = tune(b, items.data(), n_queries, stride, &best, best_ms);
    if (st != HY_OK) return st;
    b->cfg = best;
    if (n_queries) b->tuned[batch_signature(b, items.data(), n_queries)] = best;
    return fail(HY_OK);
}

hy_status hy_scan_batch(hy_batch *b, uint32_t n_queries, const uint32_t *db_of_query,
                        const uint8_t *q_res, const uint64_t *q_off, hy_hit *out,
                        uint32_t *failed_query) {
    if (!b || (n_queries && !out)) return fail(HY_ERR_INVALID_ARGUMENT);
    BatchDeviceGuard guard(b->device);
    std::vector<BatchItem> items;
    hy_status st = items_from_arrays(b, n_queries, db_of_query, q_res, q_off, items);
    if (st != HY_OK) return st;
    // Validate before any tuning so that errors are reported for the caller's batch as given.
    st = batch_stage(b, items.data(), n_queries, b->cfg, 1, failed_query);
    if (st != HY_OK) return st;
    if (b->autotune && n_queries) {
        const uint64_t sig = batch_signature(b, items.data(), n_queries);
        auto it = b->tuned.find(sig);
        if (it == b->tuned.end()) {
            BatchConfig best;
            st = tune(b, items.data(), n_queries, sample_stride(b), &best, nullptr);
            if (st != HY_OK) return st;
            b->tuned[sig] = best;
            b->cfg = best;
        } else {
            b->cfg = it->second;
        }
        st = batch_stage(b, items.data(), n_queries, b->cfg, 1, failed_query);
        if (st != HY_OK) return st;
    }
    return run_sync(b, n_queries, out);
}

}  // extern "C"
