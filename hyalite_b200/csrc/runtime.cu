// runtime.cu -- host runtime of the cuda backend: the device-resident database (build, width
// partition, length sort, packing), per-thread scratch, and the scan entry points of the C ABI.
//
// Mirrors DatabaseBuilder::build (src/database.rs:737-877), Scratch::new (965-998) and
// Database::scan / scan_all / scan_scores (83-144, 347-464, 481-515); the device kernels live in
// scan_kernel.cuh.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <numeric>
#include <vector>

#include "db_internal.h"
#include "traceback_internal.h"

using namespace hy;

struct hy_scratch {
    const hy_db *db = nullptr;
    int device = 0;  // copied from the database: destroying a scratch never reads its database
    cudaStream_t stream = nullptr;
    // The int32 part of a scan runs on a second stream, forked from and joined back into `stream`.
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

    uint8_t *d_query = nullptr;
    uint8_t *d_prof16 = nullptr, *d_prof32 = nullptr, *d_profw16 = nullptr, *d_profw32 = nullptr;
    void *d_bnd16 = nullptr, *d_bnd32 = nullptr;
    int32_t *d_scores = nullptr, *d_qend = nullptr, *d_tend = nullptr;
    unsigned long long *d_key = nullptr;
    uint32_t *d_win = nullptr;
    hy_hit *d_hit = nullptr;
    int *d_err = nullptr;
    uint8_t *h_query = nullptr;
    hy_hit *h_hit = nullptr;
    int *h_err = nullptr;
    int32_t *h_out = nullptr;  // 3 * n_seqs int32 (scores, qend, tend), allocated on first use
    uint64_t bytes = 0;
    // Optional event timing of the main scan kernels (hy_scratch_profile).
    bool profile = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    // Kernel class of each timed launch: 0 bulk int16x2 pairs, 1 int32 items, 2 long int16x2 pairs.
    std::vector<int> event_part;
    double event_cells[3] = {0.0, 0.0, 0.0};  // real DP cells the timed launches computed
    size_t n_events = 0;
    uint64_t launches = 0;        // every kernel this scratch launched since the last read
    // Traceback (Alignment search type): grow-only buffers, created on first use, and the
    // operations of the last traceback call.
    void *tb = nullptr;
    std::vector<uint8_t> tb_ops;
    // CUDA graphs of small scans (hy_scan / hy_scan_scores / hy_scan_all): one per call kind and
    // query length, captured on first use and replayed instead of launching each kernel; exec is
    // null for a call whose capture failed (it then launches directly).
    struct Graph {
        int kind;
        uint64_t qlen;
        cudaGraphExec_t exec;
        uint64_t launches;  // kernels the graph launches
        uint64_t last_use;
        uint64_t epoch;     // wait_polls_epoch() at capture
    };
    std::vector<Graph> graphs;
    uint64_t graph_clock = 0;
};

namespace hy {

void *scratch_tb(hy_scratch *sc) { return sc ? sc->tb : nullptr; }

#define HY_CK(call)                                                                  \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            cudaGetLastError();                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? HY_ERR_OUT_OF_MEMORY : HY_ERR_CUDA, e_); \
        }                                                                            \
    } while (0)

template <class A, int G, int R, int MODE, bool ENDS, bool GPROF>
static cudaError_t launch_mode(const ScanParams &p, int blocks, int threads, size_t smem,
                               cudaStream_t st) {
    auto kern = scan_kernel<A, G, R, MODE, ENDS, GPROF>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<blocks, threads, smem, st>>>(p);
    return cudaGetLastError();
}

// The launch shapes that also exist in the global-memory-profile form (large alphabets): the bulk
// pairs with 8 rows per lane and the int32 items.
template <class A, int G, int R>
constexpr bool has_gprof_form() {
    return (A::NH == 2 && G == MAIN_G && R == 8) || (A::NH == 1 && G == MAIN_G32 && R == MAIN_R32);
}

template <class A, int G, int R>
static cudaError_t launch_scan(int mode, bool ends, bool gprof, const ScanParams &p, int blocks,
                               int threads, size_t smem, cudaStream_t st) {
    if (gprof) {
        if constexpr (has_gprof_form<A, G, R>()) {
#define HY_MODE_CASE(M)                                                                   \
    case M:                                                                               \
        return ends ? launch_mode<A, G, R, M, true, true>(p, blocks, threads, smem, st)   \
                    : launch_mode<A, G, R, M, false, true>(p, blocks, threads, smem, st);
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
#define HY_MODE_CASE(M)                                                                    \
    case M:                                                                                \
        return ends ? launch_mode<A, G, R, M, true, false>(p, blocks, threads, smem, st)   \
                    : launch_mode<A, G, R, M, false, false>(p, blocks, threads, smem, st);
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

template <class A, int G, int R>
static cudaError_t launch_profile(const hy_db *db, const uint8_t *d_query, uint64_t qlen,
                                  const QueryPlan &qp, int32_t lim, uint8_t *out, cudaStream_t st) {
    const int64_t total = A::letters(db->al) * A::TABLES * G * R * qp.n_passes;
    if (total == 0) return cudaSuccess;
    int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
    const bool top_free = db->mode == MODE_SW || db->mode == MODE_HW || db->mode == MODE_OV;
    build_profile_kernel<A, G, R><<<blocks, 256, 0, st>>>(
        d_query, (int32_t)qlen, db->d_matrix, (int32_t)db->al, db->go, lim, top_free ? 1 : 0,
        qp.vrow0, qp.n_passes, reinterpret_cast<typename A::PE *>(out));
    return cudaGetLastError();
}

static constexpr int32_t LIM32 = 536870911;
static int32_t lim16(const hy_db *db) { return 32767 - db->go; }

// Fill per-target scores (and ends) for every sequence; optionally fold the best hit key.
// Items [item_base, item_end) of `part` (or the single item *item_ptr) on stream `st`.
template <class A, int G, int R>
static hy_status enqueue_partition(const hy_db *db, hy_scratch *sc, const Partition &part,
                                   uint32_t item_base, uint32_t item_end, const uint8_t *d_query,
                                   uint64_t qlen, bool ends, unsigned long long *key,
                                   int32_t *scores, uint8_t *prof, void *bnd,
                                   const uint32_t *item_ptr, int blocks, int threads,
                                   cudaStream_t st_) {
    const bool i16 = sizeof(typename A::V) == 4 && A::NH == 2;
    QueryPlan qp = plan_for<A>(qlen, G * R, db->al);
    HY_CK((launch_profile<A, G, R>(db, d_query, qlen, qp, i16 ? lim16(db) : LIM32, prof, st_)));
    sc->launches += qp.n_passes > 0 ? 2 : 1;
    ScanParams p{};
    p.meta = part.d_meta;
    p.item_base = item_base;
    p.n_items = item_end;
    p.item_ptr = item_ptr;
    p.res = part.d_res;
    p.profile = prof;
    p.pass_bytes = qp.pass_bytes;
    p.n_passes = qp.n_passes;
    p.vrow0 = qp.vrow0;
    p.qlen = (int32_t)qlen;
    p.go = db->go;
    p.ge = db->ge;
    p.sentinel = i16 ? (-32768 + db->ge) : (INT32_MIN / 4);
    p.boundary = bnd;
    p.scores = scores;
    p.qend = sc->d_qend;
    p.tend = sc->d_tend;
    p.best_key = key;
    p.err = sc->d_err;
    p.wait_polls = wait_polls();
    set_extents<A>(p, db, part, part.total_cols);
    size_t smem = 2 * (size_t)qp.pass_bytes + 16;
    const bool gprof = smem > db->smem_limit;
    if (gprof) smem = 16;
    const bool timed = sc->profile && item_ptr == nullptr;
    if (timed) {
        if (sc->n_events == sc->events.size()) {
            cudaEvent_t a, b;
            HY_CK(cudaEventCreate(&a));
            HY_CK(cudaEventCreate(&b));
            sc->events.push_back({a, b});
            sc->event_part.push_back(0);
        }
        const int cls = i16 ? 0 : 1;
        sc->event_part[sc->n_events] = cls;
        sc->event_cells[cls] +=
            (double)qlen * (double)(part.res_prefix[item_end] - part.res_prefix[item_base]);
        HY_CK(cudaEventRecord(sc->events[sc->n_events].first, st_));
    }
    HY_CK((launch_scan<A, G, R>(db->mode, ends, gprof, p, blocks, threads, smem, st_)));
    if (timed) {
        HY_CK(cudaEventRecord(sc->events[sc->n_events].second, st_));
        ++sc->n_events;
    }
    return fail(HY_OK);
}

// Per-target scores (and ends) for every sequence, optionally folding the best-hit key. The
// int32 items of this query run on the scratch's second stream, concurrently with the int16x2
// pairs, and are joined back before the call's later work.
// P is the int16x2 pair arithmetic of the database's layout (Pair16: Gathered, PairTab16:
// Precomputed).
template <class P>
static hy_status enqueue_scores_p(const hy_db *db, hy_scratch *sc, const uint8_t *d_query,
                                  uint64_t qlen, bool ends, unsigned long long *key, int32_t *scores) {
    hy_status st;
    const QuerySplit split = split_for_query(db, qlen);
    const int gpb = BLOCK / MAIN_G;
    const bool forked = split.n_i32 > 0;
    if (forked) {
        HY_CK(cudaEventRecord(sc->ev_fork, sc->stream));
        HY_CK(cudaStreamWaitEvent(sc->stream2, sc->ev_fork, 0));
        const int gpb32 = BLOCK / MAIN_G32;
        const int blocks = (int)((split.n_i32 + gpb32 - 1) / gpb32);
        st = enqueue_partition<Single32, MAIN_G32, MAIN_R32>(db, sc, db->p32, 0, split.n_i32, d_query,
                                                          qlen, ends, key, scores, sc->d_prof32,
                                                          sc->d_bnd32, nullptr, blocks, BLOCK,
                                                          sc->stream2);
        if (st != HY_OK) return st;
        HY_CK(cudaEventRecord(sc->ev_join, sc->stream2));
    }
    if (split.k0 < db->p16.n_items) {
        const int blocks = (int)((db->p16.n_items - split.k0 + gpb - 1) / gpb);
        // Rows per lane by query length: more rows amortise the per-step work, fewer keep the
        // padding of a short query's single pass small. An alphabet whose two pass slices do not
        // fit in shared memory runs with 8 rows, from the profile in global memory if need be.
        int rows = bulk_rows(qlen, db->mode == MODE_SW && !ends);
        const size_t slice = profile_slice_row_bytes<P>(db->al) * MAIN_G;
        if (2 * slice * rows + 16 > db->smem_limit) rows = 8;
#define HY_BULK(RR)                                                                              \
    enqueue_partition<P, MAIN_G, RR>(db, sc, db->p16, split.k0, db->p16.n_items, d_query,        \
                                          qlen, ends, key, scores, sc->d_prof16, sc->d_bnd16,    \
                                          nullptr, blocks, BLOCK, sc->stream)
        st = rows == 8 ? HY_BULK(8) : rows == 16 ? HY_BULK(16) : HY_BULK(32);
#undef HY_BULK
        if (st != HY_OK) return st;
    }
    if (forked) HY_CK(cudaStreamWaitEvent(sc->stream, sc->ev_join, 0));
    return fail(HY_OK);
}

static hy_status enqueue_scores(const hy_db *db, hy_scratch *sc, const uint8_t *d_query,
                                uint64_t qlen, bool ends, unsigned long long *key, int32_t *scores) {
    return db->layout == HY_LAYOUT_PRECOMPUTED
               ? enqueue_scores_p<PairTab16>(db, sc, d_query, qlen, ends, key, scores)
               : enqueue_scores_p<Pair16>(db, sc, d_query, qlen, ends, key, scores);
}

// The winner's item: its int16x2 pair when that pair ran packed for this query (pair >= k0),
// else its int32 single (the 2*k0 longest sequences). The other slot gets NO_INDEX. A key of 0
// means no item recorded a hit (a scan kernel gave up on a bounded wait): no winner then.
__global__ void winner_loc_kernel(const unsigned long long *key, const uint32_t *rank, uint32_t k0,
                                  uint32_t *win) {
    if (*key == 0) {
        win[0] = win[1] = NO_INDEX;
        return;
    }
    const uint32_t idx = ~(uint32_t)(*key & 0xffffffffu);
    const uint32_t r = rank[idx];
    const bool packed = r / 2 >= k0;
    win[0] = packed ? r / 2 : NO_INDEX;
    win[1] = packed ? NO_INDEX : r;
}

// The band kernel on one block, or on a cluster of `blocks` blocks (at most 8, the portable
// cluster size every launch shape of one block per SM can be given).
template <class A, int MODE, bool GPROF>
static cudaError_t launch_band_mode(const ScanParams &p, int warps, int blocks, size_t smem, cudaStream_t st) {
    auto kern = band_kernel<A, WIN_R, MODE, GPROF>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    if (GPROF || blocks <= 1) {
        kern<<<1, 32 * warps, smem, st>>>(p);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(32u * (unsigned)warps);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)blocks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, p);
}

// Launch shape of the band kernel for a query plan: one pass slice per warp in shared memory (a
// slice too large for that runs from the profile in global memory, 32 warps on one block); more
// passes than one block's slices hold take a cluster of blocks, so that the passes run in as few
// rounds as possible.
struct BandShape {
    bool gprof;
    int warps, blocks;
    size_t smem;
};
static BandShape band_shape(const QueryPlan &qp, size_t smem_limit) {
    BandShape sh;
    const size_t budget = std::min<size_t>(BAND_SMEM_BUDGET, smem_limit - 16);
    sh.gprof = qp.pass_bytes > budget;
    int warps = sh.gprof ? 32 : (int)std::min<size_t>(32, budget / std::max<uint32_t>(qp.pass_bytes, 1));
    warps = std::max(1, std::min(warps, std::max(qp.n_passes, 1)));
    int blocks = 1;
    if (!sh.gprof && qp.n_passes > warps) {
        blocks = std::min(BAND_CLUSTER_MAX, (qp.n_passes + warps - 1) / warps);
        const int rounds = (qp.n_passes + blocks * warps - 1) / (blocks * warps);
        warps = (qp.n_passes + rounds * blocks - 1) / (rounds * blocks);  // as few as those rounds need
    }
    sh.warps = warps;
    sh.blocks = blocks;
    sh.smem = sh.gprof ? 16 : (size_t)warps * qp.pass_bytes + 16;
    return sh;
}

}  // namespace hy

extern "C" void hy_debug_band_shape(uint32_t pass_bytes, int32_t n_passes, uint64_t smem_limit, int32_t out[4]) {
    hy::QueryPlan qp;
    qp.pass_bytes = pass_bytes;
    qp.n_passes = n_passes;
    const hy::BandShape sh = hy::band_shape(qp, (size_t)smem_limit);
    out[0] = sh.gprof ? 1 : 0;
    out[1] = sh.warps;
    out[2] = sh.blocks;
    out[3] = (n_passes + sh.warps * sh.blocks - 1) / (sh.warps * sh.blocks);
}

namespace hy {

// End positions of the single item *item_ptr with the block-cooperative band kernel.
template <class A>
static hy_status enqueue_band(const hy_db *db, hy_scratch *sc, const Partition &part,
                              uint32_t item_end, const uint8_t *d_query, uint64_t qlen,
                              uint8_t *prof, void *bnd, const uint32_t *item_ptr) {
    const bool i16 = A::NH == 2;
    QueryPlan qp = plan_for<A>(qlen, WIN_G * WIN_R, db->al);
    HY_CK((launch_profile<A, WIN_G, WIN_R>(db, d_query, qlen, qp, i16 ? lim16(db) : LIM32, prof,
                                            sc->stream)));
    ScanParams p{};
    p.meta = part.d_meta;
    p.item_base = 0;
    p.n_items = item_end;
    p.item_ptr = item_ptr;
    p.res = part.d_res;
    p.profile = prof;
    p.pass_bytes = qp.pass_bytes;
    p.n_passes = qp.n_passes;
    p.vrow0 = qp.vrow0;
    p.qlen = (int32_t)qlen;
    p.go = db->go;
    p.ge = db->ge;
    p.sentinel = i16 ? (-32768 + db->ge) : (INT32_MIN / 4);
    p.boundary = bnd;
    p.scores = sc->d_scores;
    p.qend = sc->d_qend;
    p.tend = sc->d_tend;
    p.best_key = nullptr;
    p.err = sc->d_err;
    p.wait_polls = wait_polls();
    set_extents<A>(p, db, part, part.total_cols);
    BandShape sh = band_shape(qp, db->smem_limit);
    const bool gprof = sh.gprof;
    const int warps = sh.warps, blocks = sh.blocks;
    const size_t smem = sh.smem;
    cudaError_t e = cudaErrorInvalidValue;
#define HY_BAND_CASE(M)                                                                        \
    case M:                                                                                    \
        e = gprof ? launch_band_mode<A, M, true>(p, warps, 1, smem, sc->stream)                \
                  : launch_band_mode<A, M, false>(p, warps, blocks, smem, sc->stream);         \
        break;
    switch (db->mode) {
        HY_BAND_CASE(MODE_SW)
        HY_BAND_CASE(MODE_NW)
        HY_BAND_CASE(MODE_HW)
        HY_BAND_CASE(MODE_OV)
        HY_BAND_CASE(MODE_SHW)
    }
#undef HY_BAND_CASE
    HY_CK(e);
    sc->launches += qp.n_passes > 0 ? 2 : 1;
    return fail(HY_OK);
}

// Device buffers of the long-pair band paths, grow-only, per calling thread and device.
struct BandPairContext {
    int device = -1;
    size_t smem_limit = 0;
    cudaStream_t stream = nullptr;  // band_single_pair's own
    uint8_t *prof = nullptr, *in = nullptr;
    size_t c_prof = 0, c_in = 0;
    int32_t *bnd = nullptr;
    size_t c_bnd = 0;
    // One item (32 bytes), its index (a uint32 at +32), the error word (+36) and band_single_pair's
    // score, query end and target end (+40).
    ItemMeta *meta = nullptr;
    uint8_t *h_stage = nullptr, *h_in = nullptr;
    size_t ch_in = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~BandPairContext() {
        hy::dev_free(prof);
        hy::dev_free(in);
        hy::dev_free(bnd);
        hy::dev_free(meta);
        if (h_stage) cudaFreeHost(h_stage);
        if (h_in) cudaFreeHost(h_in);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};
static thread_local std::unique_ptr<BandPairContext> g_band_pair;

template <class T>
static cudaError_t grow_dev(T *&p, size_t &cap, size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    cudaError_t e = hy::dev_free(p);
    p = nullptr;
    cap = 0;
    if (e != cudaSuccess) return e;
    e = hy::dev_malloc(&p, bytes);
    if (e == cudaSuccess) cap = bytes;
    return e;
}

bool band_long_pair_fits(uint64_t m, uint64_t al) {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const QueryPlan qp = plan_for<Single32>(m, WIN_G * WIN_R, al);
    const BandShape sh = band_shape(qp, (size_t)optin);
    return !sh.gprof && qp.n_passes <= sh.warps * sh.blocks;
}

// The calling thread's context on the current device.
static hy_status band_pair_context(BandPairContext *&out) {
    int dev = 0;
    HY_CK(cudaGetDevice(&dev));
    if (g_band_pair && g_band_pair->device != dev) g_band_pair.reset();
    if (!g_band_pair) {
        std::unique_ptr<BandPairContext> c(new BandPairContext);
        c->device = dev;
        int optin = 0;
        HY_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        c->smem_limit = (size_t)optin;
        HY_CK(hy::dev_malloc(&c->meta, 64));
        HY_CK(cudaMallocHost((void **)&c->h_stage, 64));
        HY_CK(cudaEventCreate(&c->ev[0]));
        HY_CK(cudaEventCreate(&c->ev[1]));
        HY_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        g_band_pair = std::move(c);
    }
    out = g_band_pair.get();
    return fail(HY_OK);
}

// Enqueues one long pair's profile and band kernel on `st`: the query, target and matrix already on
// the device, the item staged in c.h_stage (its first 40 bytes go with it). Records the band's time
// between c.ev[0] and c.ev[1].
static hy_status band_pair_enqueue(BandPairContext &c, const uint8_t *d_q, uint64_t m, const uint8_t *d_t, uint64_t tl,
                                   const int32_t *d_matrix, uint64_t al, int32_t go, int32_t ge, int mode,
                                   cudaStream_t st, uint32_t slot, int32_t *d_scores, int32_t *d_qend,
                                   int32_t *d_tend) {
    const QueryPlan qp = plan_for<Single32>(m, WIN_G * WIN_R, al);
    HY_CK(grow_dev(c.prof, c.c_prof, std::max<size_t>(16, (size_t)qp.pass_bytes * qp.n_passes)));
    HY_CK(grow_dev(c.bnd, c.c_bnd, sizeof(int32_t) * std::max<uint64_t>(16, 2 * tl)));
    // The item (the target as one int32 column run, the pair's slot as its index), its index and
    // a cleared error word.
    ItemMeta im{};
    im.col_off = 0;
    im.w = (uint32_t)tl;
    im.n[0] = (uint32_t)tl;
    im.n[1] = 0;
    im.idx[0] = slot;
    im.idx[1] = NO_INDEX;
    const uint32_t zero_item = 0;
    const int zero_err = 0;
    memcpy(c.h_stage, &im, sizeof(im));
    memcpy(c.h_stage + 32, &zero_item, 4);
    memcpy(c.h_stage + 36, &zero_err, 4);
    HY_CK(cudaMemcpyAsync(c.meta, c.h_stage, 40, cudaMemcpyHostToDevice, st));
    const uint8_t *base = reinterpret_cast<const uint8_t *>(c.meta);
    const bool top_free = mode == MODE_SW || mode == MODE_HW || mode == MODE_OV;
    const int64_t words = Single32::letters((int64_t)al) * WIN_G * WIN_R * (int64_t)qp.n_passes;
    if (words > 0) {
        build_profile_kernel<Single32, WIN_G, WIN_R><<<(int)std::min<int64_t>((words + 255) / 256, 148 * 16), 256, 0, st>>>(
            d_q, (int32_t)m, d_matrix, (int32_t)al, go, LIM32, top_free ? 1 : 0, qp.vrow0, qp.n_passes,
            reinterpret_cast<Single32::PE *>(c.prof));
        HY_CK(cudaGetLastError());
    }
    ScanParams p{};
    p.meta = c.meta;
    p.item_base = 0;
    p.n_items = 1;
    p.item_ptr = reinterpret_cast<const uint32_t *>(base + 32);
    p.res = d_t;
    p.profile = c.prof;
    p.pass_bytes = qp.pass_bytes;
    p.n_passes = qp.n_passes;
    p.vrow0 = qp.vrow0;
    p.qlen = (int32_t)m;
    p.go = go;
    p.ge = ge;
    p.sentinel = INT32_MIN / 4;
    p.boundary = c.bnd;
    p.bnd_col0 = 0;
    p.scores = d_scores;
    p.qend = d_qend;
    p.tend = d_tend;
    p.best_key = nullptr;
    p.err = reinterpret_cast<int *>(const_cast<uint8_t *>(base) + 36);
    p.wait_polls = wait_polls();
    p.res_cols = tl;
    p.bnd_cols = tl;
    p.n_seqs = slot + 1;
    p.letters = (uint32_t)Single32::letters((int64_t)al);
    const BandShape sh = band_shape(qp, c.smem_limit);
    cudaError_t e = cudaErrorInvalidValue;
    HY_CK(cudaEventRecord(c.ev[0], st));
#define HY_PAIR_BAND_CASE(M)                                                                      \
    case M:                                                                                       \
        e = sh.gprof ? launch_band_mode<Single32, M, true>(p, sh.warps, 1, sh.smem, st)           \
                     : launch_band_mode<Single32, M, false>(p, sh.warps, sh.blocks, sh.smem, st); \
        break;
    switch (mode) {
        HY_PAIR_BAND_CASE(MODE_SW)
        HY_PAIR_BAND_CASE(MODE_NW)
        HY_PAIR_BAND_CASE(MODE_HW)
        HY_PAIR_BAND_CASE(MODE_OV)
        HY_PAIR_BAND_CASE(MODE_SHW)
    }
#undef HY_PAIR_BAND_CASE
    HY_CK(e);
    HY_CK(cudaEventRecord(c.ev[1], st));
    return fail(HY_OK);
}

hy_status band_long_pair(const uint8_t *d_q, uint64_t m, const uint8_t *t, uint64_t tl, const int32_t *d_matrix,
                         uint64_t al, int32_t go, int32_t ge, int mode, cudaStream_t st, uint32_t slot,
                         int32_t *d_scores, int32_t *d_qend, int32_t *d_tend, double *kernel_ms) {
    BandPairContext *cp = nullptr;
    hy_status s0 = band_pair_context(cp);
    if (s0 != HY_OK) return s0;
    BandPairContext &c = *cp;
    HY_CK(grow_dev(c.in, c.c_in, std::max<uint64_t>(16, tl)));
    if (tl) HY_CK(cudaMemcpyAsync(c.in, t, tl, cudaMemcpyHostToDevice, st));
    s0 = band_pair_enqueue(c, d_q, m, c.in, tl, d_matrix, al, go, ge, mode, st, slot, d_scores, d_qend, d_tend);
    if (s0 != HY_OK) return s0;
    const uint8_t *base = reinterpret_cast<const uint8_t *>(c.meta);
    HY_CK(cudaMemcpyAsync(c.h_stage + 36, base + 36, 4, cudaMemcpyDeviceToHost, st));
    HY_CK(cudaStreamSynchronize(st));
    int err = 0;
    memcpy(&err, c.h_stage + 36, 4);
    if (err) return fail(device_error(err));
    float ms = 0.f;
    HY_CK(cudaEventElapsedTime(&ms, c.ev[0], c.ev[1]));
    if (kernel_ms) *kernel_ms += ms;
    return fail(HY_OK);
}

hy_status band_single_pair(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t tl, const int32_t *matrix,
                           uint64_t al, int32_t go, int32_t ge, int mode, int32_t out[3], double *kernel_ms) {
    BandPairContext *cp = nullptr;
    hy_status s0 = band_pair_context(cp);
    if (s0 != HY_OK) return s0;
    BandPairContext &c = *cp;
    // Query, target and matrix staged together for one copy (the matrix 4-byte aligned).
    const uint64_t mat_off = (m + tl + 3) / 4 * 4, bytes = mat_off + sizeof(int32_t) * al * al;
    if (bytes > c.ch_in) {
        if (c.h_in) cudaFreeHost(c.h_in);
        c.h_in = nullptr;
        c.ch_in = 0;
        HY_CK(cudaMallocHost((void **)&c.h_in, bytes));
        c.ch_in = bytes;
    }
    memcpy(c.h_in, q, m);
    memcpy(c.h_in + m, t, tl);
    memcpy(c.h_in + mat_off, matrix, sizeof(int32_t) * al * al);
    HY_CK(grow_dev(c.in, c.c_in, bytes));
    HY_CK(cudaMemcpyAsync(c.in, c.h_in, bytes, cudaMemcpyHostToDevice, c.stream));
    int32_t *d_res = reinterpret_cast<int32_t *>(reinterpret_cast<uint8_t *>(c.meta) + 40);
    s0 = band_pair_enqueue(c, c.in, m, c.in + m, tl, reinterpret_cast<const int32_t *>(c.in + mat_off), al, go, ge,
                           mode, c.stream, 0, d_res, d_res + 1, d_res + 2);
    if (s0 != HY_OK) return s0;
    HY_CK(cudaMemcpyAsync(c.h_stage + 36, reinterpret_cast<const uint8_t *>(c.meta) + 36, 16, cudaMemcpyDeviceToHost,
                          c.stream));
    HY_CK(cudaStreamSynchronize(c.stream));
    int err = 0;
    memcpy(&err, c.h_stage + 36, 4);
    if (err) return fail(device_error(err));
    memcpy(out, c.h_stage + 40, 12);
    float ms = 0.f;
    HY_CK(cudaEventElapsedTime(&ms, c.ev[0], c.ev[1]));
    if (kernel_ms) *kernel_ms += ms;
    return fail(HY_OK);
}

// Compose the BestHit of a single-best scan from the reduced key (and the winner's ends).
__global__ void finalize_kernel(const unsigned long long *key, const int32_t *qend,
                                const int32_t *tend, int with_ends, hy_hit *out) {
    const unsigned long long k = *key;
    const uint32_t idx = ~(uint32_t)(k & 0xffffffffu);
    hy_hit h;
    h.score = (int32_t)((uint32_t)(k >> 32) ^ 0x80000000u);
    h.reserved = 0;
    h.db_index = idx;
    // A key of 0 (no hit recorded: the call reports a timeout) names no sequence to read.
    const bool ends = with_ends && k != 0;
    h.query_end = ends ? (int64_t)qend[idx] : -1;
    h.target_end = ends ? (int64_t)tend[idx] : -1;
    *out = h;
}

static hy_status enqueue_scan(const hy_db *db, hy_scratch *sc, const uint8_t *d_query,
                              uint64_t qlen, hy_hit *d_out) {
    HY_CK(cudaMemsetAsync(sc->d_key, 0, sizeof(unsigned long long), sc->stream));
    hy_status st = enqueue_scores(db, sc, d_query, qlen, false, sc->d_key, sc->d_scores);
    if (st != HY_OK) return st;
    const bool ends = db->search_type != HY_SEARCH_SCORE;
    if (ends) {
        // End positions of the winner only (src/database.rs:186-197): rerun its item with
        // position tracking on a whole block (the band kernel).
        const QuerySplit split = split_for_query(db, qlen);
        winner_loc_kernel<<<1, 1, 0, sc->stream>>>(sc->d_key, db->d_rank, split.k0, sc->d_win);
        HY_CK(cudaGetLastError());
        ++sc->launches;
        if (split.k0 < db->p16.n_items) {
            st = db->layout == HY_LAYOUT_PRECOMPUTED
                     ? enqueue_band<PairTab16>(db, sc, db->p16, db->p16.n_items, d_query, qlen,
                                               sc->d_profw16, sc->d_bnd16, sc->d_win)
                     : enqueue_band<Pair16>(db, sc, db->p16, db->p16.n_items, d_query, qlen,
                                            sc->d_profw16, sc->d_bnd16, sc->d_win);
            if (st != HY_OK) return st;
        }
        if (split.n_i32 > 0) {
            st = enqueue_band<Single32>(db, sc, db->p32, split.n_i32, d_query, qlen, sc->d_profw32,
                                        sc->d_bnd32, sc->d_win + 1);
            if (st != HY_OK) return st;
        }
    }
    finalize_kernel<<<1, 1, 0, sc->stream>>>(sc->d_key, sc->d_qend, sc->d_tend, ends ? 1 : 0, d_out);
    HY_CK(cudaGetLastError());
    ++sc->launches;
    return fail(HY_OK);
}

static hy_status check_query(const hy_db *db, const uint8_t *query, uint64_t qlen) {
    if (qlen > db->mql) return fail(HY_ERR_QUERY_TOO_LONG, (int64_t)qlen, (int64_t)db->mql);
    if (qlen && !query) return fail(HY_ERR_INVALID_ARGUMENT);
    for (uint64_t i = 0; i < qlen; ++i)
        if (query[i] >= db->al) return fail(HY_ERR_SYMBOL_OUT_OF_RANGE, query[i], (int64_t)db->al);
    return fail(HY_OK);
}

// ---- small scans through CUDA graphs ------------------------------------------------------------
//
// A scan of a small database is launch-bound: its kernels run for tens of microseconds, and each
// of the call's ten or so stream operations costs a few microseconds of host and device time. Such
// calls capture their device work (query upload, kernels, copies back) once per query length into
// a CUDA graph and replay it.

// Calls whose query meets at most this many database residues x query rows use graphs.
constexpr double GRAPH_MAX_CELLS = 2e9;
constexpr size_t GRAPH_CACHE = 32;  // graphs a scratch keeps (least recently used evicted)
enum { GRAPH_SCAN = 0, GRAPH_SCORES = 1, GRAPH_ALL = 2 };

static uint64_t db_residues(const hy_db *db) {
    return db->p16.res_prefix.empty() ? 0 : db->p16.res_prefix.back();
}

// Enqueues a call's device work on sc->stream through `issue`: directly, or by replaying the
// scratch's graph for (kind, qlen), capturing it on first use.
template <class F>
static hy_status run_captured(const hy_db *db, hy_scratch *sc, int kind, uint64_t qlen, F issue) {
    if (sc->profile || (double)qlen * (double)db_residues(db) > GRAPH_MAX_CELLS) return issue();
    // Graphs captured under another wait limit are captured again.
    const uint64_t epoch = wait_polls_epoch();
    for (size_t i = 0; i < sc->graphs.size();) {
        if (sc->graphs[i].epoch == epoch) {
            ++i;
            continue;
        }
        if (sc->graphs[i].exec) cudaGraphExecDestroy(sc->graphs[i].exec);
        sc->graphs.erase(sc->graphs.begin() + i);
    }
    for (auto &gr : sc->graphs) {
        if (gr.kind != kind || gr.qlen != qlen) continue;
        gr.last_use = ++sc->graph_clock;
        if (!gr.exec) return issue();
        HY_CK(cudaGraphLaunch(gr.exec, sc->stream));
        sc->launches += gr.launches;
        return fail(HY_OK);
    }
    if (sc->graphs.size() >= GRAPH_CACHE) {
        auto old = std::min_element(sc->graphs.begin(), sc->graphs.end(),
                                    [](const hy_scratch::Graph &a, const hy_scratch::Graph &b) {
                                        return a.last_use < b.last_use;
                                    });
        if (old->exec) cudaGraphExecDestroy(old->exec);
        sc->graphs.erase(old);
    }
    const uint64_t launches0 = sc->launches;
    HY_CK(cudaStreamBeginCapture(sc->stream, cudaStreamCaptureModeThreadLocal));
    hy_status st = issue();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(sc->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (st == HY_OK && e == cudaSuccess && graph) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (st != HY_OK) return st;
    sc->graphs.push_back({kind, qlen, e == cudaSuccess ? exec : nullptr, sc->launches - launches0,
                          ++sc->graph_clock, epoch});
    if (!sc->graphs.back().exec) {
        // Not capturable here: this call and later ones of its kind and length launch directly.
        sc->launches = launches0;
        return issue();
    }
    HY_CK(cudaGraphLaunch(exec, sc->stream));
    return fail(HY_OK);
}

// The device error flag back with the call's results (part of a call's captured work).
static hy_status issue_err_back(hy_scratch *sc) {
    HY_CK(cudaMemcpyAsync(sc->h_err, sc->d_err, sizeof(int), cudaMemcpyDeviceToHost, sc->stream));
    return fail(HY_OK);
}

// Waits for the call's work; a set device error flag (a bounded wait that gave up) is cleared and
// reported.
static hy_status wait_and_check(hy_scratch *sc) {
    HY_CK(cudaStreamSynchronize(sc->stream));
    if (const int w = *sc->h_err) {
        *sc->h_err = 0;
        HY_CK(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream));
        HY_CK(cudaStreamSynchronize(sc->stream));
        return fail(device_error(w));
    }
    return fail(HY_OK);
}

// The query into the scratch's pinned buffer (host) and its copy to the device (enqueued).
static void stage_query(hy_scratch *sc, const uint8_t *query, uint64_t qlen) {
    if (qlen) memcpy(sc->h_query, query, qlen);
}
static hy_status issue_query(hy_scratch *sc, uint64_t qlen) {
    if (qlen) HY_CK(cudaMemcpyAsync(sc->d_query, sc->h_query, qlen, cudaMemcpyHostToDevice, sc->stream));
    return fail(HY_OK);
}

static hy_status sync_and_check(hy_scratch *sc) {
    HY_CK(cudaMemcpyAsync(sc->h_err, sc->d_err, sizeof(int), cudaMemcpyDeviceToHost, sc->stream));
    HY_CK(cudaStreamSynchronize(sc->stream));
    if (const int w = *sc->h_err) {
        *sc->h_err = 0;
        HY_CK(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream));
        HY_CK(cudaStreamSynchronize(sc->stream));
        return fail(device_error(w));
    }
    return fail(HY_OK);
}

static hy_status ensure_host_out(hy_scratch *sc) {
    if (!sc->h_out) {
        size_t bytes = 3 * sizeof(int32_t) * std::max<uint64_t>(sc->db->n_seqs, 1);
        HY_CK(cudaMallocHost(&sc->h_out, bytes));
    }
    return fail(HY_OK);
}

// Makes `dev` current for the scope of a call and restores the caller's device afterwards. Any
// error of these bookkeeping calls is cleared so it cannot surface in a later launch check.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
        cudaGetLastError();
    }
    ~DeviceGuard() {
        int cur;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
        cudaGetLastError();
    }
};

// Build one partition: `order` lists its global indices sorted by length, longest first.
// LayoutChoice::Auto (src/inter.rs:356-367 picks Precomputed when its table stays cache
// resident). On the device: Precomputed when the pair table of a 256-row pass slice, double
// buffered, stays within 100 KiB of shared memory (alphabets of at most 6 symbols, e.g. DNA), so
// two blocks of the 32-row kernel still fit on an SM; measured 7.7% faster than Gathered on DNA.
// Larger alphabets resolve to Gathered, whose per-letter tables grow linearly.
static int auto_layout(uint64_t al) {
    return 2 * profile_slice_row_bytes<PairTab16>((int64_t)al) * BULK_MAX_RPP <= 100 * 1024
               ? HY_LAYOUT_PRECOMPUTED
               : HY_LAYOUT_GATHERED;
}

static hy_status build_partition(hy_db *db, Partition &part, const std::vector<uint32_t> &order,
                                 const uint8_t *residues, const uint64_t *offsets, bool pairs) {
    part.n_seqs = order.size();
    if (order.empty()) return fail(HY_OK);
    const uint64_t per = pairs ? 2 : 1;
    const uint64_t align = pairs ? 8 : 16;
    part.n_items = (uint32_t)((order.size() + per - 1) / per);
    std::vector<ItemMeta> meta(part.n_items);
    uint64_t cols = 0;
    for (uint32_t it = 0; it < part.n_items; ++it) {
        ItemMeta &m = meta[it];
        m.col_off = cols;
        m.pad_ = 0;
        for (int h = 0; h < 2; ++h) {
            uint64_t k = (uint64_t)it * per + h;
            if (h < (int)per && k < order.size()) {
                m.idx[h] = order[k];
                m.n[h] = (uint32_t)(offsets[order[k] + 1] - offsets[order[k]]);
            } else {
                m.idx[h] = NO_INDEX;
                m.n[h] = 0;
            }
        }
        m.w = std::max(m.n[0], m.n[1]);
        cols += (m.w + align - 1) / align * align;
    }
    part.total_cols = cols;
    part.res_prefix.assign(part.n_items + 1, 0);
    for (uint32_t it = 0; it < part.n_items; ++it)
        part.res_prefix[it + 1] = part.res_prefix[it] + meta[it].n[0] + meta[it].n[1];
    HY_CK(hy::dev_malloc(&part.d_meta, sizeof(ItemMeta) * part.n_items));
    HY_CK(cudaMemcpy(part.d_meta, meta.data(), sizeof(ItemMeta) * part.n_items, cudaMemcpyHostToDevice));
    db->device_bytes += sizeof(ItemMeta) * part.n_items;
    if (pairs) {
        // Pair column codes: lo | hi << 8 (Gathered) or lo * (al + 1) + hi (Precomputed).
        const bool tab = db->layout == HY_LAYOUT_PRECOMPUTED;
        const uint32_t al = (uint32_t)db->al;
        auto code = [&](uint32_t lo, uint32_t hi) {
            return (uint16_t)(tab ? PairTab16::code(lo, hi, al) : Pair16::code(lo, hi, al));
        };
        std::vector<uint16_t> res(std::max<uint64_t>(cols, 1), code(al, al));
        for (uint32_t it = 0; it < part.n_items; ++it) {
            const ItemMeta &m = meta[it];
            const uint8_t *t0 = residues + offsets[m.idx[0]];
            const uint8_t *t1 = m.idx[1] == NO_INDEX ? nullptr : residues + offsets[m.idx[1]];
            for (uint32_t j = 0; j < m.w; ++j) {
                uint16_t lo = j < m.n[0] ? t0[j] : (uint16_t)db->al;
                uint16_t hi = (t1 && j < m.n[1]) ? t1[j] : (uint16_t)db->al;
                res[m.col_off + j] = code(lo, hi);
            }
        }
        HY_CK(hy::dev_malloc(&part.d_res, res.size() * sizeof(uint16_t)));
        HY_CK(cudaMemcpy(part.d_res, res.data(), res.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
        db->device_bytes += res.size() * sizeof(uint16_t);
    } else {
        std::vector<uint8_t> res(std::max<uint64_t>(cols, 1), 0);
        for (uint32_t it = 0; it < part.n_items; ++it) {
            const ItemMeta &m = meta[it];
            memcpy(&res[m.col_off], residues + offsets[m.idx[0]], m.n[0]);
        }
        HY_CK(hy::dev_malloc(&part.d_res, res.size()));
        HY_CK(cudaMemcpy(part.d_res, res.data(), res.size(), cudaMemcpyHostToDevice));
        db->device_bytes += res.size();
    }
    return fail(HY_OK);
}

static void free_db(hy_db *db) {
    if (!db) return;
    hy::dev_free(db->d_matrix);
    hy::dev_free(db->p16.d_meta);
    hy::dev_free(db->p16.d_res);
    hy::dev_free(db->p32.d_meta);
    hy::dev_free(db->p32.d_res);
    hy::dev_free(db->d_rank);
    hy::dev_free(db->d_tb_res);
    delete db;
}

static uint64_t npass(uint64_t mql, int rpp) { return (mql + rpp - 1) / rpp; }

}  // namespace hy

extern "C" {

hy_status hy_db_create(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                       const int32_t *matrix, uint64_t alphabet_len, int32_t gap_open,
                       int32_t gap_ext, hy_mode mode, hy_search_type search_type,
                       uint64_t traceback_max_bytes, uint64_t max_query_len, int backend_choice,
                       int layout, hy_db **out) {
    if (!out) return fail(HY_ERR_INVALID_ARGUMENT);
    *out = nullptr;
    if ((int)mode < 0 || (int)mode > 4) return fail(HY_ERR_INVALID_ARGUMENT);
    if ((int)search_type < HY_SEARCH_SCORE || (int)search_type > HY_SEARCH_ALIGNMENT)
        return fail(HY_ERR_INVALID_ARGUMENT);
    hy_status st = validate_scoring(alphabet_len, matrix, alphabet_len * alphabet_len, gap_open, gap_ext);
    if (st != HY_OK) return st;
    if (n_seqs == 0) return fail(HY_ERR_EMPTY_DATABASE);
    if (!offsets || (!residues && offsets[n_seqs] > 0)) return fail(HY_ERR_INVALID_ARGUMENT);
    for (uint64_t k = 0; k < n_seqs; ++k) {
        if (offsets[k + 1] < offsets[k]) return fail(HY_ERR_INVALID_ARGUMENT);
        for (uint64_t i = offsets[k]; i < offsets[k + 1]; ++i)
            if (residues[i] >= alphabet_len)
                return fail(HY_ERR_SYMBOL_OUT_OF_RANGE, residues[i], (int64_t)alphabet_len);
    }
    uint64_t max_t = 0;
    for (uint64_t k = 0; k < n_seqs; ++k) max_t = std::max(max_t, offsets[k + 1] - offsets[k]);
    const int32_t min_e = *std::min_element(matrix, matrix + alphabet_len * alphabet_len);
    const int32_t max_e = *std::max_element(matrix, matrix + alphabet_len * alphabet_len);
    const int64_t bound = magnitude_bound(mode, min_e, max_e, gap_open, gap_ext, max_query_len, max_t);
    const int width = narrowest_width(bound);
    if (width < 0) return fail(HY_ERR_SCORE_RANGE_TOO_WIDE, bound);
    // The Alignment budget covers every problem the database can pose (src/database.rs:776-790).
    if (search_type == HY_SEARCH_ALIGNMENT) {
        const uint64_t needed = hy_traceback_min_bytes_for_database(max_query_len, max_t);
        if (needed > traceback_max_bytes)
            return fail(HY_ERR_TRACEBACK_BUDGET_EXCEEDED, (int64_t)needed, (int64_t)traceback_max_bytes);
    }
    hy_backend backend;
    st = hy_backend_resolve(backend_choice, &backend);
    if (st != HY_OK) return st;
    if (layout != HY_LAYOUT_AUTO && layout != HY_LAYOUT_GATHERED && layout != HY_LAYOUT_PRECOMPUTED)
        return fail(HY_ERR_INVALID_ARGUMENT);
    // Device limits: 32-bit db indices (one value reserved), byte residues plus a padding symbol.
    if (n_seqs >= (uint64_t)NO_INDEX || alphabet_len > 255 || max_t >= (1ull << 31) ||
        max_query_len >= (1ull << 30))
        return fail(HY_ERR_UNSUPPORTED);

    hy_db *db = new hy_db;
    cudaGetDevice(&db->device);
    int smem_optin = 0;
    if (cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, db->device) == cudaSuccess &&
        smem_optin > 0)
        db->smem_limit = (size_t)smem_optin;
    cudaGetLastError();
    db->n_seqs = n_seqs;
    db->mql = max_query_len;
    db->max_t = max_t;
    db->al = alphabet_len;
    db->go = gap_open;
    db->ge = gap_ext;
    db->min_e = min_e;
    db->max_e = max_e;
    db->mode = mode;
    db->search_type = search_type;
    db->tb_max_bytes = search_type == HY_SEARCH_ALIGNMENT ? traceback_max_bytes : 0;
    db->layout = layout == HY_LAYOUT_AUTO ? auto_layout(alphabet_len) : layout;
    db->width = (hy_score_width)width;
    db->backend = backend;

    // One global length order (longest first, ties by index). Every sequence is packed in int16x2
    // pairs over it; the prefix the whole-database proof cannot place in int16 (plus one, so a
    // pair straddling any query's split is covered) is also packed as int32 singles.
    std::vector<uint32_t> order(n_seqs);
    for (uint64_t k = 0; k < n_seqs; ++k) order[k] = (uint32_t)k;
    auto by_len = [&](uint32_t a, uint32_t b) {
        uint64_t la = offsets[a + 1] - offsets[a], lb = offsets[b + 1] - offsets[b];
        return la != lb ? la > lb : a < b;
    };
    std::sort(order.begin(), order.end(), by_len);
    uint64_t k32 = 0;
    while (k32 < n_seqs) {
        const uint64_t len = offsets[order[k32] + 1] - offsets[order[k32]];
        if (device_fits_i16(magnitude_bound(mode, min_e, max_e, gap_open, gap_ext, max_query_len, len), gap_open))
            break;
        ++k32;
    }
    if (k32 > 0) k32 = std::min<uint64_t>(n_seqs, k32 + 1);
    std::vector<uint32_t> o32(order.begin(), order.begin() + k32);
    db->pair_w.resize((n_seqs + 1) / 2);
    for (uint64_t p = 0; p < db->pair_w.size(); ++p)
        db->pair_w[p] = (uint32_t)(offsets[order[2 * p] + 1] - offsets[order[2 * p]]);

    hy_status bst = HY_OK;
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && bst == HY_OK) {
            cudaGetLastError();
            bst = fail(e == cudaErrorMemoryAllocation ? HY_ERR_OUT_OF_MEMORY : HY_ERR_CUDA, e);
        }
    };
    ck(hy::dev_malloc(&db->d_matrix, sizeof(int32_t) * alphabet_len * alphabet_len));
    if (bst == HY_OK)
        ck(cudaMemcpy(db->d_matrix, matrix, sizeof(int32_t) * alphabet_len * alphabet_len,
                      cudaMemcpyHostToDevice));
    if (bst == HY_OK) bst = build_partition(db, db->p16, order, residues, offsets, true);
    if (bst == HY_OK) bst = build_partition(db, db->p32, o32, residues, offsets, false);
    if (bst == HY_OK) {
        std::vector<uint32_t> rank(n_seqs);
        for (uint64_t r = 0; r < n_seqs; ++r) rank[order[r]] = (uint32_t)r;
        ck(hy::dev_malloc(&db->d_rank, sizeof(uint32_t) * n_seqs));
        if (bst == HY_OK)
            ck(cudaMemcpy(db->d_rank, rank.data(), sizeof(uint32_t) * n_seqs, cudaMemcpyHostToDevice));
        db->device_bytes += sizeof(uint32_t) * n_seqs + sizeof(int32_t) * alphabet_len * alphabet_len;
    }
    // The Alignment search type traces targets back from a plain copy of the residues in db order.
    if (bst == HY_OK && search_type == HY_SEARCH_ALIGNMENT) {
        const uint64_t total = offsets[n_seqs] - offsets[0];
        db->tb_off.resize(n_seqs + 1);
        for (uint64_t k = 0; k <= n_seqs; ++k) db->tb_off[k] = offsets[k] - offsets[0];
        ck(hy::dev_malloc(&db->d_tb_res, std::max<uint64_t>(total, 16)));
        if (bst == HY_OK && total)
            ck(cudaMemcpy(db->d_tb_res, residues + offsets[0], total, cudaMemcpyHostToDevice));
        db->device_bytes += total;
    }
    if (bst != HY_OK) {
        int64_t d[3];
        hy_last_error_detail(d);
        free_db(db);
        return fail(bst, d[0], d[1], d[2]);
    }
    *out = db;
    return fail(HY_OK);
}

void hy_db_destroy(hy_db *db) {
    if (!db) return;
    DeviceGuard g(db->device);
    free_db(db);
}

uint64_t hy_db_sequence_count(const hy_db *db) { return db ? db->n_seqs : 0; }
hy_mode hy_db_mode(const hy_db *db) { return (hy_mode)db->mode; }
hy_search_type hy_db_search_type(const hy_db *db) { return (hy_search_type)db->search_type; }
uint64_t hy_db_traceback_max_bytes(const hy_db *db) { return db->tb_max_bytes; }
hy_score_width hy_db_score_width(const hy_db *db) { return db->width; }
hy_backend hy_db_backend(const hy_db *db) { return db->backend; }
int hy_db_layout(const hy_db *db) { return db->layout; }
uint64_t hy_db_max_query_len(const hy_db *db) { return db->mql; }
uint64_t hy_db_max_target_len(const hy_db *db) { return db->max_t; }
uint64_t hy_db_device_bytes(const hy_db *db) { return db->device_bytes; }
void hy_db_partition(const hy_db *db, uint64_t *n_i16, uint64_t *n_i32) {
    if (n_i16) *n_i16 = db->p16.n_seqs;
    if (n_i32) *n_i32 = db->p32.n_seqs;
}

// Profile bytes of one query row of an int16x2 pass slice in the database's layout.
static uint64_t pair_slice_row_bytes(const hy_db *db) {
    return db->layout == HY_LAYOUT_PRECOMPUTED ? profile_slice_row_bytes<PairTab16>(db->al)
                                               : profile_slice_row_bytes<Pair16>(db->al);
}

uint64_t hy_db_scratch_bytes(const hy_db *db) {
    const uint64_t mq = std::max<uint64_t>(db->mql, 1);
    uint64_t b = mq + 3 * 4 * db->n_seqs + 64 + sizeof(hy_hit);
    const uint64_t pr = pair_slice_row_bytes(db), sr = profile_slice_row_bytes<Single32>(db->al);
    b += npass(mq, BULK_MAX_RPP) * BULK_MAX_RPP * pr;
    b += npass(mq, MAIN_G32 * MAIN_R32) * MAIN_G32 * MAIN_R32 * sr;
    b += npass(mq, WIN_G * WIN_R) * WIN_G * WIN_R * (pr + sr);
    if (mq > (uint64_t)std::min({MAIN_G * 8, MAIN_G * MAIN_R16, MAIN_G32 * MAIN_R32, WIN_G * WIN_R}))
        b += 8 * (db->p16.total_cols + db->p32.total_cols);
    return b;
}

hy_status hy_scratch_create(const hy_db *db, hy_scratch **out) {
    if (!db || !out) return fail(HY_ERR_INVALID_ARGUMENT);
    DeviceGuard g(db->device);
    hy_scratch *sc = new hy_scratch;
    sc->db = db;
    sc->device = db->device;
    hy_status st = HY_OK;
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && st == HY_OK) {
            cudaGetLastError();
            st = fail(e == cudaErrorMemoryAllocation ? HY_ERR_OUT_OF_MEMORY : HY_ERR_CUDA, e);
        }
    };
    const uint64_t mq = std::max<uint64_t>(db->mql, 1);
    const uint64_t n = std::max<uint64_t>(db->n_seqs, 1);
    ck(cudaStreamCreateWithFlags(&sc->stream, cudaStreamNonBlocking));
    int prio_low = 0, prio_high = 0;
    ck(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    ck(cudaStreamCreateWithPriority(&sc->stream2, cudaStreamNonBlocking, prio_high));
    ck(cudaEventCreateWithFlags(&sc->ev_fork, cudaEventDisableTiming));
    ck(cudaEventCreateWithFlags(&sc->ev_join, cudaEventDisableTiming));
    ck(hy::dev_malloc(&sc->d_query, mq));
    auto prof_bytes = [&](int rpp, size_t slice_row_bytes) {
        return std::max<uint64_t>(1, npass(mq, rpp) * rpp * slice_row_bytes);
    };
    const uint64_t pr = pair_slice_row_bytes(db), sr = profile_slice_row_bytes<Single32>(db->al);
    ck(hy::dev_malloc(&sc->d_prof16, prof_bytes(BULK_MAX_RPP, pr)));
    ck(hy::dev_malloc(&sc->d_prof32, prof_bytes(MAIN_G32 * MAIN_R32, sr)));
    ck(hy::dev_malloc(&sc->d_profw16, prof_bytes(WIN_G * WIN_R, pr)));
    ck(hy::dev_malloc(&sc->d_profw32, prof_bytes(WIN_G * WIN_R, sr)));
    const bool multipass = mq > (uint64_t)std::min({MAIN_G * 8, MAIN_G * MAIN_R16, MAIN_G32 * MAIN_R32, WIN_G * WIN_R});
    ck(hy::dev_malloc(&sc->d_bnd16, multipass ? std::max<uint64_t>(8, 8 * db->p16.total_cols) : 8));
    ck(hy::dev_malloc(&sc->d_bnd32, multipass ? std::max<uint64_t>(8, 8 * db->p32.total_cols) : 8));
    ck(hy::dev_malloc(&sc->d_scores, 4 * n));
    ck(hy::dev_malloc(&sc->d_qend, 4 * n));
    ck(hy::dev_malloc(&sc->d_tend, 4 * n));
    ck(hy::dev_malloc(&sc->d_key, 64));
    ck(hy::dev_malloc(&sc->d_win, 64));
    ck(hy::dev_malloc(&sc->d_hit, sizeof(hy_hit)));
    ck(hy::dev_malloc(&sc->d_err, 64));
    ck(cudaMallocHost(&sc->h_query, mq));
    ck(cudaMallocHost(&sc->h_hit, sizeof(hy_hit)));
    ck(cudaMallocHost(&sc->h_err, sizeof(int)));
    if (st == HY_OK) {
        ck(cudaMemset(sc->d_err, 0, 64));
        *sc->h_err = 0;
        sc->bytes = hy_db_scratch_bytes(db);
    }
    if (st != HY_OK) {
        int64_t d[3];
        hy_last_error_detail(d);
        hy_scratch_destroy(sc);
        return fail(st, d[0], d[1], d[2]);
    }
    *out = sc;
    return fail(HY_OK);
}

void hy_scratch_destroy(hy_scratch *sc) {
    if (!sc) return;
    DeviceGuard g(sc->device);
    if (sc->stream) cudaStreamSynchronize(sc->stream);
    tb_context_destroy(sc->tb);
    hy::dev_free(sc->d_query);
    hy::dev_free(sc->d_prof16);
    hy::dev_free(sc->d_prof32);
    hy::dev_free(sc->d_profw16);
    hy::dev_free(sc->d_profw32);
    hy::dev_free(sc->d_bnd16);
    hy::dev_free(sc->d_bnd32);
    hy::dev_free(sc->d_scores);
    hy::dev_free(sc->d_qend);
    hy::dev_free(sc->d_tend);
    hy::dev_free(sc->d_key);
    hy::dev_free(sc->d_win);
    hy::dev_free(sc->d_hit);
    hy::dev_free(sc->d_err);
    cudaFreeHost(sc->h_query);
    cudaFreeHost(sc->h_hit);
    cudaFreeHost(sc->h_err);
    cudaFreeHost(sc->h_out);
    for (auto &gr : sc->graphs)
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
    for (auto &e : sc->events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (sc->stream2) cudaStreamSynchronize(sc->stream2);
    if (sc->ev_fork) cudaEventDestroy(sc->ev_fork);
    if (sc->ev_join) cudaEventDestroy(sc->ev_join);
    if (sc->stream2) cudaStreamDestroy(sc->stream2);
    if (sc->stream) cudaStreamDestroy(sc->stream);
    delete sc;
}

void *hy_scratch_stream(hy_scratch *sc) { return sc ? (void *)sc->stream : nullptr; }

hy_status hy_scratch_profile(hy_scratch *sc, int enable) {
    if (!sc) return fail(HY_ERR_INVALID_ARGUMENT);
    sc->profile = enable != 0;
    sc->n_events = 0;
    sc->launches = 0;
    sc->event_cells[0] = sc->event_cells[1] = sc->event_cells[2] = 0.0;
    return fail(HY_OK);
}

hy_status hy_scratch_profile_read(hy_scratch *sc, double kernel_ms[3], uint64_t launches[3],
                                  double cells[3], uint64_t *all_launches) {
    if (!sc || !kernel_ms || !launches) return fail(HY_ERR_INVALID_ARGUMENT);
    DeviceGuard g(sc->device);
    HY_CK(cudaStreamSynchronize(sc->stream));
    kernel_ms[0] = kernel_ms[1] = kernel_ms[2] = 0.0;
    launches[0] = launches[1] = launches[2] = 0;
    for (size_t i = 0; i < sc->n_events; ++i) {
        float ms = 0.f;
        HY_CK(cudaEventElapsedTime(&ms, sc->events[i].first, sc->events[i].second));
        kernel_ms[sc->event_part[i]] += ms;
        launches[sc->event_part[i]] += 1;
    }
    if (cells) {
        cells[0] = sc->event_cells[0];
        cells[1] = sc->event_cells[1];
        cells[2] = sc->event_cells[2];
    }
    if (all_launches) *all_launches = sc->launches + tb_context_launches(sc->tb);
    sc->n_events = 0;
    sc->launches = 0;
    sc->event_cells[0] = sc->event_cells[1] = sc->event_cells[2] = 0.0;
    return fail(HY_OK);
}

hy_status hy_host_alloc(uint64_t bytes, void **out) {
    if (!out) return fail(HY_ERR_INVALID_ARGUMENT);
    *out = nullptr;
    HY_CK(cudaMallocHost(out, std::max<uint64_t>(bytes, 1)));
    return fail(HY_OK);
}

hy_status hy_host_free(void *p) {
    if (p) HY_CK(cudaFreeHost(p));
    return fail(HY_OK);
}

hy_status hy_query_validate(const hy_db *db, const uint8_t *query, uint64_t qlen) {
    if (!db) return fail(HY_ERR_INVALID_ARGUMENT);
    return check_query(db, query, qlen);
}

hy_status hy_scratch_sync(hy_scratch *sc) {
    if (!sc) return fail(HY_ERR_INVALID_ARGUMENT);
    DeviceGuard g(sc->device);
    return sync_and_check(sc);
}

hy_status hy_scan(const hy_db *db, hy_scratch *sc, const uint8_t *query, uint64_t qlen, hy_hit *out) {
    if (!db || !sc || !out || sc->db != db) return fail(HY_ERR_INVALID_ARGUMENT);
    hy_status st = check_query(db, query, qlen);
    if (st != HY_OK) return st;
    DeviceGuard g(db->device);
    stage_query(sc, query, qlen);
    st = run_captured(db, sc, GRAPH_SCAN, qlen, [&]() -> hy_status {
        hy_status s2;
        if ((s2 = issue_query(sc, qlen)) != HY_OK) return s2;
        if ((s2 = enqueue_scan(db, sc, sc->d_query, qlen, sc->d_hit)) != HY_OK) return s2;
        HY_CK(cudaMemcpyAsync(sc->h_hit, sc->d_hit, sizeof(hy_hit), cudaMemcpyDeviceToHost, sc->stream));
        return issue_err_back(sc);
    });
    if (st != HY_OK) return st;
    if ((st = wait_and_check(sc)) != HY_OK) return st;
    *out = *sc->h_hit;
    return fail(HY_OK);
}

hy_status hy_scan_device(const hy_db *db, hy_scratch *sc, const uint8_t *d_query, uint64_t qlen,
                         hy_hit *d_out) {
    if (!db || !sc || !d_out || sc->db != db) return fail(HY_ERR_INVALID_ARGUMENT);
    if (qlen > db->mql) return fail(HY_ERR_QUERY_TOO_LONG, (int64_t)qlen, (int64_t)db->mql);
    DeviceGuard g(db->device);
    return enqueue_scan(db, sc, d_query, qlen, d_out);
}

hy_status hy_scan_scores_device(const hy_db *db, hy_scratch *sc, const uint8_t *d_query,
                                uint64_t qlen, int32_t *d_out) {
    if (!db || !sc || !d_out || sc->db != db) return fail(HY_ERR_INVALID_ARGUMENT);
    if (qlen > db->mql) return fail(HY_ERR_QUERY_TOO_LONG, (int64_t)qlen, (int64_t)db->mql);
    DeviceGuard g(db->device);
    return enqueue_scores(db, sc, d_query, qlen, false, nullptr, d_out);
}

hy_status hy_scan_scores(const hy_db *db, hy_scratch *sc, const uint8_t *query, uint64_t qlen,
                         int32_t *out) {
    if (!db || !sc || !out || sc->db != db) return fail(HY_ERR_INVALID_ARGUMENT);
    hy_status st = check_query(db, query, qlen);
    if (st != HY_OK) return st;
    DeviceGuard g(db->device);
    if ((st = ensure_host_out(sc)) != HY_OK) return st;
    stage_query(sc, query, qlen);
    st = run_captured(db, sc, GRAPH_SCORES, qlen, [&]() -> hy_status {
        hy_status s2;
        if ((s2 = issue_query(sc, qlen)) != HY_OK) return s2;
        if ((s2 = enqueue_scores(db, sc, sc->d_query, qlen, false, nullptr, sc->d_scores)) != HY_OK) return s2;
        HY_CK(cudaMemcpyAsync(sc->h_out, sc->d_scores, 4 * db->n_seqs, cudaMemcpyDeviceToHost, sc->stream));
        return issue_err_back(sc);
    });
    if (st != HY_OK) return st;
    if ((st = wait_and_check(sc)) != HY_OK) return st;
    memcpy(out, sc->h_out, 4 * db->n_seqs);
    return fail(HY_OK);
}

hy_status hy_scan_all(const hy_db *db, hy_scratch *sc, const uint8_t *query, uint64_t qlen,
                      hy_hit *out) {
    if (!db || !sc || !out || sc->db != db) return fail(HY_ERR_INVALID_ARGUMENT);
    hy_status st = check_query(db, query, qlen);
    if (st != HY_OK) return st;
    DeviceGuard g(db->device);
    const bool ends = db->search_type != HY_SEARCH_SCORE;
    const uint64_t n = db->n_seqs;
    if ((st = ensure_host_out(sc)) != HY_OK) return st;
    stage_query(sc, query, qlen);
    st = run_captured(db, sc, GRAPH_ALL, qlen, [&]() -> hy_status {
        hy_status s2;
        if ((s2 = issue_query(sc, qlen)) != HY_OK) return s2;
        if ((s2 = enqueue_scores(db, sc, sc->d_query, qlen, ends, nullptr, sc->d_scores)) != HY_OK) return s2;
        HY_CK(cudaMemcpyAsync(sc->h_out, sc->d_scores, 4 * n, cudaMemcpyDeviceToHost, sc->stream));
        if (ends) {
            HY_CK(cudaMemcpyAsync(sc->h_out + n, sc->d_qend, 4 * n, cudaMemcpyDeviceToHost, sc->stream));
            HY_CK(cudaMemcpyAsync(sc->h_out + 2 * n, sc->d_tend, 4 * n, cudaMemcpyDeviceToHost, sc->stream));
        }
        return issue_err_back(sc);
    });
    if (st != HY_OK) return st;
    if ((st = wait_and_check(sc)) != HY_OK) return st;
    for (uint64_t k = 0; k < n; ++k) {
        out[k].score = sc->h_out[k];
        out[k].reserved = 0;
        out[k].db_index = k;
        out[k].query_end = ends ? (int64_t)sc->h_out[n + k] : -1;
        out[k].target_end = ends ? (int64_t)sc->h_out[2 * n + k] : -1;
    }
    return fail(HY_OK);
}

hy_status hy_scan_aligned(const hy_db *db, hy_scratch *sc, const uint8_t *query, uint64_t qlen,
                          uint64_t *db_index, hy_alignment *out, const uint8_t **ops) {
    if (!db || !sc || !out || !ops || sc->db != db || db->search_type != HY_SEARCH_ALIGNMENT)
        return fail(HY_ERR_INVALID_ARGUMENT);
    hy_hit hit;
    hy_status st = hy_scan(db, sc, query, qlen, &hit);
    if (st != HY_OK) return st;
    DeviceGuard g(db->device);
    const uint32_t k = (uint32_t)hit.db_index;
    st = tb_scan_targets(db, &sc->tb, sc->stream, query, qlen, &k, 1, out, sc->tb_ops);
    if (st != HY_OK) return st;
    if (db_index) *db_index = hit.db_index;
    *ops = sc->tb_ops.data();
    return fail(HY_OK);
}

hy_status hy_scan_all_aligned(const hy_db *db, hy_scratch *sc, const uint8_t *query, uint64_t qlen,
                              hy_alignment *out, const uint8_t **ops) {
    if (!db || !sc || !out || !ops || sc->db != db || db->search_type != HY_SEARCH_ALIGNMENT)
        return fail(HY_ERR_INVALID_ARGUMENT);
    hy_status st = check_query(db, query, qlen);
    if (st != HY_OK) return st;
    DeviceGuard g(db->device);
    std::vector<uint32_t> idx(db->n_seqs);
    std::iota(idx.begin(), idx.end(), 0u);
    st = tb_scan_targets(db, &sc->tb, sc->stream, query, qlen, idx.data(), (uint32_t)db->n_seqs, out,
                         sc->tb_ops);
    if (st != HY_OK) return st;
    *ops = sc->tb_ops.data();
    return fail(HY_OK);
}

}  // extern "C"
