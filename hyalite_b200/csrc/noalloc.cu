// noalloc.cu -- hy_scan_scores_noalloc: the per-target score scan for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc once they are running: a process whose device memory is
// already fully reserved by another allocator (a framework's caching allocator or a fixed arena
// that owns the whole GPU), or a latency-critical loop in which cudaMalloc's implicit device
// synchronisation is not acceptable. This entry point gives them the same scores as
// hy_scan_scores without any allocation: the query and the output are the caller's device
// buffers, and the kernels' scratch (the staged query profile, the boundary rows between passes
// and the wait-timeout flag) lives in one file-scope __device__ array of fixed size.
//
// That array costs NOALLOC_SCRATCH_BYTES of device memory on every GPU that loads this library,
// held until the process exits. All calls share it and it keeps the previous call's contents;
// the timeout flag is cleared at the start of each call and every other byte a call reads it has
// first written. Calls whose kernels overlap on the GPU (two host threads, two streams) race on the
// array and corrupt each other's results: callers must serialise them.
//
// The first call on each device does a one-time set-up: it looks up the array's device address and
// loads every kernel the entry point launches (a lazily loaded kernel would otherwise allocate at
// its first launch). That first call may therefore allocate, and it should be made before the
// caller reserves all device memory and before any stream capture; later calls allocate nothing.
#include <mutex>

#include "db_internal.h"

using namespace hy;

namespace {

// 16 MiB: the profile slices of a query plus the boundary rows of a multi-pass scan must fit.
constexpr size_t NOALLOC_SCRATCH_BYTES = 16u << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// In host code `g_noalloc_scratch` only names a host-side stand-in; kernels must be given the
// device address, looked up once per device with that device current.
constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void *g_scratch_addr[MAX_DEVICES] = {};

// Under CUDA's lazy module loading a kernel's code is loaded onto the device at its first launch,
// and loading can allocate device memory. The set-up of each device therefore loads every kernel
// this entry point can launch, so that no later call loads (or allocates) anything.
template <class A, int G, int R>
cudaError_t preload_arith() {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, build_profile_kernel<A, G, R>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, scan_kernel<A, G, R, MODE_SW, false>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, scan_kernel<A, G, R, MODE_NW, false>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, scan_kernel<A, G, R, MODE_HW, false>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, scan_kernel<A, G, R, MODE_OV, false>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, scan_kernel<A, G, R, MODE_SHW, false>);
    return e;
}

// Once per device, with that device current: the array's device address, and every kernel loaded.
hy_status scratch_address(int device, uint8_t **out) {
    if (device < 0 || device >= MAX_DEVICES) return fail(HY_ERR_UNSUPPORTED);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaSuccess) e = preload_arith<Pair16, MAIN_G, MAIN_R16>();
        if (e == cudaSuccess) e = preload_arith<PairTab16, MAIN_G, MAIN_R16>();
        if (e == cudaSuccess) e = preload_arith<Single32, MAIN_G32, MAIN_R32>();
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(HY_ERR_CUDA, e);
        }
        g_scratch_addr[device] = p;
    }
    *out = (uint8_t *)g_scratch_addr[device];
    return fail(HY_OK);
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

template <class A, int G, int R, int MODE>
cudaError_t launch_scores(const ScanParams &p, int blocks, size_t smem, cudaStream_t st) {
    auto kern = scan_kernel<A, G, R, MODE, false>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<blocks, BLOCK, smem, st>>>(p);
    return cudaGetLastError();
}

template <class A, int G, int R>
cudaError_t launch_scores_mode(int mode, const ScanParams &p, int blocks, size_t smem, cudaStream_t st) {
    switch (mode) {
    case MODE_SW: return launch_scores<A, G, R, MODE_SW>(p, blocks, smem, st);
    case MODE_NW: return launch_scores<A, G, R, MODE_NW>(p, blocks, smem, st);
    case MODE_HW: return launch_scores<A, G, R, MODE_HW>(p, blocks, smem, st);
    case MODE_OV: return launch_scores<A, G, R, MODE_OV>(p, blocks, smem, st);
    case MODE_SHW: return launch_scores<A, G, R, MODE_SHW>(p, blocks, smem, st);
    }
    return cudaErrorInvalidValue;
}

struct Region {
    QueryPlan qp;
    size_t prof_off = 0, prof_bytes = 0, bnd_off = 0, bnd_bytes = 0;
};

template <class A, int G, int R>
Region plan_region(const hy_db *db, const Partition &part, uint64_t qlen, size_t &cursor) {
    Region r;
    if (!part.n_items) return r;
    r.qp = plan_for<A>(qlen, G * R, db->al);
    r.prof_off = cursor;
    r.prof_bytes = (size_t)r.qp.n_passes * r.qp.pass_bytes;
    cursor = align256(cursor + r.prof_bytes);
    r.bnd_off = cursor;
    r.bnd_bytes = r.qp.n_passes > 1 ? 2 * sizeof(typename A::V) * part.total_cols : 0;
    cursor = align256(cursor + r.bnd_bytes);
    return r;
}

template <class A, int G, int R>
hy_status run_partition(const hy_db *db, const Partition &part, uint32_t item_base,
                        uint32_t item_end, const Region &rg, uint8_t *base, const uint8_t *d_query,
                        uint64_t qlen, int32_t *d_scores, int *d_err, cudaStream_t st) {
    if (item_base >= item_end) return fail(HY_OK);
    const bool i16 = A::NH == 2;
    const int32_t lim = i16 ? 32767 - db->go : 536870911;
    const int64_t total = A::letters(db->al) * A::TABLES * G * R * rg.qp.n_passes;
    const bool top_free = db->mode == MODE_SW || db->mode == MODE_HW || db->mode == MODE_OV;
    if (total > 0) {
        int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
        build_profile_kernel<A, G, R><<<blocks, 256, 0, st>>>(
            d_query, (int32_t)qlen, db->d_matrix, (int32_t)db->al, db->go, lim, top_free ? 1 : 0,
            rg.qp.vrow0, rg.qp.n_passes, reinterpret_cast<typename A::PE *>(base + rg.prof_off));
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(HY_ERR_CUDA, e);
    }
    ScanParams p{};
    p.meta = part.d_meta;
    p.item_base = item_base;
    p.n_items = item_end;
    p.item_ptr = nullptr;
    p.res = part.d_res;
    p.profile = base + rg.prof_off;
    p.pass_bytes = rg.qp.pass_bytes;
    p.n_passes = rg.qp.n_passes;
    p.vrow0 = rg.qp.vrow0;
    p.qlen = (int32_t)qlen;
    p.go = db->go;
    p.ge = db->ge;
    p.sentinel = i16 ? (-32768 + db->ge) : (INT32_MIN / 4);
    p.boundary = base + rg.bnd_off;
    p.scores = d_scores;
    p.qend = nullptr;
    p.tend = nullptr;
    p.best_key = nullptr;
    p.err = d_err;
    p.wait_polls = wait_polls();
    set_extents<A>(p, db, part, part.total_cols);
    const int gpb = BLOCK / G;
    const int blocks = (int)((item_end - item_base + gpb - 1) / gpb);
    cudaError_t e = launch_scores_mode<A, G, R>(db->mode, p, blocks, 2 * (size_t)rg.qp.pass_bytes + 16, st);
    if (e != cudaSuccess) return fail(HY_ERR_CUDA, e);
    return fail(HY_OK);
}

}  // namespace

extern "C" hy_status hy_scan_scores_noalloc(const hy_db *db, const uint8_t *d_query, uint64_t qlen,
                                            int32_t *d_scores, void *stream) {
    if (!db || !d_scores || (qlen && !d_query)) return fail(HY_ERR_INVALID_ARGUMENT);
    if (qlen > db->mql) return fail(HY_ERR_QUERY_TOO_LONG, (int64_t)qlen, (int64_t)db->mql);
    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(HY_ERR_CUDA, e);
    if (device != db->device) return fail(HY_ERR_INVALID_ARGUMENT);
    // Lay out this call's scratch: the timeout flag, then profile and boundary rows per partition.
    size_t cursor = 256;
    const bool tab = db->layout == HY_LAYOUT_PRECOMPUTED;
    const Region r16 = tab ? plan_region<PairTab16, MAIN_G, MAIN_R16>(db, db->p16, qlen, cursor)
                           : plan_region<Pair16, MAIN_G, MAIN_R16>(db, db->p16, qlen, cursor);
    const Region r32 = plan_region<Single32, MAIN_G32, MAIN_R32>(db, db->p32, qlen, cursor);
    if (cursor > NOALLOC_SCRATCH_BYTES)
        return fail(HY_ERR_UNSUPPORTED, (int64_t)cursor, (int64_t)NOALLOC_SCRATCH_BYTES);
    // This form stages its profile slices in shared memory only (large alphabets: hy_scan_scores).
    const size_t smem_need = 2 * (size_t)std::max(r16.qp.pass_bytes, r32.qp.pass_bytes) + 16;
    if (smem_need > db->smem_limit)
        return fail(HY_ERR_UNSUPPORTED, (int64_t)smem_need, (int64_t)db->smem_limit);
    uint8_t *base = nullptr;
    hy_status st = scratch_address(device, &base);
    if (st != HY_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    int *d_err = reinterpret_cast<int *>(base);
    e = cudaMemsetAsync(d_err, 0, sizeof(int), s);
    if (e != cudaSuccess) return fail(HY_ERR_CUDA, e);
    // The same per-query split as hy_scan_scores: pairs [k0, n) packed, the 2*k0 longest in int32.
    const QuerySplit split = split_for_query(db, qlen);
    st = tab ? run_partition<PairTab16, MAIN_G, MAIN_R16>(db, db->p16, split.k0, db->p16.n_items, r16, base,
                                                d_query, qlen, d_scores, d_err, s)
             : run_partition<Pair16, MAIN_G, MAIN_R16>(db, db->p16, split.k0, db->p16.n_items, r16, base,
                                                d_query, qlen, d_scores, d_err, s);
    if (st != HY_OK) return st;
    st = run_partition<Single32, MAIN_G32, MAIN_R32>(db, db->p32, 0, split.n_i32, r32, base, d_query,
                                                  qlen, d_scores, d_err, s);
    if (st != HY_OK) return st;
    int err = 0;
    e = cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(HY_ERR_CUDA, e);
    return err ? fail(device_error(err)) : fail(HY_OK);
}
