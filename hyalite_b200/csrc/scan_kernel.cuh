// scan_kernel.cuh -- the device side of the inter-sequence database scan.
//
// One "item" is either a PAIR of database sequences packed into the two int16 halves of every
// 32-bit register (Pair16), or ONE sequence in int32 lanes (Single32). A group of G consecutive
// lanes of a warp runs one item: lane L owns R consecutive query rows of the current pass and
// sweeps the item's columns one step behind lane L-1 (an anti-diagonal wavefront); the H and F
// values of a lane's last row move to the next lane with one shuffle each per step. A pass covers
// G*R query rows; the last row of a pass is handed to the next pass through a boundary row in
// global memory. The query profile of the current pass is staged into shared memory by a TMA bulk
// copy (cp.async.bulk) with an mbarrier, double-buffered across passes.
//
// The recurrence is the Gotoh recurrence of the scalar oracle (src/kernel.rs:168-217):
//   E[i][j] = max(E[i][j-1] - ge, H[i][j-1] - go)
//   F[i][j] = max(F[i-1][j] - ge, H[i-1][j] - go)
//   H[i][j] = max(H[i-1][j-1] + sub(q_i, t_j), E[i][j], F[i][j])   (SW: also max with 0)
// carried as G = H - go, with the profile holding P = sub + go so that G_diag + P = H_diag + sub:
//   E = max(E + (-ge), G_left)           __viaddmax            (ALU pipe)
//   F = max(F + (-ge), G_up)             __viaddmax            (ALU)
//   d = G_diag + P                       __vadd2 (x2 for the two Gathered tables)   (FMA pipe)
//   H = max(d, E, F)                     __vimax3 (SW: __vimax3_relu)               (ALU)
//   G = H + (-go)                        __vadd2               (FMA)
// For SW scores the row-to-row chain is shortened to one op (see sweep_step).
// Width safety: the host routes a sequence to Pair16 only when its magnitude bound plus gap_open
// fits int16 (bound + go <= 32767), which keeps every intermediate above exactly representable,
// so the packed arithmetic never wraps on a real cell and the results equal the i32 oracle.
//
// Rows: the query is padded at the FRONT so the last query row always sits in the last slot of
// the last lane of the last pass. Virtual rows (index <= 0) reproduce the border row 0 exactly:
// left border 0 and a profile value of `go` (free top border) or 0 (penalised top border).
// Columns: in a Pair16 item the shorter sequence is padded with a symbol whose profile value is
// the most negative representable; padded columns never feed a real cell and are excluded from
// every answer region (or, for SW, can only tie a real cell at a larger column).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace hy {

enum { MODE_SW = 0, MODE_NW = 1, MODE_HW = 2, MODE_OV = 3, MODE_SHW = 4 };

// Flags::for_mode (src/kernel.rs:43-98).
template <int MODE>
struct ModeFlags {
    static constexpr bool top_free = MODE == MODE_SW || MODE == MODE_HW || MODE == MODE_OV;
    static constexpr bool left_free = MODE == MODE_SW || MODE == MODE_OV || MODE == MODE_SHW;
    static constexpr bool last_row = MODE == MODE_HW || MODE == MODE_OV;
    static constexpr bool last_col = MODE == MODE_OV || MODE == MODE_SHW;
    static constexpr bool local = MODE == MODE_SW;
    static constexpr bool corner = MODE == MODE_NW;
};

struct ItemMeta {
    uint64_t col_off;  // first column of the item in the residue / boundary arrays
    uint32_t w;        // columns swept (the longer length of the pair)
    uint32_t n[2];     // sequence lengths; a lone sequence has n[1] = 0 and idx[1] = NO_INDEX
    uint32_t idx[2];   // global db indices
    uint32_t pad_;
};
static constexpr uint32_t NO_INDEX = 0xffffffffu;

struct ScanParams {
    const ItemMeta *meta;
    uint32_t item_base;        // first item of the launch: items [item_base, n_items) run
    uint32_t n_items;
    const uint32_t *item_ptr;  // when set: run the single item *item_ptr (NO_INDEX: nothing)
    const void *res;           // Pair16: uint16 (lo | hi << 8); Single32: uint8
    const uint8_t *profile;    // pass-major profile slices, pass_bytes each
    uint32_t pass_bytes;
    int32_t n_passes;
    int32_t vrow0;  // grid row of pass 0, lane 0, slot 0 (<= 1)
    int32_t qlen;
    int32_t go, ge;
    int32_t sentinel;
    void *boundary;     // 2 values (G, F) per column, starting at column bnd_col0
    uint64_t bnd_col0;  // first column the boundary region covers
    int32_t *scores;    // per-target outputs by global index (may be null: best key only)
    int32_t *qend;
    int32_t *tend;
    unsigned long long *best_key;
    int *err;
    // Band recovery only: when set, the winner named by *best_key is written here as {score,
    // query end, target end} instead of to scores / qend / tend.
    int32_t *ends_out;
    uint32_t wait_polls;  // polls a wait for a profile copy makes before it gives up
    // Extents the bounds-checked build (HY_BOUNDS) verifies every item against before use.
    uint64_t res_cols;  // columns of the residue array
    uint64_t bnd_cols;  // columns the boundary region holds, from bnd_col0
    uint32_t n_seqs;    // db indices are below this
    uint32_t letters;   // profile letters per table
};

// Error words a kernel leaves in ScanParams::err: a bounded wait gave up, or (bounds-checked
// build) an item failed its check and was skipped.
enum { ERR_WAIT = 1, ERR_BOUNDS = 2 };

// ---- lane arithmetic -----------------------------------------------------------------------
//
// Per cell the recurrence issues three ops on the ALU pipe (two __viaddmax for E and F, one
// __vimax3 for H) and, for int16x2, three on the FMA pipe (__vadd2 for the diagonal's two profile
// words and for G = H - go); the two half-rate pipes run in parallel.

struct Pair16 {
    typedef uint32_t V;
    // Profile words: a low-half table holding (P, 0) and a high-half table holding (0, P), so the
    // two sequences' substitution values are merged by per-halfword adds on the FMA pipe.
    typedef uint32_t PE;
    typedef uint16_t RES;
    static constexpr int NH = 2;
    static constexpr int EPV = 4;     // profile words per 16-byte vector
    static constexpr int TABLES = 2;  // per pass slice: the low-half table, then the high-half one
    static constexpr int32_t VMIN = -32768, VMAX = 32767;
    __device__ __forceinline__ static V splat(int64_t x) {
        x = x < VMIN ? VMIN : (x > VMAX ? VMAX : x);
        uint32_t h = (uint16_t)(int16_t)x;
        return h | (h << 16);
    }
    __device__ __forceinline__ static V addmax(V a, V b, V c) { return __viaddmax_s16x2(a, b, c); }
    __device__ __forceinline__ static V vmax(V a, V b) { return __vmaxs2(a, b); }
    __device__ __forceinline__ static V vmax3(V a, V b, V c) { return __vimax3_s16x2(a, b, c); }
    __device__ __forceinline__ static V vmax3_relu(V a, V b, V c) { return __vimax3_s16x2_relu(a, b, c); }
    __device__ __forceinline__ static V vadd(V a, V b) { return __vadd2(a, b); }
    __device__ __forceinline__ static V diag(V g, V pa, V pb) { return __vadd2(__vadd2(g, pa), pb); }
    __device__ __forceinline__ static int32_t get(V v, int h) {
        return h ? (int32_t)(int16_t)(v >> 16) : (int32_t)(int16_t)(v & 0xffffu);
    }
    // Running maximum; up[h] is set where x is strictly greater than best in half h.
    __device__ __forceinline__ static V bmax(V best, V x, bool &up0, bool &up1) {
        bool ph, pl;
        V r = __vibmax_s16x2(best, x, &ph, &pl);
        up0 = !pl;
        up1 = !ph;
        return r;
    }
    __device__ __forceinline__ static void residues(RES r, int &a, int &b) {
        a = r & 0xff;
        b = r >> 8;
    }
    // Chunk k (EPV rows) of the profile for letters (a, b): prof_lo is the low-half table used by
    // the low sequence, prof_hi the high-half table used by the high sequence.
    template <int R, int G>
    __device__ __forceinline__ static void load_chunk(const uint8_t *prof_lo, const uint8_t *prof_hi,
                                                      int a, int b, int lane, int k, V (&pa)[EPV],
                                                      V (&pb)[EPV]) {
        constexpr int KCH = R / EPV;
        const uint4 A = reinterpret_cast<const uint4 *>(prof_lo)[((size_t)a * KCH + k) * G + lane];
        const uint4 B = reinterpret_cast<const uint4 *>(prof_hi)[((size_t)b * KCH + k) * G + lane];
        pa[0] = A.x; pa[1] = A.y; pa[2] = A.z; pa[3] = A.w;
        pb[0] = B.x; pb[1] = B.y; pb[2] = B.z; pb[3] = B.w;
    }
    // The profile word of value v in table t (0: low half, 1: high half).
    __host__ __device__ __forceinline__ static PE word(int64_t v, int t) {
        const uint32_t h = (uint16_t)(int16_t)v;
        return t ? (h << 16) : h;
    }
    // Profile letters of an alphabet of `al` symbols (the padding symbol included).
    static constexpr bool PAIRTAB = false;
    __host__ __device__ static constexpr int64_t letters(int64_t al) { return al + 1; }
    // Residue code of a pair column (low sequence's symbol lo, high sequence's hi).
    __host__ __device__ static constexpr uint32_t code(uint32_t lo, uint32_t hi, uint32_t) { return lo | (hi << 8); }
};

// The int16x2 arithmetic with a half-size query profile, for kernels whose groups each keep their
// own profile in shared memory (the pair kernel): each table holds 16-bit entries, and a row's
// word is assembled from the two tables' entries by one byte permute instead of merging two 32-bit
// words by an add. The same values; half the shared memory, so twice the groups fit on an SM.
struct Pair16H : Pair16 {
    typedef uint16_t PE;
    __device__ __forceinline__ static V diag(V g, V p, V) { return __vadd2(g, p); }
    template <int R, int G>
    __device__ __forceinline__ static void load_chunk(const uint8_t *prof_lo, const uint8_t *prof_hi,
                                                      int a, int b, int lane, int k, V (&pa)[EPV],
                                                      V (&pb)[EPV]) {
        constexpr int KCH = R / EPV;
        const uint2 A = reinterpret_cast<const uint2 *>(prof_lo)[((size_t)a * KCH + k) * G + lane];
        const uint2 B = reinterpret_cast<const uint2 *>(prof_hi)[((size_t)b * KCH + k) * G + lane];
        // Row 2i: the low entries of both tables' word i; row 2i + 1: the high entries.
        pa[0] = __byte_perm(A.x, B.x, 0x5410);
        pa[1] = __byte_perm(A.x, B.x, 0x7632);
        pa[2] = __byte_perm(A.y, B.y, 0x5410);
        pa[3] = __byte_perm(A.y, B.y, 0x7632);
        pb[0] = pb[1] = pb[2] = pb[3] = 0;
    }
    __host__ __device__ __forceinline__ static PE word(int64_t v, int) { return (uint16_t)(int16_t)v; }
};

// The Precomputed layout (src/inter.rs:317-330: "a precomputed score table, so each cell's
// substitution vector is a direct load with no gather"), restated for the device: the database
// stores each pair column as one code c = lo * (al + 1) + hi, and the pass's profile is a single
// table indexed by (c, query row) whose word already holds both halves' substitution values. A
// cell pair then costs one profile load and one add instead of two of each; the table has
// (al + 1)^2 letters, so it is compact for small alphabets only. Arithmetic as Pair16.
struct PairTab16 : Pair16 {
    static constexpr int TABLES = 1;
    static constexpr bool PAIRTAB = true;
    __host__ __device__ static constexpr int64_t letters(int64_t al) { return (al + 1) * (al + 1); }
    __host__ __device__ static constexpr uint32_t code(uint32_t lo, uint32_t hi, uint32_t al) {
        return lo * (al + 1) + hi;
    }
    __device__ __forceinline__ static V diag(V g, V p, V) { return __vadd2(g, p); }
    __device__ __forceinline__ static void residues(RES r, int &a, int &b) {
        a = r;
        b = 0;
    }
    template <int R, int G>
    __device__ __forceinline__ static void load_chunk(const uint8_t *prof, const uint8_t *, int c,
                                                      int, int lane, int k, V (&pa)[EPV],
                                                      V (&pb)[EPV]) {
        constexpr int KCH = R / EPV;
        const uint4 A = reinterpret_cast<const uint4 *>(prof)[((size_t)c * KCH + k) * G + lane];
        pa[0] = A.x; pa[1] = A.y; pa[2] = A.z; pa[3] = A.w;
        pb[0] = pb[1] = pb[2] = pb[3] = 0;
    }
    // The word of a pair code's two values (low half: the low sequence's).
    __host__ __device__ __forceinline__ static PE pair_word(int64_t lo, int64_t hi) {
        return (uint32_t)(uint16_t)(int16_t)lo | ((uint32_t)(uint16_t)(int16_t)hi << 16);
    }
};

struct Single32 {
    typedef int32_t V;
    typedef int32_t PE;
    typedef uint8_t RES;
    static constexpr int NH = 1;
    static constexpr int EPV = 4;
    static constexpr int TABLES = 1;
    static constexpr int64_t VMIN = INT32_MIN, VMAX = INT32_MAX;
    __device__ __forceinline__ static V splat(int64_t x) {
        return (V)(x < VMIN ? VMIN : (x > VMAX ? VMAX : x));
    }
    __device__ __forceinline__ static V addmax(V a, V b, V c) { return __viaddmax_s32(a, b, c); }
    __device__ __forceinline__ static V vmax(V a, V b) { return max(a, b); }
    __device__ __forceinline__ static V vmax3(V a, V b, V c) { return __vimax3_s32(a, b, c); }
    __device__ __forceinline__ static V vmax3_relu(V a, V b, V c) { return __vimax3_s32_relu(a, b, c); }
    __device__ __forceinline__ static V vadd(V a, V b) { return a + b; }
    __device__ __forceinline__ static V diag(V g, V pa, V) { return g + pa; }
    __device__ __forceinline__ static int32_t get(V v, int) { return v; }
    __device__ __forceinline__ static V bmax(V best, V x, bool &up0, bool &up1) {
        bool p;
        V r = __vibmax_s32(best, x, &p);
        up0 = !p;
        up1 = false;
        return r;
    }
    __device__ __forceinline__ static void residues(RES r, int &a, int &b) {
        a = r;
        b = r;
    }
    template <int R, int G>
    __device__ __forceinline__ static void load_chunk(const uint8_t *prof, const uint8_t *, int a,
                                                      int, int lane, int k, V (&pa)[EPV],
                                                      V (&pb)[EPV]) {
        constexpr int KCH = R / EPV;
        const int4 A = reinterpret_cast<const int4 *>(prof)[((size_t)a * KCH + k) * G + lane];
        pa[0] = A.x; pa[1] = A.y; pa[2] = A.z; pa[3] = A.w;
        pb[0] = pb[1] = pb[2] = pb[3] = 0;
    }
    __host__ __device__ __forceinline__ static PE word(int64_t v, int) { return (PE)v; }
    static constexpr bool PAIRTAB = false;
    __host__ __device__ static constexpr int64_t letters(int64_t al) { return al + 1; }
};

// Profile bytes per (letter, query row) of one lane arithmetic: every table's word.
template <class A>
__host__ __device__ constexpr size_t profile_row_bytes() {
    return A::TABLES * sizeof(typename A::PE);
}

// Profile bytes of one query row of a pass slice: every letter of every table.
template <class A>
__host__ __device__ constexpr size_t profile_slice_row_bytes(int64_t al) {
    return (size_t)A::letters(al) * profile_row_bytes<A>();
}

// ---- small helpers -------------------------------------------------------------------------

// gap_penalty (src/kernel.rs:103-109).
__device__ __forceinline__ int64_t gap_pen(int32_t go, int32_t ge, int64_t len) {
    return len <= 0 ? 0 : (int64_t)go + (len - 1) * (int64_t)ge;
}

// Answer candidate under the tie-break of Best::consider (src/kernel.rs:113-129): higher score,
// then smaller grid column, then smaller grid row.
struct Cand {
    int32_t s;
    int32_t col;
    int32_t row;
};
__device__ __forceinline__ bool better(const Cand &a, const Cand &b) {
    return a.s > b.s || (a.s == b.s && (a.col < b.col || (a.col == b.col && a.row < b.row)));
}
__device__ __forceinline__ void consider(Cand &b, int32_t s, int32_t col, int32_t row) {
    Cand c = {s, col, row};
    if (better(c, b)) b = c;
}

// Best border-cell candidate of the mode's answer region (reduce_answer, src/kernel.rs:223-260,
// restricted to row 0 and column 0), for query length m and target length n.
template <int MODE>
__device__ __forceinline__ Cand border_seed(int32_t m, int32_t n, int32_t go, int32_t ge) {
    const Cand none = {INT32_MIN, INT32_MAX, INT32_MAX};
    switch (MODE) {
    case MODE_SW: return {0, 0, 0};
    case MODE_NW:
        if (m == 0) return {(int32_t)-gap_pen(go, ge, n), n, 0};
        if (n == 0) return {(int32_t)-gap_pen(go, ge, m), 0, m};
        return none;
    case MODE_HW:
        if (m == 0) return {0, 0, 0};
        return {(int32_t)-gap_pen(go, ge, m), 0, m};
    case MODE_SHW:
        if (n == 0) return {0, 0, 0};
        return {(int32_t)-gap_pen(go, ge, n), n, 0};
    default: /* OV */
        if (m == 0 || n == 0) return {0, 0, 0};
        return {0, 0, m};
    }
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Issue one TMA bulk copy global -> shared whose completion is tracked by `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, "
        "0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after `polls` polls (each poll may itself suspend briefly).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t polls) {
    for (uint32_t it = 0; it < polls; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// After a wait gave up (one thread of the block): records the timeout and lets the copies still
// in flight into the block's shared memory land before the block exits (bounded again, by the
// default number of polls; the block's shared memory stays allocated while this thread runs).
// `pending` holds the barriers with a copy outstanding (bit b: bars[b]) and `phase` the parity
// each waits for. Out of line: the scan kernels' hot loops keep their register allocation.
static __device__ __noinline__ void wait_gave_up(int *err, uint64_t *bars, uint32_t pending, uint32_t phase) {
    atomicExch(err, ERR_WAIT);
    for (int b = 0; b < 2; ++b)
        if ((pending >> b) & 1u) mbar_wait_bounded(&bars[b], (phase >> b) & 1u, 1u << 24);
}

// ---- thread-block clusters (the band kernel's blocks) -----------------------------------------
// A block not launched as part of a cluster is a cluster of one: rank 0 of 1.
__device__ __forceinline__ int cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return (int)r;
}
__device__ __forceinline__ int cluster_size() {
    uint32_t n;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    return (int)n;
}
// Every thread of every block of the cluster; orders memory at cluster scope (release, acquire).
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// The 32-bit word at the address of `p` in the shared memory of block `rank` of the cluster.
__device__ __forceinline__ uint32_t ld_cluster_u32(const void *p, int rank) {
    uint32_t a, v;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
// The block barrier of a cluster of one, else the cluster barrier.
__device__ __forceinline__ void band_sync(const int csize) {
    if (csize > 1)
        cluster_barrier();
    else
        __syncthreads();
}
// Whether `v` holds in any block of the cluster (`v` block-uniform; every thread calls it).
// `flag` is a shared word of this block; no block returns before every block has read the others'.
__device__ __forceinline__ bool cluster_any(const bool v, uint32_t *flag, const int csize) {
    if (csize == 1) return v;
    if (threadIdx.x == 0) *flag = v ? 1u : 0u;
    cluster_barrier();
    const uint32_t o = (int)threadIdx.x < csize ? ld_cluster_u32(flag, (int)threadIdx.x) : 0u;
    const bool any = __syncthreads_or(o != 0);
    cluster_barrier();
    return any;
}

__device__ __forceinline__ unsigned long long hit_key(int32_t score, uint32_t idx) {
    return ((unsigned long long)((uint32_t)score ^ 0x80000000u) << 32) | (uint32_t)(~idx);
}

// ---- one pass of the wavefront -------------------------------------------------------------
//
// Sweeps the item's columns for the G*R query rows of one pass. Steps are warp-uniform (every
// lane of the warp shuffles every step). Lane L works on column j = s - L + 1 at step s; the G and
// F values of its last row at column j reach lane L+1 at step s+1. Lane 0 reads the row above the
// pass from the boundary row (or the top border in the first pass); lane G-1 writes the pass's
// last row to the boundary row unless this is the last pass. The state lives in a Sweep so a
// pass can be run in windows of steps (the block-cooperative band kernel interleaves warps).
template <class A, int R>
struct Sweep {
    typename A::V Gp[R], E[R];  // G (= H - go) of the previous column and E, per row slot
    typename A::V diag;         // G of the row above at the previous column (row slot 0)
    typename A::V botG, botF;   // this lane's last row at its current column, for lane L+1
    // SW end tracking within a pass: the running per-half maximum of G (= H - go) and the cell id
    // (column * R + slot) where it was first reached; column-major order inside the lane means
    // the first strict improvement is the smallest (column, row).
    typename A::V pbest;
    int32_t pid0, pid1;
    typename A::V botM;  // column maxima (COLMAX): G maximum of this column down to this lane's rows
};

// Where a COLMAX sweep writes its column maxima: per half, the pair's array indexed by target
// position (H of the column's best cell, so >= 0 in local mode); `atomic` when several passes
// combine into one array.
struct ColMaxOut {
    int32_t *p[2];
    bool atomic;
};

template <class A, int R, int MODE>
__device__ __forceinline__ void sweep_begin(Sweep<A, R> &sw, const int32_t row0, const int32_t go,
                                            const int32_t ge, const typename A::V Sv) {
    typedef ModeFlags<MODE> Fl;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int32_t row = row0 + r;
        const int64_t lb = (row <= 0 || Fl::left_free) ? 0 : -gap_pen(go, ge, row);
        sw.Gp[r] = A::splat(lb - go);
        sw.E[r] = Sv;
    }
    const int32_t row = row0 - 1;
    const int64_t lb = (row <= 0 || Fl::left_free) ? 0 : -gap_pen(go, ge, row);
    sw.diag = A::splat(lb - go);
    sw.botG = A::splat(0);
    sw.botF = A::splat(0);
    sw.pbest = A::splat(INT32_MIN);
    sw.pid0 = -1;
    sw.pid1 = -1;
}

// Constants of a sweep that do not change from step to step.
template <class A>
struct SweepConst {
    typename A::V negge, neggo, Sv;
    typename A::V top_free_g;  // G of the free top border row (H = 0)
};

// One step s of one lane. CHECKED steps test whether the lane's column is inside [1, w]; the
// caller runs unchecked steps only where every lane of the warp is live.
// With PRE the step's residue code and (lane 0) boundary-row values come from the caller, which
// loaded them one step ahead.
template <class A, int G, int R, int MODE, bool ENDS, bool CHECKED, bool PRE = false, bool COLMAX = false>
__device__ __forceinline__ void sweep_step(Sweep<A, R> &sw, const int s, const int lane,
                                           const int32_t w, const uint32_t (&n)[2],
                                           const typename A::RES *__restrict__ res,
                                           const uint8_t *prof_a, const uint8_t *prof_b,
                                           const int32_t row0, const bool first_pass,
                                           const bool last_pass, typename A::V *bnd,
                                           const int32_t qlen, const int32_t go, const int32_t ge,
                                           const SweepConst<A> &k, typename A::V &best,
                                           Cand (&cand)[2], const typename A::RES pre_r = 0,
                                           const typename A::V pre_g = 0, const typename A::V pre_f = 0,
                                           const ColMaxOut *cmo = nullptr) {
    typedef typename A::V V;
    typedef ModeFlags<MODE> Fl;
    static_assert(!COLMAX || (Fl::local && !ENDS), "column maxima are a local score-only sweep");
    const V negge = k.negge, neggo = k.neggo;
    {
        const int32_t j = s - lane + 1;
        V upG = __shfl_up_sync(0xffffffffu, sw.botG, 1, G);
        V upF = __shfl_up_sync(0xffffffffu, sw.botF, 1, G);
        // COLMAX: the column's maximum over the rows of the lanes above (lane 0: none this pass).
        V upM;
        if constexpr (COLMAX) {
            upM = __shfl_up_sync(0xffffffffu, sw.botM, 1, G);
            if (lane == 0) upM = neggo;
        }
        const bool live = !CHECKED || (j >= 1 && j <= w);
        if (lane == 0) {
            if (first_pass) {
                upG = Fl::top_free ? k.top_free_g : A::splat(-gap_pen(go, ge, j) - go);
                upF = k.Sv;
            } else if (live) {
                upG = PRE ? pre_g : bnd[2 * (j - 1)];
                upF = PRE ? pre_f : bnd[2 * (j - 1) + 1];
            }
        }
        if (live) {
            int a, b;
            A::residues(PRE ? pre_r : res[j - 1], a, b);
            V pa[A::EPV], pb[A::EPV];
            V g_up = upG, f = upF, gd = sw.diag, hprev = A::splat(0), hlast = A::splat(0);
            V xprev = A::splat(0);
            V cm;  // COLMAX: this column's G maximum, down to this lane's rows
            if constexpr (COLMAX) cm = upM;
            const int32_t jR = j * R;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r % A::EPV == 0)
                    A::template load_chunk<R, G>(prof_a, prof_b, a, b, lane, r / A::EPV, pa, pb);
                sw.E[r] = A::addmax(sw.E[r], negge, sw.Gp[r]);
                V h;
                if (Fl::local) {
                    // SW, with a one-op dependency chain from row to row: with x = max(d, E, 0) -
                    // go, G = max(F - go, x) and, since go >= ge, F of the next row = max(F - ge,
                    // G) = max(F - ge, x). x >= -go, so nothing leaves int16. h here is G; the
                    // running maximum (and with ENDS the tracked best cell) is kept in G, go added
                    // at the end.
                    f = A::addmax(f, negge, r == 0 ? g_up : xprev);
                    const V d = A::diag(gd, pa[r % A::EPV], pb[r % A::EPV]);
                    const V x = A::vadd(A::vmax3_relu(d, sw.E[r], d), neggo);
                    xprev = x;
                    h = A::addmax(f, neggo, x);
                    gd = sw.Gp[r];
                    sw.Gp[r] = h;
                    g_up = h;
                } else {
                    f = A::addmax(f, negge, g_up);
                    const V d = A::diag(gd, pa[r % A::EPV], pb[r % A::EPV]);
                    h = Fl::local ? A::vmax3_relu(d, sw.E[r], f) : A::vmax3(d, sw.E[r], f);
                    gd = sw.Gp[r];
                    const V g = A::vadd(h, neggo);
                    sw.Gp[r] = g;
                    g_up = g;
                }
                if (Fl::local) {
                    if (ENDS) {
                        bool u0, u1;
                        sw.pbest = A::bmax(sw.pbest, h, u0, u1);
                        if (u0) sw.pid0 = jR + r;
                        if (u1) sw.pid1 = jR + r;
                    } else if (COLMAX) {
                        if (r & 1)
                            cm = A::vmax3(cm, hprev, h);
                        else
                            hprev = h;
                    } else {
                        if (r & 1)
                            best = A::vmax3(best, hprev, h);
                        else
                            hprev = h;
                    }
                }
                if (r == R - 1) hlast = h;
            }
            if (Fl::local && !ENDS && (R & 1)) {
                if (COLMAX)
                    cm = A::vmax(cm, hprev);
                else
                    best = A::vmax(best, hprev);
            }
            if constexpr (COLMAX) {
                // The last lane holds the column's maximum over the pass: H = G + go.
                sw.botM = cm;
                if (lane == G - 1) {
#pragma unroll
                    for (int h = 0; h < A::NH; ++h) {
                        if (j <= (int32_t)n[h]) {
                            const int32_t v = A::get(cm, h) + go;
                            if (cmo->atomic)
                                atomicMax(cmo->p[h] + (j - 1), v);
                            else
                                cmo->p[h][j - 1] = v;
                        }
                    }
                }
            }
            sw.botG = g_up;
            sw.botF = f;
            sw.diag = upG;
            if (lane == G - 1 && !last_pass) {
                bnd[2 * (j - 1)] = sw.botG;
                bnd[2 * (j - 1) + 1] = sw.botF;
            }
            // Last query row (grid row qlen): slot R-1 of lane G-1 in the last pass.
            if ((Fl::last_row || Fl::corner) && last_pass && lane == G - 1) {
#pragma unroll
                for (int h = 0; h < A::NH; ++h) {
                    const int32_t nh = (int32_t)n[h];
                    if (Fl::last_row ? (j <= nh) : (j == nh)) consider(cand[h], A::get(hlast, h), j, qlen);
                }
            }
            // Last column of each sequence (grid column n): every real row of this lane.
            if (Fl::last_col) {
#pragma unroll
                for (int h = 0; h < A::NH; ++h) {
                    if (j == (int32_t)n[h]) {
#pragma unroll
                        for (int r = 0; r < R; ++r)
                            if (row0 + r >= 1) consider(cand[h], A::get(sw.Gp[r], h) + go, j, row0 + r);
                    }
                }
            }
        }
    }
}

// Steps [s_begin, s_end) of one lane. `w_min` is the smallest item width in the warp: steps in
// [G-1, w_min) have every lane of the warp on a real column and skip the per-lane checks. All
// bounds are warp-uniform.
// With PREFETCH the unchecked steps load the next step's residue code and boundary-row values one
// step ahead; only for callers whose boundary row was written by an earlier, completed pass (the
// band kernel's warps read rows another warp is writing and keep their exact read timing).
template <class A, int G, int R, int MODE, bool ENDS, bool PREFETCH = false, bool COLMAX = false>
__device__ __forceinline__ void sweep_run(Sweep<A, R> &sw, const int s_begin, const int s_end,
                                          const int w_min, const int lane, const int32_t w,
                                          const uint32_t (&n)[2],
                                          const typename A::RES *__restrict__ res,
                                          const uint8_t *prof_a, const uint8_t *prof_b,
                                          const int32_t row0, const bool first_pass,
                                          const bool last_pass, typename A::V *bnd,
                                          const int32_t qlen, const int32_t go, const int32_t ge,
                                          const typename A::V Sv, typename A::V &best,
                                          Cand (&cand)[2], const ColMaxOut *cmo = nullptr) {
    SweepConst<A> k;
    k.negge = A::splat(-(int64_t)ge);
    k.neggo = A::splat(-(int64_t)go);
    k.Sv = Sv;
    k.top_free_g = A::splat(-(int64_t)go);
    const int fast_lo = max(s_begin, G - 1);
    const int fast_hi = max(fast_lo, min(s_end, w_min));
    const int head_end = min(s_end, fast_lo);
    for (int s = s_begin; s < head_end; ++s)
        sweep_step<A, G, R, MODE, ENDS, true, false, COLMAX>(sw, s, lane, w, n, res, prof_a, prof_b, row0,
                                                             first_pass, last_pass, bnd, qlen, go, ge, k,
                                                             best, cand, 0, 0, 0, cmo);
    if (PREFETCH && fast_lo < fast_hi) {
        typedef typename A::V V;
        // Every lane of the warp is inside its item in [fast_lo, fast_hi): the indices below
        // (step s - lane, clamped to the range) are real columns.
        typename A::RES r_cur = res[fast_lo - lane];
        V g_cur = 0, f_cur = 0;
        if (lane == 0 && !first_pass) {
            g_cur = bnd[2 * (fast_lo - lane)];
            f_cur = bnd[2 * (fast_lo - lane) + 1];
        }
        for (int s = fast_lo; s < fast_hi; ++s) {
            const int sn = min(s + 1, fast_hi - 1);
            const typename A::RES r_next = res[sn - lane];
            V g_next = g_cur, f_next = f_cur;
            if (lane == 0 && !first_pass) {
                g_next = bnd[2 * (sn - lane)];
                f_next = bnd[2 * (sn - lane) + 1];
            }
            sweep_step<A, G, R, MODE, ENDS, false, true, COLMAX>(sw, s, lane, w, n, res, prof_a, prof_b,
                                                                 row0, first_pass, last_pass, bnd, qlen,
                                                                 go, ge, k, best, cand, r_cur, g_cur,
                                                                 f_cur, cmo);
            r_cur = r_next;
            g_cur = g_next;
            f_cur = f_next;
        }
    } else {
        for (int s = fast_lo; s < fast_hi; ++s)
            sweep_step<A, G, R, MODE, ENDS, false, false, COLMAX>(sw, s, lane, w, n, res, prof_a, prof_b,
                                                                  row0, first_pass, last_pass, bnd, qlen,
                                                                  go, ge, k, best, cand, 0, 0, 0, cmo);
    }
    for (int s = max(fast_hi, head_end); s < s_end; ++s)
        sweep_step<A, G, R, MODE, ENDS, true, false, COLMAX>(sw, s, lane, w, n, res, prof_a, prof_b, row0,
                                                             first_pass, last_pass, bnd, qlen, go, ge, k,
                                                             best, cand, 0, 0, 0, cmo);
}

// The lane's tracked best cell of the pass as a candidate (local mode: pbest holds G = H - go).
template <class A, int R, int MODE, bool ENDS>
__device__ __forceinline__ void sweep_end(const Sweep<A, R> &sw, const int32_t row0, const int32_t go,
                                          Cand (&cand)[2]) {
    if (ModeFlags<MODE>::local && ENDS) {
        if (sw.pid0 >= 0) consider(cand[0], A::get(sw.pbest, 0) + go, sw.pid0 / R, row0 + sw.pid0 % R);
        if (A::NH > 1 && sw.pid1 >= 0)
            consider(cand[1], A::get(sw.pbest, 1) + go, sw.pid1 / R, row0 + sw.pid1 % R);
    }
}

// One whole pass: begin, every step, end.
template <class A, int G, int R, int MODE, bool ENDS, bool COLMAX = false>
__device__ __forceinline__ void sweep_pass(const int lane, const int steps, const int w_min,
                                           const int32_t w, const uint32_t (&n)[2],
                                           const typename A::RES *__restrict__ res,
                                           const uint8_t *prof_a, const uint8_t *prof_b,
                                           const int32_t row0, const bool first_pass,
                                           const bool last_pass, typename A::V *bnd,
                                           const int32_t qlen, const int32_t go, const int32_t ge,
                                           const typename A::V Sv, typename A::V &best,
                                           Cand (&cand)[2], const ColMaxOut *cmo = nullptr) {
    Sweep<A, R> sw;
    sweep_begin<A, R, MODE>(sw, row0, go, ge, Sv);
    if constexpr (COLMAX) sw.botM = A::splat(-(int64_t)go);
    sweep_run<A, G, R, MODE, ENDS, true, COLMAX>(sw, 0, steps, w_min, lane, w, n, res, prof_a, prof_b,
                                                 row0, first_pass, last_pass, bnd, qlen, go, ge, Sv,
                                                 best, cand, cmo);
    sweep_end<A, R, MODE, ENDS>(sw, row0, go, cand);
}

// ---- two columns per step: the SW score sweep of int16x2 pairs and int32 items ------------------
//
// Lane L works on columns j0 = 2(s - L) + 1 and j1 = j0 + 1 at step s, R rows each: the per-step
// work (shuffles, residue and boundary loads, loop control) is spread over 2R rows of work while a
// lane keeps only R rows of state, and the F chains of the two columns (column j1 one row behind
// column j0) give the scheduler two independent dependency chains. Long form of the recurrence
// (E, F, H = max(d, E, F, 0), G = H - go); the running maximum is kept on G.

// The residue codes of two adjacent columns as one load: two 16-bit pair codes (int16x2 pairs) or
// two 8-bit residues (int32 items). OK: the lane arithmetic has a two-column form.
template <class A>
struct TwoCodes {
    static constexpr bool OK = (A::NH == 2 && sizeof(typename A::RES) == 2) || (A::NH == 1 && sizeof(typename A::RES) == 1);
    static constexpr int BITS = 8 * (int)sizeof(typename A::RES);
    typedef typename std::conditional<sizeof(typename A::RES) == 2, uint32_t, uint16_t>::type W;
};

template <class A, int R>
struct Sweep2 {
    typename A::V Gp[R], E[R];        // G of the previous column and E, per row slot
    typename A::V diag;               // G of the row above the lane at the column before j0
    typename A::V botG[2], botF[2];   // this lane's last row at columns j0, j1, for lane L + 1
};

// One column of R rows: E, F, H, G in place; returns the last row's G and F.
template <class A, int G, int R>
__device__ __forceinline__ void sweep2_column(Sweep2<A, R> &sw, const int a, const int b, const int lane,
                                              const uint8_t *prof_a, const uint8_t *prof_b,
                                              typename A::V g_up, typename A::V f, typename A::V gd,
                                              const typename A::V negge, const typename A::V neggo,
                                              typename A::V &best, typename A::V &outG,
                                              typename A::V &outF) {
    typedef typename A::V V;
    V pa[A::EPV], pb[A::EPV];
    V hprev = A::splat(0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (r % A::EPV == 0) A::template load_chunk<R, G>(prof_a, prof_b, a, b, lane, r / A::EPV, pa, pb);
        sw.E[r] = A::addmax(sw.E[r], negge, sw.Gp[r]);
        f = A::addmax(f, negge, g_up);
        const V d = A::diag(gd, pa[r % A::EPV], pb[r % A::EPV]);
        const V h = A::vmax3_relu(d, sw.E[r], f);
        const V g = A::vadd(h, neggo);
        gd = sw.Gp[r];
        sw.Gp[r] = g;
        g_up = g;
        if (r & 1)
            best = A::vmax3(best, hprev, g);
        else
            hprev = g;
    }
    if (R & 1) best = A::vmax(best, hprev);
    outG = g_up;
    outF = f;
}

// Both columns of a step, interleaved one row apart (row r of column j0 with row r - 1 of column
// j1, which needs rows r - 1 of column j0 only): the same values as sweep2_column twice, with the
// two columns' dependency chains side by side in the instruction stream.
template <class A, int G, int R>
__device__ __forceinline__ void sweep2_both(Sweep2<A, R> &sw, const int a0, const int b0, const int a1,
                                            const int b1, const int lane, const uint8_t *prof_a,
                                            const uint8_t *prof_b, const typename A::V upG0,
                                            const typename A::V upF0, const typename A::V upG1,
                                            const typename A::V upF1, const typename A::V negge,
                                            const typename A::V neggo, typename A::V &best) {
    typedef typename A::V V;
    V p0a[A::EPV], p0b[A::EPV], p1a[A::EPV], p1b[A::EPV];
    V g_up0 = upG0, f0 = upF0, gd0 = sw.diag, hprev0 = A::splat(0);
    V g_up1 = upG1, f1 = upF1, gd1 = upG0, hprev1 = A::splat(0);
#pragma unroll
    for (int t = 0; t <= R; ++t) {
        if (t < R) {  // column j0, row t
            const int r = t;
            if (r % A::EPV == 0) A::template load_chunk<R, G>(prof_a, prof_b, a0, b0, lane, r / A::EPV, p0a, p0b);
            sw.E[r] = A::addmax(sw.E[r], negge, sw.Gp[r]);
            f0 = A::addmax(f0, negge, g_up0);
            const V d = A::diag(gd0, p0a[r % A::EPV], p0b[r % A::EPV]);
            const V h = A::vmax3_relu(d, sw.E[r], f0);
            const V g = A::vadd(h, neggo);
            gd0 = sw.Gp[r];
            sw.Gp[r] = g;
            g_up0 = g;
            if (r & 1)
                best = A::vmax3(best, hprev0, g);
            else
                hprev0 = g;
        }
        if (t >= 1) {  // column j1, row t - 1
            const int r = t - 1;
            if (r % A::EPV == 0) A::template load_chunk<R, G>(prof_a, prof_b, a1, b1, lane, r / A::EPV, p1a, p1b);
            sw.E[r] = A::addmax(sw.E[r], negge, sw.Gp[r]);
            f1 = A::addmax(f1, negge, g_up1);
            const V d = A::diag(gd1, p1a[r % A::EPV], p1b[r % A::EPV]);
            const V h = A::vmax3_relu(d, sw.E[r], f1);
            const V g = A::vadd(h, neggo);
            gd1 = sw.Gp[r];
            sw.Gp[r] = g;
            g_up1 = g;
            if (r & 1)
                best = A::vmax3(best, hprev1, g);
            else
                hprev1 = g;
        }
    }
    if (R & 1) best = A::vmax3(best, hprev0, hprev1);
    sw.botG[0] = g_up0;
    sw.botF[0] = f0;
    sw.botG[1] = g_up1;
    sw.botF[1] = f1;
}

// Step s of one lane (see above). The residue codes of columns j0, j1 come as one 32-bit word
// (`codes`) and, for lane 0 after the first pass, the boundary values of both columns as one
// 16-byte word (`up`: G, F of j0, then of j1). CHECKED steps test each column against [1, w].
template <class A, int G, int R, bool CHECKED>
__device__ __forceinline__ void sweep2_step(Sweep2<A, R> &sw, const int s, const int lane, const int32_t w,
                                            const uint8_t *prof_a, const uint8_t *prof_b,
                                            const bool first_pass, const bool last_pass,
                                            typename A::V *bnd, const SweepConst<A> &k,
                                            typename A::V &best, const uint32_t codes, const uint4 up) {
    typedef typename A::V V;
    constexpr int CODE_BITS = TwoCodes<A>::BITS;
    constexpr uint32_t CODE_MASK = (1u << CODE_BITS) - 1u;
    const int32_t j0 = 2 * (s - lane) + 1;
    V upG0 = __shfl_up_sync(0xffffffffu, sw.botG[0], 1, G);
    V upF0 = __shfl_up_sync(0xffffffffu, sw.botF[0], 1, G);
    V upG1 = __shfl_up_sync(0xffffffffu, sw.botG[1], 1, G);
    V upF1 = __shfl_up_sync(0xffffffffu, sw.botF[1], 1, G);
    const bool live0 = !CHECKED || (j0 >= 1 && j0 <= w);
    const bool live1 = !CHECKED || (j0 + 1 >= 1 && j0 + 1 <= w);
    if (lane == 0) {
        if (first_pass) {
            upG0 = upG1 = k.top_free_g;
            upF0 = upF1 = k.Sv;
        } else {
            upG0 = up.x;
            upF0 = up.y;
            upG1 = up.z;
            upF1 = up.w;
        }
    }
    int a, b;
    if (!CHECKED) {
        // Both columns live: interleaved (measured 0.6% faster than one after the other).
        int a1, b1;
        A::residues((typename A::RES)(codes & CODE_MASK), a, b);
        A::residues((typename A::RES)(codes >> CODE_BITS), a1, b1);
        sweep2_both<A, G, R>(sw, a, b, a1, b1, lane, prof_a, prof_b, upG0, upF0, upG1, upF1, k.negge, k.neggo,
                             best);
    } else {
        if (live0) {
            A::residues((typename A::RES)(codes & CODE_MASK), a, b);
            sweep2_column<A, G, R>(sw, a, b, lane, prof_a, prof_b, upG0, upF0, sw.diag, k.negge, k.neggo, best,
                                   sw.botG[0], sw.botF[0]);
        }
        if (live1) {
            A::residues((typename A::RES)(codes >> CODE_BITS), a, b);
            sweep2_column<A, G, R>(sw, a, b, lane, prof_a, prof_b, upG1, upF1, upG0, k.negge, k.neggo, best,
                                   sw.botG[1], sw.botF[1]);
        }
    }
    if (live0) sw.diag = live1 ? upG1 : upG0;
    if (lane == G - 1 && !last_pass && live0)
        *reinterpret_cast<uint4 *>(bnd + 2 * (j0 - 1)) = make_uint4(sw.botG[0], sw.botF[0], sw.botG[1], sw.botF[1]);
}

// Every pass of one item's two-column sweep, the passes back to back. With W column pairs a pass
// (warp-uniform), lane L works virtual column pair v = s - L at step s, that is pass v / W at
// column pair v % W: when lane 0 has finished a pass it starts the next one while lanes 1..G-1
// finish theirs, so the G - 1 fill and drain steps of the wavefront are paid once per item, not
// once per pass. A pass p >= 1 begins with G - 1 transition steps (lanes L <= t at column pair
// t - L of pass p, the others at W + t - L of pass p - 1), then its interior steps (every lane in
// pass p; the ones with both columns of every lane inside its item run unchecked, with the next
// step's codes and boundary values loaded one step ahead).
//
// Shared memory: pass p's profile slice is in buffer p % 2. After the transition into pass p no
// lane of the block reads pass p - 1's slice any more: the block barrier there (one per pass, in
// every warp) frees that buffer for pass p + 1's copy, issued by thread 0. The boundary row: lane
// G-1 writes column pair c of pass p at step pW + c + G - 1, lane 0 reads it for pass p + 1 at
// step (p + 1)W + c (one step earlier with the prefetch). W >= 2G keeps every such read at least G
// steps after its write; the warp barrier at the start of each transition orders the writes the
// transition's reads need, and the block barrier after it orders the rest.
//
// Every thread of the block calls it with the block's `phase` (see scan_unit). Returns false if a
// profile copy did not arrive in time (the error flag is then set and the block must stop).
template <class A, int G, int R>
__device__ __forceinline__ bool sweep2_item(const ScanParams &p, const int lane, const int W, const int wfast,
                                            const int32_t w, const typename A::RES *__restrict__ res,
                                            typename A::V *bnd, uint8_t *smem, uint64_t *bars,
                                            uint32_t &phase, const typename A::V Sv, typename A::V &best) {
    typedef typename A::V V;
    typedef typename TwoCodes<A>::W W2;
    const int n_passes = p.n_passes;
    const uint32_t hi_off = (A::TABLES - 1) * (p.pass_bytes / A::TABLES);
    SweepConst<A> k;
    k.negge = A::splat(-(int64_t)p.ge);
    k.neggo = A::splat(-(int64_t)p.go);
    k.Sv = Sv;
    k.top_free_g = A::splat(-(int64_t)p.go);
    Sweep2<A, R> sw;
    // A lane's state at the start of a pass: local mode, the left border is free (H = 0).
    auto reset = [&]() {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            sw.Gp[r] = k.top_free_g;
            sw.E[r] = Sv;
        }
        sw.diag = k.top_free_g;
    };
    reset();
    sw.botG[0] = sw.botG[1] = sw.botF[0] = sw.botF[1] = A::splat(0);
    const W2 *res2 = reinterpret_cast<const W2 *>(res);  // codes of columns (2i+1, 2i+2)
    const uint4 *bnd4 = reinterpret_cast<const uint4 *>(bnd);          // boundary of the same pair
    const uint4 none = make_uint4(0, 0, 0, 0);
    // Loads for column pair c of this lane (-1: no column; a dead pair's values are never used).
    auto codes_at = [&](int c) -> uint32_t { return (c >= 0 && 2 * c < w) ? res2[c] : 0u; };
    auto up_at = [&](int c, bool first) -> uint4 {
        return (lane == 0 && !first && c >= 0 && 2 * c < w) ? bnd4[c] : none;
    };
    // One checked step of this lane at column pair c of pass lp (lp < 0 or c < 0: no column).
    auto checked = [&](int lp, int c) {
        const uint8_t *pa = smem + (size_t)(lp & 1) * p.pass_bytes;
        if (lp < 0) c = -1;
        sweep2_step<A, G, R, true>(sw, c + lane, lane, w, pa, pa + hi_off, lp == 0, lp == n_passes - 1, bnd, k,
                                   best, codes_at(c), up_at(c, lp == 0));
    };
    for (int pass = 0; pass < n_passes; ++pass) {
        const int buf = pass & 1;
        const bool ok = mbar_wait_bounded(&bars[buf], (phase >> buf) & 1u, p.wait_polls);
        phase ^= 1u << buf;
        if (W > 0) {
            __syncwarp();
            for (int t = 0; t < G - 1; ++t) {
                const bool fresh = lane <= t;  // this lane has entered pass `pass`
                if (fresh && lane == t && pass > 0) reset();
                checked(fresh ? pass : pass - 1, fresh ? t - lane : W + t - lane);
            }
            if (lane == G - 1 && pass > 0) reset();  // lane G-1 enters at the first interior step
        }
        if (__syncthreads_or(!ok)) {
            // This pass's copy and, in the first pass, the second one are still outstanding.
            if (threadIdx.x == 0)
                wait_gave_up(p.err, bars, (1u << buf) | (pass == 0 && n_passes > 1 ? 2u : 0u), phase ^ (1u << buf));
            return false;
        }
        if (threadIdx.x == 0 && pass >= 1 && pass + 1 < n_passes)
            bulk_load(smem + (size_t)(buf ^ 1) * p.pass_bytes, p.profile + (size_t)(pass + 1) * p.pass_bytes,
                      p.pass_bytes, &bars[buf ^ 1]);
        if (W == 0) continue;
        const uint8_t *pa = smem + (size_t)buf * p.pass_bytes, *pb = pa + hi_off;
        const bool first = pass == 0, last = pass == n_passes - 1;
        const int fast_hi = max(G - 1, wfast);
        if (G - 1 < fast_hi) {
            // Two steps an iteration with two sets of registers for the one-step-ahead loads (only
            // lane 0 reads the boundary row: the other lanes' copies are never used).
            const bool up_lane = lane == 0 && !first;
            uint32_t c_a = res2[G - 1 - lane], c_b = 0;
            uint4 u_a = none, u_b = none;
            if (up_lane) u_a = bnd4[G - 1];
            int s = G - 1;
            for (; s + 1 < fast_hi; s += 2) {
                c_b = res2[s + 1 - lane];
                if (up_lane) u_b = bnd4[s + 1];
                sweep2_step<A, G, R, false>(sw, s, lane, w, pa, pb, first, last, bnd, k, best, c_a, u_a);
                const int s2 = min(s + 2, fast_hi - 1);
                c_a = res2[s2 - lane];
                if (up_lane) u_a = bnd4[s2];
                sweep2_step<A, G, R, false>(sw, s + 1, lane, w, pa, pb, first, last, bnd, k, best, c_b, u_b);
            }
            if (s < fast_hi)
                sweep2_step<A, G, R, false>(sw, s, lane, w, pa, pb, first, last, bnd, k, best, c_a, u_a);
        }
        for (int s = fast_hi; s < W; ++s) checked(pass, s - lane);
    }
    // The last pass's drain: lanes L > t finish their columns W + t - L.
    if (W > 0)
        for (int t = 0; t < G - 1; ++t) checked(lane > t ? n_passes - 1 : -1, W + t - lane);
    __syncthreads();  // both profile buffers are free for the block's next unit
    return true;
}

// Group reduction of the per-lane candidates, border seeds, output and best-key fold. Every lane
// of the warp must call it (it shuffles).
template <class A, int G, int MODE, bool ENDS>
__device__ __forceinline__ void finish_item(const int lane, const bool active, const ItemMeta &meta,
                                            const int32_t qlen, const int32_t go, const int32_t ge,
                                            const typename A::V best, Cand (&cand)[2],
                                            int32_t *scores, int32_t *qend, int32_t *tend,
                                            unsigned long long *best_key) {
    typedef ModeFlags<MODE> Fl;
    if (Fl::local && !ENDS) {
#pragma unroll
        for (int h = 0; h < A::NH; ++h) cand[h].s = A::get(best, h) + go;  // best is kept in G
    }
#pragma unroll
    for (int h = 0; h < A::NH; ++h) {
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) {
            Cand o;
            o.s = __shfl_xor_sync(0xffffffffu, cand[h].s, off, G);
            o.col = __shfl_xor_sync(0xffffffffu, cand[h].col, off, G);
            o.row = __shfl_xor_sync(0xffffffffu, cand[h].row, off, G);
            if (Fl::local && !ENDS) {
                if (o.s > cand[h].s) cand[h] = o;
            } else if (better(o, cand[h])) {
                cand[h] = o;
            }
        }
    }
    unsigned long long key = 0;
    if (active && lane == 0) {
#pragma unroll
        for (int h = 0; h < A::NH; ++h) {
            const uint32_t idx = meta.idx[h];
            if (idx == NO_INDEX) continue;
            Cand c = border_seed<MODE>(qlen, (int32_t)meta.n[h], go, ge);
            if (Fl::local && !ENDS) {
                if (cand[h].s > c.s) c.s = cand[h].s;
            } else if (better(cand[h], c)) {
                c = cand[h];
            }
            if (scores) scores[idx] = c.s;
            if (ENDS) {
                qend[idx] = c.row - 1;
                tend[idx] = c.col - 1;
            }
            const unsigned long long k = hit_key(c.s, idx);
            key = k > key ? k : key;
        }
    }
    if (best_key) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            unsigned long long o = __shfl_xor_sync(0xffffffffu, key, off);
            key = o > key ? o : key;
        }
        if ((threadIdx.x & 31) == 0 && key != 0) atomicMax(best_key, key);
    }
}

// Whether a scan launch shape runs the two-column sweep: SW scores of int16x2 pairs or int32 items
// with at most 16 rows per lane. Measured on the protein benchmark: for the pairs as fast as one
// column of 32 rows, with half the per-lane state and 10% faster on 64-residue DNA queries; for the
// int32 items of a 5000-residue query 1014 against 594 GCUPS (two independent column chains per
// lane for their latency-bound warps).
template <class A, int R, int MODE, bool ENDS, bool GPROF>
__host__ __device__ constexpr bool two_col_form() {
    return TwoCodes<A>::OK && ModeFlags<MODE>::local && !ENDS && !GPROF && R <= 16;
}

#ifdef HY_BOUNDS
// The bounds-checked build: before an item is used, every index its metadata and residue codes
// can produce is checked against the extents in `p` (residue columns, boundary region, db
// indices, profile letters). All G lanes of a group call it for their group's item (`active`:
// the group has one); returns whether the item may be swept.
template <class A, int G>
__device__ bool item_in_bounds(const ScanParams &p, const ItemMeta &m, const int lane, const bool active) {
    bool ok = true;
    if (active) {
        ok = m.col_off + m.w <= p.res_cols && m.n[0] <= m.w && m.n[1] <= m.w &&
             (m.idx[0] == NO_INDEX || m.idx[0] < p.n_seqs) && (m.idx[1] == NO_INDEX || m.idx[1] < p.n_seqs) &&
             (A::NH == 2 || m.idx[1] == NO_INDEX) &&
             (p.n_passes <= 1 || (m.col_off >= p.bnd_col0 && m.col_off - p.bnd_col0 + m.w <= p.bnd_cols));
        if (ok) {
            const typename A::RES *res = reinterpret_cast<const typename A::RES *>(p.res) + m.col_off;
            for (uint32_t j = lane; j < m.w; j += G) {
                int a, b;
                A::residues(res[j], a, b);
                if ((uint32_t)a >= p.letters || (uint32_t)b >= p.letters) ok = false;
            }
        }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) ok &= __shfl_xor_sync(0xffffffffu, (int)ok, off, G) != 0;
    return ok;
}
#endif

// ---- the database scan kernel ---------------------------------------------------------------
//
// All groups of a block step through the passes together: the pass's query profile is one
// contiguous slice, brought into shared memory by a TMA bulk copy while the previous pass runs.

// Initialise the block's two profile mbarriers (thread 0; the caller synchronises the block).
__device__ __forceinline__ void init_profile_bars(uint64_t *bars) {
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
}

// One unit of work for one block: group g of the block runs item `item_first + g` if that is
// below `item_end`, through every pass of the query in `p`. The block's two profile buffers and
// mbarriers live in `smem` / `bars`; `phase` holds the parity each barrier waits for next (bit b
// for barrier b) and is carried from unit to unit by a persistent caller. Every thread of the
// block must call it with the same arguments. Returns false if a profile copy did not arrive in
// time (the error flag is then set and the block must stop). With GPROF the lanes read the pass
// slices straight from the profile in global memory (through L1) instead of shared memory: the
// form for alphabets whose slices do not fit in shared memory; `smem` and `bars` are then unused.
template <class A, int G, int R, int MODE, bool ENDS, bool GPROF = false>
__device__ __forceinline__ bool scan_unit(const ScanParams &p, const uint32_t item_first,
                                          const uint32_t item_end, uint8_t *smem, uint64_t *bars,
                                          uint32_t &phase) {
    typedef typename A::V V;
    constexpr int RPP = G * R;
    static_assert(R % A::EPV == 0, "rows per lane must fill whole profile vectors");
    static_assert(32 % G == 0, "groups must tile a warp");
    const uint8_t *prof_buf[2] = {smem, smem + p.pass_bytes};

    const int lane = threadIdx.x % G;
    const uint32_t item = item_first == NO_INDEX ? NO_INDEX : item_first + threadIdx.x / G;
    bool active = item != NO_INDEX && item < item_end;
    ItemMeta meta;
    if (active) meta = p.meta[item];
#ifdef HY_BOUNDS
    if (!item_in_bounds<A, G>(p, meta, lane, active)) {
        if (lane == 0) atomicExch(p.err, ERR_BOUNDS);
        active = false;
    }
#endif
    if (!active) {
        meta.col_off = p.bnd_col0;
        meta.w = 0;
        meta.n[0] = meta.n[1] = 0;
        meta.idx[0] = meta.idx[1] = NO_INDEX;
    }
    const V Sv = A::splat(p.sentinel);
    const typename A::RES *res = reinterpret_cast<const typename A::RES *>(p.res) + meta.col_off;
    V *bnd = reinterpret_cast<V *>(p.boundary) + 2 * (meta.col_off - p.bnd_col0);
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, meta.w);
    const int w_min = (int)__reduce_min_sync(0xffffffffu, meta.w);
    const int steps = wmax == 0 ? 0 : (int)wmax + G - 1;

    V best = A::splat(ModeFlags<MODE>::local && !ENDS ? -(int64_t)p.go : 0);
    Cand cand[2] = {{INT32_MIN, INT32_MAX, INT32_MAX}, {INT32_MIN, INT32_MAX, INT32_MAX}};

    if (!GPROF && threadIdx.x == 0 && p.n_passes > 0) {
        bulk_load(smem, p.profile, p.pass_bytes, &bars[0]);
        if (p.n_passes > 1) bulk_load(smem + p.pass_bytes, p.profile + p.pass_bytes, p.pass_bytes, &bars[1]);
    }
    if constexpr (two_col_form<A, R, MODE, ENDS, GPROF>()) {
        // Column pairs a pass: at least 2G (the boundary row's read-after-write distance).
        const int W = wmax == 0 ? 0 : max((int)(wmax + 1) / 2, 2 * G);
        if (!sweep2_item<A, G, R>(p, lane, W, min(W, w_min / 2), (int32_t)meta.w, res, bnd, smem, bars, phase, Sv,
                                  best))
            return false;
    } else {
        for (int pass = 0; pass < p.n_passes; ++pass) {
            const int buf = pass & 1;
            const uint8_t *prof;
            if (GPROF) {
                prof = p.profile + (size_t)pass * p.pass_bytes;
            } else {
                const bool ok = mbar_wait_bounded(&bars[buf], (phase >> buf) & 1u, p.wait_polls);
                phase ^= 1u << buf;
                if (__syncthreads_or(!ok)) {
                    // This pass's copy and, if issued, the next pass's are still outstanding.
                    if (threadIdx.x == 0)
                        wait_gave_up(p.err, bars, (1u << buf) | (pass + 1 < p.n_passes ? 1u << (buf ^ 1) : 0u),
                                     phase ^ (1u << buf));
                    return false;
                }
                prof = prof_buf[buf];
            }
            sweep_pass<A, G, R, MODE, ENDS>(lane, steps, w_min, (int32_t)meta.w, meta.n, res, prof,
                                            prof + (A::TABLES - 1) * (p.pass_bytes / A::TABLES),
                                            p.vrow0 + pass * RPP + lane * R, pass == 0, pass == p.n_passes - 1,
                                            bnd, p.qlen, p.go, p.ge, Sv, best, cand);
            __syncthreads();  // the profile buffer and boundary row are free again
            if (!GPROF && threadIdx.x == 0 && pass + 2 < p.n_passes)
                bulk_load(smem + (size_t)buf * p.pass_bytes, p.profile + (size_t)(pass + 2) * p.pass_bytes,
                          p.pass_bytes, &bars[buf]);
        }
    }
    finish_item<A, G, MODE, ENDS>(lane, active, meta, p.qlen, p.go, p.ge, best, cand, p.scores,
                                  p.qend, p.tend, p.best_key);
    return true;
}

// Resident 256-thread blocks per SM each launch shape is compiled for (its register budget).
// The two-column sweep of 16 rows per lane is compiled for two blocks (measured faster than three
// with the spills three would need).
template <class A, int G, int R, bool TWO_COL = false>
constexpr int scan_min_blocks() {
    return A::NH == 1 ? 2 : (G == 8 && R == 8) ? 4 : (G == 8 && R == 32) ? 2 : (TWO_COL && R == 16) ? 2 : 3;
}

template <class A, int G, int R, int MODE, bool ENDS, bool GPROF = false>
__global__ void __launch_bounds__(256, (scan_min_blocks<A, G, R, two_col_form<A, R, MODE, ENDS, GPROF>()>()))
    scan_kernel(const ScanParams p) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + (GPROF ? 0 : 2 * (size_t)p.pass_bytes));
    const int gpb = blockDim.x / G;
    uint32_t first, end;
    if (p.item_ptr) {
        // One item, run by group 0 of block 0.
        const uint32_t want = *p.item_ptr;
        first = blockIdx.x == 0 ? want : NO_INDEX;
        end = (first == NO_INDEX || first >= p.n_items) ? first : first + 1;
    } else {
        first = p.item_base + blockIdx.x * gpb;
        end = p.n_items;
    }
    init_profile_bars(bars);
    __syncthreads();
    uint32_t phase = 0;
    scan_unit<A, G, R, MODE, ENDS, GPROF>(p, first, end, smem, bars, phase);
}

// ---- the block-cooperative band kernel (one long item, with end positions) -------------------
//
// Recovers the end positions of a single item (the winner of a scan) with a whole block. Every
// warp is one 32-lane group running one pass (a band of 32*R query rows); the block takes the
// passes in rounds of W = blockDim/32. Inside a round warp w runs BAND_K*2*w steps behind warp w-1
// with a block barrier every BAND_K steps, so each boundary-row column a band reads was written
// by the band above in an earlier window (the write of column j happens 2*BAND_K - (G - 1) >
// BAND_K steps before the read). The round's profile slices are staged by one TMA bulk copy.
constexpr int BAND_K = 32;

// The band recovery of item `item` (a valid item of p.meta) by the whole block, or by every block
// of a thread-block cluster: the cluster's warps take the passes in rounds of W * (blocks), block
// b's warps the passes b * W .. b * W + W - 1 of a round, and a cluster barrier takes the place of
// the block barrier between windows (it orders the boundary-row writes of one block's warps before
// the next block's reads). `bar` is an initialised mbarrier whose next wait parity is `phase`; the
// block's dynamic shared memory (`smem`) holds W = blockDim/32 pass slices. Every thread of every
// block must call it. With GPROF (single blocks only) the warps read their pass slices from the
// profile in global memory; `smem` and `bar` are then unused.
template <class A, int R, int MODE, bool GPROF = false>
__device__ __forceinline__ void band_item(const ScanParams &p, const uint32_t item, uint8_t *smem,
                                          uint64_t *bar, uint32_t &phase) {
    typedef typename A::V V;
    constexpr int G = 32;
    constexpr int RPP = G * R;
    static_assert(BAND_K >= G, "the lag must cover the lane skew of a warp");
    static_assert(R % A::EPV == 0, "rows per lane must fill whole profile vectors");
    const int W = blockDim.x / G;
    const int warp = threadIdx.x / G, lane = threadIdx.x % G;
    const int crank = cluster_rank(), csize = cluster_size();
    const int WT = W * csize;          // warps of the cluster
    const int gw = crank * W + warp;   // this warp's index in the cluster
    __shared__ uint32_t s_flag;
    const ItemMeta meta = p.meta[item];
#ifdef HY_BOUNDS
    // Every warp checks the item (the same answer in all of them), so all skip it together.
    if (!item_in_bounds<A, G>(p, meta, lane, true)) {
        if (threadIdx.x == 0) atomicExch(p.err, ERR_BOUNDS);
        return;
    }
#endif
    const int32_t w = (int32_t)meta.w;
    const V Sv = A::splat(p.sentinel);
    const typename A::RES *res = reinterpret_cast<const typename A::RES *>(p.res) + meta.col_off;
    V *bnd = reinterpret_cast<V *>(p.boundary) + 2 * (meta.col_off - p.bnd_col0);
    V best = A::splat(0);
    Cand cand[2] = {{INT32_MIN, INT32_MAX, INT32_MAX}, {INT32_MIN, INT32_MAX, INT32_MAX}};
    const int pass_steps = w + G - 1;
    const int rounds = (p.n_passes + WT - 1) / WT;
    for (int round = 0; round < rounds; ++round) {
        const int first = round * WT;
        const int cnt = min(WT, p.n_passes - first);          // warps of the cluster with a pass
        const int bcnt = max(0, min(W, cnt - crank * W));      // ... of this block
        if (!GPROF) {
            bool fail = false;
            if (bcnt > 0) {
                if (threadIdx.x == 0)
                    bulk_load(smem, p.profile + (size_t)(first + crank * W) * p.pass_bytes,
                              (uint32_t)bcnt * p.pass_bytes, bar);
                const bool ok = mbar_wait_bounded(bar, phase & 1u, p.wait_polls);
                phase ^= 1u;
                fail = __syncthreads_or(!ok);
            }
            if (cluster_any(fail, &s_flag, csize)) {
                if (threadIdx.x == 0 && fail) wait_gave_up(p.err, bar, 1u, phase ^ 1u);  // the round's copy
                return;
            }
        }
        const int pass = first + gw;
        const bool mine = gw < cnt && w > 0;
        const int32_t row0 = p.vrow0 + pass * RPP + lane * R;
        const uint8_t *prof = GPROF ? p.profile + (size_t)min(pass, p.n_passes - 1) * p.pass_bytes
                                    : smem + (size_t)warp * p.pass_bytes;
        const uint8_t *prof_hi = prof + (A::TABLES - 1) * (p.pass_bytes / A::TABLES);
        Sweep<A, R> sw;
        sweep_begin<A, R, MODE>(sw, row0, p.go, p.ge, Sv);
        const int lag = 2 * BAND_K * gw;
        const int total = pass_steps + 2 * BAND_K * (cnt - 1);
        for (int t0 = 0; t0 < total; t0 += BAND_K) {
            const int s0 = max(t0 - lag, 0), s1 = min(t0 + BAND_K - lag, pass_steps);
            if (mine && s0 < s1)
                sweep_run<A, G, R, MODE, true>(sw, s0, s1, w, lane, w, meta.n, res, prof, prof_hi, row0,
                                               pass == 0, pass == p.n_passes - 1, bnd, p.qlen, p.go,
                                               p.ge, Sv, best, cand);
            band_sync(csize);
        }
        if (mine) sweep_end<A, R, MODE, true>(sw, row0, p.go, cand);
        __syncthreads();  // the slices may be restaged for the next round
    }
    // Reduce every lane's candidates: inside each warp, then across warps in shared memory.
    __shared__ Cand s_cand[32][2];
    __syncthreads();  // a previous item's reduction may still be reading s_cand
#pragma unroll
    for (int h = 0; h < A::NH; ++h) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            Cand o;
            o.s = __shfl_xor_sync(0xffffffffu, cand[h].s, off);
            o.col = __shfl_xor_sync(0xffffffffu, cand[h].col, off);
            o.row = __shfl_xor_sync(0xffffffffu, cand[h].row, off);
            if (better(o, cand[h])) cand[h] = o;
        }
        if (lane == 0) s_cand[warp][h] = cand[h];
    }
    band_sync(csize);  // every block's candidates are in its shared memory
    if (threadIdx.x == 0 && crank == 0) {
        for (int h = 0; h < A::NH; ++h) {
            const uint32_t idx = meta.idx[h];
            if (idx == NO_INDEX) continue;
            Cand c = border_seed<MODE>(p.qlen, (int32_t)meta.n[h], p.go, p.ge);
            for (int b = 0; b < csize; ++b)
                for (int k = 0; k < W; ++k) {
                    Cand o = s_cand[k][h];
                    if (b > 0) {
                        o.s = (int32_t)ld_cluster_u32(&s_cand[k][h].s, b);
                        o.col = (int32_t)ld_cluster_u32(&s_cand[k][h].col, b);
                        o.row = (int32_t)ld_cluster_u32(&s_cand[k][h].row, b);
                    }
                    if (better(o, c)) c = o;
                }
            if (p.ends_out) {
                if (idx == ~(uint32_t)(*p.best_key & 0xffffffffu)) {
                    p.ends_out[0] = c.s;
                    p.ends_out[1] = c.row - 1;
                    p.ends_out[2] = c.col - 1;
                }
            } else {
                p.scores[idx] = c.s;
                p.qend[idx] = c.row - 1;
                p.tend[idx] = c.col - 1;
            }
        }
    }
    if (csize > 1) cluster_barrier();  // block 0 has read every block's candidates
}

template <class A, int R, int MODE, bool GPROF = false>
__global__ void __launch_bounds__(1024) band_kernel(const ScanParams p) {
    extern __shared__ __align__(128) uint8_t smem[];
    const uint32_t item = *p.item_ptr;
    if (item == NO_INDEX || item >= p.n_items) return;  // the same for every thread of the block
    const int W = blockDim.x / 32;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + (GPROF ? 0 : (size_t)W * p.pass_bytes));
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    band_item<A, R, MODE, GPROF>(p, item, smem, bar, phase);
}

// ---- the batched pairwise kernel (align_pairs) -----------------------------------------------
//
// Every item carries its own queries (one per half, of equal length), so each group builds the
// profile slice of its own pass in its own region of shared memory, then sweeps it. Groups of a
// warp run their items' passes in step; there is no block-wide synchronisation.
struct PairParams {
    const ItemMeta *meta;  // n[h]: target lengths; idx[h]: pair indices
    const uint32_t *qlen;  // per item
    const uint64_t *qoff;  // per item and half: offset of the query residues in q_res
    uint32_t item_base;    // items [item_base, n_items) run
    uint32_t n_items;
    const uint8_t *q_res;
    const void *res;       // packed target residues, as in the scan
    const int32_t *matrix;
    int32_t al;
    int32_t lim;
    int32_t go, ge;
    int32_t sentinel;
    int top_free;
    uint32_t group_bytes;  // shared memory per group (both halves of one pass slice)
    void *boundary;
    int32_t *scores;
    int32_t *qend;
    int32_t *tend;
    // Global-memory-profile form (alphabets whose group profiles do not fit in shared memory):
    // group g of block b builds and reads its profile at gprof + (b * groups_per_block + g) *
    // group_bytes.
    uint8_t *gprof;
    // Column-maxima form (align_pair_position_max): pair half h of item i writes the maximum of H
    // over each target column to colmax + toff[2 * i + h] + column.
    int32_t *colmax;
    const uint64_t *toff;
};

template <class A, int G, int R>
__device__ __forceinline__ void build_group_profile(uint8_t *dst, const uint8_t *q, int32_t qlen,
                                                    int32_t row_base, const int32_t *matrix,
                                                    int32_t al, int32_t lim, int32_t go,
                                                    int top_free, int lane, int table) {
    static_assert(R % A::EPV == 0 && R >= A::EPV, "rows per lane must fill whole profile vectors");
    constexpr int KCH = R / A::EPV;
    typename A::PE *out = reinterpret_cast<typename A::PE *>(dst);
    const int64_t pad = -(int64_t)lim - 1 + go;
    for (int letter = 0; letter <= al; ++letter) {
#pragma unroll
        for (int k = 0; k < KCH; ++k) {
#pragma unroll
            for (int e = 0; e < A::EPV; ++e) {
                const int32_t row = row_base + lane * R + k * A::EPV + e;
                int64_t v;
                if (row <= 0) {
                    v = top_free ? go : 0;
                } else if (letter == al) {
                    v = pad;
                } else {
                    int64_t sub = matrix[(int32_t)q[row - 1] * al + letter];
                    if (sub < -(int64_t)lim - 1) sub = -(int64_t)lim - 1;
                    if (sub > lim) sub = lim;
                    v = sub + go;
                }
                out[(((size_t)letter * KCH + k) * G + lane) * A::EPV + e] = A::word(v, table);
            }
        }
    }
}

template <class A, int G, int R, int MODE, bool ENDS, bool GPROF = false, bool COLMAX = false>
__global__ void __launch_bounds__(256) pairs_kernel(const PairParams p) {
    typedef typename A::V V;
    constexpr int RPP = G * R;
    extern __shared__ __align__(128) uint8_t smem[];
    const int lane = threadIdx.x % G;
    const int gib = threadIdx.x / G;
    const uint32_t item = p.item_base + blockIdx.x * (blockDim.x / G) + gib;
    const bool active = item < p.n_items;
    ItemMeta meta;
    int32_t qlen = 0;
    if (active) {
        meta = p.meta[item];
        qlen = (int32_t)p.qlen[item];
    } else {
        meta.col_off = 0;
        meta.w = 0;
        meta.n[0] = meta.n[1] = 0;
        meta.idx[0] = meta.idx[1] = NO_INDEX;
    }
    const int32_t n_passes = (qlen + RPP - 1) / RPP;
    const int32_t vrow0 = qlen - n_passes * RPP + 1;
    const uint8_t *qa = active ? p.q_res + p.qoff[2 * (size_t)item] : p.q_res;
    const uint8_t *qb = (active && A::NH > 1 && meta.idx[1] != NO_INDEX) ? p.q_res + p.qoff[2 * (size_t)item + 1] : qa;
    // The group's region: the low-half table of query a, then (int16x2) the high-half table of b.
    uint8_t *gprof_a = GPROF ? p.gprof + ((size_t)blockIdx.x * (blockDim.x / G) + gib) * p.group_bytes
                             : smem + (size_t)gib * p.group_bytes;
    uint8_t *gprof_b = gprof_a + (A::TABLES - 1) * (p.group_bytes / A::TABLES);
    const V Sv = A::splat(p.sentinel);
    const typename A::RES *res = reinterpret_cast<const typename A::RES *>(p.res) + meta.col_off;
    V *bnd = reinterpret_cast<V *>(p.boundary) + 2 * meta.col_off;
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, meta.w);
    const int steps = wmax == 0 ? 0 : (int)wmax + G - 1;
    const int32_t pmax = (int32_t)__reduce_max_sync(0xffffffffu, (uint32_t)n_passes);
    ColMaxOut cmo;
    if constexpr (COLMAX) {
        cmo.p[0] = cmo.p[1] = p.colmax;
        if (active) {
            cmo.p[0] = p.colmax + p.toff[2 * (size_t)item];
            cmo.p[1] = p.colmax + p.toff[2 * (size_t)item + 1];
        }
        cmo.atomic = n_passes > 1;
    }

    V best = A::splat(ModeFlags<MODE>::local && !ENDS ? -(int64_t)p.go : 0);
    Cand cand[2] = {{INT32_MIN, INT32_MAX, INT32_MAX}, {INT32_MIN, INT32_MAX, INT32_MAX}};
    for (int pass = 0; pass < pmax; ++pass) {
        const bool mine = pass < n_passes;
        const int32_t row_base = vrow0 + pass * RPP;
        if (mine) {
            build_group_profile<A, G, R>(gprof_a, qa, qlen, row_base, p.matrix, p.al, p.lim, p.go,
                                         p.top_free, lane, 0);
            if (A::TABLES > 1)
                build_group_profile<A, G, R>(gprof_b, qb, qlen, row_base, p.matrix, p.al, p.lim,
                                             p.go, p.top_free, lane, 1);
        }
        __syncwarp();
        // `steps` stays warp-uniform; a group past its last pass sweeps zero columns.
        const int w_here = mine ? (int)meta.w : 0;
        const int w_min = (int)__reduce_min_sync(0xffffffffu, (uint32_t)w_here);
        sweep_pass<A, G, R, MODE, ENDS, COLMAX>(lane, steps, w_min, w_here, meta.n, res, gprof_a,
                                                gprof_b, row_base + lane * R, pass == 0,
                                                pass == n_passes - 1, bnd, qlen, p.go, p.ge, Sv, best,
                                                cand, COLMAX ? &cmo : nullptr);
        __syncwarp();
    }
    if constexpr (!COLMAX)
        finish_item<A, G, MODE, ENDS>(lane, active, meta, qlen, p.go, p.ge, best, cand, p.scores,
                                      p.qend, p.tend, nullptr);
}

// ---- query profile ----------------------------------------------------------------------------
//
// Layout of one pass slice: [table < TABLES][letter 0..al][chunk k < R/EPV][lane < G][EPV words],
// word e of chunk k of lane L being grid row vrow0 + pass*G*R + L*R + k*EPV + e. Letter `al` is the
// padding symbol. Values are P = clamp(sub, -(lim+1), lim) + go; virtual rows (<= 0) get go (free
// top border) or 0 (penalised top border); the padding symbol gets -(lim+1) + go. For int16x2 the
// first table holds each value in the low half of its word, the second in the high half.
// Words [first, total) in steps of `stride` of the profile described above.
template <class A, int G, int R>
__device__ __forceinline__ void build_profile_words(const uint8_t *q, const int32_t *matrix,
                                                    int32_t al, int32_t go, int32_t lim,
                                                    int top_free, int32_t vrow0, int32_t n_passes,
                                                    typename A::PE *out, int64_t first,
                                                    int64_t stride) {
    static_assert(R % A::EPV == 0 && R >= A::EPV, "rows per lane must fill whole profile vectors");
    constexpr int KCH = R / A::EPV;
    const int64_t per_table = A::letters(al) * G * R;
    const int64_t per_pass = per_table * A::TABLES;
    const int64_t total = per_pass * n_passes;
    for (int64_t i = first; i < total; i += stride) {
        const int64_t pass = i / per_pass;
        const int table = (int)((i % per_pass) / per_table);
        int64_t rem = i % per_table;
        const int e = (int)(rem % A::EPV);
        rem /= A::EPV;
        const int lane = (int)(rem % G);
        rem /= G;
        const int k = (int)(rem % KCH);
        const int letter = (int)(rem / KCH);
        const int64_t row = vrow0 + pass * (G * R) + (int64_t)lane * R + k * A::EPV + e;
        const int64_t pad = -(int64_t)lim - 1 + go;
        // Profile value of target symbol l at this row.
        auto value = [&](int l) -> int64_t {
            if (row <= 0) return top_free ? go : 0;
            if (l == al) return pad;
            int64_t sub = matrix[(int64_t)q[row - 1] * al + l];
            if (sub < -(int64_t)lim - 1) sub = -(int64_t)lim - 1;
            if (sub > lim) sub = lim;
            return sub + go;
        };
        if constexpr (A::PAIRTAB)
            out[i] = A::pair_word(value(letter / (al + 1)), value(letter % (al + 1)));
        else
            out[i] = A::word(value(letter), table);
    }
}

template <class A, int G, int R>
__global__ void build_profile_kernel(const uint8_t *q, int32_t qlen, const int32_t *matrix,
                                     int32_t al, int32_t go, int32_t lim, int top_free,
                                     int32_t vrow0, int32_t n_passes, typename A::PE *out) {
    (void)qlen;
    build_profile_words<A, G, R>(q, matrix, al, go, lim, top_free, vrow0, n_passes, out,
                                 blockIdx.x * (int64_t)blockDim.x + threadIdx.x,
                                 (int64_t)gridDim.x * blockDim.x);
}

}  // namespace hy
