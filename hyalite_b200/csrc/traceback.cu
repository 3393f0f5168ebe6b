// traceback.cu -- the Alignment search type on the device: align (src/align.rs:169-222),
// Database::scan_aligned and Database::scan_all_aligned (src/database.rs:527-549).
//
// The reference recovers an alignment with a scalar full-matrix DP that keeps H, E and F as three
// i32 matrices (12 bytes a cell) and walks back through their values (src/align.rs:345-545). Every
// decision of that walk is a comparison between values of one cell and its left, upper or diagonal
// neighbour, so the device instead records, per cell, the four outcomes the walk can ask for in
// one 4-bit code while the DP runs, and walks the codes:
//
//   bits 0-1  which state H(i,j) came from: 0 diagonal (H == H(i-1,j-1) + sub), 1 E (H == E),
//             2 F; the walk's H-state rule, tie-break included
//   bit 2     E(i,j) != H(i,j-1) - gap_open  (the E state extends; clear: back to H)
//   bit 3     F(i,j) != H(i-1,j) - gap_open  (the F state extends; clear: back to H)
//
// The local-mode stop (H == 0) needs no bits: the walk carries the value of the cell it stands on,
// from the end cell's score back through each operation (a diagonal step subtracts the
// substitution score, a gap step adds gap_ext while the run extends and gap_open where it opens),
// and stops where that value is 0. Half a byte a cell instead of twelve, written once and read only
// along the path. Cell values
// are int32 with the reference's arithmetic (its width proof keeps every real cell exact), so each
// code equals the outcome of the reference's comparison and the walk emits the same operations.
//
// Fill kernel: one warp per (query, target) pair, each lane R consecutive query rows, lanes
// skewed one column apart (anti-diagonal wavefront); passes of 32 * R rows joined by a boundary
// row (H and F) in global memory. Codes are stored step-major per lane: the R/2 bytes a lane
// writes at consecutive steps are contiguous, so the walk's diagonal and leftward moves inside a
// lane's rows stay within one cache line for many steps (the L2 merges the lanes' 8-byte stores
// into full sectors before they reach DRAM).
// The fill also reduces the end cell (Best::consider, src/align.rs:281-327) over the mode's answer
// region. Walk kernel: one thread per pair follows the codes from the end cell, writing the
// operations backwards into a slot of m + n bytes; a scan and a gather compact the slots.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <mutex>
#include <vector>

#include "db_internal.h"
#include "host_common.h"
#include "scan_kernel.cuh"
#include "traceback_internal.h"
#include "host_threads.h"

namespace hy {

constexpr int TB_BLOCK = 256;
constexpr int32_t TB_NEG = INT32_MIN / 4;  // kernel::NEG (src/kernel.rs:39)
// Code bytes one launch chunk may hold before the pairs are split over several chunks (a single
// pair larger than this gets a chunk of its own).
constexpr uint64_t TB_CHUNK_BYTES = 2ull << 30;

// One (query, target) pair of a launch.
struct TbPair {
    uint64_t q_off;     // query residues in q_res
    uint64_t prof_off;  // int32 elements: the query's profile, letter-major, m_pad rows a letter
    uint64_t t_off;     // target residues in t_res
    uint64_t dir_off;   // code bytes
    uint64_t bnd_off;   // int2 elements: the boundary row, n + 1 entries
    uint64_t ops_off;   // operation slot of m + n bytes
    uint64_t ends_off;  // end-cell candidates: n_ends of them (one per stripe, or one)
    uint32_t m, n, m_pad, slot;  // lengths, profile row stride, result index within the launch
    uint32_t rows;               // query rows per lane (R) of the fill
    uint32_t n_ends;
};

// Interior end-cell candidate of a pair: the best answer-region cell with i, j >= 1.
struct TbEnd {
    int32_t score;
    uint32_t row, col, valid;
};

struct TbParams {
    const TbPair *pairs;
    uint32_t n_pairs;
    const uint8_t *q_res;
    const uint8_t *t_res;
    const int32_t *prof;
    uint8_t *dir;
    int2 *bnd;
    TbEnd *ends;
    hy_alignment *out;
    uint8_t *ops;
    uint8_t *ops_out;
    uint64_t *total;
    int32_t *colmax;  // TB_COLMAX: per pair at TbPair::ops_off, n entries, zeroed before the launch
    const int32_t *matrix;  // the walk (local mode): substitution scores, al x al
    uint32_t al;
    int32_t go, ge;
};

__host__ __device__ inline int64_t tb_gap(int32_t go, int32_t ge, int64_t len) {
    return len == 0 ? 0 : (int64_t)go + (len - 1) * (int64_t)ge;
}

// H on the left border, H(i, 0) (src/align.rs:457-460), clamped for the padding rows below the
// query whose values are never read.
template <int MODE>
__device__ inline int32_t tb_left(int64_t i, int32_t go, int32_t ge) {
    if (ModeFlags<MODE>::left_free || i == 0) return 0;
    const int64_t v = -tb_gap(go, ge, i);
    return v < TB_NEG ? TB_NEG : (int32_t)v;
}

// Best::consider (src/align.rs:298-305): higher score, then smaller column, then smaller row.
__device__ inline bool tb_better(int32_t s, uint32_t r, uint32_t c, int32_t bs, uint32_t br, uint32_t bc) {
    return s > bs || (s == bs && (c < bc || (c == bc && r < br)));
}

template <int R>
struct TbWord;
template <>
struct TbWord<4> { using T = uint16_t; };
template <>
struct TbWord<8> { using T = uint32_t; };
template <>
struct TbWord<16> { using T = uint2; };

template <int R>
__device__ inline void tb_store(uint8_t *p, uint32_t lo, uint32_t hi) {
    if constexpr (R == 4) *(uint16_t *)p = (uint16_t)lo;
    else if constexpr (R == 8) *(uint32_t *)p = lo;
    else *(uint2 *)p = make_uint2(lo, hi);
}

// What a pass records besides the DP: nothing (score only), the walk codes, or the per-column
// maxima of H (align_pair_position_max; local mode, score only).
enum { TB_SCORE = 0, TB_CODES = 1, TB_COLMAX = 2 };

// Boundary rows of one pass. `in` is the row above the pass (H and F, n + 1 entries; null: row 0,
// computed), `out` the pass's last row for the next pass (null: none). Between the warps of the
// stripe kernel, `in_prog` / `out_prog` count the published columns of those rows.
struct TbRows {
    const int2 *in;
    int2 *out;
    const uint32_t *in_prog;
    uint32_t *out_prog;
    int *err;
    uint32_t spin;  // polls a wait on in_prog makes before it gives up
};

constexpr uint32_t TB_PUBLISH = 32;        // columns between two progress updates of a stripe
// Rows per lane of the stripe kernel: 128-row stripes, the most warps per pair.
constexpr uint32_t TB_STRIPE_R = 4;
// Alphabets up to this size give each stripe a shared-memory copy of its profile rows (96 KB for
// a two-warp block at the limit); larger ones read the profile from global memory.
constexpr uint64_t TB_STRIPE_SMEM_AL = 96;
inline uint32_t tb_stripe_smem_al(uint64_t al) { return al <= TB_STRIPE_SMEM_AL ? (uint32_t)al : 0u; }
// Polls (about 0.25 us each) before a wait gives up: the default bound of the library's waits
// divided down to this wait's longer poll interval.
inline uint32_t tb_spin_limit() { return wait_polls() >> 2; }

// Waits until *prog >= need (acquire); after `spin` polls without it records the timeout in *err
// and stops waiting for good (the results are then discarded by the host).
__device__ inline uint32_t tb_wait(const uint32_t *prog, uint32_t need, uint32_t avail, int *err,
                                   uint32_t spin) {
    uint32_t it = 0;
    while (avail < need) {
        avail = *(const volatile uint32_t *)prog;
        if (avail >= need) break;
        if (++it > spin) {
            atomicExch(err, 1);
            return 0xffffffffu;
        }
        __nanosleep(128);
    }
    __threadfence();
    return avail;
}

// One pass of 32 * R query rows (pass p) of pair `pr` over all its columns: the DP with the walk
// codes stored, the row for the next pass, and the pass's end-cell candidates merged into
// (bs, brow, bcol) of this lane.
template <int R, int MODE, int KIND, bool XC = false>
__device__ __forceinline__ void tb_pass(const TbParams &P, const TbPair &pr, int p, int passes, int lane,
                                        const TbRows &rows, int32_t &bs, uint32_t &brow, uint32_t &bcol,
                                        const int32_t *sprof = nullptr) {
    using F = ModeFlags<MODE>;
    constexpr bool CODES = KIND == TB_CODES;
    static_assert(KIND != TB_COLMAX || MODE == MODE_SW, "column maxima are a local-mode search");
    const int m = (int)pr.m, n = (int)pr.n;
    const int32_t go = P.go, ge = P.ge;
    const uint8_t *tq = P.t_res + pr.t_off;
    const int rpp = 32 * R;
    int32_t carry_m = 0;  // TB_COLMAX: max of H over this column's rows above and in this lane
    const uint64_t pass_stride = (uint64_t)(n + 31) * 32 * (R / 2);
    const int i0 = p * rpp + lane * R + 1;  // first DP row of this lane
    int32_t Hl[R], E[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        Hl[k] = tb_left<MODE>(i0 + k, go, ge);
        E[k] = TB_NEG;
    }
    int32_t hdiag = tb_left<MODE>(i0 - 1, go, ge);  // H(i0 - 1, 0)
    int32_t carry_h = 0, carry_f = TB_NEG;
    int32_t ps = F::local ? 0 : INT32_MIN;  // this pass's best (local mode)
    uint32_t prow = 0, pcol = 0;
    const int km = m - i0;  // row m is Hl[km] when 0 <= km < R
    const bool has_m = km >= 0 && km < R;
    const int kv = min(R, m - i0 + 1);  // rows of this lane inside the query
    uint8_t *D = P.dir + pr.dir_off + (uint64_t)p * pass_stride;
    // The profile rows of this lane: from global memory, or (sprof) from the warp's shared-memory
    // copy of this pass's 32 * R rows, letter-major.
    const int32_t *pq = sprof ? sprof + lane * R : P.prof + pr.prof_off + (i0 - 1);
    const uint64_t pstride = sprof ? (uint64_t)(32 * R) : (uint64_t)pr.m_pad;
    // The row above: in place (one warp per pair), lane 0 reads it one column ahead; between
    // stripes (published by another warp), all lanes load it 32 columns at a time from L2 once
    // those columns are published, and lane 0 takes column j from lane (j - 1) % 32.
    const bool batched = rows.in_prog != nullptr;
    auto row_above = [&](int j) -> int2 {
        if (!rows.in) {
            int32_t h = 0;
            if (!F::top_free && j > 0) h = (int32_t)-tb_gap(go, ge, j);
            return make_int2(h, TB_NEG);
        }
        return rows.in[j];
    };
    uint32_t avail = 0;
    int2 nb = make_int2(0, TB_NEG), cur = make_int2(0, TB_NEG);
    if (lane == 0 && !batched) nb = row_above(1);
    // Loads run ahead of the DP: the residue two steps ahead, its profile values one step ahead.
    // Lane l works column s - l + 1 at step s.
    auto residue = [&](int s) -> int {
        const int col = s - lane + 1;
        return (col >= 1 && col <= n) ? (int)tq[col - 1] : 0;
    };
    int4 subn[R / 4];
    auto load_profile = [&](int s, int c) {
        const int col = s - lane + 1;
        if (col >= 1 && col <= n) {
            const int32_t *pc = pq + (uint64_t)c * pstride;
#pragma unroll
            for (int k = 0; k < R / 4; ++k) subn[k] = *(const int4 *)(pc + 4 * k);
        }
    };
    load_profile(0, residue(0));
    int cnext = residue(1);
    const int steps = n + 31;
    for (int s = 0; s < steps; ++s) {
        const int j = s - lane + 1;  // this lane's DP column
        if (batched && (s & 31) == 0 && s < n) {
            const uint32_t need = min((uint32_t)n, (uint32_t)s + 32);
            if (lane == 0 && need > avail) avail = tb_wait(rows.in_prog, need, avail, rows.err, rows.spin);
            __syncwarp();
            const int col = s + 1 + lane;
            cur = col <= n ? __ldcg(rows.in + col) : make_int2(0, TB_NEG);
        }
        int32_t up_h = __shfl_up_sync(0xffffffffu, carry_h, 1);
        int32_t up_f = __shfl_up_sync(0xffffffffu, carry_f, 1);
        int32_t up_m = 0;
        if constexpr (KIND == TB_COLMAX) {
            up_m = __shfl_up_sync(0xffffffffu, carry_m, 1);
            if (lane == 0) up_m = 0;
        }
        if (batched) {
            const int32_t bh = __shfl_sync(0xffffffffu, cur.x, s & 31);
            const int32_t bf = __shfl_sync(0xffffffffu, cur.y, s & 31);
            if (lane == 0) {
                up_h = bh;
                up_f = bf;
            }
        }
        if (lane == 0 && !batched) {
            up_h = nb.x;
            up_f = nb.y;
            if (j + 1 <= n) nb = row_above(j + 1);
        }
        int32_t sub[R];
#pragma unroll
        for (int k = 0; k < R / 4; ++k) {
            sub[4 * k] = subn[k].x;
            sub[4 * k + 1] = subn[k].y;
            sub[4 * k + 2] = subn[k].z;
            sub[4 * k + 3] = subn[k].w;
        }
        load_profile(s + 1, cnext);
        cnext = residue(s + 2);
        if (j >= 1 && j <= n) {
            int32_t hd = hdiag, hu = up_h, fu = up_f;
            uint32_t w0 = 0, w1 = 0;
            int32_t colmax = 0;
            int32_t xp = 0;  // XC: the previous row's x
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if constexpr (XC) {
                    // The short-chain form for lone warps (the stripe kernel), whose steps are bound
                    // by dependent latency: with x = max(d, E[, 0]) - go, H = max(x + go, F) and the
                    // next row's F = max(F - ge, x) (go >= ge), so the row-to-row chain is the one
                    // add-max on F. Every value equals the plain form's.
                    const int32_t e = __viaddmax_s32(Hl[k], -go, E[k] - ge);
                    const int32_t d = hd + sub[k];
                    const int32_t x = (F::local ? __vimax3_s32_relu(d, e, d) : max(d, e)) - go;
                    const int32_t hgp = k == 0 ? hu - go : __viaddmax_s32(fu, -go, xp);  // H(i-1,j) - go
                    const int32_t f = k == 0 ? max(hgp, fu - ge) : __viaddmax_s32(fu, -ge, xp);
                    const int32_t h = __viaddmax_s32(x, go, f);
                    if constexpr (CODES) {
                        const uint32_t e_ext = min((uint32_t)(e - Hl[k] + go), 1u);
                        const uint32_t f_ext = min((uint32_t)(f - hgp), 1u);
                        const uint32_t d_ne = min((uint32_t)(h - d), 1u);
                        const uint32_t e_ne = min((uint32_t)(h - e), 1u);
                        uint32_t code = d_ne * e_ne + d_ne;
                        code += e_ext * 4u + f_ext * 8u;
                        if (k < 8) w0 += code << (4 * k);
                        else w1 += code << (4 * (k - 8));
                    }
                    if (F::local) colmax = max(colmax, h);
                    xp = x;
                    hd = Hl[k];
                    Hl[k] = h;
                    E[k] = e;
                    hu = h;
                    fu = f;
                    continue;
                }
                if constexpr (!CODES) {
                    // Score only (the DP of src/kernel.rs:168-232).
                    const int32_t e = __viaddmax_s32(Hl[k], -go, E[k] - ge);
                    const int32_t f = __viaddmax_s32(hu, -go, fu - ge);
                    const int32_t d = hd + sub[k];
                    const int32_t h = F::local ? __vimax3_s32_relu(d, e, f) : __vimax3_s32(d, e, f);
                    if (F::local) colmax = max(colmax, h);
                    hd = Hl[k];
                    Hl[k] = h;
                    E[k] = e;
                    hu = h;
                    fu = f;
                    continue;
                }
                // The walk's comparisons as 0/1 flags, each a difference of two values that is
                // zero exactly when they are equal (the max is never below its operands), clamped
                // to 1: no selects.
                const int32_t e = __viaddmax_s32(Hl[k], -go, E[k] - ge);
                const uint32_t e_ext = min((uint32_t)(e - Hl[k] + go), 1u);  // E != H(i,j-1) - go
                const int32_t f = __viaddmax_s32(hu, -go, fu - ge);
                const uint32_t f_ext = min((uint32_t)(f - hu + go), 1u);  // F != H(i-1,j) - go
                const int32_t d = hd + sub[k];
                int32_t h = F::local ? __vimax3_s32_relu(d, e, f) : __vimax3_s32(d, e, f);
                const uint32_t d_ne = min((uint32_t)(h - d), 1u);
                const uint32_t e_ne = min((uint32_t)(h - e), 1u);
                // Source: d_ne * (1 + e_ne) is 0 diagonal, 1 E, 2 F.
                uint32_t code = d_ne * e_ne + d_ne;
                code += e_ext * 4u + f_ext * 8u;
                if (k < 8) w0 += code << (4 * k);
                else w1 += code << (4 * (k - 8));
                if (F::local) colmax = max(colmax, h);
                hd = Hl[k];
                Hl[k] = h;
                E[k] = e;
                hu = h;
                fu = f;
            }
            if constexpr (CODES) tb_store<R>(D + ((uint64_t)lane * (n + 31) + s) * (R / 2), w0, w1);
            if (lane == 31 && rows.out) {
                rows.out[j] = make_int2(hu, fu);
                if (rows.out_prog && ((uint32_t)j % TB_PUBLISH == 0 || j == n)) {
                    __threadfence();
                    atomicExch(rows.out_prog, (uint32_t)j);
                }
            }
            carry_h = hu;
            carry_f = fu;
            hdiag = up_h;
            if constexpr (KIND == TB_COLMAX) {
                // Rows below the query (the last pass) are not part of the column.
                int32_t cm = colmax;
                if (kv < R) {
                    cm = 0;
#pragma unroll
                    for (int k = 0; k < R; ++k)
                        if (k < kv) cm = max(cm, Hl[k]);
                }
                carry_m = max(up_m, cm);
                if (lane == 31) atomicMax(P.colmax + pr.ops_off + (j - 1), carry_m);
            }
            if (F::local) {
                if (colmax > ps) {
                    int kk = 0;
#pragma unroll
                    for (int k = R - 1; k >= 0; --k)
                        if (Hl[k] == colmax) kk = k;
                    ps = colmax;
                    prow = (uint32_t)(i0 + kk);
                    pcol = (uint32_t)j;
                }
            } else {
                if (F::last_col && j == n) {
#pragma unroll
                    for (int k = 0; k < R; ++k)
                        if (k < kv && tb_better(Hl[k], i0 + k, n, bs, brow, bcol)) {
                            bs = Hl[k];
                            brow = i0 + k;
                            bcol = n;
                        }
                }
                if (has_m && (F::last_row || j == n)) {
                    int32_t v = Hl[0];
#pragma unroll
                    for (int k = 1; k < R; ++k)
                        if (k == km) v = Hl[k];
                    if (tb_better(v, m, j, bs, brow, bcol)) {
                        bs = v;
                        brow = m;
                        bcol = j;
                    }
                }
            }
        }
    }
    __syncwarp();
    if (F::local && ps > 0 && tb_better(ps, prow, pcol, bs, brow, bcol)) {
        bs = ps;
        brow = prow;
        bcol = pcol;
    }
}

// Reduces the lanes' candidates under Best::consider's order; lane 0 writes the result.
template <int MODE>
__device__ inline void tb_write_end(TbEnd *dst, int lane, int32_t bs, uint32_t brow, uint32_t bcol) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int32_t os = __shfl_xor_sync(0xffffffffu, bs, o);
        const uint32_t orow = __shfl_xor_sync(0xffffffffu, brow, o);
        const uint32_t ocol = __shfl_xor_sync(0xffffffffu, bcol, o);
        if (tb_better(os, orow, ocol, bs, brow, bcol)) {
            bs = os;
            brow = orow;
            bcol = ocol;
        }
    }
    if (lane == 0) {
        const bool valid = ModeFlags<MODE>::local ? bs > 0 : bs != INT32_MIN;
        *dst = TbEnd{bs, brow, bcol, valid ? 1u : 0u};
    }
}

// Throughput form: one warp per pair, its passes in sequence, the boundary row in place.
template <int R, int MODE>
__global__ void __launch_bounds__(TB_BLOCK) tb_fill_kernel(TbParams P) {
    using F = ModeFlags<MODE>;
    const uint32_t warp = (blockIdx.x * TB_BLOCK + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= P.n_pairs) return;
    const TbPair pr = P.pairs[warp];
    const int m = (int)pr.m, n = (int)pr.n;
    if (m == 0 || n == 0) return;  // border-only problems: the walk kernel resolves them alone
    int2 *B = P.bnd + pr.bnd_off;
    // Row 0: H(0, j) (src/align.rs:500-508) and F(0, j) = NEG.
    for (int j = lane; j <= n; j += 32) {
        int32_t h = 0;
        if (!F::top_free && j > 0) h = (int32_t)-tb_gap(P.go, P.ge, j);
        B[j] = make_int2(h, TB_NEG);
    }
    __syncwarp();
    const int passes = (m + 32 * R - 1) / (32 * R);
    int32_t bs = F::local ? 0 : INT32_MIN;
    uint32_t brow = 0, bcol = 0;
    for (int p = 0; p < passes; ++p) {
        const TbRows rows{B, p + 1 < passes ? B : nullptr, nullptr, nullptr, nullptr, 0};
        tb_pass<R, MODE, TB_CODES>(P, pr, p, passes, lane, rows, bs, brow, bcol);
    }
    tb_write_end<MODE>(P.ends + pr.ends_off, lane, bs, brow, bcol);
}

// From each pair's column maxima (at its ops_off): its BestHit and, with s2, its score2
// (position_hits). One thread per pair.
__global__ void tb_position_hits_kernel(TbParams P, int32_t *scores, int32_t *tend, int32_t matrix_max,
                                        int32_t min_score, int32_t *s2) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n_pairs) return;
    const TbPair pr = P.pairs[t];
    position_hits(P.colmax + pr.ops_off, pr.n, matrix_max, min_score, scores + pr.slot, tend + pr.slot,
                  s2 ? s2 + 2 * (uint64_t)pr.slot : nullptr);
}

// Latency form for few long pairs: every pass (stripe) of every pair on its own warp, all warps
// resident at once (cooperative launch). Stripe s reads the row stripe s - 1 publishes, column by
// column, so the stripes of one pair run as a pipeline instead of in sequence. Pair x owns the
// stripes [first[x], first[x + 1]); warp w takes stripes w, w + warps, ... in increasing order,
// so each waits only on a lower stripe that is already running or done. KIND TB_SCORE runs the
// score-only DP (the long pairs of align_pairs) and records only the end-cell candidates;
// TB_COLMAX also the column maxima (a long pair of align_pair_position_max).
struct TbStripes {
    const uint32_t *first;  // per pair: first stripe (n_pairs + 1 entries)
    uint32_t n_stripes;
    uint32_t al;            // letters; > 0: each warp copies its stripe's profile rows to shared memory
    int2 *bnd;              // per pair: (stripes - 1) rows of n + 1 entries at TbPair::bnd_off
    uint32_t *prog;         // per stripe: published columns of its last row (zeroed before launch)
    int *err;
    uint32_t spin;          // polls a wait makes before it gives up
};

template <int R, int MODE, int KIND>
__global__ void __launch_bounds__(TB_BLOCK) tb_stripe_kernel(TbParams P, TbStripes S) {
    using F = ModeFlags<MODE>;
    const uint32_t warps = gridDim.x * (blockDim.x / 32);
    const int lane = threadIdx.x & 31;
    for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < S.n_stripes; g += warps) {
        uint32_t lo = 0, hi = P.n_pairs;  // the pair x with first[x] <= g < first[x + 1]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (S.first[mid] <= g) lo = mid; else hi = mid;
        }
        const uint32_t pi = lo, s = g - S.first[pi];
        const TbPair pr = P.pairs[pi];
        const int m = (int)pr.m, n = (int)pr.n;
        if (m == 0 || n == 0) continue;
        const int passes = (m + 32 * R - 1) / (32 * R);
        if ((int)s >= passes) continue;
        int2 *B = S.bnd + pr.bnd_off;
        const TbRows rows{s == 0 ? nullptr : B + (uint64_t)(s - 1) * (n + 1),
                          (int)s + 1 < passes ? B + (uint64_t)s * (n + 1) : nullptr,
                          s == 0 ? nullptr : S.prog + g - 1, S.prog + g, S.err, S.spin};
        int32_t bs = F::local ? 0 : INT32_MIN;
        uint32_t brow = 0, bcol = 0;
        // The stripe's profile rows (al letters x 32 R rows) into this warp's shared memory: every
        // step then reads its profile words at shared-memory latency.
        int32_t *sprof = nullptr;
        if (S.al) {
            extern __shared__ int32_t tb_smem[];
            sprof = tb_smem + (size_t)(threadIdx.x >> 5) * S.al * 32 * R;
            __syncwarp();
            const int32_t *src = P.prof + pr.prof_off + (uint64_t)s * 32 * R;
            for (uint32_t x = lane; x < S.al * 32 * R; x += 32) {
                const uint32_t c = x / (32 * R), r = x - c * 32 * R;
                sprof[x] = src[(uint64_t)c * pr.m_pad + r];
            }
            __syncwarp();
        }
        tb_pass<R, MODE, KIND, true>(P, pr, (int)s, passes, lane, rows, bs, brow, bcol, sprof);
        tb_write_end<MODE>(P.ends + pr.ends_off + s, lane, bs, brow, bcol);
    }
}

// The code of interior cell (i, j), i, j >= 1, in the fill's layout (R = 1 << r_log2 rows per lane).
__device__ inline uint32_t tb_code(const uint8_t *D, uint32_t r_log2, uint64_t pass_stride, uint32_t n_cols,
                                   uint32_t i, uint32_t j) {
    const uint32_t r = i - 1, c = j - 1;
    const uint32_t p = r >> (5 + r_log2), rr = r & ((32u << r_log2) - 1);
    const uint32_t l = rr >> r_log2, k = rr & ((1u << r_log2) - 1);
    const uint64_t at = (uint64_t)p * pass_stride + (((uint64_t)l * (n_cols + 31) + (c + l)) << (r_log2 - 1)) + (k >> 1);
    return (__ldg(D + at) >> (4 * (k & 1))) & 15u;
}

// The end cell of a pair (src/align.rs:309-327 over every row): the fill's interior candidates
// merged with the border candidates. H(0, j) and H(i, 0) never increase with j or i, so among
// border cells of row 0 or column 0 the one nearest the corner (0, 0) wins.
template <int MODE>
__device__ inline void tb_end_cell(const TbPair &pr, const TbEnd *ends, int32_t go, int32_t ge, int32_t &bs,
                                   uint32_t &brow, uint32_t &bcol) {
    using F = ModeFlags<MODE>;
    const uint32_t m = pr.m, n = pr.n;
    auto top = [&](uint32_t j) -> int32_t {  // H(0, j)
        return (F::top_free || j == 0) ? 0 : (int32_t)-tb_gap(go, ge, j);
    };
    auto left = [&](uint32_t i) -> int32_t {  // H(i, 0)
        return (F::left_free || i == 0) ? 0 : (int32_t)-tb_gap(go, ge, i);
    };
    bs = INT32_MIN;
    brow = bcol = 0;
    auto consider = [&](int32_t s, uint32_t r, uint32_t c) {
        if (tb_better(s, r, c, bs, brow, bcol)) {
            bs = s;
            brow = r;
            bcol = c;
        }
    };
    if (m > 0 && n > 0) {
        for (uint32_t x = 0; x < pr.n_ends; ++x) {
            const TbEnd e = ends[pr.ends_off + x];
            if (e.valid) consider(e.score, e.row, e.col);
        }
    }
    if (F::local) {
        consider(0, 0, 0);
    } else {
        if (F::last_col) {
            consider(top(n), 0, n);
            if (n == 0) consider(0, 0, 0);
        }
        if (m == 0) consider(top(n), 0, n);
        else if (n == 0) consider(left(m), m, 0);
        if (F::last_row) {
            consider(left(m), m, 0);
            if (m == 0) consider(0, 0, 0);
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(64) tb_walk_kernel(TbParams P) {
    using F = ModeFlags<MODE>;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n_pairs) return;
    const TbPair pr = P.pairs[t];
    const uint32_t m = pr.m, n = pr.n;
    int32_t bs;
    uint32_t brow, bcol;
    tb_end_cell<MODE>(pr, P.ends, P.go, P.ge, bs, brow, bcol);
    // Walk. State 0 H, 1 E, 2 F.
    const uint8_t *D = P.dir + pr.dir_off;
    const uint32_t R = pr.rows, r_log2 = 31 - __clz(R);
    const uint64_t pass_stride = (uint64_t)(n + 31) * 32 * (R / 2);
    const uint8_t *qs = P.q_res + pr.q_off;
    const uint8_t *ts = P.t_res + pr.t_off;
    uint8_t *slot = P.ops + pr.ops_off;
    const uint64_t cap = (uint64_t)m + n;
    uint64_t cnt = 0;
    uint32_t i = brow, j = bcol;
    int state = 0;
    int32_t v = bs;  // local mode: the value of the cell the walk stands on (H, E or F by state)
    const int32_t go = P.go, ge = P.ge;
    // Each iteration emits an operation or changes state once between two operations, so the
    // walk ends within 2 (m + n) + 2 iterations.
    for (uint64_t it = 0; it < 2 * cap + 4; ++it) {
        if (i == 0 || j == 0) {
            // Border (src/align.rs:366-383): nothing but a penalised border gap remains. The E
            // and F states always return to H before reaching a border row or column.
            if constexpr (!F::local && !F::top_free) {
                if (i == 0)
                    while (j > 0 && cnt < cap) {
                        slot[cap - 1 - cnt++] = 3;
                        --j;
                    }
            }
            if constexpr (!F::local && !F::left_free) {
                if (j == 0)
                    while (i > 0 && cnt < cap) {
                        slot[cap - 1 - cnt++] = 2;
                        --i;
                    }
            }
            break;
        }
        if (F::local && state == 0 && v == 0) break;  // local && H == 0 (src/align.rs:362-365)
        const uint32_t code = tb_code(D, r_log2, pass_stride, n, i, j);
        if (state == 0) {
            const uint32_t src = code & 3u;
            if (src == 0u) {
                const uint32_t a = qs[i - 1], b = ts[j - 1];
                if (cnt < cap) slot[cap - 1 - cnt++] = a == b ? 0 : 1;
                if (F::local) v -= P.matrix[a * P.al + b];  // H(i-1, j-1) = H(i, j) - sub
                --i;
                --j;
                continue;
            }
            state = (int)src;  // the gap step below reads the same cell's code (E or F = H here)
        }
        if (state == 1) {
            if (cnt < cap) slot[cap - 1 - cnt++] = 3;
            --j;
            if (!(code & 4u)) {
                state = 0;
                if (F::local) v += go;  // H(i, j - 1) = E(i, j) + go
            } else if (F::local) {
                v += ge;  // E(i, j - 1) = E(i, j) + ge
            }
        } else {
            if (cnt < cap) slot[cap - 1 - cnt++] = 2;
            --i;
            if (!(code & 8u)) {
                state = 0;
                if (F::local) v += go;  // H(i - 1, j) = F(i, j) + go
            } else if (F::local) {
                v += ge;  // F(i - 1, j) = F(i, j) + ge
            }
        }
    }
    hy_alignment a;
    a.score = bs;
    a.query_start = i;
    a.query_end = brow;
    a.target_start = j;
    a.target_end = bcol;
    a.n_ops = cnt;
    a.ops_offset = 0;
    P.out[pr.slot] = a;
}

// Exclusive prefix sum of n_ops over the launch's results (slot order), one block.
__global__ void __launch_bounds__(1024) tb_scan_kernel(hy_alignment *out, uint32_t n, uint64_t *total) {
    __shared__ uint64_t part[1024];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (n + 1023) / 1024;
    const uint32_t a = min(n, t * per), b = min(n, a + per);
    uint64_t s = 0;
    for (uint32_t k = a; k < b; ++k) s += out[k].n_ops;
    part[t] = s;
    __syncthreads();
    for (uint32_t o = 1; o < 1024; o <<= 1) {
        const uint64_t v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint64_t run = part[t] - s;
    for (uint32_t k = a; k < b; ++k) {
        out[k].ops_offset = run;
        run += out[k].n_ops;
    }
    if (t == 1023) *total = part[1023];
}

// Copies each pair's operations from the tail of its slot to its compacted offset (one warp each).
__global__ void __launch_bounds__(TB_BLOCK) tb_gather_kernel(TbParams P) {
    const uint32_t warp = (blockIdx.x * TB_BLOCK + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= P.n_pairs) return;
    const TbPair pr = P.pairs[warp];
    const hy_alignment a = P.out[pr.slot];
    const uint8_t *src = P.ops + pr.ops_off + ((uint64_t)pr.m + pr.n - a.n_ops);
    uint8_t *dst = P.ops_out + a.ops_offset;
    for (uint64_t x = lane; x < a.n_ops; x += 32) dst[x] = src[x];
}

// align_pairs' long pairs: the end cell of each pair as a BestHit (score, 0-based ends or -1),
// written at the pair's index (src/kernel.rs:239-277 via the same Best rule).
template <int MODE>
__global__ void tb_pair_hits_kernel(TbParams P, int32_t *scores, int32_t *qend, int32_t *tend) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.n_pairs) return;
    const TbPair pr = P.pairs[t];
    int32_t bs;
    uint32_t brow, bcol;
    tb_end_cell<MODE>(pr, P.ends, P.go, P.ge, bs, brow, bcol);
    scores[pr.slot] = bs;
    qend[pr.slot] = brow == 0 ? -1 : (int32_t)(brow - 1);
    tend[pr.slot] = bcol == 0 ? -1 : (int32_t)(bcol - 1);
}

// Query profile for the fill: prof[c * m_pad + r] = matrix[q[r] * al + c] for r < m, 0 for the
// padding rows (sub = 0 there keeps every padding cell below a real cell of no larger column and
// smaller row, so padding never wins the local end cell).
__global__ void tb_profile_kernel(const uint8_t *q, uint32_t m, uint32_t m_pad, const int32_t *matrix,
                                  uint32_t al, int32_t *prof) {
    const uint64_t total = (uint64_t)al * m_pad;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)(x / m_pad), r = (uint32_t)(x - (uint64_t)c * m_pad);
        prof[x] = r < m ? matrix[(uint64_t)q[r] * al + c] : 0;
    }
}

// ---- host side ----------------------------------------------------------------------------------

// Rows per lane of the fill for a query of m rows: the fewest (steps x per-step cost) over the
// compiled choices, where a pass of 32 R rows costs (n + 31) steps of R cells plus a fixed part.
static uint32_t tb_rows(uint64_t m, uint64_t n) {
    uint32_t best = 16;
    double best_cost = 1e300;
    for (uint32_t R : {4u, 8u, 16u}) {
        const uint64_t passes = (m + 32 * R - 1) / (32 * R);
        const double cost = (double)passes * (double)(n + 31) * (R + 6.0);
        if (cost < best_cost) {
            best_cost = cost;
            best = R;
        }
    }
    return best;
}

// align_pairs sends a pair to the score-only stripe kernel when its query spans several stripes
// and it is large: the int16x2 pair kernels give one pair one 8-lane group, far too little for a
// single pair of thousands of residues each.
constexpr uint64_t TB_LONG_PAIR_ROWS = 256;
constexpr double TB_LONG_PAIR_CELLS = 1024.0 * 1024;

// Few pairs of a multi-pass query fill with the stripe kernel at 4 rows per lane (128-row
// stripes: the most warps per pair); many pairs fill one warp each at tb_rows.
constexpr uint32_t TB_STRIPE_PAIRS = 16;
static void tb_plan(uint64_t m, uint64_t max_n, uint32_t n_pairs, uint32_t *R, bool *stripes) {
    *stripes = n_pairs <= TB_STRIPE_PAIRS && m > 128;
    *R = *stripes ? TB_STRIPE_R : tb_rows(m, max_n);
}

static uint64_t tb_passes(uint64_t m, uint32_t R) { return std::max<uint64_t>(1, (m + 32 * R - 1) / (32 * R)); }

static uint64_t tb_dir_bytes(uint64_t m, uint64_t n, uint32_t R) {
    if (m == 0 || n == 0) return 0;
    return tb_passes(m, R) * (n + 31) * 32 * (R / 2);
}

static uint64_t align16(uint64_t x) { return (x + 15) & ~15ull; }

template <class T>
static cudaError_t grow(T *&p, uint64_t &cap, uint64_t need) {
    need = std::max<uint64_t>(need, 16);
    if (cap >= need) return cudaSuccess;
    hy::dev_free(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = hy::dev_malloc((void **)&p, need);
    if (e == cudaSuccess) cap = need;
    return e;
}

template <class T>
static cudaError_t grow_pinned(T *&p, uint64_t &cap, uint64_t need) {
    need = std::max<uint64_t>(need, 16);
    if (cap >= need) return cudaSuccess;
    cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost((void **)&p, need);
    if (e == cudaSuccess) cap = need;
    return e;
}

// Grow-only device and pinned buffers of one traceback caller (a scratch, or the calling thread
// for hy_align).
struct TbContext {
    int device = -1;
    cudaStream_t stream = nullptr;    // fills, then the copies back (the caller's stream)
    cudaStream_t stream_b = nullptr;  // walks and compaction, overlapping the next chunk's fill
    bool own_stream = false;
    uint8_t *d_q = nullptr, *d_t = nullptr, *d_ops = nullptr, *d_ops_out = nullptr;
    uint8_t *d_dir[2] = {nullptr, nullptr};  // codes of two chunks in flight
    int32_t *d_prof = nullptr, *d_matrix = nullptr;
    int2 *d_bnd = nullptr;
    TbPair *d_pairs = nullptr;
    TbEnd *d_ends = nullptr;
    hy_alignment *d_out = nullptr;
    uint64_t *d_total = nullptr;
    uint32_t *d_prog = nullptr;  // stripe kernel: error flag (first 16 bytes), then progress counters
    uint32_t *d_first = nullptr, *h_first = nullptr;  // stripe kernel: first stripe of each pair
    uint64_t c_prog = 0, c_first = 0, ch_first = 0;
    uint64_t c_q = 0, c_t = 0, c_ops = 0, c_ops_out = 0, c_prof = 0, c_matrix = 0, c_bnd = 0,
             c_pairs = 0, c_ends = 0, c_out = 0, c_total = 0;
    uint64_t c_dir[2] = {0, 0};
    TbPair *h_pairs = nullptr;
    hy_alignment *h_out = nullptr;
    uint8_t *h_ops = nullptr, *h_q = nullptr, *h_stage = nullptr;
    uint64_t *h_total = nullptr;
    uint64_t ch_pairs = 0, ch_out = 0, ch_ops = 0, ch_total = 0, ch_q = 0, ch_stage = 0;
    uint64_t launches = 0;
    // Per chunk: fill start / end on `stream`, walk start / end on `stream_b`.
    std::vector<cudaEvent_t> ev;
    // Timing of the last call: the fill kernels, the walk + compaction kernels, the device span
    // from the first fill to the end of compaction (CUDA events), the whole call (host clock), and
    // the DP cells traced.
    double fill_ms = 0.0, walk_ms = 0.0, device_ms = 0.0, call_ms = 0.0, cells = 0.0;
    ~TbContext() {
        if (stream) cudaStreamSynchronize(stream);
        if (stream_b) cudaStreamSynchronize(stream_b);
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        for (void *p : {(void *)d_q, (void *)d_t, (void *)d_dir[0], (void *)d_dir[1], (void *)d_ops,
                        (void *)d_ops_out, (void *)d_prof, (void *)d_matrix, (void *)d_bnd, (void *)d_pairs,
                        (void *)d_ends, (void *)d_out, (void *)d_total, (void *)d_prog, (void *)d_first})
            hy::dev_free(p);
        for (void *p : {(void *)h_pairs, (void *)h_out, (void *)h_ops, (void *)h_total, (void *)h_q,
                        (void *)h_first, (void *)h_stage})
            cudaFreeHost(p);
        if (stream_b) cudaStreamDestroy(stream_b);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

#define TB_CK(call)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            cudaGetLastError();                                                                  \
            return fail(e_ == cudaErrorMemoryAllocation ? HY_ERR_OUT_OF_MEMORY : HY_ERR_CUDA, e_); \
        }                                                                                        \
    } while (0)

template <int MODE>
static cudaError_t launch_fill(uint32_t R, const TbParams &p, cudaStream_t st) {
    const uint32_t blocks = (uint32_t)(((uint64_t)p.n_pairs * 32 + TB_BLOCK - 1) / TB_BLOCK);
    if (R == 4) tb_fill_kernel<4, MODE><<<blocks, TB_BLOCK, 0, st>>>(p);
    else if (R == 8) tb_fill_kernel<8, MODE><<<blocks, TB_BLOCK, 0, st>>>(p);
    else tb_fill_kernel<16, MODE><<<blocks, TB_BLOCK, 0, st>>>(p);
    return cudaGetLastError();
}

// The walk is one thread per pair and bound by the latency of its dependent code loads: small
// blocks spread the walkers over every SM.
constexpr int TB_WALK_BLOCK = 64;

template <int MODE>
static cudaError_t launch_walk(const TbParams &p, cudaStream_t st) {
    tb_walk_kernel<MODE><<<(p.n_pairs + TB_WALK_BLOCK - 1) / TB_WALK_BLOCK, TB_WALK_BLOCK, 0, st>>>(p);
    return cudaGetLastError();
}


// Blocks of the stripe kernel: two warps, so a pair's stripes spread over many SMs (each stripe is
// a chain of dependent steps; a warp alone on its scheduler runs it at the lowest latency).
constexpr int TB_STRIPE_BLOCK = 64;

template <int MODE, int KIND>
static cudaError_t launch_stripes(const TbParams &p, const TbStripes &S, cudaStream_t st, int device) {
    auto kern = tb_stripe_kernel<TB_STRIPE_R, MODE, KIND>;
    // The stripes read their profile rows every step from global memory: keep L1 as large as
    // the SM allows.
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxL1);
    if (e != cudaSuccess) return e;
    const size_t smem = (size_t)S.al * 32 * TB_STRIPE_R * sizeof(int32_t) * (TB_STRIPE_BLOCK / 32);
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TB_STRIPE_BLOCK, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    const uint64_t want = ((uint64_t)S.n_stripes * 32 + TB_STRIPE_BLOCK - 1) / TB_STRIPE_BLOCK;
    const uint32_t blocks = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)per_sm * sms));
    TbParams pc = p;
    TbStripes sc = S;
    void *args[] = {(void *)&pc, (void *)&sc};
    return cudaLaunchCooperativeKernel((const void *)kern, dim3(blocks), dim3(TB_STRIPE_BLOCK), args, smem, st);
}

static cudaError_t dispatch_stripes(int mode, bool codes, const TbParams &p, const TbStripes &S,
                                    cudaStream_t st, int device) {
#define TB_STRIPE_CASE(M)                                                                          \
    case M:                                                                                        \
        return codes ? launch_stripes<M, TB_CODES>(p, S, st, device) : launch_stripes<M, TB_SCORE>(p, S, st, device);
    switch (mode) {
        TB_STRIPE_CASE(MODE_SW)
        TB_STRIPE_CASE(MODE_NW)
        TB_STRIPE_CASE(MODE_HW)
        TB_STRIPE_CASE(MODE_OV)
        TB_STRIPE_CASE(MODE_SHW)
    }
#undef TB_STRIPE_CASE
    return cudaErrorInvalidValue;
}

static cudaError_t dispatch_fill(int mode, uint32_t R, const TbParams &p, cudaStream_t st) {
    switch (mode) {
    case MODE_SW: return launch_fill<MODE_SW>(R, p, st);
    case MODE_NW: return launch_fill<MODE_NW>(R, p, st);
    case MODE_HW: return launch_fill<MODE_HW>(R, p, st);
    case MODE_OV: return launch_fill<MODE_OV>(R, p, st);
    default: return launch_fill<MODE_SHW>(R, p, st);
    }
}

static cudaError_t dispatch_walk(int mode, const TbParams &p, cudaStream_t st) {
    switch (mode) {
    case MODE_SW: return launch_walk<MODE_SW>(p, st);
    case MODE_NW: return launch_walk<MODE_NW>(p, st);
    case MODE_HW: return launch_walk<MODE_HW>(p, st);
    case MODE_OV: return launch_walk<MODE_OV>(p, st);
    default: return launch_walk<MODE_SHW>(p, st);
    }
}

// One query (already on the device, with its profile built) against the targets `idx` (global
// indices into t_res by `t_off`): fills, walks and compacts in chunks, appending to `ops` and
// writing out[k] for target idx[k] (ops_offset relative to the start of the call's operations).
struct TbRun {
    int mode;
    int32_t go, ge;
    uint64_t m;
    uint32_t m_pad, R;
    const uint8_t *d_t_res;        // device targets
    const uint64_t *h_t_off;       // host offsets of the targets (n_targets + 1), or null
    const uint64_t *h_t_single;    // a single target: {offset, length} when h_t_off is null
    bool stripes;                  // fill with the stripe kernel (few long pairs)
    uint64_t al;                   // alphabet size (profile letters)
    const int32_t *d_matrix;       // substitution matrix on the device (the walk's values)
};

static hy_status tb_run(TbContext &ctx, const TbRun &run, const uint32_t *idx, uint32_t n_idx,
                        hy_alignment *out, std::vector<uint8_t> *ops_host, uint8_t *ops_direct) {
    auto t_off = [&](uint32_t k) { return run.h_t_off ? run.h_t_off[k] : run.h_t_single[0]; };
    auto t_len = [&](uint32_t k) {
        return run.h_t_off ? run.h_t_off[k + 1] - run.h_t_off[k] : run.h_t_single[1];
    };
    const auto t_start = std::chrono::steady_clock::now();
    ctx.fill_ms = ctx.walk_ms = ctx.device_ms = ctx.cells = 0.0;
    if (!ctx.stream_b) TB_CK(cudaStreamCreateWithFlags(&ctx.stream_b, cudaStreamNonBlocking));
    // Launch order: longest target first over the whole call, so every chunk holds targets of
    // similar length (short tails) and the longest start first. Results keep the caller's order.
    std::vector<uint32_t> order(n_idx);
    for (uint32_t x = 0; x < n_idx; ++x) order[x] = x;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t x, uint32_t y) { return t_len(idx[x]) > t_len(idx[y]); });
    // Operation slots in the caller's order; chunks of at most TB_CHUNK_BYTES of codes.
    TB_CK(grow_pinned(ctx.h_pairs, ctx.ch_pairs, sizeof(TbPair) * n_idx));
    std::vector<uint64_t> ops_at(n_idx);
    uint64_t oo = 0;
    for (uint32_t x = 0; x < n_idx; ++x) {
        ops_at[x] = oo;
        oo += run.m + t_len(idx[x]);
    }
    std::vector<uint32_t> chunk_at{0};
    uint64_t dir_max = 0, bnd_max = 0, dir = 0, bnd = 0;
    const uint32_t per_pair = run.stripes ? (uint32_t)tb_passes(run.m, run.R) : 1u;
    for (uint32_t x = 0; x < n_idx; ++x) {
        const uint32_t s = order[x], k = idx[s];
        const uint64_t n = t_len(k);
        const uint64_t d = align16(tb_dir_bytes(run.m, n, run.R));
        if (x > chunk_at.back() && dir + d > TB_CHUNK_BYTES) {
            chunk_at.push_back(x);
            dir = bnd = 0;
        }
        TbPair &pp = ctx.h_pairs[x];
        pp.q_off = 0;
        pp.prof_off = 0;
        pp.t_off = t_off(k);
        pp.m = (uint32_t)run.m;
        pp.n = (uint32_t)n;
        pp.m_pad = run.m_pad;
        pp.slot = s;
        pp.rows = run.R;
        pp.n_ends = per_pair;
        pp.ends_off = run.stripes ? (uint64_t)x * per_pair : s;
        pp.dir_off = dir;
        pp.bnd_off = bnd;
        pp.ops_off = ops_at[s];
        dir += d;
        bnd += run.stripes ? (uint64_t)(per_pair - 1) * (n + 1) : n + 1;
        dir_max = std::max(dir_max, dir);
        bnd_max = std::max(bnd_max, bnd);
        ctx.cells += (double)run.m * (double)n;
    }
    chunk_at.push_back(n_idx);
    const size_t n_chunks = chunk_at.size() - 1;
    TB_CK(grow(ctx.d_pairs, ctx.c_pairs, sizeof(TbPair) * n_idx));
    TB_CK(grow(ctx.d_dir[0], ctx.c_dir[0], dir_max));
    if (n_chunks > 1) TB_CK(grow(ctx.d_dir[1], ctx.c_dir[1], dir_max));
    TB_CK(grow(ctx.d_bnd, ctx.c_bnd, sizeof(int2) * bnd_max));
    TB_CK(grow(ctx.d_ops, ctx.c_ops, oo));
    TB_CK(grow(ctx.d_ops_out, ctx.c_ops_out, oo));
    TB_CK(grow(ctx.d_ends, ctx.c_ends, sizeof(TbEnd) * n_idx * per_pair));
    if (run.stripes) {
        TB_CK(grow(ctx.d_prog, ctx.c_prog, sizeof(uint32_t) * (uint64_t)n_idx * per_pair + 16));
        TB_CK(cudaMemsetAsync(ctx.d_prog, 0, 16, ctx.stream));  // the error flag sits in front
        // Every pair has per_pair stripes: chunk-local pair x owns [x, x + 1) * per_pair.
        TB_CK(grow(ctx.d_first, ctx.c_first, sizeof(uint32_t) * (n_idx + 1)));
        TB_CK(grow_pinned(ctx.h_first, ctx.ch_first, sizeof(uint32_t) * (n_idx + 1)));
        for (uint32_t x = 0; x <= n_idx; ++x) ctx.h_first[x] = x * per_pair;
        TB_CK(cudaMemcpyAsync(ctx.d_first, ctx.h_first, sizeof(uint32_t) * (n_idx + 1), cudaMemcpyHostToDevice,
                              ctx.stream));
    }
    TB_CK(grow(ctx.d_out, ctx.c_out, sizeof(hy_alignment) * n_idx));
    TB_CK(grow(ctx.d_total, ctx.c_total, 16));
    TB_CK(grow_pinned(ctx.h_out, ctx.ch_out, sizeof(hy_alignment) * n_idx));
    TB_CK(grow_pinned(ctx.h_total, ctx.ch_total, 16));
    while (ctx.ev.size() < 4 * n_chunks + 2) {
        cudaEvent_t e;
        TB_CK(cudaEventCreate(&e));
        ctx.ev.push_back(e);
    }
    TB_CK(cudaMemcpyAsync(ctx.d_pairs, ctx.h_pairs, sizeof(TbPair) * n_idx, cudaMemcpyHostToDevice, ctx.stream));
    TbParams p;
    memset(&p, 0, sizeof(p));
    p.q_res = ctx.d_q;
    p.t_res = run.d_t_res;
    p.prof = ctx.d_prof;
    p.matrix = run.d_matrix;
    p.al = (uint32_t)run.al;
    p.bnd = ctx.d_bnd;
    p.ends = ctx.d_ends;
    p.out = ctx.d_out;
    p.ops = ctx.d_ops;
    p.ops_out = ctx.d_ops_out;
    p.total = ctx.d_total;
    p.go = run.go;
    p.ge = run.ge;
    // Chunk c: fill on `stream` into codes buffer c % 2 (once the walk of chunk c - 2 is done with
    // it), walk on `stream_b` once the fill is done.
    for (size_t c = 0; c < n_chunks; ++c) {
        cudaEvent_t *e = &ctx.ev[4 * c];
        p.pairs = ctx.d_pairs + chunk_at[c];
        p.n_pairs = chunk_at[c + 1] - chunk_at[c];
        p.dir = ctx.d_dir[c & 1];
        if (c >= 2) TB_CK(cudaStreamWaitEvent(ctx.stream, ctx.ev[4 * (c - 2) + 3], 0));
        TB_CK(cudaEventRecord(e[0], ctx.stream));
        if (run.m > 0 && run.stripes) {
            const uint32_t n_str = p.n_pairs * per_pair;
            TbStripes S{ctx.d_first, n_str, tb_stripe_smem_al(run.al), ctx.d_bnd, ctx.d_prog + 4, (int *)ctx.d_prog,
                        tb_spin_limit()};
            TB_CK(cudaMemsetAsync(S.prog, 0, sizeof(uint32_t) * n_str, ctx.stream));
            TB_CK(dispatch_stripes(run.mode, true, p, S, ctx.stream, ctx.device));
            ctx.launches += 2;
        } else if (run.m > 0) {
            TB_CK(dispatch_fill(run.mode, run.R, p, ctx.stream));
            ++ctx.launches;
        }
        TB_CK(cudaEventRecord(e[1], ctx.stream));
        TB_CK(cudaStreamWaitEvent(ctx.stream_b, e[1], 0));
        TB_CK(cudaEventRecord(e[2], ctx.stream_b));
        TB_CK(dispatch_walk(run.mode, p, ctx.stream_b));
        ++ctx.launches;
        TB_CK(cudaEventRecord(e[3], ctx.stream_b));
    }
    // Compaction over the whole call, in the caller's order.
    p.pairs = ctx.d_pairs;
    p.n_pairs = n_idx;
    tb_scan_kernel<<<1, 1024, 0, ctx.stream_b>>>(ctx.d_out, n_idx, ctx.d_total);
    TB_CK(cudaGetLastError());
    tb_gather_kernel<<<(uint32_t)(((uint64_t)n_idx * 32 + TB_BLOCK - 1) / TB_BLOCK), TB_BLOCK, 0, ctx.stream_b>>>(p);
    TB_CK(cudaGetLastError());
    ctx.launches += 2;
    cudaEvent_t e_end = ctx.ev[4 * n_chunks];
    TB_CK(cudaEventRecord(e_end, ctx.stream_b));
    TB_CK(cudaStreamWaitEvent(ctx.stream, e_end, 0));
    TB_CK(cudaMemcpyAsync(ctx.h_out, ctx.d_out, sizeof(hy_alignment) * n_idx, cudaMemcpyDeviceToHost, ctx.stream));
    TB_CK(cudaMemcpyAsync(ctx.h_total, ctx.d_total, sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx.stream));
    if (run.stripes) TB_CK(cudaMemcpyAsync(ctx.h_total + 1, ctx.d_prog, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx.stream));
    TB_CK(cudaStreamSynchronize(ctx.stream));
    if (run.stripes && *(const uint32_t *)(ctx.h_total + 1)) return fail(HY_ERR_TIMEOUT);
    const uint64_t total = *ctx.h_total;
    if (ops_direct) {
        if (total) TB_CK(cudaMemcpyAsync(ops_direct, ctx.d_ops_out, total, cudaMemcpyDeviceToHost, ctx.stream));
    } else {
        TB_CK(grow_pinned(ctx.h_ops, ctx.ch_ops, total));
        if (total) TB_CK(cudaMemcpyAsync(ctx.h_ops, ctx.d_ops_out, total, cudaMemcpyDeviceToHost, ctx.stream));
    }
    TB_CK(cudaStreamSynchronize(ctx.stream));
    if (!ops_direct) ops_host->assign(ctx.h_ops, ctx.h_ops + total);
    memcpy(out, ctx.h_out, sizeof(hy_alignment) * n_idx);
    for (size_t c = 0; c < n_chunks; ++c) {
        float f_ms = 0.f, w_ms = 0.f;
        TB_CK(cudaEventElapsedTime(&f_ms, ctx.ev[4 * c], ctx.ev[4 * c + 1]));
        TB_CK(cudaEventElapsedTime(&w_ms, ctx.ev[4 * c + 2], ctx.ev[4 * c + 3]));
        ctx.fill_ms += f_ms;
        ctx.walk_ms += w_ms;
    }
    float span = 0.f, tail = 0.f;
    TB_CK(cudaEventElapsedTime(&span, ctx.ev[0], e_end));
    TB_CK(cudaEventElapsedTime(&tail, ctx.ev[4 * n_chunks - 1], e_end));
    ctx.device_ms = span;
    ctx.walk_ms += tail;
    ctx.call_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return fail(HY_OK);
}

static hy_status tb_prepare_query(TbContext &ctx, const uint8_t *query, uint64_t m, const int32_t *d_matrix,
                                  uint64_t al, uint32_t R, uint32_t *m_pad) {
    *m_pad = (uint32_t)(tb_passes(std::max<uint64_t>(m, 1), R) * 32 * R);
    TB_CK(grow(ctx.d_q, ctx.c_q, std::max<uint64_t>(m, 1)));
    TB_CK(grow(ctx.d_prof, ctx.c_prof, sizeof(int32_t) * al * *m_pad));
    if (m) {
        TB_CK(cudaStreamSynchronize(ctx.stream));  // the staging buffer of the previous call is free
        TB_CK(grow_pinned(ctx.h_q, ctx.ch_q, m));
        memcpy(ctx.h_q, query, m);
        TB_CK(cudaMemcpyAsync(ctx.d_q, ctx.h_q, m, cudaMemcpyHostToDevice, ctx.stream));
    }
    const uint64_t total = al * (uint64_t)*m_pad;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>(1024, (total + 255) / 256);
    tb_profile_kernel<<<std::max<uint32_t>(blocks, 1), 256, 0, ctx.stream>>>(ctx.d_q, (uint32_t)m, *m_pad, d_matrix,
                                                                            (uint32_t)al, ctx.d_prof);
    TB_CK(cudaGetLastError());
    ++ctx.launches;
    return fail(HY_OK);
}

// u64::isqrt (src/align.rs:210).
static uint64_t isqrt_u64(uint64_t v) {
    uint64_t r = 0;
    for (uint64_t bit = 1ull << 62; bit; bit >>= 2) {
        if (v >= r + bit) {
            v -= r + bit;
            r = (r >> 1) + bit;
        } else {
            r >>= 1;
        }
    }
    return r;
}

static uint64_t sat_mul(uint64_t a, uint64_t b) {
    unsigned __int128 p = (unsigned __int128)a * b;
    return p > (unsigned __int128)UINT64_MAX ? UINT64_MAX : (uint64_t)p;
}
// full_matrix_bytes and checkpoint_bytes (src/align.rs:252-268).
static uint64_t full_matrix_bytes(uint64_t m, uint64_t n) { return sat_mul(sat_mul(sat_mul(m + 1, n + 1), 3), 4); }
static uint64_t checkpoint_bytes(uint64_t m, uint64_t n, uint64_t k) {
    return sat_mul(sat_mul(2 * (m / k + 1) + 3 * (k + 1), n + 1), 4);
}

}  // namespace hy

using namespace hy;

// ---- runtime hooks ----------------------------------------------------------------------------

void hy::tb_context_destroy(void *ctx) { delete (TbContext *)ctx; }

// ---- C ABI ------------------------------------------------------------------------------------------

extern "C" {

uint64_t hy_traceback_needed(uint64_t m, uint64_t n, uint64_t max_bytes) {
    if (full_matrix_bytes(m, n) <= max_bytes || m == 0 || n == 0) return 0;
    const uint64_t peak = checkpoint_bytes(m, n, std::max<uint64_t>(1, isqrt_u64(m)));
    return peak > max_bytes ? peak : 0;
}

uint64_t hy_traceback_min_bytes_for_database(uint64_t max_m, uint64_t max_n) {
    uint64_t v = full_matrix_bytes(max_m, max_n);
    if (max_m > 0 && max_n > 0)
        v = std::min(v, checkpoint_bytes(max_m, max_n, std::max<uint64_t>(1, isqrt_u64(max_m))));
    return std::max({v, full_matrix_bytes(max_m, 0), full_matrix_bytes(0, max_n)});
}

// Per calling thread, freed when the thread exits.
static thread_local std::unique_ptr<TbContext> g_align_ctx;

hy_status hy_traceback_timing(hy_scratch *scratch, double out[5]) {
    if (!out) return fail(HY_ERR_INVALID_ARGUMENT);
    tb_context_timing(scratch ? scratch_tb(scratch) : (void *)g_align_ctx.get(), out);
    return fail(HY_OK);
}

hy_status hy_align(const uint8_t *query, uint64_t qlen, const uint8_t *target, uint64_t tlen,
                   const int32_t *matrix, uint64_t alphabet_len, int32_t gap_open, int32_t gap_ext,
                   hy_mode mode, uint64_t max_bytes, hy_alignment *out, uint8_t *ops) {
    if (!out || (qlen + tlen > 0 && !ops) || (qlen && !query) || (tlen && !target))
        return fail(HY_ERR_INVALID_ARGUMENT);
    if ((int)mode < 0 || (int)mode > 4) return fail(HY_ERR_INVALID_ARGUMENT);
    hy_status st = validate_scoring(alphabet_len, matrix, alphabet_len * alphabet_len, gap_open, gap_ext);
    if (st != HY_OK) return st;
    for (uint64_t x = 0; x < qlen + tlen; ++x) {
        const uint8_t s = x < qlen ? query[x] : target[x - qlen];
        if (s >= alphabet_len) return fail(HY_ERR_SYMBOL_OUT_OF_RANGE, s, (int64_t)alphabet_len);
    }
    const int32_t min_e = *std::min_element(matrix, matrix + alphabet_len * alphabet_len);
    const int32_t max_e = *std::max_element(matrix, matrix + alphabet_len * alphabet_len);
    const int64_t bound = magnitude_bound(mode, min_e, max_e, gap_open, gap_ext, qlen, tlen);
    if (narrowest_width(bound) < 0) return fail(HY_ERR_SCORE_RANGE_TOO_WIDE, bound);
    const uint64_t need = hy_traceback_needed(qlen, tlen, max_bytes);
    if (need) return fail(HY_ERR_TRACEBACK_BUDGET_EXCEEDED, (int64_t)need, (int64_t)max_bytes);
    if (qlen >= (1ull << 31) || tlen >= (1ull << 31)) return fail(HY_ERR_UNSUPPORTED);

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(HY_ERR_CUDA, cudaErrorNoDevice);
    }
    if (g_align_ctx && g_align_ctx->device != dev) g_align_ctx.reset();
    if (!g_align_ctx) {
        g_align_ctx.reset(new TbContext);
        g_align_ctx->device = dev;
        g_align_ctx->own_stream = true;
        if (cudaStreamCreateWithFlags(&g_align_ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            g_align_ctx.reset();
            return fail(HY_ERR_CUDA, cudaErrorUnknown);
        }
    }
    TbContext &ctx = *g_align_ctx;
    const uint64_t mat_bytes = sizeof(int32_t) * alphabet_len * alphabet_len;
    TB_CK(grow(ctx.d_matrix, ctx.c_matrix, mat_bytes));
    TB_CK(cudaMemcpyAsync(ctx.d_matrix, matrix, mat_bytes, cudaMemcpyHostToDevice, ctx.stream));
    TB_CK(grow(ctx.d_t, ctx.c_t, std::max<uint64_t>(tlen, 1)));
    if (tlen) TB_CK(cudaMemcpyAsync(ctx.d_t, target, tlen, cudaMemcpyHostToDevice, ctx.stream));
    uint32_t R = 0;
    bool stripes = false;
    tb_plan(qlen, tlen, 1, &R, &stripes);
    uint32_t m_pad = 0;
    st = tb_prepare_query(ctx, query, qlen, ctx.d_matrix, alphabet_len, R, &m_pad);
    if (st != HY_OK) return st;
    TbRun run;
    run.mode = mode;
    run.go = gap_open;
    run.ge = gap_ext;
    run.m = qlen;
    run.m_pad = m_pad;
    run.R = R;
    run.stripes = stripes;
    run.al = alphabet_len;
    run.d_matrix = ctx.d_matrix;
    run.d_t_res = ctx.d_t;
    run.h_t_off = nullptr;
    const uint64_t single[2] = {0, tlen};
    run.h_t_single = single;
    const uint32_t idx0 = 0;
    return tb_run(ctx, run, &idx0, 1, out, nullptr, ops);
}

}  // extern "C"

namespace hy {

// scan_all_aligned / scan_aligned over the database's plain residue copy.
hy_status tb_scan_targets(const hy_db *db, void **ctx_slot, cudaStream_t stream, const uint8_t *query,
                          uint64_t qlen, const uint32_t *idx, uint32_t n_idx, hy_alignment *out,
                          std::vector<uint8_t> &ops) {
    TbContext *ctx = (TbContext *)*ctx_slot;
    if (!ctx) {
        ctx = new TbContext;
        ctx->device = db->device;
        ctx->stream = stream;
        *ctx_slot = ctx;
    }
    uint64_t max_n = 0;
    for (uint32_t x = 0; x < n_idx; ++x)
        max_n = std::max<uint64_t>(max_n, db->tb_off[idx[x] + 1] - db->tb_off[idx[x]]);
    uint32_t R = 0;
    bool stripes = false;
    tb_plan(qlen, max_n, n_idx, &R, &stripes);
    uint32_t m_pad = 0;
    hy_status st = tb_prepare_query(*ctx, query, qlen, db->d_matrix, db->al, R, &m_pad);
    if (st != HY_OK) return st;
    TbRun run;
    run.mode = db->mode;
    run.go = db->go;
    run.ge = db->ge;
    run.m = qlen;
    run.m_pad = m_pad;
    run.R = R;
    run.stripes = stripes;
    run.al = db->al;
    run.d_matrix = db->d_matrix;
    run.d_t_res = db->d_tb_res;
    run.h_t_off = db->tb_off.data();
    run.h_t_single = nullptr;
    ops.clear();
    return tb_run(*ctx, run, idx, n_idx, out, &ops, nullptr);
}

bool tb_long_pair(uint64_t qlen, uint64_t tlen) {
    return qlen >= TB_LONG_PAIR_ROWS && (double)qlen * (double)tlen >= TB_LONG_PAIR_CELLS;
}

uint64_t tb_long_pair_stripes(uint64_t qlen) { return tb_passes(qlen, TB_STRIPE_R); }

static thread_local std::unique_ptr<TbContext> g_pairs_ctx;

hy_status tb_long_pair_scores(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                              const uint64_t *t_off, const std::vector<uint32_t> &idx, const uint8_t *d_q,
                              const int32_t *d_matrix, uint64_t al, int32_t go, int32_t ge, int mode,
                              cudaStream_t stream, int32_t *d_scores, int32_t *d_qend, int32_t *d_tend,
                              double *kernel_ms, const TbColmaxOut *cmx) {
    (void)q_res;
    const uint32_t n = (uint32_t)idx.size();
    if (n == 0) return fail(HY_OK);
    int dev = 0;
    TB_CK(cudaGetDevice(&dev));
    if (g_pairs_ctx && g_pairs_ctx->device != dev) g_pairs_ctx.reset();
    if (!g_pairs_ctx) {
        g_pairs_ctx.reset(new TbContext);
        g_pairs_ctx->device = dev;
    }
    TbContext &ctx = *g_pairs_ctx;
    // The caller's stream, borrowed for this call only: ordered after its query upload, before its
    // copy back.
    ctx.stream = stream;
    struct Unborrow {
        TbContext &c;
        ~Unborrow() { c.stream = nullptr; }
    } unborrow{ctx};
    if (ctx.ev.size() < 2) {
        for (int x = 0; x < 2; ++x) {
            cudaEvent_t e;
            TB_CK(cudaEventCreate(&e));
            ctx.ev.push_back(e);
        }
    }
    // Targets, profiles, boundary rows and stripes of every long pair.
    uint64_t t_total = 0, prof_total = 0, bnd_total = 0;
    uint32_t n_str = 0;
    TB_CK(grow_pinned(ctx.h_pairs, ctx.ch_pairs, sizeof(TbPair) * n));
    TB_CK(grow_pinned(ctx.h_first, ctx.ch_first, sizeof(uint32_t) * (n + 1)));
    for (uint32_t x = 0; x < n; ++x) {
        const uint32_t k = idx[x];
        const uint64_t m = q_off[k + 1] - q_off[k], tl = t_off[k + 1] - t_off[k];
        const uint32_t S = (uint32_t)tb_passes(m, TB_STRIPE_R);
        TbPair &pp = ctx.h_pairs[x];
        pp.q_off = q_off[k];
        pp.m = (uint32_t)m;
        pp.n = (uint32_t)tl;
        pp.m_pad = S * 32 * TB_STRIPE_R;
        pp.prof_off = prof_total;
        pp.t_off = t_total;
        pp.dir_off = 0;
        pp.bnd_off = bnd_total;
        pp.ops_off = cmx ? t_off[k] : 0;  // column maxima at the pair's target offset
        pp.ends_off = n_str;
        pp.n_ends = S;
        pp.slot = k;
        pp.rows = TB_STRIPE_R;
        ctx.h_first[x] = n_str;
        prof_total += al * pp.m_pad;
        t_total += tl;
        bnd_total += (uint64_t)(S - 1) * (tl + 1);
        n_str += S;
    }
    ctx.h_first[n] = n_str;
    TB_CK(grow_pinned(ctx.h_ops, ctx.ch_ops, t_total));
    for (uint32_t x = 0; x < n; ++x) {
        const uint32_t k = idx[x];
        memcpy(ctx.h_ops + ctx.h_pairs[x].t_off, t_res + t_off[k], t_off[k + 1] - t_off[k]);
    }
    TB_CK(grow(ctx.d_t, ctx.c_t, t_total));
    TB_CK(grow(ctx.d_prof, ctx.c_prof, sizeof(int32_t) * prof_total));
    TB_CK(grow(ctx.d_bnd, ctx.c_bnd, sizeof(int2) * std::max<uint64_t>(bnd_total, 1)));
    TB_CK(grow(ctx.d_pairs, ctx.c_pairs, sizeof(TbPair) * n));
    TB_CK(grow(ctx.d_first, ctx.c_first, sizeof(uint32_t) * (n + 1)));
    TB_CK(grow(ctx.d_ends, ctx.c_ends, sizeof(TbEnd) * n_str));
    TB_CK(grow(ctx.d_prog, ctx.c_prog, sizeof(uint32_t) * n_str + 16));
    TB_CK(grow(ctx.d_dir[0], ctx.c_dir[0], 16));
    TB_CK(cudaMemcpyAsync(ctx.d_t, ctx.h_ops, t_total, cudaMemcpyHostToDevice, stream));
    TB_CK(cudaMemcpyAsync(ctx.d_pairs, ctx.h_pairs, sizeof(TbPair) * n, cudaMemcpyHostToDevice, stream));
    TB_CK(cudaMemcpyAsync(ctx.d_first, ctx.h_first, sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice, stream));
    TB_CK(cudaMemsetAsync(ctx.d_prog, 0, sizeof(uint32_t) * n_str + 16, stream));
    for (uint32_t x = 0; x < n; ++x) {
        const TbPair &pp = ctx.h_pairs[x];
        const uint64_t total = al * (uint64_t)pp.m_pad;
        const uint32_t blocks = (uint32_t)std::min<uint64_t>(1024, (total + 255) / 256);
        tb_profile_kernel<<<blocks, 256, 0, stream>>>(d_q + pp.q_off, pp.m, pp.m_pad, d_matrix, (uint32_t)al,
                                                      ctx.d_prof + pp.prof_off);
        TB_CK(cudaGetLastError());
    }
    TbParams p;
    memset(&p, 0, sizeof(p));
    p.pairs = ctx.d_pairs;
    p.n_pairs = n;
    p.q_res = d_q;
    p.t_res = ctx.d_t;
    p.prof = ctx.d_prof;
    p.dir = ctx.d_dir[0];
    p.bnd = ctx.d_bnd;
    p.ends = ctx.d_ends;
    p.go = go;
    p.ge = ge;
    TbStripes S{ctx.d_first, n_str, tb_stripe_smem_al(al), ctx.d_bnd, ctx.d_prog + 4, (int *)ctx.d_prog,
                tb_spin_limit()};
    if (cmx) {
        p.colmax = cmx->colmax;
        TB_CK(cudaEventRecord(ctx.ev[0], stream));
        TB_CK((launch_stripes<MODE_SW, TB_COLMAX>(p, S, stream, dev)));
        TB_CK(cudaEventRecord(ctx.ev[1], stream));
        tb_position_hits_kernel<<<(n + 63) / 64, 64, 0, stream>>>(p, d_scores, d_tend, cmx->matrix_max,
                                                                  cmx->min_score, cmx->s2);
    } else {
        TB_CK(cudaEventRecord(ctx.ev[0], stream));
        TB_CK(dispatch_stripes(mode, false, p, S, stream, dev));
        TB_CK(cudaEventRecord(ctx.ev[1], stream));
        switch (mode) {
        case MODE_SW: tb_pair_hits_kernel<MODE_SW><<<(n + 63) / 64, 64, 0, stream>>>(p, d_scores, d_qend, d_tend); break;
        case MODE_NW: tb_pair_hits_kernel<MODE_NW><<<(n + 63) / 64, 64, 0, stream>>>(p, d_scores, d_qend, d_tend); break;
        case MODE_HW: tb_pair_hits_kernel<MODE_HW><<<(n + 63) / 64, 64, 0, stream>>>(p, d_scores, d_qend, d_tend); break;
        case MODE_OV: tb_pair_hits_kernel<MODE_OV><<<(n + 63) / 64, 64, 0, stream>>>(p, d_scores, d_qend, d_tend); break;
        default: tb_pair_hits_kernel<MODE_SHW><<<(n + 63) / 64, 64, 0, stream>>>(p, d_scores, d_qend, d_tend); break;
        }
    }
    TB_CK(cudaGetLastError());
    TB_CK(grow_pinned(ctx.h_total, ctx.ch_total, 16));
    TB_CK(cudaMemcpyAsync(ctx.h_total, ctx.d_prog, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    TB_CK(cudaStreamSynchronize(stream));
    if (*(const uint32_t *)ctx.h_total) return fail(HY_ERR_TIMEOUT);
    float ms = 0.f;
    TB_CK(cudaEventElapsedTime(&ms, ctx.ev[0], ctx.ev[1]));
    if (kernel_ms) *kernel_ms += ms;
    return fail(HY_OK);
}

void tb_context_timing(void *ctx, double out[5]) {
    const TbContext *c = (const TbContext *)ctx;
    out[0] = c ? c->fill_ms : 0.0;
    out[1] = c ? c->walk_ms : 0.0;
    out[2] = c ? c->device_ms : 0.0;
    out[3] = c ? c->call_ms : 0.0;
    out[4] = c ? c->cells : 0.0;
}

uint64_t tb_context_launches(void *ctx) {
    if (!ctx) return 0;
    TbContext *c = (TbContext *)ctx;
    const uint64_t v = c->launches;
    c->launches = 0;
    return v;
}

}  // namespace hy

// ---- score2 (src/kernel.rs:741-792) --------------------------------------------------------------
//
// align_pair_position_max over many pairs runs in pairs.cu (the pair kernel's column-maxima form);
// its long pairs take this file's stripe kernel through tb_long_pair_scores.

extern "C" {

int hy_score2(const int32_t *colmax, uint64_t n, int32_t best_score, uint64_t best_target_end,
              int32_t matrix_max, int32_t min_score, int32_t *score, uint64_t *pos) {
    if (matrix_max <= 0 || (n && !colmax)) return 0;
    const int64_t w = ((int64_t)std::max(best_score, 0) + matrix_max - 1) / matrix_max;
    const int64_t te = (int64_t)best_target_end, low = te - w, high = te + w;
    bool have = false, open = false;
    int32_t bs = 0, cs = 0;
    uint64_t bp = 0, cp = 0;
    auto consider = [&](int32_t sc, uint64_t p) {
        const int64_t q = (int64_t)p;
        if ((q < low || q > high) && (!have || sc > bs)) {
            have = true;
            bs = sc;
            bp = p;
        }
    };
    for (uint64_t i = 0; i < n; ++i) {
        const int32_t v = colmax[i];
        if (v < min_score) continue;
        if (open && cp + 1 == i) {
            if (cs < v) {
                cs = v;
                cp = i;
            }
        } else {
            if (open) consider(cs, cp);
            open = true;
            cs = v;
            cp = i;
        }
    }
    if (open) consider(cs, cp);
    if (have) {
        if (score) *score = bs;
        if (pos) *pos = bp;
    }
    return have ? 1 : 0;
}

}  // extern "C"
