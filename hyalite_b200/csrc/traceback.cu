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
//             2 F, 3 stop (local mode and H == 0); the walk's H-state rule, tie-break included
//   bit 2     E(i,j) == H(i,j-1) - gap_open  (leave the E state to H)
//   bit 3     F(i,j) == H(i-1,j) - gap_open  (leave the F state to H)
//
// Half a byte a cell instead of twelve, written once and read only along the path. Cell values
// are int32 with the reference's arithmetic (its width proof keeps every real cell exact), so each
// code equals the outcome of the reference's comparison and the walk emits the same operations.
//
// Fill kernel: one warp per (query, target) pair, each lane R consecutive query rows, lanes
// skewed one column apart (anti-diagonal wavefront); passes of 32 * R rows joined by a boundary
// row (H and F) in global memory. Codes are stored lane-major per step: step s of a pass writes 32
// lanes x R/2 bytes contiguously, so every store of the warp is one coalesced 32 * R/2-byte row.
// The fill also reduces the end cell (Best::consider, src/align.rs:281-327) over the mode's answer
// region. Walk kernel: one thread per pair follows the codes from the end cell, writing the
// operations backwards into a slot of m + n bytes; a scan and a gather compact the slots.
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "db_internal.h"
#include "host_common.h"
#include "scan_kernel.cuh"
#include "traceback_internal.h"

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
    uint32_t m, n, m_pad, slot;  // lengths, profile row stride, result index within the launch
    uint32_t rows;               // query rows per lane (R) of the fill
    uint32_t pad_;
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

template <int R, int MODE>
__global__ void __launch_bounds__(TB_BLOCK) tb_fill_kernel(TbParams P) {
    using F = ModeFlags<MODE>;
    const uint32_t warp = (blockIdx.x * TB_BLOCK + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= P.n_pairs) return;
    const TbPair pr = P.pairs[warp];
    const int m = (int)pr.m, n = (int)pr.n;
    if (m == 0 || n == 0) return;  // border-only problems: the walk kernel resolves them alone
    const int32_t go = P.go, ge = P.ge;
    int2 *B = P.bnd + pr.bnd_off;
    // Row 0: H(0, j) (src/align.rs:500-508) and F(0, j) = NEG.
    for (int j = lane; j <= n; j += 32) {
        int32_t h = 0;
        if (!F::top_free && j > 0) h = (int32_t)-tb_gap(go, ge, j);
        B[j] = make_int2(h, TB_NEG);
    }
    __syncwarp();
    const uint8_t *tq = P.t_res + pr.t_off;
    const int32_t *prof = P.prof + pr.prof_off;
    const int rpp = 32 * R;
    const int passes = (m + rpp - 1) / rpp;
    const uint64_t pass_stride = (uint64_t)(n + 31) * 32 * (R / 2);
    int32_t bs = F::local ? 0 : INT32_MIN;
    uint32_t brow = 0, bcol = 0;
    for (int p = 0; p < passes; ++p) {
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
        const int32_t *pq = prof + (i0 - 1);
        int2 nb = make_int2(0, TB_NEG);
        if (lane == 0) nb = B[1];
        int cnext = (lane == 0) ? tq[0] : 0;
        const int steps = n + 31;
        for (int s = 0; s < steps; ++s) {
            const int j = s - lane + 1;  // this lane's DP column
            int32_t up_h = __shfl_up_sync(0xffffffffu, carry_h, 1);
            int32_t up_f = __shfl_up_sync(0xffffffffu, carry_f, 1);
            const int c = cnext;
            if (lane == 0) {
                up_h = nb.x;
                up_f = nb.y;
                if (j + 1 <= n) {
                    nb = B[j + 1];
                    cnext = tq[j];
                }
            } else if (j + 1 >= 1 && j + 1 <= n) {
                cnext = tq[j];  // residue of the next step's column
            }
            if (j >= 1 && j <= n) {
                const int32_t *pc = pq + (uint64_t)c * pr.m_pad;
                int32_t sub[R];
#pragma unroll
                for (int k = 0; k < R; k += 4) {
                    const int4 v = *(const int4 *)(pc + k);
                    sub[k] = v.x;
                    sub[k + 1] = v.y;
                    sub[k + 2] = v.z;
                    sub[k + 3] = v.w;
                }
                int32_t hd = hdiag, hu = up_h, fu = up_f;
                uint32_t w0 = 0, w1 = 0;
                int32_t colmax = 0;
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    const int32_t hg = Hl[k] - go, eg = E[k] - ge;
                    const int32_t e = max(hg, eg);
                    const int32_t ug = hu - go, fg = fu - ge;
                    const int32_t f = max(ug, fg);
                    const int32_t d = hd + sub[k];
                    int32_t h = F::local ? __vimax3_s32_relu(d, e, f) : __vimax3_s32(d, e, f);
                    uint32_t code = h == e ? 1u : 2u;
                    code = h == d ? 0u : code;
                    if (F::local) code = h == 0 ? 3u : code;
                    code |= hg >= eg ? 4u : 0u;
                    code |= ug >= fg ? 8u : 0u;
                    if (k < 8) w0 |= code << (4 * k);
                    else w1 |= code << (4 * (k - 8));
                    if (F::local) colmax = max(colmax, h);
                    hd = Hl[k];
                    Hl[k] = h;
                    E[k] = e;
                    hu = h;
                    fu = f;
                }
                tb_store<R>(D + ((uint64_t)s * 32 + lane) * (R / 2), w0, w1);
                if (lane == 31 && p + 1 < passes) B[j] = make_int2(hu, fu);
                carry_h = hu;
                carry_f = fu;
                hdiag = up_h;
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
    // Warp reduction under the same order.
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
        const bool valid = F::local ? bs > 0 : bs != INT32_MIN;
        P.ends[pr.slot] = TbEnd{bs, brow, bcol, valid ? 1u : 0u};
    }
}

// The code of interior cell (i, j), i, j >= 1, in the fill's lane-major layout.
__device__ inline uint32_t tb_code(const uint8_t *D, uint32_t R, uint64_t pass_stride, uint32_t i,
                                   uint32_t j) {
    const uint32_t r = i - 1, c = j - 1;
    const uint32_t rpp = 32 * R;
    const uint32_t p = r / rpp, rr = r - p * rpp;
    const uint32_t l = rr / R, k = rr - l * R;
    const uint64_t at = (uint64_t)p * pass_stride + ((uint64_t)(c + l) * 32 + l) * (R / 2) + (k >> 1);
    return (D[at] >> (4 * (k & 1))) & 15u;
}

// The end cell (src/align.rs:309-327 over every row) and the walk (src/align.rs:345-420).
template <int MODE>
__global__ void __launch_bounds__(TB_BLOCK) tb_walk_kernel(TbParams P) {
    using F = ModeFlags<MODE>;
    const uint32_t t = blockIdx.x * TB_BLOCK + threadIdx.x;
    if (t >= P.n_pairs) return;
    const TbPair pr = P.pairs[t];
    const uint32_t m = pr.m, n = pr.n;
    const int32_t go = P.go, ge = P.ge;
    auto top = [&](uint32_t j) -> int32_t {  // H(0, j)
        return (F::top_free || j == 0) ? 0 : (int32_t)-tb_gap(go, ge, j);
    };
    auto left = [&](uint32_t i) -> int32_t {  // H(i, 0)
        return (F::left_free || i == 0) ? 0 : (int32_t)-tb_gap(go, ge, i);
    };
    // End cell: the fill's interior candidate merged with the border candidates. H(0, j) and
    // H(i, 0) never increase with j or i, so among border cells of row 0 or column 0 the one
    // nearest the corner (0, 0) wins.
    int32_t bs = INT32_MIN;
    uint32_t brow = 0, bcol = 0;
    auto consider = [&](int32_t s, uint32_t r, uint32_t c) {
        if (tb_better(s, r, c, bs, brow, bcol)) {
            bs = s;
            brow = r;
            bcol = c;
        }
    };
    if (m > 0 && n > 0) {
        const TbEnd e = P.ends[pr.slot];
        if (e.valid) consider(e.score, e.row, e.col);
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
    // Walk. State 0 H, 1 E, 2 F.
    const uint8_t *D = P.dir + pr.dir_off;
    const uint32_t R = pr.rows;
    const uint64_t pass_stride = (uint64_t)(n + 31) * 32 * (R / 2);
    const uint8_t *qs = P.q_res + pr.q_off;
    const uint8_t *ts = P.t_res + pr.t_off;
    uint8_t *slot = P.ops + pr.ops_off;
    const uint64_t cap = (uint64_t)m + n;
    uint64_t cnt = 0;
    uint32_t i = brow, j = bcol;
    int state = 0;
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
        const uint32_t code = tb_code(D, R, pass_stride, i, j);
        if (state == 0) {
            const uint32_t src = code & 3u;
            if (src == 3u) break;
            if (src == 0u) {
                if (cnt < cap) slot[cap - 1 - cnt++] = qs[i - 1] == ts[j - 1] ? 0 : 1;
                --i;
                --j;
            } else {
                state = (int)src;
            }
        } else if (state == 1) {
            if (cnt < cap) slot[cap - 1 - cnt++] = 3;
            --j;
            if (code & 4u) state = 0;
        } else {
            if (cnt < cap) slot[cap - 1 - cnt++] = 2;
            --i;
            if (code & 8u) state = 0;
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
    cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void **)&p, need);
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
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint8_t *d_q = nullptr, *d_t = nullptr, *d_dir = nullptr, *d_ops = nullptr, *d_ops_out = nullptr;
    int32_t *d_prof = nullptr, *d_matrix = nullptr;
    int2 *d_bnd = nullptr;
    TbPair *d_pairs = nullptr;
    TbEnd *d_ends = nullptr;
    hy_alignment *d_out = nullptr;
    uint64_t *d_total = nullptr;
    uint64_t c_q = 0, c_t = 0, c_dir = 0, c_ops = 0, c_ops_out = 0, c_prof = 0, c_matrix = 0, c_bnd = 0,
             c_pairs = 0, c_ends = 0, c_out = 0, c_total = 0;
    TbPair *h_pairs = nullptr;
    hy_alignment *h_out = nullptr;
    uint8_t *h_ops = nullptr;
    uint64_t *h_total = nullptr;
    uint64_t ch_pairs = 0, ch_out = 0, ch_ops = 0, ch_total = 0;
    uint64_t launches = 0;
    ~TbContext() {
        if (stream) cudaStreamSynchronize(stream);
        for (void *p : {(void *)d_q, (void *)d_t, (void *)d_dir, (void *)d_ops, (void *)d_ops_out,
                        (void *)d_prof, (void *)d_matrix, (void *)d_bnd, (void *)d_pairs, (void *)d_ends,
                        (void *)d_out, (void *)d_total})
            cudaFree(p);
        for (void *p : {(void *)h_pairs, (void *)h_out, (void *)h_ops, (void *)h_total}) cudaFreeHost(p);
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

template <int MODE>
static cudaError_t launch_walk(const TbParams &p, cudaStream_t st) {
    tb_walk_kernel<MODE><<<(p.n_pairs + TB_BLOCK - 1) / TB_BLOCK, TB_BLOCK, 0, st>>>(p);
    return cudaGetLastError();
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
};

static hy_status tb_run(TbContext &ctx, const TbRun &run, const uint32_t *idx, uint32_t n_idx,
                        hy_alignment *out, std::vector<uint8_t> *ops_host, uint8_t *ops_direct) {
    auto t_off = [&](uint32_t k) { return run.h_t_off ? run.h_t_off[k] : run.h_t_single[0]; };
    auto t_len = [&](uint32_t k) {
        return run.h_t_off ? run.h_t_off[k + 1] - run.h_t_off[k] : run.h_t_single[1];
    };
    uint64_t ops_base = 0;
    uint32_t a = 0;
    while (a < n_idx) {
        // Chunk [a, b): code bytes within TB_CHUNK_BYTES (at least one pair).
        uint32_t b = a;
        uint64_t dir = 0, bnd = 0, ops = 0;
        while (b < n_idx) {
            const uint64_t n = t_len(idx[b]);
            const uint64_t d = align16(tb_dir_bytes(run.m, n, run.R));
            if (b > a && dir + d > TB_CHUNK_BYTES) break;
            dir += d;
            bnd += n + 1;
            ops += run.m + n;
            ++b;
        }
        const uint32_t cnt = b - a;
        TB_CK(grow_pinned(ctx.h_pairs, ctx.ch_pairs, sizeof(TbPair) * cnt));
        // Launch order: longest target first (load balance); slots stay in the caller's order.
        std::vector<uint32_t> order(cnt);
        for (uint32_t x = 0; x < cnt; ++x) order[x] = x;
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t x, uint32_t y) { return t_len(idx[a + x]) > t_len(idx[a + y]); });
        uint64_t od = 0, ob = 0, oo = 0;
        std::vector<uint64_t> ops_at(cnt);
        for (uint32_t x = 0; x < cnt; ++x) {
            ops_at[x] = oo;
            oo += run.m + t_len(idx[a + x]);
        }
        for (uint32_t x = 0; x < cnt; ++x) {
            const uint32_t s = order[x], k = idx[a + s];
            TbPair &pp = ctx.h_pairs[x];
            pp.q_off = 0;
            pp.prof_off = 0;
            pp.t_off = t_off(k);
            pp.m = (uint32_t)run.m;
            pp.n = (uint32_t)t_len(k);
            pp.m_pad = run.m_pad;
            pp.slot = s;
            pp.rows = run.R;
            pp.pad_ = 0;
            pp.dir_off = od;
            od += align16(tb_dir_bytes(run.m, pp.n, run.R));
            pp.bnd_off = ob;
            ob += pp.n + 1;
            pp.ops_off = ops_at[s];
        }
        TB_CK(grow(ctx.d_pairs, ctx.c_pairs, sizeof(TbPair) * cnt));
        TB_CK(grow(ctx.d_dir, ctx.c_dir, od));
        TB_CK(grow(ctx.d_bnd, ctx.c_bnd, sizeof(int2) * ob));
        TB_CK(grow(ctx.d_ops, ctx.c_ops, oo));
        TB_CK(grow(ctx.d_ops_out, ctx.c_ops_out, oo));
        TB_CK(grow(ctx.d_ends, ctx.c_ends, sizeof(TbEnd) * cnt));
        TB_CK(grow(ctx.d_out, ctx.c_out, sizeof(hy_alignment) * cnt));
        TB_CK(grow(ctx.d_total, ctx.c_total, 16));
        TB_CK(grow_pinned(ctx.h_out, ctx.ch_out, sizeof(hy_alignment) * cnt));
        TB_CK(grow_pinned(ctx.h_total, ctx.ch_total, 16));
        TB_CK(cudaMemcpyAsync(ctx.d_pairs, ctx.h_pairs, sizeof(TbPair) * cnt, cudaMemcpyHostToDevice, ctx.stream));
        TbParams p;
        p.pairs = ctx.d_pairs;
        p.n_pairs = cnt;
        p.q_res = ctx.d_q;
        p.t_res = run.d_t_res;
        p.prof = ctx.d_prof;
        p.dir = ctx.d_dir;
        p.bnd = ctx.d_bnd;
        p.ends = ctx.d_ends;
        p.out = ctx.d_out;
        p.ops = ctx.d_ops;
        p.ops_out = ctx.d_ops_out;
        p.total = ctx.d_total;
        p.go = run.go;
        p.ge = run.ge;
        if (run.m > 0) {
            TB_CK(dispatch_fill(run.mode, run.R, p, ctx.stream));
            ++ctx.launches;
        }
        TB_CK(dispatch_walk(run.mode, p, ctx.stream));
        tb_scan_kernel<<<1, 1024, 0, ctx.stream>>>(ctx.d_out, cnt, ctx.d_total);
        TB_CK(cudaGetLastError());
        tb_gather_kernel<<<(uint32_t)(((uint64_t)cnt * 32 + TB_BLOCK - 1) / TB_BLOCK), TB_BLOCK, 0, ctx.stream>>>(p);
        TB_CK(cudaGetLastError());
        ctx.launches += 3;
        TB_CK(cudaMemcpyAsync(ctx.h_out, ctx.d_out, sizeof(hy_alignment) * cnt, cudaMemcpyDeviceToHost, ctx.stream));
        TB_CK(cudaMemcpyAsync(ctx.h_total, ctx.d_total, sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx.stream));
        TB_CK(cudaStreamSynchronize(ctx.stream));
        const uint64_t total = *ctx.h_total;
        if (ops_direct) {
            if (total) TB_CK(cudaMemcpy(ops_direct + ops_base, ctx.d_ops_out, total, cudaMemcpyDeviceToHost));
        } else {
            TB_CK(grow_pinned(ctx.h_ops, ctx.ch_ops, total));
            if (total) {
                TB_CK(cudaMemcpyAsync(ctx.h_ops, ctx.d_ops_out, total, cudaMemcpyDeviceToHost, ctx.stream));
                TB_CK(cudaStreamSynchronize(ctx.stream));
            }
            ops_host->insert(ops_host->end(), ctx.h_ops, ctx.h_ops + total);
        }
        for (uint32_t x = 0; x < cnt; ++x) {
            out[a + x] = ctx.h_out[x];
            out[a + x].ops_offset += ops_base;
        }
        ops_base += total;
        a = b;
    }
    return fail(HY_OK);
}

static hy_status tb_prepare_query(TbContext &ctx, const uint8_t *query, uint64_t m, const int32_t *d_matrix,
                                  uint64_t al, uint32_t R, uint32_t *m_pad) {
    *m_pad = (uint32_t)(tb_passes(std::max<uint64_t>(m, 1), R) * 32 * R);
    TB_CK(grow(ctx.d_q, ctx.c_q, std::max<uint64_t>(m, 1)));
    TB_CK(grow(ctx.d_prof, ctx.c_prof, sizeof(int32_t) * al * *m_pad));
    if (m) {
        TB_CK(grow_pinned(ctx.h_ops, ctx.ch_ops, m));
        memcpy(ctx.h_ops, query, m);
        TB_CK(cudaMemcpyAsync(ctx.d_q, ctx.h_ops, m, cudaMemcpyHostToDevice, ctx.stream));
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

static thread_local TbContext *g_align_ctx = nullptr;

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
    if (g_align_ctx && g_align_ctx->device != dev) {
        delete g_align_ctx;
        g_align_ctx = nullptr;
    }
    if (!g_align_ctx) {
        g_align_ctx = new TbContext;
        g_align_ctx->device = dev;
        g_align_ctx->own_stream = true;
        if (cudaStreamCreateWithFlags(&g_align_ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            delete g_align_ctx;
            g_align_ctx = nullptr;
            return fail(HY_ERR_CUDA, cudaErrorUnknown);
        }
    }
    TbContext &ctx = *g_align_ctx;
    const uint64_t mat_bytes = sizeof(int32_t) * alphabet_len * alphabet_len;
    TB_CK(grow(ctx.d_matrix, ctx.c_matrix, mat_bytes));
    TB_CK(cudaMemcpyAsync(ctx.d_matrix, matrix, mat_bytes, cudaMemcpyHostToDevice, ctx.stream));
    TB_CK(grow(ctx.d_t, ctx.c_t, std::max<uint64_t>(tlen, 1)));
    if (tlen) TB_CK(cudaMemcpyAsync(ctx.d_t, target, tlen, cudaMemcpyHostToDevice, ctx.stream));
    const uint32_t R = tb_rows(qlen, tlen);
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
    const uint32_t R = tb_rows(qlen, max_n);
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
    run.d_t_res = db->d_tb_res;
    run.h_t_off = db->tb_off.data();
    run.h_t_single = nullptr;
    ops.clear();
    return tb_run(*ctx, run, idx, n_idx, out, &ops, nullptr);
}

uint64_t tb_context_launches(void *ctx) {
    if (!ctx) return 0;
    TbContext *c = (TbContext *)ctx;
    const uint64_t v = c->launches;
    c->launches = 0;
    return v;
}

}  // namespace hy
