// roofline.cu -- the packed-int16 DPX roofline probe: the scan kernel's per-cell instruction mix
// run register resident, with no memory traffic, shuffles or profile loads. Per cell pair that is
// three DPX ops on the ALU pipe (__viaddmax for E and F, __vimax3_relu for H) plus half a
// __vimax3 for the running maximum, and three __vadd2 on the FMA pipe (the diagonal's two profile
// words and G = H - go). The profile words stay in registers (the same for every column), so the
// probe carries no load or register-move overhead: its cell rate is an upper bound for the scan.
#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>

#include "host_common.h"

namespace hy {

template <int R>
__global__ void __launch_bounds__(256) dpx_probe_kernel(int cols, uint32_t seed, uint32_t *sink) {
    const uint32_t negge = 0xffffffffu, neggo = 0xfff5fff5u;
    uint32_t Gp[R], E[R], PA[R], PB[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        Gp[r] = 0xfff5fff5u;
        E[r] = 0x80018001u;
        PA[r] = (seed + threadIdx.x * 7u + r * 13u) & 0x7u;
        PB[r] = ((seed + threadIdx.x * 5u + r * 11u) & 0x7u) << 16;
    }
    uint32_t best = 0, diag = 0xfff5fff5u, up = 0xfff5fff5u, fup = 0x80018001u;
    for (int j = 0; j < cols; ++j) {
        uint32_t g_up = up, f = fup, gd = diag, hprev = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            E[r] = __viaddmax_s16x2(E[r], negge, Gp[r]);
            f = __viaddmax_s16x2(f, negge, g_up);
            const uint32_t d = __vadd2(__vadd2(gd, PA[r]), PB[r]);
            const uint32_t h = __vimax3_s16x2_relu(d, E[r], f);
            gd = Gp[r];
            const uint32_t g = __vadd2(h, neggo);
            Gp[r] = g;
            g_up = g;
            if (r & 1)
                best = __vimax3_s16x2(best, hprev, h);
            else
                hprev = h;
        }
        diag = up;
        up = g_up ^ (uint32_t)j;  // keeps the column recurrence live across iterations
        fup = f;
    }
    if (best == 0xdeadbeefu) sink[threadIdx.x] = best;  // never true; defeats dead-code removal
    if (threadIdx.x == 0 && blockIdx.x == 0) sink[0] = best & 1u;
}

// The int32 form (one cell per lane op): the same recurrence with __viaddmax_s32 for E and F,
// __vimax3_s32_relu for H, a plain add for the diagonal and G, and a __vimax3_s32 running maximum
// every other row. The roofline of the int32 kernels (the traceback fill, the int32 scan items).
template <int R>
__global__ void __launch_bounds__(256) dpx_probe_i32_kernel(int cols, uint32_t seed, int32_t *sink) {
    const int32_t negge = -1, neggo = -11;
    int32_t Gp[R], E[R], P[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        Gp[r] = -11;
        E[r] = -(1 << 29);
        P[r] = (int32_t)((seed + threadIdx.x * 7u + r * 13u) & 0x7u) - 3;
    }
    int32_t best = 0, diag = -11, up = -11, fup = -(1 << 29);
    for (int j = 0; j < cols; ++j) {
        int32_t g_up = up, f = fup, gd = diag, hprev = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            E[r] = __viaddmax_s32(E[r], negge, Gp[r]);
            f = __viaddmax_s32(f, negge, g_up);
            const int32_t d = gd + P[r];
            const int32_t h = __vimax3_s32_relu(d, E[r], f);
            gd = Gp[r];
            const int32_t g = h + neggo;
            Gp[r] = g;
            g_up = g;
            if (r & 1)
                best = __vimax3_s32(best, hprev, h);
            else
                hprev = h;
        }
        diag = up;
        up = g_up ^ j;
        fup = f;
    }
    if (best == 0x5eadbeef) sink[threadIdx.x] = best;
    if (threadIdx.x == 0 && blockIdx.x == 0) sink[0] = best & 1;
}

// The packed-int8 form (four cells per 32-bit lane op, the reference's i8 lanes restated with the
// SIMD-video intrinsics): saturating __vsubss4 / __vaddss4 for the gaps and the diagonal,
// __vmaxs4 for E, F, H (with a max against 0 for the local floor) and the running maximum. It
// measures whether int8x4 lanes could beat int16x2 lanes for i8-proven sequences.
template <int R>
__global__ void __launch_bounds__(256) dpx_probe_i8x4_kernel(int cols, uint32_t seed, uint32_t *sink) {
    const uint32_t ge4 = 0x01010101u, go4 = 0x0b0b0b0bu;
    uint32_t Gp[R], E[R], P[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        Gp[r] = 0xf5f5f5f5u;
        E[r] = 0x81818181u;
        P[r] = (seed + threadIdx.x * 7u + r * 13u) & 0x07070707u;
    }
    uint32_t best = 0, diag = 0xf5f5f5f5u, up = 0xf5f5f5f5u, fup = 0x81818181u;
    for (int j = 0; j < cols; ++j) {
        uint32_t g_up = up, f = fup, gd = diag;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            E[r] = __vmaxs4(__vsubss4(E[r], ge4), Gp[r]);
            f = __vmaxs4(__vsubss4(f, ge4), g_up);
            const uint32_t d = __vaddss4(gd, P[r]);
            const uint32_t h = __vmaxs4(__vmaxs4(d, E[r]), __vmaxs4(f, 0u));
            gd = Gp[r];
            const uint32_t g = __vsubss4(h, go4);
            Gp[r] = g;
            g_up = g;
            best = __vmaxs4(best, h);
        }
        diag = up;
        up = g_up ^ (uint32_t)j;
        fup = f;
    }
    if (best == 0xdeadbeefu) sink[threadIdx.x] = best;
    if (threadIdx.x == 0 && blockIdx.x == 0) sink[0] = best & 1u;
}

template <class K>
static hy_status time_probe(K launch, double cells_per_launch, double *cells_per_second) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best_ms = 1e30f;
    for (int it = 0; it < 6; ++it) {
        cudaEventRecord(a);
        launch(it);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (it > 0 && ms < best_ms) best_ms = ms;
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return fail(HY_ERR_CUDA, e);
    *cells_per_second = cells_per_launch / (best_ms * 1e-3);
    return fail(HY_OK);
}

}  // namespace hy

extern "C" hy_status hy_measure_dpx_peak_i32(double *cells_per_second) {
    using namespace hy;
    if (!cells_per_second) return fail(HY_ERR_INVALID_ARGUMENT);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int32_t *sink = nullptr;
    if (cudaMalloc(&sink, 1024 * sizeof(int32_t)) != cudaSuccess) return fail(HY_ERR_OUT_OF_MEMORY);
    constexpr int R = 16;
    const int blocks = sms * 8, threads = 256, cols = 4096;
    hy_status st = time_probe(
        [&](int it) { dpx_probe_i32_kernel<R><<<blocks, threads>>>(cols, (uint32_t)it, sink); },
        (double)blocks * threads * cols * R, cells_per_second);
    cudaFree(sink);
    return st;
}

extern "C" hy_status hy_measure_dpx_peak(double *cells_per_second) {
    using namespace hy;
    if (!cells_per_second) return fail(HY_ERR_INVALID_ARGUMENT);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t *sink = nullptr;
    if (cudaMalloc(&sink, 1024 * sizeof(uint32_t)) != cudaSuccess) return fail(HY_ERR_OUT_OF_MEMORY);
    constexpr int R = 16;
    const int blocks = sms * 8, threads = 256, cols = 4096;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best_ms = 1e30f;
    for (int it = 0; it < 6; ++it) {
        cudaEventRecord(a);
        dpx_probe_kernel<R><<<blocks, threads>>>(cols, (uint32_t)it, sink);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (it > 0 && ms < best_ms) best_ms = ms;
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return fail(HY_ERR_CUDA, e);
    const double cells = (double)blocks * threads * cols * R * 2.0;
    *cells_per_second = cells / (best_ms * 1e-3);
    return fail(HY_OK);
}

extern "C" hy_status hy_measure_dpx_peak_i8x4(double *cells_per_second) {
    using namespace hy;
    if (!cells_per_second) return fail(HY_ERR_INVALID_ARGUMENT);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t *sink = nullptr;
    if (cudaMalloc(&sink, 1024 * sizeof(uint32_t)) != cudaSuccess) return fail(HY_ERR_OUT_OF_MEMORY);
    constexpr int R = 16;
    const int blocks = sms * 8, threads = 256, cols = 1024;
    hy_status st = time_probe(
        [&](int it) { dpx_probe_i8x4_kernel<R><<<blocks, threads>>>(cols, (uint32_t)it, sink); },
        (double)blocks * threads * cols * R * 4.0, cells_per_second);
    cudaFree(sink);
    return st;
}
