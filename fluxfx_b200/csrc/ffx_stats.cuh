// Deterministic FP64 divergence statistics (physics/pressure.py:70-80): a
// two-pass reduction shared by ffx_divergence_stats (partials in a caller
// workspace) and ffx_divergence_stats_static (partials in a library array).
// Both entry points launch these same kernels with the same block count for a
// given n, so their results are bit-identical.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ffx {
namespace stats {
// Internal linkage: every translation unit that includes this header gets its
// own copy of the kernels (the library is built without relocatable device code).
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1184;   // 8 x 148 SMs

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Pass 1: block b writes its six partials (sum b^2, sum a^2, max|b|, max|a|,
// sum b, sum a) to part[6b .. 6b+5]. Every block writes all six, so the
// partials need no clearing between calls.
__global__ void __launch_bounds__(kThreads) partial_kernel(int64_t n, const float* __restrict__ b,
                                                           const float* __restrict__ a, double* part) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double vb = b[i], va = a[i];
        s[0] += vb * vb; s[1] += va * va;
        s[2] = fmax(s[2], fabs(vb)); s[3] = fmax(s[3], fabs(va));
        s[4] += vb; s[5] += va;
    }
    __shared__ double sh[6][kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < 6; ++k) {
        const double v = (k == 2 || k == 3) ? warp_max(s[k]) : warp_sum(s[k]);
        if (lane == 0) sh[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        double v = sh[k][0];
        for (int w = 1; w < kThreads / 32; ++w) v = (k == 2 || k == 3) ? fmax(v, sh[k][w]) : v + sh[k][w];
        part[(int64_t)blockIdx.x * 6 + k] = v;
    }
}

// Pass 2: one warp combines the partials in block order; out[6] = n, out[7] = 0.
__global__ void final_kernel(int nblocks, const double* part, int64_t n, double* out) {
    const int k = threadIdx.x;
    if (k >= 6) return;
    double v = part[k];
    for (int b = 1; b < nblocks; ++b) {
        const double x = part[(int64_t)b * 6 + k];
        v = (k == 2 || k == 3) ? fmax(v, x) : v + x;
    }
    out[k] = v;
    if (k == 0) { out[6] = (double)n; out[7] = 0.0; }
}

// Blocks of pass 1 for n values (1 .. kMaxBlocks).
inline int blocks(int64_t n) {
    const int64_t b = (n + kThreads - 1) / kThreads;
    return (int)(b < kMaxBlocks ? (b < 1 ? 1 : b) : kMaxBlocks);
}

// Both passes on `stream`; `part` holds 6 * blocks(n) doubles.
inline void launch(int64_t n, const float* before, const float* after, double* part, double* out,
                   cudaStream_t stream) {
    const int nb = blocks(n);
    partial_kernel<<<nb, kThreads, 0, stream>>>(n, before, after, part);
    final_kernel<<<1, 32, 0, stream>>>(nb, part, n, out);
}

}  // namespace
}  // namespace stats
}  // namespace ffx
