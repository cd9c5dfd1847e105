// Divergence statistics without any allocation: the block partials of the
// two-pass reduction live in a fixed array of this library instead of a
// caller-provided workspace.
//
// Who needs this: callers that cannot allocate device memory at the moment
// they ask for the statistics -- a host application that has handed all
// device memory to its own pool, a real-time/plugin callback in which a
// cudaMalloc (which may synchronise the device) is not allowed, or a plain C
// caller that holds only the two input pointers and an output pointer and has
// no allocator of its own.
//
// What it costs: the array below (kStaticBlocks * 6 doubles = 56,832 bytes)
// is reserved on every GPU that loads this library, for as long as the library
// stays loaded. All calls share it, so two calls whose kernels overlap on the
// GPU (e.g. issued on different streams without ordering) race on it. Calls
// ordered on one stream are fine: each call overwrites every partial it later
// reads, so nothing carries over from the previous call.
#include <mutex>

#include "ffx_host.cuh"

namespace ffx {
namespace {

constexpr int kStaticThreads = 256;
constexpr int kStaticBlocks = 1184;          // 8 blocks per SM on a 148-SM B200
constexpr int64_t kStaticMaxCount = 2147483647;  // the count is passed to the kernels as int

static __device__ __align__(256) double g_partials[kStaticBlocks * 6];

__device__ __forceinline__ double wsum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double wmax(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Pass 1: block b writes its six partials to part[6b .. 6b+5] (every block
// writes all six, so the array needs no clearing between calls).
__global__ void __launch_bounds__(kStaticThreads) static_partial_kernel(int n, const float* __restrict__ b,
                                                                        const float* __restrict__ a, double* part) {
    double s[6] = {0, 0, 0, 0, 0, 0};   // b^2, a^2, max|b|, max|a|, sum b, sum a
    // 64-bit loop index: i + stride must not wrap for n close to 2^31 - 1
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double vb = b[i], va = a[i];
        s[0] += vb * vb; s[1] += va * va;
        s[2] = fmax(s[2], fabs(vb)); s[3] = fmax(s[3], fabs(va));
        s[4] += vb; s[5] += va;
    }
    __shared__ double sh[6][kStaticThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < 6; ++k) {
        const double v = (k == 2 || k == 3) ? wmax(s[k]) : wsum(s[k]);
        if (lane == 0) sh[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        double v = sh[k][0];
        for (int w = 1; w < kStaticThreads / 32; ++w) v = (k == 2 || k == 3) ? fmax(v, sh[k][w]) : v + sh[k][w];
        part[blockIdx.x * 6 + k] = v;
    }
}

// Pass 2: combine the partials in block order (deterministic).
__global__ void static_final_kernel(int nblocks, const double* part, int n, double* out) {
    const int k = threadIdx.x;
    if (k >= 6) return;
    double v = part[k];
    for (int b = 1; b < nblocks; ++b) {
        const double x = part[b * 6 + k];
        v = (k == 2 || k == 3) ? fmax(v, x) : v + x;
    }
    out[k] = v;
    if (k == 0) { out[6] = (double)n; out[7] = 0.0; }
}

// Device address of g_partials, looked up once per device with that device
// current (host code cannot use the symbol itself as a device pointer).
constexpr int kMaxDevices = 64;
std::mutex g_lock;
void* g_addr[kMaxDevices] = {};

int partials_address(double** out) {
    int dev = 0;
    int e = cuda_status(cudaGetDevice(&dev), "ffx_divergence_stats_static: cudaGetDevice");
    if (e) return e;
    if (dev < 0 || dev >= kMaxDevices) return fail(FFX_ERR_INVALID, "ffx_divergence_stats_static: device %d", dev);
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cuda_status(cudaGetSymbolAddress(&p, g_partials), "ffx_divergence_stats_static: cudaGetSymbolAddress");
        if (e) return e;
        g_addr[dev] = p;
    }
    *out = static_cast<double*>(g_addr[dev]);
    return FFX_OK;
}

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" int ffx_divergence_stats_static(int64_t count, const float* before, const float* after, double* out,
                                           void* stream) {
    FFX_REQUIRE(before && after && out, "ffx_divergence_stats_static: NULL pointer");
    FFX_REQUIRE(count >= 1 && count <= kStaticMaxCount,
                "ffx_divergence_stats_static: count %lld outside [1, %lld] (this variant takes a 32-bit count; "
                "use ffx_divergence_stats with a workspace for larger fields)",
                (long long)count, (long long)kStaticMaxCount);
    double* part = nullptr;
    int e = partials_address(&part);
    if (e) return e;
    const int n = (int)count;
    int64_t want = (count + kStaticThreads - 1) / kStaticThreads;
    const int nblocks = (int)(want < kStaticBlocks ? want : kStaticBlocks);
    cudaStream_t s = as_stream(stream);
    static_partial_kernel<<<nblocks, kStaticThreads, 0, s>>>(n, before, after, part);
    e = launch_status("static_partial_kernel");
    if (e) return e;
    static_final_kernel<<<1, 32, 0, s>>>(nblocks, part, n, out);
    return launch_status("static_final_kernel");
}
