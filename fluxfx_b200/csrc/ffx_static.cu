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
// What it costs: the array below (stats::kMaxBlocks * 6 doubles = 56,832
// bytes) is reserved on every GPU that loads this library, for as long as the
// library stays loaded. Its size does not depend on the field: pass 1 never
// uses more than stats::kMaxBlocks blocks (a grid-stride loop covers any
// count), so every count >= 1 fits. All calls share it, so two calls whose
// kernels overlap on the GPU (e.g. issued on different streams without
// ordering) race on it. Calls ordered on one stream are fine: each call
// overwrites every partial it later reads, so nothing carries over from the
// previous call.
//
// The kernels are the ones ffx_divergence_stats launches (ffx_stats.cuh), with
// the same block count, so the two entry points return identical results.
#include <mutex>

#include "ffx_host.cuh"
#include "ffx_stats.cuh"

namespace ffx {
namespace {

static __device__ __align__(256) double g_partials[stats::kMaxBlocks * 6];

// Device address of g_partials, looked up once per device with that device
// current (host code cannot use the symbol itself as a device pointer). The
// cached address belongs to the device's primary context as it was at the
// lookup: after cudaDeviceReset (or anything else that destroys that context)
// it is stale and must not be used -- such a caller must reload the library.
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
    FFX_REQUIRE(count >= 1, "ffx_divergence_stats_static: count %lld must be at least 1", (long long)count);
    static_assert(sizeof(g_partials) == sizeof(double) * 6 * stats::kMaxBlocks, "one record per block");
    double* part = nullptr;
    int e = partials_address(&part);
    if (e) return e;
    stats::launch(count, before, after, part, out, as_stream(stream));
    return launch_status("divergence stats kernels (static partials)");
}
