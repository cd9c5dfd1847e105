// Host-side helpers shared by the entry points: thread-local error text,
// argument checks and launch-status mapping.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>

#include "ffx_common.cuh"

namespace ffx {

std::string& last_error_buffer();

inline int fail(int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    last_error_buffer() = buf;
    return status;
}

inline int launch_status(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(FFX_ERR_LAUNCH, "%s: %s", what, cudaGetErrorString(e));
    return FFX_OK;
}

inline int cuda_status(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return fail(FFX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return FFX_OK;
}

// Whether launch_pdl launches with programmatic stream serialization
// (ffx_set_dependent_launch; on by default).
extern int g_pdl;

// Launches a kernel that begins with pdl_enter() so that it may be scheduled
// while the kernel before it in the stream finishes; launch errors map like
// launch_status.
template <typename... KArgs, typename... Args>
inline int launch_pdl(const char* what, void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st,
                      Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g_pdl ? 1 : 0;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(FFX_ERR_LAUNCH, "%s: %s", what, cudaGetErrorString(e));
    }
    return launch_status(what);
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Extents within [2^-18, 2^30]: with at most 4096 cells per axis every
// extent, cell count and spacing then lies in [2^-30, 2^30], the divisor range
// of the kernels' division by grid constants.
inline bool extent_ok(float e) { return e >= 0x1p-18f && e <= 0x1p30f; }

inline bool grid_ok(const FfxGrid* g) {
    return g && g->nx >= 1 && g->ny >= 1 && g->nz >= 1 && g->nx <= 4096 && g->ny <= 4096 && g->nz <= 4096 &&
           extent_ok(g->ex) && extent_ok(g->ey) && extent_ok(g->ez) &&
           (int64_t)(g->nx + 1) * (g->ny + 1) * (g->nz + 1) < (int64_t(1) << 31);
}

inline bool shape_ok(const int32_t n[3]) {
    return n && n[0] >= 1 && n[1] >= 1 && n[2] >= 1 && (int64_t)n[0] * n[1] * n[2] < (int64_t(1) << 31);
}

inline bool storage_ok(int s) { return s == FFX_F32 || s == FFX_BF16; }

inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// Dispatch a templated launcher on the storage type.
#define FFX_DISPATCH_STORAGE(storage, T, ...)            \
    do {                                                  \
        if ((storage) == FFX_F32) {                       \
            using T = float;                              \
            __VA_ARGS__;                                  \
        } else {                                          \
            using T = __nv_bfloat16;                      \
            __VA_ARGS__;                                  \
        }                                                 \
    } while (0)

#define FFX_REQUIRE(cond, ...)                                 \
    do {                                                       \
        if (!(cond)) return ::ffx::fail(FFX_ERR_INVALID, __VA_ARGS__); \
    } while (0)

}  // namespace ffx
