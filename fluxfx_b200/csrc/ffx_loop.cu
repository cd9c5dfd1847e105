// Device-side solve loops of the single-domain solvers: a CUDA graph whose
// WHILE node repeats a captured body (one V-cycle, the residual maximum and
// the decision) until the residual meets the tolerance or the cycle budget is
// spent, so a pressure solve to a tolerance needs no host round trip. The loop
// of backend/solid_multigrid.py:67-76 with the tolerance test of the
// extension (while cycles < max and max|r| > tol * max|rhs|: cycle) decided on
// the device in FP64.
//
// Use: ffx_loop_begin starts capturing the caller's stream; the caller issues
// the passes before the loop, ending with ffx_loop_decide (which sets the loop
// condition); ffx_loop_while adds the WHILE node and returns a stream that
// captures its body, where the caller issues one iteration ending with
// ffx_loop_decide again; ffx_loop_end_while closes the body; the caller may
// issue passes after the loop on its stream; ffx_loop_end instantiates. Every
// launch of the result (ffx_loop_launch) runs the whole solve.
#include <cmath>
#include <cstdint>

#include "ffx_host.cuh"

struct FfxLoop {
    cudaStream_t st = nullptr;       // the caller's stream (capturing between begin and end)
    cudaStream_t side = nullptr;     // captures the WHILE body
    cudaGraph_t graph = nullptr;
    cudaGraphConditionalHandle handle = 0;
    cudaGraphNode_t node = nullptr;
    cudaGraphExec_t exec = nullptr;
    int in_body = 0;
};

namespace ffx {
namespace {

// counters[0]: cycles of the current solve (zeroed by ffx_loop_reset_counter),
// counters[1]: cycles of all solves, counters[2]: decisions taken.
__global__ void loop_decide_kernel(const float* rmax, const float* scale, double tol, int max_cycles,
                                   int* counters, cudaGraphConditionalHandle handle) {
    const double r = (double)*rmax, s = (double)*scale;
    const bool go = counters[0] < max_cycles && s > 0.0 && r > tol * s;
    if (go) {
        counters[0] += 1;
        counters[1] += 1;
    }
    counters[2] += 1;
    cudaGraphSetConditional(handle, go ? 1u : 0u);
}

__global__ void loop_reset_kernel(int* counters) { counters[0] = 0; }

// p = 0 where the right-hand side is all zero (scale == 0): the solve of a
// zero right-hand side is zero pressure, whatever the warm start held.
__global__ void zero_if_unscaled_kernel(const float* scale, float* p, int64_t n) {
    if (*scale != 0.f) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = 0.f;
}

// Device-side time-step rule (the adaptive step of backend/timestep.py:35-53 in
// the form the workloads use): clock = {dt, previous dt}, time in FP64.
// previous dt = dt; time += dt; dt = min(dt_max, cfl * cell / max|u|) in FP64
// from the face maxima of the step's corrected velocity (dt_max when they are
// all zero; a non-finite velocity has a huge finite maximum, so dt stays > 0).
__global__ void next_dt_kernel(const float* maxima, float* clock, double* time, double cell, double cfl,
                               double dt_max) {
    const float dt = clock[0];
    time[0] += (double)dt;
    clock[1] = dt;
    const float umax = fmaxf(fmaxf(maxima[0], maxima[1]), maxima[2]);
    const double r = cfl * cell / (double)umax;
    clock[0] = (float)(umax > 0.f ? (r < dt_max ? r : dt_max) : dt_max);
}

// p *= dt / previous dt when they differ by more than 1e-6 relative (the
// impulse warm start of backend/pressure.py:63-75), decided in FP64 on the
// device; no previous step (previous dt <= 0) leaves p unchanged.
__global__ void scale_by_ratio_kernel(int64_t n, float* p, const float* clock) {
    const float dt = clock[0], prev = clock[1];
    if (!(prev > 0.f)) return;
    const double ratio = (double)dt / (double)prev;
    if (!(fabs(ratio - 1.0) > 1e-6)) return;
    const float f = (float)ratio;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = p[i] * f;
}

// Warm start extrapolated linearly in time. The impulse pressure of a solve is
// dt times the pressure per unit time, P. With P1 = p / d1 (the last solve,
// d1 = previous dt) and P2 = hist (the solve before it, stored by the previous
// call), the next solve (dt = d0) starts from d0 * (P1 + beta * (d0 / d1) *
// (P1 - P2)), and hist becomes P1. `first` (no older solve): P2 is not used,
// so p takes the ratio rule of scale_by_ratio_kernel and hist becomes P1.
// Coefficients in FP64, the update in FP32, four cells per thread.
__device__ __forceinline__ void extrapolate_cell(float& p, float& h, float c1, float c2, float inv, bool first) {
    const float v = p;
    p = first ? v * c1 : c1 * v - c2 * h;
    h = v * inv;
}

__global__ void extrapolate_kernel(int64_t n, float* p, float* hist, const float* clock, float beta, int first) {
    const float dt = clock[0], prev = clock[1];
    if (!(prev > 0.f)) return;
    const double d0 = dt, d1 = prev, r = d0 / d1;
    const float inv = (float)(1.0 / d1);
    const float c1 = first ? (fabs(r - 1.0) > 1e-6 ? (float)r : 1.f) : (float)(d0 * (1.0 + (double)beta * r) / d1);
    const float c2 = first ? 0.f : (float)(d0 * (double)beta * r);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t quads = n / 4;
    float4* p4 = reinterpret_cast<float4*>(p);
    float4* h4 = reinterpret_cast<float4*>(hist);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < quads; i += stride) {
        float4 v = p4[i], h = first ? make_float4(0.f, 0.f, 0.f, 0.f) : h4[i];
        extrapolate_cell(v.x, h.x, c1, c2, inv, first);
        extrapolate_cell(v.y, h.y, c1, c2, inv, first);
        extrapolate_cell(v.z, h.z, c1, c2, inv, first);
        extrapolate_cell(v.w, h.w, c1, c2, inv, first);
        p4[i] = v;
        h4[i] = h;
    }
    for (int64_t i = 4 * quads + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float h = first ? 0.f : hist[i];
        extrapolate_cell(p[i], h, c1, c2, inv, first);
        hist[i] = h;
    }
}

// Quadratic form of the same start, through the last three solves. P1 = p / d1
// and the two stored quantities P2 = h_new (solve before) and P3 = h_old (the
// one before that), taken at times 0, -d1 and -d1 - d2; the Lagrange quadratic
// through them, evaluated at d0, gives Q, and the start is
// d0 * (P1 + beta * (Q - P1)). `have` = stored solves (0: the ratio rule; 1:
// the linear form with h_new; 2: the quadratic). Every form writes P1 over
// h_old (which becomes the newest stored quantity; the caller swaps the roles)
// and d1 into dprev_w; d2 is read from dprev_r (written by the previous call).
// Coefficients in FP64, the update ((a0 v + a1 h_new) + a2 h_old) in FP32.
__global__ void extrapolate2_kernel(int64_t n, float* p, const float* h_new, float* h_old, const float* clock,
                                    const float* dprev_r, float* dprev_w, float beta, int have) {
    const float dt = clock[0], prev = clock[1];
    if (!(prev > 0.f)) return;
    const double d0 = dt, d1 = prev, r = d0 / d1, b = beta;
    float a0, a1 = 0.f, a2 = 0.f;
    if (have == 0) {
        a0 = fabs(r - 1.0) > 1e-6 ? (float)r : 1.f;
    } else if (have == 1) {
        a0 = (float)(d0 * (1.0 + b * r) / d1);
        a1 = (float)(-d0 * b * r);
    } else {
        const double d2 = *dprev_r;
        const double l0 = (d0 + d1) * (d0 + d1 + d2) / (d1 * (d1 + d2));
        const double l1 = -d0 * (d0 + d1 + d2) / (d1 * d2);
        const double l2 = d0 * (d0 + d1) / ((d1 + d2) * d2);
        a0 = (float)(d0 * (1.0 + b * (l0 - 1.0)) / d1);
        a1 = (float)(d0 * b * l1);
        a2 = (float)(d0 * b * l2);
    }
    const float inv = (float)(1.0 / d1);
    auto cell = [&](float& v, float h1, float& h2) {
        const float x = v;
        v = have == 0 ? x * a0 : (have == 1 ? a0 * x + a1 * h1 : (a0 * x + a1 * h1) + a2 * h2);
        h2 = x * inv;
    };
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t quads = n / 4;
    float4* p4 = reinterpret_cast<float4*>(p);
    const float4* n4 = reinterpret_cast<const float4*>(h_new);
    float4* o4 = reinterpret_cast<float4*>(h_old);
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < quads; i += stride) {
        float4 v = p4[i];
        const float4 a = have >= 1 ? n4[i] : zero;
        float4 b = have >= 2 ? o4[i] : zero;
        cell(v.x, a.x, b.x);
        cell(v.y, a.y, b.y);
        cell(v.z, a.z, b.z);
        cell(v.w, a.w, b.w);
        p4[i] = v;
        o4[i] = b;
    }
    for (int64_t i = 4 * quads + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float v = p[i], b = have >= 2 ? h_old[i] : 0.f;
        cell(v, have >= 1 ? h_new[i] : 0.f, b);
        p[i] = v;
        h_old[i] = b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *dprev_w = prev;
}

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" {

int ffx_loop_begin(void* stream, FfxLoop** out) {
    FFX_REQUIRE(stream && out, "ffx_loop_begin: a stream (not the legacy default stream) and an output are required");
    FfxLoop* L = new FfxLoop;
    L->st = as_stream(stream);
    int rc = cuda_status(cudaStreamCreateWithFlags(&L->side, cudaStreamNonBlocking), "ffx_loop_begin: stream");
    if (!rc) rc = cuda_status(cudaStreamBeginCapture(L->st, cudaStreamCaptureModeRelaxed), "ffx_loop_begin: capture");
    if (!rc) {
        cudaStreamCaptureStatus status;
        rc = cuda_status(cudaStreamGetCaptureInfo(L->st, &status, nullptr, &L->graph, nullptr, nullptr),
                         "ffx_loop_begin: capture info");
        if (!rc && status != cudaStreamCaptureStatusActive) rc = fail(FFX_ERR_CUDA, "ffx_loop_begin: not capturing");
    }
    if (!rc)
        rc = cuda_status(cudaGraphConditionalHandleCreate(&L->handle, L->graph, 0, cudaGraphCondAssignDefault),
                         "ffx_loop_begin: conditional handle");
    if (rc) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(L->st, &g);
        if (g) cudaGraphDestroy(g);
        if (L->side) cudaStreamDestroy(L->side);
        delete L;
        return rc;
    }
    *out = L;
    return FFX_OK;
}

int ffx_loop_decide(FfxLoop* L, const float* rmax, const float* scale, double tol, int32_t max_cycles,
                    int32_t* counters, void* stream) {
    FFX_REQUIRE(L && rmax && scale && counters && max_cycles >= 0 && tol >= 0.0, "ffx_loop_decide: invalid arguments");
    loop_decide_kernel<<<1, 1, 0, as_stream(stream)>>>(rmax, scale, tol, max_cycles, counters, L->handle);
    return launch_status("loop_decide_kernel");
}

int ffx_loop_reset_counter(int32_t* counters, void* stream) {
    FFX_REQUIRE(counters, "ffx_loop_reset_counter: invalid arguments");
    loop_reset_kernel<<<1, 1, 0, as_stream(stream)>>>(counters);
    return launch_status("loop_reset_kernel");
}

int ffx_zero_if_unscaled(const float* scale, float* p, int64_t count, void* stream) {
    FFX_REQUIRE(scale && p && count >= 1, "ffx_zero_if_unscaled: invalid arguments");
    const int64_t want = (count + 255) / 256;
    zero_if_unscaled_kernel<<<(unsigned)(want < 148 * 8 ? want : 148 * 8), 256, 0, as_stream(stream)>>>(scale, p, count);
    return launch_status("zero_if_unscaled_kernel");
}

int ffx_next_dt(const float* maxima, float* clock, double* time, double cell, double cfl, double dt_max,
                void* stream) {
    FFX_REQUIRE(maxima && clock && time && cell > 0.0 && cfl > 0.0 && dt_max > 0.0 && dt_max <= 0.1,
                "ffx_next_dt: invalid arguments (cell, cfl > 0; dt_max in (0, 0.1])");
    next_dt_kernel<<<1, 1, 0, as_stream(stream)>>>(maxima, clock, time, cell, cfl, dt_max);
    return launch_status("next_dt_kernel");
}

int ffx_scale_by_ratio(int64_t count, float* p, const float* clock, void* stream) {
    FFX_REQUIRE(count >= 1 && p && clock, "ffx_scale_by_ratio: invalid arguments");
    const int64_t want = (count + 255) / 256;
    scale_by_ratio_kernel<<<(unsigned)(want < 148 * 8 ? want : 148 * 8), 256, 0, as_stream(stream)>>>(count, p, clock);
    return launch_status("scale_by_ratio_kernel");
}

int ffx_extrapolate_pressure2(int64_t count, float* p, const float* h_new, float* h_old, const float* clock,
                              const float* dprev_r, float* dprev_w, float beta, int32_t have, void* stream) {
    FFX_REQUIRE(count >= 1 && p && h_new && h_old && clock && dprev_r && dprev_w && p != h_new && p != h_old &&
                    h_new != h_old && dprev_r != dprev_w && std::isfinite(beta) && beta >= 0.f && beta <= 1.f &&
                    have >= 0 && have <= 2,
                "ffx_extrapolate_pressure2: invalid arguments (beta in [0, 1], have 0..2, distinct buffers)");
    FFX_REQUIRE(reinterpret_cast<uintptr_t>(p) % 16 == 0 && reinterpret_cast<uintptr_t>(h_new) % 16 == 0 &&
                    reinterpret_cast<uintptr_t>(h_old) % 16 == 0,
                "ffx_extrapolate_pressure2: p, h_new and h_old must be 16-byte aligned");
    const int64_t want = (count / 4 + 255) / 256;
    const int64_t blocks = want < 1 ? 1 : (want < 148 * 8 ? want : 148 * 8);
    extrapolate2_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(
        count, p, h_new, h_old, clock, dprev_r, dprev_w, beta, have);
    return launch_status("extrapolate2_kernel");
}

int ffx_extrapolate_pressure(int64_t count, float* p, float* hist, const float* clock, float beta, int32_t first,
                             void* stream) {
    FFX_REQUIRE(count >= 1 && p && hist && clock && p != hist && std::isfinite(beta) && beta >= 0.f && beta <= 1.f &&
                    (first == 0 || first == 1),
                "ffx_extrapolate_pressure: invalid arguments (beta in [0, 1], first 0 or 1, distinct buffers)");
    FFX_REQUIRE(reinterpret_cast<uintptr_t>(p) % 16 == 0 && reinterpret_cast<uintptr_t>(hist) % 16 == 0,
                "ffx_extrapolate_pressure: p and hist must be 16-byte aligned");
    const int64_t want = (count / 4 + 255) / 256;
    const int64_t blocks = want < 1 ? 1 : (want < 148 * 8 ? want : 148 * 8);
    extrapolate_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(count, p, hist, clock, beta, first);
    return launch_status("extrapolate_kernel");
}

int ffx_loop_while(FfxLoop* L, void** body_stream) {
    FFX_REQUIRE(L && body_stream && !L->in_body && !L->node, "ffx_loop_while: one loop per graph, after begin");
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    int rc = cuda_status(cudaStreamGetCaptureInfo(L->st, &status, nullptr, &graph, &deps, &ndeps),
                         "ffx_loop_while: capture info");
    if (rc) return rc;
    cudaGraphNodeParams params = {cudaGraphNodeTypeConditional};
    params.conditional.handle = L->handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    rc = cuda_status(cudaGraphAddNode(&L->node, graph, deps, ndeps, &params), "ffx_loop_while: node");
    if (rc) return rc;
    cudaGraph_t body = params.conditional.phGraph_out[0];
    rc = cuda_status(cudaStreamBeginCaptureToGraph(L->side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
                     "ffx_loop_while: body capture");
    if (rc) return rc;
    L->in_body = 1;
    *body_stream = L->side;
    return FFX_OK;
}

int ffx_loop_end_while(FfxLoop* L) {
    FFX_REQUIRE(L && L->in_body, "ffx_loop_end_while: no open loop body");
    cudaGraph_t captured = nullptr;
    int rc = cuda_status(cudaStreamEndCapture(L->side, &captured), "ffx_loop_end_while: end of body capture");
    L->in_body = 0;
    if (rc) return rc;
    return cuda_status(cudaStreamUpdateCaptureDependencies(L->st, &L->node, 1, cudaStreamSetCaptureDependencies),
                       "ffx_loop_end_while: dependencies");
}

int ffx_loop_end(FfxLoop* L) {
    FFX_REQUIRE(L && !L->in_body && L->node && !L->exec, "ffx_loop_end: the loop body must be closed");
    cudaGraph_t graph = nullptr;
    int rc = cuda_status(cudaStreamEndCapture(L->st, &graph), "ffx_loop_end: end capture");
    if (!rc) rc = cuda_status(cudaGraphInstantiate(&L->exec, graph, 0), "ffx_loop_end: instantiate");
    if (graph) cudaGraphDestroy(graph);
    return rc;
}

int ffx_loop_launch(FfxLoop* L, void* stream) {
    FFX_REQUIRE(L && L->exec, "ffx_loop_launch: not instantiated");
    return cuda_status(cudaGraphLaunch(L->exec, as_stream(stream)), "ffx_loop_launch");
}

int ffx_loop_destroy(FfxLoop* L) {
    if (!L) return FFX_OK;
    if (L->in_body) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(L->side, &g);
    }
    if (L->exec) cudaGraphExecDestroy(L->exec);
    if (L->side) cudaStreamDestroy(L->side);
    delete L;
    return FFX_OK;
}

}  // extern "C"
