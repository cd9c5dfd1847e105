// Batched passes over many independent domains of uneven sizes.
//
// A batched launch is persistent: a grid of (a multiple of) the resident
// blocks strides over a work list of tiles, where every domain contributes the
// tiles its own single-domain launch would have had (same tile coordinates,
// same per-cell arithmetic), so a domain's results are bit-identical to a
// single-domain run. The work list is a prefix table in the kernel parameters
// (BatchMap); the per-domain pass parameters are an array of descriptors in
// device memory, copied into shared memory when a block moves to another
// domain. Per-domain scalars that change on the device (the time step, the
// solver's convergence state) live in BatchState.
#pragma once
#include <cstring>
#include <initializer_list>

#include "ffx_common.cuh"

namespace ffx {

constexpr int kBatchMax = 64;       // domains per batch
constexpr int kBatchThreads = 256;  // threads per block of every batched tile kernel
constexpr int kBatchZ0 = 8;         // z cells per thread of the level-0 sweeps

struct BatchMap {
    int count;                // entries (domains) in this launch
    int total;                // tiles over all entries
    int bw, bh;               // tile shape: bw x bh threads (bw * bh == kBatchThreads)
    int dom[kBatchMax];       // state slot of entry k
    int first[kBatchMax + 1]; // first tile of entry k; first[count] == total
    int gx[kBatchMax];        // tiles along x of entry k
    int gy[kBatchMax];        // tiles along y of entry k
    int gz[kBatchMax];        // tiles along z of entry k
};

// Per-domain device state. `dt` is the step the passes use; the solve fields
// follow the stand-alone loop `while cycles < max and res > tol * scale: cycle`.
struct BatchState {
    float dt;          // time step of the current step
    float scale;       // max |rhs| of the current solve
    float res;         // max |rhs - L p| accumulator (zeroed after each decision)
    int cycles;        // V-cycles of the current solve
    int done;          // solve finished (converged, cap reached or rhs == 0)
    int last_cycles;   // V-cycles of the previous step's solve
    int total_cycles;  // V-cycles since the plan was created
    int steps;         // steps completed
    float maxima[3];   // max |u|, |v|, |w| after the projection (CFL input)
    float last_dt;     // dt of the previous step
    float last_maxima[3];   // maxima of the previous step
    double time;       // simulated time
    double dtd;        // the time step in FP64 (as the host rule computes it); dt is its FP32 rounding
    double last_dtd;
    float pfactor;     // warm start: factor of the previous pressure (dt / previous dt)
    int pmode;         // pressure at the start of the solve: 0 zero, 1 previous, 2 previous x pfactor
};

__device__ __forceinline__ int batch_entry(const BatchMap& M, int t) {
    int lo = 0, hi = M.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (M.first[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Walk the tiles of a batched launch: for every tile of a domain that is not
// finished (when `skip_done`), stage the domain's descriptor in shared memory,
// let `prep(desc, slot)` adjust it (thread 0, e.g. the device time step), and
// run `body(desc, blk, slot)` with the tile's virtual block.
template <class Desc, class Prep, class Body>
__device__ __forceinline__ void for_tiles(const BatchMap& M, const Desc* __restrict__ descs,
                                          const BatchState* state, bool skip_done, Prep prep, Body body) {
    __shared__ __align__(16) unsigned char raw[sizeof(Desc)];
    Desc& sh = *reinterpret_cast<Desc*>(raw);
    int cur = -1;
    for (int t = blockIdx.x; t < M.total; t += gridDim.x) {
        const int k = batch_entry(M, t);
        const int slot = M.dom[k];
        if (skip_done && state[slot].done) continue;   // uniform over the block
        if (k != cur) {
            __syncthreads();
            const int* src = reinterpret_cast<const int*>(descs + k);
            int* dst = reinterpret_cast<int*>(raw);
            for (int i = threadIdx.x; i < (int)(sizeof(Desc) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
            __syncthreads();
            if (threadIdx.x == 0) prep(sh, slot);
            __syncthreads();
            cur = k;
        }
        const int local = t - M.first[k];
        Blk b;
        b.x = local % M.gx[k];
        const int r = local / M.gx[k];
        b.y = r % M.gy[k];
        b.z = r / M.gy[k];
        b.gz = M.gz[k];
        b.bw = M.bw;
        b.bh = M.bh;
        b.ox = threadIdx.x % M.bw;
        b.oy = threadIdx.x / M.bw;
        body(sh, b, slot);
        __syncthreads();
    }
}

struct NoPrep {
    template <class D>
    __device__ __forceinline__ void operator()(D&, int) const {}
};

// Pass kinds (the autotuner's keys; FFX_PASS_* in ffx.h).
enum BatchKind {
    kPredictor = 0, kVelocity, kDivergence, kScaleZero, kGradient, kScalarPredictor, kScalarReverse, kScalarFinal,
    kResidualMax, kSmooth, kResidualRestrict, kProlongSmooth, kDirect,
    // level 0 four cells per thread (link field, nx % 4 == 0): tiles of 32 x 8 threads
    kL0Smooth, kL0ProlongSmooth, kL0ResidualRestrict, kL0ResidualMax, kBatchKinds
};
constexpr bool is_l0_kind(int k) { return k >= kL0Smooth && k <= kL0ResidualMax; }
constexpr int kL0Cells = 4, kL0Rows = 8, kL0Slices = 8;   // cells per thread along x, rows per tile, z per thread

// Internal descriptor builders and launchers of the batched passes. A builder
// writes the descriptor of one domain to `out` (when not NULL) and returns its
// size; `descs` of a launcher points at `map.count` descriptors in device
// memory; `grid` is the persistent grid (0: one block per tile).
namespace batch {
size_t predictor_desc(const FfxBatchDomain& D, void* out);
size_t velocity_desc(const FfxBatchDomain& D, int parity, void* out);
size_t scalar_xport_desc(const FfxBatchDomain& D, int parity, int reverse, void* out);
size_t scalar_final_desc(const FfxBatchDomain& D, int parity, void* out);
size_t divergence_desc(const FfxBatchDomain& D, void* out);
size_t scale_zero_desc(const FfxBatchDomain& D, void* out);
size_t gradient_desc(const FfxBatchDomain& D, float* u, float* v, float* w, void* out);
// smoothing / residual / restriction / prolongation on one level: iterate p,
// sweep output q, rhs, the coarse iterate (prolongation) or coarse rhs
// (restriction), and an optional coarse iterate to zero (restriction).
size_t level_desc(const FfxGraphLevel& lv, const float* p, float* q, const float* rhs, float* coarse,
                  float* zero, void* out);
size_t tail_desc(const FfxBatchDomain& D, int pre, int post, void* out);
size_t direct_desc(const FfxBatchDomain& D, float* p, void* out);

cudaError_t face_predictor(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t advect_velocity(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t scalar_transport(const BatchMap& M, const void* descs, BatchState* state, int reverse, int grid,
                             cudaStream_t st);
cudaError_t advect_scalars(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t divergence(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t scale_zero(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t gradient(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t residual_max(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t smooth(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t residual_restrict(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t prolong_smooth(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t direct(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t tail(const BatchMap& M, const void* descs, BatchState* state, cudaStream_t st);
// Level 0, four cells per thread (ffx_level0.cu): whether a level and its
// fields qualify; descriptor (p, coarse iterate for the prolongation, rhs,
// output: the sweep's or the restriction's coarse rhs, coarse iterate to clear).
bool l0_eligible(const FfxGraphLevel& lv, std::initializer_list<const void*> f4);
size_t l0_desc(const FfxGraphLevel& lv, const float* p, const float* coarse, const float* rhs, float* out, float* zero,
               void* dst);
cudaError_t l0_smooth(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t l0_prolong_smooth(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t l0_residual_restrict(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
cudaError_t l0_residual_max(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st);
// Resident blocks per SM of a pass kind's kernel (0: not this file's kind).
int advect_resident_blocks(int kind);
int project_resident_blocks(int kind);
int level0_resident_blocks(int kind);
}  // namespace batch

}  // namespace ffx
