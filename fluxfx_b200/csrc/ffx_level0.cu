// Level 0 of the collider (aggregation) multigrid, four cells per thread.
//
// Level 0 is the full-resolution grid and carries almost all of the solve's
// memory traffic. These kernels replace the one-cell-per-thread versions in
// ffx_project.cu when the level has a precomputed link field and the x extent
// is a multiple of 4:
//
// * links: one byte per cell, bit 2a (2a+1) set when the face to the lower
//   (upper) neighbour along axis a is open, i.e. both cells are fluid and the
//   neighbour lies inside the domain; bit 6 = the cell itself is fluid. This is
//   the level-0 conductance of solid_hierarchy.py:16-25 (weight (n/extent)^2
//   on open faces, 0 elsewhere) packed into one load per cell.
// * A thread owns four consecutive cells along x (float4 rows) and walks a
//   column of kZ4 slices along z, carrying the iterate of slices z-1, z, z+1 in
//   registers. The x neighbours of its four cells come from the neighbouring
//   lanes by shuffle (a warp is one row of 128 cells); lanes 0 and 31 load the
//   cell beyond the warp. y neighbours are float4 loads of the adjacent rows.
//
// Every cell is evaluated with the operations, and in the order, of the
// scalar kernels (graph_terms: x-, x+, y-, y+, z-, z+), so both paths give
// bit-identical fields. A term is added only where its link bit is set; the
// scalar kernels instead add weight 0 for an in-domain neighbour that is not
// linked, and diag + 0 == diag, nb + 0 * v == nb for finite v, so the sums are
// the same (nb never holds -0: it starts at +0 and an exact cancellation
// rounds to +0).
#include <algorithm>
#include <cstring>

#include "ffx_batch.cuh"
#include "ffx_common.cuh"
#include "ffx_host.cuh"
#include "ffx_level0.cuh"

namespace ffx {
namespace {

constexpr unsigned kXm = 1u, kXp = 2u, kYm = 4u, kYp = 8u, kZm = 16u, kZp = 32u, kFluid = 64u;
constexpr int kZ4 = 8;           // slices per thread column (even: the restriction pairs slices)
constexpr int kRows = 8;         // warps (rows) per block
static_assert(kZ4 == kL0Slices && kRows == kL0Rows && 32 * kRows == kBatchThreads,
              "the batched level-0 tiles are this file's blocks");

struct L0 {
    int nx, ny, nz, nx4;
    const uint8_t* links;
    float wx, wy, wz;
    float cs;              // coarse-correction factor of the prolongation (1: plain)
};

inline L0 make_l0(const FfxGraphLevel* lv) {
    L0 g;
    g.nx = lv->nx; g.ny = lv->ny; g.nz = lv->nz; g.nx4 = lv->nx / 4;
    g.links = lv->links;
    g.wx = lv->w[0]; g.wy = lv->w[1]; g.wz = lv->w[2];
    g.cs = lv->coarse_scale != 0.f ? lv->coarse_scale : 1.f;
    return g;
}

__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ float4 ld4(const float* p, int i4) {
    return __ldg(reinterpret_cast<const float4*>(p) + i4);
}
__device__ __forceinline__ float2 ld2(const float* p, int i2) {
    return __ldg(reinterpret_cast<const float2*>(p) + i2);
}
__device__ __forceinline__ float el(const float4& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_el(float4& v, int k, float s) {
    if (k == 0) v.x = s;
    else if (k == 1) v.y = s;
    else if (k == 2) v.z = s;
    else v.w = s;
}
__device__ __forceinline__ uint32_t ld_links(const L0& g, int i4) {
    return __ldg(reinterpret_cast<const uint32_t*>(g.links) + i4);
}

// Operator terms of the four cells of one row segment (byte k of `lk` is the
// link byte of cell k). left/right: the iterate at x0-1 and x0+4.
__device__ __forceinline__ void terms4(const L0& g, uint32_t lk, float left, const float4& c, float right,
                                       const float4& ym, const float4& yp, const float4& lo, const float4& hi,
                                       float diag[4], float nb[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const unsigned b = (lk >> (8 * k)) & 0xffu;
        const float xm = k == 0 ? left : el(c, k - 1);
        const float xp = k == 3 ? right : el(c, k + 1);
        float d = 0.f, s = 0.f;
        if (b & kXm) { d = d + g.wx; s = s + g.wx * xm; }
        if (b & kXp) { d = d + g.wx; s = s + g.wx * xp; }
        if (b & kYm) { d = d + g.wy; s = s + g.wy * el(ym, k); }
        if (b & kYp) { d = d + g.wy; s = s + g.wy * el(yp, k); }
        if (b & kZm) { d = d + g.wz; s = s + g.wz * el(lo, k); }
        if (b & kZp) { d = d + g.wz; s = s + g.wz * el(hi, k); }
        diag[k] = d;
        nb[k] = s;
    }
}

// ------------------------------------------------------------ iterates
// The value the stencil reads at a cell: the iterate itself, the prolonged
// iterate p + coarse (solid_mg_prolong.glsl, formed on the fly), or the new
// search direction z + beta p_old.
enum class It { Plain, Prolonged, Direction };

struct ItArgs {
    const float* a;        // p (Plain, Prolonged) or z (Direction)
    const float* b;        // coarse correction (Prolonged) or p_old (Direction; NULL on the first iteration)
    const double* rz_new;  // Direction: beta = rz_new / rz_old, read on the device
    const double* rz_old;
};

template <It K>
__device__ __forceinline__ float4 it4(const L0& g, const ItArgs& A, float beta, int i4, int x4, int y, int z) {
    const float4 v = ld4(A.a, i4);
    if constexpr (K == It::Plain) {
        return v;
    } else if constexpr (K == It::Prolonged) {
        // coarse cell of (x, y, z) is (x/2, y/2, z/2); cells 4x4, 4x4+1 share
        // coarse x = 2x4 and 4x4+2, 4x4+3 share 2x4+1: one float2.
        const float2 c = ld2(A.b, x4 + g.nx4 * ((y >> 1) + (g.ny >> 1) * (z >> 1)));
        return make_float4(v.x + g.cs * c.x, v.y + g.cs * c.x, v.z + g.cs * c.y, v.w + g.cs * c.y);
    } else {
        if (!A.b) return v;
        const float4 q = ld4(A.b, i4);
        return make_float4(v.x + beta * q.x, v.y + beta * q.y, v.z + beta * q.z, v.w + beta * q.w);
    }
}

template <It K>
__device__ __forceinline__ float it1(const L0& g, const ItArgs& A, float beta, int i, int x, int y, int z) {
    const float v = __ldg(A.a + i);
    if constexpr (K == It::Plain) {
        return v;
    } else if constexpr (K == It::Prolonged) {
        return v + g.cs * __ldg(A.b + (x >> 1) + (g.nx >> 1) * ((y >> 1) + (g.ny >> 1) * (z >> 1)));
    } else {
        return A.b ? v + beta * __ldg(A.b + i) : v;
    }
}

// ------------------------------------------------------------ epilogues
enum class Ep { Smooth, SmoothDot, Apply, Residual, ResidualMax, ResidualMaxSmooth };

struct EpArgs {
    const float* rhs;
    float omega;
    float* out;       // smoothed iterate, new direction (Apply) or residual
    float* out2;      // q = A p (Apply)
    double* dsum;     // SmoothDot: += scale * rhs . out; Apply: += p . q
    double scale;
    float* fmax;      // ResidualMax
};

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ void block_sum_d(double* out, double v) {
    __shared__ double part[kRows];
    v = warp_sum_d(v);
    const int lane = threadIdx.x, wid = threadIdx.y;
    if (lane == 0) part[wid] = v;
    __syncthreads();
    if (lane == 0 && wid == 0) {
        double s = 0.0;
        for (int w = 0; w < kRows; ++w) s += part[w];
        if (s != 0.0) atomicAdd(out, s);
    }
}

// One pass of the stencil over level 0: K selects the iterate, E what is
// written. Block (32, kRows): lane = x4 within a 128-cell row segment, warp =
// row; blockIdx.z = column of kZ4 slices. Threads outside the grid stay in the
// loop (with zero data) so that shuffles and the block reduction see every lane.
//
// The body takes the block's coordinates (bx, by, bz) and the thread's lane
// and row (warp), so the same code runs as its own launch (level0_kernel) and
// as a tile of a batched persistent launch over many domains.
template <It K, Ep E>
__device__ __forceinline__ void level0_body(const L0& g, const ItArgs& A, const EpArgs& P, int bx, int by, int bz,
                                            int lane, int row) {
    const int x4 = bx * 32 + lane, y = by * kRows + row;
    const bool active = x4 < g.nx4 && y < g.ny;
    const int x0 = 4 * x4;
    const int z0 = bz * kZ4, zend = min(z0 + kZ4, g.nz);
    const int row4 = g.nx4, slice4 = g.nx4 * g.ny;
    int i4 = x4 + row4 * (y + g.ny * z0);
    const float one_minus = 1.f - P.omega;
    float beta = 0.f;
    if constexpr (K == It::Direction) beta = A.b ? (float)(*A.rz_new / *A.rz_old) : 0.f;
    double acc = 0.0;
    float m = 0.f;
    // Everything slice z needs from memory, fetched one slice ahead so that
    // two slices' loads are in flight while one is computed. `edge` is the
    // iterate beyond the warp (x0 - 1 on lane 0, x0 + 4 on lane 31).
    struct Slice {
        uint32_t lk;
        float4 hi, ym, yp, r;
        float edge;
    };
    auto fetch = [&](int z, int j4, Slice& s) {
        s.lk = active ? ld_links(g, j4) : 0u;
        s.hi = (active && z + 1 < g.nz) ? it4<K>(g, A, beta, j4 + slice4, x4, y, z + 1) : zero4();
        s.ym = (active && y > 0) ? it4<K>(g, A, beta, j4 - row4, x4, y - 1, z) : zero4();
        s.yp = (active && y + 1 < g.ny) ? it4<K>(g, A, beta, j4 + row4, x4, y + 1, z) : zero4();
        if constexpr (E != Ep::Apply) s.r = active ? ld4(P.rhs, j4) : zero4();
        s.edge = 0.f;
        if (active && lane == 0 && x0 > 0) s.edge = it1<K>(g, A, beta, 4 * j4 - 1, x0 - 1, y, z);
        if (active && lane == 31 && x0 + 4 < g.nx) s.edge = it1<K>(g, A, beta, 4 * j4 + 4, x0 + 4, y, z);
    };
    float4 lo = zero4(), c = zero4();
    if (active) {
        c = it4<K>(g, A, beta, i4, x4, y, z0);
        if (z0 > 0) lo = it4<K>(g, A, beta, i4 - slice4, x4, y, z0 - 1);
    }
    Slice cur;
    fetch(z0, i4, cur);
    for (int z = z0; z < zend; ++z, i4 += slice4) {
        Slice nxt;
        if (z + 1 < zend) fetch(z + 1, i4 + slice4, nxt);
        const uint32_t lk = cur.lk;
        float left = __shfl_up_sync(0xffffffffu, c.w, 1);
        float right = __shfl_down_sync(0xffffffffu, c.x, 1);
        if (lane == 0) left = cur.edge;
        if (lane == 31) right = cur.edge;
        float diag[4], nb[4];
        terms4(g, lk, left, c, right, cur.ym, cur.yp, lo, cur.hi, diag, nb);
        if (active) {
            if constexpr (E == Ep::Apply) {
                float4 q;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float pc = el(c, k);
                    const float qc = diag[k] > 0.f ? diag[k] * pc - nb[k] : 0.f;
                    set_el(q, k, qc);
                    acc += (double)pc * (double)qc;
                }
                reinterpret_cast<float4*>(P.out)[i4] = c;
                reinterpret_cast<float4*>(P.out2)[i4] = q;
            } else {
                const float4 r = cur.r;
                float4 o;
                if constexpr (E == Ep::ResidualMaxSmooth) {
                    // the residual maximum of the iterate and, from the same terms, its sweep
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float rk = el(r, k), d = diag[k];
                        const float res = d > 0.f ? (rk - nb[k]) + d * el(c, k) : 0.f;
                        m = fmaxf(m, finite_abs(res));
                        set_el(o, k, d > 0.f ? el(c, k) * one_minus + ((nb[k] - rk) / d) * P.omega : 0.f);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float rk = el(r, k), d = diag[k];
                        float v;
                        if constexpr (E == Ep::Residual || E == Ep::ResidualMax)
                            v = d > 0.f ? (rk - nb[k]) + d * el(c, k) : 0.f;
                        else
                            v = d > 0.f ? el(c, k) * one_minus + ((nb[k] - rk) / d) * P.omega : 0.f;
                        set_el(o, k, v);
                        if constexpr (E == Ep::SmoothDot) acc += P.scale * (double)rk * (double)v;
                        if constexpr (E == Ep::ResidualMax) m = fmaxf(m, finite_abs(v));
                    }
                }
                if constexpr (E != Ep::ResidualMax) reinterpret_cast<float4*>(P.out)[i4] = o;
            }
        }
        lo = c;
        c = cur.hi;
        cur = nxt;
    }
    if constexpr (E == Ep::SmoothDot || E == Ep::Apply) block_sum_d(P.dsum, acc);
    if constexpr (E == Ep::ResidualMax || E == Ep::ResidualMaxSmooth) block_max_to(P.fmax, m);
}

template <It K, Ep E>
__global__ void __launch_bounds__(32 * kRows, 4) level0_kernel(L0 g, ItArgs A, EpArgs P) {
    pdl_enter();
    level0_body<K, E>(g, A, P, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, (int)threadIdx.x,
                      (int)threadIdx.y);
}

// ------------------------------------------------ two sweeps in one pass
// out = S(S(p)), S being the weighted-Jacobi sweep of level0_body<K, Smooth>
// (the first sweep reads the iterate of kind K, the second the first's output).
// A block owns 128 x kRows2 x kZ2 cells. Its kRows2 + 2 warps march the slices
// z0 - 1 .. z0 + kZ2: each warp computes the first sweep of its row (the
// block's rows and one halo row on either side) at slice z into a ring of three
// slices in shared memory, 128 cells a row plus the cell on either side
// (lanes 0 and 31 compute those one at a time); after a barrier the inner warps
// compute the second sweep of slice z - 1 from the ring, with the link byte and
// right-hand side they loaded for it one slice earlier. Every value of the
// first sweep is formed by S's operations in S's order from the same inputs,
// so the result equals two launches of S bit for bit while the iterate, the
// right-hand side and the links are read from memory once for two sweeps.
constexpr int kRows2 = 8;             // output rows per block
constexpr int kWarps2 = kRows2 + 2;   // + one halo row on either side
constexpr int kZ2 = 16;               // output slices per block
constexpr int kOff2 = 4;              // ring column of cell x0 (16-byte aligned); x0 - 1 at kOff2 - 1
constexpr int kPitch2 = kOff2 + 128 + 4;

// S at one cell from its neighbours' iterate values (terms4's per-cell terms,
// in its order, and the Smooth epilogue).
__device__ __forceinline__ float sweep1(const L0& g, unsigned b, float c, float xm, float xp, float ym, float yp,
                                        float zm, float zp, float r, float omega, float one_minus) {
    float d = 0.f, s = 0.f;
    if (b & kXm) { d = d + g.wx; s = s + g.wx * xm; }
    if (b & kXp) { d = d + g.wx; s = s + g.wx * xp; }
    if (b & kYm) { d = d + g.wy; s = s + g.wy * ym; }
    if (b & kYp) { d = d + g.wy; s = s + g.wy * yp; }
    if (b & kZm) { d = d + g.wz; s = s + g.wz * zm; }
    if (b & kZp) { d = d + g.wz; s = s + g.wz * zp; }
    return d > 0.f ? c * one_minus + ((s - r) / d) * omega : 0.f;
}

__device__ __forceinline__ float4 sweep4(const L0& g, uint32_t lk, float left, const float4& c, float right,
                                         const float4& ym, const float4& yp, const float4& lo, const float4& hi,
                                         const float4& r, float omega, float one_minus) {
    float diag[4], nb[4];
    terms4(g, lk, left, c, right, ym, yp, lo, hi, diag, nb);
    float4 o;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float d = diag[k];
        set_el(o, k, d > 0.f ? el(c, k) * one_minus + ((nb[k] - el(r, k)) / d) * omega : 0.f);
    }
    return o;
}

template <It K>
__global__ void __launch_bounds__(32 * kWarps2) level0_smooth2_kernel(L0 g, ItArgs A, const float* __restrict__ rhs,
                                                                      float omega, float* __restrict__ out) {
    __shared__ __align__(16) float ring[3][kWarps2][kPitch2];
    const int lane = threadIdx.x, w = threadIdx.y;
    const int x4 = blockIdx.x * 32 + lane, x0 = 4 * x4;
    const int y = (int)blockIdx.y * kRows2 - 1 + w;
    const int z0 = blockIdx.z * kZ2, zend = min(z0 + kZ2, g.nz);
    const bool row = y >= 0 && y < g.ny;
    const bool active = row && x4 < g.nx4;
    const bool inner = w >= 1 && w <= kRows2 && active;
    const int row4 = g.nx4;
    const float one_minus = 1.f - omega;
    // the iterate (of kind K) at this thread's four cells of row yy, slice z, or zeros outside
    auto it_row = [&](int yy, int z) -> float4 {
        return (x4 < g.nx4 && yy >= 0 && yy < g.ny && z >= 0 && z < g.nz)
                   ? it4<K>(g, A, 0.f, x4 + row4 * (yy + g.ny * z), x4, yy, z) : zero4();
    };
    auto it_cell = [&](int x, int yy, int z) -> float {
        return (x >= 0 && x < g.nx && yy >= 0 && yy < g.ny && z >= 0 && z < g.nz)
                   ? it1<K>(g, A, 0.f, x + g.nx * (yy + g.ny * z), x, yy, z) : 0.f;
    };
    // the first sweep at the single cell (xe, y, z) (the ring's halo columns)
    auto edge = [&](int xe, int z) -> float {
        if (!row || xe < 0 || xe >= g.nx || z < 0 || z >= g.nz) return 0.f;
        const int i = xe + g.nx * (y + g.ny * z);
        return sweep1(g, __ldg(g.links + i), it_cell(xe, y, z), it_cell(xe - 1, y, z), it_cell(xe + 1, y, z),
                      it_cell(xe, y - 1, z), it_cell(xe, y + 1, z), it_cell(xe, y, z - 1), it_cell(xe, y, z + 1),
                      __ldg(rhs + i), omega, one_minus);
    };
    float4 lo = it_row(y, z0 - 2), c = it_row(y, z0 - 1);
    uint32_t lk_prev = 0u;
    float4 r_prev = zero4();
    for (int z = z0 - 1; z <= zend; ++z) {
        const float4 hi = it_row(y, z + 1);
        // first sweep of (row y, slice z)
        const bool zin = z >= 0 && z < g.nz;
        const int i4 = x4 + row4 * (y + g.ny * z);
        uint32_t lk = 0u;
        float4 r = zero4(), o = zero4();
        if (active && zin) {
            lk = ld_links(g, i4);
            r = ld4(rhs, i4);
        }
        float left = __shfl_up_sync(0xffffffffu, c.w, 1);
        float right = __shfl_down_sync(0xffffffffu, c.x, 1);
        if (lane == 0) left = it_cell(x0 - 1, y, z);
        if (lane == 31) right = it_cell(x0 + 4, y, z);
        if (active && zin) o = sweep4(g, lk, left, c, right, it_row(y - 1, z), it_row(y + 1, z), lo, hi, r, omega,
                                      one_minus);
        float* slot = ring[(z + 3) % 3][w];
        *reinterpret_cast<float4*>(slot + kOff2 + 4 * lane) = o;
        if (lane == 0) slot[kOff2 - 1] = edge(x0 - 1, z);
        if (lane == 31) slot[kOff2 + 128] = edge(x0 + 4, z);
        __syncthreads();
        // second sweep of (row y, slice z - 1)
        const int zo = z - 1;
        if (inner && zo >= z0 && zo < zend) {
            const float* mid = ring[(zo + 3) % 3][w];
            const float4 c2 = *reinterpret_cast<const float4*>(mid + kOff2 + 4 * lane);
            const float4 ym2 = *reinterpret_cast<const float4*>(ring[(zo + 3) % 3][w - 1] + kOff2 + 4 * lane);
            const float4 yp2 = *reinterpret_cast<const float4*>(ring[(zo + 3) % 3][w + 1] + kOff2 + 4 * lane);
            const float4 lo2 = *reinterpret_cast<const float4*>(ring[(zo + 2) % 3][w] + kOff2 + 4 * lane);
            const float4 hi2 = *reinterpret_cast<const float4*>(ring[(zo + 4) % 3][w] + kOff2 + 4 * lane);
            const float4 o2 = sweep4(g, lk_prev, mid[kOff2 + 4 * lane - 1], c2, mid[kOff2 + 4 * lane + 4], ym2, yp2,
                                     lo2, hi2, r_prev, omega, one_minus);
            reinterpret_cast<float4*>(out)[x4 + row4 * (y + g.ny * zo)] = o2;
        }
        __syncthreads();
        lk_prev = lk;
        r_prev = r;
        lo = c;
        c = hi;
    }
}

// First sweep from a zero iterate (graph_smooth_zero_kernel): no iterate is
// read, so this is a plain stream over links and rhs.
__global__ void __launch_bounds__(256) level0_smooth_zero_kernel(L0 g, const float* __restrict__ rhs, float omega,
                                                                float* __restrict__ out, int n4) {
    pdl_enter();
    const int i4 = blockIdx.x * blockDim.x + threadIdx.x;
    if (i4 >= n4) return;
    const uint32_t lk = ld_links(g, i4);
    const float4 r = ld4(rhs, i4);
    const float4 z = zero4();
    float diag[4], nb[4];
    terms4(g, lk, 0.f, z, 0.f, z, z, z, z, diag, nb);
    float4 o;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float d = diag[k];
        set_el(o, k, d > 0.f ? 0.f * (1.f - omega) + ((nb[k] - el(r, k)) / d) * omega : 0.f);
    }
    reinterpret_cast<float4*>(out)[i4] = o;
}

// Fused residual + 2x2x2 average restriction (graph_residual_restrict_kernel):
// a thread owns a 4 x 2 (x, y) patch, i.e. two coarse cells along x, and walks
// pairs of slices; each coarse value sums its eight children's residuals in
// the scalar kernel's order (dz, then dy, then dx) and divides by 8.
__device__ __forceinline__ void level0_restrict_body(const L0& g, const float* __restrict__ p,
                                                     const float* __restrict__ rhs, float* __restrict__ coarse,
                                                     float* __restrict__ zero, int bx, int by, int bz, int lane,
                                                     int row) {
    const int x4 = bx * 32 + lane, ya = 2 * (by * kRows + row), yb = ya + 1;
    const bool active = x4 < g.nx4 && ya < g.ny;
    const int z0 = bz * kZ4, zend = min(z0 + kZ4, g.nz);
    const int row4 = g.nx4, slice4 = g.nx4 * g.ny;
    int ia = x4 + row4 * (ya + g.ny * z0);
    float4 lo_a = zero4(), c_a = zero4(), lo_b = zero4(), c_b = zero4();
    if (active) {
        c_a = ld4(p, ia);
        c_b = ld4(p, ia + row4);
        if (z0 > 0) {
            lo_a = ld4(p, ia - slice4);
            lo_b = ld4(p, ia + row4 - slice4);
        }
    }
    float v0 = 0.f, v1 = 0.f;
    for (int z = z0; z < zend; ++z, ia += slice4) {
        const int ib = ia + row4;
        const bool up = active && z + 1 < g.nz;
        const float4 hi_a = up ? ld4(p, ia + slice4) : zero4();
        const float4 hi_b = up ? ld4(p, ib + slice4) : zero4();
        const float4 ym = (active && ya > 0) ? ld4(p, ia - row4) : zero4();
        const float4 yp = (active && yb + 1 < g.ny) ? ld4(p, ib + row4) : zero4();
        const uint32_t lka = active ? ld_links(g, ia) : 0u, lkb = active ? ld_links(g, ib) : 0u;
        float left_a = __shfl_up_sync(0xffffffffu, c_a.w, 1), right_a = __shfl_down_sync(0xffffffffu, c_a.x, 1);
        float left_b = __shfl_up_sync(0xffffffffu, c_b.w, 1), right_b = __shfl_down_sync(0xffffffffu, c_b.x, 1);
        if (lane == 0) {
            left_a = (lka & kXm) ? __ldg(p + 4 * ia - 1) : 0.f;
            left_b = (lkb & kXm) ? __ldg(p + 4 * ib - 1) : 0.f;
        }
        if (lane == 31) {
            right_a = ((lka >> 24) & kXp) ? __ldg(p + 4 * ia + 4) : 0.f;
            right_b = ((lkb >> 24) & kXp) ? __ldg(p + 4 * ib + 4) : 0.f;
        }
        float da[4], na[4], db[4], nbb[4];
        terms4(g, lka, left_a, c_a, right_a, ym, c_b, lo_a, hi_a, da, na);
        terms4(g, lkb, left_b, c_b, right_b, c_a, yp, lo_b, hi_b, db, nbb);
        if (active) {
            const float4 ra = ld4(rhs, ia), rb = ld4(rhs, ib);
            float res_a[4], res_b[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                res_a[k] = da[k] > 0.f ? (el(ra, k) - na[k]) + da[k] * el(c_a, k) : 0.f;
                res_b[k] = db[k] > 0.f ? (el(rb, k) - nbb[k]) + db[k] * el(c_b, k) : 0.f;
            }
            if ((z & 1) == 0) {
                v0 = 0.f;
                v1 = 0.f;
            }
            v0 = v0 + res_a[0]; v0 = v0 + res_a[1]; v0 = v0 + res_b[0]; v0 = v0 + res_b[1];
            v1 = v1 + res_a[2]; v1 = v1 + res_a[3]; v1 = v1 + res_b[2]; v1 = v1 + res_b[3];
            if (z & 1) {
                const int c2 = x4 + g.nx4 * ((ya >> 1) + (g.ny >> 1) * (z >> 1));
                reinterpret_cast<float2*>(coarse)[c2] = make_float2(v0 / 8.0f, v1 / 8.0f);
                if (zero) reinterpret_cast<float2*>(zero)[c2] = make_float2(0.f, 0.f);
            }
        }
        lo_a = c_a; c_a = hi_a;
        lo_b = c_b; c_b = hi_b;
    }
}

__global__ void __launch_bounds__(32 * kRows) level0_residual_restrict_kernel(L0 g, const float* __restrict__ p,
                                                                             const float* __restrict__ rhs,
                                                                             float* __restrict__ coarse,
                                                                             float* __restrict__ zero) {
    pdl_enter();
    level0_restrict_body(g, p, rhs, coarse, zero, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z,
                         (int)threadIdx.x, (int)threadIdx.y);
}

__global__ void __launch_bounds__(256) links_kernel(int nx, int ny, int nz, const uint8_t* __restrict__ solid,
                                                   uint8_t* __restrict__ links) {
    int x, y, z;
    if (!cell_coords(nx, ny, x, y, z)) return;
    const int sy = nx, sz = nx * ny;
    const int i = x + nx * (y + ny * z);
    unsigned b = 0;
    if (__ldg(solid + i) == 0) {
        b = kFluid;
        if (x > 0 && __ldg(solid + i - 1) == 0) b |= kXm;
        if (x + 1 < nx && __ldg(solid + i + 1) == 0) b |= kXp;
        if (y > 0 && __ldg(solid + i - sy) == 0) b |= kYm;
        if (y + 1 < ny && __ldg(solid + i + sy) == 0) b |= kYp;
        if (z > 0 && __ldg(solid + i - sz) == 0) b |= kZm;
        if (z + 1 < nz && __ldg(solid + i + sz) == 0) b |= kZp;
    }
    links[i] = (uint8_t)b;
}

// ------------------------------------------------- batched level-0 passes
// Level 0 of many domains in one persistent launch: every domain contributes
// the blocks of its own level0_kernel launch (32 lanes x kRows rows, kZ4
// slices per thread; the batched map's tiles are 32 x kRows threads), so each
// domain's cells are computed exactly as in its stand-alone launch.
constexpr float kL0Omega = (float)(2.0 / 3.0);   // the weighted-Jacobi factor of the batched sweeps

struct L0Desc {
    L0 g;
    const float* p;        // iterate
    const float* coarse;   // prolongation: the coarse iterate
    const float* rhs;
    float* out;            // sweep output, or the coarse right-hand side (restriction)
    float* zero;           // restriction: coarse iterate to clear (optional)
};

__global__ void __launch_bounds__(kBatchThreads) batch_l0_smooth_kernel(const __grid_constant__ BatchMap M,
                                                                        const L0Desc* descs,
                                                                        const BatchState* state) {
    for_tiles(M, descs, state, true, NoPrep{}, [](const L0Desc& D, const Blk& b, int) {
        const EpArgs E{D.rhs, kL0Omega, D.out, nullptr, nullptr, 0.0, nullptr};
        level0_body<It::Plain, Ep::Smooth>(D.g, ItArgs{D.p, nullptr, nullptr, nullptr}, E, b.x, b.y, b.z,
                                           (int)threadIdx.x & 31, (int)threadIdx.x >> 5);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_l0_prolong_smooth_kernel(const __grid_constant__ BatchMap M,
                                                                                const L0Desc* descs,
                                                                                const BatchState* state) {
    for_tiles(M, descs, state, true, NoPrep{}, [](const L0Desc& D, const Blk& b, int) {
        const EpArgs E{D.rhs, kL0Omega, D.out, nullptr, nullptr, 0.0, nullptr};
        level0_body<It::Prolonged, Ep::Smooth>(D.g, ItArgs{D.p, D.coarse, nullptr, nullptr}, E, b.x, b.y, b.z,
                                               (int)threadIdx.x & 31, (int)threadIdx.x >> 5);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_l0_residual_restrict_kernel(
    const __grid_constant__ BatchMap M, const L0Desc* descs, const BatchState* state) {
    for_tiles(M, descs, state, true, NoPrep{}, [](const L0Desc& D, const Blk& b, int) {
        level0_restrict_body(D.g, D.p, D.rhs, D.out, D.zero, b.x, b.y, b.z, (int)threadIdx.x & 31,
                             (int)threadIdx.x >> 5);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_l0_residual_max_kernel(const __grid_constant__ BatchMap M,
                                                                              const L0Desc* descs,
                                                                              BatchState* state) {
    for_tiles(M, descs, state, true, NoPrep{}, [state](const L0Desc& D, const Blk& b, int slot) {
        const int lane = (int)threadIdx.x & 31, row = (int)threadIdx.x >> 5;
        if (state[slot].scale == 0.f) {
            // rhs == 0: the solve's result is the zero pressure (and no cycle runs)
            const int x4 = b.x * 32 + lane, y = b.y * kRows + row;
            if (x4 < D.g.nx4 && y < D.g.ny)
                for (int z = b.z * kZ4; z < min(b.z * kZ4 + kZ4, D.g.nz); ++z)
                    reinterpret_cast<float4*>(const_cast<float*>(D.p))[x4 + D.g.nx4 * (y + D.g.ny * z)] = zero4();
            return;
        }
        const EpArgs E{D.rhs, 0.f, nullptr, nullptr, nullptr, 0.0, &state[slot].res};
        level0_body<It::Plain, Ep::ResidualMax>(D.g, ItArgs{D.p, nullptr, nullptr, nullptr}, E, b.x, b.y, b.z, lane,
                                                row);
    });
}

template <class K>
int occupancy_l0(K kernel) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kBatchThreads, 0);
    return n;
}

bool aligned(const void* p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) == 0; }

dim3 l0_grid(const L0& g) {
    return dim3((unsigned)((g.nx4 + 31) / 32), (unsigned)((g.ny + kRows - 1) / kRows),
                (unsigned)((g.nz + kZ4 - 1) / kZ4));
}

template <It K, Ep E>
int launch(const L0& g, const ItArgs& A, const EpArgs& P, cudaStream_t st, const char* name) {
    return launch_pdl(name, level0_kernel<K, E>, l0_grid(g), dim3(32, kRows), st, g, A, P);
}

}  // namespace

bool level0_x4(const FfxGraphLevel* lv, std::initializer_list<const void*> f4) {
    if (!lv || lv->edges || !lv->links || lv->nx % 4 != 0 || !aligned(lv->links, 4)) return false;
    for (const void* p : f4)
        if (p && !aligned(p, 16)) return false;
    return true;
}

int level0_smooth(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega, float* out,
                  cudaStream_t st) {
    EpArgs P{rhs, omega, out, nullptr, nullptr, 0.0, nullptr};
    return launch<It::Plain, Ep::Smooth>(make_l0(lv), ItArgs{p, nullptr, nullptr, nullptr}, P, st, "level0_smooth_kernel");
}

int level0_smooth_dot(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega, float* out,
                      double* dot, double scale, cudaStream_t st) {
    EpArgs P{rhs, omega, out, nullptr, dot, scale, nullptr};
    return launch<It::Plain, Ep::SmoothDot>(make_l0(lv), ItArgs{p, nullptr, nullptr, nullptr}, P, st,
                                            "level0_smooth_dot_kernel");
}

int level0_prolong_smooth(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                          float omega, float* out, cudaStream_t st) {
    EpArgs P{rhs, omega, out, nullptr, nullptr, 0.0, nullptr};
    return launch<It::Prolonged, Ep::Smooth>(make_l0(lv), ItArgs{p, coarse, nullptr, nullptr}, P, st,
                                             "level0_prolong_smooth_kernel");
}

int level0_prolong_smooth_dot(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                              float omega, float* out, double* dot, double scale, cudaStream_t st) {
    EpArgs P{rhs, omega, out, nullptr, dot, scale, nullptr};
    return launch<It::Prolonged, Ep::SmoothDot>(make_l0(lv), ItArgs{p, coarse, nullptr, nullptr}, P, st,
                                                "level0_prolong_smooth_dot_kernel");
}

int level0_smooth2(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega, float* out,
                   cudaStream_t st) {
    const L0 g = make_l0(lv);
    const dim3 grid((unsigned)((g.nx4 + 31) / 32), (unsigned)((g.ny + kRows2 - 1) / kRows2),
                    (unsigned)((g.nz + kZ2 - 1) / kZ2));
    level0_smooth2_kernel<It::Plain><<<grid, dim3(32, kWarps2), 0, st>>>(g, ItArgs{p, nullptr, nullptr, nullptr}, rhs,
                                                                          omega, out);
    return launch_status("level0_smooth2_kernel");
}

int level0_prolong_smooth2(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                           float omega, float* out, cudaStream_t st) {
    const L0 g = make_l0(lv);
    const dim3 grid((unsigned)((g.nx4 + 31) / 32), (unsigned)((g.ny + kRows2 - 1) / kRows2),
                    (unsigned)((g.nz + kZ2 - 1) / kZ2));
    level0_smooth2_kernel<It::Prolonged><<<grid, dim3(32, kWarps2), 0, st>>>(g, ItArgs{p, coarse, nullptr, nullptr},
                                                                              rhs, omega, out);
    return launch_status("level0_prolong_smooth2_kernel");
}

int level0_residual_max_smooth(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega, float* out,
                               float* p_out, cudaStream_t st) {
    EpArgs P{rhs, omega, p_out, nullptr, nullptr, 0.0, out};
    return launch<It::Plain, Ep::ResidualMaxSmooth>(make_l0(lv), ItArgs{p, nullptr, nullptr, nullptr}, P, st,
                                                    "level0_residual_max_smooth_kernel");
}

int level0_residual(const FfxGraphLevel* lv, const float* p, const float* rhs, float* r, cudaStream_t st) {
    EpArgs P{rhs, 0.f, r, nullptr, nullptr, 0.0, nullptr};
    return launch<It::Plain, Ep::Residual>(make_l0(lv), ItArgs{p, nullptr, nullptr, nullptr}, P, st, "level0_residual_kernel");
}

int level0_residual_max(const FfxGraphLevel* lv, const float* p, const float* rhs, float* out, cudaStream_t st) {
    EpArgs P{rhs, 0.f, nullptr, nullptr, nullptr, 0.0, out};
    return launch<It::Plain, Ep::ResidualMax>(make_l0(lv), ItArgs{p, nullptr, nullptr, nullptr}, P, st,
                                              "level0_residual_max_kernel");
}

int level0_direction_apply(const FfxGraphLevel* lv, const float* z, const float* p_old, const double* rz_new,
                           const double* rz_old, float* p_out, float* q, double* pq, cudaStream_t st) {
    EpArgs P{nullptr, 0.f, p_out, q, pq, 0.0, nullptr};
    const ItArgs A{z, rz_old ? p_old : nullptr, rz_new, rz_old};
    return launch<It::Direction, Ep::Apply>(make_l0(lv), A, P, st,
                                            "level0_direction_apply_kernel");
}

int level0_smooth_zero(const FfxGraphLevel* lv, const float* rhs, float omega, float* out, cudaStream_t st) {
    const L0 g = make_l0(lv);
    const int n4 = g.nx4 * g.ny * g.nz;
    return launch_pdl("level0_smooth_zero_kernel", level0_smooth_zero_kernel, dim3((unsigned)((n4 + 255) / 256)),
                      dim3(256), st, g, rhs, omega, out, n4);
}

int level0_residual_restrict(const FfxGraphLevel* lv, const float* p, const float* rhs, float* coarse,
                             float* zero, cudaStream_t st) {
    const L0 g = make_l0(lv);
    const dim3 grid((unsigned)((g.nx4 + 31) / 32), (unsigned)((g.ny / 2 + kRows - 1) / kRows),
                    (unsigned)((g.nz + kZ4 - 1) / kZ4));
    return launch_pdl("level0_residual_restrict_kernel", level0_residual_restrict_kernel, grid, dim3(32, kRows), st,
                      g, p, rhs, coarse, zero);
}

int level0_links(int nx, int ny, int nz, const uint8_t* solid, uint8_t* links, cudaStream_t st) {
    links_kernel<<<cell_grid(nx, ny, nz), cell_block(), 0, st>>>(nx, ny, nz, solid, links);
    return launch_status("links_kernel");
}

namespace batch {

bool l0_eligible(const FfxGraphLevel& lv, std::initializer_list<const void*> f4) { return level0_x4(&lv, f4); }

size_t l0_desc(const FfxGraphLevel& lv, const float* p, const float* coarse, const float* rhs, float* out, float* zero,
               void* dst) {
    if (dst) {
        L0Desc D;
        memset(&D, 0, sizeof D);
        D.g = make_l0(&lv);
        D.p = p;
        D.coarse = coarse;
        D.rhs = rhs;
        D.out = out;
        D.zero = zero;
        memcpy(dst, &D, sizeof D);
    }
    return sizeof(L0Desc);
}

static unsigned l0_blocks(const BatchMap& M, int grid) { return (unsigned)(grid > 0 ? std::min(grid, M.total) : M.total); }

cudaError_t l0_smooth(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_l0_smooth_kernel<<<l0_blocks(M, grid), kBatchThreads, 0, st>>>(M, (const L0Desc*)descs, state);
    return cudaGetLastError();
}
cudaError_t l0_prolong_smooth(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_l0_prolong_smooth_kernel<<<l0_blocks(M, grid), kBatchThreads, 0, st>>>(M, (const L0Desc*)descs, state);
    return cudaGetLastError();
}
cudaError_t l0_residual_restrict(const BatchMap& M, const void* descs, BatchState* state, int grid,
                                 cudaStream_t st) {
    batch_l0_residual_restrict_kernel<<<l0_blocks(M, grid), kBatchThreads, 0, st>>>(M, (const L0Desc*)descs, state);
    return cudaGetLastError();
}
cudaError_t l0_residual_max(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_l0_residual_max_kernel<<<l0_blocks(M, grid), kBatchThreads, 0, st>>>(M, (const L0Desc*)descs, state);
    return cudaGetLastError();
}
int level0_resident_blocks(int kind) {
    switch (kind) {
        case kL0Smooth: return occupancy_l0(batch_l0_smooth_kernel);
        case kL0ProlongSmooth: return occupancy_l0(batch_l0_prolong_smooth_kernel);
        case kL0ResidualRestrict: return occupancy_l0(batch_l0_residual_restrict_kernel);
        case kL0ResidualMax: return occupancy_l0(batch_l0_residual_max_kernel);
        default: return 0;
    }
}

}  // namespace batch

}  // namespace ffx
