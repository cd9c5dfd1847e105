// Shared device code of libffx_core: grid constants, storage loads/stores,
// samplers, collider tests and emitter weights.
//
// Every expression keeps the evaluation order of the reference shaders
// (fluxfx/shaders/*.glsl) and the library is compiled with --fmad=false, so a
// float result and every discrete decision (floor, clamp, trace clipping,
// MacCormack fallbacks) equal those of a strict IEEE FP32 evaluation.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <cmath>

#include "../../include/ffx.h"

namespace ffx {

// ---------------------------------------------------------------- storage
template <typename T> struct Store;
// Element i of a field. The 32-bit index forms (every field has fewer than
// 2^31 elements, checked at the entry points) let the address be one wide
// multiply-add; the 64-bit forms serve callers that index in int64_t.
template <> struct Store<float> {
    static __device__ __forceinline__ float ld(const float* p, int i) { return __ldg(p + i); }
    static __device__ __forceinline__ float ld(const float* p, int64_t i) { return __ldg(p + i); }
    static __device__ __forceinline__ void st(float* p, int i, float v) { p[i] = v; }
    static __device__ __forceinline__ void st(float* p, int64_t i, float v) { p[i] = v; }
};
template <> struct Store<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p, int i) { return __bfloat162float(p[i]); }
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p, int64_t i) {
        return __bfloat162float(p[i]);
    }
    static __device__ __forceinline__ void st(__nv_bfloat16* p, int i, float v) { p[i] = __float2bfloat16_rn(v); }
    static __device__ __forceinline__ void st(__nv_bfloat16* p, int64_t i, float v) {
        p[i] = __float2bfloat16_rn(v);
    }
};

// ---------------------------------------------------------------- grid
struct Dev {
    int nx, ny, nz;          // cells
    float nf[3];             // float(cell counts)
    float e[3];              // extent
    float h[3];              // e / n (FP32 division, as the shaders compute it)
    float inv[3];            // host-side 1/h rounded to FP32 (the invCell uniform)
    float re[3], rn[3], rh[3];   // 1/e, 1/n, 1/h rounded to nearest (exact when pow2)
    int pow2;                // every e, n and h is a power of two
};

inline bool is_pow2f(float v) {
    int ex = 0;
    return v > 0.f && std::frexp(v, &ex) == 0.5f;
}

inline Dev make_dev(const FfxGrid& g) {
    Dev d;
    d.nx = g.nx; d.ny = g.ny; d.nz = g.nz;
    int n[3] = {g.nx, g.ny, g.nz};
    float e[3] = {g.ex, g.ey, g.ez};
    double e64[3] = {g.ex, g.ey, g.ez};
    float given[3] = {g.ix, g.iy, g.iz};
    d.pow2 = 1;
    for (int i = 0; i < 3; ++i) {
        d.nf[i] = (float)n[i];
        d.e[i] = e[i];
        d.h[i] = e[i] / (float)n[i];
        d.inv[i] = given[i] != 0.f ? given[i] : (float)(1.0 / (e64[i] / (double)n[i]));
        d.re[i] = 1.f / e[i];
        d.rn[i] = 1.f / d.nf[i];
        d.rh[i] = 1.f / d.h[i];
        if (!(is_pow2f(e[i]) && is_pow2f(d.nf[i]) && is_pow2f(d.h[i]))) d.pow2 = 0;
    }
    return d;
}

// Whether the face predictor's start point (x + o) * h and the velocity
// correction's (x + o) * e / n (times the exact 1/n on power-of-two grids) are
// the same float for every face coordinate x + o (o = 0 or 1/2) of every axis,
// evaluated exactly as the kernels evaluate them (FP32, no contraction). The
// correction may then reuse the predictor's departure points: both passes
// trace the same point with the same velocity and time step. True on
// power-of-two grids, and whenever the spacing e / n is a power of two that
// e / n rounds to exactly, for moderate n (each product then has few bits).
inline bool face_starts_match(const Dev& d) {
    const int n[3] = {d.nx, d.ny, d.nz};
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k <= n[i]; ++k)
            for (int o = 0; o < 2; ++o) {
                const volatile float X = (float)k + (o ? 0.5f : 0.f);
                const volatile float a = X * d.h[i];
                const volatile float xe = X * d.e[i];
                const volatile float b = d.pow2 ? xe * d.rn[i] : xe / d.nf[i];
                if (a != b) return false;
            }
    return true;
}

// a / b rounded to nearest, as the IEEE division gives it, for a divisor b in
// [2^-30, 2^30] known in advance, with y = 1/b rounded to nearest (the host's
// IEEE division). Markstein's correction (P. W. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990): when y is 1/b rounded to nearest and q lies within one
// ulp of a / b, the remainder r = a - b q is exact in one FMA and RN(q + r y)
// is a / b rounded to nearest. q0 = RN(a y) lies within 1.5 ulp of a / b; the
// first correction brings it within half an ulp plus a term of relative size
// 2^-23 (so within one ulp), the second rounds it correctly. No branch: the
// sign copy makes -0 / b = -0, and |a| > 2^96 (infinities included) returns
// a y, which is the IEEE infinity for an infinite a; NaN stays NaN. The
// quotient is the IEEE one, bit for bit, for +-0, +-inf, NaN and every finite
// a with 2^-96 <= |a| <= 2^96, where no intermediate underflows or overflows:
// checked over all 2^32 inputs per divisor (ffx_division_mismatches). Grid
// positions are 0 or at least an ulp of half a cell, so the excluded
// magnitudes (nonzero below 2^-96, finite above 2^96) never reach it.
__device__ __forceinline__ float div_rn(float a, float b, float y) {
    float q = a * y;
    float r = fmaf(-q, b, a);
    q = fmaf(r, y, q);
    r = fmaf(-q, b, a);
    q = copysignf(fmaf(r, y, q), a);
    return fabsf(a) > 0x1p96f ? a * y : q;
}

// Division by the grid constants e, n and h. When every one of them is a power
// of two (e.g. a 256^3 unit cube) dividing is an exact rescaling, so it is done
// as a multiplication by the exact reciprocal; otherwise by div_rn. Both are
// bit-identical to the IEEE division and several times cheaper. P2 is chosen
// per launch from Dev::pow2.
template <bool P2> __device__ __forceinline__ float dv_e(const Dev& d, float x, int i) {
    return P2 ? x * d.re[i] : div_rn(x, d.e[i], d.re[i]);
}
template <bool P2> __device__ __forceinline__ float dv_n(const Dev& d, float x, int i) {
    return P2 ? x * d.rn[i] : div_rn(x, d.nf[i], d.rn[i]);
}
template <bool P2> __device__ __forceinline__ float dv_h(const Dev& d, float x, int i) {
    return P2 ? x * d.rh[i] : div_rn(x, d.h[i], d.rh[i]);
}

// Every field has fewer than 2^31 elements (checked at the entry points), so
// 32-bit index arithmetic is exact.
__device__ __forceinline__ int cidx(const Dev& d, int x, int y, int z) {
    return x + d.nx * (y + d.ny * z);
}

// ------------------------------------------------------------ launch geometry
// Cell-centric kernels run 32 x 8 thread blocks over (x, y) and one z slice per
// blockIdx.z: coordinates come straight from the launch, with no integer
// division, and each warp covers 32 consecutive x (coalesced rows).
constexpr int kBX = 32, kBY = 8;
inline dim3 cell_block() { return dim3(kBX, kBY, 1); }
inline dim3 cell_grid(int nx, int ny, int nz) {
    return dim3((unsigned)((nx + kBX - 1) / kBX), (unsigned)((ny + kBY - 1) / kBY), (unsigned)nz);
}
// The block a thread works on: the hardware block of a single-domain launch,
// or a tile of one domain inside a batched persistent launch. (x, y, z) index
// tiles of bw x bh threads; (ox, oy) is the thread's place in its tile; gz is
// the number of z tiles (the stride of z-strided reductions).
struct Blk {
    int x, y, z, gz;
    int bw, bh, ox, oy;
};
__device__ __forceinline__ Blk hw_blk() {
    return Blk{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, (int)gridDim.z, kBX, kBY, (int)threadIdx.x,
               (int)threadIdx.y};
}
__device__ __forceinline__ bool cell_coords(const Blk& b, int nx, int ny, int& x, int& y, int& z) {
    x = b.x * b.bw + b.ox;
    y = b.y * b.bh + b.oy;
    z = b.z;
    return x < nx && y < ny;
}
__device__ __forceinline__ bool cell_coords(int nx, int ny, int& x, int& y, int& z) {
    return cell_coords(hw_blk(), nx, ny, x, y, z);
}
// Face kernels: blockIdx.z runs over (axis, z) for the three face grids, each
// padded to the (nx+1, ny+1, nz+1) box.
inline dim3 face_grid(int nx, int ny, int nz) {
    return dim3((unsigned)((nx + 1 + kBX - 1) / kBX), (unsigned)((ny + 1 + kBY - 1) / kBY), (unsigned)(3 * (nz + 1)));
}

// Programmatic dependent launch (launch_pdl): a multigrid pass launched that
// way may be scheduled while the pass before it in the stream is still
// running. Its first statement lets the pass after it be scheduled the same
// way, then waits until the pass before it has finished and its memory is
// visible; only then does it read or write any field. For a pass launched
// normally both instructions have no effect.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

struct F3 { float x, y, z; };
__device__ __forceinline__ float comp(const F3& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
__device__ __forceinline__ float dot3(const F3& a, const F3& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// ---------------------------------------------------------------- samplers
// Clamped trilinear sample of a face grid of size (sx, sy, sz)
// (mac_sample.glsl:2-19).
template <typename T>
__device__ __forceinline__ float sample_face(const T* __restrict__ f, int sx, int sy, int sz,
                                             float qx, float qy, float qz) {
    qx = fminf(fmaxf(qx, 0.f), (float)(sx - 1));
    qy = fminf(fmaxf(qy, 0.f), (float)(sy - 1));
    qz = fminf(fmaxf(qz, 0.f), (float)(sz - 1));
    float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    float fx = qx - bx, fy = qy - by, fz = qz - bz;
    int ix = (int)bx, iy = (int)by, iz = (int)bz;
    int ix1 = min(ix + 1, sx - 1), iy1 = min(iy + 1, sy - 1), iz1 = min(iz + 1, sz - 1);
    int sxy = sx * sy;
    int r00 = iz * sxy + iy * sx, r01 = iz * sxy + iy1 * sx;
    int r10 = iz1 * sxy + iy * sx, r11 = iz1 * sxy + iy1 * sx;
    float gx = 1.f - fx, gy = 1.f - fy, gz = 1.f - fz;
    float v = 0.f;
    v = v + gx * gy * gz * Store<T>::ld(f, r00 + ix);
    v = v + fx * gy * gz * Store<T>::ld(f, r00 + ix1);
    v = v + gx * fy * gz * Store<T>::ld(f, r01 + ix);
    v = v + fx * fy * gz * Store<T>::ld(f, r01 + ix1);
    v = v + gx * gy * fz * Store<T>::ld(f, r10 + ix);
    v = v + fx * gy * fz * Store<T>::ld(f, r10 + ix1);
    v = v + gx * fy * fz * Store<T>::ld(f, r11 + ix);
    v = v + fx * fy * fz * Store<T>::ld(f, r11 + ix1);
    return v;
}

template <typename T>
struct Faces {
    const T* u; const T* v; const T* w;
};

// Staggered velocity at a physical point (mac_sample.glsl:20-26).
template <typename T, bool P2 = false>
__device__ __forceinline__ F3 velocity_at(const Dev& d, const Faces<T>& F, F3 p) {
    float qx = dv_e<P2>(d, p.x * d.nf[0], 0);
    float qy = dv_e<P2>(d, p.y * d.nf[1], 1);
    float qz = dv_e<P2>(d, p.z * d.nf[2], 2);
    F3 r;
    r.x = sample_face(F.u, d.nx + 1, d.ny, d.nz, qx, qy - 0.5f, qz - 0.5f);
    r.y = sample_face(F.v, d.nx, d.ny + 1, d.nz, qx - 0.5f, qy, qz - 0.5f);
    r.z = sample_face(F.w, d.nx, d.ny, d.nz + 1, qx - 0.5f, qy - 0.5f, qz);
    return r;
}

// sample_face at a point whose grid coordinates are exact integers or
// half-integers, given doubled: q = (qx2, qy2, qz2) / 2. Each fraction is then
// 0 or 1/2, every weight a power of two, and a term of zero weight adds a
// signed zero, which leaves the running sum unchanged (it starts at +0 and
// cannot become -0). Summing only the terms of nonzero weight, in
// sample_face's order and with its weight products, therefore gives
// sample_face's value for finite fields, with 1, 2, 4 or 8 loads instead of 8.
template <typename T>
__device__ __forceinline__ float sample_face_half(const T* __restrict__ f, int sx, int sy, int sz, int qx2, int qy2,
                                                  int qz2) {
    qx2 = min(max(qx2, 0), 2 * (sx - 1));
    qy2 = min(max(qy2, 0), 2 * (sy - 1));
    qz2 = min(max(qz2, 0), 2 * (sz - 1));
    const int ix = qx2 >> 1, iy = qy2 >> 1, iz = qz2 >> 1;
    const bool hx = qx2 & 1, hy = qy2 & 1, hz = qz2 & 1;
    const int ix1 = min(ix + 1, sx - 1), iy1 = min(iy + 1, sy - 1), iz1 = min(iz + 1, sz - 1);
    // every term present has the same weight: 1/2 per axis with a half fraction
    const float w = (hx ? 0.5f : 1.f) * (hy ? 0.5f : 1.f) * (hz ? 0.5f : 1.f);
    const int sxy = sx * sy;
    const int r00 = iz * sxy + iy * sx, r01 = iz * sxy + iy1 * sx, r10 = iz1 * sxy + iy * sx,
              r11 = iz1 * sxy + iy1 * sx;
    float v = 0.f;
    v = v + w * Store<T>::ld(f, r00 + ix);
    if (hx) v = v + w * Store<T>::ld(f, r00 + ix1);
    if (hy) {
        v = v + w * Store<T>::ld(f, r01 + ix);
        if (hx) v = v + w * Store<T>::ld(f, r01 + ix1);
    }
    if (hz) {
        v = v + w * Store<T>::ld(f, r10 + ix);
        if (hx) v = v + w * Store<T>::ld(f, r10 + ix1);
        if (hy) {
            v = v + w * Store<T>::ld(f, r11 + ix);
            if (hx) v = v + w * Store<T>::ld(f, r11 + ix1);
        }
    }
    return v;
}

// Staggered velocity at a point with doubled cell coordinates (X2, Y2, Z2)
// (a face centre or cell centre): velocity_at's value, exact when the grid's
// positions round-trip exactly (power-of-two extent, cells and spacing).
template <typename T>
__device__ __forceinline__ F3 velocity_at_node(const Dev& d, const Faces<T>& F, int X2, int Y2, int Z2) {
    F3 r;
    r.x = sample_face_half(F.u, d.nx + 1, d.ny, d.nz, X2, Y2 - 1, Z2 - 1);
    r.y = sample_face_half(F.v, d.nx, d.ny + 1, d.nz, X2 - 1, Y2, Z2 - 1);
    r.z = sample_face_half(F.w, d.nx, d.ny, d.nz + 1, X2 - 1, Y2 - 1, Z2);
    return r;
}

// Velocity at the node p = (X2, Y2, Z2) / 2 cells of the launch thread.
template <typename T, bool P2>
__device__ __forceinline__ F3 velocity_at_start(const Dev& d, const Faces<T>& F, F3 p, int X2, int Y2, int Z2) {
    if constexpr (P2) return velocity_at_node(d, F, X2, Y2, Z2);
    else return velocity_at<T, false>(d, F, p);
}

// Velocity of wall and solid faces: 0 for static walls, the moving colliders'
// rigid-body velocity when the FfxSolids carry wall fields (the
// FLUXFX_MOVING_COLLIDERS variant of pressure_walls.glsl / pressure_gradient.glsl).
struct Walls {
    const float* f[3];
};
inline Walls make_walls(const FfxSolids* s) {
    Walls w;
    for (int a = 0; a < 3; ++a) w.f[a] = s ? s->wall[a] : nullptr;
    return w;
}
__device__ __forceinline__ float wall_value(const Walls& w, int axis, int i) {
    const float* p = w.f[axis];
    return p ? __ldg(p + i) : 0.f;
}

// ---------------------------------------------------------------- colliders
__device__ __forceinline__ bool solid_cell(const Dev& d, const uint8_t* __restrict__ solid,
                                           int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= d.nx || y >= d.ny || z >= d.nz) return true;
    return __ldg(solid + cidx(d, x, y, z)) != 0;
}

__device__ __forceinline__ bool solid_face(const Dev& d, const uint8_t* __restrict__ solid,
                                           int x, int y, int z, int axis) {
    return solid_cell(d, solid, x, y, z) ||
           solid_cell(d, solid, x - (axis == 0), y - (axis == 1), z - (axis == 2));
}

// Voxel DDA clip of the segment origin -> target at the first solid cell, at
// most 384 crossings (solid_boundary.glsl:13-36).
//
// Fast path (exact): when the 3x3x3 blocks around the start cell and the end
// cell hold no solid (dilated mask `halo`) and the end cell is within one cell
// of the start, every cell the traversal can visit -- including a one-cell
// overshoot past the end from rounding of the crossing parameters -- is fluid,
// so the loop would run to t >= 1 and return b / count * extent. That value is
// returned directly; it is bit-identical to the loop's.
template <bool P2 = false>
__device__ __forceinline__ F3 clip_solid_trace(const Dev& d, const uint8_t* __restrict__ solid,
                                               const uint8_t* __restrict__ halo, F3 origin, F3 target) {
    float cnt[3] = {d.nf[0], d.nf[1], d.nf[2]};
    float o[3] = {origin.x, origin.y, origin.z}, t3[3] = {target.x, target.y, target.z};
    float a[3], b[3], delta[3], crossing[3], stride[3];
    int cell[3], dir[3], endc[3];
    for (int i = 0; i < 3; ++i) {
        a[i] = fminf(fmaxf(dv_e<P2>(d, o[i], i) * cnt[i], 0.0001f), cnt[i] - 0.0001f);
        b[i] = fminf(fmaxf(dv_e<P2>(d, t3[i], i) * cnt[i], 0.0001f), cnt[i] - 0.0001f);
        delta[i] = b[i] - a[i];
        cell[i] = (int)floorf(a[i]);
        endc[i] = (int)floorf(b[i]);
        dir[i] = delta[i] > 0.f ? 1 : (delta[i] < 0.f ? -1 : 0);
        crossing[i] = 1e20f;
        stride[i] = 1e20f;
    }
    if (halo && abs(endc[0] - cell[0]) <= 1 && abs(endc[1] - cell[1]) <= 1 && abs(endc[2] - cell[2]) <= 1 &&
        !__ldg(halo + cidx(d, cell[0], cell[1], cell[2])) && !__ldg(halo + cidx(d, endc[0], endc[1], endc[2]))) {
        F3 r = {dv_n<P2>(d, b[0], 0) * d.e[0], dv_n<P2>(d, b[1], 1) * d.e[1], dv_n<P2>(d, b[2], 2) * d.e[2]};
        return r;
    }
    if (solid_cell(d, solid, cell[0], cell[1], cell[2])) return origin;
    for (int i = 0; i < 3; ++i) {
        if (fabsf(delta[i]) > 1e-10f) {
            float edge = (float)(cell[i] + (dir[i] > 0 ? 1 : 0));
            crossing[i] = (edge - a[i]) / delta[i];
            stride[i] = 1.0f / fabsf(delta[i]);
        }
    }
    float len = sqrtf((delta[0] * delta[0] + delta[1] * delta[1]) + delta[2] * delta[2]);
    for (int it = 0; it < 384; ++it) {
        int axis = (crossing[0] <= crossing[1] && crossing[0] <= crossing[2]) ? 0
                   : (crossing[1] <= crossing[2] ? 1 : 2);
        float t = crossing[axis];
        if (t >= 1.0f) {
            F3 r = {dv_n<P2>(d, b[0], 0) * d.e[0], dv_n<P2>(d, b[1], 1) * d.e[1], dv_n<P2>(d, b[2], 2) * d.e[2]};
            return r;
        }
        cell[axis] += dir[axis];
        if (solid_cell(d, solid, cell[0], cell[1], cell[2])) {
            float back = fmaxf(0.f, t - 0.0001f / fmaxf(len, 1.0f));
            F3 r = {dv_n<P2>(d, a[0] + delta[0] * back, 0) * d.e[0], dv_n<P2>(d, a[1] + delta[1] * back, 1) * d.e[1],
                    dv_n<P2>(d, a[2] + delta[2] * back, 2) * d.e[2]};
            return r;
        }
        crossing[axis] += stride[axis];
    }
    return origin;
}

// Any solid (or out-of-domain) cell in the 3x3x3 block around p, read from the
// precomputed dilated mask (solid_boundary.glsl:39-44).
template <bool P2 = false>
__device__ __forceinline__ bool solid_halo(const Dev& d, const uint8_t* __restrict__ halo, F3 p) {
    // Clamp before the integer conversion so far-away (or non-finite) points
    // land outside the grid, i.e. count as solid.
    int cx = (int)fmaxf(fminf(floorf(dv_e<P2>(d, p.x, 0) * d.nf[0]), 1.0e9f), -1.0e9f);
    int cy = (int)fmaxf(fminf(floorf(dv_e<P2>(d, p.y, 1) * d.nf[1]), 1.0e9f), -1.0e9f);
    int cz = (int)fmaxf(fminf(floorf(dv_e<P2>(d, p.z, 2) * d.nf[2]), 1.0e9f), -1.0e9f);
    if (cx < 0 || cy < 0 || cz < 0 || cx >= d.nx || cy >= d.ny || cz >= d.nz) return true;
    return __ldg(halo + cidx(d, cx, cy, cz)) != 0;
}

__device__ __forceinline__ float dist3(F3 a, F3 b) {
    F3 c = {a.x - b.x, a.y - b.y, a.z - b.z};
    return sqrtf(dot3(c, c));
}

// dist3(a, b) < 1e-7f without the square root: sqrtf is correctly rounded and
// monotone, so sqrtf(q) < 1e-7f holds exactly when q < 1e-14f (the float
// nearest 1e-14, 0x1.6849b8p-47), for every q including NaN and infinity.
__device__ __forceinline__ bool within_1e7(F3 a, F3 b) {
    F3 c = {a.x - b.x, a.y - b.y, a.z - b.z};
    return dot3(c, c) < 0x1.6849b8p-47f;
}

// Grid coordinates q = t / e * n of a point and the cell floor(q), clamped
// before the integer conversion as in solid_halo.
struct Probe {
    float q[3];
    int c[3];
};
template <bool P2>
__device__ __forceinline__ bool probe_inside(const Dev& d, F3 t, Probe& r) {
    const float tt[3] = {t.x, t.y, t.z};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        r.q[i] = dv_e<P2>(d, tt[i], i) * d.nf[i];
        r.c[i] = (int)fmaxf(fminf(floorf(r.q[i]), 1.0e9f), -1.0e9f);
    }
    return r.c[0] >= 0 && r.c[1] >= 0 && r.c[2] >= 0 && r.c[0] < d.nx && r.c[1] < d.ny && r.c[2] < d.nz;
}

// Whether the MacCormack correction may be applied near colliders
// (correct_velocity_fused.glsl / correct_scalar.glsl: no solid in the 3x3x3
// blocks around the start, departure and arrival points, and none of the
// three segments from the start clipped by a collider). Evaluated as
//   !solid_halo(p) && !solid_halo(dep) && !solid_halo(arr) &&
//   dist3(clip_solid_trace(p, t), t) < 1e-7f for t = dep, mid, arr
// with the shared work done once: solid_halo's cell of an in-grid point is
// the clip's start / end cell (floor(clamp(q, 1e-4, n - 1e-4)) = floor(q) for
// q in [0, n)), so its halo tests stand for the clip's, and the clip's
// fast-path value is formed here; a segment the fast path does not cover
// takes the full clip.
template <bool P2 = false>
__device__ __forceinline__ bool safe_solid_correction(const Dev& d, const uint8_t* solid,
                                                      const uint8_t* halo, F3 p, F3 dep, F3 mid,
                                                      F3 arr) {
    Probe pp, pd, pa;
    if (!probe_inside<P2>(d, p, pp) || __ldg(halo + cidx(d, pp.c[0], pp.c[1], pp.c[2]))) return false;
    if (!probe_inside<P2>(d, dep, pd) || __ldg(halo + cidx(d, pd.c[0], pd.c[1], pd.c[2]))) return false;
    if (!probe_inside<P2>(d, arr, pa) || __ldg(halo + cidx(d, pa.c[0], pa.c[1], pa.c[2]))) return false;
    // clip_solid_trace(p, t) where t's halo cell is known (known_clear) or not
    auto clipped_ok = [&](F3 t, const Probe& pt, bool known_clear) -> bool {
        float b[3];
        int e[3];
        bool near = true;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            b[i] = fminf(fmaxf(pt.q[i], 0.0001f), d.nf[i] - 0.0001f);
            e[i] = known_clear ? pt.c[i] : (int)floorf(b[i]);
            near = near && abs(e[i] - pp.c[i]) <= 1;
        }
        if (near && (known_clear || !__ldg(halo + cidx(d, e[0], e[1], e[2])))) {
            const F3 r = {dv_n<P2>(d, b[0], 0) * d.e[0], dv_n<P2>(d, b[1], 1) * d.e[1], dv_n<P2>(d, b[2], 2) * d.e[2]};
            return within_1e7(r, t);
        }
        return within_1e7(clip_solid_trace<P2>(d, solid, halo, p, t), t);
    };
    if (!clipped_ok(dep, pd, true)) return false;
    Probe pm;
    probe_inside<P2>(d, mid, pm);
    if (!clipped_ok(mid, pm, false)) return false;
    return clipped_ok(arr, pa, true);
}

// ---------------------------------------------------------------- clearance
// `clear` (ffx_clearance, ffx_halo_clearance) holds one byte per cell:
//   1  no solid and no out-of-domain cell within Chebyshev distance 3;
//   2  no solid cell within distance 3, but an out-of-domain one (the cell lies
//      within three cells of a wall); ffx_clearance, which sees only the
//      dilated mask, never writes 2;
//   0  otherwise.
// Let p be the start point of a face or cell whose own cell c (its integer
// cell coordinates) has a nonzero value, and t a target within 0.75 h of p on
// every axis. floor(p / h * n) is c or a neighbour of c (rounding of the grid
// coordinate), and t's cell lies within one cell of that.
//  * Value 1: both cells lie at distance >= 2 from every solid or outside
//    cell, with a clear 3x3x3 block (halo 0), so clip_solid_trace(p, t) takes
//    its fast path with unclamped grid coordinates and returns t / e * n / n *
//    e (clear_clip), which is t itself when e, n and h are powers of two; and
//    safe_solid_correction(p, dep, mid, arr) with all three near p finds every
//    probe inside the grid with a clear halo and every segment on the fast
//    path, so it reduces to the three distance tests of the fast values
//    (clear_correction), always true on power-of-two grids.
//  * Value 2: every cell the functions visit lies within distance 3 of c and
//    is not a solid; only the grid's walls can matter. The clip's grid
//    coordinates are clamped to [1e-4, n - 1e-4], so a traversal of at most
//    0.75 cells (plus rounding) never crosses a wall: the crossing parameter
//    of a wall exceeds 1 by at least 1e-4 / 0.76, far beyond rounding. So
//    clip_solid_trace(p, t), fast path or traversal, returns the clamped
//    rescale (wall_clip). In safe_solid_correction a probe cell has halo 0
//    exactly when it lies in [1, n - 2] on every axis (inner); when p's cell
//    does, the midpoint is at least 0.25 cells from the walls and unclamped,
//    as are the departure and arrival points whose cells do, so the test
//    reduces to inner(p), inner(dep), inner(arr) and clear_correction
//    (wall_correction). A face of the cell is blocked only at the lower grid
//    wall (its lower cell lies outside); the cell itself is fluid, and so are
//    the clamped corners of a scalar sample within 0.75 h.
// Both forms give the functions' results bit for bit and skip their mask reads.
__device__ __forceinline__ int home_clearance(const uint8_t* __restrict__ clear, const Dev& d, int x, int y,
                                              int z) {
    return clear != nullptr && x < d.nx && y < d.ny && z < d.nz ? (int)__ldg(clear + cidx(d, x, y, z)) : 0;
}

__device__ __forceinline__ bool near_start(const Dev& d, F3 p, F3 t) {
    return fabsf(t.x - p.x) <= 0.75f * d.h[0] && fabsf(t.y - p.y) <= 0.75f * d.h[1] &&
           fabsf(t.z - p.z) <= 0.75f * d.h[2];
}

template <bool P2>
__device__ __forceinline__ F3 clear_clip(const Dev& d, F3 t) {
    if constexpr (P2) {
        return t;
    } else {
        return F3{dv_n<P2>(d, dv_e<P2>(d, t.x, 0) * d.nf[0], 0) * d.e[0],
                  dv_n<P2>(d, dv_e<P2>(d, t.y, 1) * d.nf[1], 1) * d.e[1],
                  dv_n<P2>(d, dv_e<P2>(d, t.z, 2) * d.nf[2], 2) * d.e[2]};
    }
}

// clip_solid_trace's value for a cell of clearance 2 (its fast-path formula
// with the wall clamp).
template <bool P2>
__device__ __forceinline__ F3 wall_clip(const Dev& d, F3 t) {
    const float tt[3] = {t.x, t.y, t.z};
    float r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float b = fminf(fmaxf(dv_e<P2>(d, tt[i], i) * d.nf[i], 0.0001f), d.nf[i] - 0.0001f);
        r[i] = dv_n<P2>(d, b, i) * d.e[i];
    }
    return F3{r[0], r[1], r[2]};
}

// The probe cell of t (probe_inside) lies in [1, n - 2] on every axis.
template <bool P2>
__device__ __forceinline__ bool inner_cell(const Dev& d, F3 t) {
    const float tt[3] = {t.x, t.y, t.z};
    const int n[3] = {d.nx, d.ny, d.nz};
    bool in = true;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int c = (int)fmaxf(fminf(floorf(dv_e<P2>(d, tt[i], i) * d.nf[i]), 1.0e9f), -1.0e9f);
        in = in && c >= 1 && c <= n[i] - 2;
    }
    return in;
}

template <bool P2>
__device__ __forceinline__ bool clear_correction(const Dev& d, F3 dep, F3 mid, F3 arr) {
    if constexpr (P2) {
        return true;
    } else {
        return within_1e7(clear_clip<P2>(d, dep), dep) && within_1e7(clear_clip<P2>(d, mid), mid) &&
               within_1e7(clear_clip<P2>(d, arr), arr);
    }
}

// clip_solid_trace(p, t), through the clear forms where they apply (cv: the
// start cell's clearance).
template <bool P2>
__device__ __forceinline__ F3 clip_from(const Dev& d, const uint8_t* solid, const uint8_t* halo, int cv, F3 p,
                                        F3 t) {
    if (cv != 0 && near_start(d, p, t)) return cv == 1 ? clear_clip<P2>(d, t) : wall_clip<P2>(d, t);
    return clip_solid_trace<P2>(d, solid, halo, p, t);
}

// safe_solid_correction(p, dep, mid, arr), through the clear forms where they apply.
template <bool P2>
__device__ __forceinline__ bool safe_correction_from(const Dev& d, const uint8_t* solid, const uint8_t* halo,
                                                     int cv, F3 p, F3 dep, F3 mid, F3 arr) {
    if (cv != 0 && near_start(d, p, dep) && near_start(d, p, mid) && near_start(d, p, arr))
        return (cv == 1 || (inner_cell<P2>(d, p) && inner_cell<P2>(d, dep) && inner_cell<P2>(d, arr))) &&
               clear_correction<P2>(d, dep, mid, arr);
    return safe_solid_correction<P2>(d, solid, halo, p, dep, mid, arr);
}

// solid_face for a face whose own cell has a nonzero clearance cv: only the
// lower grid wall (the face's lower cell outside) can block it.
__device__ __forceinline__ bool clear_face_blocked(int cv, int x, int y, int z, int axis) {
    return cv == 2 && (axis == 0 ? x : (axis == 1 ? y : z)) == 0;
}

// ---------------------------------------------------------------- emitters
// Exact time average of the compact sphere profile along a linear sweep
// (emission_weight.glsl:2-29).
__device__ __forceinline__ float emission_weight(F3 p, F3 center, F3 start, float radius, bool solid) {
    F3 seg = {center.x - start.x, center.y - start.y, center.z - start.z};
    float l2 = dot3(seg, seg);
    float r2 = radius * radius;
    if (l2 < 1e-12f) {
        F3 dd = {p.x - center.x, p.y - center.y, p.z - center.z};
        float q = dot3(dd, dd);
        float w = fmaxf(1.0f - q / r2, 0.0f);
        return solid ? (q < r2 ? 1.0f : 0.0f) : w * w;
    }
    float lp = sqrtf(l2);
    F3 ax = {seg.x / lp, seg.y / lp, seg.z / lp};
    F3 off = {p.x - start.x, p.y - start.y, p.z - start.z};
    float along = dot3(off, ax);
    F3 perp = {off.x - along * ax.x, off.y - along * ax.y, off.z - along * ax.z};
    float a = 1.0f - dot3(perp, perp) / r2;
    if (a <= 0.0f) return 0.0f;
    float half = radius * sqrtf(a);
    float lo = fmaxf(-along, -half);
    float hi = fminf(lp - along, half);
    if (hi <= lo) return 0.0f;
    if (solid) return (hi - lo) / lp;
    float u = lo / half, v = hi / half;
    float integral = (v - u) - (2.0f / 3.0f) * (v * v * v - u * u * u) + 0.2f * (v * v * v * v * v - u * u * u * u * u);
    return fminf(fmaxf(a * a * half / lp * integral, 0.0f), 1.0f);
}

// Reach of an emitter: an axis-aligned box outside which emission_weight is
// exactly 0.0f, so the weight need not be evaluated there.
//
// In real arithmetic the weight is non-zero only within distance r of the
// segment start..center (a capsule; a sphere around center when the segment is
// degenerate), and zero when the distance is >= r. Evaluated in FP32, the
// perpendicular distance and the along-axis position of a point p carry
// absolute errors of at most ~12 eps |p - start| (eps = 2^-24), and
// |p - start| <= sqrt(3) * 2M for M = max(|extent|, |start|, |center|, r)
// since grid positions lie in [0, extent]. So a point farther than
// r + 1e-3 * 4M from the segment evaluates to exactly zero (the a <= 0 or
// hi <= lo branch; both return +0.0f), and every point outside the box
// [min(start, center) - r - 4e-3 M, max(start, center) + r + 4e-3 M] is that
// far. The bounds are rounded outwards to float. A NaN anywhere leaves the
// box unusable (comparisons are false), and the weight is then evaluated.
struct Reach {
    float lo[3], hi[3];
};

inline float round_down_f(double x) {
    float f = (float)x;
    return (double)f > x ? std::nextafter(f, -INFINITY) : f;
}
inline float round_up_f(double x) {
    float f = (float)x;
    return (double)f < x ? std::nextafter(f, INFINITY) : f;
}

inline Reach make_reach(const float* center, const float* start, float radius, const float* extent) {
    double m = std::fabs((double)radius);
    for (int a = 0; a < 3; ++a)
        m = std::fmax(m, std::fmax(std::fabs((double)extent[a]),
                                   std::fmax(std::fabs((double)center[a]), std::fabs((double)start[a]))));
    double margin = std::fabs((double)radius) + 4e-3 * m;
    Reach r;
    for (int a = 0; a < 3; ++a) {
        r.lo[a] = round_down_f(std::fmin((double)center[a], (double)start[a]) - margin);
        r.hi[a] = round_up_f(std::fmax((double)center[a], (double)start[a]) + margin);
    }
    return r;
}

__device__ __forceinline__ bool outside(const Reach& r, F3 p) {
    return p.x < r.lo[0] || p.x > r.hi[0] || p.y < r.lo[1] || p.y > r.hi[1] || p.z < r.lo[2] || p.z > r.hi[2];
}

struct SrcDev {
    int count;
    int single_solid;
    F3 center, start, jet;
    float radius, coupling;
    float table[128];
    Reach reach[9];   // table rows 0..7, then the single emitter
    Reach any;        // a box holding the reach of every table row in use
};

inline SrcDev make_src(const FfxSources* s, const float* extent) {
    SrcDev r;
    r.count = s ? s->count : -1;
    r.single_solid = s ? s->single_solid_profile : 0;
    r.center = {s ? s->single_center[0] : 0.f, s ? s->single_center[1] : 0.f, s ? s->single_center[2] : 0.f};
    r.start = {s ? s->single_start[0] : 0.f, s ? s->single_start[1] : 0.f, s ? s->single_start[2] : 0.f};
    r.jet = {s ? s->single_jet[0] : 0.f, s ? s->single_jet[1] : 0.f, s ? s->single_jet[2] : 0.f};
    r.radius = s ? s->single_radius : 1.f;
    r.coupling = s ? s->single_coupling : 0.f;
    for (int i = 0; i < 128; ++i) r.table[i] = s ? s->table[i] : 0.f;
    for (int i = 0; i < 8; ++i) {
        const float* row = r.table + 16 * i;
        r.reach[i] = make_reach(row, row + 4, row[3], extent);
    }
    const float c[3] = {r.center.x, r.center.y, r.center.z}, st[3] = {r.start.x, r.start.y, r.start.z};
    r.reach[8] = make_reach(c, st, r.radius, extent);
    // the union of the rows' boxes (NaN if any bound is NaN: never outside);
    // a point outside it is outside every row's box
    for (int a = 0; a < 3; ++a) {
        float lo = INFINITY, hi = -INFINITY;
        bool nan = false;
        for (int i = 0; i < r.count && i < 8; ++i) {
            nan = nan || std::isnan(r.reach[i].lo[a]) || std::isnan(r.reach[i].hi[a]);
            lo = std::fmin(lo, r.reach[i].lo[a]);
            hi = std::fmax(hi, r.reach[i].hi[a]);
        }
        r.any.lo[a] = nan ? NAN : lo;
        r.any.hi[a] = nan ? NAN : hi;
    }
    return r;
}

__device__ __forceinline__ float table_weight(const SrcDev& s, int i, F3 p) {
    if (outside(s.reach[i], p)) return 0.0f;
    const float* row = s.table + 16 * i;
    F3 c = {row[0], row[1], row[2]}, st = {row[4], row[5], row[6]};
    return emission_weight(p, c, st, row[3], row[14] > 0.5f);
}

__device__ __forceinline__ float single_weight(const SrcDev& s, F3 p) {
    if (outside(s.reach[8], p)) return 0.0f;
    return emission_weight(p, s.center, s.start, s.radius, s.single_solid != 0);
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ float finite_abs(float v) {
    return isfinite(v) ? fabsf(v) : 3.4e38f;
}
// Non-negative floats order like their bit patterns.
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
    atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}
__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// Block-wide max then one atomic per block (block size a multiple of 32, <= 1024).
__device__ __forceinline__ void block_max_to(float* out, float v) {
    __shared__ float part[32];
    v = warp_max(v);
    int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) part[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
        float m = lane < nw ? part[lane] : 0.f;
        m = warp_max(m);
        if (lane == 0 && m > 0.f) atomic_max_nonneg(out, m);
    }
}

// out[k] raised to the block-wide max of v[k] for k < count (count <= K), with
// one barrier for all of them (the same maxima as K calls of block_max_to). A
// caller that runs it again in the same block (a persistent loop) puts a
// barrier in between.
template <int K>
__device__ __forceinline__ void block_max_to_n(float* out, const float (&v)[K], int count) {
    __shared__ float part[K][32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const float w = warp_max(v[k]);
        if (lane == 0) part[k][wid] = w;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            float m = lane < nw ? part[k][lane] : 0.f;
            m = warp_max(m);
            if (k < count && lane == 0 && m > 0.f) atomic_max_nonneg(out + k, m);
        }
    }
}

}  // namespace ffx
