// Shared-memory tiles for the transport passes.
//
// A block owns 32 x 8 columns of the grid (x, y) and marches up a chunk of z
// slices. For every field it reads (velocity faces, predictor faces, scalars)
// it keeps a ring of four z slices in shared memory: slices z-1 .. z+2 while
// it works on slice z. Each slice holds a 36 x 12 window, global indices
// x0-1 .. x0+34 and y0-1 .. y0+10, and every entry is staged from the CLAMPED
// global index (clamp(x, 0, sx-1) and likewise for y and z, per field). That
// replication is what a clamped trilinear sample reads anyway: for a lower
// corner index i in [0, s-1] the upper corner min(i+1, s-1) is exactly the
// window entry after i, so a sample reads its eight corners at constant
// offsets from one base with no per-corner clamping.
//
// A face or cell at (x, y, z) traced by at most half a cell (the CFL bound of
// the step's time step) samples lower corners in [x-1, x+1] on every axis, so
// it stays in the window. Any sample outside it (a larger time step, a trace
// that ran farther) is taken from global memory by the untiled sampler; the
// tiled and untiled samples read the same values and do the same arithmetic in
// the same order, so they are bit-identical.
#pragma once
#include <type_traits>

#include "ffx_common.cuh"

namespace ffx {
namespace tile {

constexpr int kTX = 32, kTY = 8;                 // threads (columns) of a block
constexpr int kPitch = kTX + 4;                  // window x: x0-1 .. x0+34
constexpr int kRows = kTY + 4;                   // window y: y0-1 .. y0+10
constexpr int kSlice = kPitch * kRows;           // floats per slice
constexpr int kRingSlices = 4;
constexpr int kRing = kRingSlices * kSlice;      // floats per field
constexpr int kThreads = kTX * kTY;
constexpr int kMaxLowX = kPitch - 2, kMaxLowY = kRows - 2;   // largest lower-corner offsets

// The window a block works on.
struct Window {
    const float* s;    // ring of field 0; field k at s + k * kRing
    int wx, wy;        // global index of window entry (0, 0)
    int zlo;           // lowest slice in the ring: z - 1 while slice z is worked on
};

__device__ __forceinline__ const float* slice_of(const float* ring, int zg) {
    return ring + (zg & (kRingSlices - 1)) * kSlice;
}

// Stage global slice zg of a field of size (sx, sy, sz) into its ring slot.
template <typename T>
__device__ __forceinline__ void stage(float* ring, const T* __restrict__ g, int sx, int sy, int sz, int wx, int wy,
                                      int zg, int tid) {
    float* dst = ring + (zg & (kRingSlices - 1)) * kSlice;
    const int gz = min(max(zg, 0), sz - 1);
    const int64_t plane = (int64_t)sx * sy * gz;
    for (int e = tid; e < kSlice; e += kThreads) {
        const int ly = e / kPitch, lx = e - ly * kPitch;
        const int gx = min(max(wx + lx, 0), sx - 1), gy = min(max(wy + ly, 0), sy - 1);
        dst[e] = Store<T>::ld(g, plane + (int64_t)sx * gy + gx);
    }
}

// Whether the lower corner (ix, iy, iz) and its +1 neighbours lie in the window.
__device__ __forceinline__ bool inside(const Window& w, int ix, int iy, int iz) {
    return (unsigned)(ix - w.wx) <= (unsigned)kMaxLowX && (unsigned)(iy - w.wy) <= (unsigned)kMaxLowY &&
           (unsigned)(iz - w.zlo) <= 2u;
}

// The eight corners of field k around lower corner (ix, iy, iz): c0 is the
// (iz) slice, c1 the (iz + 1) slice; corner (ox, oy) at c[oy * kPitch + ox].
struct Corners {
    const float* c0;
    const float* c1;
};
__device__ __forceinline__ Corners corners(const Window& w, int k, int ix, int iy, int iz) {
    const float* ring = w.s + k * kRing;
    const int off = (iy - w.wy) * kPitch + (ix - w.wx);
    return Corners{slice_of(ring, iz) + off, slice_of(ring, iz + 1) + off};
}

// sample_face (mac_sample.glsl:2-19) of field k from the window, else `g`.
template <typename T>
__device__ __forceinline__ float sample(const Window& w, int k, const T* __restrict__ g, int sx, int sy, int sz,
                                        float qx, float qy, float qz) {
    qx = fminf(fmaxf(qx, 0.f), (float)(sx - 1));
    qy = fminf(fmaxf(qy, 0.f), (float)(sy - 1));
    qz = fminf(fmaxf(qz, 0.f), (float)(sz - 1));
    const float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    const int ix = (int)bx, iy = (int)by, iz = (int)bz;
    if (!inside(w, ix, iy, iz)) return sample_face(g, sx, sy, sz, qx, qy, qz);
    const float fx = qx - bx, fy = qy - by, fz = qz - bz;
    const Corners c = corners(w, k, ix, iy, iz);
    const float gx = 1.f - fx, gy = 1.f - fy, gz = 1.f - fz;
    float v = 0.f;
    v = v + gx * gy * gz * c.c0[0];
    v = v + fx * gy * gz * c.c0[1];
    v = v + gx * fy * gz * c.c0[kPitch];
    v = v + fx * fy * gz * c.c0[kPitch + 1];
    v = v + gx * gy * fz * c.c1[0];
    v = v + fx * gy * fz * c.c1[1];
    v = v + gx * fy * fz * c.c1[kPitch];
    v = v + fx * fy * fz * c.c1[kPitch + 1];
    return v;
}

// sample_face_half (a node sample: doubled coordinates) of field k.
template <typename T>
__device__ __forceinline__ float sample_half(const Window& w, int k, const T* __restrict__ g, int sx, int sy, int sz,
                                             int qx2, int qy2, int qz2) {
    qx2 = min(max(qx2, 0), 2 * (sx - 1));
    qy2 = min(max(qy2, 0), 2 * (sy - 1));
    qz2 = min(max(qz2, 0), 2 * (sz - 1));
    const int ix = qx2 >> 1, iy = qy2 >> 1, iz = qz2 >> 1;
    if (!inside(w, ix, iy, iz)) return sample_face_half(g, sx, sy, sz, qx2, qy2, qz2);
    const bool hx = qx2 & 1, hy = qy2 & 1, hz = qz2 & 1;
    const float wt = (hx ? 0.5f : 1.f) * (hy ? 0.5f : 1.f) * (hz ? 0.5f : 1.f);
    const Corners c = corners(w, k, ix, iy, iz);
    float v = 0.f;
    v = v + wt * c.c0[0];
    if (hx) v = v + wt * c.c0[1];
    if (hy) {
        v = v + wt * c.c0[kPitch];
        if (hx) v = v + wt * c.c0[kPitch + 1];
    }
    if (hz) {
        v = v + wt * c.c1[0];
        if (hx) v = v + wt * c.c1[1];
        if (hy) {
            v = v + wt * c.c1[kPitch];
            if (hx) v = v + wt * c.c1[kPitch + 1];
        }
    }
    return v;
}

}  // namespace tile

// ------------------------------------------------------- closed sampling
__device__ __forceinline__ int floor_int(float v) {
    return (int)fmaxf(fminf(floorf(v), 1.0e9f), -1.0e9f);
}

// sample_closed split in two for several scalars sampled at one point: the
// stencil (clamped corners, fractions and, with colliders, which corners are
// fluid and the sum of their weights) is formed once, then applied to each
// field with sample_closed's operations in its order, so every channel's
// value is sample_closed's.
struct ClosedStencil {
    int rows[4];          // cidx(0, y, z) of (y0, z0), (y1, z0), (y0, z1), (y1, z1)
    int x0, x1;
    float fx, fy, fz;
    unsigned fluid;       // MASK: bit k set when corner k (z, y, x order) is fluid
    float total;          // MASK: sum of the fluid corners' weights
};

// fluid: every corner is known to be fluid (a departure point near a clear
// cell's centre: its corners lie within one cell of it), so the mask is not read.
template <bool MASK>
__device__ __forceinline__ ClosedStencil closed_stencil(const Dev& d, const uint8_t* solid, float qx, float qy,
                                                        float qz, bool fluid = false) {
    ClosedStencil S;
    float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    S.fx = qx - bx;
    S.fy = qy - by;
    S.fz = qz - bz;
    int ix = floor_int(qx), iy = floor_int(qy), iz = floor_int(qz);
    S.x0 = min(max(ix, 0), d.nx - 1);
    S.x1 = min(max(ix + 1, 0), d.nx - 1);
    const int y0 = min(max(iy, 0), d.ny - 1), y1 = min(max(iy + 1, 0), d.ny - 1);
    const int z0 = min(max(iz, 0), d.nz - 1), z1 = min(max(iz + 1, 0), d.nz - 1);
    S.rows[0] = cidx(d, 0, y0, z0);
    S.rows[1] = cidx(d, 0, y1, z0);
    S.rows[2] = cidx(d, 0, y0, z1);
    S.rows[3] = cidx(d, 0, y1, z1);
    S.fluid = 0u;
    S.total = 0.f;
    if (MASK) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int c = S.rows[k >> 1] + ((k & 1) ? S.x1 : S.x0);
            if (!fluid && __ldg(solid + c)) continue;
            const float wz = (k & 4) ? S.fz : 1.f - S.fz, wy = (k & 2) ? S.fy : 1.f - S.fy,
                        wx = (k & 1) ? S.fx : 1.f - S.fx;
            S.fluid |= 1u << k;
            S.total = S.total + wx * wy * wz;
        }
    }
    return S;
}

template <typename T, bool MASK>
__device__ __forceinline__ float apply_closed(const ClosedStencil& S, const T* __restrict__ f) {
    if (MASK) {
        float value = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (!(S.fluid & (1u << k))) continue;
            const float wz = (k & 4) ? S.fz : 1.f - S.fz, wy = (k & 2) ? S.fy : 1.f - S.fy,
                        wx = (k & 1) ? S.fx : 1.f - S.fx;
            value = value + wx * wy * wz * Store<T>::ld(f, S.rows[k >> 1] + ((k & 1) ? S.x1 : S.x0));
        }
        return S.total > 1e-8f ? value / S.total : 0.f;
    }
    float f000 = Store<T>::ld(f, S.rows[0] + S.x0), f100 = Store<T>::ld(f, S.rows[0] + S.x1);
    float f010 = Store<T>::ld(f, S.rows[1] + S.x0), f110 = Store<T>::ld(f, S.rows[1] + S.x1);
    float f001 = Store<T>::ld(f, S.rows[2] + S.x0), f101 = Store<T>::ld(f, S.rows[2] + S.x1);
    float f011 = Store<T>::ld(f, S.rows[3] + S.x0), f111 = Store<T>::ld(f, S.rows[3] + S.x1);
    const float fx = S.fx, fy = S.fy, fz = S.fz;
    float gx = 1.f - fx, gy = 1.f - fy, gz = 1.f - fz;
    float a0 = f000 * gx + f100 * fx, a1 = f010 * gx + f110 * fx;
    float b0 = f001 * gx + f101 * fx, b1 = f011 * gx + f111 * fx;
    float zz0 = a0 * gy + a1 * fy, zz1 = b0 * gy + b1 * fy;
    return zz0 * gz + zz1 * fz;
}

// ------------------------------------------------------------------ samplers
// The transport bodies read their fields through a sampler: field k < 3 is
// velocity component k; fields 3..5 are the predictor faces (FaceFields) or
// the transported scalars (CellFields). GlobalSampler gathers from global
// memory; TileSampler reads the block's shared-memory window and falls back to
// the global gather outside it. The field tables refer to the launch
// parameters, so pointers and sizes are read where they are used instead of
// being held in registers.
template <typename T>
struct FaceFields {
    const Dev& d;
    const Faces<T>& A;    // velocity
    const Faces<T>& B;    // predictor faces
    __device__ __forceinline__ const T* ptr(int k) const {
        const Faces<T>& F = k < 3 ? A : B;
        const int a = k < 3 ? k : k - 3;
        return a == 0 ? F.u : (a == 1 ? F.v : F.w);
    }
    __device__ __forceinline__ void dims(int k, int& sx, int& sy, int& sz) const {
        const int a = k < 3 ? k : k - 3;
        sx = d.nx + (a == 0);
        sy = d.ny + (a == 1);
        sz = d.nz + (a == 2);
    }
};

template <typename T>
struct CellFields {
    const Dev& d;
    const Faces<T>& A;    // velocity
    const T* const* C;    // scalar fields 3, 4, 5 (C[0], C[1], C[2])
    __device__ __forceinline__ const T* ptr(int k) const {
        return k == 0 ? A.u : (k == 1 ? A.v : (k == 2 ? A.w : C[k - 3]));
    }
    __device__ __forceinline__ void dims(int k, int& sx, int& sy, int& sz) const {
        sx = d.nx + (k == 0);
        sy = d.ny + (k == 1);
        sz = d.nz + (k == 2);
    }
};

template <class Fields>
struct GlobalSampler {
    Fields f;

    __device__ __forceinline__ float sample(int k, float qx, float qy, float qz) const {
        int sx, sy, sz;
        f.dims(k, sx, sy, sz);
        return sample_face(f.ptr(k), sx, sy, sz, qx, qy, qz);
    }
    __device__ __forceinline__ float half(int k, int qx2, int qy2, int qz2) const {
        int sx, sy, sz;
        f.dims(k, sx, sy, sz);
        return sample_face_half(f.ptr(k), sx, sy, sz, qx2, qy2, qz2);
    }
    // sample_face_half of field k at the node whose doubled coordinates have the
    // parities (HX, HY, HZ) and lower corner (ix, iy, iz), for a node where no
    // coordinate is clamped (the corners ix..ix+HX etc. lie in the field): the
    // same terms in the same order with the same power-of-two weight, with the
    // parities known when compiling.
    template <int HX, int HY, int HZ>
    __device__ __forceinline__ float node(int k, int ix, int iy, int iz) const {
        int sx, sy, sz;
        f.dims(k, sx, sy, sz);
        const auto* g = f.ptr(k);
        using E = typename std::remove_cv<typename std::remove_pointer<decltype(g)>::type>::type;
        constexpr float w = (HX ? 0.5f : 1.f) * (HY ? 0.5f : 1.f) * (HZ ? 0.5f : 1.f);
        const int sxy = sx * sy;
        const int b = iz * sxy + iy * sx + ix;
        float v = 0.f;
        v = v + w * Store<E>::ld(g, b);
        if (HX) v = v + w * Store<E>::ld(g, b + 1);
        if (HY) {
            v = v + w * Store<E>::ld(g, b + sx);
            if (HX) v = v + w * Store<E>::ld(g, b + sx + 1);
        }
        if (HZ) {
            v = v + w * Store<E>::ld(g, b + sxy);
            if (HX) v = v + w * Store<E>::ld(g, b + sxy + 1);
            if (HY) {
                v = v + w * Store<E>::ld(g, b + sxy + sx);
                if (HX) v = v + w * Store<E>::ld(g, b + sxy + sx + 1);
            }
        }
        return v;
    }
    // min / max over the eight corners of field k around lower corner (bx, by,
    // bz), each index clamped to the field (correct_velocity_fused.glsl:19-24,
    // correct_scalar.glsl:12-17)
    __device__ __forceinline__ void minmax8(int k, int bx, int by, int bz, float& lo, float& hi) const {
        int sx, sy, sz;
        f.dims(k, sx, sy, sz);
        const auto* g = f.ptr(k);
        const int cx0 = min(max(bx, 0), sx - 1), cx1 = min(max(bx + 1, 0), sx - 1);
        const int cy0 = min(max(by, 0), sy - 1), cy1 = min(max(by + 1, 0), sy - 1);
        const int cz0 = min(max(bz, 0), sz - 1), cz1 = min(max(bz + 1, 0), sz - 1);
        const int sxy = sx * sy;
        const int r0 = cz0 * sxy + cy0 * sx, r1 = cz0 * sxy + cy1 * sx, r2 = cz1 * sxy + cy0 * sx,
                  r3 = cz1 * sxy + cy1 * sx;
        using E = typename std::remove_cv<typename std::remove_pointer<decltype(g)>::type>::type;
        const float c[8] = {Store<E>::ld(g, r0 + cx0), Store<E>::ld(g, r0 + cx1), Store<E>::ld(g, r1 + cx0),
                            Store<E>::ld(g, r1 + cx1), Store<E>::ld(g, r2 + cx0), Store<E>::ld(g, r2 + cx1),
                            Store<E>::ld(g, r3 + cx0), Store<E>::ld(g, r3 + cx1)};
        lo = c[0];
        hi = lo;
#pragma unroll
        for (int j = 1; j < 8; ++j) {
            lo = fminf(lo, c[j]);
            hi = fmaxf(hi, c[j]);
        }
    }
    template <bool MASK>
    __device__ __forceinline__ ClosedStencil closed(const uint8_t* solid, float qx, float qy, float qz,
                                                    bool fluid = false) const {
        return closed_stencil<MASK>(f.d, solid, qx, qy, qz, fluid);
    }
    template <bool MASK>
    __device__ __forceinline__ float apply(int k, const ClosedStencil& S) const {
        return apply_closed<typename std::remove_cv<typename std::remove_pointer<decltype(f.ptr(k))>::type>::type,
                            MASK>(S, f.ptr(k));
    }
};

// Closed scalar sampling (closed_sample.glsl) through a sampler: the stencil
// (clamped corners, fractions, fluid corners) is formed once per point and
// applied to each scalar field in apply_closed's order.
template <class Fields>
struct TileSampler;

template <class Fields>
struct TileSampler {
    GlobalSampler<Fields> G;
    tile::Window w;

    __device__ __forceinline__ float sample(int k, float qx, float qy, float qz) const {
        int sx, sy, sz;
        G.f.dims(k, sx, sy, sz);
        return tile::sample(w, k, G.f.ptr(k), sx, sy, sz, qx, qy, qz);
    }
    __device__ __forceinline__ float half(int k, int qx2, int qy2, int qz2) const {
        int sx, sy, sz;
        G.f.dims(k, sx, sy, sz);
        return tile::sample_half(w, k, G.f.ptr(k), sx, sy, sz, qx2, qy2, qz2);
    }
    template <int HX, int HY, int HZ>
    __device__ __forceinline__ float node(int k, int ix, int iy, int iz) const {
        return G.template node<HX, HY, HZ>(k, ix, iy, iz);
    }
    __device__ __forceinline__ void minmax8(int k, int bx, int by, int bz, float& lo, float& hi) const {
        // the window holds clamp(index) at every entry, so the clamped corners
        // of an unclamped lower corner are the entries at and after it
        if (!tile::inside(w, bx, by, bz)) {
            G.minmax8(k, bx, by, bz, lo, hi);
            return;
        }
        const tile::Corners c = tile::corners(w, k, bx, by, bz);
        lo = c.c0[0];
        hi = lo;
        const float v[7] = {c.c0[1], c.c0[tile::kPitch], c.c0[tile::kPitch + 1], c.c1[0], c.c1[1], c.c1[tile::kPitch],
                            c.c1[tile::kPitch + 1]};
#pragma unroll
        for (int j = 0; j < 7; ++j) {
            lo = fminf(lo, v[j]);
            hi = fmaxf(hi, v[j]);
        }
    }
    // The global stencil plus, when the lower corner (floor of the unclamped
    // point) lies in the window, the window offsets of its two slices: the
    // entries at and after that corner hold the clamped corners.
    struct Stencil {
        ClosedStencil S;
        int s0, s1;     // slice offset + in-slice offset of the lower corner (z0 and z1 slices); s0 < 0: global
    };
    template <bool MASK>
    __device__ __forceinline__ Stencil closed(const uint8_t* solid, float qx, float qy, float qz,
                                              bool fluid = false) const {
        Stencil t;
        t.S = closed_stencil<MASK>(G.f.d, solid, qx, qy, qz, fluid);
        const int ix = floor_int(qx), iy = floor_int(qy), iz = floor_int(qz);
        if (tile::inside(w, ix, iy, iz)) {
            const int off = (iy - w.wy) * tile::kPitch + (ix - w.wx);
            t.s0 = (iz & (tile::kRingSlices - 1)) * tile::kSlice + off;
            t.s1 = ((iz + 1) & (tile::kRingSlices - 1)) * tile::kSlice + off;
        } else {
            t.s0 = t.s1 = -1;
        }
        return t;
    }
    template <bool MASK>
    __device__ __forceinline__ float apply(int k, const Stencil& t) const {
        if (t.s0 < 0) return G.template apply<MASK>(k, t.S);
        const float* ring = w.s + k * tile::kRing;
        const float* c0 = ring + t.s0;
        const float* c1 = ring + t.s1;
        const ClosedStencil& S = t.S;
        // corner j: bit 0 = x1, bit 1 = y1, bit 2 = z1 (closed_stencil's order)
        auto corner = [&](int j) -> float {
            const float* r = (j & 4) ? c1 : c0;
            return r[((j & 2) ? tile::kPitch : 0) + (j & 1)];
        };
        if (MASK) {
            float value = 0.f;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (!(S.fluid & (1u << j))) continue;
                const float wz = (j & 4) ? S.fz : 1.f - S.fz, wy = (j & 2) ? S.fy : 1.f - S.fy,
                            wx = (j & 1) ? S.fx : 1.f - S.fx;
                value = value + wx * wy * wz * corner(j);
            }
            return S.total > 1e-8f ? value / S.total : 0.f;
        }
        const float f000 = corner(0), f100 = corner(1), f010 = corner(2), f110 = corner(3);
        const float f001 = corner(4), f101 = corner(5), f011 = corner(6), f111 = corner(7);
        const float fx = S.fx, fy = S.fy, fz = S.fz;
        const float gx = 1.f - fx, gy = 1.f - fy, gz = 1.f - fz;
        const float a0 = f000 * gx + f100 * fx, a1 = f010 * gx + f110 * fx;
        const float b0 = f001 * gx + f101 * fx, b1 = f011 * gx + f111 * fx;
        const float zz0 = a0 * gy + a1 * fy, zz1 = b0 * gy + b1 * fy;
        return zz0 * gz + zz1 * fz;
    }
};

// Staggered velocity at a physical point through a sampler (velocity_at).
template <bool P2, class S>
__device__ __forceinline__ F3 velocity_s(const Dev& d, const S& smp, F3 p) {
    const float qx = dv_e<P2>(d, p.x * d.nf[0], 0);
    const float qy = dv_e<P2>(d, p.y * d.nf[1], 1);
    const float qz = dv_e<P2>(d, p.z * d.nf[2], 2);
    F3 r;
    r.x = smp.sample(0, qx, qy - 0.5f, qz - 0.5f);
    r.y = smp.sample(1, qx - 0.5f, qy, qz - 0.5f);
    r.z = smp.sample(2, qx - 0.5f, qy - 0.5f, qz);
    return r;
}

// Velocity at the node p = (X2, Y2, Z2) / 2 cells (velocity_at_start).
template <bool P2, class S>
__device__ __forceinline__ F3 start_velocity_s(const Dev& d, const S& smp, F3 p, int X2, int Y2, int Z2) {
    if constexpr (P2) {
        F3 r;
        r.x = smp.half(0, X2, Y2 - 1, Z2 - 1);
        r.y = smp.half(1, X2 - 1, Y2, Z2 - 1);
        r.z = smp.half(2, X2 - 1, Y2 - 1, Z2);
        return r;
    } else {
        return velocity_s<false>(d, smp, p);
    }
}

// Velocity at the centre p of face (x, y, z) of face grid `axis`
// (start_velocity_s at its doubled coordinates). On power-of-two grids, for a
// face off the domain walls along its axis, no doubled coordinate is clamped
// and the parities of every component's node are fixed by the axis: the U face
// (2x, 2y+1, 2z+1) reads u at (x, y, z), v at (x-1..x, y..y+1, z) and w at
// (x-1..x, y, z..z+1), and likewise for V and W faces.
template <bool P2, class S>
__device__ __forceinline__ F3 start_velocity_face(const Dev& d, const S& smp, F3 p, int axis, int x, int y, int z) {
    if constexpr (P2) {
        const int c = axis == 0 ? x : (axis == 1 ? y : z);
        const int n = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
        if (c >= 1 && c <= n - 1) {
            if (axis == 0)
                return F3{smp.template node<0, 0, 0>(0, x, y, z), smp.template node<1, 1, 0>(1, x - 1, y, z),
                          smp.template node<1, 0, 1>(2, x - 1, y, z)};
            if (axis == 1)
                return F3{smp.template node<1, 1, 0>(0, x, y - 1, z), smp.template node<0, 0, 0>(1, x, y, z),
                          smp.template node<0, 1, 1>(2, x, y - 1, z)};
            return F3{smp.template node<1, 0, 1>(0, x, y, z - 1), smp.template node<0, 1, 1>(1, x, y, z - 1),
                      smp.template node<0, 0, 0>(2, x, y, z)};
        }
    }
    return start_velocity_s<P2>(d, smp, p, 2 * x + (axis != 0), 2 * y + (axis != 1), 2 * z + (axis != 2));
}

// Midpoint backtrace through a sampler (the `backtrace` of the transport
// passes); `cv`: the clearance of the start point's own cell (home_clearance).
template <bool MASK, bool P2, class S>
__device__ __forceinline__ F3 backtrace_s(const Dev& d, const S& smp, const uint8_t* solid, const uint8_t* halo, F3 p,
                                          F3 v0, float dt, int cv = 0) {
    const float s = 0.5f * dt;
    F3 mid = {p.x - s * v0.x, p.y - s * v0.y, p.z - s * v0.z};
    if (MASK) mid = clip_from<P2>(d, solid, halo, cv, p, mid);
    const F3 vm = velocity_s<P2>(d, smp, mid);
    F3 dep = {p.x - dt * vm.x, p.y - dt * vm.y, p.z - dt * vm.z};
    if (MASK) dep = clip_from<P2>(d, solid, halo, cv, p, dep);
    return dep;
}

}  // namespace ffx
