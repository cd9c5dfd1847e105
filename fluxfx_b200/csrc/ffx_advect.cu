// Transport kernels: MacCormack face predictor, fused velocity transport
// (+ emitters, buoyancy, walls), closed scalar transport and the final scalar
// pass, and the P0.2/P0.3 open-boundary forms.
//
// One thread per output sample. Face passes cover all three face grids in one
// launch (blockIdx.z enumerates axis and z; 32 x 8 threads over x and y).
// Gathers go through the read-only path; the 8-corner stencils of
// neighbouring threads overlap, so the L1/L2 hit rate is high and HBM traffic
// stays close to one read of each field per pass.
#include "ffx_host.cuh"
#include "ffx_batch.cuh"
#include "ffx_tile.cuh"

namespace ffx {
namespace {

constexpr int kThreads = 256;

// Minimum resident blocks per SM asked of the compiler for the transport
// kernels: the register budget against the warps resident to hide the
// gathers' latency, chosen by measurement at 256^3 (a build can override
// each with -DFFX_MINB_<KERNEL>=n; 0 leaves the choice to the compiler).
#ifndef FFX_MINB_PREDICTOR
#define FFX_MINB_PREDICTOR 8
#endif
#ifndef FFX_MINB_VELOCITY
#define FFX_MINB_VELOCITY 5
#endif
#ifndef FFX_MINB_SCALAR_PREDICTOR
#define FFX_MINB_SCALAR_PREDICTOR 0
#endif
#ifndef FFX_MINB_SCALARS
#define FFX_MINB_SCALARS 4
#endif
#if FFX_MINB_PREDICTOR > 0
#define FFX_LB_PREDICTOR __launch_bounds__(kThreads, FFX_MINB_PREDICTOR)
#else
#define FFX_LB_PREDICTOR __launch_bounds__(kThreads)
#endif
#if FFX_MINB_VELOCITY > 0
#define FFX_LB_VELOCITY __launch_bounds__(kThreads, FFX_MINB_VELOCITY)
#else
#define FFX_LB_VELOCITY __launch_bounds__(kThreads)
#endif
#if FFX_MINB_SCALAR_PREDICTOR > 0
#define FFX_LB_SCALAR_PREDICTOR __launch_bounds__(kThreads, FFX_MINB_SCALAR_PREDICTOR)
#else
#define FFX_LB_SCALAR_PREDICTOR __launch_bounds__(kThreads)
#endif
#if FFX_MINB_SCALARS > 0
#define FFX_LB_SCALARS __launch_bounds__(kThreads, FFX_MINB_SCALARS)
#else
#define FFX_LB_SCALARS __launch_bounds__(kThreads)
#endif

struct FaceIdx {
    int axis, x, y, z, sx, sy, sz;
    int i;
};

// Face of the thread (face_grid geometry): block z = axis*(nz+1) + z.
__device__ __forceinline__ bool face_coords(const Blk& b, const Dev& d, FaceIdx& f) {
    const int nz1 = d.nz + 1;
    const int zz = b.z;
    f.axis = zz >= 2 * nz1 ? 2 : (zz >= nz1 ? 1 : 0);
    f.z = zz - f.axis * nz1;
    f.sx = d.nx + (f.axis == 0);
    f.sy = d.ny + (f.axis == 1);
    f.sz = d.nz + (f.axis == 2);
    f.x = b.x * b.bw + b.ox;
    f.y = b.y * b.bh + b.oy;
    if (f.x >= f.sx || f.y >= f.sy || f.z >= f.sz) return false;
    f.i = f.x + f.sx * (f.y + f.sy * f.z);
    return true;
}

// Midpoint backtrace p -> departure (transport_face.glsl:8-17 and the same
// lines of every advection shader); clipped at colliders when MASK.
template <typename T, bool MASK, bool P2 = false>
__device__ __forceinline__ F3 backtrace(const Dev& d, const Faces<T>& F, const uint8_t* solid, const uint8_t* halo,
                                        F3 p, F3 v0,
                                        float dt) {
    float s = 0.5f * dt;
    F3 mid = {p.x - s * v0.x, p.y - s * v0.y, p.z - s * v0.z};
    if (MASK) mid = clip_solid_trace<P2>(d, solid, halo, p, mid);
    F3 vm = velocity_at<T, P2>(d, F, mid);
    F3 dep = {p.x - dt * vm.x, p.y - dt * vm.y, p.z - dt * vm.z};
    if (MASK) dep = clip_solid_trace<P2>(d, solid, halo, p, dep);
    return dep;
}

// Closed scalar sample (closed_sample.glsl:7-29).
template <typename T, bool MASK>
__device__ __forceinline__ float sample_closed(const Dev& d, const uint8_t* solid, const T* __restrict__ f,
                                               float qx, float qy, float qz) {
    float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    float fx = qx - bx, fy = qy - by, fz = qz - bz;
    int ix = floor_int(qx), iy = floor_int(qy), iz = floor_int(qz);
    int x0 = min(max(ix, 0), d.nx - 1), x1 = min(max(ix + 1, 0), d.nx - 1);
    int y0 = min(max(iy, 0), d.ny - 1), y1 = min(max(iy + 1, 0), d.ny - 1);
    int z0 = min(max(iz, 0), d.nz - 1), z1 = min(max(iz + 1, 0), d.nz - 1);
    if (MASK) {
        int xs[2] = {x0, x1}, ys[2] = {y0, y1}, zs[2] = {z0, z1};
        float value = 0.f, total = 0.f;
        for (int oz = 0; oz < 2; ++oz) {
            float wz = oz ? fz : 1.f - fz;
            for (int oy = 0; oy < 2; ++oy) {
                float wy = oy ? fy : 1.f - fy;
                for (int ox = 0; ox < 2; ++ox) {
                    float wx = ox ? fx : 1.f - fx;
                    int c = cidx(d, xs[ox], ys[oy], zs[oz]);
                    if (__ldg(solid + c)) continue;
                    float weight = wx * wy * wz;
                    value = value + weight * Store<T>::ld(f, c);
                    total = total + weight;
                }
            }
        }
        return total > 1e-8f ? value / total : 0.f;
    }
    float f000 = Store<T>::ld(f, cidx(d, x0, y0, z0)), f100 = Store<T>::ld(f, cidx(d, x1, y0, z0));
    float f010 = Store<T>::ld(f, cidx(d, x0, y1, z0)), f110 = Store<T>::ld(f, cidx(d, x1, y1, z0));
    float f001 = Store<T>::ld(f, cidx(d, x0, y0, z1)), f101 = Store<T>::ld(f, cidx(d, x1, y0, z1));
    float f011 = Store<T>::ld(f, cidx(d, x0, y1, z1)), f111 = Store<T>::ld(f, cidx(d, x1, y1, z1));
    float gx = 1.f - fx, gy = 1.f - fy, gz = 1.f - fz;
    float a0 = f000 * gx + f100 * fx, a1 = f010 * gx + f110 * fx;
    float b0 = f001 * gx + f101 * fx, b1 = f011 * gx + f111 * fx;
    float zz0 = a0 * gy + a1 * fy, zz1 = b0 * gy + b1 * fy;
    return zz0 * gz + zz1 * fz;
}

// The time step of a pass: the launch parameter, or the value a device-side
// time-step rule left at dtp (a step that never reads dt back to the host).
template <class Pm>
__device__ __forceinline__ float step_dt(const Pm& P) {
    return P.dtp ? P.dt_sign * __ldg(P.dtp) : P.dt;
}

// ------------------------------------------------------------ face predictor
template <typename T>
struct PredParams {
    Dev d;
    const uint8_t* solid;
    const uint8_t* halo;
    const uint8_t* clear;     // optional: ffx_clearance of the mask (collider tests skipped in clear cells)
    Faces<T> F;
    float dt;
    const float* dtp;     // optional: the time step read on the device (times dt_sign) instead of dt
    float dt_sign;
    T* out[3];
    float* dep[3];    // optional: departure points per face grid (three planes of nf floats), for reuse
    int nf[3];
};

// Face index of face (x, y, z) of face grid `axis`.
__device__ __forceinline__ FaceIdx face_at(const Dev& d, int axis, int x, int y, int z) {
    FaceIdx f;
    f.axis = axis;
    f.x = x;
    f.y = y;
    f.z = z;
    f.sx = d.nx + (axis == 0);
    f.sy = d.ny + (axis == 1);
    f.sz = d.nz + (axis == 2);
    f.i = x + f.sx * (y + f.sy * z);
    return f;
}

// Velocity faces as sampler fields 0..2 and the second face set (the
// predictor faces of the velocity pass) as fields 3..5.
template <typename T>
__device__ __forceinline__ GlobalSampler<FaceFields<T>> face_sampler(const Dev& d, const Faces<T>& F,
                                                                    const Faces<T>& second) {
    return GlobalSampler<FaceFields<T>>{FaceFields<T>{d, F, second}};
}

template <typename T, bool MASK, bool P2, class Smp>
__device__ __forceinline__ void face_predictor_face(const PredParams<T>& P, const FaceIdx& f, const Smp& smp) {
    const Dev& d = P.d;
    const uint8_t* __restrict__ solid = P.solid;
    const uint8_t* __restrict__ halo = P.halo;
    const float dt = step_dt(P);
    T* out = P.out[f.axis];
    // a clear cell and its lower neighbours are fluid: the face is open (but
    // for the lower grid wall next to a cell of clearance 2)
    const int cv = MASK ? home_clearance(P.clear, d, f.x, f.y, f.z) : 0;
    if (MASK && (cv == 0 ? solid_face(d, solid, f.x, f.y, f.z, f.axis)
                         : clear_face_blocked(cv, f.x, f.y, f.z, f.axis))) {
        Store<T>::st(out, f.i, 0.f);
        return;
    }
    float ox = f.axis == 0 ? 0.f : 0.5f, oy = f.axis == 1 ? 0.f : 0.5f, oz = f.axis == 2 ? 0.f : 0.5f;
    F3 p = {((float)f.x + ox) * d.h[0], ((float)f.y + oy) * d.h[1], ((float)f.z + oz) * d.h[2]};
    F3 v0 = start_velocity_face<P2>(d, smp, p, f.axis, f.x, f.y, f.z);
    F3 dep = backtrace_s<MASK, P2>(d, smp, solid, halo, p, v0, dt, cv);
    float value = smp.sample(f.axis, dv_h<P2>(d, dep.x, 0) - ox, dv_h<P2>(d, dep.y, 1) - oy,
                             dv_h<P2>(d, dep.z, 2) - oz);
    Store<T>::st(out, f.i, value);
    if (float* D = P.dep[f.axis]) {
        const int nf = P.nf[f.axis];
        D[f.i] = dep.x;
        D[f.i + nf] = dep.y;
        D[f.i + 2 * nf] = dep.z;
        // 16-bit storage rounds the stored predictor: its FP32 value, the
        // correction's semi-Lagrangian sample, goes to a fourth plane
        if (sizeof(T) == 2) D[f.i + 3 * nf] = value;
        // the start velocity, which the correction would form again at the same point
        constexpr int kV0 = sizeof(T) == 2 ? 4 : 3;
        D[f.i + kV0 * nf] = v0.x;
        D[f.i + (kV0 + 1) * nf] = v0.y;
        D[f.i + (kV0 + 2) * nf] = v0.z;
    }
}

template <typename T, bool MASK, bool P2>
__device__ __forceinline__ void face_predictor_body(const PredParams<T>& P, const Blk& b) {
    FaceIdx f;
    if (!face_coords(b, P.d, f)) return;
    face_predictor_face<T, MASK, P2>(P, f, face_sampler<T>(P.d, P.F, P.F));
}

template <typename T, bool MASK, bool P2>
__global__ void FFX_LB_PREDICTOR face_predictor_kernel(const __grid_constant__ PredParams<T> P) {
    face_predictor_body<T, MASK, P2>(P, hw_blk());
}

// ------------------------------------------------------- velocity transport
template <typename T>
struct VelParams {
    Dev d;
    const uint8_t* solid;
    const uint8_t* halo;
    const uint8_t* clear;   // optional: ffx_clearance of the mask
    Faces<T> F;       // velocity at the start of the step
    Faces<T> P;       // MacCormack predictor
    float dt, blend, lift, weight;
    const float* dtp;     // optional: the time step read on the device (times dt_sign) instead of dt
    float dt_sign;
    int corrected, apply_walls;
    const T* density;
    const T* temperature;
    T* out[3];
    Walls walls;      // wall velocities of the fused wall condition (moving colliders)
    const float* dep[3];   // optional: the predictor's departure points (reused on power-of-two grids,
    int nf[3];             // where both passes form the same start point)
    SrcDev src;
};

template <typename T, bool MASK, bool P2, class Smp>
__device__ __forceinline__ void advect_velocity_face(const VelParams<T>& P, const FaceIdx& f, const Smp& smp) {
    const Dev& d = P.d;
    const int axis = f.axis;
    if (P.apply_walls) {
        // a boundary face ends as its wall value whatever was advected into it
        // (the wall condition below), so its advection is skipped
        const int c = axis == 0 ? f.x : (axis == 1 ? f.y : f.z);
        const int n = axis == 0 ? f.sx : (axis == 1 ? f.sy : f.sz);
        if (c == 0 || c == n - 1) {
            Store<T>::st(P.out[axis], f.i, wall_value(P.walls, axis, f.i));
            return;
        }
    }
    const float dt = step_dt(P);
    const int cv = MASK ? home_clearance(P.clear, d, f.x, f.y, f.z) : 0;
    bool blocked = MASK && (cv == 0 ? solid_face(d, P.solid, f.x, f.y, f.z, axis)
                                    : clear_face_blocked(cv, f.x, f.y, f.z, axis));
    float value = 0.f;
    if (!blocked) {
        float off[3] = {axis == 0 ? 0.f : 0.5f, axis == 1 ? 0.f : 0.5f, axis == 2 ? 0.f : 0.5f};
        F3 p = {dv_n<P2>(d, ((float)f.x + off[0]) * d.e[0], 0), dv_n<P2>(d, ((float)f.y + off[1]) * d.e[1], 1),
                dv_n<P2>(d, ((float)f.z + off[2]) * d.e[2], 2)};
        // The host passes the predictor's traces only when both passes form the
        // same start point at every face (face_starts_match); the predictor then
        // traced this face's start point with the same velocity, so its start
        // velocity, its departure point, and in FP32 storage its sample, are this
        // pass's.
        const bool reuse = P.corrected && P.dep[axis] != nullptr;
        F3 v0, dep;
        if (reuse) {
            const float* D = P.dep[axis];
            const int nf = P.nf[axis];
            constexpr int kV0 = sizeof(T) == 2 ? 4 : 3;
            dep = {__ldg(D + f.i), __ldg(D + f.i + nf), __ldg(D + f.i + 2 * nf)};
            v0 = {__ldg(D + f.i + kV0 * nf), __ldg(D + f.i + (kV0 + 1) * nf), __ldg(D + f.i + (kV0 + 2) * nf)};
        } else {
            v0 = start_velocity_face<P2>(d, smp, p, axis, f.x, f.y, f.z);
            dep = backtrace_s<MASK, P2>(d, smp, P.solid, P.halo, p, v0, dt, cv);
        }
        const T* orig = axis == 0 ? P.F.u : (axis == 1 ? P.F.v : P.F.w);
        const T* pred = axis == 0 ? P.P.u : (axis == 1 ? P.P.v : P.P.w);
        float qx = dv_h<P2>(d, dep.x, 0) - off[0], qy = dv_h<P2>(d, dep.y, 1) - off[1],
              qz = dv_h<P2>(d, dep.z, 2) - off[2];
        // the predictor's sample at the same departure point: the stored value
        // (FP32) or its unrounded copy in the fourth trace plane (BF16)
        float low = !reuse ? smp.sample(axis, qx, qy, qz)
                           : (sizeof(T) == 4 ? Store<T>::ld(pred, f.i) : __ldg(P.dep[axis] + f.i + 3 * P.nf[axis]));
        value = low;
        if (P.corrected) {
            // correct_velocity_fused.glsl:5-27
            float size[3] = {(float)(f.sx - 1), (float)(f.sy - 1), (float)(f.sz - 1)};
            float lob[3], hib[3];
            for (int k = 0; k < 3; ++k) {
                lob[k] = off[k] * d.h[k];
                hib[k] = (size[k] + off[k]) * d.h[k];
            }
            float s = 0.5f * dt;
            F3 mid2 = {p.x + s * v0.x, p.y + s * v0.y, p.z + s * v0.z};
            F3 vm2 = velocity_s<P2>(d, smp, mid2);
            F3 arr = {p.x + dt * vm2.x, p.y + dt * vm2.y, p.z + dt * vm2.z};
            bool ok = !(dep.x < lob[0] || dep.y < lob[1] || dep.z < lob[2] || dep.x > hib[0] || dep.y > hib[1] ||
                        dep.z > hib[2] || arr.x < lob[0] || arr.y < lob[1] || arr.z < lob[2] || arr.x > hib[0] ||
                        arr.y > hib[1] || arr.z > hib[2]);
            if (MASK && ok) ok = safe_correction_from<P2>(d, P.solid, P.halo, cv, p, dep, mid2, arr);
            if (ok) {
                float pa = smp.sample(3 + axis, dv_h<P2>(d, arr.x, 0) - off[0], dv_h<P2>(d, arr.y, 1) - off[1],
                                      dv_h<P2>(d, arr.z, 2) - off[2]);
                float val = Store<T>::ld(pred, f.i) + 0.5f * (Store<T>::ld(orig, f.i) - pa);
                // min / max of the 8 corners around the departure point, clamped to the grid
                float lo, hi;
                smp.minmax8(axis, (int)floorf(qx), (int)floorf(qy), (int)floorf(qz), lo, hi);
                float cl = fminf(fmaxf(val, lo), hi);
                value = low * (1.f - P.blend) + cl * P.blend;
            }
        }
        const SrcDev& S = P.src;
        if (S.count < 0) {
            float w = single_weight(S, p);
            if (w != 0.f) {
                float bl = 1.f - expf(-S.coupling * dt * w);
                value = value * (1.f - bl) + comp(S.jet, axis) * bl;
            } else {
                // expf(+-0) = 1, so bl = 0 and the blend is value * 1 + jet * 0
                value = value + comp(S.jet, axis) * 0.f;
            }
        } else if (S.count > 0 && !outside(S.any, p)) {
            // (outside every row's reach all weights are +0: total stays +-0
            // and the blend below is not taken, so the value is unchanged)
            float total = 0.f, target = 0.f;
            for (int i = 0; i < S.count; ++i) {
                float rate = S.table[16 * i + 7] * table_weight(S, i, p);
                total = total + rate;
                target = target + rate * S.table[16 * i + 8 + axis];
            }
            if (total > 0.f) {
                float bl = 1.f - expf(-dt * total);
                value = value * (1.f - bl) + (target / total) * bl;
            }
        }
    }
    if (axis == 2 && P.density) {
        // buoyancy.glsl:1-14 with the previous step's scalars
        int below = min(max(f.z - 1, 0), d.nz - 1), above = min(max(f.z, 0), d.nz - 1);
        int ib = cidx(d, f.x, f.y, below), ia = cidx(d, f.x, f.y, above);
        float rho = 0.5f * (Store<T>::ld(P.density, ib) + Store<T>::ld(P.density, ia));
        float theta = 0.5f * (Store<T>::ld(P.temperature, ib) + Store<T>::ld(P.temperature, ia));
        float a = P.lift * theta - P.weight * rho;
        value = value + dt * a;
    }
    if (P.apply_walls) {
        int c = axis == 0 ? f.x : (axis == 1 ? f.y : f.z);
        int n = axis == 0 ? f.sx : (axis == 1 ? f.sy : f.sz);
        if (c == 0 || c == n - 1 || blocked) value = wall_value(P.walls, axis, f.i);
    }
    Store<T>::st(P.out[axis], f.i, value);
}

template <typename T, bool MASK, bool P2>
__device__ __forceinline__ void advect_velocity_body(const VelParams<T>& P, const Blk& b) {
    FaceIdx f;
    if (!face_coords(b, P.d, f)) return;
    advect_velocity_face<T, MASK, P2>(P, f, face_sampler<T>(P.d, P.F, P.P));
}

template <typename T, bool MASK, bool P2>
__global__ void FFX_LB_VELOCITY advect_velocity_kernel(const __grid_constant__ VelParams<T> P) {
    advect_velocity_body<T, MASK, P2>(P, hw_blk());
}

// ------------------------------------------------- tiled face passes
// The face predictor and the velocity pass over shared-memory windows
// (ffx_tile.cuh): a block owns 32 x 8 (x, y) columns and a chunk of z slices;
// at slice z a thread works the U face (x, y, z), the V face and the W face
// of its column (the thread at x = nx - 1 also the U face x = nx, the thread
// at y = ny - 1 also the V face y = ny; the last chunk adds z = nz for the W
// faces). Results are bit-identical to the untiled kernels.
#ifndef FFX_MINB_PREDICTOR_TILED
#define FFX_MINB_PREDICTOR_TILED 6
#endif
#ifndef FFX_MINB_VELOCITY_TILED
#define FFX_MINB_VELOCITY_TILED 5
#endif
#ifndef FFX_TILE_ZCHUNK
#define FFX_TILE_ZCHUNK 16
#endif

// Slices [z0, z_end) of the block's chunk: the last chunk of a face pass
// includes z = nz (W faces only).
struct Chunk {
    int z0, z1;
};
__device__ __forceinline__ Chunk face_chunk(int nz, int zchunk) {
    const int z0 = blockIdx.z * zchunk;
    return Chunk{z0, z0 + zchunk >= nz ? nz + 1 : z0 + zchunk};
}

// The faces of column (x, y) at slice z, in U, V, W order: up to five (U at x
// and x + 1 = nx, V at y and y + 1 = ny, W), visited from one call site so
// the face body is inlined once.
template <class Face>
__device__ __forceinline__ void column_faces(const Dev& d, int x, int y, int z, Face&& face) {
    const bool in = x < d.nx && y < d.ny;
#pragma unroll 1
    for (int j = 0; j < 5; ++j) {
        int axis, fx = x, fy = y;
        bool active;
        switch (j) {
            case 0: axis = 0; active = in && z < d.nz; break;
            case 1: axis = 0; fx = d.nx; active = x == d.nx - 1 && y < d.ny && z < d.nz; break;
            case 2: axis = 1; active = in && z < d.nz; break;
            case 3: axis = 1; fy = d.ny; active = y == d.ny - 1 && x < d.nx && z < d.nz; break;
            default: axis = 2; active = in; break;
        }
        if (active) face(axis, fx, fy, z);
    }
}

// Marches the block's chunk: stages the first `nfields` sampler fields slice
// by slice (z-1 .. z+2 resident while slice z is worked) and calls work(z)
// per slice.
template <int NF, class Fields, class Work>
__device__ __forceinline__ void march(TileSampler<Fields>& smp, float* ring, int nfields, Chunk c, Work&& work) {
    const int tid = threadIdx.x + tile::kTX * threadIdx.y;
    auto stage_all = [&](int zg) {
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            if (k >= nfields) break;
            int sx, sy, sz;
            smp.G.f.dims(k, sx, sy, sz);
            tile::stage(ring + k * tile::kRing, smp.G.f.ptr(k), sx, sy, sz, smp.w.wx, smp.w.wy, zg, tid);
        }
    };
    stage_all(c.z0 - 1);
    stage_all(c.z0);
    stage_all(c.z0 + 1);
#pragma unroll 1
    for (int z = c.z0; z < c.z1; ++z) {
        stage_all(z + 2);
        __syncthreads();
        smp.w.zlo = z - 1;
        work(z);
        __syncthreads();
    }
}

template <class Fields>
__device__ __forceinline__ TileSampler<Fields> tile_sampler(const GlobalSampler<Fields>& g, float* ring) {
    return TileSampler<Fields>{g, tile::Window{ring, (int)blockIdx.x * tile::kTX - 1, (int)blockIdx.y * tile::kTY - 1, 0}};
}

template <typename T, bool MASK, bool P2>
__global__ void __launch_bounds__(tile::kThreads, FFX_MINB_PREDICTOR_TILED)
    face_predictor_tiled_kernel(const __grid_constant__ PredParams<T> P, int zchunk) {
    __shared__ float ring[3 * tile::kRing];
    auto smp = tile_sampler(face_sampler<T>(P.d, P.F, P.F), ring);
    const int x = (int)blockIdx.x * tile::kTX + (int)threadIdx.x, y = (int)blockIdx.y * tile::kTY + (int)threadIdx.y;
    march<3>(smp, ring, 3, face_chunk(P.d.nz, zchunk), [&](int z) {
        column_faces(P.d, x, y, z, [&](int axis, int fx, int fy, int fz) {
            face_predictor_face<T, MASK, P2>(P, face_at(P.d, axis, fx, fy, fz), smp);
        });
    });
}

template <typename T, bool MASK, bool P2>
__global__ void __launch_bounds__(tile::kThreads, FFX_MINB_VELOCITY_TILED)
    advect_velocity_tiled_kernel(const __grid_constant__ VelParams<T> P, int zchunk) {
    __shared__ float ring[6 * tile::kRing];
    auto smp = tile_sampler(face_sampler<T>(P.d, P.F, P.P), ring);
    const int x = (int)blockIdx.x * tile::kTX + (int)threadIdx.x, y = (int)blockIdx.y * tile::kTY + (int)threadIdx.y;
    // the predictor faces are read only by the MacCormack correction
    march<6>(smp, ring, P.corrected ? 6 : 3, face_chunk(P.d.nz, zchunk), [&](int z) {
        column_faces(P.d, x, y, z, [&](int axis, int fx, int fy, int fz) {
            advect_velocity_face<T, MASK, P2>(P, face_at(P.d, axis, fx, fy, fz), smp);
        });
    });
}

dim3 tiled_grid(int nx, int ny, int nz, int zchunk) {
    return dim3((unsigned)((nx + tile::kTX - 1) / tile::kTX), (unsigned)((ny + tile::kTY - 1) / tile::kTY),
                (unsigned)((nz + zchunk - 1) / zchunk));
}

// Whether the transport passes run tiled (ffx_set_transport_tiling). Off by
// default: on the 256^3 collider scene the tiled forms measured slower than the
// gathers (face predictor 1.98 vs 1.68 ms, velocity 2.98 vs 2.44, scalar
// predictor + reverse 2.21 vs 1.30, scalar final 1.51 vs 1.01): the passes are
// bound by instruction issue, and staging adds instructions and a block
// barrier per slice without removing arithmetic.
int g_tiling = 0;

// P0.3 plain face self-advection (mac_advect_velocity.glsl).
template <typename T>
__global__ void __launch_bounds__(kThreads) mac_advect_velocity_kernel(Dev d, Faces<T> F, float dt, T* ou, T* ov,
                                                                       T* ow) {
    FaceIdx f;
    if (!face_coords(hw_blk(), d, f)) return;
    float ox = f.axis == 0 ? 0.f : 0.5f, oy = f.axis == 1 ? 0.f : 0.5f, oz = f.axis == 2 ? 0.f : 0.5f;
    F3 p = {((float)f.x + ox) * d.e[0] / d.nf[0], ((float)f.y + oy) * d.e[1] / d.nf[1],
            ((float)f.z + oz) * d.e[2] / d.nf[2]};
    F3 v0 = velocity_at(d, F, p);
    F3 dep = backtrace<T, false>(d, F, nullptr, nullptr, p, v0, dt);
    F3 v = velocity_at(d, F, dep);
    T* out = f.axis == 0 ? ou : (f.axis == 1 ? ov : ow);
    Store<T>::st(out, f.i, comp(v, f.axis));
}

template <typename T>
__global__ void buoyancy_kernel(Dev d, const T* w_in, const T* density, const T* temperature, float dt, float lift,
                                float weight, T* w_out) {
    int x, y, z;
    if (!cell_coords(d.nx, d.ny, x, y, z)) return;
    const int i = cidx(d, x, y, z);
    int below = min(max(z - 1, 0), d.nz - 1), above = min(max(z, 0), d.nz - 1);
    int ib = cidx(d, x, y, below), ia = cidx(d, x, y, above);
    float rho = 0.5f * (Store<T>::ld(density, ib) + Store<T>::ld(density, ia));
    float theta = 0.5f * (Store<T>::ld(temperature, ib) + Store<T>::ld(temperature, ia));
    float a = lift * theta - weight * rho;
    Store<T>::st(w_out, i, Store<T>::ld(w_in, i) + dt * a);
}

// ------------------------------------------------------------- scalar passes
template <typename T>
struct ScalarXport {
    Dev d;
    const uint8_t* solid;
    const uint8_t* halo;
    const uint8_t* clear;   // optional: ffx_clearance of the mask
    Faces<T> F;
    float dt;
    const float* dtp;     // optional: the time step read on the device (times dt_sign) instead of dt
    float dt_sign;
    int count;
    const T* in[3];
    T* out[3];
    float* dep;       // optional: departure points (three planes of n floats) for the final pass
    int n;
    // optional, on the reverse pass: the forward pass's departure points (read)
    // and the final pass's correction decision per cell (written)
    const float* fdep;
    uint8_t* ok;
};

// correct_scalar.glsl:1-21's conditions for the MacCormack correction of a
// cell: departure and arrival points at least half a cell inside the domain
// and, with colliders, safe_solid_correction at start, departure, midpoint and
// arrival.
template <bool MASK, bool P2>
__device__ __forceinline__ bool scalar_correction_ok(const Dev& d, const uint8_t* solid, const uint8_t* halo,
                                                     int cv, F3 p, F3 dep, F3 mid2, F3 arr) {
    const float lb[3] = {0.5f * d.h[0], 0.5f * d.h[1], 0.5f * d.h[2]};
    const float hb[3] = {d.e[0] - 0.5f * d.h[0], d.e[1] - 0.5f * d.h[1], d.e[2] - 0.5f * d.h[2]};
    bool ok = !(dep.x < lb[0] || dep.y < lb[1] || dep.z < lb[2] || dep.x > hb[0] || dep.y > hb[1] ||
                dep.z > hb[2] || arr.x < lb[0] || arr.y < lb[1] || arr.z < lb[2] || arr.x > hb[0] ||
                arr.y > hb[1] || arr.z > hb[2]);
    if (MASK && ok) ok = safe_correction_from<P2>(d, solid, halo, cv, p, dep, mid2, arr);
    return ok;
}

__device__ __forceinline__ bool same_bits(F3 a, F3 b) {
    return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
           __float_as_uint(a.z) == __float_as_uint(b.z);
}

// Velocity faces as sampler fields 0..2, the scalar fields C[0..2] as 3..5.
template <typename T>
__device__ __forceinline__ GlobalSampler<CellFields<T>> cell_sampler(const Dev& d, const Faces<T>& F,
                                                                    const T* const* C) {
    return GlobalSampler<CellFields<T>>{CellFields<T>{d, F, C}};
}

// DECIDE: the reverse pass that also writes P.ok (its own instantiation, so
// the other passes keep their registers).
template <typename T, bool MASK, bool P2, class Smp, bool DECIDE = false>
__device__ __forceinline__ void scalar_transport_cell(const ScalarXport<T>& P, int x, int y, int z, const Smp& smp) {
    const Dev& d = P.d;
    const int i = cidx(d, x, y, z);
    const int cv = MASK ? home_clearance(P.clear, d, x, y, z) : 0;
    const bool clear = cv != 0;
    if (MASK && !clear && __ldg(P.solid + i)) {
        for (int c = 0; c < P.count; ++c) Store<T>::st(P.out[c], i, 0.f);
        return;
    }
    F3 p = {((float)x + 0.5f) * d.h[0], ((float)y + 0.5f) * d.h[1], ((float)z + 0.5f) * d.h[2]};
    F3 v0 = start_velocity_s<P2>(d, smp, p, 2 * x + 1, 2 * y + 1, 2 * z + 1);
    F3 dep;
    if (DECIDE) {
        // backtrace_s, keeping the unclipped midpoint and departure point: with
        // the reverse step -dt they are the final pass's forward midpoint
        // p + (dt/2) v0 and, where the midpoint was not clipped, its arrival
        // point p + dt v(mid) (x - (-a) b == x + a b exactly), so the final
        // pass's correction test is decided here
        const float dtr = step_dt(P), s = 0.5f * dtr;
        const F3 mid = {p.x - s * v0.x, p.y - s * v0.y, p.z - s * v0.z};
        const F3 midc = MASK ? clip_from<P2>(d, P.solid, P.halo, cv, p, mid) : mid;
        const F3 vm = velocity_s<P2>(d, smp, midc);
        F3 arr = {p.x - dtr * vm.x, p.y - dtr * vm.y, p.z - dtr * vm.z};
        dep = MASK ? clip_from<P2>(d, P.solid, P.halo, cv, p, arr) : arr;
        if (!same_bits(midc, mid)) {
            const F3 vm2 = velocity_s<P2>(d, smp, mid);
            arr = {p.x - dtr * vm2.x, p.y - dtr * vm2.y, p.z - dtr * vm2.z};
        }
        const F3 fdep = {__ldg(P.fdep + i), __ldg(P.fdep + i + P.n), __ldg(P.fdep + i + 2 * P.n)};
        P.ok[i] = scalar_correction_ok<MASK, P2>(d, P.solid, P.halo, cv, p, fdep, mid, arr) ? 1 : 0;
    } else {
        dep = backtrace_s<MASK, P2>(d, smp, P.solid, P.halo, p, v0, step_dt(P), cv);
    }
    float qx = dv_h<P2>(d, dep.x, 0) - 0.5f, qy = dv_h<P2>(d, dep.y, 1) - 0.5f,
          qz = dv_h<P2>(d, dep.z, 2) - 0.5f;
    const auto S = smp.template closed<MASK>(P.solid, qx, qy, qz, clear && near_start(d, p, dep));
    for (int c = 0; c < P.count; ++c) Store<T>::st(P.out[c], i, smp.template apply<MASK>(3 + c, S));
    if (P.dep) {
        P.dep[i] = dep.x;
        P.dep[i + P.n] = dep.y;
        P.dep[i + 2 * P.n] = dep.z;
    }
}

template <typename T, bool MASK, bool P2, bool DECIDE = false>
__device__ __forceinline__ void scalar_transport_body(const ScalarXport<T>& P, const Blk& b) {
    int x, y, z;
    if (!cell_coords(b, P.d.nx, P.d.ny, x, y, z)) return;
    using S = GlobalSampler<CellFields<T>>;
    scalar_transport_cell<T, MASK, P2, S, DECIDE>(P, x, y, z, cell_sampler<T>(P.d, P.F, P.in));
}

template <typename T, bool MASK, bool P2>
__global__ void FFX_LB_SCALAR_PREDICTOR scalar_transport_kernel(const __grid_constant__ ScalarXport<T> P) {
    scalar_transport_body<T, MASK, P2>(P, hw_blk());
}

#ifndef FFX_MINB_SCALAR_REVERSE
#define FFX_MINB_SCALAR_REVERSE 5
#endif
#if FFX_MINB_SCALAR_REVERSE > 0
#define FFX_LB_SCALAR_REVERSE __launch_bounds__(kThreads, FFX_MINB_SCALAR_REVERSE)
#else
#define FFX_LB_SCALAR_REVERSE __launch_bounds__(kThreads)
#endif

template <typename T, bool MASK, bool P2>
__global__ void FFX_LB_SCALAR_REVERSE scalar_reverse_ok_kernel(const __grid_constant__ ScalarXport<T> P) {
    scalar_transport_body<T, MASK, P2, true>(P, hw_blk());
}

template <typename T>
struct Channel {
    const T* field;
    const T* pred;
    const T* rev;
    T* out;
    float rate, decay, target;
    int channel, table_target;
};

template <typename T>
struct ScalarFinal {
    Dev d;
    const uint8_t* solid;
    const uint8_t* halo;
    const uint8_t* clear;   // optional: ffx_clearance of the mask
    Faces<T> F;
    float dt;
    const float* dtp;     // optional: the time step read on the device (times dt_sign) instead of dt
    float dt_sign;
    int corrected, count;
    Channel<T> ch[3];
    const T* fields[3];   // ch[c].field, as the sampler's scalar fields
    float* maxima;
    const float* dep;   // optional: the forward predictor's departure points (same start point, reused)
    int n;
    const uint8_t* ok;  // optional, with dep: the correction decisions of the reverse pass
    SrcDev src;
};

// One cell of the final scalar pass; vmax[c] is raised to |result of channel c|.
template <typename T, bool MASK, bool P2, class Smp>
__device__ __forceinline__ void advect_scalars_cell(const ScalarFinal<T>& P, int x, int y, int z, const Smp& smp,
                                                    float vmax[3]) {
    const Dev& d = P.d;
    const int i = cidx(d, x, y, z);
    const int cv = MASK ? home_clearance(P.clear, d, x, y, z) : 0;
    const bool clear = cv != 0;
    if (MASK && !clear && __ldg(P.solid + i)) {
        for (int c = 0; c < P.count; ++c) Store<T>::st(P.ch[c].out, i, 0.f);
        return;
    }
    const float dt = step_dt(P);
    F3 p = {((float)x + 0.5f) * d.h[0], ((float)y + 0.5f) * d.h[1], ((float)z + 0.5f) * d.h[2]};
    // the forward predictor traced this cell's start point with the same
    // velocity: its departure point, and in FP32 storage its samples, are this pass's
    const bool reuse = P.corrected && P.dep != nullptr;
    // the reverse pass decided the correction (scalar_transport_cell with ok)
    const bool decided = reuse && P.ok != nullptr;
    F3 v0 = {0.f, 0.f, 0.f};
    if (!decided) v0 = start_velocity_s<P2>(d, smp, p, 2 * x + 1, 2 * y + 1, 2 * z + 1);
    F3 dep;
    if (reuse) dep = {__ldg(P.dep + i), __ldg(P.dep + i + P.n), __ldg(P.dep + i + 2 * P.n)};
    else dep = backtrace_s<MASK, P2>(d, smp, P.solid, P.halo, p, v0, dt, cv);
    float qx = dv_h<P2>(d, dep.x, 0) - 0.5f, qy = dv_h<P2>(d, dep.y, 1) - 0.5f,
          qz = dv_h<P2>(d, dep.z, 2) - 0.5f;
    bool ok = false;
    if (decided) {
        ok = __ldg(P.ok + i) != 0;
    } else if (P.corrected) {
        // correct_scalar.glsl:1-21
        float s = 0.5f * dt;
        F3 mid2 = {p.x + s * v0.x, p.y + s * v0.y, p.z + s * v0.z};
        F3 vm2 = velocity_s<P2>(d, smp, mid2);
        F3 arr = {p.x + dt * vm2.x, p.y + dt * vm2.y, p.z + dt * vm2.z};
        ok = scalar_correction_ok<MASK, P2>(d, P.solid, P.halo, cv, p, dep, mid2, arr);
    }
    // lower corner of the departure cell (the clamp bounds: its 8 corners clamped to the grid)
    const int bx = ok ? (int)floorf(qx) : 0, by = ok ? (int)floorf(qy) : 0, bz = ok ? (int)floorf(qz) : 0;
    const SrcDev& S = P.src;
    // the semi-Lagrangian sample (the stored predictor value when it is the same)
    const bool stored = reuse && sizeof(T) == 4;
    const bool none = S.count > 0 && outside(S.any, p);
    // (where the correction applies it replaces the semi-Lagrangian value, which
    // is then not formed)
    decltype(smp.template closed<MASK>(P.solid, qx, qy, qz)) St;
    if (!stored && !ok) St = smp.template closed<MASK>(P.solid, qx, qy, qz, clear && near_start(d, p, dep));
    // at most three channels, unrolled: per-channel state stays in registers
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (c >= P.count) break;
        const Channel<T>& C = P.ch[c];
        float value;
        if (ok) {
            float val = Store<T>::ld(C.pred, i) + 0.5f * (Store<T>::ld(C.field, i) - Store<T>::ld(C.rev, i));
            float lo, hi;
            smp.minmax8(3 + c, bx, by, bz, lo, hi);
            value = fminf(fmaxf(val, lo), hi);
        } else {
            value = stored ? Store<T>::ld(C.pred, i) : smp.template apply<MASK>(3 + c, St);
        }
        // expf(-0) = 1 and v * 1 = v: no decay leaves the value as it is
        if (C.decay != 0.f) value = value * expf(-C.decay * dt);
        if (S.count < 0) {
            float w = single_weight(S, p);
            value = C.target >= 0.f ? fmaxf(value, C.target * w) : value + dt * C.rate * w;
        } else {
            float tgt = 0.f;
            for (int k = 0; k < S.count; ++k) {
                const float* row = S.table + 16 * k;
                float r = C.channel == 0 ? row[11] : (C.channel == 1 ? row[12] : row[15]);
                // table_weight is +0 outside every row's reach
                float w = none ? 0.f : table_weight(S, k, p);
                bool is_target = (C.channel == 0 && row[13] > 0.5f) || (C.channel == 1 && C.table_target);
                if (is_target) tgt = fmaxf(tgt, r * w);
                else value = value + dt * r * w;
            }
            if (C.channel == 0 || (C.channel == 1 && C.table_target)) value = fmaxf(value, tgt);
        }
        Store<T>::st(C.out, i, value);
        vmax[c] = fmaxf(vmax[c], finite_abs(value));
    }
}

template <typename T, bool MASK, bool P2>
__device__ __forceinline__ void advect_scalars_body(const ScalarFinal<T>& P, const Blk& b) {
    const Dev& d = P.d;
    int x, y, z;
    float vmax[3] = {0.f, 0.f, 0.f};
    if (cell_coords(b, d.nx, d.ny, x, y, z))
        advect_scalars_cell<T, MASK, P2>(P, x, y, z, cell_sampler<T>(d, P.F, P.fields), vmax);
    if (P.maxima) {
        block_max_to_n<3>(P.maxima, vmax, P.count);
        __syncthreads();
    }
}

template <typename T, bool MASK, bool P2>
__global__ void FFX_LB_SCALARS advect_scalars_kernel(const __grid_constant__ ScalarFinal<T> P) {
    advect_scalars_body<T, MASK, P2>(P, hw_blk());
}

// ------------------------------------------------ tiled scalar passes
// The scalar predictor/reverse and final passes over shared-memory windows of
// the velocity faces and the transported scalars (ffx_tile.cuh); a thread
// works the cell (x, y, z) of its column at each slice of the block's chunk.
#ifndef FFX_MINB_SCALAR_PREDICTOR_TILED
#define FFX_MINB_SCALAR_PREDICTOR_TILED 4
#endif
#ifndef FFX_MINB_SCALARS_TILED
#define FFX_MINB_SCALARS_TILED 4
#endif

__device__ __forceinline__ Chunk cell_chunk(int nz, int zchunk) {
    const int z0 = blockIdx.z * zchunk;
    return Chunk{z0, min(z0 + zchunk, nz)};
}

template <typename T, bool MASK, bool P2>
__global__ void __launch_bounds__(tile::kThreads, FFX_MINB_SCALAR_PREDICTOR_TILED)
    scalar_transport_tiled_kernel(const __grid_constant__ ScalarXport<T> P, int zchunk) {
    __shared__ float ring[6 * tile::kRing];
    auto smp = tile_sampler(cell_sampler<T>(P.d, P.F, P.in), ring);
    const int x = (int)blockIdx.x * tile::kTX + (int)threadIdx.x, y = (int)blockIdx.y * tile::kTY + (int)threadIdx.y;
    const bool in = x < P.d.nx && y < P.d.ny;
    using S = decltype(smp);
    march<6>(smp, ring, 3 + P.count, cell_chunk(P.d.nz, zchunk), [&](int z) {
        if (!in) return;
        if (P.ok) scalar_transport_cell<T, MASK, P2, S, true>(P, x, y, z, smp);
        else scalar_transport_cell<T, MASK, P2, S, false>(P, x, y, z, smp);
    });
}

template <typename T, bool MASK, bool P2>
__global__ void __launch_bounds__(tile::kThreads, FFX_MINB_SCALARS_TILED)
    advect_scalars_tiled_kernel(const __grid_constant__ ScalarFinal<T> P, int zchunk) {
    __shared__ float ring[6 * tile::kRing];
    auto smp = tile_sampler(cell_sampler<T>(P.d, P.F, P.fields), ring);
    const int x = (int)blockIdx.x * tile::kTX + (int)threadIdx.x, y = (int)blockIdx.y * tile::kTY + (int)threadIdx.y;
    const bool in = x < P.d.nx && y < P.d.ny;
    float vmax[3] = {0.f, 0.f, 0.f};
    march<6>(smp, ring, 3 + P.count, cell_chunk(P.d.nz, zchunk), [&](int z) {
        if (in) advect_scalars_cell<T, MASK, P2>(P, x, y, z, smp, vmax);
    });
    if (P.maxima) {
        block_max_to_n<3>(P.maxima, vmax, P.count);
        __syncthreads();
    }
}

// P0.2 open-boundary transport in an analytic flow (advect.glsl).
__device__ __forceinline__ F3 analytic_velocity(const Dev& d, F3 p, F3 base, float w) {
    float qx = p.x - 0.5f * d.e[0], qy = p.y - 0.5f * d.e[1];
    F3 r = {base.x + (-w * qy), base.y + w * qx, base.z};
    return r;
}

template <typename T>
__device__ __forceinline__ float sample_zero(const Dev& d, const T* __restrict__ f, float qx, float qy, float qz) {
    float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    float fx = qx - bx, fy = qy - by, fz = qz - bz;
    int ix = floor_int(qx), iy = floor_int(qy), iz = floor_int(qz);
    auto fz_ = [&](int ox, int oy, int oz) -> float {
        int x = ix + ox, y = iy + oy, z = iz + oz;
        if (x < 0 || y < 0 || z < 0 || x >= d.nx || y >= d.ny || z >= d.nz) return 0.f;
        return Store<T>::ld(f, cidx(d, x, y, z));
    };
    float gx = 1.f - fx, gy = 1.f - fy, gz = 1.f - fz;
    float a0 = fz_(0, 0, 0) * gx + fz_(1, 0, 0) * fx, a1 = fz_(0, 1, 0) * gx + fz_(1, 1, 0) * fx;
    float b0 = fz_(0, 0, 1) * gx + fz_(1, 0, 1) * fx, b1 = fz_(0, 1, 1) * gx + fz_(1, 1, 1) * fx;
    float z0 = a0 * gy + a1 * fy, z1 = b0 * gy + b1 * fy;
    return z0 * gz + z1 * fz;
}

struct OpenParams {
    Dev d;
    float dt, angular, radius, rate, decay;
    F3 base, center;
};

template <typename T>
__global__ void advect_open_kernel(OpenParams P, const T* in, T* out) {
    const Dev& d = P.d;
    int x, y, z;
    if (!cell_coords(d.nx, d.ny, x, y, z)) return;
    const int i = cidx(d, x, y, z);
    F3 p = {((float)x + 0.5f) * d.h[0], ((float)y + 0.5f) * d.h[1], ((float)z + 0.5f) * d.h[2]};
    F3 v = analytic_velocity(d, p, P.base, P.angular);
    float s = 0.5f * P.dt;
    F3 mid = {p.x - s * v.x, p.y - s * v.y, p.z - s * v.z};
    F3 vm = analytic_velocity(d, mid, P.base, P.angular);
    F3 dep = {p.x - P.dt * vm.x, p.y - P.dt * vm.y, p.z - P.dt * vm.z};
    float value = sample_zero(d, in, dep.x / d.h[0] - 0.5f, dep.y / d.h[1] - 0.5f, dep.z / d.h[2] - 0.5f) *
                  expf(-P.decay * P.dt);
    F3 off = {p.x - P.center.x, p.y - P.center.y, p.z - P.center.z};
    float w = fmaxf(1.0f - dot3(off, off) / (P.radius * P.radius), 0.0f);
    Store<T>::st(out, i, value + P.dt * P.rate * w * w);
}

template <typename T>
__global__ void mac_advect_density_kernel(OpenParams P, Faces<T> F, const T* in, T* out) {
    const Dev& d = P.d;
    int x, y, z;
    if (!cell_coords(d.nx, d.ny, x, y, z)) return;
    const int i = cidx(d, x, y, z);
    F3 p = {((float)x + 0.5f) * d.h[0], ((float)y + 0.5f) * d.h[1], ((float)z + 0.5f) * d.h[2]};
    F3 v0 = velocity_at(d, F, p);
    F3 dep = backtrace<T, false>(d, F, nullptr, nullptr, p, v0, P.dt);
    float value = sample_zero(d, in, dep.x / d.h[0] - 0.5f, dep.y / d.h[1] - 0.5f, dep.z / d.h[2] - 0.5f) *
                  expf(-P.decay * P.dt);
    F3 off = {p.x - P.center.x, p.y - P.center.y, p.z - P.center.z};
    float w = fmaxf(1.0f - dot3(off, off) / (P.radius * P.radius), 0.0f);
    Store<T>::st(out, i, value + P.dt * P.rate * w * w);
}

// Launch the (collider mask, power-of-two grid) instantiation of a kernel.
#define FFX_DISPATCH_MASK_P2(mask, p2, M, P, ...)             \
    do {                                                       \
        if (mask) {                                            \
            if (p2) { constexpr bool M = true, P = true; __VA_ARGS__; }   \
            else { constexpr bool M = true, P = false; __VA_ARGS__; }     \
        } else {                                               \
            if (p2) { constexpr bool M = false, P = true; __VA_ARGS__; }  \
            else { constexpr bool M = false, P = false; __VA_ARGS__; }    \
        }                                                      \
    } while (0)

bool solids_ok(const FfxSolids* s) {
    if (!s) return true;
    const bool walls = s->wall[0] || s->wall[1] || s->wall[2];
    if (walls && !(s->wall[0] && s->wall[1] && s->wall[2] && s->solid)) return false;   // all three, with a mask
    if (s->clear && !s->solid) return false;                  // clearance only with a mask
    return (!s->solid && !s->halo) || (s->solid && s->halo);
}
bool has_mask(const FfxSolids* s) { return s && s->solid; }

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" {

int ffx_set_transport_tiling(int enable) {
    const int previous = g_tiling;
    g_tiling = enable ? 1 : 0;
    return previous;
}

static int face_predictor_impl(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                               const void* w, float dt, const float* dtp, void* pu, void* pv, void* pw,
                               float* const dep[3], void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solids_ok(s) && u && v && w && pu && pv && pw,
                "ffx_face_predictor: invalid arguments");
    FFX_REQUIRE(pu != u && pv != v && pw != w, "ffx_face_predictor: outputs must not alias inputs");
    Dev d = make_dev(*g);
    dim3 blocks = face_grid(d.nx, d.ny, d.nz), threads = cell_block();
    cudaStream_t st = as_stream(stream);
    const uint8_t* solid = has_mask(s) ? s->solid : nullptr;
    FFX_DISPATCH_STORAGE(storage, T, {
        Faces<T> F = {(const T*)u, (const T*)v, (const T*)w};
        const uint8_t* halo = solid ? s->halo : nullptr;
        PredParams<T> Q;
        Q.d = d;
        Q.solid = solid;
        Q.halo = halo;
        Q.clear = solid ? s->clear : nullptr;
        Q.F = F;
        Q.dt = dt;
        Q.dtp = dtp;
        Q.dt_sign = 1.f;
        Q.out[0] = (T*)pu; Q.out[1] = (T*)pv; Q.out[2] = (T*)pw;
        for (int a = 0; a < 3; ++a) {
            Q.dep[a] = dep ? dep[a] : nullptr;
            Q.nf[a] = (d.nx + (a == 0)) * (d.ny + (a == 1)) * (d.nz + (a == 2));
        }
        if (g_tiling) {
            const int zc = FFX_TILE_ZCHUNK;
            FFX_DISPATCH_MASK_P2(solid != nullptr, d.pow2 != 0, M, P,
                                 (face_predictor_tiled_kernel<T, M, P><<<tiled_grid(d.nx, d.ny, d.nz, zc), threads, 0, st>>>(Q, zc)));
        } else {
            FFX_DISPATCH_MASK_P2(solid != nullptr, d.pow2 != 0, M, P, (face_predictor_kernel<T, M, P><<<blocks, threads, 0, st>>>(Q)));
        }
    });
    return launch_status("face_predictor_kernel");
}

int ffx_face_predictor_trace(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                             const void* w, float dt, void* pu, void* pv, void* pw, float* const dep[3],
                             void* stream) {
    return face_predictor_impl(g, s, storage, u, v, w, dt, nullptr, pu, pv, pw, dep, stream);
}

int ffx_face_predictor_dt(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                          const void* w, const float* dt, void* pu, void* pv, void* pw, float* const dep[3],
                          void* stream) {
    FFX_REQUIRE(dt, "ffx_face_predictor_dt: NULL time step");
    return face_predictor_impl(g, s, storage, u, v, w, 0.f, dt, pu, pv, pw, dep, stream);
}

int ffx_face_predictor(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                       const void* w, float dt, void* pu, void* pv, void* pw, void* stream) {
    return ffx_face_predictor_trace(g, s, storage, u, v, w, dt, pu, pv, pw, nullptr, stream);
}

static int advect_velocity_impl(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                                const void* w, const void* pu, const void* pv, const void* pw, float dt,
                                const float* dtp, int corrected, float blend, const FfxSources* src,
                                const void* density, const void* temperature, float lift, float weight,
                                int apply_walls, void* ou, void* ov, void* ow, const float* const dep[3],
                                void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solids_ok(s) && u && v && w && ou && ov && ow,
                "ffx_advect_velocity: invalid arguments");
    FFX_REQUIRE(!corrected || (pu && pv && pw), "ffx_advect_velocity: MacCormack needs the predictor faces");
    FFX_REQUIRE(ou != u && ov != v && ow != w, "ffx_advect_velocity: outputs must not alias inputs");
    FFX_REQUIRE(!src || src->count <= 8, "ffx_advect_velocity: at most eight sources");
    FFX_REQUIRE((density == nullptr) == (temperature == nullptr), "ffx_advect_velocity: density and temperature "
                "must both be given for buoyancy");
    FFX_REQUIRE(blend >= 0.f && blend <= 1.f, "ffx_advect_velocity: blend must lie in [0, 1]");
    Dev d = make_dev(*g);
    // departure points are reused only where both passes form the same start points
    const bool starts = dep && corrected && face_starts_match(d);
    dim3 blocks = face_grid(d.nx, d.ny, d.nz), threads = cell_block();
    cudaStream_t st = as_stream(stream);
    FFX_DISPATCH_STORAGE(storage, T, {
        VelParams<T> P;
        P.d = d;
        P.solid = has_mask(s) ? s->solid : nullptr;
        P.halo = has_mask(s) ? s->halo : nullptr;
        P.clear = has_mask(s) ? s->clear : nullptr;
        P.F = {(const T*)u, (const T*)v, (const T*)w};
        P.P = corrected ? Faces<T>{(const T*)pu, (const T*)pv, (const T*)pw} : P.F;
        P.dt = dt;
        P.dtp = dtp;
        P.dt_sign = 1.f;
        P.blend = blend;
        P.lift = lift;
        P.weight = weight;
        P.corrected = corrected;
        P.apply_walls = apply_walls;
        P.density = (const T*)density;
        P.temperature = (const T*)temperature;
        P.out[0] = (T*)ou; P.out[1] = (T*)ov; P.out[2] = (T*)ow;
        P.walls = make_walls(s);
        for (int a = 0; a < 3; ++a) {
            P.dep[a] = (dep && corrected && starts) ? dep[a] : nullptr;
            P.nf[a] = (d.nx + (a == 0)) * (d.ny + (a == 1)) * (d.nz + (a == 2));
        }
        const float extent[3] = {g->ex, g->ey, g->ez};
        P.src = make_src(src, extent);
        if (!src) P.src.count = 0;
        if (g_tiling) {
            const int zc = FFX_TILE_ZCHUNK;
            FFX_DISPATCH_MASK_P2(P.solid != nullptr, d.pow2 != 0, M, Q,
                                 (advect_velocity_tiled_kernel<T, M, Q><<<tiled_grid(d.nx, d.ny, d.nz, zc), threads, 0, st>>>(P, zc)));
        } else {
            FFX_DISPATCH_MASK_P2(P.solid != nullptr, d.pow2 != 0, M, Q, (advect_velocity_kernel<T, M, Q><<<blocks, threads, 0, st>>>(P)));
        }
    });
    return launch_status("advect_velocity_kernel");
}

int ffx_advect_velocity_trace(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                              const void* w, const void* pu, const void* pv, const void* pw, float dt,
                              int corrected, float blend, const FfxSources* src, const void* density,
                              const void* temperature, float lift, float weight, int apply_walls, void* ou,
                              void* ov, void* ow, const float* const dep[3], void* stream) {
    return advect_velocity_impl(g, s, storage, u, v, w, pu, pv, pw, dt, nullptr, corrected, blend, src, density,
                                temperature, lift, weight, apply_walls, ou, ov, ow, dep, stream);
}

int ffx_advect_velocity_dt(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                           const void* w, const void* pu, const void* pv, const void* pw, const float* dt,
                           int corrected, float blend, const FfxSources* src, const void* density,
                           const void* temperature, float lift, float weight, int apply_walls, void* ou,
                           void* ov, void* ow, const float* const dep[3], void* stream) {
    FFX_REQUIRE(dt, "ffx_advect_velocity_dt: NULL time step");
    return advect_velocity_impl(g, s, storage, u, v, w, pu, pv, pw, 0.f, dt, corrected, blend, src, density,
                                temperature, lift, weight, apply_walls, ou, ov, ow, dep, stream);
}

int ffx_advect_velocity(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                        const void* w, const void* pu, const void* pv, const void* pw, float dt, int corrected,
                        float blend, const FfxSources* src, const void* density, const void* temperature,
                        float lift, float weight, int apply_walls, void* ou, void* ov, void* ow, void* stream) {
    return ffx_advect_velocity_trace(g, s, storage, u, v, w, pu, pv, pw, dt, corrected, blend, src, density,
                                     temperature, lift, weight, apply_walls, ou, ov, ow, nullptr, stream);
}

int ffx_mac_advect_velocity(const FfxGrid* g, int storage, const void* u, const void* v, const void* w, float dt,
                            void* ou, void* ov, void* ow, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && u && v && w && ou && ov && ow && ou != u && ov != v && ow != w,
                "ffx_mac_advect_velocity: invalid arguments");
    Dev d = make_dev(*g);
    dim3 blocks = face_grid(d.nx, d.ny, d.nz), threads = cell_block();
    FFX_DISPATCH_STORAGE(storage, T, {
        Faces<T> F = {(const T*)u, (const T*)v, (const T*)w};
        mac_advect_velocity_kernel<T><<<blocks, threads, 0, as_stream(stream)>>>(d, F, dt, (T*)ou, (T*)ov, (T*)ow);
    });
    return launch_status("mac_advect_velocity_kernel");
}

int ffx_buoyancy(const FfxGrid* g, int storage, const void* w_in, const void* density, const void* temperature,
                 float dt, float lift, float weight, void* w_out, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && w_in && density && temperature && w_out && w_in != w_out,
                "ffx_buoyancy: invalid arguments");
    Dev d = make_dev(*g);
    dim3 grid = cell_grid(g->nx, g->ny, g->nz + 1), block = cell_block();
    FFX_DISPATCH_STORAGE(storage, T,
        buoyancy_kernel<T><<<grid, block, 0, as_stream(stream)>>>(
            d, (const T*)w_in, (const T*)density, (const T*)temperature, dt, lift, weight, (T*)w_out));
    return launch_status("buoyancy_kernel");
}

static int scalar_transport_impl(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                                 const void* w, float dt, const float* dtp, float sign, int count,
                                 const void* const* in, void* const* out, float* dep, void* stream,
                                 const float* fdep = nullptr, uint8_t* ok = nullptr) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solids_ok(s) && u && v && w && count >= 1 && count <= 3 && in &&
                out, "ffx_scalar_transport: invalid arguments");
    for (int c = 0; c < count; ++c)
        FFX_REQUIRE(in[c] && out[c] && in[c] != out[c], "ffx_scalar_transport: channel %d invalid or aliased", c);
    Dev d = make_dev(*g);
    dim3 grid = cell_grid(g->nx, g->ny, g->nz), block = cell_block();
    cudaStream_t st = as_stream(stream);
    FFX_DISPATCH_STORAGE(storage, T, {
        ScalarXport<T> P;
        P.d = d;
        P.solid = has_mask(s) ? s->solid : nullptr;
        P.halo = has_mask(s) ? s->halo : nullptr;
        P.clear = has_mask(s) ? s->clear : nullptr;
        P.F = {(const T*)u, (const T*)v, (const T*)w};
        P.dt = dt;
        P.dtp = dtp;
        P.dt_sign = sign;
        P.count = count;
        for (int c = 0; c < 3; ++c) {
            P.in[c] = c < count ? (const T*)in[c] : nullptr;
            P.out[c] = c < count ? (T*)out[c] : nullptr;
        }
        P.dep = dep;
        P.n = g->nx * g->ny * g->nz;
        P.fdep = fdep;
        P.ok = ok;
        if (g_tiling) {
            const int zc = FFX_TILE_ZCHUNK;
            FFX_DISPATCH_MASK_P2(P.solid != nullptr, d.pow2 != 0, M, Q,
                                 (scalar_transport_tiled_kernel<T, M, Q><<<tiled_grid(d.nx, d.ny, d.nz, zc), block, 0, st>>>(P, zc)));
        } else {
            if (ok) {
                FFX_DISPATCH_MASK_P2(P.solid != nullptr, d.pow2 != 0, M, Q,
                                     (scalar_reverse_ok_kernel<T, M, Q><<<grid, block, 0, st>>>(P)));
            } else {
                FFX_DISPATCH_MASK_P2(P.solid != nullptr, d.pow2 != 0, M, Q,
                                     (scalar_transport_kernel<T, M, Q><<<grid, block, 0, st>>>(P)));
            }
        }
    });
    return launch_status("scalar_transport_kernel");
}

int ffx_scalar_transport_trace(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                               const void* w, float dt, int count, const void* const* in, void* const* out,
                               float* dep, void* stream) {
    return scalar_transport_impl(g, s, storage, u, v, w, dt, nullptr, 1.f, count, in, out, dep, stream);
}

int ffx_scalar_transport_dt(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                            const void* w, const float* dt, float sign, int count, const void* const* in,
                            void* const* out, float* dep, void* stream) {
    FFX_REQUIRE(dt && (sign == 1.f || sign == -1.f), "ffx_scalar_transport_dt: NULL time step or sign not +-1");
    return scalar_transport_impl(g, s, storage, u, v, w, 0.f, dt, sign, count, in, out, dep, stream);
}

int ffx_scalar_transport(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                         const void* w, float dt, int count, const void* const* in, void* const* out, void* stream) {
    return ffx_scalar_transport_trace(g, s, storage, u, v, w, dt, count, in, out, nullptr, stream);
}

int ffx_scalar_reverse_ok(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                          const void* w, float dt, const float* dtp, int count, const void* const* in,
                          void* const* out, const float* dep, uint8_t* ok, void* stream) {
    FFX_REQUIRE(dep && ok, "ffx_scalar_reverse_ok: NULL departure points or decisions");
    FFX_REQUIRE(dtp || dt < 0.f, "ffx_scalar_reverse_ok: the reverse pass runs with a negative time step");
    return scalar_transport_impl(g, s, storage, u, v, w, dt, dtp, -1.f, count, in, out, nullptr, stream, dep, ok);
}

static int advect_scalars_impl(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                               const void* w, float dt, const float* dtp, int corrected, const FfxSources* src,
                               int count, const FfxScalarChannel* channels, float* maxima, const float* dep,
                               void* stream, const uint8_t* ok = nullptr) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solids_ok(s) && u && v && w && count >= 1 && count <= 3 &&
                channels && src && src->count <= 8, "ffx_advect_scalars: invalid arguments");
    for (int c = 0; c < count; ++c) {
        const FfxScalarChannel& C = channels[c];
        FFX_REQUIRE(C.field && C.out && C.out != C.field, "ffx_advect_scalars: channel %d invalid or aliased", c);
        FFX_REQUIRE(!corrected || (C.predictor && C.reverse), "ffx_advect_scalars: channel %d lacks predictor", c);
    }
    Dev d = make_dev(*g);
    dim3 grid = cell_grid(g->nx, g->ny, g->nz), block = cell_block();
    cudaStream_t st = as_stream(stream);
    if (maxima) {
        int e = cuda_status(cudaMemsetAsync(maxima, 0, sizeof(float) * count, st), "ffx_advect_scalars memset");
        if (e) return e;
    }
    FFX_DISPATCH_STORAGE(storage, T, {
        ScalarFinal<T> P;
        P.d = d;
        P.solid = has_mask(s) ? s->solid : nullptr;
        P.halo = has_mask(s) ? s->halo : nullptr;
        P.clear = has_mask(s) ? s->clear : nullptr;
        P.F = {(const T*)u, (const T*)v, (const T*)w};
        P.dt = dt;
        P.dtp = dtp;
        P.dt_sign = 1.f;
        P.corrected = corrected;
        P.count = count;
        for (int c = 0; c < 3; ++c) {
            Channel<T> C = {};
            if (c < count) {
                const FfxScalarChannel& H = channels[c];
                C.field = (const T*)H.field;
                C.pred = (const T*)(H.predictor ? H.predictor : H.field);
                C.rev = (const T*)(H.reverse ? H.reverse : H.field);
                C.out = (T*)H.out;
                C.rate = H.rate;
                C.decay = H.decay;
                C.target = H.target;
                C.channel = H.channel;
                C.table_target = H.table_target;
            }
            P.ch[c] = C;
            P.fields[c] = C.field;
        }
        P.maxima = maxima;
        P.dep = corrected ? dep : nullptr;
        P.n = g->nx * g->ny * g->nz;
        P.ok = corrected ? ok : nullptr;
        const float extent[3] = {g->ex, g->ey, g->ez};
        P.src = make_src(src, extent);
        if (g_tiling) {
            const int zc = FFX_TILE_ZCHUNK;
            FFX_DISPATCH_MASK_P2(P.solid != nullptr, d.pow2 != 0, M, Q,
                                 (advect_scalars_tiled_kernel<T, M, Q><<<tiled_grid(d.nx, d.ny, d.nz, zc), block, 0, st>>>(P, zc)));
        } else {
            FFX_DISPATCH_MASK_P2(P.solid != nullptr, d.pow2 != 0, M, Q, (advect_scalars_kernel<T, M, Q><<<grid, block, 0, st>>>(P)));
        }
    });
    return launch_status("advect_scalars_kernel");
}

int ffx_advect_scalars_trace(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                             const void* w, float dt, int corrected, const FfxSources* src, int count,
                             const FfxScalarChannel* channels, float* maxima, const float* dep, void* stream) {
    return advect_scalars_impl(g, s, storage, u, v, w, dt, nullptr, corrected, src, count, channels, maxima, dep,
                               stream);
}

int ffx_advect_scalars_dt(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                          const void* w, const float* dt, int corrected, const FfxSources* src, int count,
                          const FfxScalarChannel* channels, float* maxima, const float* dep, void* stream) {
    FFX_REQUIRE(dt, "ffx_advect_scalars_dt: NULL time step");
    return advect_scalars_impl(g, s, storage, u, v, w, 0.f, dt, corrected, src, count, channels, maxima, dep,
                               stream);
}

int ffx_advect_scalars(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                       const void* w, float dt, int corrected, const FfxSources* src, int count,
                       const FfxScalarChannel* channels, float* maxima, void* stream) {
    return ffx_advect_scalars_trace(g, s, storage, u, v, w, dt, corrected, src, count, channels, maxima, nullptr,
                                    stream);
}

int ffx_advect_scalars_ok(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                          const void* w, float dt, const float* dtp, int corrected, const FfxSources* src,
                          int count, const FfxScalarChannel* channels, float* maxima, const float* dep,
                          const uint8_t* ok, void* stream) {
    FFX_REQUIRE(!corrected || (dep && ok), "ffx_advect_scalars_ok: NULL departure points or decisions");
    return advect_scalars_impl(g, s, storage, u, v, w, dt, dtp, corrected, src, count, channels, maxima, dep,
                               stream, ok);
}

int ffx_advect_open(const FfxGrid* g, int storage, const void* in, float dt, const float base[3], float angular,
                    const float center[3], float radius, float rate, float decay, void* out, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && in && out && in != out && base && center && radius > 0.f,
                "ffx_advect_open: invalid arguments");
    OpenParams P;
    P.d = make_dev(*g);
    P.dt = dt; P.angular = angular; P.radius = radius; P.rate = rate; P.decay = decay;
    P.base = {base[0], base[1], base[2]};
    P.center = {center[0], center[1], center[2]};
    dim3 grid = cell_grid(g->nx, g->ny, g->nz), block = cell_block();
    FFX_DISPATCH_STORAGE(storage, T,
        advect_open_kernel<T><<<grid, block, 0, as_stream(stream)>>>(P, (const T*)in, (T*)out));
    return launch_status("advect_open_kernel");
}

int ffx_mac_advect_density(const FfxGrid* g, int storage, const void* u, const void* v, const void* w, const void* in,
                           float dt, const float center[3], float radius, float rate, float decay, void* out,
                           void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && u && v && w && in && out && in != out && center && radius > 0.f,
                "ffx_mac_advect_density: invalid arguments");
    OpenParams P;
    P.d = make_dev(*g);
    P.dt = dt; P.angular = 0.f; P.radius = radius; P.rate = rate; P.decay = decay;
    P.base = {0.f, 0.f, 0.f};
    P.center = {center[0], center[1], center[2]};
    dim3 grid = cell_grid(g->nx, g->ny, g->nz), block = cell_block();
    FFX_DISPATCH_STORAGE(storage, T, {
        Faces<T> F = {(const T*)u, (const T*)v, (const T*)w};
        mac_advect_density_kernel<T><<<grid, block, 0, as_stream(stream)>>>(P, F, (const T*)in,
                                                                                                (T*)out);
    });
    return launch_status("mac_advect_density_kernel");
}

}  // extern "C"

// ----------------------------------------------------------- batched passes
// Persistent launches over the tiles of many domains (ffx_batch.cuh). Every
// domain is on the collider path; pow2 (exact reciprocal division) is chosen
// per domain, as the single-domain launch chooses it per launch.
namespace ffx {
namespace {

// Occupancy targets of the batched transport kernels (their loops carry both
// the power-of-two and the general body; 0: the compiler's choice), chosen by
// measurement on the 48-domain batch.
#ifndef FFX_MINB_BATCH_PREDICTOR
#define FFX_MINB_BATCH_PREDICTOR 0
#endif
#ifndef FFX_MINB_BATCH_VELOCITY
#define FFX_MINB_BATCH_VELOCITY 5
#endif
#ifndef FFX_MINB_BATCH_SCALARS
#define FFX_MINB_BATCH_SCALARS 4
#endif
#if FFX_MINB_BATCH_PREDICTOR > 0
#define FFX_LB_BATCH_PREDICTOR __launch_bounds__(kBatchThreads, FFX_MINB_BATCH_PREDICTOR)
#else
#define FFX_LB_BATCH_PREDICTOR __launch_bounds__(kBatchThreads)
#endif
#if FFX_MINB_BATCH_VELOCITY > 0
#define FFX_LB_BATCH_VELOCITY __launch_bounds__(kBatchThreads, FFX_MINB_BATCH_VELOCITY)
#else
#define FFX_LB_BATCH_VELOCITY __launch_bounds__(kBatchThreads)
#endif
#if FFX_MINB_BATCH_SCALARS > 0
#define FFX_LB_BATCH_SCALARS __launch_bounds__(kBatchThreads, FFX_MINB_BATCH_SCALARS)
#else
#define FFX_LB_BATCH_SCALARS __launch_bounds__(kBatchThreads)
#endif

// prep: the descriptor's time step is the domain's device dt (times `sign`).
struct DeviceDt {
    const BatchState* state;
    float sign;
    template <class D>
    __device__ __forceinline__ void operator()(D& sh, int slot) const { sh.dt = sign * state[slot].dt; }
};

__global__ void FFX_LB_BATCH_PREDICTOR batch_predictor_kernel(const __grid_constant__ BatchMap M,
                                                                        const PredParams<float>* descs,
                                                                        const BatchState* state) {
    for_tiles(M, descs, state, false, DeviceDt{state, 1.f}, [](const PredParams<float>& P, const Blk& b, int) {
        if (P.d.pow2) face_predictor_body<float, true, true>(P, b);
        else face_predictor_body<float, true, false>(P, b);
    });
}

__global__ void FFX_LB_BATCH_VELOCITY batch_velocity_kernel(const __grid_constant__ BatchMap M,
                                                                       const VelParams<float>* descs,
                                                                       const BatchState* state) {
    for_tiles(M, descs, state, false, DeviceDt{state, 1.f}, [](const VelParams<float>& P, const Blk& b, int) {
        if (P.d.pow2) advect_velocity_body<float, true, true>(P, b);
        else advect_velocity_body<float, true, false>(P, b);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_scalar_transport_kernel(const __grid_constant__ BatchMap M,
                                                                               const ScalarXport<float>* descs,
                                                                               const BatchState* state, float sign) {
    for_tiles(M, descs, state, false, DeviceDt{state, sign}, [](const ScalarXport<float>& P, const Blk& b, int) {
        if (P.d.pow2) scalar_transport_body<float, true, true>(P, b);
        else scalar_transport_body<float, true, false>(P, b);
    });
}

// The reverse pass: domains with decision buffers decide the final pass's corrections.
__global__ void __launch_bounds__(kBatchThreads) batch_scalar_reverse_kernel(const __grid_constant__ BatchMap M,
                                                                             const ScalarXport<float>* descs,
                                                                             const BatchState* state) {
    using S = GlobalSampler<CellFields<float>>;
    for_tiles(M, descs, state, false, DeviceDt{state, -1.f}, [](const ScalarXport<float>& P, const Blk& b, int) {
        int x, y, z;
        if (!cell_coords(b, P.d.nx, P.d.ny, x, y, z)) return;
        const auto smp = cell_sampler<float>(P.d, P.F, P.in);
        if (P.ok) {
            if (P.d.pow2) scalar_transport_cell<float, true, true, S, true>(P, x, y, z, smp);
            else scalar_transport_cell<float, true, false, S, true>(P, x, y, z, smp);
        } else {
            if (P.d.pow2) scalar_transport_cell<float, true, true, S, false>(P, x, y, z, smp);
            else scalar_transport_cell<float, true, false, S, false>(P, x, y, z, smp);
        }
    });
}

__global__ void FFX_LB_BATCH_SCALARS batch_scalars_kernel(const __grid_constant__ BatchMap M,
                                                                      const ScalarFinal<float>* descs,
                                                                      const BatchState* state) {
    for_tiles(M, descs, state, false, DeviceDt{state, 1.f}, [](const ScalarFinal<float>& P, const Blk& b, int) {
        if (P.d.pow2) advect_scalars_body<float, true, true>(P, b);
        else advect_scalars_body<float, true, false>(P, b);
    });
}

template <class K>
int occupancy(K kernel) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kBatchThreads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

unsigned grid_of(const BatchMap& M, int grid) { return (unsigned)(grid > 0 && grid < M.total ? grid : M.total); }

}  // namespace

namespace batch {

size_t predictor_desc(const FfxBatchDomain& D, void* out) {
    if (out) {
        PredParams<float> P;
        memset(&P, 0, sizeof P);   // no departure output in the batched pass
        P.d = make_dev(D.grid);
        P.solid = D.solid;
        P.halo = D.halo;
        P.clear = D.clear;
        P.F = {D.u, D.v, D.w};
        P.dt = 0.f;
        P.out[0] = D.pu; P.out[1] = D.pv; P.out[2] = D.pw;
        const int nx = D.grid.nx, ny = D.grid.ny, nz = D.grid.nz;
        for (int a = 0; a < 3; ++a) {
            P.dep[a] = D.face_trace[a];
            P.nf[a] = (nx + (a == 0)) * (ny + (a == 1)) * (nz + (a == 2));
        }
        memcpy(out, &P, sizeof P);
    }
    return sizeof(PredParams<float>);
}

size_t velocity_desc(const FfxBatchDomain& D, int parity, void* out) {
    if (out) {
        VelParams<float> P;
        memset(&P, 0, sizeof P);
        P.d = make_dev(D.grid);
        P.solid = D.solid;
        P.halo = D.halo;
        P.clear = D.clear;
        P.F = {D.u, D.v, D.w};
        P.P = D.velocity_corrected ? Faces<float>{D.pu, D.pv, D.pw} : P.F;
        P.dt = 0.f;
        P.blend = D.blend;
        P.lift = D.lift;
        P.weight = D.weight;
        P.corrected = D.velocity_corrected;
        P.apply_walls = 1;
        P.density = D.density[parity];
        P.temperature = D.temperature[parity];
        P.out[0] = D.bu; P.out[1] = D.bv; P.out[2] = D.bw;
        P.walls = make_walls(nullptr);
        const int nx = D.grid.nx, ny = D.grid.ny, nz = D.grid.nz;
        const bool starts = D.velocity_corrected && face_starts_match(P.d);
        for (int a = 0; a < 3; ++a) {
            P.dep[a] = starts ? D.face_trace[a] : nullptr;
            P.nf[a] = (nx + (a == 0)) * (ny + (a == 1)) * (nz + (a == 2));
        }
        const float extent[3] = {D.grid.ex, D.grid.ey, D.grid.ez};
        P.src = make_src(&D.sources, extent);
        memcpy(out, &P, sizeof P);
    }
    return sizeof(VelParams<float>);
}

size_t scalar_xport_desc(const FfxBatchDomain& D, int parity, int reverse, void* out) {
    if (out) {
        ScalarXport<float> P;
        memset(&P, 0, sizeof P);
        P.d = make_dev(D.grid);
        P.solid = D.solid;
        P.halo = D.halo;
        P.F = {D.u, D.v, D.w};
        P.dt = 0.f;
        P.count = 2;
        P.in[0] = reverse ? D.predictor[0] : D.density[parity];
        P.in[1] = reverse ? D.predictor[1] : D.temperature[parity];
        P.out[0] = reverse ? D.reverse[0] : D.predictor[0];
        P.out[1] = reverse ? D.reverse[1] : D.predictor[1];
        P.dep = reverse ? nullptr : D.cell_trace;     // the forward pass stores its departure points
        P.n = D.grid.nx * D.grid.ny * D.grid.nz;
        P.clear = D.clear;
        if (reverse && D.cell_trace && D.cell_ok) {  // the reverse pass decides the final pass's corrections
            P.fdep = D.cell_trace;
            P.ok = D.cell_ok;
        }
        memcpy(out, &P, sizeof P);
    }
    return sizeof(ScalarXport<float>);
}

size_t scalar_final_desc(const FfxBatchDomain& D, int parity, void* out) {
    if (out) {
        ScalarFinal<float> P;
        memset(&P, 0, sizeof P);
        P.d = make_dev(D.grid);
        P.solid = D.solid;
        P.halo = D.halo;
        P.F = {D.u, D.v, D.w};
        P.dt = 0.f;
        P.corrected = D.scalar_corrected;
        P.count = 2;
        const FfxScalarChannel* H[2] = {&D.density_channel, &D.heat_channel};
        const float* field[2] = {D.density[parity], D.temperature[parity]};
        float* dst[2] = {D.density[1 - parity], D.temperature[1 - parity]};
        for (int c = 0; c < 2; ++c) {
            Channel<float> C = {};
            C.field = field[c];
            C.pred = D.scalar_corrected ? D.predictor[c] : field[c];
            C.rev = D.scalar_corrected ? D.reverse[c] : field[c];
            C.out = dst[c];
            C.rate = H[c]->rate;
            C.decay = H[c]->decay;
            C.target = H[c]->target;
            C.channel = H[c]->channel;
            C.table_target = H[c]->table_target;
            P.ch[c] = C;
            P.fields[c] = C.field;
        }
        P.maxima = nullptr;
        P.dep = D.scalar_corrected ? D.cell_trace : nullptr;
        P.n = D.grid.nx * D.grid.ny * D.grid.nz;
        P.clear = D.clear;
        P.ok = (D.scalar_corrected && D.cell_trace) ? D.cell_ok : nullptr;
        const float extent[3] = {D.grid.ex, D.grid.ey, D.grid.ez};
        P.src = make_src(&D.sources, extent);
        memcpy(out, &P, sizeof P);
    }
    return sizeof(ScalarFinal<float>);
}

cudaError_t face_predictor(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_predictor_kernel<<<grid_of(M, grid), kBatchThreads, 0, st>>>(M, (const PredParams<float>*)descs, state);
    return cudaGetLastError();
}
cudaError_t advect_velocity(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_velocity_kernel<<<grid_of(M, grid), kBatchThreads, 0, st>>>(M, (const VelParams<float>*)descs, state);
    return cudaGetLastError();
}
cudaError_t scalar_transport(const BatchMap& M, const void* descs, BatchState* state, int reverse, int grid,
                             cudaStream_t st) {
    if (reverse)
        batch_scalar_reverse_kernel<<<grid_of(M, grid), kBatchThreads, 0, st>>>(M, (const ScalarXport<float>*)descs,
                                                                               state);
    else
        batch_scalar_transport_kernel<<<grid_of(M, grid), kBatchThreads, 0, st>>>(
            M, (const ScalarXport<float>*)descs, state, 1.f);
    return cudaGetLastError();
}
cudaError_t advect_scalars(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_scalars_kernel<<<grid_of(M, grid), kBatchThreads, 0, st>>>(M, (const ScalarFinal<float>*)descs, state);
    return cudaGetLastError();
}

int advect_resident_blocks(int kind) {
    switch (kind) {
        case kPredictor: return occupancy(batch_predictor_kernel);
        case kVelocity: return occupancy(batch_velocity_kernel);
        case kScalarPredictor:
        case kScalarReverse: return occupancy(batch_scalar_reverse_kernel);
        case kScalarFinal: return occupancy(batch_scalars_kernel);
        default: return 0;
    }
}

}  // namespace batch
}  // namespace ffx
