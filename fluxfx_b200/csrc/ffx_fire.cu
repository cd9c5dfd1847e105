// Fire-configuration passes: vorticity confinement, combustion and moving
// colliders (mask refresh, rigid wall velocities, field remap).
//
// Each kernel evaluates the reference shader's expression in the same FP32
// operation order (component-wise vector arithmetic, dot sums x, y, z[, w]
// left to right), under the library-wide --fmad=false.
#include "ffx_common.cuh"
#include "ffx_host.cuh"

namespace ffx {
namespace {

// centeredVelocity (curl.glsl:1-7): face averages at the clamped cell.
template <typename T>
__device__ __forceinline__ F3 centered(const Dev& d, const Faces<T>& F, int x, int y, int z) {
    x = min(max(x, 0), d.nx - 1);
    y = min(max(y, 0), d.ny - 1);
    z = min(max(z, 0), d.nz - 1);
    const int iu = x + (d.nx + 1) * (y + d.ny * z);
    const int iv = x + d.nx * (y + (d.ny + 1) * z);
    const int iw = cidx(d, x, y, z);
    return {0.5f * (Store<T>::ld(F.u, iu) + Store<T>::ld(F.u, iu + 1)),
            0.5f * (Store<T>::ld(F.v, iv) + Store<T>::ld(F.v, iv + d.nx)),
            0.5f * (Store<T>::ld(F.w, iw) + Store<T>::ld(F.w, iw + d.nx * d.ny))};
}

// curl.glsl:8-17: omega = curl of the cell-centred velocity (central
// differences, clamped), w = |omega|.
template <typename T>
__global__ void __launch_bounds__(256) curl_kernel(Dev d, Faces<T> F, float4* out) {
    int x, y, z;
    if (!cell_coords(d.nx, d.ny, x, y, z)) return;
    F3 a = centered(d, F, x + 1, y, z), b = centered(d, F, x - 1, y, z);
    const F3 dx = {((a.x - b.x) * 0.5f) * d.inv[0], ((a.y - b.y) * 0.5f) * d.inv[0], ((a.z - b.z) * 0.5f) * d.inv[0]};
    a = centered(d, F, x, y + 1, z);
    b = centered(d, F, x, y - 1, z);
    const F3 dy = {((a.x - b.x) * 0.5f) * d.inv[1], ((a.y - b.y) * 0.5f) * d.inv[1], ((a.z - b.z) * 0.5f) * d.inv[1]};
    a = centered(d, F, x, y, z + 1);
    b = centered(d, F, x, y, z - 1);
    const F3 dz = {((a.x - b.x) * 0.5f) * d.inv[2], ((a.y - b.y) * 0.5f) * d.inv[2], ((a.z - b.z) * 0.5f) * d.inv[2]};
    const F3 om = {dy.z - dz.y, dz.x - dx.z, dx.y - dy.x};
    out[cidx(d, x, y, z)] = make_float4(om.x, om.y, om.z, sqrtf(dot3(om, om)));
}

__device__ __forceinline__ float4 curl_at(const Dev& d, const float4* __restrict__ c4, int x, int y, int z) {
    x = min(max(x, 0), d.nx - 1);
    y = min(max(y, 0), d.ny - 1);
    z = min(max(z, 0), d.nz - 1);
    return __ldg(c4 + cidx(d, x, y, z));
}

// forceAt (confinement.glsl:5-15): strength * h * (grad|w| / |grad|w||) x omega,
// capped at `limit` in magnitude; 0 where |grad| < 1e-8.
__device__ __forceinline__ F3 force_at(const Dev& d, const float4* __restrict__ c4, int x, int y, int z,
                                       float strength, float limit) {
    const F3 g = {(0.5f * d.inv[0]) * (curl_at(d, c4, x + 1, y, z).w - curl_at(d, c4, x - 1, y, z).w),
                  (0.5f * d.inv[1]) * (curl_at(d, c4, x, y + 1, z).w - curl_at(d, c4, x, y - 1, z).w),
                  (0.5f * d.inv[2]) * (curl_at(d, c4, x, y, z + 1).w - curl_at(d, c4, x, y, z - 1).w)};
    const float mag = sqrtf(dot3(g, g));
    if (mag < 1e-8f) return {0.f, 0.f, 0.f};
    const float h = 1.0f / fmaxf(d.inv[0], fmaxf(d.inv[1], d.inv[2]));
    const F3 n = {g.x / mag, g.y / mag, g.z / mag};
    const float4 o = curl_at(d, c4, x, y, z);
    const F3 cr = {n.y * o.z - n.z * o.y, n.z * o.x - n.x * o.z, n.x * o.y - n.y * o.x};
    const float sh = strength * h;
    F3 f = {sh * cr.x, sh * cr.y, sh * cr.z};
    const float scale = fminf(1.0f, limit / fmaxf(sqrtf(dot3(f, f)), 1e-12f));
    return {f.x * scale, f.y * scale, f.z * scale};
}

// confinement.glsl:16-23: face value += dt * (average of the two cells' force).axis
template <typename T>
__global__ void __launch_bounds__(256) confine_kernel(Dev d, const float4* __restrict__ c4, Faces<T> F, float dt,
                                                     float strength, float limit, T* ou, T* ov, T* ow) {
    const int nz1 = d.nz + 1;
    const int zz = blockIdx.z;
    const int axis = zz >= 2 * nz1 ? 2 : (zz >= nz1 ? 1 : 0);
    const int z = zz - axis * nz1;
    const int sx = d.nx + (axis == 0), sy = d.ny + (axis == 1), sz = d.nz + (axis == 2);
    const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
    if (x >= sx || y >= sy || z >= sz) return;
    const int i = x + sx * (y + sy * z);
    const F3 fa = force_at(d, c4, x, y, z, strength, limit);
    const F3 fb = force_at(d, c4, x - (axis == 0), y - (axis == 1), z - (axis == 2), strength, limit);
    const float f = 0.5f * (comp(fa, axis) + comp(fb, axis));
    const T* in = axis == 0 ? F.u : (axis == 1 ? F.v : F.w);
    T* out = axis == 0 ? ou : (axis == 1 ? ov : ow);
    Store<T>::st(out, i, Store<T>::ld(in, i) + dt * f);
}

// combustion_burn.glsl + combustion_apply.glsl (backend/combustion.py:21-31) in
// one pass: flame = burned fuel per second; fuel, density and temperature take
// dt * yield * flame (fuel with yield -1, clamped at 0).
template <typename T>
__global__ void __launch_bounds__(256) combustion_kernel(int64_t n, const T* fuel, const T* temperature,
                                                        const T* density, float dt, float ignition, float rate,
                                                        float smoke_yield, float heat_yield, float* flame,
                                                        T* fuel_out, T* density_out, T* temperature_out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float fu = Store<T>::ld(fuel, i), t = Store<T>::ld(temperature, i), rho = Store<T>::ld(density, i);
    const float avail = fmaxf(fu, 0.0f);
    const float burned = t >= ignition ? avail * (1.0f - expf(-rate * dt)) : 0.0f;
    const float fl = burned / dt;
    flame[i] = fl;
    Store<T>::st(fuel_out, i, fmaxf(fu + (dt * -1.0f) * fl, 0.0f));
    Store<T>::st(density_out, i, rho + (dt * smoke_yield) * fl);
    Store<T>::st(temperature_out, i, t + (dt * heat_yield) * fl);
}

// moving_mask.glsl: owner id (1-based collider index, first one wins) of every
// cell centre inside a collider, FP32 point test.
struct MovingColliders {
    int count;
    float rows[FFX_MOVING_MAX][12];
    int box[FFX_MOVING_MAX];
};

__global__ void __launch_bounds__(256) moving_mask_kernel(Dev d, MovingColliders C, uint8_t* owners) {
    int x, y, z;
    if (!cell_coords(d.nx, d.ny, x, y, z)) return;
    const float px = dv_n<false>(d, ((float)x + 0.5f) * d.e[0], 0);
    const float py = dv_n<false>(d, ((float)y + 0.5f) * d.e[1], 1);
    const float pz = dv_n<false>(d, ((float)z + 0.5f) * d.e[2], 2);
    unsigned value = 0;
    for (int k = 0; k < C.count && value == 0; ++k) {
        const float* r = C.rows[k];
        const float q0 = ((r[0] * px + r[1] * py) + r[2] * pz) + r[3] * 1.0f;
        const float q1 = ((r[4] * px + r[5] * py) + r[6] * pz) + r[7] * 1.0f;
        const float q2 = ((r[8] * px + r[9] * py) + r[10] * pz) + r[11] * 1.0f;
        const bool inside = C.box[k] ? (fabsf(q0) <= 1.0f && fabsf(q1) <= 1.0f && fabsf(q2) <= 1.0f)
                                     : ((q0 * q0 + q1 * q1) + q2 * q2) <= 1.0f;
        if (inside) value = (unsigned)(k + 1);
    }
    owners[cidx(d, x, y, z)] = (uint8_t)value;
}

// moving_wall.glsl: velocity of the owning collider's rigid motion on every
// interior face next to a solid cell (the lower cell's owner first), else 0.
struct WallTable {
    float rows[FFX_MOVING_MAX][3][4];
};

__global__ void __launch_bounds__(256) moving_wall_kernel(Dev d, const uint8_t* __restrict__ owners, WallTable W,
                                                         float* wu, float* wv, float* ww) {
    const int nz1 = d.nz + 1;
    const int zz = blockIdx.z;
    const int axis = zz >= 2 * nz1 ? 2 : (zz >= nz1 ? 1 : 0);
    const int z = zz - axis * nz1;
    const int sx = d.nx + (axis == 0), sy = d.ny + (axis == 1), sz = d.nz + (axis == 2);
    const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
    if (x >= sx || y >= sy || z >= sz) return;
    const int c[3] = {x, y, z}, n[3] = {sx, sy, sz};
    float value = 0.f;
    if (c[axis] > 0 && c[axis] < n[axis] - 1) {
        const int hi = __ldg(owners + cidx(d, x, y, z));
        const int lo = __ldg(owners + cidx(d, x - (axis == 0), y - (axis == 1), z - (axis == 2)));
        const int owner = lo > 0 ? lo : hi;
        if (owner > 0 && owner <= FFX_MOVING_MAX) {
            const float off[3] = {axis == 0 ? 0.f : 0.5f, axis == 1 ? 0.f : 0.5f, axis == 2 ? 0.f : 0.5f};
            const float px = dv_n<false>(d, ((float)x + off[0]) * d.e[0], 0);
            const float py = dv_n<false>(d, ((float)y + off[1]) * d.e[1], 1);
            const float pz = dv_n<false>(d, ((float)z + off[2]) * d.e[2], 2);
            const float* r = W.rows[owner - 1][axis];
            value = ((r[0] * px + r[1] * py) + r[2] * pz) + r[3] * 1.0f;
        }
    }
    float* out = axis == 0 ? wu : (axis == 1 ? wv : ww);
    out[x + sx * (y + sy * z)] = value;
}

// moving_remap_scalar.glsl (in place): a cell covered now or before the move
// starts empty.
template <typename T>
__global__ void __launch_bounds__(256) remap_scalars_kernel(int64_t n, const uint8_t* __restrict__ owners,
                                                           const uint8_t* __restrict__ old_owners, T* a, T* b, T* c) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (__ldg(owners + i) || __ldg(old_owners + i)) {
        Store<T>::st(a, i, 0.f);
        if (b) Store<T>::st(b, i, 0.f);
        if (c) Store<T>::st(c, i, 0.f);
    }
}

// moving_remap_face.glsl (in place): interior faces of covered cells take the
// wall velocity, faces uncovered by the move start at 0, domain walls are 0.
template <typename T>
__global__ void __launch_bounds__(256) remap_faces_kernel(Dev d, const uint8_t* __restrict__ owners,
                                                         const uint8_t* __restrict__ old_owners, T* u, T* v, T* w,
                                                         const float* __restrict__ wu, const float* __restrict__ wv,
                                                         const float* __restrict__ ww) {
    const int nz1 = d.nz + 1;
    const int zz = blockIdx.z;
    const int axis = zz >= 2 * nz1 ? 2 : (zz >= nz1 ? 1 : 0);
    const int z = zz - axis * nz1;
    const int sx = d.nx + (axis == 0), sy = d.ny + (axis == 1), sz = d.nz + (axis == 2);
    const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
    if (x >= sx || y >= sy || z >= sz) return;
    const int c[3] = {x, y, z}, n[3] = {sx, sy, sz};
    const int i = x + sx * (y + sy * z);
    T* f = axis == 0 ? u : (axis == 1 ? v : w);
    const float* wall = axis == 0 ? wu : (axis == 1 ? wv : ww);
    float value = 0.f;
    if (c[axis] > 0 && c[axis] < n[axis] - 1) {
        const int hi = cidx(d, x, y, z), lo = cidx(d, x - (axis == 0), y - (axis == 1), z - (axis == 2));
        const bool blocked = __ldg(owners + hi) || __ldg(owners + lo);
        const bool before = __ldg(old_owners + hi) || __ldg(old_owners + lo);
        value = blocked ? __ldg(wall + i) : (before ? 0.f : Store<T>::ld(f, i));
    }
    Store<T>::st(f, i, value);
}

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" {

int ffx_curl(const FfxGrid* g, int storage, const void* u, const void* v, const void* w, float* curl4,
             void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && u && v && w && curl4 && ((uintptr_t)curl4 & 15) == 0,
                "ffx_curl: invalid arguments (16-byte aligned float4 output)");
    Dev d = make_dev(*g);
    cudaStream_t st = as_stream(stream);
    FFX_DISPATCH_STORAGE(storage, T, {
        curl_kernel<T><<<cell_grid(d.nx, d.ny, d.nz), cell_block(), 0, st>>>(
            d, Faces<T>{(const T*)u, (const T*)v, (const T*)w}, reinterpret_cast<float4*>(curl4));
    });
    return launch_status("curl_kernel");
}

int ffx_confine(const FfxGrid* g, int storage, const float* curl4, const void* u, const void* v, const void* w,
                float dt, float strength, float limit, void* ou, void* ov, void* ow, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && curl4 && ((uintptr_t)curl4 & 15) == 0 && u && v && w && ou &&
                    ov && ow && ou != u && ov != v && ow != w,
                "ffx_confine: invalid arguments (outputs must not alias inputs)");
    Dev d = make_dev(*g);
    cudaStream_t st = as_stream(stream);
    FFX_DISPATCH_STORAGE(storage, T, {
        confine_kernel<T><<<face_grid(d.nx, d.ny, d.nz), cell_block(), 0, st>>>(
            d, reinterpret_cast<const float4*>(curl4), Faces<T>{(const T*)u, (const T*)v, (const T*)w}, dt,
            strength, limit, (T*)ou, (T*)ov, (T*)ow);
    });
    return launch_status("confine_kernel");
}

int ffx_combustion(const FfxGrid* g, int storage, const void* fuel, const void* temperature, const void* density,
                   float dt, float ignition, float burn_rate, float smoke_yield, float heat_yield, float* flame,
                   void* fuel_out, void* density_out, void* temperature_out, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && fuel && temperature && density && flame && fuel_out &&
                    density_out && temperature_out && dt > 0.f,
                "ffx_combustion: invalid arguments");
    const int64_t n = (int64_t)g->nx * g->ny * g->nz;
    cudaStream_t st = as_stream(stream);
    FFX_DISPATCH_STORAGE(storage, T, {
        combustion_kernel<T><<<blocks_for(n, 256), 256, 0, st>>>(
            n, (const T*)fuel, (const T*)temperature, (const T*)density, dt, ignition, burn_rate, smoke_yield,
            heat_yield, flame, (T*)fuel_out, (T*)density_out, (T*)temperature_out);
    });
    return launch_status("combustion_kernel");
}

int ffx_moving_mask(const FfxGrid* g, int count, const float* rows12, const int32_t* is_box, uint8_t* owners,
                    void* stream) {
    FFX_REQUIRE(grid_ok(g) && count >= 0 && count <= FFX_MOVING_MAX && (count == 0 || (rows12 && is_box)) && owners,
                "ffx_moving_mask: invalid arguments (at most %d colliders)", FFX_MOVING_MAX);
    MovingColliders C;
    C.count = count;
    for (int k = 0; k < count; ++k) {
        for (int j = 0; j < 12; ++j) C.rows[k][j] = rows12[12 * k + j];
        C.box[k] = is_box[k] != 0;
    }
    Dev d = make_dev(*g);
    moving_mask_kernel<<<cell_grid(d.nx, d.ny, d.nz), cell_block(), 0, as_stream(stream)>>>(d, C, owners);
    return launch_status("moving_mask_kernel");
}

int ffx_moving_walls(const FfxGrid* g, const uint8_t* owners, int count, const float* table, float* wu, float* wv,
                     float* ww, void* stream) {
    FFX_REQUIRE(grid_ok(g) && owners && count >= 0 && count <= FFX_MOVING_MAX && (count == 0 || table) && wu && wv &&
                    ww,
                "ffx_moving_walls: invalid arguments");
    WallTable W = {};
    for (int k = 0; k < count; ++k)
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 4; ++j) W.rows[k][a][j] = table[12 * k + 4 * a + j];
    Dev d = make_dev(*g);
    moving_wall_kernel<<<face_grid(d.nx, d.ny, d.nz), cell_block(), 0, as_stream(stream)>>>(d, owners, W, wu, wv,
                                                                                           ww);
    return launch_status("moving_wall_kernel");
}

int ffx_moving_remap(const FfxGrid* g, int storage, const uint8_t* owners, const uint8_t* old_owners, void* scalar0,
                     void* scalar1, void* scalar2, void* u, void* v, void* w, const float* wu, const float* wv,
                     const float* ww, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && owners && old_owners && scalar0 && u && v && w && wu && wv &&
                    ww,
                "ffx_moving_remap: invalid arguments");
    Dev d = make_dev(*g);
    const int64_t n = (int64_t)g->nx * g->ny * g->nz;
    cudaStream_t st = as_stream(stream);
    FFX_DISPATCH_STORAGE(storage, T, {
        remap_scalars_kernel<T><<<blocks_for(n, 256), 256, 0, st>>>(n, owners, old_owners, (T*)scalar0,
                                                                     (T*)scalar1, (T*)scalar2);
        int e = launch_status("remap_scalars_kernel");
        if (e) return e;
        remap_faces_kernel<T><<<face_grid(d.nx, d.ny, d.nz), cell_block(), 0, st>>>(d, owners, old_owners, (T*)u,
                                                                                   (T*)v, (T*)w, wu, wv, ww);
    });
    return launch_status("remap_faces_kernel");
}

}  // extern "C"
