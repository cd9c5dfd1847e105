// Projection kernels: walls, divergence, gradient (fused cell-centric passes),
// Jacobi, geometric multigrid operators, aggregation multigrid operators and
// the FP64 direct coarse solve.
//
// The fused cell-centric passes give each thread one cell: it evaluates the
// six faces of that cell, writes its three lower faces (and the upper face on
// the far domain boundary), and forms the divergence from the six values, so
// a face pass and the divergence that reads its result are one kernel and
// one read of every face.
//
// All stencil kernels use the 32 x 8 (x, y) block / z-per-blockIdx.z launch of
// ffx_common.cuh; reductions stride over z with a bounded number of blocks so
// each block issues one atomic.
#include "ffx_host.cuh"
#include "ffx_batch.cuh"
#include "ffx_level0.cuh"

namespace ffx {
namespace {

// Value after a round trip through storage type T.
template <typename T>
__device__ __forceinline__ float rt(float v);
template <>
__device__ __forceinline__ float rt<float>(float v) { return v; }
template <>
__device__ __forceinline__ float rt<__nv_bfloat16>(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// Bounded z extent of reduction grids: (x, y) tiles x this many z blocks.
inline unsigned reduce_z(int nz) { return (unsigned)(nz < 8 ? nz : 8); }

// ------------------------------------------------------ walls + divergence
// pressure_walls.glsl + pressure_divergence.glsl (DIV = false: walls only).
template <typename T, bool MASK, bool DIV>
__global__ void __launch_bounds__(256) walls_div_kernel(Dev d, const uint8_t* __restrict__ solid, Walls W,
                                                       Faces<T> F, T* ou, T* ov, T* ow, float* div) {
    int x, y, z;
    if (!cell_coords(d.nx, d.ny, x, y, z)) return;
    const int i = cidx(d, x, y, z);
    const int iu = x + (d.nx + 1) * (y + d.ny * z);
    const int iv = x + d.nx * (y + (d.ny + 1) * z);
    const int iw = i;
    const int sv = d.nx, sw = d.nx * d.ny;
    auto bounded = [&](const T* f, int idx, int c, int nf, int fx, int fy, int fz, int axis) -> float {
        bool wall = c == 0 || c == nf - 1;
        if (MASK) wall = wall || solid_face(d, solid, fx, fy, fz, axis);
        return wall ? wall_value(W, axis, idx) : Store<T>::ld(f, idx);
    };
    float ul = bounded(F.u, iu, x, d.nx + 1, x, y, z, 0);
    float vl = bounded(F.v, iv, y, d.ny + 1, x, y, z, 1);
    float wl = bounded(F.w, iw, z, d.nz + 1, x, y, z, 2);
    Store<T>::st(ou, iu, ul);
    Store<T>::st(ov, iv, vl);
    Store<T>::st(ow, iw, wl);
    float uu = 0.f, vu = 0.f, wu = 0.f;
    if (DIV || x == d.nx - 1) uu = bounded(F.u, iu + 1, x + 1, d.nx + 1, x + 1, y, z, 0);
    if (DIV || y == d.ny - 1) vu = bounded(F.v, iv + sv, y + 1, d.ny + 1, x, y + 1, z, 1);
    if (DIV || z == d.nz - 1) wu = bounded(F.w, iw + sw, z + 1, d.nz + 1, x, y, z + 1, 2);
    if (x == d.nx - 1) Store<T>::st(ou, iu + 1, uu);
    if (y == d.ny - 1) Store<T>::st(ov, iv + sv, vu);
    if (z == d.nz - 1) Store<T>::st(ow, iw + sw, wu);
    if (DIV) {
        float dv = (uu - ul) * d.inv[0] + (vu - vl) * d.inv[1] + (wu - wl) * d.inv[2];
        if (MASK && __ldg(solid + i)) dv = 0.f;
        div[i] = dv;
    }
}

// Plain divergence of stored faces (pressure_divergence.glsl).
template <typename T>
struct DivDesc {
    Dev d;
    const uint8_t* solid;
    Faces<T> F;
    float* div;
};

template <typename T, bool MASK>
__device__ __forceinline__ void divergence_body(const DivDesc<T>& P, const Blk& b) {
    const Dev& d = P.d;
    const uint8_t* __restrict__ solid = P.solid;
    const Faces<T>& F = P.F;
    float* div = P.div;
    int x, y, z;
    if (!cell_coords(b, d.nx, d.ny, x, y, z)) return;
    const int i = cidx(d, x, y, z);
    if (MASK && __ldg(solid + i)) { div[i] = 0.f; return; }
    const int iu = x + (d.nx + 1) * (y + d.ny * z);
    const int iv = x + d.nx * (y + (d.ny + 1) * z);
    const int sz = d.nx * d.ny;
    div[i] = (Store<T>::ld(F.u, iu + 1) - Store<T>::ld(F.u, iu)) * d.inv[0] +
             (Store<T>::ld(F.v, iv + d.nx) - Store<T>::ld(F.v, iv)) * d.inv[1] +
             (Store<T>::ld(F.w, i + sz) - Store<T>::ld(F.w, i)) * d.inv[2];
}

template <typename T, bool MASK>
__global__ void __launch_bounds__(256) divergence_kernel(Dev d, const uint8_t* __restrict__ solid, Faces<T> F,
                                                        float* div) {
    divergence_body<T, MASK>(DivDesc<T>{d, solid, F, div}, hw_blk());
}

// ------------------------------------------------- gradient + divergence
template <typename T>
struct GradDesc {
    Dev d;
    const uint8_t* solid;
    Walls W;
    Faces<T> F;
    const float* p;
    float dt;
    T* out[3];
    float* div;
    const uint8_t* links;   // optional level-0 link bytes of the same mask (ffx_graph_links), MASK only
    float* div_exact;       // optional: divergence of the corrected faces before rounding to storage
};

template <typename T, bool MASK>
__device__ __forceinline__ void gradient_body(const GradDesc<T>& P, const Blk& b, float* maxima) {
    const Dev& d = P.d;
    const uint8_t* __restrict__ solid = P.solid;
    const Walls& W = P.W;
    const Faces<T>& F = P.F;
    const float* __restrict__ p = P.p;
    const float dt = P.dt;
    T* ou = P.out[0];
    T* ov = P.out[1];
    T* ow = P.out[2];
    float* div = P.div;
    int x, y, z;
    float mx[3] = {0.f, 0.f, 0.f};
    if (cell_coords(b, d.nx, d.ny, x, y, z)) {
        const int i = cidx(d, x, y, z);
        const int iu = x + (d.nx + 1) * (y + d.ny * z);
        const int iv = x + d.nx * (y + (d.ny + 1) * z);
        const int iw = i;
        const int sy = d.nx, sz = d.nx * d.ny;
        float pc = __ldg(p + i);
        // With the link byte of the cell, bit 2a (2a + 1) says whether the face to the lower
        // (upper) neighbour along axis a joins two fluid cells inside the domain -- exactly the
        // test below (interior face, neither adjacent cell solid) -- and bit 6 that the cell is fluid.
        const unsigned lk = (MASK && P.links) ? (unsigned)__ldg(P.links + i) : 0u;
        // face between cells (face - e_axis) and (face); phi / plo are their pressures;
        // bit: the face's link bit in this cell's byte
        auto face_out = [&](const T* f, int idx, int c, int nf, int fx, int fy, int fz, int axis, float phi,
                            float plo, unsigned bit) -> float {
            bool open;
            if (MASK && P.links) {
                open = (lk & bit) != 0u;
            } else {
                open = c > 0 && c < nf - 1;
                if (MASK) open = open && !solid_face(d, solid, fx, fy, fz, axis);
            }
            if (!open) return wall_value(W, axis, idx);
            float gr = (phi - plo) * d.inv[axis];
            return Store<T>::ld(f, idx) - dt * gr;
        };
        float p_xm = x > 0 ? __ldg(p + i - 1) : 0.f, p_xp = x + 1 < d.nx ? __ldg(p + i + 1) : 0.f;
        float p_ym = y > 0 ? __ldg(p + i - sy) : 0.f, p_yp = y + 1 < d.ny ? __ldg(p + i + sy) : 0.f;
        float p_zm = z > 0 ? __ldg(p + i - sz) : 0.f, p_zp = z + 1 < d.nz ? __ldg(p + i + sz) : 0.f;
        const float ul0 = face_out(F.u, iu, x, d.nx + 1, x, y, z, 0, pc, p_xm, 1u);
        const float vl0 = face_out(F.v, iv, y, d.ny + 1, x, y, z, 1, pc, p_ym, 4u);
        const float wl0 = face_out(F.w, iw, z, d.nz + 1, x, y, z, 2, pc, p_zm, 16u);
        const float uu0 = face_out(F.u, iu + 1, x + 1, d.nx + 1, x + 1, y, z, 0, p_xp, pc, 2u);
        const float vu0 = face_out(F.v, iv + d.nx, y + 1, d.ny + 1, x, y + 1, z, 1, p_yp, pc, 8u);
        const float wu0 = face_out(F.w, iw + sz, z + 1, d.nz + 1, x, y, z + 1, 2, p_zp, pc, 32u);
        float ul = rt<T>(ul0), vl = rt<T>(vl0), wl = rt<T>(wl0);
        float uu = rt<T>(uu0), vu = rt<T>(vu0), wu = rt<T>(wu0);
        Store<T>::st(ou, iu, ul);
        Store<T>::st(ov, iv, vl);
        Store<T>::st(ow, iw, wl);
        mx[0] = finite_abs(ul); mx[1] = finite_abs(vl); mx[2] = finite_abs(wl);
        if (x == d.nx - 1) { Store<T>::st(ou, iu + 1, uu); mx[0] = fmaxf(mx[0], finite_abs(uu)); }
        if (y == d.ny - 1) { Store<T>::st(ov, iv + d.nx, vu); mx[1] = fmaxf(mx[1], finite_abs(vu)); }
        if (z == d.nz - 1) { Store<T>::st(ow, iw + sz, wu); mx[2] = fmaxf(mx[2], finite_abs(wu)); }
        if (div) {
            float dv = (uu - ul) * d.inv[0] + (vu - vl) * d.inv[1] + (wu - wl) * d.inv[2];
            if (MASK && (P.links ? (lk & 64u) == 0u : __ldg(solid + i) != 0)) dv = 0.f;
            div[i] = dv;
        }
        if (P.div_exact) {
            // the projection's own result, before the storage rounding (BF16 storage rounds the faces)
            float dv = (uu0 - ul0) * d.inv[0] + (vu0 - vl0) * d.inv[1] + (wu0 - wl0) * d.inv[2];
            if (MASK && (P.links ? (lk & 64u) == 0u : __ldg(solid + i) != 0)) dv = 0.f;
            P.div_exact[i] = dv;
        }
    }
    if (maxima) {
        block_max_to_n<3>(maxima, mx, 3);
        __syncthreads();
    }
}

template <typename T, bool MASK>
__global__ void __launch_bounds__(256) gradient_kernel(Dev d, const uint8_t* __restrict__ solid, Walls W,
                                                      Faces<T> F, const float* __restrict__ p, float dt, T* ou,
                                                      T* ov, T* ow, float* div, float* maxima,
                                                      const uint8_t* __restrict__ links, float* div_exact) {
    gradient_body<T, MASK>(GradDesc<T>{d, solid, W, F, p, dt, {ou, ov, ow}, div, links, div_exact}, hw_blk(),
                           maxima);
}

// ---------------------------------------------------------------- Jacobi
struct Lvl {
    int nx, ny, nz;
    float w[3];   // inv*inv per axis (the FP32 product pressure_jacobi.glsl forms)
};

inline Lvl make_lvl(const int32_t n[3], const float inv[3]) {
    Lvl L;
    L.nx = n[0]; L.ny = n[1]; L.nz = n[2];
    for (int a = 0; a < 3; ++a) L.w[a] = inv[a] * inv[a];
    return L;
}

// pressure_jacobi.glsl:1-34
template <bool MASK>
__global__ void __launch_bounds__(256) jacobi_kernel(Lvl L, const uint8_t* __restrict__ solid,
                                                    const float* __restrict__ p, const float* __restrict__ rhs,
                                                    float dt, float omega, float* out) {
    int x, y, z;
    if (!cell_coords(L.nx, L.ny, x, y, z)) return;
    const int i = x + L.nx * (y + L.ny * z);
    if (MASK && __ldg(solid + i)) { out[i] = 0.f; return; }
    const int c[3] = {x, y, z}, size[3] = {L.nx, L.ny, L.nz};
    const int stride[3] = {1, L.nx, L.nx * L.ny};
    float nb = 0.f, diag = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float w = L.w[a];
        bool lower = c[a] > 0, upper = c[a] + 1 < size[a];
        if (MASK) {
            lower = lower && !__ldg(solid + i - stride[a]);
            upper = upper && !__ldg(solid + i + stride[a]);
        }
        if (lower) { nb = nb + w * __ldg(p + i - stride[a]); diag = diag + w; }
        if (upper) { nb = nb + w * __ldg(p + i + stride[a]); diag = diag + w; }
    }
    if (diag == 0.f) { out[i] = 0.f; return; }
    float cand = (nb - __ldg(rhs + i) / dt) / diag;
    float old = __ldg(p + i);
    out[i] = old * (1.f - omega) + cand * omega;
}

__global__ void scale_kernel(int64_t n, const float* in, float f, float* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i] * f;
}

__global__ void add_kernel(int64_t n, const float* a, const float* b, float* out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] + b[i];
}

// ---------------------------------------------------- geometric multigrid
// Laplacian term of mg_residual.glsl at cell (x, y, z), index i.
__device__ __forceinline__ float neumann_lap(const Lvl& L, const float* __restrict__ p, int i, int x, int y, int z) {
    float c = __ldg(p + i);
    float lap = 0.f;
    const int cc[3] = {x, y, z}, size[3] = {L.nx, L.ny, L.nz};
    const int stride[3] = {1, L.nx, L.nx * L.ny};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float w = L.w[a];
        if (cc[a] > 0) lap = lap + w * (__ldg(p + i - stride[a]) - c);
        if (cc[a] + 1 < size[a]) lap = lap + w * (__ldg(p + i + stride[a]) - c);
    }
    return lap;
}

__global__ void __launch_bounds__(256) mg_residual_kernel(Lvl L, const float* __restrict__ p,
                                                         const float* __restrict__ rhs, float dt, float* r) {
    int x, y, z;
    if (!cell_coords(L.nx, L.ny, x, y, z)) return;
    const int i = x + L.nx * (y + L.ny * z);
    r[i] = __ldg(rhs + i) / dt - neumann_lap(L, p, i, x, y, z);
}

__global__ void __launch_bounds__(256) mg_residual_max_kernel(Lvl L, const float* __restrict__ p,
                                                             const float* __restrict__ rhs, float dt, float* out) {
    int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
    float m = 0.f;
    if (x < L.nx && y < L.ny)
        for (int z = blockIdx.z; z < L.nz; z += gridDim.z) {
            const int i = x + L.nx * (y + L.ny * z);
            m = fmaxf(m, finite_abs(__ldg(rhs + i) / dt - neumann_lap(L, p, i, x, y, z)));
        }
    block_max_to(out, m);
}

// mg_restrict.glsl: coarse cell c averages fine cells 2c + {0,1}^3 (z, y, x order).
__global__ void __launch_bounds__(256) mg_restrict_kernel(int fx, int fy, int fz, const float* __restrict__ f,
                                                         float* c) {
    const int cx = fx / 2, cy = fy / 2;
    int x, y, z;
    if (!cell_coords(cx, cy, x, y, z)) return;
    float v = 0.f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) v = v + __ldg(f + (2 * x + dx) + fx * ((2 * y + dy) + fy * (2 * z + dz)));
    c[x + cx * (y + cy * z)] = v / 8.0f;
}

__global__ void __launch_bounds__(256) mg_residual_restrict_kernel(Lvl L, const float* __restrict__ p,
                                                                  const float* __restrict__ rhs, float dt, float* c) {
    const int cx = L.nx / 2, cy = L.ny / 2;
    int x, y, z;
    if (!cell_coords(cx, cy, x, y, z)) return;
    float v = 0.f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
                const int fi = X + L.nx * (Y + L.ny * Z);
                v = v + (__ldg(rhs + fi) / dt - neumann_lap(L, p, fi, X, Y, Z));
            }
    c[x + cx * (y + cy * z)] = v / 8.0f;
}

// mg_prolong.glsl: cell-centred trilinear interpolation, clamped at the edges.
__global__ void __launch_bounds__(256) mg_prolong_kernel(int nx, int ny, int nz, const float* __restrict__ p,
                                                        const float* __restrict__ coarse, float* out) {
    int c[3];
    if (!cell_coords(nx, ny, c[0], c[1], c[2])) return;
    const int cs[3] = {nx / 2, ny / 2, nz / 2};
    int b[3];
    float fr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float q = ((float)c[a] + 0.5f) * 0.5f - 0.5f;
        float fb = floorf(q);
        fr[a] = q - fb;
        b[a] = (int)fb;
    }
    float v = 0.f;
#pragma unroll
    for (int oz = 0; oz < 2; ++oz) {
        float wz = oz ? fr[2] : 1.f - fr[2];
        int iz = min(max(b[2] + oz, 0), cs[2] - 1);
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
            float wy = oy ? fr[1] : 1.f - fr[1];
            int iy = min(max(b[1] + oy, 0), cs[1] - 1);
#pragma unroll
            for (int ox = 0; ox < 2; ++ox) {
                float wx = ox ? fr[0] : 1.f - fr[0];
                int ix = min(max(b[0] + ox, 0), cs[0] - 1);
                v = v + wx * wy * wz * __ldg(coarse + ix + cs[0] * (iy + cs[1] * iz));
            }
        }
    }
    const int i = c[0] + nx * (c[1] + ny * c[2]);
    out[i] = __ldg(p + i) + v;
}

// Dense FP64 mat-vec, one warp per row (coarse_pressure.glsl, solid_mg_direct.glsl).
__global__ void direct_kernel(int n, const double* __restrict__ inv, const float* __restrict__ rhs, float dt,
                              float* p) {
    pdl_enter();
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double* row = inv + (int64_t)warp * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += row[j] * (double)rhs[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) p[warp] = (float)(s / (double)dt);
}

// ------------------------------------------------- aggregation multigrid
struct GLvl {
    int nx, ny, nz;
    const float4* edges;     // NULL: derive from the mask
    const uint8_t* solid;
    float w[3];
    float cs;                // coarse-correction factor of the prolongation into this level (1: plain)
};

inline GLvl make_glvl(const FfxGraphLevel* lv) {
    GLvl g;
    g.nx = lv->nx; g.ny = lv->ny; g.nz = lv->nz;
    g.edges = reinterpret_cast<const float4*>(lv->edges);
    g.solid = lv->solid;
    for (int a = 0; a < 3; ++a) g.w[a] = lv->w[a];
    g.cs = lv->coarse_scale != 0.f ? lv->coarse_scale : 1.f;
    return g;
}

__device__ __forceinline__ bool g_fluid(const GLvl& g, int i) { return __ldg(g.solid + i) == 0; }
__device__ __forceinline__ float comp4(const float4& e, int a) { return a == 0 ? e.x : (a == 1 ? e.y : e.z); }

// Record (+x, +y, +z, active) of cell i = (x, y, z)  (solid_hierarchy.py:16-25 for level 0).
__device__ __forceinline__ float4 g_edge(const GLvl& g, int i, int x, int y, int z) {
    if (g.edges) return __ldg(g.edges + i);
    float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!g_fluid(g, i)) return e;
    e.w = 1.f;
    if (x + 1 < g.nx && g_fluid(g, i + 1)) e.x = g.w[0];
    if (y + 1 < g.ny && g_fluid(g, i + g.nx)) e.y = g.w[1];
    if (z + 1 < g.nz && g_fluid(g, i + g.nx * g.ny)) e.z = g.w[2];
    return e;
}

// solid_mg_operator.glsl: diagonal and neighbour sums. `pv(j, x, y, z)` supplies
// the iterate at cell j. Level 0 (no records) reads each mask byte once.
template <typename PV>
__device__ __forceinline__ void graph_terms(const GLvl& g, int i, int x, int y, int z, PV pv, float& diag,
                                            float& nb) {
    diag = 0.f;
    nb = 0.f;
    const int c[3] = {x, y, z}, size[3] = {g.nx, g.ny, g.nz};
    const int stride[3] = {1, g.nx, g.nx * g.ny};
    if (g.edges) {
        const float4 here = __ldg(g.edges + i);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (c[a] > 0) {
                int lc[3] = {x, y, z};
                lc[a] -= 1;
                float w = comp4(__ldg(g.edges + i - stride[a]), a);
                diag = diag + w;
                nb = nb + w * pv(i - stride[a], lc[0], lc[1], lc[2]);
            }
            if (c[a] + 1 < size[a]) {
                int uc[3] = {x, y, z};
                uc[a] += 1;
                float w = comp4(here, a);
                diag = diag + w;
                nb = nb + w * pv(i + stride[a], uc[0], uc[1], uc[2]);
            }
        }
        return;
    }
    const bool fluid = g_fluid(g, i);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (c[a] > 0) {
            int lc[3] = {x, y, z};
            lc[a] -= 1;
            float w = (fluid && g_fluid(g, i - stride[a])) ? g.w[a] : 0.f;
            diag = diag + w;
            nb = nb + w * pv(i - stride[a], lc[0], lc[1], lc[2]);
        }
        if (c[a] + 1 < size[a]) {
            int uc[3] = {x, y, z};
            uc[a] += 1;
            float w = (fluid && g_fluid(g, i + stride[a])) ? g.w[a] : 0.f;
            diag = diag + w;
            nb = nb + w * pv(i + stride[a], uc[0], uc[1], uc[2]);
        }
    }
}

__device__ __forceinline__ void graph_smooth_body(const GLvl& g, const float* __restrict__ p,
                                                  const float* __restrict__ rhs, float omega, float* out,
                                                  const Blk& b) {
    int x, y, z;
    if (!cell_coords(b, g.nx, g.ny, x, y, z)) return;
    const int i = x + g.nx * (y + g.ny * z);
    float diag, nb;
    graph_terms(g, i, x, y, z, [&](int j, int, int, int) { return __ldg(p + j); }, diag, nb);
    out[i] = diag > 0.f ? __ldg(p + i) * (1.f - omega) + ((nb - __ldg(rhs + i)) / diag) * omega : 0.f;
}

__global__ void __launch_bounds__(256) graph_smooth_kernel(GLvl g, const float* __restrict__ p,
                                                          const float* __restrict__ rhs, float omega, float* out) {
    pdl_enter();
    graph_smooth_body(g, p, rhs, omega, out, hw_blk());
}

// Level-0 (mask-derived) sweep, streamed along z: each thread owns one (x, y)
// column of kZ cells and carries p and the fluid flag of the z-1 / z / z+1
// cells in registers, so every cell loads p and the mask once for its own z
// neighbours; x/y neighbours come from the L1 lines its warp-mates load. The
// operator terms are summed in the same order as graph_terms.
constexpr int kZ = 8;
static_assert(kZ == kBatchZ0, "batched level-0 sweeps tile z like the single-domain ones");
__device__ __forceinline__ void graph_smooth_level0_body(const GLvl& g, const float* __restrict__ p,
                                                         const float* __restrict__ rhs, float omega, float* out,
                                                         const Blk& b) {
    const int x = b.x * b.bw + b.ox, y = b.y * b.bh + b.oy;
    if (x >= g.nx || y >= g.ny) return;
    const int z0 = b.z * kZ;
    const int sy = g.nx, sz = g.nx * g.ny;
    int i = x + g.nx * (y + g.ny * z0);
    const float wx = g.w[0], wy = g.w[1], wz = g.w[2];
    float p_lo = 0.f, p_c = __ldg(p + i);
    bool f_lo = false, f_c = __ldg(g.solid + i) == 0;
    if (z0 > 0) {
        p_lo = __ldg(p + i - sz);
        f_lo = __ldg(g.solid + i - sz) == 0;
    }
    const int zend = min(z0 + kZ, g.nz);
    for (int z = z0; z < zend; ++z, i += sz) {
        const bool up = z + 1 < g.nz;
        const float p_hi = up ? __ldg(p + i + sz) : 0.f;
        const bool f_hi = up && __ldg(g.solid + i + sz) == 0;
        float diag = 0.f, nb = 0.f;
        if (x > 0) {
            const float w = (f_c && __ldg(g.solid + i - 1) == 0) ? wx : 0.f;
            diag = diag + w;
            nb = nb + w * __ldg(p + i - 1);
        }
        if (x + 1 < g.nx) {
            const float w = (f_c && __ldg(g.solid + i + 1) == 0) ? wx : 0.f;
            diag = diag + w;
            nb = nb + w * __ldg(p + i + 1);
        }
        if (y > 0) {
            const float w = (f_c && __ldg(g.solid + i - sy) == 0) ? wy : 0.f;
            diag = diag + w;
            nb = nb + w * __ldg(p + i - sy);
        }
        if (y + 1 < g.ny) {
            const float w = (f_c && __ldg(g.solid + i + sy) == 0) ? wy : 0.f;
            diag = diag + w;
            nb = nb + w * __ldg(p + i + sy);
        }
        if (z > 0) {
            const float w = (f_c && f_lo) ? wz : 0.f;
            diag = diag + w;
            nb = nb + w * p_lo;
        }
        if (up) {
            const float w = (f_c && f_hi) ? wz : 0.f;
            diag = diag + w;
            nb = nb + w * p_hi;
        }
        out[i] = diag > 0.f ? p_c * (1.f - omega) + ((nb - __ldg(rhs + i)) / diag) * omega : 0.f;
        p_lo = p_c; p_c = p_hi;
        f_lo = f_c; f_c = f_hi;
    }
}

__global__ void __launch_bounds__(256) graph_smooth_level0_kernel(GLvl g, const float* __restrict__ p,
                                                                 const float* __restrict__ rhs, float omega,
                                                                 float* out) {
    pdl_enter();
    graph_smooth_level0_body(g, p, rhs, omega, out, hw_blk());
}

__device__ __forceinline__ float graph_res(const GLvl& g, const float* __restrict__ p, const float* __restrict__ rhs,
                                           int i, int x, int y, int z) {
    float diag, nb;
    graph_terms(g, i, x, y, z, [&](int j, int, int, int) { return __ldg(p + j); }, diag, nb);
    return diag > 0.f ? (__ldg(rhs + i) - nb) + diag * __ldg(p + i) : 0.f;
}

__global__ void __launch_bounds__(256) graph_residual_kernel(GLvl g, const float* __restrict__ p,
                                                            const float* __restrict__ rhs, float* r) {
    int x, y, z;
    if (!cell_coords(g.nx, g.ny, x, y, z)) return;
    const int i = x + g.nx * (y + g.ny * z);
    r[i] = graph_res(g, p, rhs, i, x, y, z);
}

__device__ __forceinline__ void graph_residual_max_body(const GLvl& g, const float* __restrict__ p,
                                                        const float* __restrict__ rhs, float* out, const Blk& b) {
    int x = b.x * b.bw + b.ox, y = b.y * b.bh + b.oy;
    float m = 0.f;
    if (x < g.nx && y < g.ny)
        for (int z = b.z; z < g.nz; z += b.gz) {
            const int i = x + g.nx * (y + g.ny * z);
            m = fmaxf(m, finite_abs(graph_res(g, p, rhs, i, x, y, z)));
        }
    block_max_to(out, m);
}

__global__ void __launch_bounds__(256) graph_residual_max_kernel(GLvl g, const float* __restrict__ p,
                                                                const float* __restrict__ rhs, float* out) {
    pdl_enter();
    graph_residual_max_body(g, p, rhs, out, hw_blk());
}

__device__ __forceinline__ void graph_residual_restrict_body(const GLvl& g, const float* __restrict__ p,
                                                             const float* __restrict__ rhs, float* c,
                                                             float* zero, const Blk& b) {
    const int cx = g.nx / 2, cy = g.ny / 2;
    int x, y, z;
    if (!cell_coords(b, cx, cy, x, y, z)) return;
    float v = 0.f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
                v = v + graph_res(g, p, rhs, X + g.nx * (Y + g.ny * Z), X, Y, Z);
            }
    c[x + cx * (y + cy * z)] = v / 8.0f;
    if (zero) zero[x + cx * (y + cy * z)] = 0.f;
}

__global__ void __launch_bounds__(256) graph_residual_restrict_zero_kernel(GLvl g, const float* __restrict__ p,
                                                                          const float* __restrict__ rhs, float* c,
                                                                          float* zero) {
    pdl_enter();
    graph_residual_restrict_body(g, p, rhs, c, zero, hw_blk());
}

__device__ __forceinline__ bool g_active(const GLvl& g, int i) {
    return g.edges ? __ldg(g.edges + i).w > 0.f : g_fluid(g, i);
}

// solid_mg_prolong.glsl
__device__ __forceinline__ float prolonged(const GLvl& g, const float* __restrict__ p,
                                           const float* __restrict__ coarse, int i, int x, int y, int z) {
    if (!g_active(g, i)) return 0.f;
    const int cx = g.nx / 2, cy = g.ny / 2;
    return __ldg(p + i) + g.cs * __ldg(coarse + (x >> 1) + cx * ((y >> 1) + cy * (z >> 1)));
}

__global__ void __launch_bounds__(256) graph_prolong_kernel(GLvl g, const float* __restrict__ p,
                                                           const float* __restrict__ coarse, float* out) {
    int x, y, z;
    if (!cell_coords(g.nx, g.ny, x, y, z)) return;
    const int i = x + g.nx * (y + g.ny * z);
    out[i] = prolonged(g, p, coarse, i, x, y, z);
}

__device__ __forceinline__ void graph_prolong_smooth_body(const GLvl& g, const float* __restrict__ p,
                                                          const float* __restrict__ coarse,
                                                          const float* __restrict__ rhs, float omega, float* out,
                                                          const Blk& b) {
    int x, y, z;
    if (!cell_coords(b, g.nx, g.ny, x, y, z)) return;
    const int i = x + g.nx * (y + g.ny * z);
    float diag, nb;
    graph_terms(g, i, x, y, z,
                [&](int j, int jx, int jy, int jz) { return prolonged(g, p, coarse, j, jx, jy, jz); }, diag, nb);
    float pc = prolonged(g, p, coarse, i, x, y, z);
    out[i] = diag > 0.f ? pc * (1.f - omega) + ((nb - __ldg(rhs + i)) / diag) * omega : 0.f;
}

__global__ void __launch_bounds__(256) graph_prolong_smooth_kernel(GLvl g, const float* __restrict__ p,
                                                                  const float* __restrict__ coarse,
                                                                  const float* __restrict__ rhs, float omega,
                                                                  float* out) {
    pdl_enter();
    graph_prolong_smooth_body(g, p, coarse, rhs, omega, out, hw_blk());
}

// ------------------------------------------ coarse (edge-record) levels: residual + restriction
// graph_residual_restrict_zero_kernel's pass on levels with edge records,
// streamed along z (ffx_set_edge_streaming, on by default): every fine
// residual is formed by the same operations in graph_terms' order (x-, x+, y-,
// y+, z-, z+) and the eight are added in the restriction's order, so the
// coarse fields are bit-identical. Measured at 256^3 (levels 128^3 .. 8^3):
// 18.2 -> 14.4 us on 128^3 and 6.2 -> 4.6-5.1 us on the small levels. The
// same streaming of the sweep and of prolongation + sweep (x neighbours by
// shuffle, the slice below carried) was slower than one cell per thread
// (15.2 against 13.7 us on 128^3; 6.2 against 4.5-5.2 us for the small
// prolongations): with eight slices per thread the level keeps too few threads
// in flight to hide L2 latency, so those passes keep their one-cell kernels.
int g_edge_streaming = 1;   // ffx_set_edge_streaming

__device__ __forceinline__ float edge_comp(const GLvl& g, int i, int c) {
    return __ldg(reinterpret_cast<const float*>(g.edges) + 4 * i + c);
}

// Residual + restriction: a thread owns one coarse column (its 2 x 2 fine
// cells per slice) and walks 2 * chunk fine slices, carrying the iterate and z
// edge weights of the fine slice below. Each fine slice's four residuals are
// formed as graph_res forms them and added in the restriction's order
// (dz, dy, dx).
__device__ __forceinline__ void graph_residual_restrict_edges_body(const GLvl& g, const float* __restrict__ p,
                                                                   const float* __restrict__ rhs, float* c,
                                                                   float* zero, int chunk, const Blk& b) {
    const int cx = g.nx / 2, cy = g.ny / 2, cz = g.nz / 2;
    const int X = b.x * b.bw + b.ox, Y = b.y * b.bh + b.oy;
    if (X >= cx || Y >= cy) return;
    const int Z0 = b.z * chunk, Zend = min(Z0 + chunk, cz);
    const int sy = g.nx, sz = g.nx * g.ny;
    const int x0 = 2 * X, y0 = 2 * Y;
    // k = 2 * dy + dx indexes the four fine cells of a slice
    float p_lo[4], wz_lo[4], p_c[4];
    int base = x0 + g.nx * (y0 + g.ny * (2 * Z0));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j = base + (k & 1) + sy * (k >> 1);
        p_c[k] = __ldg(p + j);
        p_lo[k] = Z0 > 0 ? __ldg(p + j - sz) : 0.f;
        wz_lo[k] = Z0 > 0 ? edge_comp(g, j - sz, 2) : 0.f;
    }
    float v = 0.f;
    for (int fz = 2 * Z0; fz < 2 * Zend; ++fz, base += sz) {
        const bool up = fz + 1 < g.nz;
        float p_hi[4], res[4];
        float4 E[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int j = base + (k & 1) + sy * (k >> 1);
            E[k] = __ldg(g.edges + j);
            p_hi[k] = up ? __ldg(p + j + sz) : 0.f;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int dx = k & 1, dy = k >> 1;
            const int fx = x0 + dx, fy = y0 + dy;
            const int j = base + dx + sy * dy;
            const float4 here = E[k];
            float diag = 0.f, nb = 0.f;
            if (fx > 0) {
                const float w = dx ? E[k - 1].x : edge_comp(g, j - 1, 0);
                diag = diag + w;
                nb = nb + w * (dx ? p_c[k - 1] : __ldg(p + j - 1));
            }
            if (fx + 1 < g.nx) { diag = diag + here.x; nb = nb + here.x * (dx ? __ldg(p + j + 1) : p_c[k + 1]); }
            if (fy > 0) {
                const float w = dy ? E[k - 2].y : edge_comp(g, j - sy, 1);
                diag = diag + w;
                nb = nb + w * (dy ? p_c[k - 2] : __ldg(p + j - sy));
            }
            if (fy + 1 < g.ny) { diag = diag + here.y; nb = nb + here.y * (dy ? __ldg(p + j + sy) : p_c[k + 2]); }
            if (fz > 0) { diag = diag + wz_lo[k]; nb = nb + wz_lo[k] * p_lo[k]; }
            if (up) { diag = diag + here.z; nb = nb + here.z * p_hi[k]; }
            res[k] = diag > 0.f ? (__ldg(rhs + j) - nb) + diag * p_c[k] : 0.f;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) v = v + res[k];
        if (fz & 1) {
            const int ci = X + cx * (Y + cy * (fz >> 1));
            c[ci] = v / 8.0f;
            if (zero) zero[ci] = 0.f;
            v = 0.f;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            p_lo[k] = p_c[k];
            p_c[k] = p_hi[k];
            wz_lo[k] = E[k].z;
        }
    }
}

__global__ void __launch_bounds__(256) graph_residual_restrict_edges_kernel(GLvl g, const float* __restrict__ p,
                                                                           const float* __restrict__ rhs, float* c,
                                                                           float* zero, int chunk) {
    pdl_enter();
    graph_residual_restrict_edges_body(g, p, rhs, c, zero, chunk, hw_blk());
}

// Fine z slices per thread of the streamed restriction: long columns where the
// level has enough columns to fill the GPU, short ones on small levels.
inline int edge_chunk(int nx, int ny, int nz) { return (int64_t)nx * ny * nz >= (1 << 20) ? 8 : 2; }

// physics/solid_hierarchy.py:27-53 for one coarse cell.
__global__ void __launch_bounds__(256) graph_coarsen_kernel(GLvl g, float4* coarse, int* disconnected) {
    const int cx = g.nx / 2, cy = g.ny / 2;
    int x, y, z;
    if (!cell_coords(cx, cy, x, y, z)) return;
    float4 rec[8];
    unsigned active = 0;
    for (int j = 0; j < 8; ++j) {
        const int X = 2 * x + (j & 1), Y = 2 * y + ((j >> 1) & 1), Z = 2 * z + ((j >> 2) & 1);
        rec[j] = g_edge(g, X + g.nx * (Y + g.ny * Z), X, Y, Z);
        if (rec[j].w > 0.f) active |= 1u << j;
    }
    if (active) {
        unsigned seen = active & (~active + 1u);   // lowest active child
        for (int it = 0; it < 8; ++it) {
            unsigned grow = seen;
            for (int j = 0; j < 8; ++j) {
                if (!(seen >> j & 1u)) continue;
                for (int a = 0; a < 3; ++a) {
                    const int k = j ^ (1 << a);
                    const int lower = (j >> a & 1) ? k : j;
                    if ((active >> k & 1u) && comp4(rec[lower], a) > 0.f) grow |= 1u << k;
                }
            }
            if (grow == seen) break;
            seen = grow;
        }
        if (seen != active) atomicExch(disconnected, 1);
    }
    double s[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 8; ++j)
            if (j >> a & 1) s[a] += (double)comp4(rec[j], a);
    float4 out;
    out.x = (float)(s[0] / 8.0);
    out.y = (float)(s[1] / 8.0);
    out.z = (float)(s[2] / 8.0);
    out.w = active ? 1.f : 0.f;
    coarse[x + cx * (y + cy * z)] = out;
}

__global__ void __launch_bounds__(256) graph_level0_kernel(GLvl g, float4* out) {
    int x, y, z;
    if (!cell_coords(g.nx, g.ny, x, y, z)) return;
    const int i = x + g.nx * (y + g.ny * z);
    out[i] = g_edge(g, i, x, y, z);
}

// ------------------------------------------------ coarse tail of a V-cycle
// The small coarse levels (<= kTailCells cells each) of one V-cycle in a single
// 1024-thread block: every pass of solid_multigrid.py:46-65 on those levels
// (pre-smoothing, fused residual + restriction, the FP64 direct solve or the
// 80 masked sweeps on the coarsest level, fused prolongation + smoothing,
// post-smoothing), separated by __syncthreads instead of kernel launches. Each
// cell is evaluated with the same operations and order as the per-level
// kernels, and the direct solve sums its rows as direct_kernel does, so the
// results are bit-identical. Fields written inside the kernel are read with
// plain (coherent) loads, never the read-only path.
constexpr int kTailThreads = 1024;
constexpr int kTailCells = 32768;

struct TailLvl {
    GLvl g;
    float* p;
    float* q;
    float* rhs;
    int n;
};
struct TailArgs {
    int count, pre, post;
    float omega;
    const double* inverse;
    TailLvl lv[FFX_TAIL_LEVELS];
};

__device__ __forceinline__ void tail_xyz(const GLvl& g, int i, int& x, int& y, int& z) {
    x = i % g.nx;
    const int r = i / g.nx;
    y = r % g.ny;
    z = r / g.ny;
}

__device__ __forceinline__ void tail_smooth(const TailLvl& L, const float* p, float* out, float omega, bool zero) {
    const GLvl& g = L.g;
    for (int i = threadIdx.x; i < L.n; i += kTailThreads) {
        int x, y, z;
        tail_xyz(g, i, x, y, z);
        float diag, nb;
        graph_terms(g, i, x, y, z, [&](int j, int, int, int) { return zero ? 0.f : p[j]; }, diag, nb);
        const float pc = zero ? 0.f : p[i];
        out[i] = diag > 0.f ? pc * (1.f - omega) + ((nb - L.rhs[i]) / diag) * omega : 0.f;
    }
    __syncthreads();
}

__device__ __forceinline__ float tail_res(const TailLvl& L, const float* p, int i, int x, int y, int z) {
    float diag, nb;
    graph_terms(L.g, i, x, y, z, [&](int j, int, int, int) { return p[j]; }, diag, nb);
    return diag > 0.f ? (L.rhs[i] - nb) + diag * p[i] : 0.f;
}

__device__ __forceinline__ void graph_tail_body(const TailArgs& A) {
    float* cur[FFX_TAIL_LEVELS];
    float* spare[FFX_TAIL_LEVELS];
    for (int k = 0; k < A.count; ++k) {
        cur[k] = A.lv[k].p;
        spare[k] = A.lv[k].q;
    }
    const int last = A.count - 1;
    // down: zero iterate, pre-smoothing, residual restricted to the next level
    for (int k = 0; k < last; ++k) {
        const TailLvl& L = A.lv[k];
        for (int s = 0; s < A.pre; ++s) {
            tail_smooth(L, cur[k], spare[k], A.omega, s == 0);
            float* t = cur[k]; cur[k] = spare[k]; spare[k] = t;
        }
        if (A.pre == 0) {
            for (int i = threadIdx.x; i < L.n; i += kTailThreads) cur[k][i] = 0.f;
            __syncthreads();
        }
        const TailLvl& C = A.lv[k + 1];
        const GLvl& g = L.g;
        for (int c = threadIdx.x; c < C.n; c += kTailThreads) {
            int x, y, z;
            tail_xyz(C.g, c, x, y, z);
            float v = 0.f;
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx) {
                        const int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
                        v = v + tail_res(L, cur[k], X + g.nx * (Y + g.ny * Z), X, Y, Z);
                    }
            C.rhs[c] = v / 8.0f;
        }
        __syncthreads();
    }
    // coarsest level: FP64 pseudoinverse (direct_kernel's summation order) or 80 sweeps
    {
        const TailLvl& L = A.lv[last];
        if (A.inverse) {
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            for (int row = warp; row < L.n; row += kTailThreads / 32) {
                const double* r = A.inverse + (int64_t)row * L.n;
                double s = 0.0;
                for (int j = lane; j < L.n; j += 32) s += r[j] * (double)L.rhs[j];
                for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
                if (lane == 0) cur[last][row] = (float)(s / (double)1.0f);
            }
            __syncthreads();
        } else {
            for (int s = 0; s < 80; ++s) {
                tail_smooth(L, cur[last], spare[last], A.omega, s == 0);
                float* t = cur[last]; cur[last] = spare[last]; spare[last] = t;
            }
        }
    }
    // up: prolongation fused with the first post-sweep, then the other post-sweeps
    for (int k = last - 1; k >= 0; --k) {
        const TailLvl& L = A.lv[k];
        const GLvl& g = L.g;
        const float* p = cur[k];
        const float* coarse = cur[k + 1];
        const int cx = g.nx / 2, cy = g.ny / 2;
        auto pro = [&](int j, int jx, int jy, int jz) {
            return g_active(g, j) ? p[j] + g.cs * coarse[(jx >> 1) + cx * ((jy >> 1) + cy * (jz >> 1))] : 0.f;
        };
        for (int i = threadIdx.x; i < L.n; i += kTailThreads) {
            int x, y, z;
            tail_xyz(g, i, x, y, z);
            if (A.post > 0) {
                float diag, nb;
                graph_terms(g, i, x, y, z, pro, diag, nb);
                const float pc = pro(i, x, y, z);
                spare[k][i] = diag > 0.f ? pc * (1.f - A.omega) + ((nb - L.rhs[i]) / diag) * A.omega : 0.f;
            } else {
                spare[k][i] = pro(i, x, y, z);
            }
        }
        __syncthreads();
        float* t = cur[k]; cur[k] = spare[k]; spare[k] = t;
        for (int s = 1; s < A.post; ++s) {
            tail_smooth(L, cur[k], spare[k], A.omega, false);
            float* u = cur[k]; cur[k] = spare[k]; spare[k] = u;
        }
    }
}

__global__ void __launch_bounds__(kTailThreads) graph_tail_kernel(const __grid_constant__ TailArgs A) {
    pdl_enter();
    graph_tail_body(A);
}

// ------------------------------------------ Krylov acceleration (MG-PCG)
// The projection solves L p = rhs with L the (negative semi-definite) graph
// Laplacian. Conjugate gradients run on A = -L; `res` stores the residual in
// the multigrid convention res = rhs - L x (= -(b - A x) for b = -rhs), so a
// V-cycle applied to res approximates A^-1 r directly.
__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Block-wide FP64 sum then one atomicAdd per block (block of 256 threads).
__device__ __forceinline__ void block_sum_to(double* out, double v) {
    __shared__ double part[8];
    v = warp_sum_d(v);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    if ((tid & 31) == 0) part[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; ++w) s += part[w];
        if (s != 0.0) atomicAdd(out, s);
    }
}

// Last sweep of the preconditioning V-cycle fused with dot += scale * rhs . out.
__global__ void __launch_bounds__(256) graph_smooth_dot_kernel(GLvl g, const float* __restrict__ p,
                                                              const float* __restrict__ rhs, float omega, float* out,
                                                              double* dot, double scale) {
    int x, y, z;
    double acc = 0.0;
    if (cell_coords(g.nx, g.ny, x, y, z)) {
        const int i = x + g.nx * (y + g.ny * z);
        float diag, nb;
        graph_terms(g, i, x, y, z, [&](int j, int, int, int) { return __ldg(p + j); }, diag, nb);
        const float r = __ldg(rhs + i);
        const float v = diag > 0.f ? __ldg(p + i) * (1.f - omega) + ((nb - r) / diag) * omega : 0.f;
        out[i] = v;
        acc = scale * (double)r * (double)v;
    }
    block_sum_to(dot, acc);
}

// Prolongation + first post-sweep fused with dot += scale * rhs . out (the
// last sweep of a preconditioning V-cycle with one post-sweep).
__global__ void __launch_bounds__(256) graph_prolong_smooth_dot_kernel(GLvl g, const float* __restrict__ p,
                                                                      const float* __restrict__ coarse,
                                                                      const float* __restrict__ rhs, float omega,
                                                                      float* out, double* dot, double scale) {
    int x, y, z;
    double acc = 0.0;
    if (cell_coords(g.nx, g.ny, x, y, z)) {
        const int i = x + g.nx * (y + g.ny * z);
        float diag, nb;
        graph_terms(g, i, x, y, z,
                    [&](int j, int jx, int jy, int jz) { return prolonged(g, p, coarse, j, jx, jy, jz); }, diag, nb);
        const float pc = prolonged(g, p, coarse, i, x, y, z);
        const float r = __ldg(rhs + i);
        const float v = diag > 0.f ? pc * (1.f - omega) + ((nb - r) / diag) * omega : 0.f;
        out[i] = v;
        acc = scale * (double)r * (double)v;
    }
    block_sum_to(dot, acc);
}

// First sweep from a zero iterate: p_out = omega * (0 - rhs) / diag on active cells.
__global__ void __launch_bounds__(256) graph_smooth_zero_kernel(GLvl g, const float* __restrict__ rhs, float omega,
                                                               float* out) {
    pdl_enter();
    int x, y, z;
    if (!cell_coords(g.nx, g.ny, x, y, z)) return;
    const int i = x + g.nx * (y + g.ny * z);
    float diag, nb;
    graph_terms(g, i, x, y, z, [&](int, int, int, int) { return 0.f; }, diag, nb);
    out[i] = diag > 0.f ? 0.f * (1.f - omega) + ((nb - __ldg(rhs + i)) / diag) * omega : 0.f;
}

// New search direction p = z + beta p_old (beta = rz_new / rz_old; p = z when
// rz_old is NULL), written out, and q = A p = diag p - nb(p), with pq += p . q.
__global__ void __launch_bounds__(256) pcg_direction_apply_kernel(GLvl g, const float* __restrict__ zv,
                                                                 const float* __restrict__ p_old,
                                                                 const double* rz_new, const double* rz_old,
                                                                 float* p_out, float* q, double* pq) {
    int x, y, z;
    const float beta = rz_old ? (float)(*rz_new / *rz_old) : 0.f;
    double acc = 0.0;
    if (cell_coords(g.nx, g.ny, x, y, z)) {
        const int i = x + g.nx * (y + g.ny * z);
        auto dir = [&](int j) { return rz_old ? __ldg(zv + j) + beta * __ldg(p_old + j) : __ldg(zv + j); };
        float diag, nb;
        graph_terms(g, i, x, y, z, [&](int j, int, int, int) { return dir(j); }, diag, nb);
        const float pc = dir(i);
        const float qc = diag > 0.f ? diag * pc - nb : 0.f;
        p_out[i] = pc;
        q[i] = qc;
        acc = (double)pc * (double)qc;
    }
    block_sum_to(pq, acc);
}

// x += alpha p; res += alpha q; resmax = max|res| (alpha = rz / pq).
__global__ void __launch_bounds__(256) pcg_update_kernel(int64_t n, const double* rz, const double* pq,
                                                        float* __restrict__ xv, const float* __restrict__ p,
                                                        float* __restrict__ res, const float* __restrict__ q,
                                                        float* resmax) {
    const double den = *pq;
    const float alpha = den > 0.0 ? (float)(*rz / den) : 0.f;
    float m = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        xv[i] = xv[i] + alpha * p[i];
        const float r = res[i] + alpha * q[i];
        res[i] = r;
        m = fmaxf(m, finite_abs(r));
    }
    block_max_to(resmax, m);
}

bool solids_ok(const FfxSolids* s) {
    if (!s) return true;
    const bool walls = s->wall[0] || s->wall[1] || s->wall[2];
    if (walls && !(s->wall[0] && s->wall[1] && s->wall[2] && s->solid)) return false;   // all three, with a mask
    return (!s->solid && !s->halo) || (s->solid && s->halo);
}
bool has_mask(const FfxSolids* s) { return s && s->solid; }

bool glvl_ok(const FfxGraphLevel* lv) {
    if (!lv || lv->nx < 1 || lv->ny < 1 || lv->nz < 1 || lv->nz > 65535) return false;
    if ((int64_t)lv->nx * lv->ny * lv->nz >= (int64_t(1) << 31)) return false;
    if (lv->edges) return ((uintptr_t)lv->edges & 15) == 0;
    return lv->solid != nullptr;
}

bool nz_ok(const int32_t n[3]) { return n[2] <= 65535; }

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" {

int ffx_walls(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v, const void* w,
              void* ou, void* ov, void* ow, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solids_ok(s) && u && v && w && ou && ov && ow,
                "ffx_walls: invalid arguments");
    FFX_REQUIRE(ou != u && ov != v && ow != w, "ffx_walls: outputs must not alias inputs");
    Dev d = make_dev(*g);
    cudaStream_t st = as_stream(stream);
    dim3 grid = cell_grid(g->nx, g->ny, g->nz), block = cell_block();
    FFX_DISPATCH_STORAGE(storage, T, {
        Faces<T> F = {(const T*)u, (const T*)v, (const T*)w};
        if (has_mask(s)) walls_div_kernel<T, true, false><<<grid, block, 0, st>>>(d, s->solid, make_walls(s), F, (T*)ou, (T*)ov,
                                                                                  (T*)ow, nullptr);
        else walls_div_kernel<T, false, false><<<grid, block, 0, st>>>(d, nullptr, Walls{}, F, (T*)ou, (T*)ov, (T*)ow, nullptr);
    });
    return launch_status("walls_kernel");
}

int ffx_divergence(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v, const void* w,
                   float* div, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solids_ok(s) && u && v && w && div,
                "ffx_divergence: invalid arguments");
    Dev d = make_dev(*g);
    cudaStream_t st = as_stream(stream);
    dim3 grid = cell_grid(g->nx, g->ny, g->nz), block = cell_block();
    FFX_DISPATCH_STORAGE(storage, T, {
        Faces<T> F = {(const T*)u, (const T*)v, (const T*)w};
        if (has_mask(s)) divergence_kernel<T, true><<<grid, block, 0, st>>>(d, s->solid, F, div);
        else divergence_kernel<T, false><<<grid, block, 0, st>>>(d, nullptr, F, div);
    });
    return launch_status("divergence_kernel");
}

int ffx_walls_divergence(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                         const void* w, void* ou, void* ov, void* ow, float* div, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solids_ok(s) && u && v && w && ou && ov && ow && div,
                "ffx_walls_divergence: invalid arguments");
    FFX_REQUIRE(ou != u && ov != v && ow != w, "ffx_walls_divergence: outputs must not alias inputs");
    Dev d = make_dev(*g);
    cudaStream_t st = as_stream(stream);
    dim3 grid = cell_grid(g->nx, g->ny, g->nz), block = cell_block();
    FFX_DISPATCH_STORAGE(storage, T, {
        Faces<T> F = {(const T*)u, (const T*)v, (const T*)w};
        if (has_mask(s)) walls_div_kernel<T, true, true><<<grid, block, 0, st>>>(d, s->solid, make_walls(s), F, (T*)ou, (T*)ov,
                                                                                 (T*)ow, div);
        else walls_div_kernel<T, false, true><<<grid, block, 0, st>>>(d, nullptr, Walls{}, F, (T*)ou, (T*)ov, (T*)ow, div);
    });
    return launch_status("walls_divergence_kernel");
}

static int gradient_impl(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                         const void* w, const float* pressure, float dt, void* ou, void* ov, void* ow,
                         float* div_after, float* maxima, const uint8_t* links, float* div_exact,
                         void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solids_ok(s) && u && v && w && pressure && ou && ov && ow,
                "ffx_gradient: invalid arguments");
    FFX_REQUIRE(ou != u && ov != v && ow != w, "ffx_gradient: outputs must not alias inputs");
    Dev d = make_dev(*g);
    cudaStream_t st = as_stream(stream);
    if (maxima) {
        int e = cuda_status(cudaMemsetAsync(maxima, 0, 3 * sizeof(float), st), "ffx_gradient memset");
        if (e) return e;
    }
    dim3 grid = cell_grid(g->nx, g->ny, g->nz), block = cell_block();
    FFX_DISPATCH_STORAGE(storage, T, {
        Faces<T> F = {(const T*)u, (const T*)v, (const T*)w};
        if (has_mask(s)) gradient_kernel<T, true><<<grid, block, 0, st>>>(d, s->solid, make_walls(s), F, pressure, dt, (T*)ou,
                                                                          (T*)ov, (T*)ow, div_after, maxima, links,
                                                                          div_exact);
        else gradient_kernel<T, false><<<grid, block, 0, st>>>(d, nullptr, Walls{}, F, pressure, dt, (T*)ou, (T*)ov, (T*)ow,
                                                               div_after, maxima, nullptr, div_exact);
    });
    return launch_status("gradient_kernel");
}

int ffx_gradient(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v, const void* w,
                 const float* pressure, float dt, void* ou, void* ov, void* ow, float* div_after, float* maxima,
                 void* stream) {
    return gradient_impl(g, s, storage, u, v, w, pressure, dt, ou, ov, ow, div_after, maxima, nullptr, nullptr,
                         stream);
}

int ffx_gradient_links(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v,
                       const void* w, const float* pressure, float dt, void* ou, void* ov, void* ow,
                       float* div_after, float* maxima, const uint8_t* links, void* stream) {
    return gradient_impl(g, s, storage, u, v, w, pressure, dt, ou, ov, ow, div_after, maxima, links, nullptr,
                         stream);
}

int ffx_gradient_ex(const FfxGrid* g, const FfxSolids* s, int storage, const void* u, const void* v, const void* w,
                    const float* pressure, float dt, void* ou, void* ov, void* ow, float* div_after, float* maxima,
                    const uint8_t* links, float* div_unrounded, void* stream) {
    return gradient_impl(g, s, storage, u, v, w, pressure, dt, ou, ov, ow, div_after, maxima, links, div_unrounded,
                         stream);
}

int ffx_jacobi(const int32_t n[3], const float inv[3], const uint8_t* solid, const float* p_in, const float* rhs,
               float dt, float omega, float* p_out, void* stream) {
    FFX_REQUIRE(shape_ok(n) && nz_ok(n) && inv && p_in && rhs && p_out && p_in != p_out && dt != 0.f,
                "ffx_jacobi: invalid arguments");
    Lvl L = make_lvl(n, inv);
    cudaStream_t st = as_stream(stream);
    dim3 grid = cell_grid(n[0], n[1], n[2]), block = cell_block();
    if (solid) jacobi_kernel<true><<<grid, block, 0, st>>>(L, solid, p_in, rhs, dt, omega, p_out);
    else jacobi_kernel<false><<<grid, block, 0, st>>>(L, nullptr, p_in, rhs, dt, omega, p_out);
    return launch_status("jacobi_kernel");
}

int ffx_scale(int64_t count, const float* in, float factor, float* out, void* stream) {
    FFX_REQUIRE(count >= 0 && (count == 0 || (in && out)), "ffx_scale: invalid arguments");
    if (count == 0) return FFX_OK;
    scale_kernel<<<blocks_for(count, 256), 256, 0, as_stream(stream)>>>(count, in, factor, out);
    return launch_status("scale_kernel");
}

int ffx_add(int64_t count, const float* a, const float* b, float* out, void* stream) {
    FFX_REQUIRE(count >= 1 && a && b && out, "ffx_add: invalid arguments");
    const int64_t want = (count + 255) / 256;
    add_kernel<<<(unsigned)(want < 148 * 8 ? want : 148 * 8), 256, 0, as_stream(stream)>>>(count, a, b, out);
    return launch_status("add_kernel");
}

int ffx_mg_residual(const int32_t n[3], const float inv[3], const float* p, const float* rhs, float dt, float* r,
                    void* stream) {
    FFX_REQUIRE(shape_ok(n) && nz_ok(n) && inv && p && rhs && r && dt != 0.f, "ffx_mg_residual: invalid arguments");
    Lvl L = make_lvl(n, inv);
    mg_residual_kernel<<<cell_grid(n[0], n[1], n[2]), cell_block(), 0, as_stream(stream)>>>(L, p, rhs, dt, r);
    return launch_status("mg_residual_kernel");
}

int ffx_mg_restrict(const int32_t fine_n[3], const float* fine, float* coarse, void* stream) {
    FFX_REQUIRE(shape_ok(fine_n) && nz_ok(fine_n) && fine && coarse && fine_n[0] % 2 == 0 && fine_n[1] % 2 == 0 &&
                fine_n[2] % 2 == 0, "ffx_mg_restrict: invalid arguments (even fine shape required)");
    mg_restrict_kernel<<<cell_grid(fine_n[0] / 2, fine_n[1] / 2, fine_n[2] / 2), cell_block(), 0,
                         as_stream(stream)>>>(fine_n[0], fine_n[1], fine_n[2], fine, coarse);
    return launch_status("mg_restrict_kernel");
}

int ffx_mg_residual_restrict(const int32_t n[3], const float inv[3], const float* p, const float* rhs, float dt,
                             float* coarse_rhs, void* stream) {
    FFX_REQUIRE(shape_ok(n) && nz_ok(n) && inv && p && rhs && coarse_rhs && dt != 0.f && n[0] % 2 == 0 &&
                n[1] % 2 == 0 && n[2] % 2 == 0, "ffx_mg_residual_restrict: invalid arguments");
    Lvl L = make_lvl(n, inv);
    mg_residual_restrict_kernel<<<cell_grid(n[0] / 2, n[1] / 2, n[2] / 2), cell_block(), 0, as_stream(stream)>>>(
        L, p, rhs, dt, coarse_rhs);
    return launch_status("mg_residual_restrict_kernel");
}

int ffx_mg_prolong(const int32_t fine_n[3], const float* p, const float* coarse, float* p_out, void* stream) {
    FFX_REQUIRE(shape_ok(fine_n) && nz_ok(fine_n) && p && coarse && p_out && p != p_out && fine_n[0] % 2 == 0 &&
                fine_n[1] % 2 == 0 && fine_n[2] % 2 == 0, "ffx_mg_prolong: invalid arguments");
    mg_prolong_kernel<<<cell_grid(fine_n[0], fine_n[1], fine_n[2]), cell_block(), 0, as_stream(stream)>>>(
        fine_n[0], fine_n[1], fine_n[2], p, coarse, p_out);
    return launch_status("mg_prolong_kernel");
}

int ffx_direct_solve(int32_t n, const double* inverse, const float* rhs, float dt, float* p, void* stream) {
    FFX_REQUIRE(n >= 1 && n <= 1024 && inverse && rhs && p && rhs != p && dt != 0.f,
                "ffx_direct_solve: invalid arguments (n in [1, 1024])");
    int threads = 256;
    int blocks = (n * 32 + threads - 1) / threads;
    return launch_pdl("direct_kernel", direct_kernel, dim3(blocks), dim3(threads), as_stream(stream), n, inverse, rhs,
                      dt, p);
}

int ffx_mg_residual_max(const int32_t n[3], const float inv[3], const float* p, const float* rhs, float dt,
                        float* out, void* stream) {
    FFX_REQUIRE(shape_ok(n) && nz_ok(n) && inv && p && rhs && out && dt != 0.f,
                "ffx_mg_residual_max: invalid arguments");
    Lvl L = make_lvl(n, inv);
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(out, 0, sizeof(float), st), "ffx_mg_residual_max memset");
    if (e) return e;
    dim3 grid = cell_grid(n[0], n[1], 1);
    grid.z = reduce_z(n[2]);
    mg_residual_max_kernel<<<grid, cell_block(), 0, st>>>(L, p, rhs, dt, out);
    return launch_status("mg_residual_max_kernel");
}

int ffx_graph_smooth(const FfxGraphLevel* lv, const float* p_in, const float* rhs, float omega, float* p_out,
                     void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p_in && rhs && p_out && p_in != p_out, "ffx_graph_smooth: invalid arguments");
    if (level0_x4(lv, {p_in, rhs, p_out})) return level0_smooth(lv, p_in, rhs, omega, p_out, as_stream(stream));
    GLvl g = make_glvl(lv);
    if (!g.edges) {
        dim3 grid = cell_grid(g.nx, g.ny, (g.nz + kZ - 1) / kZ);
        return launch_pdl("graph_smooth_level0_kernel", graph_smooth_level0_kernel, grid, cell_block(),
                          as_stream(stream), g, p_in, rhs, omega, p_out);
    }
    return launch_pdl("graph_smooth_kernel", graph_smooth_kernel, cell_grid(g.nx, g.ny, g.nz), cell_block(),
                      as_stream(stream), g, p_in, rhs, omega, p_out);
}

int ffx_graph_smooth2(const FfxGraphLevel* lv, const float* p_in, const float* rhs, float omega, float* tmp,
                      float* p_out, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p_in && rhs && p_out && p_in != p_out && (!tmp || (tmp != p_in && tmp != p_out)),
                "ffx_graph_smooth2: invalid arguments");
    if (level0_x4(lv, {p_in, rhs, p_out})) return level0_smooth2(lv, p_in, rhs, omega, p_out, as_stream(stream));
    FFX_REQUIRE(tmp, "ffx_graph_smooth2: this level needs the intermediate buffer");
    const int e = ffx_graph_smooth(lv, p_in, rhs, omega, tmp, stream);
    return e ? e : ffx_graph_smooth(lv, tmp, rhs, omega, p_out, stream);
}

int ffx_graph_prolong_smooth2(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                              float omega, float* tmp, float* p_out, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p && coarse && rhs && p_out && p != p_out && lv->nx % 2 == 0 && lv->ny % 2 == 0 &&
                lv->nz % 2 == 0 && (!tmp || (tmp != p && tmp != p_out)),
                "ffx_graph_prolong_smooth2: invalid arguments");
    if (level0_x4(lv, {p, rhs, p_out}) && ((uintptr_t)coarse & 7) == 0)
        return level0_prolong_smooth2(lv, p, coarse, rhs, omega, p_out, as_stream(stream));
    FFX_REQUIRE(tmp, "ffx_graph_prolong_smooth2: this level needs the intermediate buffer");
    const int e = ffx_graph_prolong_smooth(lv, p, coarse, rhs, omega, tmp, stream);
    return e ? e : ffx_graph_smooth(lv, tmp, rhs, omega, p_out, stream);
}

int ffx_graph_residual(const FfxGraphLevel* lv, const float* p, const float* rhs, float* r, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p && rhs && r && r != p, "ffx_graph_residual: invalid arguments");
    if (level0_x4(lv, {p, rhs, r})) return level0_residual(lv, p, rhs, r, as_stream(stream));
    GLvl g = make_glvl(lv);
    graph_residual_kernel<<<cell_grid(g.nx, g.ny, g.nz), cell_block(), 0, as_stream(stream)>>>(g, p, rhs, r);
    return launch_status("graph_residual_kernel");
}

int ffx_graph_residual_restrict_zero(const FfxGraphLevel* lv, const float* p, const float* rhs, float* coarse_rhs,
                                     float* coarse_p, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p && rhs && coarse_rhs && lv->nx % 2 == 0 && lv->ny % 2 == 0 && lv->nz % 2 == 0,
                "ffx_graph_residual_restrict: invalid arguments");
    FFX_REQUIRE(coarse_p != coarse_rhs || !coarse_p, "ffx_graph_residual_restrict: coarse iterate aliases its rhs");
    if (level0_x4(lv, {p, rhs}) && ((uintptr_t)coarse_rhs & 7) == 0 && ((uintptr_t)coarse_p & 7) == 0)
        return level0_residual_restrict(lv, p, rhs, coarse_rhs, coarse_p, as_stream(stream));
    GLvl g = make_glvl(lv);
    if (g_edge_streaming && g.edges) {
        const int cz = g.nz / 2, chunk = edge_chunk(g.nx, g.ny, g.nz) / 2;
        return launch_pdl("graph_residual_restrict_edges_kernel", graph_residual_restrict_edges_kernel,
                          cell_grid(g.nx / 2, g.ny / 2, (cz + chunk - 1) / chunk), cell_block(), as_stream(stream), g,
                          p, rhs, coarse_rhs, coarse_p, chunk);
    }
    return launch_pdl("graph_residual_restrict_kernel", graph_residual_restrict_zero_kernel,
                      cell_grid(g.nx / 2, g.ny / 2, g.nz / 2), cell_block(), as_stream(stream), g, p, rhs, coarse_rhs,
                      coarse_p);
}

int ffx_graph_residual_restrict(const FfxGraphLevel* lv, const float* p, const float* rhs, float* coarse_rhs,
                                void* stream) {
    return ffx_graph_residual_restrict_zero(lv, p, rhs, coarse_rhs, nullptr, stream);
}

int ffx_graph_prolong(const FfxGraphLevel* lv, const float* p, const float* coarse, float* p_out, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p && coarse && p_out && p != p_out && lv->nx % 2 == 0 && lv->ny % 2 == 0 &&
                lv->nz % 2 == 0, "ffx_graph_prolong: invalid arguments");
    GLvl g = make_glvl(lv);
    graph_prolong_kernel<<<cell_grid(g.nx, g.ny, g.nz), cell_block(), 0, as_stream(stream)>>>(g, p, coarse, p_out);
    return launch_status("graph_prolong_kernel");
}

int ffx_graph_prolong_smooth(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                             float omega, float* p_out, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p && coarse && rhs && p_out && p != p_out && lv->nx % 2 == 0 && lv->ny % 2 == 0 &&
                lv->nz % 2 == 0, "ffx_graph_prolong_smooth: invalid arguments");
    if (level0_x4(lv, {p, rhs, p_out}) && ((uintptr_t)coarse & 7) == 0)
        return level0_prolong_smooth(lv, p, coarse, rhs, omega, p_out, as_stream(stream));
    GLvl g = make_glvl(lv);
    return launch_pdl("graph_prolong_smooth_kernel", graph_prolong_smooth_kernel, cell_grid(g.nx, g.ny, g.nz),
                      cell_block(), as_stream(stream), g, p, coarse, rhs, omega, p_out);
}

int ffx_set_edge_streaming(int enable) {
    const int previous = g_edge_streaming;
    g_edge_streaming = enable ? 1 : 0;
    return previous;
}

int ffx_graph_residual_max(const FfxGraphLevel* lv, const float* p, const float* rhs, float* out, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p && rhs && out, "ffx_graph_residual_max: invalid arguments");
    GLvl g = make_glvl(lv);
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(out, 0, sizeof(float), st), "ffx_graph_residual_max memset");
    if (e) return e;
    if (level0_x4(lv, {p, rhs})) return level0_residual_max(lv, p, rhs, out, st);
    dim3 grid = cell_grid(g.nx, g.ny, 1);
    grid.z = reduce_z(g.nz);
    return launch_pdl("graph_residual_max_kernel", graph_residual_max_kernel, grid, cell_block(), st, g, p, rhs, out);
}

int ffx_graph_residual_max_smooth(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega,
                                  float* out, float* p_out, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p && rhs && out && p_out && p_out != p,
                "ffx_graph_residual_max_smooth: invalid arguments");
    cudaStream_t st = as_stream(stream);
    if (level0_x4(lv, {p, rhs, p_out})) {
        int e = cuda_status(cudaMemsetAsync(out, 0, sizeof(float), st), "ffx_graph_residual_max_smooth memset");
        return e ? e : level0_residual_max_smooth(lv, p, rhs, omega, out, p_out, st);
    }
    const int e = ffx_graph_residual_max(lv, p, rhs, out, stream);
    return e ? e : ffx_graph_smooth(lv, p, rhs, omega, p_out, stream);
}

int ffx_graph_coarsen(const FfxGraphLevel* fine, float* coarse_edges, int32_t* disconnected, void* stream) {
    FFX_REQUIRE(glvl_ok(fine) && coarse_edges && disconnected && ((uintptr_t)coarse_edges & 15) == 0 &&
                fine->nx % 2 == 0 && fine->ny % 2 == 0 && fine->nz % 2 == 0,
                "ffx_graph_coarsen: invalid arguments (even shape, 16-byte aligned records)");
    GLvl g = make_glvl(fine);
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(disconnected, 0, sizeof(int32_t), st), "ffx_graph_coarsen memset");
    if (e) return e;
    graph_coarsen_kernel<<<cell_grid(g.nx / 2, g.ny / 2, g.nz / 2), cell_block(), 0, st>>>(
        g, reinterpret_cast<float4*>(coarse_edges), disconnected);
    return launch_status("graph_coarsen_kernel");
}

int ffx_graph_tail(const FfxGraphTail* t, void* stream) {
    FFX_REQUIRE(t && t->count >= 1 && t->count <= FFX_TAIL_LEVELS && t->pre >= 0 && t->post >= 0 &&
                t->pre <= 64 && t->post <= 64, "ffx_graph_tail: invalid arguments");
    TailArgs A;
    A.count = t->count;
    A.pre = t->pre;
    A.post = t->post;
    A.omega = t->omega;
    A.inverse = t->inverse;
    for (int k = 0; k < t->count; ++k) {
        const FfxTailLevel& L = t->levels[k];
        const FfxGraphLevel& lv = L.level;
        FFX_REQUIRE(glvl_ok(&lv) && lv.edges && L.p && L.q && L.rhs && L.p != L.q && L.p != L.rhs &&
                    L.q != L.rhs && (int64_t)lv.nx * lv.ny * lv.nz <= kTailCells,
                    "ffx_graph_tail: level %d invalid (edges, distinct p/q/rhs, <= %d cells)", k, kTailCells);
        if (k > 0) {
            const FfxGraphLevel& up = t->levels[k - 1].level;
            FFX_REQUIRE(up.nx == 2 * lv.nx && up.ny == 2 * lv.ny && up.nz == 2 * lv.nz,
                        "ffx_graph_tail: level %d is not the 2x coarsening of level %d", k, k - 1);
        }
        A.lv[k].g = make_glvl(&lv);
        A.lv[k].p = L.p;
        A.lv[k].q = L.q;
        A.lv[k].rhs = L.rhs;
        A.lv[k].n = lv.nx * lv.ny * lv.nz;
    }
    FFX_REQUIRE(!t->inverse || A.lv[t->count - 1].n <= 1024, "ffx_graph_tail: direct solve limited to 1024 cells");
    return launch_pdl("graph_tail_kernel", graph_tail_kernel, dim3(1), dim3(kTailThreads), as_stream(stream), A);
}

int ffx_graph_links(const FfxGraphLevel* lv, uint8_t* links, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && !lv->edges && lv->solid && links, "ffx_graph_links: invalid arguments");
    return level0_links(lv->nx, lv->ny, lv->nz, lv->solid, links, as_stream(stream));
}

int ffx_graph_level0_edges(const FfxGraphLevel* lv, float* edges, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && !lv->edges && edges && ((uintptr_t)edges & 15) == 0,
                "ffx_graph_level0_edges: invalid arguments");
    GLvl g = make_glvl(lv);
    graph_level0_kernel<<<cell_grid(g.nx, g.ny, g.nz), cell_block(), 0, as_stream(stream)>>>(
        g, reinterpret_cast<float4*>(edges));
    return launch_status("graph_level0_kernel");
}

}  // extern "C"

namespace ffx {
namespace {

__global__ void __launch_bounds__(256) dot_kernel(int64_t n, const float* __restrict__ a,
                                                 const float* __restrict__ b, double scale, double* out) {
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += (double)a[i] * (double)b[i];
    block_sum_to(out, scale * acc);
}

unsigned flat_blocks(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 8 ? (b < 1 ? 1 : b) : 148 * 8);
}

}  // namespace
}  // namespace ffx

extern "C" {

int ffx_graph_smooth_zero(const FfxGraphLevel* lv, const float* rhs, float omega, float* p_out, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && rhs && p_out && rhs != p_out, "ffx_graph_smooth_zero: invalid arguments");
    if (level0_x4(lv, {rhs, p_out})) return level0_smooth_zero(lv, rhs, omega, p_out, as_stream(stream));
    GLvl g = make_glvl(lv);
    return launch_pdl("graph_smooth_zero_kernel", graph_smooth_zero_kernel, cell_grid(g.nx, g.ny, g.nz), cell_block(),
                      as_stream(stream), g, rhs, omega, p_out);
}

int ffx_graph_smooth_dot(const FfxGraphLevel* lv, const float* p_in, const float* rhs, float omega, float* p_out,
                         double* dot, double scale, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p_in && rhs && p_out && dot && p_in != p_out,
                "ffx_graph_smooth_dot: invalid arguments");
    GLvl g = make_glvl(lv);
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(dot, 0, sizeof(double), st), "ffx_graph_smooth_dot memset");
    if (e) return e;
    if (level0_x4(lv, {p_in, rhs, p_out})) return level0_smooth_dot(lv, p_in, rhs, omega, p_out, dot, scale, st);
    graph_smooth_dot_kernel<<<cell_grid(g.nx, g.ny, g.nz), cell_block(), 0, st>>>(g, p_in, rhs, omega, p_out, dot,
                                                                                 scale);
    return launch_status("graph_smooth_dot_kernel");
}

int ffx_graph_prolong_smooth_dot(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                                 float omega, float* p_out, double* dot, double scale, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && p && coarse && rhs && p_out && dot && p != p_out && lv->nx % 2 == 0 &&
                lv->ny % 2 == 0 && lv->nz % 2 == 0, "ffx_graph_prolong_smooth_dot: invalid arguments");
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(dot, 0, sizeof(double), st), "ffx_graph_prolong_smooth_dot memset");
    if (e) return e;
    if (level0_x4(lv, {p, rhs, p_out}) && ((uintptr_t)coarse & 7) == 0)
        return level0_prolong_smooth_dot(lv, p, coarse, rhs, omega, p_out, dot, scale, st);
    GLvl g = make_glvl(lv);
    graph_prolong_smooth_dot_kernel<<<cell_grid(g.nx, g.ny, g.nz), cell_block(), 0, st>>>(g, p, coarse, rhs, omega,
                                                                                         p_out, dot, scale);
    return launch_status("graph_prolong_smooth_dot_kernel");
}

int ffx_pcg_direction_apply(const FfxGraphLevel* lv, const float* z, const float* p_old, const double* rz_new,
                            const double* rz_old, float* p_out, float* q, double* pq, void* stream) {
    FFX_REQUIRE(glvl_ok(lv) && z && p_out && q && pq && (!rz_old || (rz_new && p_old)) && p_out != p_old &&
                p_out != z && q != z, "ffx_pcg_direction_apply: invalid arguments");
    GLvl g = make_glvl(lv);
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(pq, 0, sizeof(double), st), "ffx_pcg_direction_apply memset");
    if (e) return e;
    if (level0_x4(lv, {z, rz_old ? p_old : nullptr, p_out, q}))
        return level0_direction_apply(lv, z, p_old, rz_new, rz_old, p_out, q, pq, st);
    pcg_direction_apply_kernel<<<cell_grid(g.nx, g.ny, g.nz), cell_block(), 0, st>>>(g, z, p_old, rz_new, rz_old,
                                                                                    p_out, q, pq);
    return launch_status("pcg_direction_apply_kernel");
}

int ffx_pcg_update(int64_t count, const double* rz, const double* pq, float* x, const float* p, float* res,
                   const float* q, float* resmax, void* stream) {
    FFX_REQUIRE(count >= 1 && rz && pq && x && p && res && q && resmax, "ffx_pcg_update: invalid arguments");
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(resmax, 0, sizeof(float), st), "ffx_pcg_update memset");
    if (e) return e;
    pcg_update_kernel<<<flat_blocks(count), 256, 0, st>>>(count, rz, pq, x, p, res, q, resmax);
    return launch_status("pcg_update_kernel");
}

int ffx_dot(int64_t count, const float* a, const float* b, double scale, double* out, void* stream) {
    FFX_REQUIRE(count >= 1 && a && b && out, "ffx_dot: invalid arguments");
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(out, 0, sizeof(double), st), "ffx_dot memset");
    if (e) return e;
    dot_kernel<<<flat_blocks(count), 256, 0, st>>>(count, a, b, scale, out);
    return launch_status("dot_kernel");
}

}  // extern "C"

// ----------------------------------------------------------- batched passes
// Persistent launches over the tiles of many domains (ffx_batch.cuh) running
// the bodies of the single-domain kernels above on the collider path.
namespace ffx {
namespace {

constexpr float kOmega = (float)(2.0 / 3.0);   // the weighted-Jacobi factor the host passes

struct ScaleDesc {        // max |rhs| into the state, iterate zeroed
    int n;
    const float* rhs;
    float* p;
};
struct GDesc {            // one multigrid level
    GLvl g;
    const float* p;
    float* q;
    const float* rhs;
    float* coarse;
    float* zero;
};
struct DirectDesc {
    int n;
    const double* inverse;
    const float* rhs;
    float* p;
};

__global__ void __launch_bounds__(kBatchThreads) batch_divergence_kernel(const __grid_constant__ BatchMap M,
                                                                         const DivDesc<float>* descs,
                                                                         const BatchState* state) {
    for_tiles(M, descs, state, false, NoPrep{},
              [](const DivDesc<float>& P, const Blk& b, int) { divergence_body<float, true>(P, b); });
}

__global__ void __launch_bounds__(kBatchThreads) batch_scale_kernel(const __grid_constant__ BatchMap M,
                                                                    const ScaleDesc* descs, BatchState* state) {
    for_tiles(M, descs, state, false, NoPrep{}, [state](const ScaleDesc& P, const Blk& b, int slot) {
        const int i = b.x * kBatchThreads + (int)threadIdx.x;
        const int mode = state[slot].pmode;
        const float f = state[slot].pfactor;
        float v = 0.f;
        if (i < P.n) {
            v = finite_abs(__ldg(P.rhs + i));
            if (mode == 0) P.p[i] = 0.f;
            else if (mode == 2) P.p[i] = P.p[i] * f;   // ffx_scale's product
        }
        block_max_to(&state[slot].scale, v);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_gradient_kernel(const __grid_constant__ BatchMap M,
                                                                       const GradDesc<float>* descs,
                                                                       BatchState* state) {
    for_tiles(M, descs, state, false, NoPrep{}, [state](const GradDesc<float>& P, const Blk& b, int slot) {
        gradient_body<float, true>(P, b, state[slot].maxima);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_residual_max_kernel(const __grid_constant__ BatchMap M,
                                                                           const GDesc* descs, BatchState* state) {
    for_tiles(M, descs, state, true, NoPrep{}, [state](const GDesc& P, const Blk& b, int slot) {
        if (state[slot].scale == 0.f) {
            // rhs == 0: the solve's result is the zero pressure (and no cycle runs)
            int x, y, z;
            if (cell_coords(b, P.g.nx, P.g.ny, x, y, z))
                for (int zz = z; zz < P.g.nz; zz += b.gz) const_cast<float*>(P.p)[x + P.g.nx * (y + P.g.ny * zz)] = 0.f;
            return;
        }
        graph_residual_max_body(P.g, P.p, P.rhs, &state[slot].res, b);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_smooth_kernel(const __grid_constant__ BatchMap M,
                                                                     const GDesc* descs, const BatchState* state) {
    // level 0 (mask-derived terms) streams kBatchZ0 cells along z per thread
    for_tiles(M, descs, state, true, NoPrep{}, [](const GDesc& P, const Blk& b, int) {
        if (P.g.edges) graph_smooth_body(P.g, P.p, P.rhs, kOmega, P.q, b);
        else graph_smooth_level0_body(P.g, P.p, P.rhs, kOmega, P.q, b);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_residual_restrict_kernel(const __grid_constant__ BatchMap M,
                                                                                const GDesc* descs,
                                                                                const BatchState* state) {
    for_tiles(M, descs, state, true, NoPrep{}, [](const GDesc& P, const Blk& b, int) {
        graph_residual_restrict_body(P.g, P.p, P.rhs, P.coarse, P.zero, b);
    });
}

__global__ void __launch_bounds__(kBatchThreads) batch_prolong_smooth_kernel(const __grid_constant__ BatchMap M,
                                                                             const GDesc* descs,
                                                                             const BatchState* state) {
    for_tiles(M, descs, state, true, NoPrep{}, [](const GDesc& P, const Blk& b, int) {
        graph_prolong_smooth_body(P.g, P.p, P.coarse, P.rhs, kOmega, P.q, b);
    });
}

// direct_kernel's rows, eight per tile (one warp each).
__global__ void __launch_bounds__(kBatchThreads) batch_direct_kernel(const __grid_constant__ BatchMap M,
                                                                     const DirectDesc* descs,
                                                                     const BatchState* state) {
    for_tiles(M, descs, state, true, NoPrep{}, [](const DirectDesc& P, const Blk& b, int) {
        const int row = b.x * (kBatchThreads / 32) + (int)(threadIdx.x >> 5), lane = threadIdx.x & 31;
        if (row >= P.n) return;
        const double* r = P.inverse + (int64_t)row * P.n;
        double s = 0.0;
        for (int j = lane; j < P.n; j += 32) s += r[j] * (double)P.rhs[j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) P.p[row] = (float)(s / (double)1.0f);
    });
}

// One 1024-thread block per domain with a tail.
__global__ void __launch_bounds__(kTailThreads) batch_tail_kernel(const __grid_constant__ BatchMap M,
                                                                  const TailArgs* descs, const BatchState* state) {
    __shared__ __align__(16) unsigned char raw[sizeof(TailArgs)];
    const int k = blockIdx.x;
    if (k >= M.count || state[M.dom[k]].done) return;
    const int* src = reinterpret_cast<const int*>(descs + k);
    int* dst = reinterpret_cast<int*>(raw);
    for (int i = threadIdx.x; i < (int)(sizeof(TailArgs) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
    graph_tail_body(*reinterpret_cast<const TailArgs*>(raw));
}

template <class K>
int occupancy_of(K kernel) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kBatchThreads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

unsigned persistent(const BatchMap& M, int grid) {
    return (unsigned)(grid > 0 && grid < M.total ? grid : M.total);
}

GLvl batch_glvl(const FfxGraphLevel& lv) { return make_glvl(&lv); }

}  // namespace

namespace batch {

size_t divergence_desc(const FfxBatchDomain& D, void* out) {
    if (out) {
        DivDesc<float> P = {make_dev(D.grid), D.solid, {D.bu, D.bv, D.bw}, D.level[0].rhs};
        memcpy(out, &P, sizeof P);
    }
    return sizeof(DivDesc<float>);
}

size_t scale_zero_desc(const FfxBatchDomain& D, void* out) {
    if (out) {
        ScaleDesc P = {D.grid.nx * D.grid.ny * D.grid.nz, D.level[0].rhs, D.level[0].p};
        memcpy(out, &P, sizeof P);
    }
    return sizeof(ScaleDesc);
}

size_t gradient_desc(const FfxBatchDomain& D, float* u, float* v, float* w, void* out) {
    if (out) {
        GradDesc<float> P;
        memset(&P, 0, sizeof P);
        P.d = make_dev(D.grid);
        P.solid = D.solid;
        P.W = make_walls(nullptr);
        P.F = {D.bu, D.bv, D.bw};
        P.p = D.level[0].p;
        P.dt = 1.0f;   // impulse form: the solve used dt = 1
        P.out[0] = u; P.out[1] = v; P.out[2] = w;
        P.div = D.after;
        P.links = D.level[0].level.links;   // level-0 link bytes of the same mask (or NULL)
        memcpy(out, &P, sizeof P);
    }
    return sizeof(GradDesc<float>);
}

size_t level_desc(const FfxGraphLevel& lv, const float* p, float* q, const float* rhs, float* coarse, float* zero,
                  void* out) {
    if (out) {
        GDesc P = {batch_glvl(lv), p, q, rhs, coarse, zero};
        memcpy(out, &P, sizeof P);
    }
    return sizeof(GDesc);
}

size_t tail_desc(const FfxBatchDomain& D, int pre, int post, void* out) {
    if (out) {
        TailArgs A;
        memset(&A, 0, sizeof A);
        const int start = D.tail_start;
        A.count = D.levels - start;
        A.pre = pre;
        A.post = post;
        A.omega = kOmega;
        A.inverse = D.inverse;
        for (int k = 0; k < A.count; ++k) {
            const FfxBatchLevel& L = D.level[start + k];
            A.lv[k].g = batch_glvl(L.level);
            A.lv[k].p = L.p;
            A.lv[k].q = L.q;
            A.lv[k].rhs = L.rhs;
            A.lv[k].n = L.level.nx * L.level.ny * L.level.nz;
        }
        memcpy(out, &A, sizeof A);
    }
    return sizeof(TailArgs);
}

size_t direct_desc(const FfxBatchDomain& D, float* p, void* out) {
    if (out) {
        const FfxBatchLevel& L = D.level[D.levels - 1];
        DirectDesc P = {L.level.nx * L.level.ny * L.level.nz, D.inverse, L.rhs, p};
        memcpy(out, &P, sizeof P);
    }
    return sizeof(DirectDesc);
}

cudaError_t divergence(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_divergence_kernel<<<persistent(M, grid), kBatchThreads, 0, st>>>(M, (const DivDesc<float>*)descs, state);
    return cudaGetLastError();
}
cudaError_t scale_zero(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_scale_kernel<<<persistent(M, grid), kBatchThreads, 0, st>>>(M, (const ScaleDesc*)descs, state);
    return cudaGetLastError();
}
cudaError_t gradient(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_gradient_kernel<<<persistent(M, grid), kBatchThreads, 0, st>>>(M, (const GradDesc<float>*)descs, state);
    return cudaGetLastError();
}
cudaError_t residual_max(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_residual_max_kernel<<<persistent(M, grid), kBatchThreads, 0, st>>>(M, (const GDesc*)descs, state);
    return cudaGetLastError();
}
cudaError_t smooth(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_smooth_kernel<<<persistent(M, grid), kBatchThreads, 0, st>>>(M, (const GDesc*)descs, state);
    return cudaGetLastError();
}
cudaError_t residual_restrict(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_residual_restrict_kernel<<<persistent(M, grid), kBatchThreads, 0, st>>>(M, (const GDesc*)descs, state);
    return cudaGetLastError();
}
cudaError_t prolong_smooth(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_prolong_smooth_kernel<<<persistent(M, grid), kBatchThreads, 0, st>>>(M, (const GDesc*)descs, state);
    return cudaGetLastError();
}
cudaError_t direct(const BatchMap& M, const void* descs, BatchState* state, int grid, cudaStream_t st) {
    batch_direct_kernel<<<persistent(M, grid), kBatchThreads, 0, st>>>(M, (const DirectDesc*)descs, state);
    return cudaGetLastError();
}
cudaError_t tail(const BatchMap& M, const void* descs, BatchState* state, cudaStream_t st) {
    batch_tail_kernel<<<(unsigned)M.count, kTailThreads, 0, st>>>(M, (const TailArgs*)descs, state);
    return cudaGetLastError();
}

int project_resident_blocks(int kind) {
    switch (kind) {
        case kDivergence: return occupancy_of(batch_divergence_kernel);
        case kScaleZero: return occupancy_of(batch_scale_kernel);
        case kGradient: return occupancy_of(batch_gradient_kernel);
        case kResidualMax: return occupancy_of(batch_residual_max_kernel);
        case kSmooth: return occupancy_of(batch_smooth_kernel);
        case kResidualRestrict: return occupancy_of(batch_residual_restrict_kernel);
        case kProlongSmooth: return occupancy_of(batch_prolong_smooth_kernel);
        case kDirect: return occupancy_of(batch_direct_kernel);
        default: return 0;
    }
}

}  // namespace batch
}  // namespace ffx
