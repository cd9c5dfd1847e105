// Runtime entry points: error text, device query and probe, seeds, collider
// masks and reductions.
#include <cstring>

#include "ffx_host.cuh"
#include "ffx_stats.cuh"

namespace ffx {

std::string& last_error_buffer() {
    static thread_local std::string buf;
    return buf;
}

int g_pdl = 1;

namespace {

__global__ void probe_kernel(float* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 7 * 5 * 3) return;
    int x = i % 7, y = (i / 7) % 5, z = i / 35;
    out[i] = (float)(x + 10 * y + 100 * z);
}

// seed.glsl / temperature_seed.glsl
template <typename T>
__global__ void seed_scalar_kernel(Dev d, F3 center, float radius, float scale, int use_scale, T* out) {
    int64_t n = (int64_t)d.nx * d.ny * d.nz;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x = (int)(i % d.nx), y = (int)((i / d.nx) % d.ny), z = (int)(i / ((int64_t)d.nx * d.ny));
    F3 p = {((float)x + 0.5f) * d.e[0] / d.nf[0], ((float)y + 0.5f) * d.e[1] / d.nf[1],
            ((float)z + 0.5f) * d.e[2] / d.nf[2]};
    F3 off = {p.x - center.x, p.y - center.y, p.z - center.z};
    float w = fmaxf(1.0f - dot3(off, off) / (radius * radius), 0.0f);
    Store<T>::st(out, i, use_scale ? scale * w * w : w * w);
}

// mac_seed.glsl (all three components)
template <typename T>
__global__ void seed_faces_kernel(Dev d, F3 base, float angular, T* u, T* v, T* w) {
    int64_t nu = (int64_t)(d.nx + 1) * d.ny * d.nz, nv = (int64_t)d.nx * (d.ny + 1) * d.nz;
    int64_t nw = (int64_t)d.nx * d.ny * (d.nz + 1);
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int axis;
    int sx, sy;
    T* out;
    if (i < nu) { axis = 0; sx = d.nx + 1; sy = d.ny; out = u; }
    else if (i < nu + nv) { i -= nu; axis = 1; sx = d.nx; sy = d.ny + 1; out = v; }
    else if (i < nu + nv + nw) { i -= nu + nv; axis = 2; sx = d.nx; sy = d.ny; out = w; }
    else return;
    int x = (int)(i % sx), y = (int)((i / sx) % sy), z = (int)(i / ((int64_t)sx * sy));
    float ox = axis == 0 ? 0.f : 0.5f, oy = axis == 1 ? 0.f : 0.5f, oz = axis == 2 ? 0.f : 0.5f;
    float px = ((float)x + ox) * d.e[0] / d.nf[0];
    float py = ((float)y + oy) * d.e[1] / d.nf[1];
    float qx = px - 0.5f * d.e[0], qy = py - 0.5f * d.e[1];
    float val = axis == 0 ? base.x + (-angular * qy) : (axis == 1 ? base.y + angular * qx : base.z);
    (void)oz;
    Store<T>::st(out, i, val);
}

// FP64 voxelisation in the operation order of physics/collision.py:23-37.
__global__ void raster_kernel(Dev d, double ex, double ey, double ez, int count, const double* __restrict__ rows, uint8_t* solid) {
    int64_t n = (int64_t)d.nx * d.ny * d.nz;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x = (int)(i % d.nx), y = (int)((i / d.nx) % d.ny), z = (int)(i / ((int64_t)d.nx * d.ny));
    double hx = ex / d.nx, hy = ey / d.ny, hz = ez / d.nz;
    double px = (x + .5) * hx, py = (y + .5) * hy, pz = (z + .5) * hz;
    uint8_t inside = 0;
    for (int c = 0; c < count && !inside; ++c) {
        const double* r = rows + 13 * c;
        double q[3];
        for (int k = 0; k < 3; ++k) {
            const double* row = r + 4 * k;
            q[k] = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(row[0], px), __dmul_rn(row[1], py)),
                                       __dmul_rn(row[2], pz)), row[3]);
        }
        if (r[12] < 0.5) {
            double s = __dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2]));
            inside = s <= 1.0;
        } else {
            double m = fmax(fmax(fabs(q[0]), fabs(q[1])), fabs(q[2]));
            inside = m <= 1.0;
        }
    }
    solid[i] = inside;
}

__global__ void dilate_kernel(Dev d, const uint8_t* __restrict__ solid, uint8_t* halo) {
    int64_t n = (int64_t)d.nx * d.ny * d.nz;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x = (int)(i % d.nx), y = (int)((i / d.nx) % d.ny), z = (int)(i / ((int64_t)d.nx * d.ny));
    uint8_t any = 0;
    for (int dz = -1; dz <= 1 && !any; ++dz)
        for (int dy = -1; dy <= 1 && !any; ++dy)
            for (int dx = -1; dx <= 1 && !any; ++dx) any = solid_cell(d, solid, x + dx, y + dy, z + dz);
    halo[i] = any;
}

// 1 where no cell of the 5x5x5 block around the cell is set in `halo` or lies
// outside the grid (ffx_clearance).
__global__ void clearance_kernel(Dev d, const uint8_t* __restrict__ halo, uint8_t* clear) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= d.nx || y >= d.ny) return;
    bool any = x < 2 || y < 2 || z < 2 || x >= d.nx - 2 || y >= d.ny - 2 || z >= d.nz - 2;
    for (int dz = -2; dz <= 2 && !any; ++dz)
        for (int dy = -2; dy <= 2 && !any; ++dy) {
            const uint8_t* row = halo + cidx(d, x, y + dy, z + dz);
            any = row[-2] | row[-1] | row[0] | row[1] | row[2];
        }
    clear[cidx(d, x, y, z)] = any ? 0 : 1;
}

// The dilated mask and the clearance of a mask in one pass (ffx_halo_clearance):
// halo = any solid or outside cell in the 3x3x3 block (dilate_kernel's field);
// clear = 1 where the 7x7x7 block holds no solid and no outside cell
// (clearance_kernel's value), 2 where it holds no solid but reaches outside the
// grid, 0 where it holds a solid. A block owns 32 x 8 columns and a chunk of
// kHZ slices; per slice it stages the 38 x 14 window of the mask (outside = 0),
// dilates it along x and then y in shared memory, and every thread keeps the
// last seven slices' (x, y) dilations as bits, so the z dilation is a mask of
// those bits; the outside cells within distance 1 or 3 follow from the cell's
// coordinates.
constexpr int kHX = 32, kHY = 8, kHZ = 16, kHR = 3;
constexpr int kWinX = kHX + 2 * kHR, kWinY = kHY + 2 * kHR;

__global__ void __launch_bounds__(kHX * kHY) halo_clear_kernel(Dev d, const uint8_t* __restrict__ solid,
                                                               uint8_t* __restrict__ halo, uint8_t* __restrict__ clear) {
    __shared__ uint8_t win[kWinY][kWinX];
    __shared__ uint8_t rx1[kWinY][kHX], rx3[kWinY][kHX];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kHX + tx;
    const int x0 = blockIdx.x * kHX, y0 = blockIdx.y * kHY, z0 = blockIdx.z * kHZ;
    const int x = x0 + tx, y = y0 + ty;
    const int zend = min(z0 + kHZ, d.nz);
    unsigned h1 = 0u, h3 = 0u;   // bit k: the (x, y) dilation of slice zs - k
    for (int zs = z0 - kHR; zs < zend + kHR; ++zs) {
        for (int e = tid; e < kWinY * kWinX; e += kHX * kHY) {
            const int wy = e / kWinX, wx = e - wy * kWinX;
            const int gx = x0 - kHR + wx, gy = y0 - kHR + wy;
            const bool out = gx < 0 || gy < 0 || zs < 0 || gx >= d.nx || gy >= d.ny || zs >= d.nz;
            win[wy][wx] = out ? 0 : (__ldg(solid + cidx(d, gx, gy, zs)) != 0);
        }
        __syncthreads();
        for (int e = tid; e < kWinY * kHX; e += kHX * kHY) {
            const int wy = e / kHX, cx = e - wy * kHX;
            const uint8_t* r = win[wy] + cx;    // r[0 .. 6]: x - 3 .. x + 3
            rx1[wy][cx] = r[2] | r[3] | r[4];
            rx3[wy][cx] = r[0] | r[1] | r[2] | r[3] | r[4] | r[5] | r[6];
        }
        __syncthreads();
        const unsigned d1 = rx1[ty + 2][tx] | rx1[ty + 3][tx] | rx1[ty + 4][tx];
        unsigned d3 = 0u;
#pragma unroll
        for (int k = 0; k < 2 * kHR + 1; ++k) d3 |= rx3[ty + k][tx];
        h1 = (h1 << 1) | d1;
        h3 = (h3 << 1) | d3;
        const int z = zs - kHR;   // slices z - 3 .. z + 3 are bits 6 .. 0
        if (z >= z0 && z < zend && x < d.nx && y < d.ny) {
            const int i = cidx(d, x, y, z);
            const bool wall1 = x < 1 || y < 1 || z < 1 || x > d.nx - 2 || y > d.ny - 2 || z > d.nz - 2;
            const bool wall3 = x < 3 || y < 3 || z < 3 || x > d.nx - 4 || y > d.ny - 4 || z > d.nz - 4;
            halo[i] = wall1 || ((h1 >> 2) & 7u) != 0u;
            clear[i] = (h3 & 0x7fu) != 0u ? 0 : (wall3 ? 2 : 1);
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void solid_clear_kernel(int64_t n, const uint8_t* __restrict__ solid, const T* in, T* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Store<T>::st(out, i, solid[i] ? 0.f : Store<T>::ld(in, i));
}

template <typename T>
__global__ void max_abs_kernel(int64_t n, const T* __restrict__ x, float* out) {
    float m = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = fmaxf(m, finite_abs(Store<T>::ld(x, i)));
    block_max_to(out, m);
}

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" {

int ffx_abi_version(void) { return FFX_ABI_VERSION; }

const char* ffx_last_error(void) { return last_error_buffer().c_str(); }

int ffx_set_dependent_launch(int enable) {
    const int previous = g_pdl;
    g_pdl = enable ? 1 : 0;
    return previous;
}

int ffx_device_info(int device, FfxDeviceInfo* out) {
    FFX_REQUIRE(out, "ffx_device_info: out is NULL");
    cudaDeviceProp prop;
    int st = cuda_status(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (st) return st;
    std::memset(out, 0, sizeof *out);
    out->device = device;
    out->sm_count = prop.multiProcessorCount;
    out->cc_major = prop.major;
    out->cc_minor = prop.minor;
    out->total_bytes = (int64_t)prop.totalGlobalMem;
    std::strncpy(out->name, prop.name, sizeof out->name - 1);
    return FFX_OK;
}

int ffx_probe_3d(float* out, void* stream) {
    FFX_REQUIRE(out, "ffx_probe_3d: out is NULL");
    probe_kernel<<<1, 128, 0, as_stream(stream)>>>(out);
    return launch_status("probe_kernel");
}

int ffx_seed_scalar(const FfxGrid* g, int storage, const float center[3], float radius, float scale,
                    void* out, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && center && out && radius > 0.f,
                "ffx_seed_scalar: invalid arguments");
    Dev d = make_dev(*g);
    int64_t n = (int64_t)g->nx * g->ny * g->nz;
    F3 c = {center[0], center[1], center[2]};
    FFX_DISPATCH_STORAGE(storage, T,
        seed_scalar_kernel<T><<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(d, c, radius, scale,
                                                                                   scale != 1.0f, (T*)out));
    return launch_status("seed_scalar_kernel");
}

int ffx_seed_faces(const FfxGrid* g, int storage, const float base[3], float angular, void* u, void* v,
                   void* w, void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && base && u && v && w, "ffx_seed_faces: invalid arguments");
    Dev d = make_dev(*g);
    int64_t n = (int64_t)(g->nx + 1) * g->ny * g->nz + (int64_t)g->nx * (g->ny + 1) * g->nz +
                (int64_t)g->nx * g->ny * (g->nz + 1);
    F3 b = {base[0], base[1], base[2]};
    FFX_DISPATCH_STORAGE(storage, T,
        seed_faces_kernel<T><<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(d, b, angular, (T*)u, (T*)v,
                                                                                  (T*)w));
    return launch_status("seed_faces_kernel");
}

int ffx_raster_colliders(const FfxGrid* g, const double extent[3], int count, const double* rows13,
                         uint8_t* solid, void* stream) {
    FFX_REQUIRE(grid_ok(g) && extent && solid && count >= 0 && count <= 64 && (count == 0 || rows13),
                "ffx_raster_colliders: invalid arguments");
    Dev d = make_dev(*g);
    int64_t n = (int64_t)g->nx * g->ny * g->nz;
    raster_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(d, extent[0], extent[1], extent[2], count,
                                                                          rows13, solid);
    return launch_status("raster_kernel");
}

int ffx_dilate_mask(const FfxGrid* g, const uint8_t* solid, uint8_t* halo, void* stream) {
    FFX_REQUIRE(grid_ok(g) && solid && halo && solid != halo, "ffx_dilate_mask: invalid arguments");
    Dev d = make_dev(*g);
    int64_t n = (int64_t)g->nx * g->ny * g->nz;
    dilate_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(d, solid, halo);
    return launch_status("dilate_kernel");
}

// Inputs a, over all 2^32 bit patterns, whose div_rn quotient by b differs
// from the IEEE division a / b (NaN against NaN counts as equal): count[0]
// those in div_rn's exact class (+-0, +-inf, NaN, 2^-96 <= |a| <= 2^96),
// count[1] the others.
__global__ void __launch_bounds__(256) division_check_kernel(float b, float y, unsigned long long* count) {
    unsigned long long bad[2] = {0, 0};
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < (1ull << 32); k += stride) {
        const float a = __uint_as_float((uint32_t)k);
        const float q = div_rn(a, b, y), ref = a / b;
        const bool same = __float_as_uint(q) == __float_as_uint(ref) || (q != q && ref != ref);
        const float m = fabsf(a);
        const bool exact_class = m == 0.f || m == INFINITY || a != a || (m >= 0x1p-96f && m <= 0x1p96f);
        bad[exact_class ? 0 : 1] += !same;
    }
    for (int j = 0; j < 2; ++j) {
        unsigned long long v = bad[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(count + j, v);
    }
}

int ffx_division_mismatches(float divisor, int64_t* count, void* stream) {
    FFX_REQUIRE(count && divisor >= 0x1p-30f && divisor <= 0x1p30f, "ffx_division_mismatches: invalid arguments");
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(cudaMemsetAsync(count, 0, 2 * sizeof(int64_t), st), "ffx_division_mismatches: clear");
    if (e) return e;
    division_check_kernel<<<148 * 8, 256, 0, st>>>(divisor, 1.f / divisor,
                                                    reinterpret_cast<unsigned long long*>(count));
    return launch_status("division_check_kernel");
}

int ffx_halo_clearance(const FfxGrid* g, const uint8_t* solid, uint8_t* halo, uint8_t* clear, void* stream) {
    FFX_REQUIRE(grid_ok(g) && solid && halo && clear && solid != halo && solid != clear && halo != clear,
                "ffx_halo_clearance: invalid arguments");
    Dev d = make_dev(*g);
    const dim3 grid((unsigned)((g->nx + kHX - 1) / kHX), (unsigned)((g->ny + kHY - 1) / kHY),
                    (unsigned)((g->nz + kHZ - 1) / kHZ));
    halo_clear_kernel<<<grid, dim3(kHX, kHY), 0, as_stream(stream)>>>(d, solid, halo, clear);
    return launch_status("halo_clear_kernel");
}

int ffx_clearance(const FfxGrid* g, const uint8_t* halo, uint8_t* clear, void* stream) {
    FFX_REQUIRE(grid_ok(g) && halo && clear && halo != clear, "ffx_clearance: invalid arguments");
    Dev d = make_dev(*g);
    clearance_kernel<<<cell_grid(g->nx, g->ny, g->nz), cell_block(), 0, as_stream(stream)>>>(d, halo, clear);
    return launch_status("clearance_kernel");
}

int ffx_solid_clear(const FfxGrid* g, int storage, const uint8_t* solid, const void* in, void* out,
                    void* stream) {
    FFX_REQUIRE(grid_ok(g) && storage_ok(storage) && solid && in && out, "ffx_solid_clear: invalid arguments");
    int64_t n = (int64_t)g->nx * g->ny * g->nz;
    FFX_DISPATCH_STORAGE(storage, T,
        solid_clear_kernel<T><<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(n, solid, (const T*)in, (T*)out));
    return launch_status("solid_clear_kernel");
}

int ffx_max_abs(int64_t count, int storage, const void* x, float* out, void* stream) {
    FFX_REQUIRE(count >= 0 && storage_ok(storage) && out && (count == 0 || x), "ffx_max_abs: invalid arguments");
    cudaStream_t s = as_stream(stream);
    int st = cuda_status(cudaMemsetAsync(out, 0, sizeof(float), s), "ffx_max_abs memset");
    if (st || count == 0) return st;
    int64_t b = (count + 255) / 256;
    unsigned blocks = (unsigned)(b < 148 * 16 ? b : 148 * 16);
    FFX_DISPATCH_STORAGE(storage, T, max_abs_kernel<T><<<blocks, 256, 0, s>>>(count, (const T*)x, out));
    return launch_status("max_abs_kernel");
}

size_t ffx_divergence_stats_workspace(int64_t count) {
    return (size_t)stats::blocks(count < 1 ? 1 : count) * 6 * sizeof(double);
}

int ffx_divergence_stats(int64_t count, const float* before, const float* after, double* out, void* workspace,
                         size_t workspace_bytes, void* stream) {
    FFX_REQUIRE(count >= 1 && before && after && out, "ffx_divergence_stats: invalid arguments");
    size_t need = ffx_divergence_stats_workspace(count);
    FFX_REQUIRE(workspace && workspace_bytes >= need,
                "ffx_divergence_stats: workspace of %zu bytes required, %zu given", need, workspace_bytes);
    FFX_REQUIRE(((uintptr_t)workspace & 7) == 0, "ffx_divergence_stats: workspace must be 8-byte aligned");
    stats::launch(count, before, after, (double*)workspace, out, as_stream(stream));
    return launch_status("divergence stats kernels");
}

}  // extern "C"
