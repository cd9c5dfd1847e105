// Sparse brick path: a brick pool (host topology) and the pressure projection
// on the cells of active bricks only, with the dense layout as its twin.
//
// Counterpart of FluxFX's native prototype (FluxFX_Source/native/bricks.hpp,
// arena.hpp, projection.mm:15-120): domains whose work is confined to part of
// the grid store and sweep only the bricks that part touches.
//
// Topology (host, BrickPool): a fixed-capacity table of brick coordinates ->
// storage slots. Open addressing with linear probing over a power-of-two table
// of at least twice the capacity, tombstones on removal, slots from a LIFO free
// list (a removed slot is the next one handed out), an active list with O(1)
// removal, and an atomic box activation that checks capacity before changing
// anything. All storage is reserved at creation.
//
// Device layout of a level (SpLevel): n^3 cells (n a multiple of the brick
// side S, S = 8 or 16). A cell field stores S^3 values per brick slot, local
// index (z * S + y) * S + x; a face field stores, per axis, the faces at the
// lower side of each cell of the brick (faces 0 .. S - 1 of the brick along
// the axis), so every interior face has exactly one owner; the faces on the
// domain's upper walls (index n) are always zero and not stored. The dense
// twin stores n^3 cells and (n + 1) n^2 faces per axis in x-fast order. A
// brick is active when any cell within one cell of the solve region lies in
// it, so every face of a solve cell has its owner. The kernels are templated
// on the layout and do the same arithmetic in the same order in both, so the
// sparse results equal the dense ones bit for bit on the solve region.
//
// Units are cells (h = 1) and the pressure is the impulse q = dt p, as in the
// prototype: Jacobi with omega = 2/3 over the in-domain neighbours, residual
// rhs - L q, restriction 1/2 * the sum of the eight children (four times their
// average: the coarse spacing is doubled), trilinear prolongation (clamped).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "ffx_host.cuh"

// ------------------------------------------------------------- topology
struct FfxBrickPool {
    struct Entry { int32_t x, y, z, slot; };   // slot: -1 empty, -2 tombstone, >= 0 live
    std::vector<Entry> table;
    std::vector<int32_t> coords;                // 3 per slot
    std::vector<uint32_t> position;             // slot -> index in `active`
    std::vector<uint32_t> free_slots;           // LIFO
    std::vector<uint32_t> active;
    uint32_t capacity = 0;

    static uint64_t mix(int32_t x, int32_t y, int32_t z) {
        // a multiply-xorshift mix of the three coordinates
        uint64_t h = (uint64_t)(uint32_t)x * 0x9e3779b97f4a7c15ull;
        h ^= (uint64_t)(uint32_t)y * 0xbf58476d1ce4e5b9ull + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)z * 0x94d049bb133111ebull + (h << 6) + (h >> 2);
        h ^= h >> 31;
        h *= 0xd6e8feb86659fd93ull;
        return h ^ (h >> 32);
    }
    // the entry holding (x, y, z), or the first empty entry of its probe chain
    size_t find(int32_t x, int32_t y, int32_t z) const {
        const size_t m = table.size() - 1;
        size_t pos = mix(x, y, z) & m;
        for (size_t k = 0; k < table.size(); ++k, pos = (pos + 1) & m) {
            const Entry& e = table[pos];
            if (e.slot == -1 || (e.slot >= 0 && e.x == x && e.y == y && e.z == z)) return pos;
        }
        return table.size();
    }
    int32_t lookup(int32_t x, int32_t y, int32_t z) const {
        const size_t i = find(x, y, z);
        return i < table.size() && table[i].slot >= 0 ? table[i].slot : -1;
    }
};

// ------------------------------------------------------------- arena
// A GPU-independent suballocator of one buffer (FluxFX_Source/native/arena.hpp):
// spans aligned to 256 bytes, first fit over the free spans in address order,
// adjacent free spans merged on release, handles unique across all arenas and
// never reused, at most 65536 live spans.
struct FfxArena {
    struct Span { uint64_t offset, bytes, requested; };
    uint64_t capacity = 0, used = 0, peak = 0, allocations = 0;
    std::vector<Span> free_spans;       // sorted by offset, disjoint, not adjacent
    std::vector<std::pair<uint64_t, Span>> live;   // (handle, span), sorted by handle
};

namespace ffx {
namespace {

std::atomic<uint64_t> g_next_handle{1};

FfxArena::Span* find_live(FfxArena* A, uint64_t id) {
    auto it = std::lower_bound(A->live.begin(), A->live.end(), id,
                               [](const std::pair<uint64_t, FfxArena::Span>& e, uint64_t v) { return e.first < v; });
    return it != A->live.end() && it->first == id ? &it->second : nullptr;
}

constexpr int32_t kCoordLimit = 1048576;   // coordinates in [-2^20, 2^20 - 1]

bool coord_ok(int32_t x, int32_t y, int32_t z) {
    return x >= -kCoordLimit && x < kCoordLimit && y >= -kCoordLimit && y < kCoordLimit && z >= -kCoordLimit &&
           z < kCoordLimit;
}

int activate_one(FfxBrickPool* P, int32_t x, int32_t y, int32_t z, int32_t* slot) {
    const int32_t prior = P->lookup(x, y, z);
    if (prior >= 0) {
        *slot = prior;
        return FFX_OK;
    }
    if (P->free_slots.empty()) return fail(FFX_ERR_INVALID, "ffx_bricks_activate: brick pool capacity exhausted");
    const size_t m = P->table.size() - 1;
    size_t pos = FfxBrickPool::mix(x, y, z) & m;
    while (P->table[pos].slot >= 0) pos = (pos + 1) & m;    // first empty or tombstone
    const uint32_t s = P->free_slots.back();
    P->free_slots.pop_back();
    P->table[pos] = {x, y, z, (int32_t)s};
    P->coords[3 * s] = x;
    P->coords[3 * s + 1] = y;
    P->coords[3 * s + 2] = z;
    P->position[s] = (uint32_t)P->active.size();
    P->active.push_back(s);
    *slot = (int32_t)s;
    return FFX_OK;
}

// ------------------------------------------------------------- device side
struct SpLevel {
    int n, side, lg;          // cells per axis, brick side, log2(side)
    int grid;                 // bricks per axis
    int mode;                 // solve region: 0 all, 1 central box, 2 two boxes
    const int32_t* map;       // grid^3 slots (-1: inactive); sparse only
    const int32_t* active;    // active slots; sparse only
    const int32_t* coords;    // 3 per slot; sparse only
    int count;                // active bricks (sparse) or 1 (dense)
};

__host__ __device__ __forceinline__ bool solve_cell(int x, int y, int z, int n, int mode) {
    if (x < 0 || y < 0 || z < 0 || x >= n || y >= n || z >= n) return false;
    if (mode != 1 && mode != 2) return true;
    auto box = [&](int lo, int hi) { return x >= lo && y >= lo && z >= lo && x < hi && y < hi && z < hi; };
    return mode == 1 ? box(n / 4, 3 * n / 4) : (box(n / 8, 3 * n / 8) || box(5 * n / 8, 7 * n / 8));
}

template <bool SP>
__device__ __forceinline__ int cell_index(const SpLevel& L, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= L.n || y >= L.n || z >= L.n) return -1;
    if (!SP) return (z * L.n + y) * L.n + x;
    const int m = L.side - 1, g = L.grid;
    const int slot = __ldg(L.map + ((z >> L.lg) * g + (y >> L.lg)) * g + (x >> L.lg));
    if (slot < 0) return -1;
    return (slot << (3 * L.lg)) + (((z & m) << L.lg | (y & m)) << L.lg | (x & m));
}

// face (x, y, z) of axis a: between cells c - e_a and c; index n along a is a wall
template <bool SP>
__device__ __forceinline__ int face_index(const SpLevel& L, int a, int x, int y, int z) {
    if (!SP) {
        const int dx = L.n + (a == 0), dy = L.n + (a == 1), dz = L.n + (a == 2);
        if (x < 0 || y < 0 || z < 0 || x >= dx || y >= dy || z >= dz) return -1;
        return (z * dy + y) * dx + x;
    }
    return cell_index<true>(L, x, y, z);      // the wall face at index n falls outside: -1
}

template <bool SP>
__device__ __forceinline__ float pressure_at(const SpLevel& L, const float* q, int x, int y, int z) {
    if (!solve_cell(x, y, z, L.n, L.mode)) return 0.f;
    const int i = cell_index<SP>(L, x, y, z);
    return i < 0 ? 0.f : __ldg(q + i);
}

template <bool SP>
__device__ __forceinline__ float face_at(const SpLevel& L, const float* u, int faces, int a, int x, int y, int z) {
    const int i = face_index<SP>(L, a, x, y, z);
    return i < 0 ? 0.f : __ldg(u + (size_t)a * faces + i);
}

// Cell (or face-owner) coordinates of storage index i; false past the end.
template <bool SP>
__device__ __forceinline__ bool stored_cell(const SpLevel& L, int i, int& x, int& y, int& z) {
    if (SP) {
        const int per = 1 << (3 * L.lg);
        const int b = i >> (3 * L.lg);
        if (b >= L.count) return false;
        const int slot = __ldg(L.active + b), j = i & (per - 1), m = L.side - 1;
        x = (__ldg(L.coords + 3 * slot) << L.lg) + (j & m);
        y = (__ldg(L.coords + 3 * slot + 1) << L.lg) + ((j >> L.lg) & m);
        z = (__ldg(L.coords + 3 * slot + 2) << L.lg) + (j >> (2 * L.lg));
        return true;
    }
    const int n = L.n;
    if (i >= n * n * n) return false;
    x = i % n;
    y = (i / n) % n;
    z = i / (n * n);
    return true;
}

// Cells touched by a launch: active bricks x S^3, or n^3.
template <bool SP>
inline int cell_count(const SpLevel& L) {
    return SP ? (L.count << (3 * L.lg)) : L.n * L.n * L.n;
}

template <bool SP>
__global__ void sp_divergence_kernel(SpLevel L, const float* __restrict__ u, int faces, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (!stored_cell<SP>(L, i, x, y, z)) return;
    float v = 0.f;
    if (solve_cell(x, y, z, L.n, L.mode)) {
        v = v + (face_at<SP>(L, u, faces, 0, x + 1, y, z) - face_at<SP>(L, u, faces, 0, x, y, z));
        v = v + (face_at<SP>(L, u, faces, 1, x, y + 1, z) - face_at<SP>(L, u, faces, 1, x, y, z));
        v = v + (face_at<SP>(L, u, faces, 2, x, y, z + 1) - face_at<SP>(L, u, faces, 2, x, y, z));
    }
    out[cell_index<SP>(L, x, y, z)] = v;
}

template <bool SP>
__global__ void sp_jacobi_kernel(SpLevel L, const float* __restrict__ old, const float* __restrict__ rhs,
                                 float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (!stored_cell<SP>(L, i, x, y, z)) return;
    const int c = cell_index<SP>(L, x, y, z);
    if (!solve_cell(x, y, z, L.n, L.mode)) {
        out[c] = 0.f;
        return;
    }
    float sum = 0.f, diag = 0.f;
    const int nb[6][3] = {{x - 1, y, z}, {x + 1, y, z}, {x, y - 1, z}, {x, y + 1, z}, {x, y, z - 1}, {x, y, z + 1}};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int vx = nb[k][0], vy = nb[k][1], vz = nb[k][2];
        if (vx >= 0 && vy >= 0 && vz >= 0 && vx < L.n && vy < L.n && vz < L.n) {
            diag = diag + 1.f;
            sum = sum + pressure_at<SP>(L, old, vx, vy, vz);
        }
    }
    const float a = 2.f / 3.f;
    out[c] = __ldg(old + c) * (1.f - a) + ((sum - __ldg(rhs + c)) / diag) * a;
}

template <bool SP>
__global__ void sp_residual_kernel(SpLevel L, const float* __restrict__ q, const float* __restrict__ rhs,
                                   float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (!stored_cell<SP>(L, i, x, y, z)) return;
    const int c = cell_index<SP>(L, x, y, z);
    if (!solve_cell(x, y, z, L.n, L.mode)) {
        out[c] = 0.f;
        return;
    }
    const float qc = __ldg(q + c);
    float lap = 0.f;
    const int nb[6][3] = {{x - 1, y, z}, {x + 1, y, z}, {x, y - 1, z}, {x, y + 1, z}, {x, y, z - 1}, {x, y, z + 1}};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int vx = nb[k][0], vy = nb[k][1], vz = nb[k][2];
        if (vx >= 0 && vy >= 0 && vz >= 0 && vx < L.n && vy < L.n && vz < L.n)
            lap = lap + (pressure_at<SP>(L, q, vx, vy, vz) - qc);
    }
    out[c] = __ldg(rhs + c) - lap;
}

// Faces of axis a: sparse, the S^3 faces owned by each active brick; dense, all.
template <bool SP>
__global__ void sp_gradient_kernel(SpLevel L, int a, const float* __restrict__ u, const float* __restrict__ q,
                                   int faces, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (SP) {
        if (!stored_cell<true>(L, i, x, y, z)) return;
    } else {
        const int dx = L.n + (a == 0), dy = L.n + (a == 1), dz = L.n + (a == 2);
        if (i >= dx * dy * dz) return;
        x = i % dx;
        y = (i / dx) % dy;
        z = i / (dx * dy);
    }
    const int c[3] = {x, y, z};
    const int lx = x - (a == 0), ly = y - (a == 1), lz = z - (a == 2);
    float v = 0.f;
    if (c[a] > 0 && c[a] < L.n && (solve_cell(x, y, z, L.n, L.mode) || solve_cell(lx, ly, lz, L.n, L.mode)))
        v = __ldg(u + (size_t)a * faces + face_index<SP>(L, a, x, y, z)) -
            (pressure_at<SP>(L, q, x, y, z) - pressure_at<SP>(L, q, lx, ly, lz));
    out[(size_t)a * faces + face_index<SP>(L, a, x, y, z)] = v;
}

// coarse rhs = 1/2 * sum of the eight children's residuals (4 x their average)
template <bool SF, bool SC>
__global__ void sp_restrict_kernel(SpLevel F, const float* __restrict__ fine, SpLevel Cl, float* __restrict__ coarse) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (!stored_cell<SC>(Cl, i, x, y, z)) return;
    float sum = 0.f;
    if (solve_cell(x, y, z, Cl.n, Cl.mode))
        for (int oz = 0; oz < 2; ++oz)
            for (int oy = 0; oy < 2; ++oy)
                for (int ox = 0; ox < 2; ++ox) sum = sum + pressure_at<SF>(F, fine, 2 * x + ox, 2 * y + oy, 2 * z + oz);
    coarse[cell_index<SC>(Cl, x, y, z)] = sum * 0.5f;
}

// fine += trilinear (clamped) interpolation of the coarse correction
template <bool SF, bool SC>
__global__ void sp_prolong_kernel(SpLevel Cl, const float* __restrict__ coarse, SpLevel F, float* __restrict__ fine) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (!stored_cell<SF>(F, i, x, y, z)) return;
    if (!solve_cell(x, y, z, F.n, F.mode)) return;
    const float px = ((float)x + 0.5f) * 0.5f - 0.5f, py = ((float)y + 0.5f) * 0.5f - 0.5f,
                pz = ((float)z + 0.5f) * 0.5f - 0.5f;
    const float bx = floorf(px), by = floorf(py), bz = floorf(pz);
    const float fx = px - bx, fy = py - by, fz = pz - bz;
    const int ix = (int)bx, iy = (int)by, iz = (int)bz, m = Cl.n - 1;
    float sum = 0.f;
    for (int oz = 0; oz < 2; ++oz)
        for (int oy = 0; oy < 2; ++oy)
            for (int ox = 0; ox < 2; ++ox) {
                const float wx = ox ? fx : 1.f - fx, wy = oy ? fy : 1.f - fy, wz = oz ? fz : 1.f - fz;
                const int qx = min(max(ix + ox, 0), m), qy = min(max(iy + oy, 0), m), qz = min(max(iz + oz, 0), m);
                sum = sum + wx * wy * wz * pressure_at<SC>(Cl, coarse, qx, qy, qz);
            }
    const int c = cell_index<SF>(F, x, y, z);
    fine[c] = fine[c] + sum;
}

SpLevel to_level(const FfxSparseLevel* l) {
    SpLevel L;
    L.n = l->n;
    L.side = l->side;
    L.lg = l->side == 16 ? 4 : 3;
    L.grid = l->n / l->side;
    L.mode = l->mode;
    L.map = l->map;
    L.active = l->active;
    L.coords = l->coords;
    L.count = l->sparse ? l->count : 1;
    return L;
}

bool level_ok(const FfxSparseLevel* l) {
    return l && (l->side == 8 || l->side == 16) && l->n >= l->side && l->n % l->side == 0 && l->n <= 1024 &&
           l->mode >= 0 && l->mode <= 2 && (!l->sparse || (l->map && l->active && l->coords && l->count >= 0 &&
                                                           l->count <= (l->n / l->side) * (l->n / l->side) *
                                                                            (l->n / l->side)));
}

inline unsigned blocks256(int n) { return (unsigned)((n + 255) / 256); }

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" {

// ---------------------------------------------------------- pool (host)
int ffx_bricks_create(uint32_t capacity, FfxBrickPool** out) {
    FFX_REQUIRE(out && capacity >= 1 && capacity <= 262144, "ffx_bricks_create: capacity must be 1..262144");
    FfxBrickPool* P = new FfxBrickPool;
    size_t n = 2;
    while (n < (size_t)capacity * 2) n *= 2;
    P->table.assign(n, FfxBrickPool::Entry{0, 0, 0, -1});
    P->coords.assign((size_t)capacity * 3, 0);
    P->position.assign(capacity, 0);
    P->free_slots.reserve(capacity);
    P->active.reserve(capacity);
    for (uint32_t s = capacity; s > 0; --s) P->free_slots.push_back(s - 1);
    P->capacity = capacity;
    *out = P;
    return FFX_OK;
}

int ffx_bricks_destroy(FfxBrickPool* P) {
    delete P;
    return FFX_OK;
}

int ffx_bricks_lookup(const FfxBrickPool* P, int32_t x, int32_t y, int32_t z, int32_t* slot) {
    FFX_REQUIRE(P && slot, "ffx_bricks_lookup: invalid arguments");
    FFX_REQUIRE(coord_ok(x, y, z), "ffx_bricks_lookup: brick coordinates must lie in [-1048576, 1048575]");
    *slot = P->lookup(x, y, z);
    return FFX_OK;
}

int ffx_bricks_activate(FfxBrickPool* P, int32_t x, int32_t y, int32_t z, int32_t* slot) {
    FFX_REQUIRE(P && slot, "ffx_bricks_activate: invalid arguments");
    FFX_REQUIRE(coord_ok(x, y, z), "ffx_bricks_activate: brick coordinates must lie in [-1048576, 1048575]");
    return activate_one(P, x, y, z, slot);
}

int ffx_bricks_deactivate(FfxBrickPool* P, int32_t x, int32_t y, int32_t z, int32_t* was_active) {
    FFX_REQUIRE(P && was_active, "ffx_bricks_deactivate: invalid arguments");
    FFX_REQUIRE(coord_ok(x, y, z), "ffx_bricks_deactivate: brick coordinates must lie in [-1048576, 1048575]");
    const size_t i = P->find(x, y, z);
    if (i >= P->table.size() || P->table[i].slot < 0) {
        *was_active = 0;
        return FFX_OK;
    }
    const uint32_t s = (uint32_t)P->table[i].slot, pos = P->position[s], last = P->active.back();
    P->active[pos] = last;
    P->position[last] = pos;
    P->active.pop_back();
    P->table[i].slot = -2;
    P->free_slots.push_back(s);
    *was_active = 1;
    return FFX_OK;
}

int ffx_bricks_neighbors(const FfxBrickPool* P, int32_t x, int32_t y, int32_t z, int32_t out[6]) {
    FFX_REQUIRE(P && out, "ffx_bricks_neighbors: invalid arguments");
    FFX_REQUIRE(coord_ok(x, y, z), "ffx_bricks_neighbors: brick coordinates must lie in [-1048576, 1048575]");
    const int32_t d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int k = 0; k < 6; ++k) out[k] = P->lookup(x + d[k][0], y + d[k][1], z + d[k][2]);
    return FFX_OK;
}

int ffx_bricks_activate_box(FfxBrickPool* P, const int32_t lo[3], const int32_t extent[3]) {
    FFX_REQUIRE(P && lo && extent, "ffx_bricks_activate_box: invalid arguments");
    FFX_REQUIRE(coord_ok(lo[0], lo[1], lo[2]), "ffx_bricks_activate_box: brick coordinates must lie in [-1048576, 1048575]");
    for (int a = 0; a < 3; ++a)
        FFX_REQUIRE(extent[a] >= 1 && extent[a] <= 4096, "ffx_bricks_activate_box: box extent must be 1..4096 per axis");
    FFX_REQUIRE(coord_ok(lo[0] + extent[0] - 1, lo[1] + extent[1] - 1, lo[2] + extent[2] - 1),
                "ffx_bricks_activate_box: brick coordinates must lie in [-1048576, 1048575]");
    FFX_REQUIRE((uint64_t)extent[0] * extent[1] * extent[2] <= P->capacity, "ffx_bricks_activate_box: box exceeds pool capacity");
    // preflight: nothing changes unless every missing brick fits
    uint64_t needed = 0;
    for (int z = 0; z < extent[2]; ++z)
        for (int y = 0; y < extent[1]; ++y)
            for (int x = 0; x < extent[0]; ++x) needed += P->lookup(lo[0] + x, lo[1] + y, lo[2] + z) < 0;
    FFX_REQUIRE(needed <= P->free_slots.size(), "ffx_bricks_activate_box: brick pool capacity exhausted");
    int32_t slot;
    for (int z = 0; z < extent[2]; ++z)
        for (int y = 0; y < extent[1]; ++y)
            for (int x = 0; x < extent[0]; ++x) activate_one(P, lo[0] + x, lo[1] + y, lo[2] + z, &slot);
    return FFX_OK;
}

int ffx_bricks_stats(const FfxBrickPool* P, FfxBrickStats* out) {
    FFX_REQUIRE(P && out, "ffx_bricks_stats: invalid arguments");
    out->capacity = P->capacity;
    out->active = (uint32_t)P->active.size();
    out->metadata_bytes = (uint64_t)P->table.capacity() * sizeof(FfxBrickPool::Entry) +
                          (uint64_t)P->coords.capacity() * sizeof(int32_t) +
                          (uint64_t)(P->position.capacity() + P->free_slots.capacity() + P->active.capacity()) *
                              sizeof(uint32_t);
    return FFX_OK;
}

// active slots in activation order (swap-removal keeps it compact) and, per
// slot, its coordinates
int ffx_bricks_active(const FfxBrickPool* P, int32_t* slots, int32_t* coords_by_slot, uint32_t room) {
    FFX_REQUIRE(P && slots && coords_by_slot && room >= P->capacity, "ffx_bricks_active: room for capacity entries");
    for (size_t k = 0; k < P->active.size(); ++k) slots[k] = (int32_t)P->active[k];
    std::memcpy(coords_by_slot, P->coords.data(), sizeof(int32_t) * 3 * (size_t)P->capacity);
    return FFX_OK;
}

// ---------------------------------------------------------- arena (host)
int ffx_arena_create(uint64_t capacity, FfxArena** out) {
    FFX_REQUIRE(out && capacity > 0 && capacity % 256 == 0, "ffx_arena_create: capacity must be a positive multiple of 256");
    FfxArena* A = new FfxArena;
    A->capacity = capacity;
    A->free_spans.push_back({0, capacity, capacity});
    *out = A;
    return FFX_OK;
}

int ffx_arena_destroy(FfxArena* A) {
    delete A;
    return FFX_OK;
}

int ffx_arena_allocate(FfxArena* A, uint64_t bytes, uint64_t* id) {
    FFX_REQUIRE(A && id, "ffx_arena_allocate: invalid arguments");
    FFX_REQUIRE(bytes > 0 && bytes <= A->capacity, "ffx_arena_allocate: allocation is empty or exceeds the arena");
    FFX_REQUIRE(A->live.size() < 65536, "ffx_arena_allocate: 65536 live allocations");
    const uint64_t aligned = (bytes + 255) & ~uint64_t(255);
    for (size_t i = 0; i < A->free_spans.size(); ++i) {
        FfxArena::Span& f = A->free_spans[i];
        if (f.bytes < aligned) continue;
        const uint64_t handle = g_next_handle.fetch_add(1);
        const FfxArena::Span span{f.offset, aligned, bytes};
        f.offset += aligned;
        f.bytes -= aligned;
        if (!f.bytes) A->free_spans.erase(A->free_spans.begin() + (long)i);
        A->live.emplace_back(handle, span);        // handles increase: the list stays sorted
        A->used += aligned;
        A->peak = std::max(A->peak, A->used);
        A->allocations += 1;
        *id = handle;
        return FFX_OK;
    }
    return fail(FFX_ERR_INVALID, "ffx_arena_allocate: arena exhausted or fragmented; release allocations first");
}

int ffx_arena_get(const FfxArena* A, uint64_t id, uint64_t* offset, uint64_t* bytes, uint64_t* requested) {
    FFX_REQUIRE(A && offset && bytes && requested, "ffx_arena_get: invalid arguments");
    const FfxArena::Span* s = find_live(const_cast<FfxArena*>(A), id);
    FFX_REQUIRE(s, "ffx_arena_get: unknown, released or foreign allocation handle");
    *offset = s->offset;
    *bytes = s->bytes;
    *requested = s->requested;
    return FFX_OK;
}

int ffx_arena_release(FfxArena* A, uint64_t id) {
    FFX_REQUIRE(A, "ffx_arena_release: invalid arguments");
    auto it = std::lower_bound(A->live.begin(), A->live.end(), id,
                               [](const std::pair<uint64_t, FfxArena::Span>& e, uint64_t v) { return e.first < v; });
    FFX_REQUIRE(it != A->live.end() && it->first == id,
                "ffx_arena_release: unknown, released or foreign allocation handle");
    const FfxArena::Span span = it->second;
    A->live.erase(it);
    auto pos = std::lower_bound(A->free_spans.begin(), A->free_spans.end(), span.offset,
                                [](const FfxArena::Span& f, uint64_t o) { return f.offset < o; });
    pos = A->free_spans.insert(pos, FfxArena::Span{span.offset, span.bytes, span.bytes});
    // merge with the following and the preceding free span
    if (pos + 1 != A->free_spans.end() && pos->offset + pos->bytes == (pos + 1)->offset) {
        pos->bytes += (pos + 1)->bytes;
        A->free_spans.erase(pos + 1);
    }
    if (pos != A->free_spans.begin() && (pos - 1)->offset + (pos - 1)->bytes == pos->offset) {
        (pos - 1)->bytes += pos->bytes;
        A->free_spans.erase(pos);
    }
    A->used -= span.bytes;
    return FFX_OK;
}

int ffx_arena_stats(const FfxArena* A, FfxArenaStats* out) {
    FFX_REQUIRE(A && out, "ffx_arena_stats: invalid arguments");
    out->capacity = A->capacity;
    out->used = A->used;
    out->peak = A->peak;
    out->allocations = A->allocations;
    out->live = A->live.size();
    uint64_t largest = 0;
    for (const auto& f : A->free_spans) largest = std::max(largest, f.bytes);
    out->largest_free = largest;
    return FFX_OK;
}

// ------------------------------------------------------------ projection
#define FFX_SP_DISPATCH(l, SP, ...)                     \
    do {                                                \
        if ((l)->sparse) { constexpr bool SP = true; __VA_ARGS__; }   \
        else { constexpr bool SP = false; __VA_ARGS__; }              \
    } while (0)

int ffx_sparse_divergence(const FfxSparseLevel* l, const float* u, int32_t faces, float* out, void* stream) {
    FFX_REQUIRE(level_ok(l) && u && out && faces >= 1, "ffx_sparse_divergence: invalid arguments");
    SpLevel L = to_level(l);
    FFX_SP_DISPATCH(l, SP, sp_divergence_kernel<SP><<<blocks256(cell_count<SP>(L)), 256, 0, as_stream(stream)>>>(L, u, faces, out));
    return launch_status("sp_divergence_kernel");
}

int ffx_sparse_jacobi(const FfxSparseLevel* l, const float* old, const float* rhs, float* out, void* stream) {
    FFX_REQUIRE(level_ok(l) && old && rhs && out && old != out, "ffx_sparse_jacobi: invalid arguments");
    SpLevel L = to_level(l);
    FFX_SP_DISPATCH(l, SP, sp_jacobi_kernel<SP><<<blocks256(cell_count<SP>(L)), 256, 0, as_stream(stream)>>>(L, old, rhs, out));
    return launch_status("sp_jacobi_kernel");
}

int ffx_sparse_residual(const FfxSparseLevel* l, const float* q, const float* rhs, float* out, void* stream) {
    FFX_REQUIRE(level_ok(l) && q && rhs && out && q != out, "ffx_sparse_residual: invalid arguments");
    SpLevel L = to_level(l);
    FFX_SP_DISPATCH(l, SP, sp_residual_kernel<SP><<<blocks256(cell_count<SP>(L)), 256, 0, as_stream(stream)>>>(L, q, rhs, out));
    return launch_status("sp_residual_kernel");
}

int ffx_sparse_gradient(const FfxSparseLevel* l, const float* u, const float* q, int32_t faces, float* out,
                        void* stream) {
    FFX_REQUIRE(level_ok(l) && u && q && out && u != out && faces >= 1, "ffx_sparse_gradient: invalid arguments");
    SpLevel L = to_level(l);
    for (int a = 0; a < 3; ++a) {
        const int count = l->sparse ? cell_count<true>(L) : (L.n + 1) * L.n * L.n;
        FFX_SP_DISPATCH(l, SP, sp_gradient_kernel<SP><<<blocks256(count), 256, 0, as_stream(stream)>>>(L, a, u, q, faces, out));
    }
    return launch_status("sp_gradient_kernel");
}

int ffx_sparse_restrict(const FfxSparseLevel* fine, const float* residual, const FfxSparseLevel* coarse,
                        float* coarse_rhs, void* stream) {
    FFX_REQUIRE(level_ok(fine) && level_ok(coarse) && residual && coarse_rhs && coarse->n * 2 == fine->n &&
                coarse->mode == fine->mode, "ffx_sparse_restrict: invalid arguments");
    SpLevel F = to_level(fine), Cl = to_level(coarse);
    cudaStream_t st = as_stream(stream);
    FFX_SP_DISPATCH(fine, SF, FFX_SP_DISPATCH(coarse, SC,
        (sp_restrict_kernel<SF, SC><<<blocks256(cell_count<SC>(Cl)), 256, 0, st>>>(F, residual, Cl, coarse_rhs))));
    return launch_status("sp_restrict_kernel");
}

int ffx_sparse_prolong(const FfxSparseLevel* coarse, const float* correction, const FfxSparseLevel* fine, float* q,
                       void* stream) {
    FFX_REQUIRE(level_ok(fine) && level_ok(coarse) && correction && q && coarse->n * 2 == fine->n &&
                coarse->mode == fine->mode, "ffx_sparse_prolong: invalid arguments");
    SpLevel F = to_level(fine), Cl = to_level(coarse);
    cudaStream_t st = as_stream(stream);
    FFX_SP_DISPATCH(fine, SF, FFX_SP_DISPATCH(coarse, SC,
        (sp_prolong_kernel<SF, SC><<<blocks256(cell_count<SF>(F)), 256, 0, st>>>(Cl, correction, F, q))));
    return launch_status("sp_prolong_kernel");
}

}  // extern "C"
