// Batched uneven domains: plan, V-cycle schedule, CUDA graph with device-side
// convergence, and the C ABI (ffx_batch_*). No counterpart in the reference,
// which runs one domain per solver object.
//
// A step of every domain is the single-domain step of backend/projected.py
// (149-202) on the collider path, issued as one persistent launch per pass
// over all domains (ffx_advect.cu / ffx_project.cu batched kernels):
//   face predictor, velocity transport (+ emitters, buoyancy, walls),
//   divergence, max |rhs| (+ zeroed pressure),
//   WHILE any domain unconverged { residual max, decision, one V-cycle of the
//                                  unconverged domains },
//   gradient (+ velocity maxima), scalar predictor, reverse, final scalars,
//   step end (next dt = min(dt_max, cfl * h / max |u|) on the device).
// The V-cycle of backend/solid_multigrid.py:46-65 is scheduled level by level
// over the domains that have the level; each domain keeps its own hierarchy
// depth, single-block tail, direct coarse solve and buffer roles, so the
// sequence of operations on each domain's data is exactly its stand-alone one.
#include <vector>

#include "ffx_host.cuh"
#include "ffx_batch.cuh"

struct FfxBatchPlan {
    int count = 0;
    std::vector<FfxBatchDomain> dom;
    char* ws = nullptr;
    int64_t ws_bytes = 0;
    ffx::BatchState* state = nullptr;
    struct Solve { double tol; int max_cycles; int warm; }* solve = nullptr;
    const void* rules = nullptr;
    struct Guard { int iterations; int tripped; long long total; }* guard = nullptr;   // solve-loop bound (device)
    struct Entry { int slot, X, Y, Z; };
    struct Launch {
        int kind;             // ffx::BatchKind, or kTail
        size_t offset;        // descriptor array in the workspace
        std::vector<Entry> entries;
    };
    // per parity: the passes before and after the solve; the solve body
    std::vector<Launch> pre[2], post[2], cycle;
    Launch resmax;
    Launch tune[ffx::kBatchKinds];
    int shape[ffx::kBatchKinds] = {};
    int grid[ffx::kBatchKinds] = {};
    int sms = 148;
    int parity = 0;
};

namespace ffx {
namespace {

constexpr int kTail = 100;        // launch kind of the single-block tail
constexpr int kShapes[4][2] = {{32, 8}, {64, 4}, {128, 2}, {16, 16}};

// Iterations of one solve loop after which it stops whatever the domains'
// state says (every domain stops by its own cycle cap, at most 256, first).
constexpr int kLoopCap = 300;

__global__ void batch_decide_kernel(BatchState* state, const FfxBatchPlan::Solve* solve, int count,
                                    FfxBatchPlan::Guard* guard, cudaGraphConditionalHandle handle) {
    __shared__ int iteration;
    if (threadIdx.x == 0) {
        iteration = ++guard->iterations;
        guard->total += 1;
    }
    __syncthreads();
    int open = 0;
    for (int d = threadIdx.x; d < count; d += blockDim.x) {
        BatchState& S = state[d];
        if (!S.done) {
            // while cycles < max and res > tol * scale: cycle
            const bool go = S.cycles < solve[d].max_cycles && (double)S.res > solve[d].tol * (double)S.scale;
            if (go) S.cycles += 1;
            else S.done = 1;
        }
        S.res = 0.f;
        open |= !S.done;
    }
    open = __syncthreads_or(open);
    if (open && iteration >= kLoopCap) {
        open = 0;
        if (threadIdx.x == 0) guard->tripped = 1;
        for (int d = threadIdx.x; d < count; d += blockDim.x) state[d].done = 1;
    }
    if (threadIdx.x == 0) cudaGraphSetConditional(handle, open ? 1u : 0u);
}

struct StepRule { double cell, cfl, dt_max; };

__global__ void batch_step_end_kernel(BatchState* state, const StepRule* rule, const FfxBatchPlan::Solve* solve,
                                      int count, FfxBatchPlan::Guard* guard) {
    if (threadIdx.x == 0) guard->iterations = 0;
    for (int d = threadIdx.x; d < count; d += blockDim.x) {
        BatchState& S = state[d];
        S.last_cycles = S.cycles;
        S.last_maxima[0] = S.maxima[0];
        S.last_maxima[1] = S.maxima[1];
        S.last_maxima[2] = S.maxima[2];
        S.total_cycles += S.cycles;
        S.steps += 1;
        S.time += S.dtd;
        S.last_dt = S.dt;
        S.last_dtd = S.dtd;
        const float umax = fmaxf(fmaxf(S.maxima[0], S.maxima[1]), S.maxima[2]);
        const double r = rule[d].cfl * rule[d].cell / (double)umax;
        S.dtd = umax > 0.f ? (r < rule[d].dt_max ? r : rule[d].dt_max) : rule[d].dt_max;
        S.dt = (float)S.dtd;
        // impulse warm start: the previous pressure times dt / previous dt when they differ
        const double ratio = S.dtd / S.last_dtd;
        S.pfactor = (float)ratio;
        S.pmode = solve[d].warm ? (fabs(ratio - 1.0) > 1e-6 ? 2 : 1) : 0;
        S.scale = 0.f;
        S.res = 0.f;
        S.cycles = 0;
        S.done = 0;
        S.maxima[0] = S.maxima[1] = S.maxima[2] = 0.f;
    }
}

// Clears the accumulators a tuning launch may have touched.
__global__ void batch_clear_kernel(BatchState* state, int count) {
    for (int d = threadIdx.x; d < count; d += blockDim.x) {
        state[d].scale = 0.f;
        state[d].res = 0.f;
        state[d].maxima[0] = state[d].maxima[1] = state[d].maxima[2] = 0.f;
    }
}

size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

int64_t cells_of(const FfxGraphLevel& lv) { return (int64_t)lv.nx * lv.ny * lv.nz; }

// Descriptor size of a launch kind.
size_t desc_size(int kind) {
    FfxBatchDomain z;
    memset(&z, 0, sizeof z);
    switch (kind) {
        case kPredictor: return batch::predictor_desc(z, nullptr);
        case kVelocity: return batch::velocity_desc(z, 0, nullptr);
        case kDivergence: return batch::divergence_desc(z, nullptr);
        case kScaleZero: return batch::scale_zero_desc(z, nullptr);
        case kGradient: return batch::gradient_desc(z, nullptr, nullptr, nullptr, nullptr);
        case kScalarPredictor:
        case kScalarReverse: return batch::scalar_xport_desc(z, 0, 0, nullptr);
        case kScalarFinal: return batch::scalar_final_desc(z, 0, nullptr);
        case kDirect: return batch::direct_desc(z, nullptr, nullptr);
        case kTail: return batch::tail_desc(z, 0, 0, nullptr);
        case kL0Smooth:
        case kL0ProlongSmooth:
        case kL0ResidualRestrict:
        case kL0ResidualMax: return batch::l0_desc(FfxGraphLevel{}, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
        default: return batch::level_desc(FfxGraphLevel{}, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    }
}

bool domain_ok(const FfxBatchDomain& D, int i, int D_first_pre, int D_first_post) {
    const FfxGrid& g = D.grid;
    if (!grid_ok(&g)) return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: invalid grid", i), false;
    if (!D.solid || !D.halo || !D.u || !D.v || !D.w || !D.bu || !D.bv || !D.bw || !D.after)
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: missing mask or face buffer", i), false;
    if (D.velocity_corrected && (!D.pu || !D.pv || !D.pw))
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: MacCormack velocity needs predictor faces", i), false;
    for (int c = 0; c < 2; ++c) {
        if (!D.density[c] || !D.temperature[c] || D.density[c] == D.density[1 - c] ||
            D.temperature[c] == D.temperature[1 - c])
            return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: scalar ping-pong buffers", i), false;
        if (D.scalar_corrected && (!D.predictor[c] || !D.reverse[c]))
            return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: MacCormack scalars need scratch", i), false;
    }
    if (D.sources.count > 8) return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: at most eight sources", i), false;
    if (!(D.blend >= 0.f && D.blend <= 1.f))
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: blend outside [0, 1]", i), false;
    if (!(D.cell > 0.0 && D.cfl > 0.0 && D.dt_max > 0.0 && D.dt0 > 0.f))
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: invalid time-step rule", i), false;
    if (D.levels < 2 || D.levels > FFX_BATCH_LEVELS)
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: needs 2..%d multigrid levels", i, FFX_BATCH_LEVELS),
               false;
    if (D.pre < 1 || D.post < 1 || D.pre > 16 || D.post > 16 || (D.pre + D.post) % 2)
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: sweeps must be 1..16 with an even sum", i), false;
    if (i > 0 && (D.pre != D_first_pre || D.post != D_first_post))
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: every domain needs the same sweeps", i), false;
    if (D.max_cycles < 1 || D.max_cycles > 256 || !(D.tolerance > 0.0))
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: cycle cap 1..256 and tolerance > 0", i), false;
    for (int k = 0; k < D.levels; ++k) {
        const FfxBatchLevel& L = D.level[k];
        const FfxGraphLevel& lv = L.level;
        if (!L.p || !L.q || !L.rhs || L.p == L.q || L.p == L.rhs || L.q == L.rhs || lv.nx < 1 || lv.ny < 1 ||
            lv.nz < 1)
            return fail(FFX_ERR_INVALID, "ffx_batch: domain %d level %d: buffers", i, k), false;
        if (k == 0 && (lv.edges || lv.solid != D.solid || lv.nx != g.nx || lv.ny != g.ny || lv.nz != g.nz))
            return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: level 0 must be the mask-derived grid", i), false;
        if (k > 0) {
            const FfxGraphLevel& up = D.level[k - 1].level;
            if (!lv.edges || ((uintptr_t)lv.edges & 15) || up.nx != 2 * lv.nx || up.ny != 2 * lv.ny ||
                up.nz != 2 * lv.nz)
                return fail(FFX_ERR_INVALID, "ffx_batch: domain %d level %d: not a 2x coarsening with records", i,
                            k), false;
        }
    }
    const int last = D.levels - 1;
    if (D.inverse && cells_of(D.level[last].level) > 1024)
        return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: direct solve limited to 1024 cells", i), false;
    if (D.tail_start >= 0) {
        if (D.tail_start < 1 || D.tail_start > last || D.levels - D.tail_start > FFX_TAIL_LEVELS)
            return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: tail start", i), false;
        for (int k = D.tail_start; k < D.levels; ++k)
            if (cells_of(D.level[k].level) > 32768)
                return fail(FFX_ERR_INVALID, "ffx_batch: domain %d: tail level over 32768 cells", i), false;
    }
    return true;
}

// Extent (x, y, z tiles-axis) of a domain for a launch kind.
FfxBatchPlan::Entry entry_for(int kind, int slot, int nx, int ny, int nz) {
    switch (kind) {
        case kPredictor:
        case kVelocity: return {slot, nx + 1, ny + 1, 3 * (nz + 1)};
        case kResidualRestrict: return {slot, nx / 2, ny / 2, nz / 2};
        // level 0, four cells per thread: x in units of 4 cells, kL0Slices z per thread
        case kL0Smooth:
        case kL0ProlongSmooth:
        case kL0ResidualMax: return {slot, nx / kL0Cells, ny, (nz + kL0Slices - 1) / kL0Slices};
        case kL0ResidualRestrict: return {slot, nx / kL0Cells, ny / 2, (nz + kL0Slices - 1) / kL0Slices};
        case kScaleZero: return {slot, nx * ny * nz, 1, 1};
        case kDirect: return {slot, nx * ny * nz, 1, 1};
        default: return {slot, nx, ny, nz};
    }
}

// Work list of a launch for the kind's current tile shape.
BatchMap make_map(const FfxBatchPlan& P, const FfxBatchPlan::Launch& L) {
    BatchMap M;
    memset(&M, 0, sizeof M);
    const int kind = L.kind;
    int bw = kShapes[P.shape[kind < kBatchKinds ? kind : 0]][0], bh = kShapes[P.shape[kind < kBatchKinds ? kind : 0]][1];
    if (is_l0_kind(kind)) {   // the four-cell kernels' block: 32 lanes x kL0Rows rows
        bw = 32;
        bh = kL0Rows;
    }
    M.count = (int)L.entries.size();
    int64_t total = 0;
    for (int k = 0; k < M.count; ++k) {
        const FfxBatchPlan::Entry& e = L.entries[k];
        int gx, gy, gz;
        if (kind == kScaleZero) { gx = (e.X + kBatchThreads - 1) / kBatchThreads; gy = 1; gz = 1; }
        else if (kind == kDirect) { gx = (e.X + kBatchThreads / 32 - 1) / (kBatchThreads / 32); gy = 1; gz = 1; }
        else { gx = (e.X + bw - 1) / bw; gy = (e.Y + bh - 1) / bh; gz = e.Z; }
        M.dom[k] = e.slot;
        M.first[k] = (int)total;
        M.gx[k] = gx;
        M.gy[k] = gy;
        M.gz[k] = gz;
        total += (int64_t)gx * gy * gz;
    }
    M.first[M.count] = (int)total;
    M.total = (int)total;
    M.bw = (kind == kScaleZero || kind == kDirect) ? kBatchThreads : bw;
    M.bh = (kind == kScaleZero || kind == kDirect) ? 1 : bh;
    return M;
}

int resident(int kind) {
    int r = batch::advect_resident_blocks(kind);
    if (!r) r = batch::project_resident_blocks(kind);
    if (!r) r = batch::level0_resident_blocks(kind);
    return r > 0 ? r : 1;
}

cudaError_t issue(FfxBatchPlan& P, const FfxBatchPlan::Launch& L, cudaStream_t st) {
    if (L.entries.empty()) return cudaSuccess;
    BatchMap M = make_map(P, L);
    if (M.total == 0) return cudaSuccess;
    const void* d = P.ws + L.offset;
    const int kind = L.kind;
    if (kind == kTail) return batch::tail(M, d, P.state, st);
    const int g = P.grid[kind] > 0 ? P.grid[kind] * resident(kind) * P.sms : 0;
    switch (kind) {
        case kPredictor: return batch::face_predictor(M, d, P.state, g, st);
        case kVelocity: return batch::advect_velocity(M, d, P.state, g, st);
        case kDivergence: return batch::divergence(M, d, P.state, g, st);
        case kScaleZero: return batch::scale_zero(M, d, P.state, g, st);
        case kGradient: return batch::gradient(M, d, P.state, g, st);
        case kScalarPredictor: return batch::scalar_transport(M, d, P.state, 0, g, st);
        case kScalarReverse: return batch::scalar_transport(M, d, P.state, 1, g, st);
        case kScalarFinal: return batch::advect_scalars(M, d, P.state, g, st);
        case kResidualMax: return batch::residual_max(M, d, P.state, g, st);
        case kSmooth: return batch::smooth(M, d, P.state, g, st);
        case kResidualRestrict: return batch::residual_restrict(M, d, P.state, g, st);
        case kProlongSmooth: return batch::prolong_smooth(M, d, P.state, g, st);
        case kDirect: return batch::direct(M, d, P.state, g, st);
        case kL0Smooth: return batch::l0_smooth(M, d, P.state, g, st);
        case kL0ProlongSmooth: return batch::l0_prolong_smooth(M, d, P.state, g, st);
        case kL0ResidualRestrict: return batch::l0_residual_restrict(M, d, P.state, g, st);
        case kL0ResidualMax: return batch::l0_residual_max(M, d, P.state, g, st);
        default: return cudaErrorInvalidValue;
    }
}

// Builder of the plan's launches and descriptor bytes.
struct Builder {
    FfxBatchPlan& P;
    std::vector<char> host;
    explicit Builder(FfxBatchPlan& p) : P(p) {}

    size_t reserve(size_t bytes) {
        const size_t off = align_up(host.size());
        host.resize(off + bytes);
        return off;
    }
    template <class F>
    FfxBatchPlan::Launch launch(int kind, const std::vector<int>& slots, F fill) {
        FfxBatchPlan::Launch L;
        L.kind = kind;
        const size_t sz = desc_size(kind);
        L.offset = reserve(sz * slots.size());
        for (size_t k = 0; k < slots.size(); ++k) {
            FfxBatchPlan::Entry e;
            fill(slots[k], host.data() + L.offset + k * sz, e);
            L.entries.push_back(e);
        }
        return L;
    }
};

// Level 0 of a domain qualifies for the four-cell kernels: link field, x a
// multiple of 4, 16-byte aligned fields, even y and z, and a level below it
// (whose rhs and iterate the restriction and prolongation address as float2).
bool l0_domain(const FfxBatchDomain& D) {
    if (D.levels < 2) return false;
    const FfxBatchLevel& L = D.level[0];
    const FfxBatchLevel& C = D.level[1];
    return batch::l0_eligible(L.level, {L.p, L.q, L.rhs}) && L.level.ny % 2 == 0 && L.level.nz % 2 == 0 &&
           ((uintptr_t)C.rhs & 7) == 0 && ((uintptr_t)C.p & 7) == 0 && ((uintptr_t)C.q & 7) == 0;
}

std::vector<int> all_slots(const FfxBatchPlan& P) {
    std::vector<int> s;
    for (int d = 0; d < P.count; ++d) s.push_back(d);
    return s;
}

// The V-cycle schedule: down over the stand-alone levels, the coarse stage
// (tail, direct solve or 80 sweeps), up again; every domain's buffer roles
// are tracked exactly as the stand-alone cycle swaps them.
void build_cycle(Builder& B) {
    FfxBatchPlan& P = B.P;
    const int n = P.count;
    std::vector<int> top(n);
    std::vector<std::vector<int>> role(n);   // 0: p holds the iterate, 1: q does
    int K = 0;
    for (int d = 0; d < n; ++d) {
        const FfxBatchDomain& D = P.dom[d];
        top[d] = D.tail_start >= 0 ? D.tail_start : D.levels - 1;
        role[d].assign(D.levels, 0);
        if (top[d] > K) K = top[d];
    }
    auto cur = [&](int d, int k) { const FfxBatchLevel& L = P.dom[d].level[k]; return role[d][k] ? L.q : L.p; };
    auto other = [&](int d, int k) { const FfxBatchLevel& L = P.dom[d].level[k]; return role[d][k] ? L.p : L.q; };
    auto level_entry = [&](int kind, int d, int k) {
        const FfxGraphLevel& lv = P.dom[d].level[k].level;
        FfxBatchPlan::Entry e = entry_for(kind, d, lv.nx, lv.ny, lv.nz);
        if (kind == kSmooth && k == 0) e.Z = (lv.nz + kBatchZ0 - 1) / kBatchZ0;   // streamed along z
        return e;
    };
    // level 0 runs four cells per thread when every domain of the launch qualifies
    auto x4 = [&](int k, const std::vector<int>& slots) {
        if (k != 0) return false;
        for (int d : slots)
            if (!l0_domain(P.dom[d])) return false;
        return true;
    };
    auto l0_entry = [&](int kind, int d) {
        const FfxGraphLevel& lv = P.dom[d].level[0].level;
        return entry_for(kind, d, lv.nx, lv.ny, lv.nz);
    };
    auto smooth_at = [&](int k, const std::vector<int>& slots) {
        if (x4(k, slots)) {
            P.cycle.push_back(B.launch(kL0Smooth, slots, [&](int d, char* out, FfxBatchPlan::Entry& e) {
                const FfxBatchLevel& L = P.dom[d].level[0];
                batch::l0_desc(L.level, cur(d, 0), nullptr, L.rhs, other(d, 0), nullptr, out);
                e = l0_entry(kL0Smooth, d);
            }));
        } else {
            P.cycle.push_back(B.launch(kSmooth, slots, [&](int d, char* out, FfxBatchPlan::Entry& e) {
                const FfxBatchLevel& L = P.dom[d].level[k];
                batch::level_desc(L.level, cur(d, k), other(d, k), L.rhs, nullptr, nullptr, out);
                e = level_entry(kSmooth, d, k);
            }));
        }
        for (int d : slots) role[d][k] ^= 1;
    };
    // down
    for (int k = 0; k < K; ++k) {
        std::vector<int> act;
        for (int d = 0; d < n; ++d)
            if (k < top[d]) act.push_back(d);
        for (int s = 0; s < P.dom[act[0]].pre; ++s) smooth_at(k, act);
        const bool four = x4(k, act);
        P.cycle.push_back(B.launch(four ? kL0ResidualRestrict : kResidualRestrict, act,
                                   [&](int d, char* out, FfxBatchPlan::Entry& e) {
            const FfxBatchDomain& D = P.dom[d];
            const FfxBatchLevel& L = D.level[k];
            const bool tail_next = D.tail_start == k + 1;
            float* zero = tail_next ? nullptr : cur(d, k + 1);
            if (four) {
                batch::l0_desc(L.level, cur(d, 0), nullptr, L.rhs, D.level[1].rhs, zero, out);
                e = l0_entry(kL0ResidualRestrict, d);
            } else {
                batch::level_desc(L.level, cur(d, k), nullptr, L.rhs, D.level[k + 1].rhs, zero, out);
                e = level_entry(kResidualRestrict, d, k);
            }
        }));
    }
    // coarse stage
    std::vector<int> tails, directs, sweeps;
    for (int d = 0; d < n; ++d) {
        const FfxBatchDomain& D = P.dom[d];
        if (D.tail_start >= 0) tails.push_back(d);
        else if (D.inverse) directs.push_back(d);
        else sweeps.push_back(d);
    }
    if (!tails.empty()) {
        P.cycle.push_back(B.launch(kTail, tails, [&](int d, char* out, FfxBatchPlan::Entry& e) {
            const FfxBatchDomain& D = P.dom[d];
            batch::tail_desc(D, D.pre, D.post, out);
            e = {d, 1, 1, 1};
        }));
    }
    if (!directs.empty()) {
        P.cycle.push_back(B.launch(kDirect, directs, [&](int d, char* out, FfxBatchPlan::Entry& e) {
            const FfxBatchDomain& D = P.dom[d];
            const int last = D.levels - 1;
            batch::direct_desc(D, cur(d, last), out);
            e = level_entry(kDirect, d, last);
        }));
    }
    if (!sweeps.empty()) {
        // 80 sweeps from the zeroed iterate, on each domain's coarsest level
        for (int s = 0; s < 80; ++s) {
            P.cycle.push_back(B.launch(kSmooth, sweeps, [&](int d, char* out, FfxBatchPlan::Entry& e) {
                const FfxBatchDomain& D = P.dom[d];
                const int last = D.levels - 1;
                const FfxBatchLevel& L = D.level[last];
                batch::level_desc(L.level, cur(d, last), other(d, last), L.rhs, nullptr, nullptr, out);
                e = level_entry(kSmooth, d, last);
            }));
            for (int d : sweeps) role[d][P.dom[d].levels - 1] ^= 1;
        }
    }
    // up
    for (int k = K - 1; k >= 0; --k) {
        std::vector<int> act;
        for (int d = 0; d < n; ++d)
            if (k < top[d]) act.push_back(d);
        const bool four = x4(k, act);
        P.cycle.push_back(B.launch(four ? kL0ProlongSmooth : kProlongSmooth, act,
                                   [&](int d, char* out, FfxBatchPlan::Entry& e) {
            const FfxBatchLevel& L = P.dom[d].level[k];
            if (four) {
                batch::l0_desc(L.level, cur(d, 0), cur(d, 1), L.rhs, other(d, 0), nullptr, out);
                e = l0_entry(kL0ProlongSmooth, d);
            } else {
                batch::level_desc(L.level, cur(d, k), other(d, k), L.rhs, cur(d, k + 1), nullptr, out);
                e = level_entry(kProlongSmooth, d, k);
            }
        }));
        for (int d : act) role[d][k] ^= 1;
        for (int s = 1; s < P.dom[act[0]].post; ++s) smooth_at(k, act);
    }
}

int build(FfxBatchPlan& P, std::vector<char>& host) {
    Builder B(P);
    const std::vector<int> all = all_slots(P);
    const size_t state_off = B.reserve(sizeof(BatchState) * P.count);
    const size_t solve_off = B.reserve(sizeof(FfxBatchPlan::Solve) * P.count);
    const size_t rule_off = B.reserve(sizeof(StepRule) * P.count);
    const size_t guard_off = B.reserve(sizeof(FfxBatchPlan::Guard));
    for (int d = 0; d < P.count; ++d) {
        const FfxBatchDomain& D = P.dom[d];
        BatchState S;
        memset(&S, 0, sizeof S);
        S.dt = D.dt0;
        S.dtd = D.dt0;
        S.pmode = 0;
        memcpy(B.host.data() + state_off + d * sizeof(BatchState), &S, sizeof S);
        FfxBatchPlan::Solve V = {D.tolerance, D.max_cycles, D.warm_start ? 1 : 0};
        memcpy(B.host.data() + solve_off + d * sizeof V, &V, sizeof V);
        StepRule R = {D.cell, D.cfl, D.dt_max};
        memcpy(B.host.data() + rule_off + d * sizeof R, &R, sizeof R);
    }
    auto cells = [&](int kind, int d) {
        const FfxGrid& g = P.dom[d].grid;
        return entry_for(kind, d, g.nx, g.ny, g.nz);
    };
    std::vector<int> vcorr, scorr;
    for (int d = 0; d < P.count; ++d) {
        if (P.dom[d].velocity_corrected) vcorr.push_back(d);
        if (P.dom[d].scalar_corrected) scorr.push_back(d);
    }
    for (int par = 0; par < 2; ++par) {
        auto& pre = P.pre[par];
        auto& post = P.post[par];
        if (!vcorr.empty())
            pre.push_back(B.launch(kPredictor, vcorr, [&](int d, char* out, FfxBatchPlan::Entry& e) {
                batch::predictor_desc(P.dom[d], out);
                e = cells(kPredictor, d);
            }));
        pre.push_back(B.launch(kVelocity, all, [&](int d, char* out, FfxBatchPlan::Entry& e) {
            batch::velocity_desc(P.dom[d], par, out);
            e = cells(kVelocity, d);
        }));
        pre.push_back(B.launch(kDivergence, all, [&](int d, char* out, FfxBatchPlan::Entry& e) {
            batch::divergence_desc(P.dom[d], out);
            e = cells(kDivergence, d);
        }));
        pre.push_back(B.launch(kScaleZero, all, [&](int d, char* out, FfxBatchPlan::Entry& e) {
            batch::scale_zero_desc(P.dom[d], out);
            e = cells(kScaleZero, d);
        }));
        post.push_back(B.launch(kGradient, all, [&](int d, char* out, FfxBatchPlan::Entry& e) {
            const FfxBatchDomain& D = P.dom[d];
            batch::gradient_desc(D, D.u, D.v, D.w, out);
            e = cells(kGradient, d);
        }));
        if (!scorr.empty()) {
            post.push_back(B.launch(kScalarPredictor, scorr, [&](int d, char* out, FfxBatchPlan::Entry& e) {
                batch::scalar_xport_desc(P.dom[d], par, 0, out);
                e = cells(kScalarPredictor, d);
            }));
            post.push_back(B.launch(kScalarReverse, scorr, [&](int d, char* out, FfxBatchPlan::Entry& e) {
                batch::scalar_xport_desc(P.dom[d], par, 1, out);
                e = cells(kScalarReverse, d);
            }));
        }
        post.push_back(B.launch(kScalarFinal, all, [&](int d, char* out, FfxBatchPlan::Entry& e) {
            batch::scalar_final_desc(P.dom[d], par, out);
            e = cells(kScalarFinal, d);
        }));
    }
    bool four = true;
    for (int d = 0; d < P.count; ++d) four = four && l0_domain(P.dom[d]);
    P.resmax = B.launch(four ? kL0ResidualMax : kResidualMax, all, [&](int d, char* out, FfxBatchPlan::Entry& e) {
        const FfxBatchLevel& L = P.dom[d].level[0];
        if (four) {
            batch::l0_desc(L.level, L.p, nullptr, L.rhs, nullptr, nullptr, out);
            e = entry_for(kL0ResidualMax, d, L.level.nx, L.level.ny, L.level.nz);
        } else {
            batch::level_desc(L.level, L.p, nullptr, L.rhs, nullptr, nullptr, out);
            e = cells(kResidualMax, d);
        }
    });
    build_cycle(B);
    // tuning launches: each kind once over every domain, writing scratch only
    // (the launch of the kind that covers the most cells: level 0 for the multigrid kinds)
    auto volume = [](const FfxBatchPlan::Launch& L) {
        int64_t v = 0;
        for (const auto& e : L.entries) v += (int64_t)e.X * e.Y * e.Z;
        return v;
    };
    for (int kind = 0; kind < kBatchKinds; ++kind) {
        FfxBatchPlan::Launch* found = nullptr;
        for (auto* list : {&P.pre[0], &P.post[0], &P.cycle})
            for (auto& L : *list)
                if (L.kind == kind && (!found || volume(L) > volume(*found))) found = &L;
        if ((kind == kResidualMax || kind == kL0ResidualMax) && P.resmax.kind == kind) found = &P.resmax;
        if (kind == kGradient) {
            P.tune[kind] = B.launch(kGradient, all, [&](int d, char* out, FfxBatchPlan::Entry& e) {
                const FfxBatchDomain& D = P.dom[d];
                // velocity kept: the outputs go to the predictor faces (same shapes)
                batch::gradient_desc(D, D.pu ? D.pu : D.bu, D.pv ? D.pv : D.bv, D.pw ? D.pw : D.bw, out);
                e = cells(kGradient, d);
            });
            if (!P.dom[0].pu) P.tune[kind].entries.clear();   // no scratch faces: not tunable
        } else if (found) {
            P.tune[kind] = *found;
        } else {
            P.tune[kind].kind = kind;
        }
    }
    P.state = reinterpret_cast<BatchState*>(P.ws + state_off);
    P.solve = reinterpret_cast<FfxBatchPlan::Solve*>(P.ws + solve_off);
    P.rules = P.ws + rule_off;
    P.guard = reinterpret_cast<FfxBatchPlan::Guard*>(P.ws + guard_off);
    host.swap(B.host);
    return FFX_OK;
}

const StepRule* rules_of(const FfxBatchPlan& P) { return reinterpret_cast<const StepRule*>(P.rules); }

cudaError_t issue_list(FfxBatchPlan& P, const std::vector<FfxBatchPlan::Launch>& list, cudaStream_t st) {
    for (const auto& L : list) {
        cudaError_t e = issue(P, L, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// One step captured on `st` (capturing) with the solve loop as a WHILE node
// whose body is captured on `side`.
int capture_step(FfxBatchPlan& P, int par, cudaStream_t st, cudaStream_t side) {
    cudaError_t e = issue_list(P, P.pre[par], st);
    if (e != cudaSuccess) return cuda_status(e, "ffx_batch_graph: passes before the solve");
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    e = cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess || status != cudaStreamCaptureStatusActive)
        return cuda_status(e != cudaSuccess ? e : cudaErrorStreamCaptureInvalidated, "ffx_batch_graph: capture info");
    cudaGraphConditionalHandle handle;
    e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return cuda_status(e, "ffx_batch_graph: conditional handle");
    cudaGraphNodeParams params = {cudaGraphNodeTypeConditional};
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, graph, deps, ndeps, &params);
    if (e != cudaSuccess) return cuda_status(e, "ffx_batch_graph: conditional node");
    cudaGraph_t body = params.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return cuda_status(e, "ffx_batch_graph: body capture");
    cudaError_t eb = issue(P, P.resmax, side);
    if (eb == cudaSuccess) {
        batch_decide_kernel<<<1, 64, 0, side>>>(P.state, P.solve, P.count, P.guard, handle);
        eb = cudaGetLastError();
    }
    if (eb == cudaSuccess) eb = issue_list(P, P.cycle, side);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(side, &captured);
    if (eb != cudaSuccess) return cuda_status(eb, "ffx_batch_graph: solve body");
    if (e != cudaSuccess) return cuda_status(e, "ffx_batch_graph: end of body capture");
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return cuda_status(e, "ffx_batch_graph: capture dependencies");
    e = issue_list(P, P.post[par], st);
    if (e != cudaSuccess) return cuda_status(e, "ffx_batch_graph: passes after the solve");
    batch_step_end_kernel<<<1, 64, 0, st>>>(P.state, rules_of(P), P.solve, P.count, P.guard);
    return cuda_status(cudaGetLastError(), "ffx_batch_graph: step end");
}

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" {

int ffx_batch_workspace_bytes(const FfxBatchDomain* domains, int32_t count, int64_t* bytes) {
    FFX_REQUIRE(domains && bytes && count >= 1 && count <= FFX_BATCH_MAX && count <= kBatchMax,
                "ffx_batch_workspace_bytes: 1..%d domains", FFX_BATCH_MAX);
    for (int d = 0; d < count; ++d)
        if (!domain_ok(domains[d], d, domains[0].pre, domains[0].post)) return FFX_ERR_INVALID;
    FfxBatchPlan P;
    P.count = count;
    P.dom.assign(domains, domains + count);
    std::vector<char> host;
    build(P, host);
    *bytes = (int64_t)align_up(host.size());
    return FFX_OK;
}

int ffx_batch_create(const FfxBatchDomain* domains, int32_t count, void* workspace, int64_t bytes,
                     FfxBatchPlan** plan) {
    FFX_REQUIRE(domains && plan && workspace && count >= 1 && count <= FFX_BATCH_MAX && count <= kBatchMax,
                "ffx_batch_create: invalid arguments");
    FFX_REQUIRE(((uintptr_t)workspace & 255) == 0, "ffx_batch_create: workspace must be 256-byte aligned");
    for (int d = 0; d < count; ++d)
        if (!domain_ok(domains[d], d, domains[0].pre, domains[0].post)) return FFX_ERR_INVALID;
    FfxBatchPlan* P = new FfxBatchPlan;
    P->count = count;
    P->dom.assign(domains, domains + count);
    P->ws = reinterpret_cast<char*>(workspace);
    P->ws_bytes = bytes;
    std::vector<char> host;
    build(*P, host);
    if ((int64_t)host.size() > bytes) {
        delete P;
        return fail(FFX_ERR_INVALID, "ffx_batch_create: workspace of %lld bytes, %lld needed", (long long)bytes,
                    (long long)host.size());
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&P->sms, cudaDevAttrMultiProcessorCount, dev);
    int e = cuda_status(cudaMemcpy(workspace, host.data(), host.size(), cudaMemcpyHostToDevice),
                        "ffx_batch_create: upload");
    if (e) {
        delete P;
        return e;
    }
    *plan = P;
    return FFX_OK;
}

int ffx_batch_set_config(FfxBatchPlan* plan, int32_t kind, int32_t shape, int32_t grid) {
    FFX_REQUIRE(plan && kind >= 0 && kind < kBatchKinds && shape >= 0 && shape < 4 && grid >= 0 && grid <= 64,
                "ffx_batch_set_config: invalid arguments");
    plan->shape[kind] = shape;
    plan->grid[kind] = grid;
    return FFX_OK;
}

int ffx_batch_tune_pass(FfxBatchPlan* plan, int32_t kind, void* stream) {
    FFX_REQUIRE(plan && kind >= 0 && kind < kBatchKinds, "ffx_batch_tune_pass: invalid arguments");
    cudaStream_t st = as_stream(stream);
    int e = cuda_status(issue(*plan, plan->tune[kind], st), "ffx_batch_tune_pass");
    if (e) return e;
    if (kind == kScaleZero || kind == kGradient || kind == kResidualMax || kind == kL0ResidualMax) {
        batch_clear_kernel<<<1, 64, 0, st>>>(plan->state, plan->count);
        return launch_status("ffx_batch_tune_pass: clear");
    }
    return FFX_OK;
}

int ffx_batch_graph(FfxBatchPlan* plan, int32_t steps, void** graph_exec) {
    FFX_REQUIRE(plan && graph_exec && steps >= 1 && steps <= 1024, "ffx_batch_graph: invalid arguments");
    cudaStream_t st = nullptr, side = nullptr;
    int rc = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "ffx_batch_graph: stream");
    if (!rc) rc = cuda_status(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking), "ffx_batch_graph: stream");
    cudaGraph_t graph = nullptr;
    if (!rc) rc = cuda_status(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "ffx_batch_graph: capture");
    if (!rc) {
        int par = plan->parity;
        for (int s = 0; s < steps && !rc; ++s, par ^= 1) rc = capture_step(*plan, par, st, side);
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        if (!rc) rc = cuda_status(e, "ffx_batch_graph: end capture");
    }
    cudaGraphExec_t exec = nullptr;
    if (!rc) rc = cuda_status(cudaGraphInstantiate(&exec, graph, 0), "ffx_batch_graph: instantiate");
    if (graph) cudaGraphDestroy(graph);
    if (side) cudaStreamDestroy(side);
    if (st) cudaStreamDestroy(st);
    if (rc) return rc;
    *graph_exec = exec;
    return FFX_OK;
}

int ffx_batch_launch(FfxBatchPlan* plan, void* graph_exec, int32_t steps, void* stream) {
    FFX_REQUIRE(plan && graph_exec && steps >= 1, "ffx_batch_launch: invalid arguments");
    int rc = cuda_status(cudaGraphLaunch(reinterpret_cast<cudaGraphExec_t>(graph_exec), as_stream(stream)),
                         "ffx_batch_launch");
    if (!rc) plan->parity ^= (steps & 1);
    return rc;
}

int ffx_batch_graph_free(void* graph_exec) {
    if (graph_exec) cudaGraphExecDestroy(reinterpret_cast<cudaGraphExec_t>(graph_exec));
    return FFX_OK;
}

int ffx_batch_stats(const FfxBatchPlan* plan, FfxBatchStats* out, void* stream) {
    FFX_REQUIRE(plan && out, "ffx_batch_stats: invalid arguments");
    std::vector<BatchState> S(plan->count);
    FfxBatchPlan::Guard G = {0, 0, 0};
    cudaStream_t st = as_stream(stream);
    int rc = cuda_status(cudaMemcpyAsync(S.data(), plan->state, sizeof(BatchState) * plan->count,
                                         cudaMemcpyDeviceToHost, st), "ffx_batch_stats: copy");
    if (!rc) rc = cuda_status(cudaMemcpyAsync(&G, plan->guard, sizeof G, cudaMemcpyDeviceToHost, st),
                              "ffx_batch_stats: copy");
    if (!rc) rc = cuda_status(cudaStreamSynchronize(st), "ffx_batch_stats: synchronise");
    if (rc) return rc;
    for (int d = 0; d < plan->count; ++d) {
        out[d].dt = S[d].dt;
        out[d].last_dt = S[d].last_dt;
        out[d].last_cycles = S[d].last_cycles;
        out[d].total_cycles = S[d].total_cycles;
        out[d].steps = S[d].steps;
        for (int a = 0; a < 3; ++a) out[d].maxima[a] = S[d].last_maxima[a];
        out[d].time = S[d].time;
        out[d].loop_iterations = G.total;
    }
    if (G.tripped) return fail(FFX_ERR_TIMEOUT, "ffx_batch_stats: a solve loop reached %d iterations", kLoopCap);
    return FFX_OK;
}

int ffx_batch_parity(const FfxBatchPlan* plan) { return plan ? plan->parity : -1; }

int ffx_batch_destroy(FfxBatchPlan* plan) {
    delete plan;
    return FFX_OK;
}

}  // extern "C"
