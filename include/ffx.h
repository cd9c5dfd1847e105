/*
 * ffx.h -- C ABI of libffx_core.so, the B200 (sm_100a) kernels of the dense
 * MAC-grid smoke step.
 *
 * Conventions
 *   - Plain C: no exceptions cross this boundary. Every entry point returns an
 *     FfxStatus; ffx_last_error() gives a thread-local message for the last
 *     failure on the calling thread.
 *   - All buffers are DEVICE pointers owned by the caller (allocated by any
 *     allocator, e.g. torch). The library allocates nothing and frees nothing.
 *     Work is enqueued on `stream` (a cudaStream_t passed as void*; NULL is the
 *     legacy default stream); calls are asynchronous unless stated otherwise.
 *   - Cell fields are x-fast: index x + nx*(y + ny*z). Face grids are
 *     (nx+1, ny, nz), (nx, ny+1, nz), (nx, ny, nz+1) in the same order.
 *   - `storage` selects the element type of velocity/scalar fields:
 *     FFX_F32 (float) or FFX_BF16 (bfloat16). Arithmetic is always FP32;
 *     pressure, divergence and multigrid buffers are always float.
 *   - Colliders are two uint8 cell masks (FfxSolids): `solid` (1 = solid) and
 *     `halo` (1 = a solid or out-of-domain cell lies in the 3x3x3 block), the
 *     latter made by ffx_dilate_mask. Both NULL = no colliders.
 *
 * Each entry point names the reference interface it replaces
 * (FluxFX, paths relative to the add-on package `fluxfx/`).
 */
#ifndef FFX_H
#define FFX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFX_ABI_VERSION 3

typedef enum FfxStatus {
    FFX_OK = 0,
    FFX_ERR_INVALID = 1,       /* bad argument (shape, pointer, range) */
    FFX_ERR_LAUNCH = 2,        /* kernel launch failed */
    FFX_ERR_NOT_CONVERGED = 3, /* iterative solve hit its cycle cap */
    FFX_ERR_TIMEOUT = 4,       /* a bounded device wait gave up */
    FFX_ERR_CUDA = 5           /* other CUDA runtime error */
} FfxStatus;

enum { FFX_F32 = 0, FFX_BF16 = 1 };

typedef struct FfxGrid {
    int32_t nx, ny, nz;   /* cells per axis, 1 to 4096 */
    float ex, ey, ez;     /* domain extent in metres, 2^-18 to 2^30 */
    float ix, iy, iz;     /* 1/h of divergence and gradient (the reference's
                             invCell uniform: 1/(extent/n) in FP64, rounded);
                             0 = derive it from ex..ez */
} FfxGrid;

typedef struct FfxSolids {
    const uint8_t* solid; /* nx*ny*nz, nonzero = solid cell; NULL = no colliders */
    const uint8_t* halo;  /* nx*ny*nz dilated mask (ffx_dilate_mask) */
    const float* wall[3]; /* moving colliders: velocity of every wall and solid face
                             (face grids, ffx_moving_walls); NULL = 0 (static walls) */
    const uint8_t* clear; /* optional, with a mask: nx*ny*nz clearance (ffx_clearance: 0/1;
                             ffx_halo_clearance: 0/1/2, 2 = no solid within three cells but
                             a wall); the transport passes skip the collider tests of traces
                             that start in a cell of nonzero clearance and stay within 0.75
                             cells (same results) */
} FfxSolids;

/* Moving colliders per solver (the reference's wall table holds 8). */
#define FFX_MOVING_MAX 8

/* Emitters. count < 0: one swept sphere described by the `single_*` fields
 * (backend/projected.py:155-159, emission_weight.glsl). count in [0, 8]: rows
 * of `table`, 16 floats per source in the layout of physics/emission.py:49-58
 * (center.xyz, radius | start.xyz, coupling | jet.xyz, density_rate |
 *  heat_rate, target_flag, solid_flag, fuel_rate). */
typedef struct FfxSources {
    int32_t count;
    int32_t single_solid_profile;
    float single_center[3];
    float single_start[3];
    float single_radius;
    float single_jet[3];
    float single_coupling;
    float table[128];
} FfxSources;

typedef struct FfxDeviceInfo {
    int32_t device, sm_count, cc_major, cc_minor;
    int64_t total_bytes;
    char name[128];
} FfxDeviceInfo;

/* ------------------------------------------------------------------ runtime */
int ffx_abi_version(void);
const char* ffx_last_error(void);
/* Device capability query; replaces backend/device.py:15-28 (capability gate). */
int ffx_device_info(int device, FfxDeviceInfo* out);
/* Writes x + 10y + 100z over a 7x5x3 float buffer; replaces backend/device.py:83-96. */
int ffx_probe_3d(float* out, void* stream);

/* -------------------------------------------------------------- seeds/masks */
/* Soft-sphere scalar seed * scale; replaces shaders/seed.glsl, temperature_seed.glsl. */
int ffx_seed_scalar(const FfxGrid* g, int storage, const float center[3], float radius,
                    float scale, void* out, void* stream);
/* Analytic rotation + translation face seed; replaces shaders/mac_seed.glsl. */
int ffx_seed_faces(const FfxGrid* g, int storage, const float base[3], float angular,
                   void* u, void* v, void* w, void* stream);
/* Voxelise `count` colliders (13 doubles each: 3x4 inverse rows, shape 0=sphere
 * 1=box) at cell centres in FP64 using the FP64 `extent`; replaces backend/collision.py:22-41 +
 * shaders/solid_mask.glsl, bit-exact with physics/collision.py:35-37. */
int ffx_raster_colliders(const FfxGrid* g, const double extent[3], int count,
                         const double* rows13, uint8_t* solid, void* stream);
/* 3x3x3 dilation with out-of-domain = solid (precomputes solidHalo,
 * shaders/solid_boundary.glsl:39-44). */
int ffx_dilate_mask(const FfxGrid* g, const uint8_t* solid, uint8_t* halo, void* stream);

/* Clearance of a mask: clear[c] = 1 where no cell within Chebyshev distance 2
 * of c is set in `halo` (ffx_dilate_mask of the mask) or lies outside the grid,
 * i.e. no solid or outside cell lies within distance 3 of c; else 0. An
 * extension with no reference counterpart: it lets the transport passes skip
 * the collider tests (solid_boundary.glsl, correct_*.glsl) where they cannot
 * change the result. One-time work per collider layout. */
int ffx_clearance(const FfxGrid* g, const uint8_t* halo, uint8_t* clear, void* stream);
/* ffx_dilate_mask and the clearance of a mask in one pass (an extension:
 * moving colliders refresh both after every move). halo is ffx_dilate_mask's
 * field bit for bit; clear is 1 where ffx_clearance writes 1 (no solid and no
 * outside cell within distance 3), 2 where no solid but an outside cell lies
 * within distance 3, 0 elsewhere. The transport passes take both nonzero
 * values through FfxSolids.clear. */
int ffx_halo_clearance(const FfxGrid* g, const uint8_t* solid, uint8_t* halo, uint8_t* clear, void* stream);
/* Counts the inputs a, over all 2^32 FP32 bit patterns, whose quotient by
 * `divisor` (in [2^-30, 2^30]) as the kernels form it on grids that are not
 * powers of two (a reciprocal with two remainder corrections) differs from the
 * IEEE division a / divisor: count[0] (device int64) over the inputs the form
 * is exact for (+-0, +-inf, NaN and 2^-96 <= |a| <= 2^96; must be 0),
 * count[1] over the others (nonzero |a| < 2^-96, finite |a| > 2^96; no grid
 * position). A check of the library's own arithmetic: no reference
 * counterpart. */
int ffx_division_mismatches(float divisor, int64_t* count, void* stream);
/* out = solid ? 0 : in; replaces shaders/solid_clear.glsl. */
int ffx_solid_clear(const FfxGrid* g, int storage, const uint8_t* solid, const void* in,
                    void* out, void* stream);

/* ---------------------------------------------------------- velocity passes */
/* The transport passes (face predictor, velocity, scalar predictor/reverse and
 * final scalar pass) run as global-memory gathers by default (enable = 0), or,
 * with enable != 0, over shared-memory windows of a rolling z slab (measured
 * slower on B200: the passes are bound by instruction issue). Both forms give
 * bit-identical results; the switch is process-wide and returns the previous
 * setting. No counterpart in the reference (an A/B switch). */
int ffx_set_transport_tiling(int enable);
/* Whether the edge-record (coarse) multigrid levels run the residual +
 * restriction streamed along z (default on) or one coarse cell per thread.
 * Both give the same fields bit for bit; returns the previous setting. */
int ffx_set_edge_streaming(int enable);
/* Whether the multigrid passes of the collider solver (level-0 and coarse
 * sweeps, residual + restriction, prolongation + sweep, the single-block tail,
 * the convergence test) are launched as programmatic dependent launches, so a
 * pass is scheduled while the one before it finishes (default on). Results are
 * the same either way; returns the previous setting. */
int ffx_set_dependent_launch(int enable);
/* MacCormack predictor of all three face components in one launch; replaces
 * backend/detail.py:27-37 + shaders/transport_face.glsl. */
int ffx_face_predictor(const FfxGrid* g, const FfxSolids* s, int storage,
                       const void* u, const void* v, const void* w, float dt,
                       void* pu, void* pv, void* pw, void* stream);
/* The same, also storing each open face's trace in dep[axis], planes of
 * (nx+a0)(ny+a1)(nz+a2) floats for ffx_advect_velocity_trace: FFX_F32 storage
 * six planes (departure point x, y, z; start velocity x, y, z), FFX_BF16 seven
 * (departure point x, y, z; the face's sample before rounding to storage, which
 * the velocity correction reads as its semi-Lagrangian value; start velocity
 * x, y, z). */
int ffx_face_predictor_trace(const FfxGrid* g, const FfxSolids* s, int storage,
                             const void* u, const void* v, const void* w, float dt,
                             void* pu, void* pv, void* pw, float* const dep[3], void* stream);
/* Velocity transport (SL or MacCormack: corrected != 0, blended by `blend`),
 * emitter coupling, and -- fused -- buoyancy on W from the previous density and
 * temperature (NULL to skip) and the wall condition (apply_walls != 0). Replaces
 * shaders/emitting_advect_velocity.glsl, multi_advect_velocity.glsl,
 * correct_velocity_fused.glsl, buoyancy.glsl and pressure_walls.glsl as
 * sequenced by backend/projected.py:150-177. Faces out must not alias faces in. */
int ffx_advect_velocity(const FfxGrid* g, const FfxSolids* s, int storage,
                        const void* u, const void* v, const void* w,
                        const void* pu, const void* pv, const void* pw,
                        float dt, int corrected, float blend, const FfxSources* src,
                        const void* density, const void* temperature, float lift, float weight,
                        int apply_walls, void* ou, void* ov, void* ow, void* stream);
/* The same, reusing the predictor's departure points `dep` (ffx_face_predictor_trace
 * of the same faces and dt) instead of tracing again; used on grids whose extent, cell
 * count and spacing are powers of two, where both passes form the same start point, so
 * the result is unchanged (and the semi-Lagrangian sample is the predictor's value:
 * the stored face in FP32 storage, the fourth trace plane in BF16 storage; the
 * start velocity is the predictor's too).
 * dep == NULL or other grids: ffx_advect_velocity. */
int ffx_advect_velocity_trace(const FfxGrid* g, const FfxSolids* s, int storage,
                              const void* u, const void* v, const void* w,
                              const void* pu, const void* pv, const void* pw,
                              float dt, int corrected, float blend, const FfxSources* src,
                              const void* density, const void* temperature, float lift, float weight,
                              int apply_walls, void* ou, void* ov, void* ow,
                              const float* const dep[3], void* stream);
/* Plain face self-advection; replaces shaders/mac_advect_velocity.glsl. */
int ffx_mac_advect_velocity(const FfxGrid* g, int storage, const void* u, const void* v,
                            const void* w, float dt, void* ou, void* ov, void* ow, void* stream);
/* w_out = w_in + dt (lift*T - weight*rho), face averaged; replaces shaders/buoyancy.glsl. */
int ffx_buoyancy(const FfxGrid* g, int storage, const void* w_in, const void* density,
                 const void* temperature, float dt, float lift, float weight, void* w_out,
                 void* stream);

/* ------------------------------------------------------------ scalar passes */
typedef struct FfxScalarChannel {
    const void* field;      /* current scalar */
    const void* predictor;  /* MacCormack predictor (or == field) */
    const void* reverse;    /* MacCormack reverse (or == field) */
    void* out;
    float rate, decay;      /* emission rate; exp(-decay dt) */
    float target;           /* single-emitter form: >= 0 selects TARGET */
    int32_t channel;        /* table form: 0 density, 1 heat, 2 fuel */
    int32_t table_target;   /* table form: TARGET for this channel (heat extension) */
} FfxScalarChannel;

/* Closed (clamp-to-edge / collider-renormalised) semi-Lagrangian transport of
 * up to 3 scalars sharing one backtrace; dt < 0 gives the MacCormack reverse.
 * Replaces backend/detail.py:16-25 + shaders/transport_scalar.glsl. */
int ffx_scalar_transport(const FfxGrid* g, const FfxSolids* s, int storage,
                         const void* u, const void* v, const void* w, float dt, int count,
                         const void* const* in, void* const* out, void* stream);
/* The same, also storing each fluid cell's departure point in dep (three planes of
 * nx*ny*nz floats) for ffx_advect_scalars_trace (use it on the forward, +dt, pass). */
int ffx_scalar_transport_trace(const FfxGrid* g, const FfxSolids* s, int storage,
                               const void* u, const void* v, const void* w, float dt, int count,
                               const void* const* in, void* const* out, float* dep, void* stream);
/* Final scalar pass for up to 3 channels: MacCormack correction + clamp,
 * decay, emission. Replaces shaders/closed_advect_scalar.glsl,
 * multi_advect_scalar.glsl, correct_scalar.glsl (backend/projected.py:185-195).
 * If maxima != NULL, atomically raises maxima[c] to max|out_c|. */
int ffx_advect_scalars(const FfxGrid* g, const FfxSolids* s, int storage,
                       const void* u, const void* v, const void* w, float dt, int corrected,
                       const FfxSources* src, int count, const FfxScalarChannel* channels,
                       float* maxima, void* stream);
/* The same, reusing the forward predictor's departure points (same cells, velocity
 * and dt: the same start point), so the result is unchanged; in FP32 storage the
 * semi-Lagrangian samples are the predictor's values. */
int ffx_advect_scalars_trace(const FfxGrid* g, const FfxSolids* s, int storage,
                             const void* u, const void* v, const void* w, float dt, int corrected,
                             const FfxSources* src, int count, const FfxScalarChannel* channels,
                             float* maxima, const float* dep, void* stream);
/* The four transport passes above with the time step read on the device: `dt`
 * points at a float (the solver's clock, ffx_next_dt) that the kernels read,
 * times `sign` (+1 or -1: the reverse scalar pass) for ffx_scalar_transport_dt,
 * so a step whose dt the device chose needs no host readback. Results equal the
 * host-dt forms given the same dt value. */
int ffx_face_predictor_dt(const FfxGrid* g, const FfxSolids* s, int storage,
                          const void* u, const void* v, const void* w, const float* dt,
                          void* pu, void* pv, void* pw, float* const dep[3], void* stream);
int ffx_advect_velocity_dt(const FfxGrid* g, const FfxSolids* s, int storage,
                           const void* u, const void* v, const void* w,
                           const void* pu, const void* pv, const void* pw, const float* dt,
                           int corrected, float blend, const FfxSources* src,
                           const void* density, const void* temperature, float lift, float weight,
                           int apply_walls, void* ou, void* ov, void* ow, const float* const dep[3],
                           void* stream);
int ffx_scalar_transport_dt(const FfxGrid* g, const FfxSolids* s, int storage,
                            const void* u, const void* v, const void* w, const float* dt, float sign,
                            int count, const void* const* in, void* const* out, float* dep, void* stream);
int ffx_advect_scalars_dt(const FfxGrid* g, const FfxSolids* s, int storage,
                          const void* u, const void* v, const void* w, const float* dt, int corrected,
                          const FfxSources* src, int count, const FfxScalarChannel* channels,
                          float* maxima, const float* dep, void* stream);
/* The reverse scalar pass (ffx_scalar_transport with the forward pass's step
 * negated: `dt` < 0, or dtp != NULL: minus the device float *dtp) that also
 * decides the final pass's MacCormack correction of every fluid cell
 * (correct_scalar.glsl's conditions): its backtrace with -dt starts with the
 * final pass's forward midpoint and arrival point, so ok[c] = 1 exactly where
 * ffx_advect_scalars would correct cell c. `dep`: the forward pass's departure
 * points (ffx_scalar_transport_trace / _dt). An extension with no reference
 * counterpart; results equal those of the passes it replaces. */
int ffx_scalar_reverse_ok(const FfxGrid* g, const FfxSolids* s, int storage,
                          const void* u, const void* v, const void* w, float dt, const float* dtp,
                          int count, const void* const* in, void* const* out, const float* dep,
                          uint8_t* ok, void* stream);
/* The final scalar pass reading those decisions (and the forward departure
 * points) instead of tracing forward again: the result of ffx_advect_scalars_trace
 * (dtp == NULL) or ffx_advect_scalars_dt (dtp != NULL) with the same arguments. */
int ffx_advect_scalars_ok(const FfxGrid* g, const FfxSolids* s, int storage,
                          const void* u, const void* v, const void* w, float dt, const float* dtp,
                          int corrected, const FfxSources* src, int count,
                          const FfxScalarChannel* channels, float* maxima, const float* dep,
                          const uint8_t* ok, void* stream);
/* P0.2 open-boundary transport in an analytic flow; replaces shaders/advect.glsl. */
int ffx_advect_open(const FfxGrid* g, int storage, const void* in, float dt,
                    const float base[3], float angular, const float center[3], float radius,
                    float rate, float decay, void* out, void* stream);
/* P0.3 open-boundary transport by MAC velocity; replaces shaders/mac_advect_density.glsl. */
int ffx_mac_advect_density(const FfxGrid* g, int storage, const void* u, const void* v,
                           const void* w, const void* in, float dt, const float center[3],
                           float radius, float rate, float decay, void* out, void* stream);

/* --------------------------------------------------------------- projection */
/* Zero normal velocity on box walls and solid faces; replaces
 * backend/pressure.py:49-51 + shaders/pressure_walls.glsl. */
int ffx_walls(const FfxGrid* g, const FfxSolids* s, int storage, const void* u,
              const void* v, const void* w, void* ou, void* ov, void* ow, void* stream);
/* Cell divergence (0 in solids); replaces shaders/pressure_divergence.glsl. */
int ffx_divergence(const FfxGrid* g, const FfxSolids* s, int storage, const void* u,
                   const void* v, const void* w, float* div, void* stream);
/* Fused walls + divergence in one pass (backend/pressure.py:61-62). */
int ffx_walls_divergence(const FfxGrid* g, const FfxSolids* s, int storage,
                         const void* u, const void* v, const void* w,
                         void* ou, void* ov, void* ow, float* div, void* stream);
/* out = bounded - dt grad p on open faces, 0 on walls/solid faces; fused with
 * the divergence of the result (div_after, may be NULL) and the face maxima
 * max|u|,|v|,|w| (maxima[0..2], atomically raised, may be NULL). Replaces
 * backend/pressure.py:77-81 + shaders/pressure_gradient.glsl. */
int ffx_gradient(const FfxGrid* g, const FfxSolids* s, int storage,
                 const void* u, const void* v, const void* w, const float* pressure, float dt,
                 void* ou, void* ov, void* ow, float* div_after, float* maxima, void* stream);
/* The same with the collider test read from the level-0 link bytes of the same mask
 * (ffx_graph_links: one byte per cell, the open-face bits and the fluid bit): one load
 * per cell instead of twelve mask loads, the same result. */
int ffx_gradient_links(const FfxGrid* g, const FfxSolids* s, int storage,
                       const void* u, const void* v, const void* w, const float* pressure, float dt,
                       void* ou, void* ov, void* ow, float* div_after, float* maxima,
                       const uint8_t* links, void* stream);
/* Either of the two (links may be NULL), also writing to div_unrounded (may be
 * NULL) the divergence of the corrected faces before they are rounded to the
 * storage type: with BF16 storage the projection's FP32 result, which meets the
 * solve tolerance where the stored faces cannot (a BF16 face holds ~3 digits). */
int ffx_gradient_ex(const FfxGrid* g, const FfxSolids* s, int storage,
                    const void* u, const void* v, const void* w, const float* pressure, float dt,
                    void* ou, void* ov, void* ow, float* div_after, float* maxima,
                    const uint8_t* links, float* div_unrounded, void* stream);
/* One weighted-Jacobi sweep of the (masked) Neumann Laplacian on a level of
 * shape n[3] with 1/h = inv[3]; solid may be NULL. Replaces
 * shaders/pressure_jacobi.glsl. p_out must not alias p_in. */
int ffx_jacobi(const int32_t n[3], const float inv[3], const uint8_t* solid,
               const float* p_in, const float* rhs, float dt, float omega, float* p_out,
               void* stream);
/* out[i] = in[i] * factor; replaces shaders/pressure_scale.glsl. */
int ffx_scale(int64_t count, const float* in, float factor, float* out, void* stream);
/* out = a + b elementwise (FP32; out may alias a or b). */
int ffx_add(int64_t count, const float* a, const float* b, float* out, void* stream);

/* ------------------------------------------------- geometric multigrid (MG) */
/* r = rhs/dt - L p; replaces shaders/mg_residual.glsl. */
int ffx_mg_residual(const int32_t n[3], const float inv[3], const float* p, const float* rhs,
                    float dt, float* r, void* stream);
/* 2x2x2 average onto the coarse grid n/2; replaces shaders/mg_restrict.glsl. */
int ffx_mg_restrict(const int32_t fine_n[3], const float* fine, float* coarse, void* stream);
/* Fused residual + restriction (the fine residual is never stored). */
int ffx_mg_residual_restrict(const int32_t n[3], const float inv[3], const float* p,
                             const float* rhs, float dt, float* coarse_rhs, void* stream);
/* p_out = p + trilinear(coarse); replaces shaders/mg_prolong.glsl. */
int ffx_mg_prolong(const int32_t fine_n[3], const float* p, const float* coarse, float* p_out,
                   void* stream);
/* p = (inverse . rhs) / dt with an FP64 n x n pseudoinverse, FP64 accumulation;
 * replaces shaders/coarse_pressure.glsl (4^3) and shaders/solid_mg_direct.glsl
 * (dt = 1). n <= 1024. */
int ffx_direct_solve(int32_t n, const double* inverse, const float* rhs, float dt, float* p,
                     void* stream);
/* max|rhs/dt - L p| raised into *out (zeroed by the call). */
int ffx_mg_residual_max(const int32_t n[3], const float inv[3], const float* p,
                        const float* rhs, float dt, float* out, void* stream);

/* ------------------------------------- collider (aggregation) multigrid */
/* A level of the graph Laplacian. Level 0 derives its conductances from the
 * solid mask (edges == NULL): w[a] between two fluid cells, 0 otherwise. Coarse
 * levels carry explicit float4 (+x, +y, +z conductance, active) records. */
typedef struct FfxGraphLevel {
    int32_t nx, ny, nz;
    const float* edges;     /* 4 floats per cell, or NULL for level 0 */
    const uint8_t* solid;   /* level-0 mask when edges == NULL */
    float w[3];             /* level-0 conductances (n/extent)^2 */
    float coarse_scale;     /* factor of the coarse correction prolonged into this level
                               (over-correction); 0 or 1 = the plain prolongation */
    const uint8_t* links;   /* optional level-0 link bytes (ffx_graph_links); with
                               nx % 4 == 0 and 16-byte aligned fields the level-0
                               passes run four cells per thread. NULL: derive
                               the links from `solid` in every pass. */
} FfxGraphLevel;

/* The small coarse levels of one V-cycle in one kernel launch (one 1024-thread
 * block). Runs, on levels[0..count-1] (coarsest last), exactly the passes of
 * solid_multigrid.py:46-65 below the level that restricted into levels[0]:
 * levels[k].p is zeroed, `pre` sweeps, residual restricted into
 * levels[k+1].rhs; on the coarsest level the FP64 pseudoinverse `inverse`
 * (n x n, n <= 1024) is applied, or, with inverse == NULL, 80 sweeps from
 * zero; going up, prolongation fused with the first of `post` sweeps. Results
 * are bit-identical to the per-level entry points. Each sweep alternates a
 * level's p and q; the final iterate of levels[k] is in p when the level saw
 * an even number of sweeps (pre + post, or 80 / 0 on the coarsest), else in q.
 * Every level needs edges (no level 0), at most 32768 cells, and halves the
 * shape of the one before. Replaces that part of the per-level launch
 * sequence; no counterpart shader. */
#define FFX_TAIL_LEVELS 8
typedef struct FfxTailLevel {
    FfxGraphLevel level;
    float* p;
    float* q;
    float* rhs;
} FfxTailLevel;
typedef struct FfxGraphTail {
    int32_t count, pre, post;
    float omega;
    const double* inverse;
    FfxTailLevel levels[FFX_TAIL_LEVELS];
} FfxGraphTail;
int ffx_graph_tail(const FfxGraphTail* tail, void* stream);

/* Level-0 link bytes from the mask: bit 2a / 2a+1 = the face to the lower /
 * upper neighbour along axis a joins two fluid cells inside the domain, bit 6
 * = the cell is fluid. The level-0 conductances of
 * physics/solid_hierarchy.py:16-25 (w[a] on linked faces), one byte per cell.
 * Needs lv->solid and lv->edges == NULL; links holds nx*ny*nz bytes. */
int ffx_graph_links(const FfxGraphLevel* lv, uint8_t* links, void* stream);

/* omega-Jacobi on the graph Laplacian; replaces shaders/solid_mg_smooth.glsl
 * (omega = 2/3 there). p_out must not alias p_in. */
int ffx_graph_smooth(const FfxGraphLevel* lv, const float* p_in, const float* rhs,
                     float omega, float* p_out, void* stream);
/* ffx_graph_residual_max and ffx_graph_smooth of the same p in one pass: out[0]
 * = max |rhs - L p| (out is set first) and p_out = the sweep of p, both
 * bit-identical to the two entry points (on level 0 with links the terms are
 * formed once; other levels run the two launches). A solve loop that tests
 * convergence with it has the next cycle's first pre-sweep ready when it goes
 * on. An extension with no reference counterpart. */
int ffx_graph_residual_max_smooth(const FfxGraphLevel* lv, const float* p, const float* rhs,
                                  float omega, float* out, float* p_out, void* stream);
/* Two sweeps of ffx_graph_smooth in one pass: p_out = S(S(p_in)), bit-identical
 * to two ffx_graph_smooth launches. On a level-0 field with links (nx % 4 == 0,
 * aligned rows) the first sweep stays in shared memory (the iterate, right-hand
 * side and links are read once); on other levels it runs as two launches
 * through `tmp` (a field of the level's size, distinct from p_in and p_out; may
 * be NULL on level 0). An extension with no reference counterpart. */
int ffx_graph_smooth2(const FfxGraphLevel* lv, const float* p_in, const float* rhs, float omega,
                      float* tmp, float* p_out, void* stream);
/* The same for ffx_graph_prolong_smooth followed by one ffx_graph_smooth. */
int ffx_graph_prolong_smooth2(const FfxGraphLevel* lv, const float* p, const float* coarse,
                              const float* rhs, float omega, float* tmp, float* p_out, void* stream);
/* r = rhs - L p on active cells; replaces shaders/solid_mg_residual.glsl. */
int ffx_graph_residual(const FfxGraphLevel* lv, const float* p, const float* rhs, float* r,
                       void* stream);
/* Fused residual + 2x2x2 average restriction (solid_multigrid.py:56-59). */
int ffx_graph_residual_restrict(const FfxGraphLevel* lv, const float* p, const float* rhs,
                                float* coarse_rhs, void* stream);
/* The same, and coarse_p (the coarse level's iterate, may be NULL) set to zero
 * in the same pass: the next level of the V-cycle starts from it. */
int ffx_graph_residual_restrict_zero(const FfxGraphLevel* lv, const float* p, const float* rhs,
                                     float* coarse_rhs, float* coarse_p, void* stream);
/* p_out = active ? p + coarse[c/2] : 0; replaces shaders/solid_mg_prolong.glsl. */
int ffx_graph_prolong(const FfxGraphLevel* lv, const float* p, const float* coarse,
                      float* p_out, void* stream);
/* Fused prolongation + one smoothing sweep (the prolonged field is formed on the
 * fly for the 7-point stencil and never stored). */
int ffx_graph_prolong_smooth(const FfxGraphLevel* lv, const float* p, const float* coarse,
                             const float* rhs, float omega, float* p_out, void* stream);
/* max|rhs - L p| over active cells raised into *out (zeroed by the call). */
int ffx_graph_residual_max(const FfxGraphLevel* lv, const float* p, const float* rhs,
                           float* out, void* stream);
/* One Galerkin aggregation level (physics/solid_hierarchy.py:27-53): coarse
 * edges = boundary sums / 8, active = any active child. *disconnected (int32,
 * zeroed by the call) becomes nonzero if any aggregate joins children that are
 * not connected inside it; the caller then discards the level. */
int ffx_graph_coarsen(const FfxGraphLevel* fine, float* coarse_edges, int32_t* disconnected,
                      void* stream);
/* Materialise level-0 records (4 floats per cell) from the mask. */
int ffx_graph_level0_edges(const FfxGraphLevel* lv, float* edges, void* stream);

/* --------------------------------------- Krylov acceleration (MG-PCG) */
/* Conjugate gradients on A = -L (L the graph Laplacian of `lv`) preconditioned
 * by the aggregation V-cycle; an extension with no counterpart in the reference,
 * which cycles plain V-cycles (backend/solid_multigrid.py:67-76). Residuals use
 * the multigrid convention res = rhs - L x. FP64 scalars stay on the device. */
/* First smoothing sweep from a zero iterate (reads no iterate). */
int ffx_graph_smooth_zero(const FfxGraphLevel* lv, const float* rhs, float omega, float* p_out,
                          void* stream);
/* Smoothing sweep fused with *dot = scale * sum(rhs * p_out) (FP64; zeroed by the call). */
int ffx_graph_smooth_dot(const FfxGraphLevel* lv, const float* p_in, const float* rhs, float omega,
                         float* p_out, double* dot, double scale, void* stream);
/* ffx_graph_prolong_smooth fused with *dot = scale * (rhs . p_out) (FP64,
 * zeroed by the call): the last sweep of a preconditioning V-cycle that has
 * one post-sweep. No counterpart shader (MG-PCG extension). */
int ffx_graph_prolong_smooth_dot(const FfxGraphLevel* lv, const float* p, const float* coarse,
                                 const float* rhs, float omega, float* p_out, double* dot,
                                 double scale, void* stream);
/* p_out = z + (*rz_new / *rz_old) p_old (p_out = z when rz_old is NULL), q = A p_out,
 * *pq = sum(p_out * q) in FP64 (zeroed by the call). p_out must not alias p_old or z. */
int ffx_pcg_direction_apply(const FfxGraphLevel* lv, const float* z, const float* p_old,
                            const double* rz_new, const double* rz_old, float* p_out, float* q,
                            double* pq, void* stream);
/* alpha = *rz / *pq; x += alpha p; res += alpha q; *resmax = max|res| (zeroed by the call). */
int ffx_pcg_update(int64_t count, const double* rz, const double* pq, float* x, const float* p,
                   float* res, const float* q, float* resmax, void* stream);
/* *out = scale * sum(a * b), FP64 accumulation (zeroed by the call). */
int ffx_dot(int64_t count, const float* a, const float* b, double scale, double* out, void* stream);

/* --------------------------------------------------------------- reductions */
/* max|x| with NaN/Inf -> 3.4e38 into *out (zeroed by the call); replaces the
 * shaders/max_reduce.glsl chains of backend/timestep.py:24-33. */
int ffx_max_abs(int64_t count, int storage, const void* x, float* out, void* stream);
/* Divergence statistics (physics/pressure.py:70-80) of two float fields:
 * out[0..7] = sum(b^2), sum(a^2), max|b|, max|a|, sum(b), sum(a), n, 0 in FP64,
 * deterministic (fixed-order two-pass reduction). Needs `workspace` of
 * ffx_divergence_stats_workspace(count) bytes. */
size_t ffx_divergence_stats_workspace(int64_t count);
int ffx_divergence_stats(int64_t count, const float* before, const float* after,
                         double* out, void* workspace, size_t workspace_bytes, void* stream);
/* The same statistics for callers that cannot allocate device memory when they
 * ask for them (a host whose device memory is all owned by its own pool, a
 * real-time callback where cudaMalloc -- which may synchronise the device -- is
 * not allowed, a C caller with no allocator). No counterpart in the reference.
 * Allocates nothing: the block partials live in a fixed 56,832-byte array of
 * the library (at most 1184 blocks of six FP64 partials, whatever the count),
 * reserved on every GPU that loads it until the library is unloaded. Any
 * count >= 1 is accepted (count < 1 gives FFX_ERR_INVALID), and the result is
 * bit-identical to ffx_divergence_stats'. The first call on a device looks up
 * that array's device address (cudaGetSymbolAddress) with the device current;
 * make that first call before any stream capture. The address is cached per
 * device: after cudaDeviceReset it is stale, so reload the library. All calls
 * share the array: calls whose kernels overlap on the GPU race; calls ordered
 * on one stream do not, since each call rewrites every partial it reads. */
int ffx_divergence_stats_static(int64_t count, const float* before, const float* after,
                                double* out, void* stream);

/* ------------------------------------------------------- device solve loops */
/* A pressure solve to a tolerance as one CUDA graph with a WHILE node, so it
 * needs no host round trip (the V-cycle loop of backend/solid_multigrid.py:67-76
 * with the tolerance test decided on the device). ffx_loop_begin starts
 * capturing `stream` (a created stream, not the legacy default stream); the
 * caller issues the passes before the loop, the last of them ffx_loop_decide;
 * ffx_loop_while adds the WHILE node and returns in *body_stream a stream that
 * captures the loop body (one iteration, again ending with ffx_loop_decide);
 * ffx_loop_end_while closes the body; passes after the loop go to `stream`;
 * ffx_loop_end instantiates the graph and ffx_loop_launch runs the whole solve.
 * ffx_loop_decide: continue while counters[0] < max_cycles and
 * max|r| (*rmax) > tol * (*scale) with *scale > 0, in FP64; a continuing
 * decision adds one to counters[0] (this solve) and counters[1] (all solves);
 * counters[2] counts decisions. The loop ends by the cycle budget at the latest.
 * ffx_loop_reset_counter sets counters[0] = 0; ffx_zero_if_unscaled zeroes p
 * when *scale == 0 (a zero right-hand side). */
typedef struct FfxLoop FfxLoop;
int ffx_loop_begin(void* stream, FfxLoop** loop);
int ffx_loop_decide(FfxLoop* loop, const float* rmax, const float* scale, double tol,
                    int32_t max_cycles, int32_t* counters, void* stream);
int ffx_loop_reset_counter(int32_t* counters, void* stream);
int ffx_zero_if_unscaled(const float* scale, float* p, int64_t count, void* stream);
int ffx_loop_while(FfxLoop* loop, void** body_stream);
int ffx_loop_end_while(FfxLoop* loop);
int ffx_loop_end(FfxLoop* loop);
int ffx_loop_launch(FfxLoop* loop, void* stream);
int ffx_loop_destroy(FfxLoop* loop);
/* Device-side time-step rule (backend/timestep.py:35-53 in the workloads' form):
 * clock = float[2] {dt, previous dt}, time = one double. Sets previous dt = dt,
 * time += dt, and dt = min(dt_max, cfl * cell / max(maxima[0..2])) in FP64
 * (dt_max when the maxima are zero); cell, cfl > 0, dt_max in (0, 0.1]. */
int ffx_next_dt(const float* maxima, float* clock, double* time, double cell, double cfl,
                double dt_max, void* stream);
/* p *= clock[0] / clock[1] when clock[1] > 0 and the ratio differs from 1 by more
 * than 1e-6 (FP64): the impulse warm start's rescaling (backend/pressure.py:63-75)
 * with the time steps on the device. */
int ffx_scale_by_ratio(int64_t count, float* p, const float* clock, void* stream);
/* Warm start extrapolated linearly in time (an extension; the reference's warm
 * start is the ratio rule of ffx_scale_by_ratio, backend/pressure.py:63-75). The
 * impulse pressure is dt times the pressure per unit time P. With P1 = p / clock[1]
 * (the last solve) and P2 = hist (the same quantity from the solve before), sets
 * p = clock[0] * (P1 + beta * (clock[0] / clock[1]) * (P1 - P2)) and hist = P1.
 * first = 1 (no older solve): p takes ffx_scale_by_ratio's rule and hist = P1.
 * Nothing changes when clock[1] <= 0. beta in [0, 1]; p and hist distinct,
 * 16-byte aligned, count floats each. */
int ffx_extrapolate_pressure(int64_t count, float* p, float* hist, const float* clock, float beta,
                             int32_t first, void* stream);
/* Quadratic form (an extension): P1 = p / clock[1], P2 = h_new and P3 = h_old (the
 * two earlier solves, per unit time) at times 0, -clock[1] and -clock[1] - *dprev_r;
 * Q = their Lagrange quadratic at clock[0]; p = clock[0] * (P1 + beta * (Q - P1)).
 * have = earlier solves stored: 0 applies ffx_scale_by_ratio's rule, 1 the linear
 * form of ffx_extrapolate_pressure with h_new, 2 the quadratic. Every call writes
 * P1 over h_old and clock[1] to *dprev_w; the caller then swaps h_new / h_old and
 * dprev_r / dprev_w. Nothing changes when clock[1] <= 0. p, h_new and h_old are
 * distinct, 16-byte aligned, count floats each. */
int ffx_extrapolate_pressure2(int64_t count, float* p, const float* h_new, float* h_old,
                              const float* clock, const float* dprev_r, float* dprev_w, float beta,
                              int32_t have, void* stream);

/* ------------------------------------------------------- sparse brick path */
/* Brick pool: the topology of FluxFX_Source/native/bricks.hpp:14-94 (fixed
 * capacity 1..262144, brick coordinates in [-2^20, 2^20 - 1], open addressing with
 * tombstones, a removed slot is the next one handed out, atomic box activation
 * with a capacity preflight). Host memory only. */
typedef struct FfxBrickPool FfxBrickPool;
typedef struct FfxBrickStats {
    uint32_t capacity, active;
    uint64_t metadata_bytes;   /* constant after creation: all storage is reserved */
} FfxBrickStats;
int ffx_bricks_create(uint32_t capacity, FfxBrickPool** pool);
int ffx_bricks_destroy(FfxBrickPool* pool);
int ffx_bricks_lookup(const FfxBrickPool* pool, int32_t x, int32_t y, int32_t z, int32_t* slot);
int ffx_bricks_activate(FfxBrickPool* pool, int32_t x, int32_t y, int32_t z, int32_t* slot);
int ffx_bricks_deactivate(FfxBrickPool* pool, int32_t x, int32_t y, int32_t z, int32_t* was_active);
/* slots of the -x, +x, -y, +y, -z, +z neighbours (-1: inactive) */
int ffx_bricks_neighbors(const FfxBrickPool* pool, int32_t x, int32_t y, int32_t z, int32_t out[6]);
int ffx_bricks_activate_box(FfxBrickPool* pool, const int32_t lo[3], const int32_t extent[3]);
int ffx_bricks_stats(const FfxBrickPool* pool, FfxBrickStats* out);
/* active slots (stats.active of them) and the coordinates of every slot (3 per
 * slot); both arrays hold room >= capacity entries */
int ffx_bricks_active(const FfxBrickPool* pool, int32_t* slots, int32_t* coords_by_slot, uint32_t room);
/* Arena: a GPU-independent suballocator of one buffer (FluxFX_Source/native/
 * arena.hpp:12-57): capacity a positive multiple of 256; spans aligned to 256 bytes,
 * first fit in address order, adjacent free spans merged on release; handles are
 * unique across all arenas and never reused; at most 65536 live spans. */
typedef struct FfxArena FfxArena;
typedef struct FfxArenaStats {
    uint64_t capacity, used, peak, allocations, live, largest_free;
} FfxArenaStats;
int ffx_arena_create(uint64_t capacity, FfxArena** arena);
int ffx_arena_destroy(FfxArena* arena);
int ffx_arena_allocate(FfxArena* arena, uint64_t bytes, uint64_t* handle);
int ffx_arena_get(const FfxArena* arena, uint64_t handle, uint64_t* offset, uint64_t* bytes, uint64_t* requested);
int ffx_arena_release(FfxArena* arena, uint64_t handle);
int ffx_arena_stats(const FfxArena* arena, FfxArenaStats* out);
/* One level of the sparse projection (FluxFX_Source/native/projection.mm:15-120):
 * n^3 unit cells (n a multiple of side, side 8 or 16), solve region `mode` (0 all,
 * 1 the central box [n/4, 3n/4)^3, 2 the boxes [n/8, 3n/8)^3 and [5n/8, 7n/8)^3).
 * sparse != 0: fields hold side^3 values per brick slot, local (z*side + y)*side + x,
 * faces the side^3 faces at the lower side of each cell per axis (upper-wall faces
 * are zero, not stored); map = (n/side)^3 slots (-1 inactive), active = the
 * `count` slots to sweep, coords = 3 per slot. sparse == 0: n^3 cells and
 * (n+1) n^2 faces per axis, x-fast. `faces` is the per-axis stride of a face
 * array. Sparse and dense give identical values on the solve region. */
typedef struct FfxSparseLevel {
    int32_t n, side, mode, sparse;
    const int32_t* map;
    const int32_t* active;
    const int32_t* coords;
    int32_t count;
} FfxSparseLevel;
int ffx_sparse_divergence(const FfxSparseLevel* l, const float* u, int32_t faces, float* out, void* stream);
/* out = q + 2/3 ((sum of in-domain neighbours - rhs) / their count - q) on solve cells, 0 elsewhere */
int ffx_sparse_jacobi(const FfxSparseLevel* l, const float* q, const float* rhs, float* out, void* stream);
int ffx_sparse_residual(const FfxSparseLevel* l, const float* q, const float* rhs, float* out, void* stream);
/* out = u - (q(c) - q(c - e)) on faces with a solve cell beside them, 0 elsewhere */
int ffx_sparse_gradient(const FfxSparseLevel* l, const float* u, const float* q, int32_t faces, float* out,
                        void* stream);
int ffx_sparse_restrict(const FfxSparseLevel* fine, const float* residual, const FfxSparseLevel* coarse,
                        float* coarse_rhs, void* stream);
int ffx_sparse_prolong(const FfxSparseLevel* coarse, const float* correction, const FfxSparseLevel* fine,
                       float* q, void* stream);

/* ------------------------------------------------------------- bake readback */
/* Storage code of a uint8 field (the collider mask) for ffx_pack_channels. */
enum { FFX_PACK_U8 = 2 };
/* Packs `channels` (1..8) fields of `count` values each -- kinds[c] is FFX_F32,
 * FFX_BF16 or FFX_PACK_U8 -- into out[c * count + i] as FP32: the frame layout of
 * the playback cache (channel after channel, x-fast), so one device-to-host copy
 * of `out` carries a whole baked frame. Replaces the per-channel texture reads of
 * backend/cache.py:7-11 (capture). */
int ffx_pack_channels(int64_t count, int channels, const void* const* fields, const int* kinds,
                      float* out, void* stream);

/* ------------------------------------------------------ fire configuration */
/* Cell vorticity (omega.xyz, |omega|) as float4 per cell, central differences of
 * the cell-centred velocity with clamped reads; replaces shaders/curl.glsl
 * (backend/detail.py:39-49). */
int ffx_curl(const FfxGrid* g, int storage, const void* u, const void* v, const void* w,
             float* curl4, void* stream);
/* Vorticity confinement on every face: out = in + dt * (force(c) + force(c - e_a)) / 2 . e_a,
 * force = strength * h * normalize(grad|omega|) x omega capped at `limit`; replaces
 * shaders/confinement.glsl. Outputs must not alias inputs. */
int ffx_confine(const FfxGrid* g, int storage, const float* curl4, const void* u, const void* v,
                const void* w, float dt, float strength, float limit, void* ou, void* ov,
                void* ow, void* stream);
/* Combustion in one pass (backend/combustion.py:21-31, combustion_burn.glsl,
 * combustion_apply.glsl): flame = (T >= ignition ? max(fuel,0)(1 - exp(-rate dt)) : 0)/dt;
 * fuel -= dt flame (clamped at 0), density += dt smoke_yield flame, temperature +=
 * dt heat_yield flame. Outputs may alias their inputs (elementwise). */
int ffx_combustion(const FfxGrid* g, int storage, const void* fuel, const void* temperature,
                   const void* density, float dt, float ignition, float burn_rate,
                   float smoke_yield, float heat_yield, float* flame, void* fuel_out,
                   void* density_out, void* temperature_out, void* stream);
/* Owner mask of moving colliders: 1-based index of the first collider holding
 * each cell centre (FP32 test of 12 inverse-affine coefficients per collider,
 * sphere or box), 0 = fluid; replaces shaders/moving_mask.glsl
 * (backend/moving_collision.py:44-58). count <= FFX_MOVING_MAX. rows12 and
 * is_box are HOST arrays (passed to the kernel by value). */
int ffx_moving_mask(const FfxGrid* g, int count, const float* rows12, const int32_t* is_box,
                    uint8_t* owners, void* stream);
/* Rigid wall velocity (row . (p, 1), 3 rows of 4 per collider in the HOST array
 * `table`) on every interior face next to a solid cell, 0 elsewhere; replaces
 * shaders/moving_wall.glsl. */
int ffx_moving_walls(const FfxGrid* g, const uint8_t* owners, int count, const float* table,
                     float* wu, float* wv, float* ww, void* stream);
/* In-place remap after a move (backend/moving_collision.py:64-80,
 * moving_remap_scalar.glsl, moving_remap_face.glsl): scalars (scalar1, scalar2
 * may be NULL) zeroed in cells solid now or before; faces take the wall velocity
 * where blocked, 0 where just uncovered, 0 on domain walls. */
int ffx_moving_remap(const FfxGrid* g, int storage, const uint8_t* owners,
                     const uint8_t* old_owners, void* scalar0, void* scalar1, void* scalar2,
                     void* u, void* v, void* w, const float* wu, const float* wv,
                     const float* ww, void* stream);

/* ------------------------------------------------ batched domains (a19) */
/* No counterpart in the reference (it runs one domain per solver object): many
 * independent FP32 collider-path smoke domains of uneven sizes advance
 * together, one persistent launch per pass over all of them. Each domain
 * follows exactly the single-domain step of backend/projected.py:149-202 with
 * static colliders, MacCormack (or semi-Lagrangian) transport, buoyancy,
 * table emitters, the aggregation multigrid of backend/solid_multigrid.py:46-76
 * run as stand-alone V-cycles until max|rhs - L p| <= tolerance * max|rhs|
 * (pressure from zero every step, or warm-started), and the time step
 * dt = min(dt_max, cfl * cell / max|u|) computed on the device from the
 * projection's velocity maxima. Results are bit-identical to running each
 * domain alone through the single-domain entry points. */
#define FFX_BATCH_MAX 64
#define FFX_BATCH_LEVELS 8
typedef struct FfxBatchLevel {
    FfxGraphLevel level;   /* level 0: edges NULL, solid = the collider mask */
    float* p;              /* iterate (level 0: the pressure) */
    float* q;              /* sweep partner (level 0: the spare pressure) */
    float* rhs;            /* right-hand side (level 0: the divergence) */
} FfxBatchLevel;
typedef struct FfxBatchDomain {
    FfxGrid grid;
    const uint8_t* solid;  /* collider mask (all zero for a domain without colliders) */
    const uint8_t* halo;   /* its dilation (ffx_dilate_mask) */
    float* u; float* v; float* w;      /* velocity faces, updated in place every step */
    float* pu; float* pv; float* pw;   /* face predictor scratch */
    float* bu; float* bv; float* bw;   /* walled (bounded) faces scratch */
    float* density[2];                 /* [front, back]: front holds the field before an even step */
    float* temperature[2];
    float* predictor[2];               /* scalar MacCormack predictor scratch (density, temperature) */
    float* reverse[2];
    float* after;                      /* divergence after the projection */
    FfxSources sources;                /* emitter table (count 0..8) or single emitter (count < 0) */
    int32_t velocity_corrected, scalar_corrected;   /* MacCormack (1) or semi-Lagrangian (0) */
    float blend, lift, weight;
    FfxScalarChannel density_channel;  /* rate, decay, target, channel, table_target (pointers unused) */
    FfxScalarChannel heat_channel;
    double cell, cfl, dt_max;          /* time step rule */
    float dt0;                         /* time step of the first step */
    int32_t levels;                    /* multigrid hierarchy, finest first */
    FfxBatchLevel level[FFX_BATCH_LEVELS];
    int32_t tail_start;                /* first level run by the single-block tail, or -1 */
    const double* inverse;             /* FP64 pseudoinverse of the coarsest level, or NULL */
    int32_t pre, post, max_cycles;     /* sweeps per V-cycle (both >= 1), cycle cap per solve */
    int32_t warm_start;                /* 1: start each solve from the previous step's pressure scaled by
                                          dt / previous dt (backend/pressure.py:63-75), 0: from zero */
    double tolerance;                  /* relative max-norm residual target (> 0) */
    float* face_trace[3];              /* optional traces of the face predictor (six planes per face
                                          grid, the FP32 layout of ffx_face_predictor_trace;
                                          power-of-two grids only), reused by the velocity pass as in
                                          ffx_advect_velocity_trace */
    float* cell_trace;                 /* optional departure points of the scalar predictor (three
                                          planes of cells), reused by the final scalar pass */
    const uint8_t* clear;              /* optional clearance of the mask (ffx_clearance), as FfxSolids.clear */
    uint8_t* cell_ok;                  /* optional, with cell_trace: one byte per cell, the reverse scalar
                                          pass's correction decisions (as ffx_scalar_reverse_ok) */
} FfxBatchDomain;
typedef struct FfxBatchStats {
    float dt, last_dt;                 /* dt of the next step, of the last step */
    int32_t last_cycles, total_cycles, steps;
    float maxima[3];
    double time;
    int64_t loop_iterations;           /* solve-loop iterations of the whole batch since creation */
} FfxBatchStats;
typedef struct FfxBatchPlan FfxBatchPlan;
/* Device bytes the plan of these domains needs (descriptors and state). */
int ffx_batch_workspace_bytes(const FfxBatchDomain* domains, int32_t count, int64_t* bytes);
/* Build a plan in the caller's device workspace (synchronous upload). */
int ffx_batch_create(const FfxBatchDomain* domains, int32_t count, void* workspace, int64_t bytes,
                     FfxBatchPlan** plan);
/* Pass kinds of a batched step (the autotuner's keys). */
enum {
    FFX_PASS_PREDICTOR = 0, FFX_PASS_VELOCITY, FFX_PASS_DIVERGENCE, FFX_PASS_SCALE, FFX_PASS_GRADIENT,
    FFX_PASS_SCALAR_PREDICTOR, FFX_PASS_SCALAR_REVERSE, FFX_PASS_SCALAR_FINAL, FFX_PASS_RESIDUAL_MAX,
    FFX_PASS_SMOOTH, FFX_PASS_RESIDUAL_RESTRICT, FFX_PASS_PROLONG_SMOOTH, FFX_PASS_DIRECT,
    /* level 0 four cells per thread (link field, nx % 4 == 0; fixed 32 x 8 tiles, grid tuned) */
    FFX_PASS_L0_SMOOTH, FFX_PASS_L0_PROLONG_SMOOTH, FFX_PASS_L0_RESIDUAL_RESTRICT, FFX_PASS_L0_RESIDUAL_MAX,
    FFX_PASS_KINDS
};
/* Tile shape (0: 32x8, 1: 64x4, 2: 128x2, 3: 16x16 threads) and persistent grid
 * (0: one block per tile; m >= 1: m x the resident blocks of the GPU) of one
 * pass kind. Takes effect for graphs captured afterwards. */
int ffx_batch_set_config(FfxBatchPlan* plan, int32_t kind, int32_t shape, int32_t grid);
/* Launch one pass kind alone over the plan's buffers (autotuning; the pass only
 * writes scratch fields that the step recomputes, the gradient pass writes the
 * predictor faces instead of the velocity). */
int ffx_batch_tune_pass(FfxBatchPlan* plan, int32_t kind, void* stream);
/* Capture `steps` steps (starting from the plan's current parity) into an
 * instantiated CUDA graph with one conditional WHILE node per solve. */
int ffx_batch_graph(FfxBatchPlan* plan, int32_t steps, void** graph_exec);
/* Launch such a graph; advances the plan's parity by its step count. */
int ffx_batch_launch(FfxBatchPlan* plan, void* graph_exec, int32_t steps, void* stream);
int ffx_batch_graph_free(void* graph_exec);
/* Host copy of every domain's FfxBatchStats (synchronises `stream`). */
int ffx_batch_stats(const FfxBatchPlan* plan, FfxBatchStats* out, void* stream);
/* Current parity: 0 = density[0]/temperature[0] hold the fields. */
int ffx_batch_parity(const FfxBatchPlan* plan);
int ffx_batch_destroy(FfxBatchPlan* plan);

/* ------------------------------------------------- learned warm start (a18) */
/* No counterpart in the reference: a 3D U-Net predicts the pressure from the
 * divergence and the collider mask. Activations are NDHWC bfloat16 addressed
 * through views (data, elements per voxel, first channel); every channel
 * count, pitch and offset is a multiple of 8 and data is 16-byte aligned. */
typedef struct FfxTensorView {
    const void* data;
    int32_t pitch, offset;
} FfxTensorView;
typedef struct FfxConv {
    int32_t batch;
    int32_t in_dims[3];      /* d, h, w of the input grid */
    int32_t out_dims[3];     /* d, h, w of the output grid */
    int32_t c1, c2, cout;    /* input channels read from in1, then in2 (concatenated; c2 may be 0) */
    int32_t ksize, stride, pad;
    int32_t transposed;      /* 1: 2^3 stride-2 transposed convolution onto the doubled grid */
    FfxTensorView in1, in2;
    const void* weight;      /* bf16 [taps][c1 + c2][cout] (transposed: taps = 8 parity classes) */
    const float* bias;       /* optional, FP32 [cout] */
    int32_t relu, accumulate; /* ReLU on the result; add to the existing BF16 output */
    void* out; int32_t out_pitch, out_offset;   /* optional BF16 output view */
    float* out_f32; int32_t out_f32_pitch;      /* optional FP32 output */
} FfxConv;
/* Convolution as an implicit GEMM on the BF16 tensor cores (FP32 accumulation). */
int ffx_conv_forward(const FfxConv* conv, void* stream);
/* The same on the 5th-generation tensor cores (tcgen05.mma, accumulator in tensor
 * memory, bounded completion waits). */
int ffx_conv_forward_tc(const FfxConv* conv, void* stream);
/* 3x3x3 stride-1 pad-1 convolutions without an operand gather: each block stages its
 * input halo tile by TMA tensor loads (cp.async.bulk.tensor, zero fill = padding) and runs
 * every tap as a shifted shared-memory descriptor into tcgen05.mma (accumulators in tensor
 * memory). The weights come pre-packed (ffx_conv_pack_weights, `packed_bytes` from
 * ffx_conv_packed_bytes; 0 for shapes the kernel does not tile). 1x1 and transposed 2^3
 * layers with 8 or 16 output channels run a per-voxel CUDA-core kernel, the other shapes
 * (2^3 stride 2, wider layers) the ffx_conv_forward kernel; both ignore `packed`. */
int ffx_conv_packed_bytes(const FfxConv* conv, int64_t* packed_bytes);
int ffx_conv_pack_weights(const FfxConv* conv, void* packed, void* stream);
int ffx_conv_forward_tma(const FfxConv* conv, const void* packed, void* stream);
/* Number of tcgen05 convolution launches that gave up waiting (synchronous; reset != 0
 * clears it). */
int ffx_conv_timeouts(int32_t* out, int32_t reset);
/* dweight[k][cout] += sum over output voxels of input(k) * grad (FP32, caller zeroes);
 * `grad` is the BF16 gradient of the convolution's output (ReLU already applied). */
int ffx_conv_weight_grad(const FfxConv* conv, const void* grad, int32_t grad_pitch, float* dweight,
                         void* stream);
/* dy *= (y > 0) in place. */
int ffx_relu_backward(int64_t voxels, int32_t channels, void* dy, int32_t dy_pitch, const void* y,
                      int32_t y_pitch, int32_t y_offset, void* stream);
/* dbias[c] += sum over voxels of g[v][c] (channels <= 128, dividing 256). */
int ffx_bias_grad(int64_t voxels, int32_t channels, const void* g, int32_t pitch, float* dbias,
                  void* stream);
/* Weights of the data-gradient convolution: dst[t][co][ci] = src[flip ? taps-1-t : t][ci][co]. */
int ffx_weight_transpose(int32_t taps, int32_t cin, int32_t cout, int32_t flip, const void* src,
                         void* dst, void* stream);
/* Adam step on FP32 master weights w (moments m, v) with gradient g; w_bf16 (optional)
 * receives the rounded weights. */
int ffx_adam(int64_t n, float* w, float* m, float* v, const float* g, void* w_bf16, float lr,
             float beta1, float beta2, float eps, int32_t step, void* stream);
/* Network input, 8 BF16 channels per voxel: scale * div, solid mask, zeros. */
int ffx_pack_input(int64_t voxels, const float* div, const uint8_t* mask, float scale, void* out,
                   void* stream);
/* The same with scale = 1 / *max_abs (0 when *max_abs is 0) formed on the device, so the
 * caller need not read max |div| back (max_abs: ffx_max_abs of div). */
int ffx_pack_input_scaled(int64_t voxels, const float* div, const uint8_t* mask, const float* max_abs,
                          void* out, void* stream);
/* Collider mask of the 2x coarser grid (dims coarse_n): 1 where at least `threshold`
 * of the eight children are nonzero. */
int ffx_mask_restrict(const int32_t coarse_n[3], const uint8_t* fine, int32_t threshold, uint8_t* coarse,
                      void* stream);
/* out[v] = src[v * pitch] * scale: one channel of the FP32 network output as a cell field. */
int ffx_unpack_channel(int64_t voxels, const float* src, int32_t pitch, float scale, float* out,
                       void* stream);
/* The same with scale = 1 / ((1 / *max_abs) * weight) formed on the device in FP64 (0 when
 * *max_abs is 0): the factor that undoes ffx_pack_input_scaled's normalisation. */
int ffx_unpack_channel_scaled(int64_t voxels, const float* src, int32_t pitch, const float* max_abs,
                              double weight, float* out, void* stream);
/* *loss += sum over fluid voxels of (pred - target)^2 * inv_count; grad (8 BF16
 * channels per voxel) = its derivative in channel 0. */
int ffx_mse_grad(int64_t voxels, const float* pred, int32_t pred_pitch, const float* target,
                 const uint8_t* mask, float inv_count, void* grad, double* loss, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FFX_H */
