// The reference's hot-path compute shaders compiled for the CPU -- TEST
// INFRASTRUCTURE ONLY (the checker's "reference" leg).
//
// Each kernel is one namespace holding the shader sources exactly as the
// reference's device adapter concatenates them (includes first, then the
// kernel file; collider variants prepend solid_boundary.glsl, see
// fluxfx/backend/device.py:43-55 and fluxfx/backend/collision.py:51-58). The
// sources are pulled in with #include from the directory given by the build
// recipe (oracle/glsl_ref/build.py), never copied into this repository.
//
// C ABI (ctypes): pick a kernel by shader file name, set uniforms and
// samplers by their GLSL names, bind the output image, dispatch over a grid.
// A dispatch runs main() once per invocation with OpenMP over z slices.
#include <cstring>
#include <string>
#include <vector>

#include "glsl.hpp"

namespace glsl {
thread_local long long g_out_of_range = 0;
thread_local InvocationID gl_GlobalInvocationID;
}  // namespace glsl

namespace glsl_state {
using namespace glsl;
// uniforms (push constants) of every hot-path shader
ivec3 gridSize;
vec3 domainExtent, cellCount, faceOffset, axisMask, invCell, sourceCenter, sourceStart, baseVelocity,
    emissionVelocity;
vec4 row0, row1, row2;
float dt, relaxation, componentAxis, factor, sourceRadius, sourceProfile, sourceRate, dissipation, targetDensity,
    correctedTransport, correctedVelocity, emissionCoupling, sourceCount, scalarChannel, thermalLift, densityWeight,
    seedTemperature, angularSpeed, shapeKind, curlStrength, forceLimit, ignitionTemperature, burnRate, yieldValue,
    owner;
// samplers and the output image
sampler3D inputField, velocityU, velocityV, velocityW, divergenceField, pressureField, coarseField, inverseField,
    edgeField, solidField, densityField, temperatureField, predictorField, reverseField, originalFaceField,
    facePredictor, sourceTable, curlField, burnField, boundaryField, oldSolidField, wallTable;
image3D outputField;
}  // namespace glsl_state

#define FFX_KERNEL_BEGIN(NS) namespace NS { using namespace glsl; using namespace glsl_state;
#define FFX_KERNEL_END }

// ------------------------------------------------------------- plain kernels
FFX_KERNEL_BEGIN(k_seed)
#include "seed.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_temperature_seed)
#include "temperature_seed.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_mac_seed)
#include "mac_seed.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_advect)
#include "advect.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_mac_advect_velocity)
#include "mac_sample.glsl"
#include "mac_advect_velocity.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_mac_advect_density)
#include "mac_sample.glsl"
#include "mac_advect_density.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_buoyancy)
#include "buoyancy.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_pressure_walls)
#include "pressure_walls.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_pressure_divergence)
#include "pressure_divergence.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_pressure_jacobi)
#include "pressure_jacobi.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_pressure_gradient)
#include "pressure_gradient.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_pressure_scale)
#include "pressure_scale.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_mg_residual)
#include "mg_residual.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_mg_restrict)
#include "mg_restrict.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_mg_prolong)
#include "mg_prolong.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_coarse_pressure)
#include "coarse_pressure.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_transport_face)
#include "mac_sample.glsl"
#include "transport_face.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_transport_scalar)
#include "mac_sample.glsl"
#include "closed_sample.glsl"
#include "transport_scalar.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_closed_advect_scalar)
#include "mac_sample.glsl"
#include "emission_weight.glsl"
#include "closed_sample.glsl"
#include "correct_scalar.glsl"
#include "closed_advect_scalar.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_emitting_advect_velocity)
#include "mac_sample.glsl"
#include "emission_weight.glsl"
#include "correct_velocity_fused.glsl"
#include "emitting_advect_velocity.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_multi_advect_velocity)
#include "mac_sample.glsl"
#include "source_table.glsl"
#include "correct_velocity_fused.glsl"
#include "multi_advect_velocity.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_multi_advect_scalar)
#include "mac_sample.glsl"
#include "source_table.glsl"
#include "closed_sample.glsl"
#include "correct_scalar.glsl"
#include "multi_advect_scalar.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_max_reduce)
#include "max_reduce.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_solid_mask)
#include "solid_mask.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_solid_mg_smooth)
#include "solid_mg_operator.glsl"
#include "solid_mg_smooth.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_solid_mg_residual)
#include "solid_mg_operator.glsl"
#include "solid_mg_residual.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_solid_mg_prolong)
#include "solid_mg_prolong.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_solid_mg_direct)
#include "solid_mg_direct.glsl"
FFX_KERNEL_END

// ------------------------------------------- fire-config passes (C5 rows)
FFX_KERNEL_BEGIN(k_curl)
#include "curl.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_confinement)
#include "confinement.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_combustion_burn)
#include "combustion_burn.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_combustion_apply)
#include "combustion_apply.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_moving_mask)
#include "moving_mask.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_moving_wall)
#include "moving_wall.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_moving_remap_scalar)
#include "moving_remap_scalar.glsl"
FFX_KERNEL_END
FFX_KERNEL_BEGIN(k_moving_remap_face)
#include "moving_remap_face.glsl"
FFX_KERNEL_END

// ---------------------------------------------- collider-decorated variants
// solid_boundary.glsl #defines FLUXFX_COLLISIONS; it is undefined again after
// every variant so the next namespace starts clean.
FFX_KERNEL_BEGIN(ks_pressure_walls)
#include "solid_boundary.glsl"
#include "pressure_walls.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_pressure_jacobi)
#include "solid_boundary.glsl"
#include "pressure_jacobi.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_pressure_gradient)
#include "solid_boundary.glsl"
#include "pressure_gradient.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_solid_clear)
#include "solid_boundary.glsl"
#include "solid_clear.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_transport_face)
#include "solid_boundary.glsl"
#include "mac_sample.glsl"
#include "transport_face.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_transport_scalar)
#include "solid_boundary.glsl"
#include "mac_sample.glsl"
#include "closed_sample.glsl"
#include "transport_scalar.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_closed_advect_scalar)
#include "solid_boundary.glsl"
#include "mac_sample.glsl"
#include "emission_weight.glsl"
#include "closed_sample.glsl"
#include "correct_scalar.glsl"
#include "closed_advect_scalar.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_emitting_advect_velocity)
#include "solid_boundary.glsl"
#include "mac_sample.glsl"
#include "emission_weight.glsl"
#include "correct_velocity_fused.glsl"
#include "emitting_advect_velocity.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_multi_advect_velocity)
#include "solid_boundary.glsl"
#include "mac_sample.glsl"
#include "source_table.glsl"
#include "correct_velocity_fused.glsl"
#include "multi_advect_velocity.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
FFX_KERNEL_BEGIN(ks_multi_advect_scalar)
#include "solid_boundary.glsl"
#include "mac_sample.glsl"
#include "source_table.glsl"
#include "closed_sample.glsl"
#include "correct_scalar.glsl"
#include "multi_advect_scalar.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS

// Moving colliders (backend/moving_collision.py:23-37): walls and gradient get
// solid_boundary.glsl + moving_boundary.glsl (FLUXFX_MOVING_COLLIDERS, wall
// velocities from boundaryField; variant 2); the divergence gets
// solid_boundary.glsl (variant 1).
FFX_KERNEL_BEGIN(km_pressure_walls)
#include "solid_boundary.glsl"
#include "moving_boundary.glsl"
#include "pressure_walls.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
#undef FLUXFX_MOVING_COLLIDERS
FFX_KERNEL_BEGIN(km_pressure_gradient)
#include "solid_boundary.glsl"
#include "moving_boundary.glsl"
#include "pressure_gradient.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS
#undef FLUXFX_MOVING_COLLIDERS
FFX_KERNEL_BEGIN(km_pressure_divergence)
#include "solid_boundary.glsl"
#include "pressure_divergence.glsl"
FFX_KERNEL_END
#undef FLUXFX_COLLISIONS

// ------------------------------------------------------------------ tables
namespace {
using namespace glsl;
using namespace glsl_state;

struct KernelEntry {
    const char* file;
    int collisions;
    void (*main)();
};

const KernelEntry kKernels[] = {
    {"seed.glsl", 0, k_seed::main},
    {"temperature_seed.glsl", 0, k_temperature_seed::main},
    {"mac_seed.glsl", 0, k_mac_seed::main},
    {"advect.glsl", 0, k_advect::main},
    {"mac_advect_velocity.glsl", 0, k_mac_advect_velocity::main},
    {"mac_advect_density.glsl", 0, k_mac_advect_density::main},
    {"buoyancy.glsl", 0, k_buoyancy::main},
    {"pressure_walls.glsl", 0, k_pressure_walls::main},
    {"pressure_divergence.glsl", 0, k_pressure_divergence::main},
    {"pressure_jacobi.glsl", 0, k_pressure_jacobi::main},
    {"pressure_gradient.glsl", 0, k_pressure_gradient::main},
    {"pressure_scale.glsl", 0, k_pressure_scale::main},
    {"mg_residual.glsl", 0, k_mg_residual::main},
    {"mg_restrict.glsl", 0, k_mg_restrict::main},
    {"mg_prolong.glsl", 0, k_mg_prolong::main},
    {"coarse_pressure.glsl", 0, k_coarse_pressure::main},
    {"transport_face.glsl", 0, k_transport_face::main},
    {"transport_scalar.glsl", 0, k_transport_scalar::main},
    {"closed_advect_scalar.glsl", 0, k_closed_advect_scalar::main},
    {"emitting_advect_velocity.glsl", 0, k_emitting_advect_velocity::main},
    {"multi_advect_velocity.glsl", 0, k_multi_advect_velocity::main},
    {"multi_advect_scalar.glsl", 0, k_multi_advect_scalar::main},
    {"max_reduce.glsl", 0, k_max_reduce::main},
    {"solid_mask.glsl", 0, k_solid_mask::main},
    {"solid_mg_smooth.glsl", 0, k_solid_mg_smooth::main},
    {"solid_mg_residual.glsl", 0, k_solid_mg_residual::main},
    {"solid_mg_prolong.glsl", 0, k_solid_mg_prolong::main},
    {"solid_mg_direct.glsl", 0, k_solid_mg_direct::main},
    {"pressure_walls.glsl", 1, ks_pressure_walls::main},
    {"pressure_jacobi.glsl", 1, ks_pressure_jacobi::main},
    {"pressure_gradient.glsl", 1, ks_pressure_gradient::main},
    {"solid_clear.glsl", 1, ks_solid_clear::main},
    {"transport_face.glsl", 1, ks_transport_face::main},
    {"transport_scalar.glsl", 1, ks_transport_scalar::main},
    {"closed_advect_scalar.glsl", 1, ks_closed_advect_scalar::main},
    {"emitting_advect_velocity.glsl", 1, ks_emitting_advect_velocity::main},
    {"multi_advect_velocity.glsl", 1, ks_multi_advect_velocity::main},
    {"multi_advect_scalar.glsl", 1, ks_multi_advect_scalar::main},
    {"curl.glsl", 0, k_curl::main},
    {"confinement.glsl", 0, k_confinement::main},
    {"combustion_burn.glsl", 0, k_combustion_burn::main},
    {"combustion_apply.glsl", 0, k_combustion_apply::main},
    {"moving_mask.glsl", 0, k_moving_mask::main},
    {"moving_wall.glsl", 0, k_moving_wall::main},
    {"moving_remap_scalar.glsl", 0, k_moving_remap_scalar::main},
    {"moving_remap_face.glsl", 0, k_moving_remap_face::main},
    {"pressure_walls.glsl", 2, km_pressure_walls::main},
    {"pressure_gradient.glsl", 2, km_pressure_gradient::main},
    {"pressure_divergence.glsl", 1, km_pressure_divergence::main},
};

struct FloatSlot {
    const char* name;
    float* data;
    int n;
};
const FloatSlot kFloats[] = {
    {"domainExtent", domainExtent.v, 3}, {"cellCount", cellCount.v, 3}, {"faceOffset", faceOffset.v, 3},
    {"axisMask", axisMask.v, 3}, {"invCell", invCell.v, 3}, {"sourceCenter", sourceCenter.v, 3},
    {"sourceStart", sourceStart.v, 3}, {"baseVelocity", baseVelocity.v, 3},
    {"emissionVelocity", emissionVelocity.v, 3}, {"row0", row0.v, 4}, {"row1", row1.v, 4}, {"row2", row2.v, 4},
    {"dt", &dt, 1}, {"relaxation", &relaxation, 1}, {"componentAxis", &componentAxis, 1}, {"factor", &factor, 1},
    {"sourceRadius", &sourceRadius, 1}, {"sourceProfile", &sourceProfile, 1}, {"sourceRate", &sourceRate, 1},
    {"dissipation", &dissipation, 1}, {"targetDensity", &targetDensity, 1},
    {"correctedTransport", &correctedTransport, 1}, {"correctedVelocity", &correctedVelocity, 1},
    {"emissionCoupling", &emissionCoupling, 1}, {"sourceCount", &sourceCount, 1},
    {"scalarChannel", &scalarChannel, 1}, {"thermalLift", &thermalLift, 1}, {"densityWeight", &densityWeight, 1},
    {"seedTemperature", &seedTemperature, 1}, {"angularSpeed", &angularSpeed, 1}, {"shapeKind", &shapeKind, 1},
    {"curlStrength", &curlStrength, 1}, {"forceLimit", &forceLimit, 1},
    {"ignitionTemperature", &ignitionTemperature, 1}, {"burnRate", &burnRate, 1}, {"yieldValue", &yieldValue, 1},
    {"owner", &owner, 1},
};

struct SamplerSlot {
    const char* name;
    sampler3D* s;
};
const SamplerSlot kSamplers[] = {
    {"inputField", &inputField}, {"velocityU", &velocityU}, {"velocityV", &velocityV}, {"velocityW", &velocityW},
    {"divergenceField", &divergenceField}, {"pressureField", &pressureField}, {"coarseField", &coarseField},
    {"inverseField", &inverseField}, {"edgeField", &edgeField}, {"solidField", &solidField},
    {"densityField", &densityField}, {"temperatureField", &temperatureField}, {"predictorField", &predictorField},
    {"reverseField", &reverseField}, {"originalFaceField", &originalFaceField}, {"facePredictor", &facePredictor},
    {"sourceTable", &sourceTable}, {"curlField", &curlField}, {"burnField", &burnField},
    {"boundaryField", &boundaryField}, {"oldSolidField", &oldSolidField}, {"wallTable", &wallTable},
};

long long g_total_out_of_range = 0;
}  // namespace

extern "C" {

int glsl_ref_kernel(const char* file, int collisions) {
    for (size_t k = 0; k < sizeof kKernels / sizeof kKernels[0]; ++k)
        if (!std::strcmp(kKernels[k].file, file) && kKernels[k].collisions == collisions) return (int)k;
    return -1;
}

int glsl_ref_set_uniform(const char* name, const float* values, int n) {
    for (const FloatSlot& s : kFloats)
        if (!std::strcmp(s.name, name)) {
            if (n != s.n) return -2;
            for (int i = 0; i < n; ++i) s.data[i] = values[i];
            return 0;
        }
    return -1;
}

int glsl_ref_bind_sampler(const char* name, const float* data, int sx, int sy, int sz, int channels) {
    for (const SamplerSlot& s : kSamplers)
        if (!std::strcmp(s.name, name)) {
            *s.s = sampler3D{data, sx, sy, sz, channels};
            return 0;
        }
    return -1;
}

void glsl_ref_clear_bindings(void) {
    for (const SamplerSlot& s : kSamplers) *s.s = sampler3D{};
    outputField = image3D{};
}

void glsl_ref_bind_output(float* data, int sx, int sy, int sz, int channels) {
    outputField = image3D{data, sx, sy, sz, channels};
}

// Runs main() for every invocation of a gx x gy x gz grid (gridSize uniform).
int glsl_ref_dispatch(int kernel, int gx, int gy, int gz) {
    if (kernel < 0 || kernel >= (int)(sizeof kKernels / sizeof kKernels[0])) return -1;
    gridSize = ivec3(gx, gy, gz);
    void (*fn)() = kKernels[kernel].main;
    long long oor = 0;
#pragma omp parallel for schedule(static) reduction(+ : oor)
    for (int z = 0; z < gz; ++z) {
        g_out_of_range = 0;
        for (int y = 0; y < gy; ++y)
            for (int x = 0; x < gx; ++x) {
                gl_GlobalInvocationID.xyz = ivec3(x, y, z);
                fn();
            }
        oor += g_out_of_range;
    }
    g_total_out_of_range += oor;
    return 0;
}

long long glsl_ref_out_of_range(void) { return g_total_out_of_range; }

int glsl_ref_kernel_count(void) { return (int)(sizeof kKernels / sizeof kKernels[0]); }

}  // extern "C"
