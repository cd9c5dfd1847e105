"""Single-pass dispatch by reference shader name (``CudaDevice.dispatch``).

Scripts and tests written against FluxFX drive individual passes through
``device.dispatch(kernel, output, shape, uniforms, input_field, sources)``
(e.g. ``scripts/multigrid_operators_validate.py``, ``detail_validate.py``,
``motion_detail_validate.py``). This maps those passes onto the native entry
points with the reference's uniform and sampler names: the multigrid
operators, the pressure passes (walls, divergence, gradient, Jacobi, scale,
direct solve), the transport passes (face and scalar predictors, the emitting
velocity and closed scalar passes in their single-emitter and table forms),
buoyancy and the benchmark fence. Face passes run one face grid
(``componentAxis`` or ``axisMask``): the native passes take all three grids
at once, so the other two run on scratch buffers and are discarded; each
grid's result depends only on its own inputs, so the requested grid's values
are those of the fused step. Collider variants follow the device's mask when
the device is a collider device (``SolidDevice``).
"""
import ctypes as C
from math import prod

import torch

from .. import _native as N
from .device import ptr, solids_struct


def _f32(t):
    if t.dtype != torch.float32:
        raise ValueError("single-pass dispatch works on float32 fields")
    return ptr(t)


def _storage(t):
    if t.dtype == torch.float32:
        return N.FFX_F32
    if t.dtype == torch.bfloat16:
        return N.FFX_BF16
    raise ValueError("dispatch fields must be float32 or bfloat16")


def _grid(uniforms, shape):
    """FfxGrid of the pass's cells (``cellCount`` or the dispatch shape of a
    cell pass) and ``domainExtent``; ``invCell`` as given."""
    cells = tuple(int(round(c)) for c in uniforms.get('cellCount', shape))
    g = N.grid_struct(cells, tuple(float(e) for e in uniforms.get('domainExtent', (1.0, 1.0, 1.0))))
    if 'invCell' in uniforms:
        g.ix, g.iy, g.iz = (float(v) for v in uniforms['invCell'])
    return g


def _axis(uniforms):
    if 'componentAxis' in uniforms:
        return int(round(float(uniforms['componentAxis'])))
    mask = tuple(float(v) for v in uniforms.get('axisMask', (1.0, 0.0, 0.0)))
    return mask.index(1.0)


def _face_set(dev, g, axis, field, like):
    """Three face grids: ``field`` on ``axis``, zero scratch on the others."""
    n = (g.nx, g.ny, g.nz)
    out = []
    for a in range(3):
        if a == axis:
            out.append(field)
        else:
            shape = tuple(n[k] + (k == a) for k in range(3))
            with dev.ordered():
                out.append(torch.zeros(shape[::-1], dtype=like.dtype, device=like.device))
    return out


def _velocity(sources):
    return [sources[k] for k in ('velocityU', 'velocityV', 'velocityW')]


def _single_source(uniforms):
    src = N.FfxSources()
    src.count = -1
    center = uniforms.get('sourceCenter', (0.5, 0.5, 0.5))
    src.single_solid_profile = int(float(uniforms.get('sourceProfile', 0.0)) >= 0.5)
    src.single_center = N.f3(*center)
    src.single_start = N.f3(*uniforms.get('sourceStart', center))
    src.single_radius = float(uniforms.get('sourceRadius', 0.0))
    src.single_jet = N.f3(*uniforms.get('emissionVelocity', (0.0, 0.0, 0.0)))
    src.single_coupling = float(uniforms.get('emissionCoupling', 0.0))
    return src


def _table_source(dev, uniforms, sources):
    """The 8-row emitter table (16 floats a row, ``physics/emission.py``)
    from the ``sourceTable`` field, copied into the launch parameters."""
    src = N.FfxSources()
    src.count = int(round(float(uniforms['sourceCount'])))
    values = dev.fetch(sources['sourceTable'].reshape(-1).to(torch.float32))
    for i, v in enumerate(values[:128].tolist()):
        src.table[i] = v
    return src


def run(dev, shader, output, shape, uniforms, input_field, sources):
    name = shader.name
    s = dev.s
    n3 = N.n3(*shape)
    if name in _PASSES:
        return _PASSES[name](dev, output, shape, uniforms, input_field, sources)
    if name == 'mg_residual.glsl':
        dev.call('ffx_mg_residual', n3, N.f3(*uniforms['invCell']), _f32(input_field),
                 _f32(sources['divergenceField']), float(uniforms['dt']), _f32(output), s)
    elif name == 'mg_restrict.glsl':
        fine = tuple(2 * n for n in shape)
        dev.call('ffx_mg_restrict', N.n3(*fine), _f32(input_field), _f32(output), s)
    elif name == 'mg_prolong.glsl':
        dev.call('ffx_mg_prolong', n3, _f32(input_field), _f32(sources['coarseField']), _f32(output), s)
    elif name == 'pressure_jacobi.glsl':
        mask = getattr(dev, 'mask', None)
        dev.call('ffx_jacobi', n3, N.f3(*uniforms['invCell']), ptr(mask), _f32(input_field),
                 _f32(sources['divergenceField']), float(uniforms['dt']), float(uniforms['relaxation']),
                 _f32(output), s)
    elif name == 'pressure_scale.glsl':
        dev.call('ffx_scale', prod(shape), _f32(input_field), float(uniforms['factor']), _f32(output), s)
    elif name in ('coarse_pressure.glsl', 'solid_mg_direct.glsl'):
        inverse = sources['inverseField']
        if inverse.dtype != torch.float64:
            inverse = inverse.to(torch.float64)
        dt = float(uniforms.get('dt', 1.0))
        dev.call('ffx_direct_solve', prod(shape), ptr(inverse), _f32(input_field), dt, _f32(output), s)
    elif name == 'max_reduce.glsl':
        dev.call('ffx_max_abs', input_field.numel(), N.FFX_F32, _f32(input_field), _f32(output.view(-1)[0:1]), s)
    else:
        raise NotImplementedError(f"{name} runs through the solver objects, not single-pass dispatch")


# ---------------------------------------------------------------- face and cell passes
def _walls(dev, output, shape, uniforms, field, sources):
    g = _grid(uniforms, tuple(n - (k == _axis(uniforms)) for k, n in enumerate(shape)))
    a = _axis(uniforms)
    ins = _face_set(dev, g, a, field, field)
    outs = _face_set(dev, g, a, output, field)
    dev.call('ffx_walls', C.byref(g), C.byref(solids_struct(dev)), _storage(field), *[ptr(f) for f in ins],
             *[ptr(f) for f in outs], dev.s)


def _divergence(dev, output, shape, uniforms, field, sources):
    g = _grid(uniforms, shape)
    vel = _velocity(sources)
    dev.call('ffx_divergence', C.byref(g), C.byref(solids_struct(dev)), _storage(vel[0]), *[ptr(f) for f in vel],
             _f32(output), dev.s)


def _gradient(dev, output, shape, uniforms, field, sources):
    a = _axis(uniforms)
    g = _grid(uniforms, tuple(n - (k == a) for k, n in enumerate(shape)))
    ins = _face_set(dev, g, a, field, field)
    outs = _face_set(dev, g, a, output, field)
    dev.call('ffx_gradient', C.byref(g), C.byref(solids_struct(dev)), _storage(field), *[ptr(f) for f in ins],
             _f32(sources['pressureField']), float(uniforms.get('dt', 1.0)), *[ptr(f) for f in outs], None, None,
             dev.s)


def _transport_face(dev, output, shape, uniforms, field, sources):
    a = _axis(uniforms)
    g = _grid(uniforms, shape)
    vel = _velocity(sources)
    if field is not vel[a]:
        raise ValueError('transport_face: inputField must be the velocity component of its axis')
    outs = _face_set(dev, g, a, output, field)
    dev.call('ffx_face_predictor', C.byref(g), C.byref(solids_struct(dev)), _storage(field), *[ptr(f) for f in vel],
             float(uniforms['dt']), *[ptr(f) for f in outs], dev.s)


def _transport_scalar(dev, output, shape, uniforms, field, sources):
    g = _grid(uniforms, shape)
    vel = _velocity(sources)
    ins = (C.c_void_p * 1)(field.data_ptr())
    outs = (C.c_void_p * 1)(output.data_ptr())
    dev.call('ffx_scalar_transport', C.byref(g), C.byref(solids_struct(dev)), _storage(field), *[ptr(f) for f in vel],
             float(uniforms['dt']), 1, ins, outs, dev.s)


def _velocity_pass(dev, output, shape, uniforms, field, sources, src):
    a = _axis(uniforms)
    g = _grid(uniforms, shape)
    vel = _velocity(sources)
    if sources.get('originalFaceField', vel[a]) is not vel[a]:
        raise ValueError('the original face field must be the velocity component of its axis')
    corrected = float(uniforms.get('correctedVelocity', 0.0)) >= 0.5
    pred = [sources['facePredictor'] if k == a else vel[k] for k in range(3)]
    outs = _face_set(dev, g, a, output, vel[a])
    dev.call('ffx_advect_velocity', C.byref(g), C.byref(solids_struct(dev)), _storage(vel[a]),
             *[ptr(f) for f in vel], *[ptr(f) for f in pred], float(uniforms['dt']), int(corrected), 0.5,
             C.byref(src), None, None, 0.0, 0.0, 0, *[ptr(f) for f in outs], dev.s)


def _emitting_velocity(dev, output, shape, uniforms, field, sources):
    _velocity_pass(dev, output, shape, uniforms, field, sources, _single_source(uniforms))


def _multi_velocity(dev, output, shape, uniforms, field, sources):
    _velocity_pass(dev, output, shape, uniforms, field, sources, _table_source(dev, uniforms, sources))


def _scalar_pass(dev, output, shape, uniforms, field, sources, src, rate, target, channel):
    g = _grid(uniforms, shape)
    vel = _velocity(sources)
    corrected = float(uniforms.get('correctedTransport', 0.0)) >= 0.5
    ch = N.FfxScalarChannel(ptr(field), ptr(sources.get('predictorField', field)),
                            ptr(sources.get('reverseField', field)), ptr(output), rate,
                            float(uniforms.get('dissipation', 0.0)), target, channel, 0)
    dev.call('ffx_advect_scalars', C.byref(g), C.byref(solids_struct(dev)), _storage(field), *[ptr(f) for f in vel],
             float(uniforms['dt']), int(corrected), C.byref(src), 1, C.byref(ch), None, dev.s)


def _closed_scalar(dev, output, shape, uniforms, field, sources):
    _scalar_pass(dev, output, shape, uniforms, field, sources, _single_source(uniforms),
                 float(uniforms.get('sourceRate', 0.0)), float(uniforms.get('targetDensity', -1.0)), 0)


def _multi_scalar(dev, output, shape, uniforms, field, sources):
    _scalar_pass(dev, output, shape, uniforms, field, sources, _table_source(dev, uniforms, sources), 0.0, -1.0,
                 int(round(float(uniforms['scalarChannel']))))


def _buoyancy(dev, output, shape, uniforms, field, sources):
    g = _grid(uniforms, (shape[0], shape[1], shape[2] - 1))
    dev.call('ffx_buoyancy', C.byref(g), _storage(field), ptr(field), ptr(sources['densityField']),
             ptr(sources['temperatureField']), float(uniforms['dt']), float(uniforms['thermalLift']),
             float(uniforms['densityWeight']), ptr(output), dev.s)


_FENCE_FIELDS = ('densityField', 'temperatureField', 'velocityU', 'velocityV', 'velocityW', 'divergenceField',
                 'fuelField', 'flameField')


def _fence(dev, output, shape, uniforms, field, sources):
    """benchmark_fence.glsl: every output texel holds the sum of the first
    texel of each bound field (a completion dependency on all of them)."""
    with dev.ordered():
        total = torch.zeros((), dtype=torch.float32, device=output.device)
        for name in _FENCE_FIELDS:
            if sources.get(name) is not None:
                total = total + sources[name].reshape(-1)[0].to(torch.float32)
        output.fill_(total)


_PASSES = {
    'pressure_walls.glsl': _walls,
    'pressure_divergence.glsl': _divergence,
    'pressure_gradient.glsl': _gradient,
    'transport_face.glsl': _transport_face,
    'transport_scalar.glsl': _transport_scalar,
    'emitting_advect_velocity.glsl': _emitting_velocity,
    'multi_advect_velocity.glsl': _multi_velocity,
    'closed_advect_scalar.glsl': _closed_scalar,
    'multi_advect_scalar.glsl': _multi_scalar,
    'buoyancy.glsl': _buoyancy,
    'benchmark_fence.glsl': _fence,
}
