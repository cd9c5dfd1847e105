"""Single-pass dispatch by reference shader name (``CudaDevice.dispatch``).

Scripts and tests written against FluxFX drive individual passes through
``device.dispatch(kernel, output, shape, uniforms, input_field, sources)``
(e.g. ``scripts/multigrid_operators_validate.py``). This maps the passes of
the projection and multigrid path onto the native entry points with the
reference's uniform and sampler names. Face passes that the native library
runs for all three axes at once (walls, gradient, transport) are driven
through the solver objects instead.
"""
import ctypes as C
from math import prod

import torch

from .. import _native as N
from .device import ptr


def _f32(t):
    if t.dtype != torch.float32:
        raise ValueError("single-pass dispatch works on float32 fields")
    return ptr(t)


def run(dev, shader, output, shape, uniforms, input_field, sources):
    name = shader.name
    s = dev.s
    n3 = N.n3(*shape)
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
