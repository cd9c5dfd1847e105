"""Static voxel colliders: device raster, dilated halo mask, masked Jacobi projector.

Drop-in for FluxFX ``fluxfx/backend/collision.py:12-88``. ``SolidDevice`` wraps a
``CudaDevice``: every pass that the reference "decorates" with the solid mask
(``VARIANTS``) reads ``mask`` (uint8, 1 = solid) and ``halo`` (uint8, a solid or
out-of-domain cell in the 3x3x3 block) through the projector and solver, and
everything else is delegated unchanged.
"""
import ctypes as C
from math import prod

import torch

from .. import _native as N
from .device import CudaDevice, ptr
from .pressure import PressureProjector

VARIANTS = {'pressure_walls.glsl', 'pressure_jacobi.glsl', 'pressure_gradient.glsl',
            'closed_advect_scalar.glsl', 'multi_advect_scalar.glsl',
            'emitting_advect_velocity.glsl', 'multi_advect_velocity.glsl', 'solid_clear.glsl',
            'transport_scalar.glsl', 'transport_face.glsl'}


def collider_rows(colliders):
    """13 FP64 values per collider: three affine inverse rows and the shape code."""
    rows = []
    for c in colliders:
        if c.shape == 'MESH':
            raise ValueError('Mesh colliders need the Blender mesh SDF, which this build does not provide')
        rows.extend(float(v) for r in c.inverse_rows for v in r)
        rows.append(float(c.shape == 'BOX'))
    return rows


class SolidDevice:
    """Delegates ordinary passes; carries the static mask for the masked forms."""

    def __init__(self, grid, colliders, device=None):
        if not 1 <= len(colliders) <= 8:
            raise ValueError('Use one to eight static colliders')
        self.base = device or CudaDevice()
        self.grid = grid
        self.decorated = []
        self.mesh_sdf = None
        self.mesh_reports = []
        nx, ny, nz = grid.shape
        dev = self.base.device
        self.mask = torch.zeros((nz, ny, nx), dtype=torch.uint8, device=dev)
        self.halo = torch.zeros((nz, ny, nx), dtype=torch.uint8, device=dev)
        rows = torch.tensor(collider_rows(colliders), dtype=torch.float64).to(dev)
        g = N.grid_struct(grid.shape, grid.extent)
        self.base.call('ffx_raster_colliders', C.byref(g), (C.c_double * 3)(*grid.extent), len(colliders),
                       ptr(rows), ptr(self.mask), self.base.s)
        # the dilated mask and the cells with no collider or wall within three cells
        # (the transport passes skip their collider tests there), refreshed with the mask
        self.clear = torch.zeros((nz, ny, nx), dtype=torch.uint8, device=dev)
        self.base.call('ffx_halo_clearance', C.byref(g), ptr(self.mask), ptr(self.halo), ptr(self.clear),
                       self.base.s)
        self._rows = rows
        self.colliders = tuple(colliders)

    @property
    def calls(self):
        return self.base.calls

    @calls.setter
    def calls(self, value):
        self.base.calls = value

    def __getattr__(self, name):
        base = self.__dict__.get('base')
        if base is None:
            raise AttributeError(name)
        return getattr(base, name)

    @property
    def allocated_bytes(self):
        return 3 * prod(self.grid.shape)

    def kernel(self, filename, constants=(), sample_input=False, samplers=(), includes=(), output_format='R32F'):
        handle = self.base.kernel(filename, constants)
        if filename in VARIANTS:
            self.decorated.append(handle)
        return handle

    def dispatch(self, shader, output, shape, uniforms=None, input_field=None, sources=None):
        # through this device, so the passes read its mask (the collider variants)
        CudaDevice.dispatch(self, shader, output, shape, uniforms, input_field, sources)

    def clear_solid(self, source, target):
        """target = source outside solids, 0 inside (``solid_clear.glsl``)."""
        code = N.FFX_F32 if source.dtype == torch.float32 else N.FFX_BF16
        g = N.grid_struct(self.grid.shape, self.grid.extent)
        self.base.call('ffx_solid_clear', C.byref(g), code, ptr(self.mask), ptr(source), ptr(target), self.base.s)

    def close(self):
        self.mask = self.halo = self.clear = None
        self.decorated = []
        self.mesh_sdf = None
        self.mesh_reports = []


class SolidPressureProjector(PressureProjector):
    """Masked Jacobi projection; the pressure starts from zero every step."""

    @property
    def uses_impulse(self):
        return True

    def solve_pressure(self, dt, previous_dt):
        # A short masked Jacobi solve cannot reliably remove a stale guess when
        # the new divergence is tiny: start from zero for stable damping.
        self.pressure.zero_()
        super().solve_pressure(dt, previous_dt)

    def metrics(self):
        moving = self.settings.moving_colliders
        return super().metrics() | {
            'solver': 'MOVING_JACOBI' if moving else 'SOLID_JACOBI',
            'boundary': 'moving_voxel_free_slip' if moving else 'static_voxel_free_slip', 'warm_start': False}
