"""Interactive (moving) colliders: mask refresh, rigid wall velocities, remap.

Drop-in for FluxFX ``fluxfx/backend/moving_collision.py:7-87``
(``MovingSolidDevice``). The collider mask holds owner ids (1-based collider
index, first collider wins, 0 = fluid; ``moving_mask.glsl``), rebuilt in place
by ``update`` together with the dilated mask and the wall velocity of every
face next to a solid cell (``moving_wall.glsl``). The pressure passes read
those wall velocities through the solver's FfxSolids (the
FLUXFX_MOVING_COLLIDERS variants of ``pressure_walls.glsl`` and
``pressure_gradient.glsl``). ``remap`` empties cells covered before or after
the move and gives covered faces the wall velocity (``moving_remap_*.glsl``),
in place.
"""
import ctypes as C
from math import prod

import torch

from .. import _native as N
from ..physics.collider_motion import collider_rows12, validate_motion, velocity_rows
from .collision import SolidDevice
from .device import ptr


class MovingSolidDevice(SolidDevice):
    def __init__(self, grid, colliders, device=None):
        validate_motion(colliders, colliders)
        if len(colliders) > N.MOVING_MAX:
            raise ValueError(f'Use at most {N.MOVING_MAX} moving colliders')
        super().__init__(grid, colliders, device)
        dev = self.base.device
        nx, ny, nz = grid.shape
        self.previous_mask = torch.zeros((nz, ny, nx), dtype=torch.uint8, device=dev)
        self.walls = [torch.zeros((s[2], s[1], s[0]), dtype=torch.float32, device=dev) for s in grid.face_shapes]
        self._g = N.grid_struct(grid.shape, grid.extent)
        self._owner_mask(colliders)       # the FP32 owner test of moving_mask.glsl from the start

    @property
    def allocated_bytes(self):
        return 4 * prod(self.grid.shape) + 4 * sum(prod(s) for s in self.grid.face_shapes)

    def _owner_mask(self, colliders):
        rows, box = collider_rows12(colliders)
        # host arrays: the library copies them into the launch parameters
        rows_h = (C.c_float * len(rows))(*rows)
        box_h = (C.c_int32 * len(box))(*box)
        self.base.call('ffx_moving_mask', C.byref(self._g), len(colliders), rows_h, box_h, ptr(self.mask),
                       self.base.s)
        self.base.call('ffx_halo_clearance', C.byref(self._g), ptr(self.mask), ptr(self.halo), ptr(self.clear),
                       self.base.s)

    def update(self, colliders, dt):
        """New poses: owner mask, dilated mask and wall velocities, in place."""
        validate_motion(self.colliders, colliders)
        self.previous_mask.copy_(self.mask)
        self._owner_mask(colliders)
        table = [v for old, new in zip(self.colliders, colliders) for row in velocity_rows(old, new, dt) for v in row]
        table_h = (C.c_float * len(table))(*table)
        self.base.call('ffx_moving_walls', C.byref(self._g), ptr(self.mask), len(colliders), table_h,
                       *[ptr(w) for w in self.walls], self.base.s)
        self.colliders = tuple(colliders)

    def remap(self, solver):
        storage = N.FFX_F32 if solver._front.dtype == torch.float32 else N.FFX_BF16
        fuel = solver.combustion.fuel if solver.combustion is not None else None
        self.base.call('ffx_moving_remap', C.byref(self._g), storage, ptr(self.mask), ptr(self.previous_mask),
                       ptr(solver._front), ptr(solver._temperature), ptr(fuel), *[ptr(v) for v in solver._velocity],
                       *[ptr(w) for w in self.walls], self.base.s)
        if solver.combustion is not None:
            solver.combustion.flame.zero_()

    def close(self):
        self.previous_mask = None
        self.walls = None
        super().close()
