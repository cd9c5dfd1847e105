"""Fuel storage and the combustion pass.

Drop-in for FluxFX ``fluxfx/backend/combustion.py:4-33`` (``CombustionPasses``):
``fuel`` is transported with the other scalars (third channel, table column
``fuel_rate`` or ``settings.fuel_source_rate``); after transport one
``ffx_combustion`` launch burns fuel above the ignition temperature and feeds
smoke and heat (``combustion_burn.glsl`` + ``combustion_apply.glsl``), in
place. ``flame`` holds the consumed fuel per second of the last step.
"""
import ctypes as C
from math import prod

import torch

from .. import _native as N
from .device import ptr


class CombustionPasses:
    def __init__(self, grid, device, dtype=torch.float32):
        self.grid, self.device = grid, device
        self._g = N.grid_struct(grid.shape, grid.extent)
        self._storage = N.FFX_F32 if dtype == torch.float32 else N.FFX_BF16
        self.fuel = device.texture(grid.shape, dtype=dtype)
        self.spare = device.texture(grid.shape, dtype=dtype)
        self.flame = device.texture(grid.shape)

    @property
    def allocated_bytes(self):
        return (2 * self.fuel.element_size() + 4) * prod(self.grid.shape)

    def reset(self):
        for field in (self.fuel, self.spare, self.flame):
            field.zero_()

    def react(self, solver, dt):
        s = solver.settings
        self.device.call('ffx_combustion', C.byref(self._g), self._storage, ptr(self.fuel), ptr(solver.temperature),
                         ptr(solver.density), dt, s.ignition_temperature, s.burn_rate, s.smoke_yield, s.heat_yield,
                         ptr(self.flame), ptr(self.fuel), ptr(solver.density), ptr(solver.temperature),
                         self.device.s)

    def close(self):
        self.fuel = self.spare = self.flame = None
