"""Temperature transport with explicit vertical buoyancy (P0.4).

Drop-in for FluxFX ``fluxfx/backend/thermal.py:9-80``.
"""
from math import prod

from .. import _native as N
from ..physics.config import validate_dt
from ..physics.thermal import ThermalSettings
from .device import ptr
from .mac import DenseMACAdvection


class DenseThermalAdvection(DenseMACAdvection):
    def __init__(self, grid=None, settings=None, device=None):
        self._temperature = self._temperature_back = self._buoyancy_scratch = None
        super().__init__(grid, settings or ThermalSettings(), device)
        self._temperature = self._texture(self.grid.shape)
        self._temperature_back = self._texture(self.grid.shape)
        self._buoyancy_scratch = self._texture(self.grid.face_shapes[2])
        self.reset()

    @property
    def temperature(self):
        return self._temperature

    @property
    def allocated_bytes(self):
        return self.grid.mac_bytes + 8 * prod(self.grid.shape) + 4 * prod(self.grid.face_shapes[2])

    def reset(self, seed=True):
        super().reset(seed)
        if self._temperature is None:
            return
        for t in (self._temperature, self._temperature_back, self._buoyancy_scratch):
            t.zero_()
        if seed:
            s = self.settings
            self._call('ffx_seed_scalar', self._gp, self._storage, N.f3(*s.source_center), s.source_radius,
                       s.initial_temperature, ptr(self._temperature), self.device.s)

    def upload_temperature(self, values):
        self._temperature = self._texture(self.grid.shape, values, nonnegative=False)

    def read_temperature(self):
        return self.device.read(self._temperature, self.grid.shape)

    def step(self, dt=1.0 / 30.0):
        validate_dt(dt)
        s = self.settings
        vel = self._face_ptrs(self._velocity)
        back = self._face_ptrs(self._velocity_back)
        self._call('ffx_mac_advect_velocity', self._gp, self._storage, *vel, dt, *back, self.device.s)
        # The previous scalars drive buoyancy; newly injected heat acts next step.
        self._call('ffx_buoyancy', self._gp, self._storage, back[2], ptr(self._front), ptr(self._temperature), dt,
                   s.thermal_lift, s.density_weight, ptr(self._buoyancy_scratch), self.device.s)
        nxt = [self._velocity_back[0], self._velocity_back[1], self._buoyancy_scratch]
        nv = self._face_ptrs(nxt)
        self._call('ffx_mac_advect_density', self._gp, self._storage, *nv, ptr(self._front), dt,
                   N.f3(*s.source_center), s.source_radius, s.source_rate, s.dissipation, ptr(self._back),
                   self.device.s)
        # The same scalar pass transports the signed temperature excess.
        self._call('ffx_mac_advect_density', self._gp, self._storage, *nv, ptr(self._temperature), dt,
                   N.f3(*s.source_center), s.source_radius, s.heat_source_rate, s.cooling,
                   ptr(self._temperature_back), self.device.s)
        spare_w = self._velocity_back[2]
        self._velocity_back, self._velocity = self._velocity, nxt
        self._buoyancy_scratch = spare_w
        self._front, self._back = self._back, self._front
        self._temperature, self._temperature_back = self._temperature_back, self._temperature
        self.time += dt
        self.steps += 1

    def close(self):
        self._temperature = self._temperature_back = self._buoyancy_scratch = None
        super().close()
