"""Dense ping-pong density transport in a prescribed flow (P0.2).

Drop-in for FluxFX ``fluxfx/backend/dense.py:12-65`` (same constructor, methods
and attributes). Fields are CUDA tensors; the pass is ``ffx_advect_open``.
"""
import torch

from .. import _native as N
from ..physics.config import AdvectionSettings, GridSpec, validate_dt
from .device import CudaDevice, ptr

SEED_CONSTANTS = (("VEC3", "domainExtent"), ("VEC3", "sourceCenter"), ("FLOAT", "sourceRadius"))
ADVECTION_CONSTANTS = SEED_CONSTANTS + (
    ("VEC3", "baseVelocity"), ("FLOAT", "angularSpeed"), ("FLOAT", "dt"),
    ("FLOAT", "sourceRate"), ("FLOAT", "dissipation"),
)


class DenseAdvection:
    _field_dtype = torch.float32

    def __init__(self, grid=None, settings=None, device=None):
        self.grid = grid or GridSpec()
        self.settings = settings or AdvectionSettings()
        self.device = device or CudaDevice()
        self._g = N.grid_struct(self.grid.shape, self.grid.extent)
        self._storage = N.FFX_F32 if self._field_dtype == torch.float32 else N.FFX_BF16
        self._front = self._texture(self.grid.shape)
        self._back = self._texture(self.grid.shape)
        self.time = 0.0
        self.steps = 0
        self.reset()

    # ------------------------------------------------------------ helpers
    def _texture(self, shape, values=None, nonnegative=True):
        return self.device.texture(shape, values, nonnegative=nonnegative, dtype=self._field_dtype)

    def _call(self, name, *args):
        self.device.call(name, *args)

    @property
    def _gp(self):
        import ctypes
        return ctypes.byref(self._g)

    @property
    def density(self):
        return self._front

    def _source_uniforms(self):
        """The seed/source uniforms of the reference's passes (``backend/dense.py:29-31``),
        for scripts that drive single passes through ``device.dispatch``."""
        return {"domainExtent": self.grid.extent, "sourceCenter": self.settings.source_center,
                "sourceRadius": self.settings.source_radius}

    def reset(self, seed=True):
        self._front.zero_()
        self._back.zero_()
        if seed:
            s = self.settings
            self._call('ffx_seed_scalar', self._gp, self._storage, N.f3(*s.source_center), s.source_radius, 1.0,
                       ptr(self._front), self.device.s)
        self.time = 0.0
        self.steps = 0

    def upload(self, values):
        """Test/debug entry point, not part of the playback path."""
        self._front = self._texture(self.grid.shape, values)
        self._back.zero_()
        self.time = 0.0
        self.steps = 0

    def step(self, dt=1.0 / 30.0):
        validate_dt(dt)
        s = self.settings
        self._call('ffx_advect_open', self._gp, self._storage, ptr(self._front), dt, N.f3(*s.velocity),
                   s.angular_speed, N.f3(*s.source_center), s.source_radius, s.source_rate, s.dissipation,
                   ptr(self._back), self.device.s)
        self._front, self._back = self._back, self._front
        self.time += dt
        self.steps += 1

    def read_density(self):
        return self.device.read(self._front, self.grid.shape)

    def close(self):
        self._front = self._back = None
