"""Staggered (MAC) face velocity storage and plain self-advection (P0.3).

Drop-in for FluxFX ``fluxfx/backend/mac.py:12-81``. U, V, W are CUDA tensors
of shapes (nz, ny, nx+1), (nz, ny+1, nx), (nz+1, ny, nx).
"""
from .. import _native as N
from ..physics.config import validate_dt
from .dense import DenseAdvection, SEED_CONSTANTS
from .device import ptr

FACE_OFFSETS = ((0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0))
AXIS_MASKS = ((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0))
VELOCITY_NAMES = ("velocityU", "velocityV", "velocityW")
FACE_CONSTANTS = (("VEC3", "domainExtent"), ("VEC3", "cellCount"),
                  ("VEC3", "faceOffset"), ("VEC3", "axisMask"))

__all__ = ['DenseMACAdvection', 'FACE_OFFSETS', 'AXIS_MASKS', 'VELOCITY_NAMES', 'FACE_CONSTANTS', 'SEED_CONSTANTS']


class DenseMACAdvection(DenseAdvection):
    def __init__(self, grid=None, settings=None, device=None):
        self._velocity = self._velocity_back = None
        super().__init__(grid, settings, device)
        self._velocity = [self._texture(shape) for shape in self.grid.face_shapes]
        self._velocity_back = [self._texture(shape) for shape in self.grid.face_shapes]
        self.reset()

    @property
    def allocated_bytes(self):
        return self.grid.mac_bytes

    def _face_uniforms(self, axis):
        """The face-pass uniforms of the reference (``backend/mac.py:33-35``)."""
        return {"domainExtent": self.grid.extent, "cellCount": self.grid.shape,
                "faceOffset": FACE_OFFSETS[axis], "axisMask": AXIS_MASKS[axis]}

    def _face_ptrs(self, faces):
        return [ptr(f) for f in faces]

    def reset(self, seed=True):
        super().reset(seed)
        if self._velocity is None:
            return
        s = self.settings
        self._call('ffx_seed_faces', self._gp, self._storage, N.f3(*s.velocity), s.angular_speed,
                   *self._face_ptrs(self._velocity), self.device.s)
        for f in self._velocity_back:
            f.zero_()

    def upload_velocity(self, components):
        """Signed face-centred data for numerical tests/debugging only."""
        if len(components) != 3:
            raise ValueError("MAC velocity requires U, V, W components")
        # Build all three before replacing, so invalid data cannot half-modify state.
        fields = [self._texture(shape, values, nonnegative=False)
                  for shape, values in zip(self.grid.face_shapes, components)]
        self._velocity = fields

    def read_velocity(self):
        return tuple(self.device.read(f, s) for f, s in zip(self._velocity, self.grid.face_shapes))

    def step(self, dt=1.0 / 30.0):
        validate_dt(dt)
        s = self.settings
        # All components gather from the same old velocity before any swap.
        self._call('ffx_mac_advect_velocity', self._gp, self._storage, *self._face_ptrs(self._velocity), dt,
                   *self._face_ptrs(self._velocity_back), self.device.s)
        self._call('ffx_mac_advect_density', self._gp, self._storage, *self._face_ptrs(self._velocity_back),
                   ptr(self._front), dt, N.f3(*s.source_center), s.source_radius, s.source_rate, s.dissipation,
                   ptr(self._back), self.device.s)
        # Commit the complete step only after every pass was enqueued.
        self._velocity, self._velocity_back = self._velocity_back, self._velocity
        self._front, self._back = self._back, self._front
        self.time += dt
        self.steps += 1

    def close(self):
        self._velocity = self._velocity_back = None
        super().close()
