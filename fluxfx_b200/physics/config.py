"""Grid and advection descriptors (SI units: metres, seconds).

Behaviour follows FluxFX ``fluxfx/physics/config.py:6-62``: the same fields,
defaults and validation messages. One extension: ``GridSpec.axis_limit``
lifts the reference's 128-cells-per-axis cap (``config.py:12``) for callers
that opt in (256^3 and 192x192x320 domains fit easily in HBM).
"""
from dataclasses import dataclass
from math import ceil, isfinite, prod

REFERENCE_AXIS_LIMIT = 128
HARD_AXIS_LIMIT = 2048


def _finite(values):
    return all(isfinite(v) for v in values)


@dataclass(frozen=True)
class GridSpec:
    """Cell-centred grid: ``shape`` = (nx, ny, nz) cells over ``extent`` metres.

    Field storage is x-fast (index ``x + nx*(y + ny*z)``), i.e. a torch tensor of
    shape (nz, ny, nx). Face grids add one sample along their own axis.
    """
    shape: tuple = (64, 64, 64)
    extent: tuple = (1.0, 1.0, 1.0)
    axis_limit: int = REFERENCE_AXIS_LIMIT

    def __post_init__(self):
        if type(self.axis_limit) is not int or not REFERENCE_AXIS_LIMIT <= self.axis_limit <= HARD_AXIS_LIMIT:
            raise ValueError(f"axis_limit must be an integer in [{REFERENCE_AXIS_LIMIT}, {HARD_AXIS_LIMIT}]")
        shape_ok = len(self.shape) == 3 and all(type(n) is int and 2 <= n <= self.axis_limit for n in self.shape)
        if not shape_ok:
            if self.axis_limit == REFERENCE_AXIS_LIMIT:
                raise ValueError("P0 grid dimensions must be integers in [2, 128]")
            raise ValueError(f"Grid dimensions must be integers in [2, {self.axis_limit}]")
        if len(self.extent) != 3 or not all(isfinite(x) and x > 0 for x in self.extent):
            raise ValueError("Domain extents must be finite and positive")

    @property
    def cells(self):
        return prod(self.shape)

    @property
    def cell_size(self):
        return tuple(e / n for e, n in zip(self.extent, self.shape))

    @property
    def face_shapes(self):
        nx, ny, nz = self.shape
        return ((nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1))

    @property
    def density_bytes(self):
        # Two FP32 scalar fields (front/back), as the reference accounts it.
        return 8 * prod(self.shape)

    @property
    def mac_bytes(self):
        return self.density_bytes + 8 * sum(prod(s) for s in self.face_shapes)


@dataclass(frozen=True)
class AdvectionSettings:
    velocity: tuple = (0.0, 0.0, 0.25)
    angular_speed: float = 0.8
    source_center: tuple = (0.5, 0.5, 0.16)
    source_radius: float = 0.12
    source_rate: float = 2.0
    dissipation: float = 0.1

    def __post_init__(self):
        if len(self.velocity) != 3 or len(self.source_center) != 3:
            raise ValueError("Velocity and source center must have three components")
        if not _finite((*self.velocity, self.angular_speed, *self.source_center,
                        self.source_radius, self.source_rate, self.dissipation)):
            raise ValueError("Simulation parameters must be finite")
        if self.source_radius <= 0 or self.source_rate < 0 or self.dissipation < 0:
            raise ValueError("Radius must be positive; source rate and dissipation nonnegative")


def workgroups(shape, local_size=(4, 4, 4)):
    """Ceil-divided launch extents (kept for API parity with the reference)."""
    if len(shape) != 3 or len(local_size) != 3 or min(*shape, *local_size) <= 0:
        raise ValueError("Dispatch requires three positive dimensions")
    return tuple(ceil(n / b) for n, b in zip(shape, local_size))


def validate_dt(dt):
    if not (isfinite(dt) and 0 < dt <= 0.1):
        raise ValueError("P0 timestep must be finite and in (0, 0.1] seconds")
