"""Emitter descriptors and the 8-source table layout.

Follows FluxFX ``fluxfx/physics/emission.py:6-58``. The table is the format the
device kernels read: 16 floats per source, four rows of four:

    row 0: center.x, center.y, center.z, radius
    row 1: start.x,  start.y,  start.z,  coupling
    row 2: jet.x,    jet.y,    jet.z,    density_rate
    row 3: heat_rate, target_flag, solid_flag, fuel_rate
"""
from dataclasses import dataclass
from math import isfinite, sqrt

MAX_SOURCES = 8
SOURCE_TABLE_SHAPE = (4, 4, MAX_SOURCES)
SOURCE_FLOATS = 16


@dataclass(frozen=True)
class Emission:
    """Single-emitter motion: swept start point, jet velocity and coupling rate."""
    start: tuple
    velocity: tuple = (0., 0., 0.)
    coupling: float = 0.

    def __post_init__(self):
        ok = (len(self.start) == 3 and len(self.velocity) == 3
              and all(isfinite(x) for x in (*self.start, *self.velocity, self.coupling))
              and self.coupling >= 0)
        if not ok:
            raise ValueError("Invalid emission parameters")


def motion_velocity(previous, current, interval, inheritance, jet, speed_limit):
    """Inherited emitter translation, capped at ``speed_limit``, plus a jet."""
    vectors_ok = all(len(v) == 3 for v in (previous, current, jet))
    scalars = (*previous, *current, *jet, interval, inheritance, speed_limit) if vectors_ok else ()
    if (not vectors_ok or not all(isfinite(v) for v in scalars) or interval <= 0
            or inheritance < 0 or speed_limit <= 0):
        raise ValueError("Invalid motion interval or limits")
    moved = [(b - a) / interval * inheritance for a, b in zip(previous, current)]
    speed = sqrt(sum(v * v for v in moved))
    scale = min(1., speed_limit / max(speed, 1e-20))
    return tuple(v * scale + j for v, j in zip(moved, jet))


@dataclass(frozen=True)
class Source:
    center: tuple
    radius: float
    density_rate: float
    heat_rate: float
    motion: Emission
    density_mode: str = "RATE"
    profile: str = "SOFT"
    fuel_rate: float = 0.0

    def __post_init__(self):
        if not isfinite(self.fuel_rate) or self.fuel_rate < 0:
            raise ValueError("Fuel rate must be finite and nonnegative")
        if self.density_mode not in {"RATE", "TARGET"} or self.profile not in {"SOFT", "SOLID"}:
            raise ValueError("Unknown source mode/profile")
        ok = (len(self.center) == 3
              and all(isfinite(v) for v in (*self.center, self.radius, self.density_rate, self.heat_rate))
              and self.radius > 0 and self.density_rate >= 0 and isinstance(self.motion, Emission))
        if not ok:
            raise ValueError("Invalid spherical source")


def pack_sources(sources):
    """Flatten up to eight sources into the 128-float device table."""
    if len(sources) > MAX_SOURCES:
        raise ValueError("At most eight sources are supported")
    table = []
    for s in sources:
        if not isinstance(s, Source):
            raise TypeError("Expected Source")
        table += [*s.center, s.radius,
                  *s.motion.start, s.motion.coupling,
                  *s.motion.velocity, s.density_rate,
                  s.heat_rate, float(s.density_mode == "TARGET"), float(s.profile == "SOLID"), s.fuel_rate]
    table += [0.] * (SOURCE_FLOATS * MAX_SOURCES - len(table))
    return tuple(table)
