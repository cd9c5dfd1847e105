"""CFL timestep selection.

``choose_timestep`` follows FluxFX ``fluxfx/physics/timestep.py:6-23`` (stable
quadratic root, or power-of-two halving in the quantized policy).
``cfl_timestep`` is the simple rule dt = min(max_dt, cfl * dx / max|u|) used by
the 64^3/256^3 smoke workloads.
"""
from math import hypot, isfinite, sqrt

from .config import validate_dt

MIN_TIMESTEP = 1e-6


def choose_timestep(max_dt, cfl, rate, acceleration_rate=0.0, *, quantized=True):
    validate_dt(max_dt)
    finite = all(isfinite(v) for v in (cfl, rate, acceleration_rate))
    if not finite or not 0 < cfl <= 2 or min(rate, acceleration_rate) < 0:
        raise ValueError('CFL and rate bounds must be finite and valid')

    def courant(dt):
        return rate * dt + acceleration_rate * dt * dt

    if not quantized:
        if courant(max_dt) <= cfl:
            return max_dt
        # Positive root of a dt^2 + r dt = cfl in the cancellation-free form, 1% margin.
        dt = .99 * (2 * cfl / (rate + hypot(rate, 2 * sqrt(acceleration_rate) * sqrt(cfl))))
        if dt < MIN_TIMESTEP:
            raise RuntimeError('Required timestep below 1 microsecond; reduce forces or reset')
        return min(max_dt, dt)
    dt = max_dt
    while courant(dt) > cfl:
        dt *= 0.5
        if dt < MIN_TIMESTEP:
            raise RuntimeError('Required timestep below 1 microsecond; reduce forces or reset')
    return dt


def cfl_timestep(max_dt, cfl, cell_size, max_speed):
    """dt = min(max_dt, cfl * min(h) / max|u|); max_dt when the flow is at rest."""
    validate_dt(max_dt)
    if not (isfinite(max_speed) and max_speed >= 0 and isfinite(cfl) and cfl > 0):
        raise ValueError('CFL and speed must be finite and valid')
    if max_speed <= 0:
        return max_dt
    dt = min(max_dt, cfl * min(cell_size) / max_speed)
    if dt < MIN_TIMESTEP:
        raise RuntimeError('Required timestep below 1 microsecond; reduce forces or reset')
    return dt
