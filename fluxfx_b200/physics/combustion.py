"""Single-cell fuel kinetics (FluxFX ``fluxfx/physics/combustion.py:6-11``)."""
from math import expm1, isfinite

from .config import validate_dt


def react(fuel, temperature, dt, ignition, burn_rate):
    """Fuel consumed in dt by exact first-order decay when temperature >= ignition."""
    validate_dt(dt)
    if not all(isfinite(v) for v in (fuel, temperature, ignition, burn_rate)) or min(fuel, ignition, burn_rate) < 0:
        raise ValueError("Invalid combustion state")
    if temperature < ignition:
        return 0.
    return -fuel * expm1(-burn_rate * dt)
