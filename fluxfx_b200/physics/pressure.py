"""Pressure/solver settings and divergence statistics.

Fields, defaults and validation follow FluxFX ``fluxfx/physics/pressure.py:7-80``.
Extensions (all default to the reference's behaviour):

* ``pressure_tolerance`` -- 0 keeps the reference's fixed V-cycle budget; a
  positive value runs V-cycles until the relative max-norm divergence
  (max|div_after| / max|div_before|) is at or below it, capped by
  ``pressure_max_cycles``.
* ``mg_pre_sweeps`` / ``mg_post_sweeps`` -- 0 keeps the reference's sweeps
  (3/3 geometric, 4/4 collider aggregation).
* ``mg_coarse_sweeps`` -- collider multigrid: 0 keeps the level-0 sweep counts
  on every level (the reference); N runs N pre- and N post-sweeps on every
  level below level 0 (level 0 keeps ``mg_pre_sweeps`` / ``mg_post_sweeps``).
* ``mg_max_levels`` -- 0 keeps the reference's hierarchy (halve while all axes
  are even and the smallest is >= 8); N caps it at N levels.
* ``heat_mode`` -- "RATE" (reference: temperature emission is additive) or
  "TARGET" (temperature is raised to ``heat_source_rate * weight``).
* ``velocity_blend`` -- weight of the clamped MacCormack value against the
  first-order value; 0.5 is the reference (``correct_velocity_fused.glsl:26``).
* ``storage`` -- "FP32" or "BF16" storage of velocity and advected scalars
  (arithmetic is FP32 either way).
* ``solid_warm_start`` -- reuse the previous step's pressure with colliders
  instead of the reference's cold start.
* ``learned_correction`` -- with ``learned_warm_start`` and
  ``solid_warm_start``: on warm starts, add the network's answer for the
  residual of the previous pressure to it (a learned correction) instead of
  using the previous pressure alone.
* ``pressure_method`` -- "VCYCLE" (reference: stand-alone V-cycles) or "PCG"
  (conjugate gradients preconditioned by the same symmetric aggregation
  V-cycle; collider multigrid only). Both solve the same system to the same
  tolerance. "IR": iterative refinement -- every outer iteration recomputes the
  true FP32 residual of the pressure, decides convergence in FP64, solves the
  correction equation from zero with ``ir_inner_cycles`` V-cycles and adds the
  correction (collider multigrid with a tolerance).
* ``warm_start_extrapolation`` -- with ``solid_warm_start`` (and no learned
  warm start): beta in [0, 1]. The solve starts from the previous two
  pressures extrapolated linearly in time, P1 + beta (dt / dt1) (P1 - P2) in
  pressure per unit time, instead of the previous pressure alone (0, the
  default). Same system, same tolerance; only the start differs.
  ``warm_start_order`` 2 extrapolates with the quadratic through the last
  three pressures instead (P1 + beta (Q - P1)).
"""
from dataclasses import dataclass
from math import fsum, isfinite, sqrt

from .thermal import ThermalSettings

_CHOICES = {
    "coarse_solver": ({"DIRECT", "SMOOTH"}, "Unknown coarse pressure solver"),
    "timestep_policy": ({"AUTO", "CONTINUOUS", "QUANTIZED"}, "Unknown timestep policy"),
    "velocity_advection": ({"SEMI_LAGRANGIAN", "MACCORMACK"}, "Unknown velocity advection"),
    "pressure_warm_start": ({"AUTO", "IMPULSE", "LEGACY"}, "Unknown pressure warm start"),
    "density_mode": ({"RATE", "TARGET"}, "Unknown emission mode/profile"),
    "source_profile": ({"SOFT", "SOLID"}, "Unknown emission mode/profile"),
    "scalar_advection": ({"SEMI_LAGRANGIAN", "MACCORMACK"}, "Unknown scalar advection"),
    "pressure_solver": ({"AUTO", "JACOBI", "MULTIGRID"}, "Unknown pressure solver"),
    "heat_mode": ({"RATE", "TARGET"}, "Unknown heat emission mode"),
    "storage": ({"FP32", "BF16"}, "Unknown field storage"),
    "pressure_method": ({"VCYCLE", "PCG", "IR"}, "Unknown pressure method"),
}

_TURBULENCE_RANGES = (
    ("turbulence_strength", 0, 20), ("turbulence_scale", .01, 4), ("turbulence_speed", 0, 10),
    ("turbulence_limit", .01, 20), ("turbulence_threshold", .001, 2000))

_INT_RANGES = (
    ("pressure_cycles", 1, 16, "Multigrid cycles must be an integer in [1, 16]"),
    ("pressure_iterations", 1, 4096, "Pressure iterations must be an integer in [1, 4096]"),
    ("pressure_cold_multiplier", 1, 8, "Cold-start multiplier must be an integer in [1, 8]"),
    ("pressure_max_cycles", 1, 256, "Maximum V-cycles must be an integer in [1, 256]"),
    ("mg_pre_sweeps", 0, 16, "Multigrid sweeps must be integers in [0, 16]"),
    ("mg_post_sweeps", 0, 16, "Multigrid sweeps must be integers in [0, 16]"),
    ("mg_max_levels", 0, 16, "Multigrid level cap must be an integer in [0, 16]"),
    ("mg_coarse_sweeps", 0, 16, "Coarse-level sweeps must be an integer in [0, 16]"),
    ("ir_inner_cycles", 1, 16, "Inner refinement cycles must be an integer in [1, 16]"),
)


@dataclass(frozen=True)
class PressureSettings(ThermalSettings):
    turbulence_strength: float = 0.0
    turbulence_scale: float = 0.5
    turbulence_speed: float = 0.5
    turbulence_seed: int = 0
    turbulence_octaves: int = 3
    turbulence_limit: float = 2.0
    turbulence_mask: str = 'DENSITY'
    turbulence_threshold: float = 0.2
    combustion_enabled: bool = False
    fuel_source_rate: float = 1.0
    ignition_temperature: float = 150.0
    burn_rate: float = 4.0
    heat_yield: float = 600.0
    smoke_yield: float = 1.0
    moving_colliders: bool = False
    velocity_advection: str = "SEMI_LAGRANGIAN"
    timestep_policy: str = "AUTO"
    pressure_warm_start: str = "AUTO"
    coarse_solver: str = "DIRECT"
    density_mode: str = "RATE"
    source_profile: str = "SOFT"
    scalar_advection: str = "SEMI_LAGRANGIAN"
    vorticity_strength: float = 0.0
    vorticity_limit: float = 2.0
    pressure_solver: str = "AUTO"
    pressure_cycles: int = 2
    pressure_iterations: int = 80
    pressure_relaxation: float = 2.0 / 3.0
    pressure_cold_multiplier: int = 4
    # --- extensions (defaults reproduce the reference) ---
    pressure_tolerance: float = 0.0
    pressure_max_cycles: int = 64
    mg_pre_sweeps: int = 0
    mg_post_sweeps: int = 0
    mg_max_levels: int = 0
    heat_mode: str = "RATE"
    velocity_blend: float = 0.5
    storage: str = "FP32"
    solid_warm_start: bool = False
    pressure_method: str = "VCYCLE"
    learned_warm_start: bool = False
    mg_coarse_scale: float = 1.0
    learned_correction: bool = False
    ir_inner_cycles: int = 1
    warm_start_extrapolation: float = 0.0
    mg_coarse_sweeps: int = 0
    warm_start_order: int = 1

    def __post_init__(self):
        super().__post_init__()
        for name, low, high in _TURBULENCE_RANGES:
            value = getattr(self, name)
            if not isfinite(value) or not low <= value <= high:
                raise ValueError('Invalid turbulence parameter')
        if type(self.turbulence_seed) is not int or not 0 <= self.turbulence_seed <= 65535:
            raise ValueError('Invalid turbulence seed')
        if type(self.turbulence_octaves) is not int or not 1 <= self.turbulence_octaves <= 4:
            raise ValueError('Use one to four turbulence scales')
        if self.turbulence_mask not in {'ALL', 'DENSITY', 'HEAT'}:
            raise ValueError('Invalid turbulence mask')
        if type(self.combustion_enabled) is not bool:
            raise ValueError("Combustion enabled must be boolean")
        kinetics = (self.fuel_source_rate, self.ignition_temperature, self.burn_rate,
                    self.heat_yield, self.smoke_yield)
        if not all(isfinite(v) and v >= 0 for v in kinetics):
            raise ValueError("Combustion parameters must be finite and nonnegative")
        for name, (allowed, message) in _CHOICES.items():
            if getattr(self, name) not in allowed:
                raise ValueError(message)
        if not isfinite(self.vorticity_strength) or not 0 <= self.vorticity_strength <= 20:
            raise ValueError("Curl strength must lie in [0,20]")
        if not isfinite(self.vorticity_limit) or not 0 < self.vorticity_limit <= 20:
            raise ValueError("Curl acceleration limit must lie in (0,20]")
        for name, low, high, message in _INT_RANGES:
            value = getattr(self, name)
            if type(value) is not int or not low <= value <= high:
                raise ValueError(message)
        if not isfinite(self.pressure_relaxation) or not 0 < self.pressure_relaxation < 1:
            raise ValueError("Jacobi relaxation must lie strictly between zero and one")
        if not isfinite(self.pressure_tolerance) or not 0 <= self.pressure_tolerance < 1:
            raise ValueError("Pressure tolerance must lie in [0, 1)")
        if not isfinite(self.velocity_blend) or not 0 <= self.velocity_blend <= 1:
            raise ValueError("Velocity blend must lie in [0, 1]")
        if type(self.solid_warm_start) is not bool:
            raise ValueError("Collider warm start must be boolean")
        if type(self.learned_correction) is not bool:
            raise ValueError("Learned correction must be boolean")
        if type(self.learned_warm_start) is not bool:
            raise ValueError("Learned warm start must be boolean")
        if not isfinite(self.mg_coarse_scale) or not 0 < self.mg_coarse_scale < 2:
            raise ValueError("Coarse-correction factor must lie in (0, 2)")
        if (type(self.warm_start_extrapolation) not in (int, float) or not isfinite(self.warm_start_extrapolation)
                or not 0 <= self.warm_start_extrapolation <= 1):
            raise ValueError("Warm-start extrapolation must lie in [0, 1]")
        if type(self.warm_start_order) is not int or self.warm_start_order not in (1, 2):
            raise ValueError("Warm-start extrapolation order must be 1 or 2")


def divergence_stats(before, after):
    """rms/max/mean of the divergence before and after projection (FP64 sums)."""
    if not before or len(before) != len(after):
        raise ValueError("Divergence arrays must be nonempty and equal in length")
    if not all(isfinite(v) for v in before) or not all(isfinite(v) for v in after):
        raise ValueError("Non-finite divergence")
    n = len(before)
    rms_before = sqrt(fsum(v * v for v in before) / n)
    rms_after = sqrt(fsum(v * v for v in after) / n)
    if rms_before > 0:
        ratio = rms_after / rms_before
    else:
        ratio = 0.0 if rms_after == 0 else None
    return {"rms_before": rms_before, "rms_after": rms_after, "ratio": ratio,
            "max_before": max(abs(v) for v in before), "max_after": max(abs(v) for v in after),
            "mean_before": fsum(before) / n, "mean_after": fsum(after) / n}
