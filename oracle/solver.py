"""CPU oracle of the solver objects -- TEST INFRASTRUCTURE ONLY.

Restates the host-side orchestration of FluxFX's backend on top of the
per-cell formulas in ``oracle/smoke.py``:

* ``OracleProjector`` -- ``backend/pressure.py:57-98`` (walls, divergence,
  impulse warm start and dt rescale, Jacobi budget), ``backend/multigrid.py:
  83-95`` (geometric V-cycles), ``backend/collision.py:75-88`` (masked Jacobi,
  cold start) and ``backend/solid_multigrid.py:67-76`` (aggregation V-cycles,
  cold multiplier on the first step).
* ``OracleSmoke`` -- ``backend/projected.py:61-202`` (reset and the step order:
  velocity transport + emission, buoyancy from the previous scalars,
  projection, scalar transport + emission).

Settings objects are duck-typed: anything with the attributes of
``PressureSettings``. The tolerance-driven cycle count (``pressure_tolerance``
> 0) stops when max|r| <= tol * max|rhs| for the level-0 residual r, checked
before every V-cycle, exactly as the device solver does.
"""
from math import ceil

import numpy as np

from . import fire as F
from . import smoke as S


class OracleProjector:
    def __init__(self, g, settings, kind, mask=None):
        self.g = g
        self.s = settings
        self.kind = kind                      # JACOBI | MULTIGRID | SOLID_JACOBI | SOLID_MULTIGRID
        self.pressure = g.zeros(g.cell_shape)
        self.history = None          # the extrapolated warm start's previous pressure per unit time
        self.last_dt = None
        self.last_iterations = 0
        self.last_cycles = 0
        self.mg = None
        self.levels = ()
        s = settings
        if kind == 'MULTIGRID':
            shapes = S.hierarchy_shapes(g.shape, s.mg_max_levels)
            self.levels = shapes
            inverse = None
            if s.coarse_solver == 'DIRECT' and (shapes[-1] == (4, 4, 4) or (s.mg_max_levels and np.prod(shapes[-1]) <= 512)):
                from fluxfx_b200.physics.coarse_pressure import neumann_inverse
                inverse = neumann_inverse(shapes[-1], g.extent64)
            self.mg = S.GeometricMG(g, s.mg_pre_sweeps or 3, s.mg_post_sweeps or 3, s.mg_max_levels,
                                    inverse, s.coarse_solver)
        elif kind == 'SOLID_MULTIGRID':
            self.refresh()

    def refresh(self):
        """(Re)build the aggregation hierarchy from the grid's current mask (at
        construction, and after a collider move: the multigrid-with-moving-
        colliders extension of the fire configuration)."""
        g, s = self.g, self.s
        if self.kind == 'SOLID_MULTIGRID':
            hier = S.build_hierarchy(g.shape, g.extent64, g.mask, s.mg_max_levels)
            self.levels = [h[0] for h in hier]
            self.mg = S.SolidMG(hier, s.mg_pre_sweeps or 4, s.mg_post_sweeps or 4, s.coarse_solver, g.dt,
                                getattr(s, 'mg_coarse_scale', 1.0), getattr(s, 'mg_coarse_sweeps', 0))

    @property
    def uses_impulse(self):
        if self.kind.startswith('SOLID'):
            return True
        ws = self.s.pressure_warm_start
        return ws == 'IMPULSE' or (ws == 'AUTO' and len(self.levels) > 1)

    def reset(self):
        self.pressure = self.g.zeros(self.g.cell_shape)
        self.history = None
        self.last_dt = None
        self.last_iterations = 0
        self.last_cycles = 0

    def _mask(self):
        return self.g.mask if self.kind.startswith('SOLID') else None

    def _jacobi_solve(self, rhs, dt, previous_dt):
        s = self.s
        if previous_dt != dt:
            self.pressure = self.g.zeros(self.g.cell_shape)
        scaled = ceil(s.pressure_iterations * max(1.0, (max(self.g.shape) / 64) ** 2))
        mult = s.pressure_cold_multiplier if previous_dt != dt else 1
        self.last_iterations = min(4096, scaled * mult)
        for _ in range(self.last_iterations):
            self.pressure = S.jacobi(self.g, self.pressure, rhs, dt, s.pressure_relaxation, mask=self._mask())

    def _residual_max(self, rhs, dt):
        if self.kind == 'MULTIGRID':
            r = S.residual(self.g, self.pressure, rhs, dt, self.mg.invs[0])
        else:
            r = S.graph_residual(self.pressure, rhs, self.mg.levels[0][1])
        return float(np.abs(r.astype(np.float64)).max())

    def _cycles(self, rhs, dt, budget):
        s = self.s
        tol = s.pressure_tolerance
        self.last_cycles = 0
        if tol <= 0:
            for _ in range(budget):
                self._one_cycle(rhs, dt)
                self.last_cycles += 1
            return
        scale = float(np.abs(rhs.astype(np.float64)).max()) / (dt if self.kind == 'MULTIGRID' else 1.0)
        if scale == 0:
            self.pressure = self.g.zeros(self.g.cell_shape)
            return
        while self.last_cycles < s.pressure_max_cycles and self._residual_max(rhs, dt) > tol * scale:
            self._one_cycle(rhs, dt)
            self.last_cycles += 1

    def _one_cycle(self, rhs, dt):
        if self.kind == 'MULTIGRID':
            self.pressure = self.mg.cycle(0, self.pressure, rhs, dt)
        else:
            self.pressure = self.mg.cycle(0, self.pressure, rhs)

    def solve(self, rhs, dt, previous_dt):
        s = self.s
        if self.kind == 'JACOBI':
            self.last_cycles = 0
            return self._jacobi_solve(rhs, dt, previous_dt)
        if self.kind == 'SOLID_JACOBI':
            self.pressure = self.g.zeros(self.g.cell_shape)
            self.last_cycles = 0
            return self._jacobi_solve(rhs, dt, previous_dt)
        if self.kind == 'MULTIGRID':
            if len(self.levels) == 1:
                self.last_cycles = 0
                return self._jacobi_solve(rhs, dt, previous_dt)
            if previous_dt != dt:
                self.pressure = self.g.zeros(self.g.cell_shape)
            self.mg.sweeps = 0
            self._cycles(rhs, dt, s.pressure_cycles)
            self.last_iterations = self.mg.sweeps
            return
        # SOLID_MULTIGRID
        if len(self.levels) == 1:
            self.last_cycles = 0
            self.pressure = self.g.zeros(self.g.cell_shape)
            return self._jacobi_solve(rhs, dt, previous_dt)
        if not (s.solid_warm_start and previous_dt is not None):
            self.pressure = self.g.zeros(self.g.cell_shape)
        self.mg.sweeps = 0
        budget = s.pressure_cycles * (s.pressure_cold_multiplier if previous_dt is None else 1)
        self._cycles(rhs, dt, budget)
        self.last_iterations = self.mg.sweeps

    def project(self, vel, dt):
        """Returns (corrected faces, divergence before, divergence after)."""
        g = self.g
        previous_dt, self.last_dt = self.last_dt, None
        bounded = S.walls(g, vel)
        before = S.divergence(g, bounded)
        impulse = self.uses_impulse
        solve_dt = 1.0 if impulse else dt
        previous_solve = (1.0 if previous_dt is not None else None) if impulse else previous_dt
        beta = getattr(self.s, 'warm_start_extrapolation', 0.0)
        extrapolates = (beta > 0 and self.kind == 'SOLID_MULTIGRID' and len(self.levels) > 1
                        and self.s.solid_warm_start
                        and not (getattr(self.s, 'learned_warm_start', False) and getattr(self.s, 'learned_correction', False)))
        if impulse and previous_dt is not None and extrapolates and getattr(self.s, 'warm_start_order', 1) == 2:
            hist = self.history or []
            self.pressure, newest = extrapolate2(self.pressure, hist, dt, previous_dt, beta)
            # (P1, its dt) first, then the solve before it
            self.history = [(newest, float(np.float32(previous_dt)))] + hist[:1]
        elif impulse and previous_dt is not None and extrapolates:
            self.pressure, self.history = extrapolate(self.pressure, self.history, dt, previous_dt, beta)
        elif impulse and previous_dt is not None and abs(dt / previous_dt - 1.0) > 1e-6:
            self.pressure = self.pressure * g.f(dt / previous_dt)
        if previous_dt is None:
            self.history = None
        self.solve(before, solve_dt, previous_solve)
        out = S.gradient(g, bounded, self.pressure, solve_dt)
        after = S.divergence(g, out)
        self.last_dt = dt
        return out, before, after


def extrapolate(p, history, dt, previous_dt, beta):
    """The extrapolated warm start (an extension of the solver, not in the
    reference): with P1 = p / previous dt and P2 = history, the start is
    dt (P1 + beta (dt / previous dt) (P1 - P2)); returns (start, P1). The time
    steps are rounded to FP32 first (the device keeps them as floats), the
    coefficients formed in FP64 and the update done in FP32, as the device
    pass does; without a history (the first warm solve) the start is the
    dt / previous dt rescale."""
    d0, d1 = float(np.float32(dt)), float(np.float32(previous_dt))
    r = d0 / d1
    p = np.asarray(p, np.float32)
    new_history = p * np.float32(1.0 / d1)
    if history is None:
        c1 = np.float32(r) if abs(r - 1.0) > 1e-6 else np.float32(1.0)
        return p * c1, new_history
    c1 = np.float32(d0 * (1.0 + beta * r) / d1)
    c2 = np.float32(d0 * beta * r)
    return c1 * p - c2 * np.asarray(history, np.float32), new_history


def extrapolate2(p, history, dt, previous_dt, beta):
    """The quadratic form of the extrapolated start (``warm_start_order`` 2):
    ``history`` holds up to two earlier solves as (pressure per unit time, the
    dt of that solve), newest first. With P1 = p / previous dt at time 0 and
    the stored ones at -d1 and -d1 - d2, the start is d0 (P1 + beta (Q - P1))
    with Q their Lagrange quadratic at d0 (the linear form with one stored
    solve, the dt rescale with none). FP32 time steps, FP64 coefficients,
    FP32 update ((a0 v + a1 h1) + a2 h2), as the device pass does; returns
    (start, P1)."""
    d0, d1 = float(np.float32(dt)), float(np.float32(previous_dt))
    r, b = d0 / d1, beta
    v = np.asarray(p, np.float32)
    newest = v * np.float32(1.0 / d1)
    if not history:
        c = np.float32(r) if abs(r - 1.0) > 1e-6 else np.float32(1.0)
        return v * c, newest
    if len(history) == 1:
        a0, a1 = np.float32(d0 * (1.0 + b * r) / d1), np.float32(-d0 * b * r)
        return a0 * v + a1 * history[0][0], newest
    d2 = history[0][1]
    l0 = (d0 + d1) * (d0 + d1 + d2) / (d1 * (d1 + d2))
    l1 = -d0 * (d0 + d1 + d2) / (d1 * d2)
    l2 = d0 * (d0 + d1) / ((d1 + d2) * d2)
    a0 = np.float32(d0 * (1.0 + b * (l0 - 1.0)) / d1)
    a1, a2 = np.float32(d0 * b * l1), np.float32(d0 * b * l2)
    return (a0 * v + a1 * history[0][0]) + a2 * history[1][0], newest


def projector_kind(grid_shape, settings, has_mask):
    """Which projector DenseProjectedSmoke builds (``backend/projected.py:26-40``)."""
    shapes = S.hierarchy_shapes(grid_shape)
    use_mg = len(shapes) > 1 and (settings.pressure_solver == 'MULTIGRID' or
                                  (settings.pressure_solver == 'AUTO' and min(grid_shape) >= 16))
    if has_mask:
        return 'SOLID_MULTIGRID' if (not settings.moving_colliders and use_mg) else 'SOLID_JACOBI'
    return 'MULTIGRID' if use_mg else 'JACOBI'


class OracleSmoke:
    """Field state and step sequence of ``DenseProjectedSmoke``."""

    def __init__(self, shape, extent, settings, dtype=np.float32, mask=None, kind=None, colliders=None):
        """``colliders``: ((shape, inverse_rows), ...) of moving colliders
        (settings.moving_colliders); their FP32 owner mask replaces ``mask``."""
        self.colliders = tuple(colliders) if colliders is not None else None
        if self.colliders is not None:
            g0 = S.Grid(shape, extent, dtype)
            self.owners = F.moving_mask(g0, self.colliders)
            mask = self.owners > 0.5
        self.g = S.Grid(shape, extent, dtype, mask)
        if self.colliders is not None:
            self.g.boundary = tuple(self.g.zeros(fs) for fs in self.g.face_shapes)
        self.s = settings
        self.kind = kind or projector_kind(tuple(shape), settings, mask is not None)
        self.projector = OracleProjector(self.g, settings, self.kind)
        self.time = 0.0
        self.steps = 0
        self.before = self.after = None
        self.reset()

    def reset(self, seed=True):
        g, s = self.g, self.s
        if seed:
            self.density = S.seed_scalar(g, s.source_center, s.source_radius)
            self.temperature = S.seed_scalar(g, s.source_center, s.source_radius, s.initial_temperature)
            self.velocity = S.seed_faces(g, s.velocity, s.angular_speed)
        else:
            self.density = g.zeros(g.cell_shape)
            self.temperature = g.zeros(g.cell_shape)
            self.velocity = tuple(g.zeros(fs) for fs in g.face_shapes)
        if g.mask is not None:
            self.density = np.where(g.mask, g.f(0), self.density)
            self.temperature = np.where(g.mask, g.f(0), self.temperature)
        self.fuel = g.zeros(g.cell_shape) if s.combustion_enabled else None
        self.flame = g.zeros(g.cell_shape) if s.combustion_enabled else None
        self.projector.reset()
        self.velocity = S.walls(g, self.velocity)
        self.time = 0.0
        self.steps = 0

    def upload(self, density=None, temperature=None, velocity=None):
        g = self.g
        if density is not None:
            self.density = np.asarray(density, dtype=g.dt).reshape(g.cell_shape)
            if g.mask is not None:
                self.density = np.where(g.mask, g.f(0), self.density)
        if temperature is not None:
            self.temperature = np.asarray(temperature, dtype=g.dt).reshape(g.cell_shape)
            if g.mask is not None:
                self.temperature = np.where(g.mask, g.f(0), self.temperature)
        if velocity is not None:
            self.velocity = tuple(np.asarray(v, dtype=g.dt).reshape(fs) for v, fs in zip(velocity, g.face_shapes))
            if g.mask is not None:
                self.velocity = S.walls(g, self.velocity)
        self.projector.reset()

    def step(self, dt, emission=None, sources=None):
        """One step. ``emission``: object with start/velocity/coupling (the
        reference's ``Emission``), default a static emitter at the source
        centre; ``sources``: (packed 128-float table, count)."""
        g, s = self.g, self.s
        vel = self.velocity
        detail = s.velocity_advection == 'MACCORMACK'
        emitter = None
        table = None
        if sources is not None:
            table = sources          # (128 floats, count)
        else:
            start = emission.start if emission is not None else s.source_center
            jet = emission.velocity if emission is not None else (0.0, 0.0, 0.0)
            coupling = emission.coupling if emission is not None else 0.0
            emitter = dict(center=s.source_center, start=start, radius=s.source_radius,
                           solid=s.source_profile == 'SOLID', jet=jet, coupling=coupling)
        preds = [S.face_predictor(g, vel, a, dt) for a in range(3)] if detail else list(vel)
        new = [S.advect_velocity_face(g, vel, preds[a], a, dt, detail, s.velocity_blend,
                                      emitter=emitter, sources=table) for a in range(3)]
        new[2] = S.buoyancy(g, new[2], self.density, self.temperature, dt, s.thermal_lift, s.density_weight)
        if s.vorticity_strength > 0:
            # confinement of the provisional (unwalled) velocity before projection (projected.py:172-175)
            new = F.confine(g, new, F.curl(g, new), dt, s.vorticity_strength, s.vorticity_limit)
        out, self.before, self.after = self.projector.project(tuple(new), dt)
        self.velocity = out
        corrected = s.scalar_advection == 'MACCORMACK'
        channels = [(0, self.density, s.source_rate, s.dissipation,
                     s.source_rate if s.density_mode == 'TARGET' else -1.0),
                    (1, self.temperature, s.heat_source_rate, s.cooling,
                     s.heat_source_rate if s.heat_mode == 'TARGET' else -1.0)]
        if self.fuel is not None:
            channels.append((2, self.fuel, s.fuel_source_rate, 0.0, -1.0))
        results = []
        for ch, field, rate, decay, target in channels:
            if corrected:
                pred = S.scalar_transport(g, out, field, dt)
                rev = S.scalar_transport(g, out, pred, -dt)
            else:
                pred = rev = field
            results.append(S.advect_scalar(g, out, field, pred, rev, dt, corrected, rate, decay, target,
                                           emitter=emitter, sources=table, channel=ch,
                                           target_heat=s.heat_mode == 'TARGET'))
        self.density, self.temperature = results[:2]
        if self.fuel is not None:
            # combustion after transport (backend/combustion.py:21-31)
            self.fuel = results[2]
            self.flame = F.burn(g, self.fuel, self.temperature, dt, s.ignition_temperature, s.burn_rate)
            self.fuel = F.apply_burn(g, self.fuel, self.flame, dt, -1.0)
            self.density = F.apply_burn(g, self.density, self.flame, dt, s.smoke_yield)
            self.temperature = F.apply_burn(g, self.temperature, self.flame, dt, s.heat_yield)
        self.time += dt
        self.steps += 1

    def move_colliders(self, colliders, dt):
        """New collider poses before a step (backend/moving_collision.py:44-82):
        owner mask, rigid wall velocities, remap of the fields."""
        g = self.g
        colliders = tuple(colliders)
        old = self.owners
        self.owners = F.moving_mask(g, colliders)
        table = F.velocity_table([c[1] for c in self.colliders], [c[1] for c in colliders], dt)
        g.boundary = F.moving_walls(g, self.owners, table)
        self.colliders = colliders
        g.set_mask(self.owners > 0.5)
        self.projector.refresh()
        self.density = F.remap_scalar(g, self.density, self.owners, old)
        self.temperature = F.remap_scalar(g, self.temperature, self.owners, old)
        self.velocity = F.remap_faces(g, self.velocity, self.owners, old, g.boundary)
        if self.fuel is not None:
            self.fuel = F.remap_scalar(g, self.fuel, self.owners, old)
            self.flame = g.zeros(g.cell_shape)

    def rel_div(self):
        b = float(np.abs(self.before.astype(np.float64)).max())
        a = float(np.abs(self.after.astype(np.float64)).max())
        return a / b if b > 0 else 0.0
