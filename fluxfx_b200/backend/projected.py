"""The dense smoke step: transport, buoyancy, projection, scalar transport.

Drop-in for FluxFX ``fluxfx/backend/projected.py:13-229``
(``DenseProjectedSmoke``): same constructor, step order and state machine
(``faulted`` after a failed step until ``reset``). One step enqueues:

1. ``ffx_face_predictor`` (MacCormack velocity only);
2. ``ffx_advect_velocity`` -- transport of U, V, W, emitter coupling, buoyancy
   on W from the previous density/temperature and the wall condition, written
   straight into the projector's bounded faces;
3. the projection (divergence, pressure solve, gradient + divergence after);
4. ``ffx_scalar_transport`` x2 (MacCormack predictor and reverse of density and
   temperature together) and ``ffx_advect_scalars`` (both channels, decay and
   emission) -- one launch per pass for both scalars.

Fire configuration (``projected.py:161-200``): vorticity confinement between
buoyancy and projection (``ffx_curl`` + ``ffx_confine``), fuel as a third
transported scalar and ``ffx_combustion`` after transport, moving colliders
through ``move_colliders`` (``MovingSolidDevice``).

Extensions: ``settings.storage == 'BF16'`` stores velocity and scalars in
bfloat16 (FP32 arithmetic); ``heat_mode == 'TARGET'`` raises temperature to the
emitter value instead of adding a rate.
"""
import ctypes as C

import torch

from .. import _native as N
from ..physics.config import GridSpec, validate_dt
from ..physics.emission import Emission, pack_sources, SOURCE_TABLE_SHAPE
from ..physics.interaction import validate_live_update
from ..physics.pressure import PressureSettings
from .dense import SEED_CONSTANTS
from .detail import DetailPasses
from .device import ptr, solids_struct
from .mac import FACE_CONSTANTS, VELOCITY_NAMES
from .pressure import PressureProjector
from .thermal import DenseThermalAdvection


class DenseProjectedSmoke(DenseThermalAdvection):
    def __init__(self, grid=None, settings=None, device=None, projector_class=None, *, colliders=()):
        settings = settings or PressureSettings()
        self._field_dtype = torch.bfloat16 if settings.storage == 'BF16' else torch.float32
        self.combustion = None
        self.solids = None
        if colliders:
            from .collision import SolidDevice, SolidPressureProjector
            from .multigrid import use_multigrid
            from .solid_multigrid import SolidMultigridProjector
            grid = grid or GridSpec()
            if settings.moving_colliders:
                from .moving_collision import MovingSolidDevice
                device = self.solids = MovingSolidDevice(grid, colliders, device)
                # the reference projects moving-collider scenes with masked Jacobi (projected.py:28)
                projector_class = projector_class or SolidPressureProjector
            else:
                device = self.solids = SolidDevice(grid, colliders, device)
                projector_class = SolidMultigridProjector if use_multigrid(grid, settings) else SolidPressureProjector
        if settings.turbulence_strength > 0:
            raise ValueError('Turbulence is not part of this build')
        self.projector = None
        self.detail = None
        self.turbulence = None
        self.pass_timer = None
        self.faulted = False
        self._source_data = None
        self._sources = N.FfxSources()
        self._sources.count = -1
        super().__init__(grid, settings, device)
        if projector_class is None:
            from .multigrid import MultigridPressureProjector, use_multigrid
            projector_class = MultigridPressureProjector if use_multigrid(self.grid, self.settings) else PressureProjector
        self.projector = projector_class(self.grid, self.settings, self.device)
        self.detail = DetailPasses(self.grid, self.device, self._field_dtype)
        if self.settings.combustion_enabled:
            from .combustion import CombustionPasses
            self.combustion = CombustionPasses(self.grid, self.device, self._field_dtype)
        self._solids = solids_struct(self.solids) if self.solids is not None else N.FfxSolids()
        # the reference's pass handles, for scripts that drive single passes
        # through device.dispatch (backend/projected.py:47-54, 135-146)
        self._closed_scalar = self.device.kernel('closed_advect_scalar.glsl')
        self._emitting_velocity = self.device.kernel('emitting_advect_velocity.glsl')
        self._multi_scalar = self._multi_velocity = None
        self._source_table = None
        self._maxima = torch.zeros(3, dtype=torch.float32, device=self.device.device)
        # device-side time step (step_cfl): clock = (dt, previous dt), time in FP64
        self._clock = torch.zeros(2, dtype=torch.float32, device=self.device.device)
        self._clock_time = torch.zeros(1, dtype=torch.float64, device=self.device.device)
        self._clock_live = False
        self.reset()

    # Simulation time: host steps add dt here; device-timed steps (step_cfl)
    # accumulate it on the device, read (once, synchronising) when asked.
    @property
    def time(self):
        if getattr(self, '_clock_live', False):
            return self._time_host + float(self.device.fetch(self._clock_time))
        return self._time_host

    @time.setter
    def time(self, value):
        self._time_host = float(value)
        if getattr(self, '_clock_live', False):
            self._clock_time.zero_()

    @property
    def allocated_bytes(self):
        extra = (self.solids.allocated_bytes if self.solids else 0) + (self.combustion.allocated_bytes
                                                                       if self.combustion else 0)
        return super().allocated_bytes + extra + self.projector.allocated_bytes + self.detail.allocated_bytes

    def reset(self, seed=True):
        with self.device.ordered():
            super().reset(seed)
            self._clock_live = False      # the next step_cfl starts again from dt_max
            self.faulted = False
            if self.combustion is not None:
                self.combustion.reset()
            if self.solids is not None:
                self.solids.clear_solid(self._front, self._back)
                self._front, self._back = self._back, self._front
                if self._temperature is not None:
                    self.solids.clear_solid(self._temperature, self._temperature_back)
                    self._temperature, self._temperature_back = self._temperature_back, self._temperature
            if self.projector is not None:
                self.projector.reset()
                self.projector.enforce_walls(self._velocity, self._velocity_back)
                self._velocity, self._velocity_back = self._velocity_back, self._velocity

    def upload_velocity(self, components):
        with self.device.ordered():
            super().upload_velocity(components)
            if self.solids is not None:
                self.projector.enforce_walls(self._velocity, self._velocity_back)
                self._velocity, self._velocity_back = self._velocity_back, self._velocity
            self.projector.reset()

    def upload(self, values):
        with self.device.ordered():
            super().upload(values)
            if self.solids is not None:
                self.solids.clear_solid(self._front, self._back)
                self._front, self._back = self._back, self._front
            self.projector.reset()

    def upload_temperature(self, values):
        with self.device.ordered():
            super().upload_temperature(values)
            if self.solids is not None:
                self.solids.clear_solid(self._temperature, self._temperature_back)
                self._temperature, self._temperature_back = self._temperature_back, self._temperature
            self.projector.reset()

    def update_settings(self, settings):
        """Apply live parameters between steps, preserving all fields and pressure."""
        validate_live_update(self.settings, settings)
        self.settings = settings
        self.projector.settings = settings

    def move_colliders(self, colliders, dt):
        """New collider poses before a step (``projected.py:103-115``)."""
        with self.device.ordered():
            if not self.settings.moving_colliders or self.solids is None:
                raise ValueError('Enable Moving colliders and Reset first')
            validate_dt(dt)
            if self.faulted:
                raise RuntimeError('Reset required after a failed GPU step')
            try:
                self.solids.update(colliders, dt)
                self.solids.remap(self)
                refresh = getattr(self.projector, 'refresh_hierarchy', None)
                if refresh is not None:
                    refresh()            # multigrid with moving colliders (extension): follow the new mask
                self.projector.ready = False
            except Exception:
                self.faulted = True
                raise

    def measure_projection(self):
        return self.projector.metrics() | {"step": self.steps, "simulation_time": self.time}

    def step_cfl(self, cfl=0.5, dt_max=0.02, emission=None, sources=None):
        """One step whose time step lives on the device: the first step of a
        run (after construction or ``reset``) uses ``dt_max``; every step ends
        by setting the next dt = min(dt_max, cfl * cell / max|u|) on the device
        from the face maxima of its corrected velocity (cell = the smallest cell
        spacing), in FP64 -- the rule the workloads state. Nothing is read back:
        with the device-side V-cycle loop a step is queued without waiting for
        the GPU. ``time`` and ``current_dt()`` read the clock when asked. Needs
        the impulse pressure form (multigrid or colliders); not with
        confinement, combustion or moving colliders."""
        with self.device.ordered():
            if not (0 < cfl <= 10 and 0 < dt_max <= 0.1):
                raise ValueError('cfl must lie in (0, 10] and dt_max in (0, 0.1]')
            s = self.settings
            if s.vorticity_strength > 0 or self.combustion is not None or s.moving_colliders:
                raise ValueError('Device time steps cover the smoke step without confinement, combustion '
                                 'or moving colliders')
            if sources is not None:
                self._prepare_sources(sources)
            if self.faulted:
                raise RuntimeError("Reset required after a failed GPU step")
            if not self._clock_live:
                previous = self.projector.previous_dt()
                self._clock[0] = dt_max
                self._clock[1] = previous if previous is not None else 0.0
                self._clock_time.zero_()
                self._clock_live = True
            try:
                self._step(None, emission or Emission(self.settings.source_center), sources, clock=self._clock)
                cell = min(e / n for e, n in zip(self.grid.extent, self.grid.shape))
                self.device.call('ffx_next_dt', ptr(self.projector._scalars[0:3]), ptr(self._clock),
                                 ptr(self._clock_time), cell, float(cfl), float(dt_max), self.device.s)
            except Exception:
                self.faulted = True
                self.projector.ready = False
                raise

    def current_dt(self):
        """The dt the next ``step_cfl`` will take (one readback)."""
        return float(self.device.fetch(self._clock[0]))

    def step(self, dt=1.0 / 30.0, emission=None, sources=None):
        with self.device.ordered():
            validate_dt(dt)
            if sources is not None:
                self._prepare_sources(sources)
            if self.faulted:
                raise RuntimeError("Reset required after a failed GPU step")
            try:
                self._step(dt, emission or Emission(self.settings.source_center), sources)
            except Exception:
                self.faulted = True
                self.projector.ready = False
                raise

    def _prepare_sources(self, sources):
        data = pack_sources(sources)
        if data != self._source_data:
            self._source_data = data
            # the table as a device field (the reference's sourceTable texture), for
            # single-pass dispatch of the table forms
            with self.device.ordered():
                self._source_table = torch.tensor(list(data) + [0.0] * (128 - len(data)), dtype=torch.float32,
                                                  device=self.device.device)
            if self._multi_velocity is None:
                self._multi_velocity = self.device.kernel('multi_advect_velocity.glsl')
                self._multi_scalar = self.device.kernel('multi_advect_scalar.glsl')
        self._source_count = len(sources)

    def _fill_sources(self, emission, emitters):
        src = self._sources
        s = self.settings
        if emitters is not None:
            src.count = len(emitters)
            for i, v in enumerate(self._source_data):
                src.table[i] = v
        else:
            src.count = -1
            src.single_solid_profile = int(s.source_profile == "SOLID")
            src.single_center = N.f3(*s.source_center)
            src.single_start = N.f3(*emission.start)
            src.single_radius = s.source_radius
            src.single_jet = N.f3(*emission.velocity)
            src.single_coupling = emission.coupling
        return src

    def _mark(self, name):
        if self.pass_timer is not None:
            self.pass_timer.mark(name)

    def _step(self, dt, emission, emitters=None, clock=None):
        """One step with the time step ``dt``, or, with ``clock``, the device
        float clock[0] (the ``ffx_*_dt`` forms of the passes)."""
        s = self.settings
        dev = self.device
        gp = C.byref(self._g)
        sp = C.byref(self._solids)
        st = dev.s
        src = self._fill_sources(emission, emitters)
        corrected_v = s.velocity_advection == "MACCORMACK"
        vel = [ptr(f) for f in self._velocity]
        dtp = ptr(clock[0:1]) if clock is not None else None
        if clock is None and self._clock_live:
            # a host step after device steps: fold the device time into the host time
            self.time = self.time
            self._clock_live = False
        self._mark('start')
        if corrected_v:
            self.detail.transport_velocity(self._velocity, dt, dtp)
            pred = [ptr(f) for f in self.detail.face_predictor]
            self._mark('velocity_predictor')
        else:
            pred = [None, None, None]
        proj = self.projector
        confine = s.vorticity_strength > 0
        # with confinement the wall condition waits for the projection, as in
        # the reference (confinement reads the provisional, unwalled faces)
        dev.call('ffx_advect_velocity_dt' if dtp is not None else 'ffx_advect_velocity_trace', gp, sp, self._storage,
                 *vel, *pred, dtp if dtp is not None else dt, int(corrected_v), s.velocity_blend, C.byref(src),
                 ptr(self._front), ptr(self._temperature), s.thermal_lift, s.density_weight, int(not confine),
                 *[ptr(b) for b in proj.bounded], self.detail.face_traces() if corrected_v else None, st)
        self._mark('velocity_transport')
        # The old velocity is consumed: the corrected field is written over it.
        if confine:
            self.detail.confine(proj.bounded, self._velocity, dt, s.vorticity_strength, s.vorticity_limit)
            self._mark('confinement')
            proj.project(self._velocity, self._velocity, dt)
        elif clock is not None:
            proj.project_bounded_device(self._velocity, clock)
        else:
            proj.project_bounded(self._velocity, dt)
        self._mark('projection')
        corrected_s = s.scalar_advection == "MACCORMACK"
        fields = [self._front, self._temperature]
        if self.combustion is not None:
            fields.append(self.combustion.fuel)
        if corrected_s:
            preds, revs = self.detail.transport_many(fields, self._velocity, dt, dtp)
            self._mark('scalar_predictor_reverse')
        else:
            preds = revs = fields
        outs = [self._back, self._temperature_back]
        density_target = s.source_rate if s.density_mode == "TARGET" else -1.0
        heat_target = s.heat_source_rate if s.heat_mode == "TARGET" else -1.0
        chans = [N.FfxScalarChannel(ptr(fields[0]), ptr(preds[0]), ptr(revs[0]), ptr(outs[0]), s.source_rate,
                                    s.dissipation, density_target, 0, 0),
                 N.FfxScalarChannel(ptr(fields[1]), ptr(preds[1]), ptr(revs[1]), ptr(outs[1]), s.heat_source_rate,
                                    s.cooling, heat_target, 1, int(s.heat_mode == "TARGET"))]
        if self.combustion is not None:
            # fuel: third channel, additive emission (fuel_rate column / fuel_source_rate), no decay
            chans.append(N.FfxScalarChannel(ptr(fields[2]), ptr(preds[2]), ptr(revs[2]), ptr(self.combustion.spare),
                                            s.fuel_source_rate, 0.0, -1.0, 2, 0))
        arr = (N.FfxScalarChannel * len(chans))(*chans)
        decisions = self.detail.cell_decisions() if corrected_s else None
        if decisions is not None:
            # the reverse pass decided the corrections (ffx_scalar_reverse_ok)
            dev.call('ffx_advect_scalars_ok', gp, sp, self._storage, *[ptr(f) for f in self._velocity],
                     0.0 if dtp is not None else dt, dtp, int(corrected_s), C.byref(src), len(chans), arr,
                     ptr(self._maxima), self.detail.cell_traces(), decisions, st)
        else:
            dev.call('ffx_advect_scalars_dt' if dtp is not None else 'ffx_advect_scalars_trace', gp, sp,
                     self._storage, *[ptr(f) for f in self._velocity], dtp if dtp is not None else dt,
                     int(corrected_s), C.byref(src), len(chans), arr, ptr(self._maxima),
                     self.detail.cell_traces() if corrected_s else None, st)
        self._mark('scalar_transport')
        self._front, self._back = self._back, self._front
        self._temperature, self._temperature_back = self._temperature_back, self._temperature
        if self.combustion is not None:
            c = self.combustion
            c.fuel, c.spare = c.spare, c.fuel
            c.react(self, dt)
            self._mark('combustion')
        if clock is None:
            self.time += dt
        self.steps += 1

    def scalar_maxima(self):
        """max |density|, |temperature| of the last step (one readback)."""
        return [float(v) for v in self.device.fetch(self._maxima[0:2])]

    def preview_field(self, channel):
        if channel == 'COLLISION':
            if self.solids is None:
                raise ValueError('Add a collider and Reset for collision display')
            return self.solids.mask
        if channel in {'FUEL', 'FLAME'}:
            if self.combustion is None:
                raise ValueError('Enable combustion and Reset for fuel/flame display')
            return self.combustion.fuel if channel == 'FUEL' else self.combustion.flame
        return self.temperature if channel == 'TEMPERATURE' else self.density

    def close(self):
        if self.projector is not None:
            self.projector.close()
        self.projector = None
        if self.detail is not None:
            self.detail.close()
        self.detail = None
        if self.combustion is not None:
            self.combustion.close()
        self.combustion = None
        super().close()
        if self.solids is not None:
            self.solids.close()
        self.solids = None
