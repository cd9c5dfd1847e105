"""Closed-box (optionally masked) pressure projection, weighted-Jacobi solver.

Drop-in for FluxFX ``fluxfx/backend/pressure.py:9-120``: same state machine
(impulse storage q = dt p, dt-ratio rescale of the warm start, cold-start
iteration multiplier) and the same attributes. Walls + divergence and
gradient + post-divergence run as two fused native passes; a device whose
``mask`` attribute is set (``SolidDevice``) switches every pass to its masked
form.
"""
import ctypes as C
from math import ceil, prod

import torch

from .. import _native as N
from ..physics.config import validate_dt
from ..physics.pressure import PressureSettings
from .device import CudaDevice, KernelHandle, ptr, solids_struct


class PressureProjector:
    def __init__(self, grid, settings=None, device=None):
        self.grid = grid
        self.settings = settings or PressureSettings()
        self.device = device or CudaDevice()
        self.inv_cell = tuple(1 / h for h in grid.cell_size)
        self._g = N.grid_struct(grid.shape, grid.extent)
        self._field_dtype = torch.bfloat16 if self.settings.storage == 'BF16' else torch.float32
        self._storage = N.FFX_F32 if self._field_dtype == torch.float32 else N.FFX_BF16
        self._mask = getattr(self.device, 'mask', None)
        self._solids = solids_struct(self.device)
        self.wall = KernelHandle('pressure_walls.glsl')
        self.divergence = KernelHandle('pressure_divergence.glsl')
        self.jacobi = KernelHandle('pressure_jacobi.glsl')
        self.gradient = KernelHandle('pressure_gradient.glsl')
        self.scale = KernelHandle('pressure_scale.glsl')
        dev = self.device
        self.bounded = [dev.texture(s, dtype=self._field_dtype) for s in grid.face_shapes]
        self.pressure = dev.texture(grid.shape)
        self.spare = dev.texture(grid.shape)
        self.before = dev.texture(grid.shape)
        self.after = dev.texture(grid.shape)
        self._scalars = torch.zeros(8, dtype=torch.float32, device=dev.device)   # device-side maxima
        # warm-start extrapolation: the previous solve's pressure per unit time
        # (allocated on first use) and whether it holds one
        self._history = None
        self._history_valid = False
        self._host_clock = None
        # quadratic form: two stored solves (newest first), their count, and the
        # previous dt in two alternating device slots
        self._histories = None
        self._history_count = 0
        self._dprev = None
        self.ready = False
        self.last_dt = None
        self.last_iterations = 0

    # -------------------------------------------------------------- helpers
    @property
    def _gp(self):
        return C.byref(self._g)

    @property
    def _sp(self):
        return C.byref(self._solids)

    @property
    def _n3(self):
        return N.n3(*self.grid.shape)

    @property
    def _inv3(self):
        return N.f3(*self.inv_cell)

    def _mask_ptr(self):
        return ptr(self._mask)

    @property
    def uses_impulse(self):
        ws = self.settings.pressure_warm_start
        return ws == "IMPULSE" or (ws == "AUTO" and len(getattr(self, "levels", ())) > 1)

    @property
    def allocated_bytes(self):
        face = 2 if self._field_dtype == torch.bfloat16 else 4
        return 4 * 4 * prod(self.grid.shape) + face * sum(prod(s) for s in self.grid.face_shapes)

    def reset(self):
        self.ready = False
        self.last_dt = None
        self.last_iterations = 0
        self._history_valid = False
        self._history_count = 0
        for t in (self.pressure, self.spare, self.before, self.after, *self.bounded):
            t.zero_()

    def enforce_walls(self, fields, outputs):
        self.device.call('ffx_walls', self._gp, self._sp, self._storage, *[ptr(f) for f in fields],
                         *[ptr(o) for o in outputs], self.device.s)

    def compute_divergence(self, fields, target):
        self.device.call('ffx_divergence', self._gp, self._sp, self._storage, *[ptr(f) for f in fields],
                         ptr(target), self.device.s)

    # ------------------------------------------------------------ projection
    def project(self, fields, outputs, dt):
        """Walls + divergence, pressure solve, gradient correction, divergence after."""
        validate_dt(dt)
        self.device.call('ffx_walls_divergence', self._gp, self._sp, self._storage, *[ptr(f) for f in fields],
                         *[ptr(b) for b in self.bounded], ptr(self.before), self.device.s)
        self._finish(outputs, dt)

    def project_bounded(self, outputs, dt):
        """Projection of velocity already written to ``self.bounded`` with the
        wall condition applied (the fused velocity pass does that)."""
        validate_dt(dt)
        self.compute_divergence(self.bounded, self.before)
        self._finish(outputs, dt)

    def project_bounded_device(self, outputs, clock):
        """``project_bounded`` with the time step on the device: ``clock`` is the
        solver's float32 device pair (dt, previous dt). Needs the impulse form
        (the solve is dt-independent; only the warm start's dt / previous dt
        rescaling reads the clock, on the device)."""
        if not self.uses_impulse:
            raise ValueError('Device time steps need the impulse pressure form (multigrid or colliders)')
        self.compute_divergence(self.bounded, self.before)
        self.ready = False
        previous = self.last_dt is not None
        if previous and self.extrapolation_beta() > 0:
            self._extrapolate(clock)
        elif previous:
            self.device.call('ffx_scale_by_ratio', self.pressure.numel(), ptr(self.pressure), ptr(clock),
                             self.device.s)
        else:
            self._history_valid = False
            self._history_count = 0
        self.solve_pressure(1.0, 1.0 if previous else None)
        self._gradient(outputs, 1.0)
        self.last_dt = clock        # the previous dt now lives on the device (clock[1] after the step)
        self.ready = True

    def previous_dt(self):
        """The last projection's dt on the host (one readback after device steps)."""
        if self.last_dt is None or isinstance(self.last_dt, float):
            return self.last_dt
        return float(self.device.fetch(self.last_dt[1]))

    def _gradient(self, outputs, solve_dt):
        links = self.gradient_links()
        if self._field_dtype == torch.bfloat16:
            # BF16 storage: also the divergence of the FP32 result before rounding
            if getattr(self, 'after_fp32', None) is None:
                self.after_fp32 = self.device.texture(self.grid.shape)
            self.device.call('ffx_gradient_ex', self._gp, self._sp, self._storage, *[ptr(b) for b in self.bounded],
                             ptr(self.pressure), solve_dt, *[ptr(o) for o in outputs], ptr(self.after),
                             ptr(self._scalars[0:3]), ptr(links) if links is not None else None,
                             ptr(self.after_fp32), self.device.s)
        elif links is not None:
            self.device.call('ffx_gradient_links', self._gp, self._sp, self._storage, *[ptr(b) for b in self.bounded],
                             ptr(self.pressure), solve_dt, *[ptr(o) for o in outputs], ptr(self.after),
                             ptr(self._scalars[0:3]), ptr(links), self.device.s)
        else:
            self.device.call('ffx_gradient', self._gp, self._sp, self._storage, *[ptr(b) for b in self.bounded],
                             ptr(self.pressure), solve_dt, *[ptr(o) for o in outputs], ptr(self.after),
                             ptr(self._scalars[0:3]), self.device.s)

    def _finish(self, outputs, dt):
        self.ready = False
        previous_dt, self.last_dt = self.previous_dt(), None
        impulse = self.uses_impulse
        solve_dt = 1.0 if impulse else dt
        previous_solve_dt = (1.0 if previous_dt is not None else None) if impulse else previous_dt
        if impulse and previous_dt is not None and self.extrapolation_beta() > 0:
            if self._host_clock is None:
                self._host_clock = torch.zeros(2, dtype=torch.float32, device=self.device.device)
            self._host_clock.copy_(torch.tensor([dt, previous_dt], dtype=torch.float32))
            self._extrapolate(self._host_clock)
        elif impulse and previous_dt is not None and abs(dt / previous_dt - 1.0) > 1e-6:
            # The incremental pressure force scales with physical dt: rescale the
            # guess (in place, so the pressure keeps its buffer from step to step).
            self.device.call('ffx_scale', self.pressure.numel(), ptr(self.pressure), dt / previous_dt,
                             ptr(self.pressure), self.device.s)
        if previous_dt is None:
            self._history_valid = False
            self._history_count = 0
        self.solve_pressure(solve_dt, previous_solve_dt)
        self._gradient(outputs, solve_dt)
        self.last_dt = dt
        self.ready = True

    def extrapolation_beta(self):
        """beta of the warm start extrapolated in time, or 0 where the solve
        does not start from the previous pressure."""
        return 0.0

    def _extrapolate(self, clock):
        """Start the next solve from the last two pressures extrapolated in
        time (ffx_extrapolate_pressure; ``clock`` = device (dt, previous dt)).
        The first call after a cold solve has one pressure only and applies the
        ratio rule."""
        if self.settings.warm_start_order == 2:
            if self._histories is None:
                self._histories = [self.device.texture(self.grid.shape) for _ in range(2)]
                self._dprev = torch.zeros(2, dtype=torch.float32, device=self.device.device)
            newest, oldest = self._histories
            k = self._history_count
            self.device.call('ffx_extrapolate_pressure2', self.pressure.numel(), ptr(self.pressure), ptr(newest),
                             ptr(oldest), ptr(clock), ptr(self._dprev[(k + 1) % 2:(k + 1) % 2 + 1]),
                             ptr(self._dprev[k % 2:k % 2 + 1]), float(self.extrapolation_beta()), min(k, 2),
                             self.device.s)
            # the pass wrote the last solve over the oldest: it is now the newest
            self._histories = [oldest, newest]
            self._history_count = k + 1
            return
        if self._history is None:
            self._history = self.device.texture(self.grid.shape)
        self.device.call('ffx_extrapolate_pressure', self.pressure.numel(), ptr(self.pressure), ptr(self._history),
                         ptr(clock), float(self.extrapolation_beta()), 0 if self._history_valid else 1,
                         self.device.s)
        self._history_valid = True

    def gradient_links(self):
        """Level-0 link bytes of the collider mask (ffx_graph_links) for the
        gradient pass, or None: the pass then tests the mask itself."""
        return None

    def solve_pressure(self, dt, previous_dt):
        if previous_dt != dt:
            self.pressure.zero_()
        # Jacobi smooths across cells: scale the work with resolution squared.
        scaled = ceil(self.settings.pressure_iterations * max(1.0, (max(self.grid.shape) / 64) ** 2))
        multiplier = self.settings.pressure_cold_multiplier if previous_dt != dt else 1
        self.last_iterations = min(4096, scaled * multiplier)
        omega = self.settings.pressure_relaxation
        for _ in range(self.last_iterations):
            self.device.call('ffx_jacobi', self._n3, self._inv3, self._mask_ptr(), ptr(self.pressure),
                             ptr(self.before), dt, omega, ptr(self.spare), self.device.s)
            self.pressure, self.spare = self.spare, self.pressure

    # ------------------------------------------------------------- diagnostics
    def velocity_maxima(self):
        """max |u|, |v|, |w| of the last corrected velocity (one readback)."""
        return [float(v) for v in self.device.fetch(self._scalars[0:3])]

    def divergence_summary(self):
        """FP64 statistics of ``before``/``after`` on the device (one readback)."""
        with self.device.ordered():
            return self._divergence_summary()

    def _divergence_summary(self):
        n = self.before.numel()
        ws = torch.empty(int(self.device.lib.ffx_divergence_stats_workspace(n)) // 8 + 1,
                         dtype=torch.float64, device=self.device.device)
        out = torch.empty(8, dtype=torch.float64, device=self.device.device)
        self.device.call('ffx_divergence_stats', n, ptr(self.before), ptr(self.after), ptr(out), ptr(ws),
                         ws.numel() * 8, self.device.s)
        b2, a2, mb, ma, sb, sa, count, _ = out.cpu().tolist()
        rms_b, rms_a = (b2 / count) ** 0.5, (a2 / count) ** 0.5
        ratio = rms_a / rms_b if rms_b > 0 else (0.0 if rms_a == 0 else None)
        out = {"rms_before": rms_b, "rms_after": rms_a, "ratio": ratio, "max_before": mb, "max_after": ma,
               "mean_before": sb / count, "mean_after": sa / count,
               "rel_div_inf": (ma / mb) if mb > 0 else 0.0}
        exact = getattr(self, 'after_fp32', None)
        if exact is not None:
            # BF16 storage: rel_div_inf is of the stored (rounded) faces; this one is
            # of the projection's FP32 result before rounding, the solve's own measure
            ma32 = float(exact.abs().max())
            out.update(max_after_fp32=ma32, rel_div_inf_fp32=(ma32 / mb) if mb > 0 else 0.0)
        return out

    def metrics(self):
        """Explicit synchronous readback; never invoked by the step itself."""
        if not self.ready:
            raise RuntimeError("Take a simulation step before measuring projection")
        return self.divergence_summary() | {
            "solver": "JACOBI",
            "pressure_storage": "IMPULSE" if self.uses_impulse else "LEGACY",
            "iterations": self.last_iterations,
            "base_iterations_at_64": self.settings.pressure_iterations,
            "relaxation": self.settings.pressure_relaxation,
            "boundary": "closed_free_slip", "units": "1/s",
            "before_stage": "after_wall_conditioning"}

    def close(self):
        self.ready = False
        self.last_dt = None
        self.bounded = None
        self.pressure = self.spare = self.before = self.after = None
