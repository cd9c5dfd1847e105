"""Geometric V-cycle pressure solver for evenly coarsenable grids.

Drop-in for FluxFX ``fluxfx/backend/multigrid.py:6-106``: weighted Jacobi
(omega = 2/3), rediscretised Neumann Laplacian per level, 2x2x2 averaging,
clamped trilinear prolongation, coarse levels solved with dt = 1, and the 4^3
closed-form pseudoinverse on the coarsest level. Residual and restriction run
as one fused pass. Extensions (``PressureSettings``): sweep counts, a level cap
(the coarsest level up to 512 cells then uses the same closed-form inverse in
FP64), and cycling to a relative max-norm tolerance.
"""
import ctypes as C
from math import prod

import torch

from .. import _native as N
from ..physics.coarse_pressure import MAX_DIRECT_CELLS, neumann_inverse
from .device import KernelHandle, ptr
from .pressure import PressureProjector


def hierarchy_shapes(shape, max_levels=0):
    """Halve while all axes are even and the smallest is >= 8; optional level cap."""
    result = [tuple(shape)]
    while min(shape) >= 8 and all(n % 2 == 0 for n in shape):
        if max_levels and len(result) >= max_levels:
            break
        shape = tuple(n // 2 for n in shape)
        result.append(shape)
    return result


def use_multigrid(grid, settings):
    return (len(hierarchy_shapes(grid.shape)) > 1 and
            (settings.pressure_solver == "MULTIGRID" or
             (settings.pressure_solver == "AUTO" and min(grid.shape) >= 16)))


class MultigridPressureProjector(PressureProjector):
    def __init__(self, grid, settings=None, device=None):
        super().__init__(grid, settings, device)
        s = self.settings
        self.levels = []
        self.coarse_kernel = self.coarse_matrix = None
        shapes = hierarchy_shapes(grid.shape, s.mg_max_levels)
        self.residual_kernel = KernelHandle('mg_residual.glsl')
        self.restrict_kernel = KernelHandle('mg_restrict.glsl')
        self.prolong_kernel = KernelHandle('mg_prolong.glsl')
        dev = self.device
        for i, shape in enumerate(shapes):
            self.levels.append({
                'shape': shape, 'inv': tuple(n / e for n, e in zip(shape, grid.extent)),
                'p': self.pressure if i == 0 else dev.texture(shape),
                'q': self.spare if i == 0 else dev.texture(shape),
                'rhs': self.before if i == 0 else dev.texture(shape),
                'residual': None})
        coarsest = shapes[-1]
        if len(shapes) > 1 and s.coarse_solver == 'DIRECT' and (
                coarsest == (4, 4, 4) or (s.mg_max_levels and prod(coarsest) <= MAX_DIRECT_CELLS)):
            inv = neumann_inverse(coarsest, grid.extent)
            self.coarse_matrix = torch.as_tensor(inv, dtype=torch.float64).to(dev.device)
            self.coarse_kernel = KernelHandle('coarse_pressure.glsl')
        self.pre_sweeps = s.mg_pre_sweeps or 3
        self.post_sweeps = s.mg_post_sweeps or 3
        self.last_cycles = 0
        self.last_coarse_solves = 0
        self._rmax = torch.zeros(2, dtype=torch.float32, device=dev.device)

    @property
    def allocated_bytes(self):
        extra = 4 * sum(3 * prod(v['shape']) for v in self.levels[1:])
        return super().allocated_bytes + extra + (8 * self.coarse_matrix.numel() if self.coarse_matrix is not None else 0)

    def reset(self):
        super().reset()
        self.last_cycles = 0
        for level in self.levels[1:]:
            for name in ('p', 'q', 'rhs'):
                level[name].zero_()

    def _n3(self, level):
        return N.n3(*level['shape'])

    def _inv3(self, level):
        return N.f3(*level['inv'])

    def smooth(self, level, dt, count):
        s = self.device.s
        for _ in range(count):
            self.device.call('ffx_jacobi', self._n3(level), self._inv3(level), None, ptr(level['p']),
                             ptr(level['rhs']), dt, 2.0 / 3.0, ptr(level['q']), s)
            level['p'], level['q'] = level['q'], level['p']
            self.last_iterations += 1

    def cycle(self, index, dt):
        level = self.levels[index]
        s = self.device.s
        if index == len(self.levels) - 1:
            if self.coarse_matrix is not None:
                self.device.call('ffx_direct_solve', prod(level['shape']), ptr(self.coarse_matrix),
                                 ptr(level['rhs']), dt, ptr(level['p']), s)
                self.last_coarse_solves += 1
            else:
                self.smooth(level, dt, 80)
            return
        self.smooth(level, dt, self.pre_sweeps)
        coarse = self.levels[index + 1]
        self.device.call('ffx_mg_residual_restrict', self._n3(level), self._inv3(level), ptr(level['p']),
                         ptr(level['rhs']), dt, ptr(coarse['rhs']), s)
        coarse['p'].zero_()
        self.cycle(index + 1, 1.0)
        self.device.call('ffx_mg_prolong', self._n3(level), ptr(level['p']), ptr(coarse['p']), ptr(level['q']), s)
        level['p'], level['q'] = level['q'], level['p']
        self.smooth(level, dt, self.post_sweeps)

    def _residual_max(self, dt):
        level = self.levels[0]
        self.device.call('ffx_mg_residual_max', self._n3(level), self._inv3(level), ptr(level['p']),
                         ptr(level['rhs']), dt, ptr(self._rmax[0:1]), self.device.s)
        return float(self.device.fetch(self._rmax[0]))

    def _run_cycles(self, dt, budget):
        s = self.settings
        self.last_cycles = 0
        if s.pressure_tolerance <= 0:
            for _ in range(budget):
                self.cycle(0, dt)
                self.last_cycles += 1
            return
        self.device.call('ffx_max_abs', self.before.numel(), N.FFX_F32, ptr(self.before), ptr(self._rmax[1:2]),
                         self.device.s)
        scale = float(self.device.fetch(self._rmax[1])) / dt
        if scale == 0:
            self.levels[0]['p'].zero_()
            return
        while self.last_cycles < s.pressure_max_cycles and self._residual_max(dt) > s.pressure_tolerance * scale:
            self.cycle(0, dt)
            self.last_cycles += 1

    def solve_pressure(self, dt, previous_dt):
        self.last_coarse_solves = 0
        if len(self.levels) == 1:
            self.last_cycles = 0
            super().solve_pressure(dt, previous_dt)
            return
        if previous_dt != dt:
            self.pressure.zero_()
        self.levels[0]['p'], self.levels[0]['q'] = self.pressure, self.spare
        self.last_iterations = 0
        self._run_cycles(dt, self.settings.pressure_cycles)
        self.pressure, self.spare = self.levels[0]['p'], self.levels[0]['q']

    def metrics(self):
        return super().metrics() | {
            'solver': 'MULTIGRID' if self.last_cycles else 'JACOBI_FALLBACK',
            'v_cycles': self.last_cycles, 'direct_coarse_solves': self.last_coarse_solves,
            'levels': [v['shape'] for v in self.levels],
            'iteration_meaning': 'Jacobi smoothing passes summed across all levels'}

    def close(self):
        self.levels = []
        self.coarse_kernel = self.coarse_matrix = None
        super().close()
