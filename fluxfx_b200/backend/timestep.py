"""Device max reductions for the CFL timestep.

Drop-in for FluxFX ``fluxfx/backend/timestep.py:6-57``: five max-abs reductions
(U, V, W, density, temperature; NaN/Inf count as 3.4e38), one readback of five
floats, then ``choose_timestep``. ``cfl_dt`` is the simpler rule
dt = min(max_dt, cfl * min(h) / max|u|).
"""
from math import isfinite, prod

import torch

from .. import _native as N
from ..physics.timestep import cfl_timestep, choose_timestep
from .device import ptr


class AdaptiveTimestep:
    def __init__(self, grid, device):
        self.device = device
        self.grid = grid
        self._out = torch.zeros(5, dtype=torch.float32, device=device.device)

    @property
    def allocated_bytes(self):
        return 4 * 5

    def bounds(self, solver):
        fields = (*solver._velocity, solver.density, solver.temperature)
        for k, f in enumerate(fields):
            code = N.FFX_F32 if f.dtype == torch.float32 else N.FFX_BF16
            self.device.call('ffx_max_abs', f.numel(), code, ptr(f), ptr(self._out[k:k + 1]), self.device.s)
        maxima = [float(v) for v in self.device.fetch(self._out)]
        if any(not isfinite(v) or v >= 1e30 for v in maxima):
            raise RuntimeError('Nonfinite or excessive field values; reset simulation')
        return maxima

    def select(self, solver, max_dt, cfl, emission=None, sources=None):
        u, v, w, density, temperature = self.bounds(solver)
        motions = [s.motion for s in sources] if sources is not None else ([emission] if emission is not None else [])
        for motion in motions:
            if motion.coupling > 0:
                u, v, w = (max(cur, abs(t)) for cur, t in zip((u, v, w), motion.velocity))
        h = self.grid.cell_size
        rate = sum(speed / spacing for speed, spacing in zip((u, v, w), h))
        st = solver.settings
        accel = (st.thermal_lift * temperature + st.density_weight * density) / h[2]
        if st.vorticity_strength > 0:
            accel += st.vorticity_limit * sum(1 / spacing for spacing in h)
        if st.turbulence_strength > 0:
            accel += min(st.turbulence_strength, st.turbulence_limit) * sum(1 / spacing for spacing in h)
        quantized = st.timestep_policy == "QUANTIZED" or (st.timestep_policy == "AUTO"
                                                          and not solver.projector.uses_impulse)
        dt = choose_timestep(max_dt, cfl, rate, accel, quantized=quantized)
        return {'dt': dt, 'max_dt': max_dt, 'target': cfl, 'rate_bound': rate, 'acceleration_rate_bound': accel,
                'estimated_courant': rate * dt + accel * dt * dt,
                'policy': 'QUANTIZED' if quantized else 'CONTINUOUS', 'max_abs_velocity': [u, v, w],
                'mode': 'ADAPTIVE'}

    def cfl_dt(self, solver, max_dt, cfl):
        u, v, w = self.bounds(solver)[:3]
        return cfl_timestep(max_dt, cfl, self.grid.cell_size, max(u, v, w))

    def close(self):
        self._out = None
