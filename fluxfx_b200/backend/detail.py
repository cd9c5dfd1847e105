"""MacCormack predictor/reverse passes (scalar and face).

Drop-in for FluxFX ``fluxfx/backend/detail.py:5-54`` (``transport``,
``transport_velocity``). The scalar passes transport up to three channels that
share one backtrace in a single launch (``transport_many``). Vorticity
confinement (``confine``) belongs to the combustion/fire configuration and is
not part of this build.
"""
import ctypes as C
from math import prod

import torch

from .. import _native as N
from .device import ptr, solids_struct
from .mac import VELOCITY_NAMES


class DetailPasses:
    def __init__(self, grid, device, dtype=torch.float32):
        self.grid = grid
        self.device = device
        self.dtype = dtype
        self._storage = N.FFX_F32 if dtype == torch.float32 else N.FFX_BF16
        self._g = N.grid_struct(grid.shape, grid.extent)
        self._solids = solids_struct(device)
        self.predictor = self.reverse = None
        self.predictors = self.reverses = None
        self.face_predictor = None
        self.curl = None
        # departure points of the predictor passes, reused by the correction passes
        # (faces only where both passes form the same start point at every face)
        self.reuse_traces = True
        self.face_trace = None
        self.cell_trace = None
        self.cell_ok = None       # the reverse pass's correction decisions (uint8 per cell)
        self._face_reuse = N.face_starts_match(grid.shape, grid.extent)

    @property
    def allocated_bytes(self):
        size = 2 if self.dtype == torch.bfloat16 else 4
        scalar = sum(t.numel() for t in (self.predictors or []) + (self.reverses or [])) * size
        faces = size * sum(prod(s) for s in self.grid.face_shapes) if self.face_predictor is not None else 0
        traces = sum(4 * t.numel() for t in (self.face_trace or [])) + (
            4 * self.cell_trace.numel() if self.cell_trace is not None else 0) + (
            self.cell_ok.numel() if self.cell_ok is not None else 0)
        return scalar + faces + traces + (self.curl.numel() * 4 if self.curl is not None else 0)

    def _ensure_scalar(self, count):
        if self.predictors is None or len(self.predictors) < count:
            self.predictors = [self.device.texture(self.grid.shape, dtype=self.dtype) for _ in range(count)]
            self.reverses = [self.device.texture(self.grid.shape, dtype=self.dtype) for _ in range(count)]
            self.predictor, self.reverse = self.predictors[0], self.reverses[0]

    def transport_many(self, fields, velocities, dt, dt_device=None):
        """Predictor (+dt) and reverse (-dt) of up to three scalars; returns
        (predictors, reverses) tensors aligned with ``fields``. ``dt_device``:
        a device float holding dt (``ffx_*_dt`` entry points) instead of ``dt``."""
        count = len(fields)
        self._ensure_scalar(count)
        vel = [ptr(velocities[name]) if isinstance(velocities, dict) else ptr(velocities[i])
               for i, name in enumerate(VELOCITY_NAMES)]
        ins = (C.c_void_p * count)(*[f.data_ptr() for f in fields])
        preds = (C.c_void_p * count)(*[p.data_ptr() for p in self.predictors[:count]])
        revs = (C.c_void_p * count)(*[r.data_ptr() for r in self.reverses[:count]])
        gp, sp, s = C.byref(self._g), C.byref(self._solids), self.device.s
        if self.reuse_traces and self.cell_trace is None:
            self.cell_trace = torch.empty(3 * prod(self.grid.shape), dtype=torch.float32, device=self.device.device)
        trace = ptr(self.cell_trace) if self.reuse_traces else None
        if self.reuse_traces:
            # the reverse pass also decides the final pass's corrections (cell_decisions)
            if self.cell_ok is None:
                nx, ny, nz = self.grid.shape
                self.cell_ok = torch.empty((nz, ny, nx), dtype=torch.uint8, device=self.device.device)
            if dt_device is not None:
                self.device.call('ffx_scalar_transport_dt', gp, sp, self._storage, *vel, dt_device, 1.0, count, ins,
                                 preds, trace, s)
            else:
                self.device.call('ffx_scalar_transport_trace', gp, sp, self._storage, *vel, dt, count, ins, preds,
                                 trace, s)
            self.device.call('ffx_scalar_reverse_ok', gp, sp, self._storage, *vel, 0.0 if dt_device is not None
                             else -dt, dt_device, count, preds, revs, trace, ptr(self.cell_ok), s)
        elif dt_device is not None:
            self.device.call('ffx_scalar_transport_dt', gp, sp, self._storage, *vel, dt_device, 1.0, count, ins, preds,
                             trace, s)
            self.device.call('ffx_scalar_transport_dt', gp, sp, self._storage, *vel, dt_device, -1.0, count, preds,
                             revs, None, s)
        else:
            self.device.call('ffx_scalar_transport_trace', gp, sp, self._storage, *vel, dt, count, ins, preds, trace,
                             s)
            self.device.call('ffx_scalar_transport', gp, sp, self._storage, *vel, -dt, count, preds, revs, s)
        return self.predictors[:count], self.reverses[:count]

    def transport(self, field, velocities, dt):
        preds, revs = self.transport_many([field], velocities, dt)
        return {'predictorField': preds[0], 'reverseField': revs[0]}

    def transport_velocity(self, fields, dt, dt_device=None):
        """Predict each signed face component; the reverse sample is fused with the correction."""
        if self.face_predictor is None:
            self.face_predictor = [self.device.texture(s, dtype=self.dtype) for s in self.grid.face_shapes]
        if self.reuse_traces and self._face_reuse and self.face_trace is None:
            # x, y, z of each departure point, plus (16-bit storage) the unrounded sample
            # departure point, (BF16) the unrounded sample, start velocity
            planes = 6 if self.dtype == torch.float32 else 7
            self.face_trace = [torch.empty(planes * prod(s), dtype=torch.float32, device=self.device.device)
                               for s in self.grid.face_shapes]
        name, step = ('ffx_face_predictor_dt', dt_device) if dt_device is not None else ('ffx_face_predictor_trace', dt)
        self.device.call(name, C.byref(self._g), C.byref(self._solids), self._storage, *[ptr(f) for f in fields],
                         step, *[ptr(p) for p in self.face_predictor], self.face_traces(), self.device.s)

    def face_traces(self):
        """The face departure points as a C array of three pointers, or NULL."""
        if not (self.reuse_traces and self._face_reuse and self.face_trace is not None):
            return None
        return (C.c_void_p * 3)(*[t.data_ptr() for t in self.face_trace])

    def cell_traces(self):
        return ptr(self.cell_trace) if (self.reuse_traces and self.cell_trace is not None) else None

    def cell_decisions(self):
        """The reverse pass's correction decisions (ffx_scalar_reverse_ok), or NULL."""
        return ptr(self.cell_ok) if (self.reuse_traces and self.cell_ok is not None) else None

    def confine(self, fields, outputs, dt, strength, limit):
        """Vorticity confinement (``backend/detail.py:39-49``): cell curl
        (omega, |omega|) into ``self.curl``, then every face of ``outputs`` =
        ``fields`` + dt * confinement force."""
        if self.curl is None:
            nx, ny, nz = self.grid.shape
            self.curl = torch.zeros((nz, ny, nx, 4), dtype=torch.float32, device=self.device.device)
        gp, s = C.byref(self._g), self.device.s
        self.device.call('ffx_curl', gp, self._storage, *[ptr(f) for f in fields], ptr(self.curl), s)
        self.device.call('ffx_confine', gp, self._storage, ptr(self.curl), *[ptr(f) for f in fields], dt, strength,
                         limit, *[ptr(o) for o in outputs], s)

    def close(self):
        self.predictor = self.reverse = self.predictors = self.reverses = None
        self.face_predictor = None
        self.face_trace = self.cell_trace = None
        self.curl = None
