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

    @property
    def allocated_bytes(self):
        size = 2 if self.dtype == torch.bfloat16 else 4
        scalar = sum(t.numel() for t in (self.predictors or []) + (self.reverses or [])) * size
        faces = size * sum(prod(s) for s in self.grid.face_shapes) if self.face_predictor is not None else 0
        return scalar + faces + (self.curl.numel() * 4 if self.curl is not None else 0)

    def _ensure_scalar(self, count):
        if self.predictors is None or len(self.predictors) < count:
            self.predictors = [self.device.texture(self.grid.shape, dtype=self.dtype) for _ in range(count)]
            self.reverses = [self.device.texture(self.grid.shape, dtype=self.dtype) for _ in range(count)]
            self.predictor, self.reverse = self.predictors[0], self.reverses[0]

    def transport_many(self, fields, velocities, dt):
        """Predictor (+dt) and reverse (-dt) of up to three scalars; returns
        (predictors, reverses) tensors aligned with ``fields``."""
        count = len(fields)
        self._ensure_scalar(count)
        vel = [ptr(velocities[name]) if isinstance(velocities, dict) else ptr(velocities[i])
               for i, name in enumerate(VELOCITY_NAMES)]
        ins = (C.c_void_p * count)(*[f.data_ptr() for f in fields])
        preds = (C.c_void_p * count)(*[p.data_ptr() for p in self.predictors[:count]])
        revs = (C.c_void_p * count)(*[r.data_ptr() for r in self.reverses[:count]])
        gp, sp, s = C.byref(self._g), C.byref(self._solids), self.device.s
        self.device.call('ffx_scalar_transport', gp, sp, self._storage, *vel, dt, count, ins, preds, s)
        self.device.call('ffx_scalar_transport', gp, sp, self._storage, *vel, -dt, count, preds, revs, s)
        return self.predictors[:count], self.reverses[:count]

    def transport(self, field, velocities, dt):
        preds, revs = self.transport_many([field], velocities, dt)
        return {'predictorField': preds[0], 'reverseField': revs[0]}

    def transport_velocity(self, fields, dt):
        """Predict each signed face component; the reverse sample is fused with the correction."""
        if self.face_predictor is None:
            self.face_predictor = [self.device.texture(s, dtype=self.dtype) for s in self.grid.face_shapes]
        self.device.call('ffx_face_predictor', C.byref(self._g), C.byref(self._solids), self._storage,
                         *[ptr(f) for f in fields], dt, *[ptr(p) for p in self.face_predictor], self.device.s)

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
        self.curl = None
