"""GPU readback for baking: one frame's preview channels to host memory.

Drop-in for FluxFX ``fluxfx/backend/cache.py:7-11`` (``capture``): the
channels DENSITY and TEMPERATURE, FUEL and FLAME with combustion, COLLISION
(the mask as 0/1) with colliders, each a flat x-fast FP32 array.

``BakeRecorder`` writes a run into a playback cache (``physics.cache``)
without stalling the solver: after a step it enqueues, on a copy stream,
one ``ffx_pack_channels`` launch that snapshots the channels into a device
staging buffer (already the frame's file layout), makes the solver's stream
wait only for that snapshot, and copies the staging buffer into pinned host
memory while the next steps compute. A writer thread waits for the copy,
validates, compresses and writes the frame (frames stay in order). ``depth``
staging/pinned buffers bound the frames in flight; a frame that would reuse a
buffer still being written waits for it.
"""
import ctypes as C
import threading
from concurrent.futures import ThreadPoolExecutor
from math import prod

import torch

from .. import _native as N
from .device import ptr


def channels_of(solver):
    """Preview channels of a solver, in the reference's order."""
    names = ['DENSITY', 'TEMPERATURE']
    if solver.combustion is not None:
        names += ['FUEL', 'FLAME']
    if solver.solids is not None:
        names += ['COLLISION']
    return names


def _kind(t):
    if t.dtype == torch.float32:
        return N.FFX_F32
    if t.dtype == torch.bfloat16:
        return N.FFX_BF16
    if t.dtype == torch.uint8:
        return N.FFX_PACK_U8
    raise ValueError(f'Unsupported preview field type {t.dtype}')


def _pack(solver, names, out, stream):
    fields = [solver.preview_field(name) for name in names]
    arr = (C.c_void_p * len(fields))(*[f.data_ptr() for f in fields])
    kinds = (C.c_int * len(fields))(*[_kind(f) for f in fields])
    solver.device.call('ffx_pack_channels', prod(solver.grid.shape), len(fields), arr, kinds, ptr(out),
                       stream.cuda_stream)


def capture(solver):
    """{channel: host FP32 array} of the solver's current fields (synchronous)."""
    names = channels_of(solver)
    n = prod(solver.grid.shape)
    stream = solver.device.stream
    staging = torch.empty(len(names) * n, dtype=torch.float32, device=solver.device.device)
    with torch.cuda.stream(stream):
        _pack(solver, names, staging, stream)
        host = staging.cpu()
    return {name: host[i * n:(i + 1) * n].numpy() for i, name in enumerate(names)}


class BakeRecorder:
    """Asynchronous bake of ``solver``'s frames into ``writer`` (a
    ``physics.cache.CacheWriter`` whose channels are the solver's preview
    channels). Call ``record(frame)`` after each baked step, ``finish()`` at
    the end (or ``close()`` to abandon); errors of the writer thread surface
    from the next ``record`` or from ``finish``."""

    def __init__(self, solver, writer, depth=2):
        names = list(writer.meta['channels'])
        if set(names) != set(channels_of(solver)):
            raise ValueError('Cache channels differ from the solver preview channels')
        if tuple(writer.meta['shape']) != tuple(solver.grid.shape):
            raise ValueError('Cache grid differs from the solver grid')
        if depth < 1:
            raise ValueError('depth must be at least 1')
        self.solver = solver
        self.writer = writer
        self.names = names
        self.n = prod(solver.grid.shape)
        dev = solver.device.device
        size = len(names) * self.n
        self.staging = [torch.empty(size, dtype=torch.float32, device=dev) for _ in range(depth)]
        self.host = [torch.empty(size, dtype=torch.float32, pin_memory=True) for _ in range(depth)]
        self.copier = torch.cuda.Stream(device=dev)
        self.pending = [None] * depth       # future of the write that still reads host[slot]
        self.pool = ThreadPoolExecutor(max_workers=1, thread_name_prefix='fluxfx-bake')
        self.lock = threading.Lock()
        self.frames = 0
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    def _slot_free(self, slot):
        fut = self.pending[slot]
        if fut is not None:
            fut.result()              # re-raises a failed write
            self.pending[slot] = None

    def record(self, frame):
        """Snapshot the solver's current fields as cache frame ``frame``."""
        slot = self.frames % len(self.staging)
        self._slot_free(slot)
        solver_stream = self.solver.device.stream
        ready = torch.cuda.Event()
        ready.record(solver_stream)
        self.copier.wait_event(ready)
        with torch.cuda.stream(self.copier):
            _pack(self.solver, self.names, self.staging[slot], self.copier)
            packed = torch.cuda.Event()
            packed.record(self.copier)
            self.host[slot].copy_(self.staging[slot], non_blocking=True)
            landed = torch.cuda.Event()
            landed.record(self.copier)
        # the solver may overwrite its fields once the snapshot exists
        solver_stream.wait_event(packed)
        self.d2h_bytes += self.host[slot].numel() * 4
        self.pending[slot] = self.pool.submit(self._write, frame, slot, landed)
        self.frames += 1

    def _write(self, frame, slot, landed):
        landed.synchronize()
        data = self.host[slot].numpy()
        fields = {name: data[i * self.n:(i + 1) * self.n] for i, name in enumerate(self.names)}
        with self.lock:
            self.writer.write(frame, fields)

    def drain(self):
        for slot in range(len(self.pending)):
            self._slot_free(slot)

    def finish(self, status='COMPLETE', message=''):
        try:
            self.drain()
        except Exception as exc:
            self.writer.finish('FAILED', str(exc))
            self.close()
            raise
        self.writer.finish(status, message)
        self.close()

    def close(self):
        self.pool.shutdown(wait=True)
        self.staging = self.host = []
        self.pending = []
