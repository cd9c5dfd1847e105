"""CUDA device boundary: torch tensors for storage, libffx_core for the passes.

Replaces FluxFX ``fluxfx/backend/device.py`` (the Blender ``gpu`` adapter). The
names ``texture``, ``kernel``, ``dispatch``, ``read`` and ``probe_3d`` keep
their meaning:

* ``texture(shape, values=None)`` allocates a zero-filled (or uploaded) field.
  ``shape`` is the reference's (nx, ny, nz); the tensor is (nz, ny, nx),
  x-fast, so ``tensor.flatten()`` is the reference's flat list order.
* ``read(texture, shape)`` is a synchronous readback to a Python list.
* ``kernel(name)`` / ``dispatch(...)`` run one of the native passes by the
  reference shader file name with the reference's uniform names, for scripts
  and tests that drive single passes (e.g. multigrid operators).

All work is enqueued on ``self.stream`` (the current torch stream of the device
at construction unless one is given). There is no CPU fallback.
"""
import ctypes as C
from math import isfinite, prod

import torch

from .. import _native as N

LOCAL_SIZE = (4, 4, 4)


class GPUUnavailable(RuntimeError):
    pass


def _shape3(shape):
    if len(shape) != 3 or any(int(n) <= 0 for n in shape):
        raise ValueError("Dispatch requires three positive dimensions")
    return tuple(int(n) for n in shape)


class KernelHandle:
    """A native pass addressed by the reference shader name."""

    def __init__(self, name, constants=()):
        self.name = name
        self.constants = tuple(constants)

    def __repr__(self):
        return f"KernelHandle({self.name!r})"


class CudaDevice:
    def __init__(self, index=None, stream=None):
        if not torch.cuda.is_available():
            raise GPUUnavailable("CUDA device required: no CUDA device is visible")
        try:
            self.lib = N.load()
        except N.NativeUnavailable as exc:
            raise GPUUnavailable(str(exc)) from exc
        self.index = torch.cuda.current_device() if index is None else int(index)
        self.device = torch.device('cuda', self.index)
        info = N.FfxDeviceInfo()
        status = self.lib.ffx_device_info(self.index, C.byref(info))
        if status != N.FFX_OK:
            raise GPUUnavailable(f"device query failed: {self.lib.ffx_last_error().decode()}")
        self.info = info
        if (info.cc_major, info.cc_minor) != (10, 0):
            raise GPUUnavailable(f"libffx_core is built for sm_100a (B200); found sm_{info.cc_major}{info.cc_minor}")
        self.sm_count = info.sm_count
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        self.max_groups = (2 ** 31 - 1, 65535, 65535)
        self.calls = 0

    # ------------------------------------------------------------------ basics
    @property
    def s(self):
        """Raw cudaStream_t for the C ABI."""
        return C.c_void_p(self.stream.cuda_stream)

    def call(self, name, *args):
        """Invoke a native entry point (each enqueues one kernel, two for the
        divergence statistics) and count it in ``calls``."""
        self.calls += 1
        N.check(getattr(self.lib, name)(*args))

    def synchronize(self):
        self.stream.synchronize()

    def ordered(self):
        """Context in which torch ops run on this device's stream, after the
        passes queued there (a solver may run on a stream other than torch's
        current one)."""
        return torch.cuda.stream(self.stream)

    def fetch(self, tensor):
        """Synchronous host copy of a device tensor, ordered after the passes
        queued on this device's stream."""
        with torch.cuda.stream(self.stream):
            return tensor.cpu()

    def capture(self, fn):
        """Record the passes ``fn`` enqueues into a CUDA graph (not executed now).

        Capture runs on a side stream: every native call made by ``fn`` goes to
        ``self.stream``, which points at that stream for the duration, and torch
        ops inside ``fn`` follow the capturing stream. ``fn`` must allocate
        nothing and must not synchronise."""
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(self.stream)
        saved = self.stream
        self.stream = side
        try:
            with torch.cuda.graph(graph, stream=side):
                fn()
        finally:
            self.stream = saved
        self.stream.wait_stream(side)
        return graph

    def replay(self, graph):
        with torch.cuda.stream(self.stream):
            graph.replay()

    def texture(self, shape, values=None, *, nonnegative=True, channels=1, dtype=torch.float32):
        if channels not in (1, 4):
            raise ValueError("Only scalar or four-channel fields are supported")
        nx, ny, nz = _shape3(shape)
        dims = (nz, ny, nx) if channels == 1 else (nz, ny, nx, 4)
        if values is None:
            with torch.cuda.stream(self.stream):
                return torch.zeros(dims, dtype=dtype, device=self.device)
        if isinstance(values, torch.Tensor):
            host = values.detach().to('cpu', torch.float64).reshape(-1)
        else:
            host = torch.as_tensor(list(values) if not hasattr(values, '__len__') else values,
                                   dtype=torch.float64).reshape(-1)
        if host.numel() != prod(dims):
            raise ValueError("Field upload must match grid and satisfy finite/sign constraints")
        if not bool(torch.isfinite(host).all()) or (nonnegative and bool((host < 0).any())):
            raise ValueError("Field upload must match grid and satisfy finite/sign constraints")
        with torch.cuda.stream(self.stream):
            return host.to(dtype).reshape(dims).to(self.device, non_blocking=False)

    def read(self, texture, shape=None):
        """Synchronous readback (diagnostics and tests)."""
        self.stream.synchronize()
        return texture.detach().to(torch.float64).flatten().cpu().tolist()

    def probe_3d(self):
        shape = (7, 5, 3)
        out = self.texture(shape)
        self.call('ffx_probe_3d', C.c_void_p(out.data_ptr()), self.s)
        actual = self.read(out)
        expected = [float(x + 10 * y + 100 * z) for z in range(3) for y in range(5) for x in range(7)]
        error = max(abs(a - b) for a, b in zip(actual, expected))
        if not all(isfinite(v) for v in actual) or error > 1e-6:
            raise GPUUnavailable(f"3D store/readback mismatch: {error}")
        return {"status": "PASS", "format": "R32F", "shape": shape, "texels_checked": len(actual),
                "max_abs_error": error, "device": self.info.name.decode(), "sm_count": self.sm_count}

    # ------------------------------------------------------- reference-style
    def kernel(self, filename, constants=(), sample_input=False, samplers=(), includes=(), output_format='R32F'):
        return KernelHandle(filename, constants)

    def dispatch(self, shader, output, shape, uniforms=None, input_field=None, sources=None):
        """Run one native pass by shader name with the reference's uniforms."""
        from . import _dispatch
        if output is input_field or any(output is t for t in (sources or {}).values()):
            raise ValueError("Advection input/output textures must be distinct")
        _dispatch.run(self, shader, output, _shape3(shape), uniforms or {}, input_field, sources or {})


class PassTimer:
    """CUDA events between the passes of a step, on the solver's stream.

    ``mark(name)`` closes the interval that started at the previous mark and
    books it under ``name``; ``totals_ms()`` synchronises and returns the summed
    milliseconds per name. Off unless a solver is given one."""

    def __init__(self, stream):
        self.stream = stream
        self.events = []     # (name, event)

    def mark(self, name):
        e = torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        self.events.append((name, e))

    def totals_ms(self):
        if len(self.events) < 2:
            return {}
        self.events[-1][1].synchronize()
        out = {}
        for (_, a), (name, b) in zip(self.events, self.events[1:]):
            if name == 'start':
                continue
            out[name] = out.get(name, 0.0) + a.elapsed_time(b)
        return out


def ptr(t):
    """Device address of a tensor (or NULL for None)."""
    return C.c_void_p(0 if t is None else t.data_ptr())


def solids_struct(device):
    """FfxSolids of a (collider) device: its mask and dilated mask, plus the
    wall-velocity faces of moving colliders. The tensors are updated in place
    when colliders move, so the struct stays valid."""
    mask = getattr(device, 'mask', None)
    halo = getattr(device, 'halo', None)
    walls = getattr(device, 'walls', None)
    clear = getattr(device, 'clear', None)
    s = N.FfxSolids(ptr(mask) if mask is not None else None, ptr(halo) if halo is not None else None)
    if clear is not None and mask is not None:
        s.clear = clear.data_ptr()
    if walls is not None:
        for a in range(3):
            s.wall[a] = walls[a].data_ptr()
    return s


def storage_code(dtype):
    if dtype == torch.float32:
        return N.FFX_F32
    if dtype == torch.bfloat16:
        return N.FFX_BF16
    raise ValueError(f"unsupported field storage {dtype}")
