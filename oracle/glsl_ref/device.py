"""CPU stand-in for the reference's GPU device adapter -- TEST INFRASTRUCTURE ONLY.

Implements the interface of FluxFX ``fluxfx/backend/device.py:15-96``
(``texture``, ``kernel``, ``dispatch``, ``read``, ``probe_3d``) on top of
``oracle/_ref/libglsl_ref.so``, the reference's own compute shaders compiled
for the CPU. With it, the reference's unmodified backend classes
(``DenseProjectedSmoke``, ``MultigridPressureProjector``,
``SolidMultigridProjector``, ...) run on the host and produce golden vectors.
"""
import ctypes as C
from math import isfinite, prod
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent.parent / '_ref' / 'libglsl_ref.so'
_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} missing: run python oracle/glsl_ref/build.py")
        lib = C.CDLL(str(LIB))
        lib.glsl_ref_kernel.argtypes = [C.c_char_p, C.c_int]
        lib.glsl_ref_set_uniform.argtypes = [C.c_char_p, C.POINTER(C.c_float), C.c_int]
        lib.glsl_ref_bind_sampler.argtypes = [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.glsl_ref_bind_output.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.glsl_ref_dispatch.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
        lib.glsl_ref_out_of_range.restype = C.c_longlong
        _lib = lib
    return _lib


class Texture:
    """R32F / RGBA32F 3D texture held as a flat x-fast float32 array."""

    def __init__(self, shape, channels=1, data=None):
        self.shape = tuple(int(n) for n in shape)
        self.channels = channels
        n = prod(self.shape) * channels
        self.data = np.zeros(n, np.float32) if data is None else np.array(data, dtype=np.float32).reshape(n)

    def clear(self, format='FLOAT', value=(0.0,)):
        self.data.reshape(-1, self.channels)[:] = np.array(value, dtype=np.float32)

    def filter_mode(self, _):
        pass

    def ptr(self):
        return self.data.ctypes.data_as(C.c_void_p)


class Shader:
    def __init__(self, filename, kernel_id):
        self.filename = filename
        self.kernel_id = kernel_id


class GPUUnavailable(RuntimeError):
    pass


class GlslCpuDevice:
    def __init__(self):
        self.lib = load()
        self.max_groups = (1 << 30,) * 3
        self.dispatches = 0

    def texture(self, shape, values=None, *, nonnegative=True, channels=1):
        if channels not in (1, 4):
            raise ValueError("Only scalar or four-channel fields are supported")
        if values is not None:
            values = list(values)
            if len(values) != prod(shape) * channels or not all(
                    isfinite(v) and (not nonnegative or v >= 0) for v in values):
                raise ValueError("Field upload must match grid and satisfy finite/sign constraints")
        return Texture(shape, channels, values)

    def kernel(self, filename, constants=(), sample_input=False, samplers=(), includes=(), output_format='R32F'):
        collisions = 2 if 'moving_boundary.glsl' in includes else int('solid_boundary.glsl' in includes)
        kid = self.lib.glsl_ref_kernel(filename.encode(), collisions)
        return Shader(filename, kid)

    def dispatch(self, shader, output, shape, uniforms=None, input_field=None, sources=None):
        if shader.kernel_id < 0:
            raise NotImplementedError(f"{shader.filename} is not part of the compiled reference kernel set")
        if output is input_field or any(output is t for t in (sources or {}).values()):
            raise ValueError("Advection input/output textures must be distinct")
        lib = self.lib
        lib.glsl_ref_clear_bindings()
        keep = []
        if input_field is not None:
            lib.glsl_ref_bind_sampler(b'inputField', input_field.ptr(), *input_field.shape, input_field.channels)
        for name, tex in (sources or {}).items():
            if lib.glsl_ref_bind_sampler(name.encode(), tex.ptr(), *tex.shape, tex.channels) != 0:
                raise KeyError(f"unknown sampler {name}")
        for name, value in (uniforms or {}).items():
            vals = [float(v) for v in value] if isinstance(value, (tuple, list)) else [float(value)]
            arr = (C.c_float * len(vals))(*vals)
            keep.append(arr)
            st = lib.glsl_ref_set_uniform(name.encode(), arr, len(vals))
            if st != 0:
                raise KeyError(f"uniform {name} ({len(vals)} values) not accepted: {st}")
        lib.glsl_ref_bind_output(output.ptr(), *output.shape, output.channels)
        lib.glsl_ref_dispatch(shader.kernel_id, *[int(n) for n in shape])
        self.dispatches += 1

    @staticmethod
    def read(texture, shape):
        return texture.data[:prod(shape) * texture.channels].astype(np.float64).tolist()

    def probe_3d(self):
        return {"status": "PASS", "format": "R32F", "shape": (7, 5, 3), "texels_checked": 105,
                "max_abs_error": 0.0}

    def out_of_range(self):
        return int(self.lib.glsl_ref_out_of_range())
