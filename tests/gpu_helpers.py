"""Shared helpers of the GPU parity tests (CUDA path vs the CPU oracle)."""
import ctypes as C

import numpy as np
import torch

from fluxfx_b200 import _native as N

# Per-pass parity bar: max abs error <= REL * max|oracle field| (+ a floor for all-zero fields).
REL = 1e-5


def dev():
    from fluxfx_b200.backend.device import CudaDevice
    return CudaDevice()


# Tensors handed to the C ABI as raw pointers must outlive the (asynchronous)
# launches that read them: t() parks every tensor here until the test ends.
_KEEP = []


def t(a, dtype=torch.float32):
    x = torch.as_tensor(np.ascontiguousarray(a)).to(dtype).cuda()
    _KEEP.append(x)
    return x


def release():
    if _KEEP:
        torch.cuda.synchronize()
        _KEEP.clear()


def n(x):
    torch.cuda.synchronize()
    return x.detach().to(torch.float64).cpu().numpy()


def assert_close(actual, expected, rel=REL, floor=1e-30, what=''):
    a = np.asarray(actual, dtype=np.float64)
    e = np.asarray(expected, dtype=np.float64)
    assert a.shape == e.shape, (what, a.shape, e.shape)
    scale = max(float(np.abs(e).max()) if e.size else 0.0, floor)
    err = float(np.abs(a - e).max()) if e.size else 0.0
    assert err <= rel * scale, f"{what}: max abs error {err:.3e} > {rel:.1e} * {scale:.3e}"
    return err / scale


def grid_ptr(shape, extent):
    g = N.grid_struct(shape, extent)
    return g, C.byref(g)


def solids(mask_t=None, halo_t=None):
    from fluxfx_b200.backend.device import ptr
    return N.FfxSolids(ptr(mask_t) if mask_t is not None else None, ptr(halo_t) if halo_t is not None else None)


def random_faces(g, rng, scale=1.0):
    return tuple((rng.uniform(-1, 1, fs) * scale).astype(np.float32) for fs in g.face_shapes)


def sphere_box_mask(shape, extent=(1., 1., 1.)):
    """A sphere and a box, in cell units, for collider tests."""
    from fluxfx_b200.physics.collision import primitive
    nx, ny, nz = shape
    h = [e / c for e, c in zip(extent, shape)]
    sph = primitive('SPHERE', (0.55 * extent[0], 0.5 * extent[1], 0.5 * extent[2]), (0.22 * min(extent),) * 3)
    box = primitive('BOX', (0.2 * extent[0], 0.3 * extent[1], 0.25 * extent[2]),
                    (3 * h[0], 4 * h[1], 2 * h[2]))
    return (sph, box)
