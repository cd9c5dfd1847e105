"""Galerkin aggregation hierarchy of the masked pressure graph.

Behaviour of FluxFX ``fluxfx/physics/solid_hierarchy.py:11-75``: level 0 holds,
per cell, the +x/+y/+z conductances (n/extent)^2 between fluid neighbours and an
active flag; each coarser level aggregates 2x2x2 children (restriction P^T/8,
so coarse conductances are boundary sums / 8) and coarsening stops before an
aggregate would join children that are not connected inside it.

In this package the hierarchy is built on the device by
``SolidMultigridProjector`` (``ffx_graph_coarsen``); ``build_hierarchy`` here
runs the same native kernel on a mask given from the host and returns host
arrays, for callers that want the levels themselves.
"""
from math import prod

import numpy as np


def build_hierarchy(shape, extent, mask, device=None):
    """[(shape, edges)] fine to coarse; edges are float32 arrays (nz, ny, nx, 4)."""
    import ctypes as C
    import torch
    from .. import _native as N
    from ..backend.device import CudaDevice, ptr
    if len(mask) != prod(shape):
        raise ValueError('Mask size must match grid')
    dev = device or CudaDevice()
    nx, ny, nz = shape
    solid = torch.as_tensor(np.asarray(mask, dtype=np.float64).reshape(nz, ny, nx) > .5).to(torch.uint8).to(dev.device)
    w = [float(np.float32((n / e) ** 2)) for n, e in zip(shape, extent)]
    level = N.FfxGraphLevel(*shape, None, ptr(solid), N.f3(*w))
    out = torch.empty((nz, ny, nx, 4), dtype=torch.float32, device=dev.device)
    dev.call('ffx_graph_level0_edges', C.byref(level), ptr(out), dev.s)
    levels = [(tuple(shape), out.cpu().numpy())]
    flag = torch.zeros(1, dtype=torch.int32, device=dev.device)
    keep = [solid, out]
    shape = tuple(shape)
    while min(shape) >= 8 and all(n % 2 == 0 for n in shape):
        cs = tuple(n // 2 for n in shape)
        edges = torch.empty((cs[2], cs[1], cs[0], 4), dtype=torch.float32, device=dev.device)
        dev.call('ffx_graph_coarsen', C.byref(level), ptr(edges), ptr(flag), dev.s)
        if int(flag.item()):
            break
        keep.append(edges)
        level = N.FfxGraphLevel(*cs, ptr(edges), None, N.f3(0.0, 0.0, 0.0))
        levels.append((cs, edges.cpu().numpy()))
        shape = cs
    return levels


def graph_inverse(shape, edges):
    """FP64 pseudoinverse of a small graph Laplacian (<= 256 cells)."""
    from ..backend.solid_multigrid import graph_pseudoinverse
    return graph_pseudoinverse(shape, edges)
