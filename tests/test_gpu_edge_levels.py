"""Coarse (edge-record) multigrid levels: the residual + restriction
streamed along z (ffx_set_edge_streaming(1), the default) against one coarse
cell per thread, bit for bit -- with the coarse iterate cleared, and with the
sweep and prolongation + sweep (one cell per thread in both settings) checked
alongside -- on random edge records (zero and nonzero conductances, inactive
cells) over extents that are and are not multiples of the 32 x 8 block and of
the z chunks (8 fine slices from 2^20 cells up, else 2), and whole
collider-multigrid solves with the same cycle counts and fields."""
import ctypes as C

import numpy as np
import pytest
import torch

from fluxfx_b200 import _native as N
from tests.gpu_helpers import dev, t

pytestmark = pytest.mark.gpu


def ptr(x):
    return C.c_void_p(0 if x is None else x.data_ptr())


def _bits(x):
    torch.cuda.synchronize()
    return x.detach().cpu().numpy().view(np.uint32)


def _edges(shape, rng):
    nx, ny, nz = shape
    e = rng.uniform(0.0, 3.0, (nz, ny, nx, 4)).astype(np.float32)
    e[..., :3][rng.uniform(size=(nz, ny, nx, 3)) < 0.2] = 0.0       # closed faces
    e[..., 3] = (rng.uniform(size=(nz, ny, nx)) < 0.9).astype(np.float32)   # active flag
    return t(e)


@pytest.mark.parametrize('shape', [(128, 128, 66), (130, 18, 20), (64, 32, 70), (33, 7, 9), (2, 2, 2)])
def test_streamed_edge_passes_equal_one_cell_passes(shape):
    D = dev()
    nx, ny, nz = shape
    rng = np.random.default_rng(nx + 3 * ny + 7 * nz)
    edges = _edges(shape, rng)
    cell = (nz, ny, nx)
    p, rhs = t(rng.uniform(-1, 1, cell)), t(rng.uniform(-1, 1, cell))
    even = nx % 2 == 0 and ny % 2 == 0 and nz % 2 == 0
    coarse_shape = (max(nz // 2, 1), max(ny // 2, 1), max(nx // 2, 1))
    coarse = t(rng.uniform(-1, 1, coarse_shape))
    for scale in (0.0, 1.9):
        lv = N.FfxGraphLevel(*shape, ptr(edges), None, N.f3(0.0, 0.0, 0.0))
        lv.coarse_scale = scale
        outs = {}
        for stream_on in (1, 0):
            D.lib.ffx_set_edge_streaming(stream_on)
            try:
                sm = t(np.full(cell, np.nan))
                D.call('ffx_graph_smooth', C.byref(lv), ptr(p), ptr(rhs), 2 / 3, ptr(sm), D.s)
                got = [sm]
                if even:
                    ps = t(np.full(cell, np.nan))
                    D.call('ffx_graph_prolong_smooth', C.byref(lv), ptr(p), ptr(coarse), ptr(rhs), 2 / 3, ptr(ps),
                           D.s)
                    crhs, cp = t(np.full(coarse_shape, np.nan)), t(np.full(coarse_shape, np.nan))
                    D.call('ffx_graph_residual_restrict_zero', C.byref(lv), ptr(p), ptr(rhs), ptr(crhs), ptr(cp),
                           D.s)
                    got += [ps, crhs, cp]
                outs[stream_on] = [_bits(x) for x in got]
            finally:
                D.lib.ffx_set_edge_streaming(1)
        for k, (a, b) in enumerate(zip(outs[1], outs[0])):
            assert np.array_equal(a, b), (shape, scale, ['smooth', 'prolong_smooth', 'restrict', 'zero'][k])


@pytest.mark.parametrize('variant, storage', [('fast', 'BF16'), ('plain', 'FP32')])
def test_solve_with_streamed_edge_levels_equals_one_cell_solve(variant, storage):
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    D = dev()
    runs = []
    try:
        for stream_on in (1, 0):
            D.lib.ffx_set_edge_streaming(stream_on)
            grid, s, colliders, emitters, noise = bench.scene(64, storage, 9, **bench.VARIANTS[variant])
            sv = DenseProjectedSmoke(grid, s, D, colliders=colliders)
            sv.upload(torch.zeros(grid.cells))
            sv.upload_temperature(torch.zeros(grid.cells))
            sv.upload_velocity([torch.as_tensor(v * 300) for v in noise])
            runs.append((sv, emitters, stream_on))
        for k in range(3):
            for sv, em, stream_on in runs:
                D.lib.ffx_set_edge_streaming(stream_on)
                sv.step(0.02, sources=em)
            (a, _, _), (b, _, _) = runs
            assert a.projector.last_cycles == b.projector.last_cycles > 0, k
            torch.cuda.synchronize()
            for x, y in zip([a.density, a.temperature, a.projector.pressure, *a._velocity],
                            [b.density, b.temperature, b.projector.pressure, *b._velocity]):
                assert torch.equal(x, y), (variant, k)
    finally:
        D.lib.ffx_set_edge_streaming(1)
        for sv, _, _ in runs:
            sv.close()
