"""Two level-0 sweeps in one pass (ffx_graph_smooth2, ffx_graph_prolong_smooth2)
against two launches of the single sweep, bit for bit: grids whose extents are
and are not multiples of the fused kernel's tile (128 x 8 x 16 cells), with a
collider mask and random solid cells, the plain and the prolonged first sweep,
and the one-cell (edge record) level path through the intermediate buffer. The
collider-multigrid solve with fused sweeps takes the same cycles and gives the
same fields as the sweep-by-sweep solve."""
import ctypes as C

import numpy as np
import pytest
import torch

from fluxfx_b200 import _native as N
from tests.gpu_helpers import dev, sphere_box_mask, t

pytestmark = pytest.mark.gpu


def ptr(x):
    return C.c_void_p(0 if x is None else x.data_ptr())


def _bits(x):
    torch.cuda.synchronize()
    return x.detach().cpu().numpy().view(np.uint32)


@pytest.mark.parametrize('shape', [(256, 16, 32), (48, 42, 36), (132, 9, 17), (8, 8, 8)])
def test_fused_sweeps_equal_two_sweeps(shape):
    D = dev()
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 7 + ny * 3 + nz)
    from fluxfx_b200.physics.collision import raster_reference
    from fluxfx_b200.physics.config import GridSpec
    grid = GridSpec(shape, axis_limit=256)
    mask = np.asarray(raster_reference(grid, sphere_box_mask(shape))).reshape(nz, ny, nx) > 0.5
    mask |= rng.uniform(size=mask.shape) < 0.1
    solid_t = t(mask, torch.uint8)
    w = [float(np.float32(c ** 2)) for c in shape]
    lv = N.FfxGraphLevel(*shape, None, ptr(solid_t), N.f3(*w))
    links = torch.zeros((nz, ny, nx), dtype=torch.uint8, device='cuda')
    D.call('ffx_graph_links', C.byref(lv), ptr(links), D.s)
    lv.links = links.data_ptr()
    cell = (nz, ny, nx)
    p, rhs = t(rng.uniform(-1, 1, cell)), t(rng.uniform(-1, 1, cell))
    coarse = t(rng.uniform(-1, 1, (max(nz // 2, 1), max(ny // 2, 1), max(nx // 2, 1))))
    for omega in (2 / 3, 0.8):
        mid, two, fused = (t(np.full(cell, np.nan)) for _ in range(3))
        D.call('ffx_graph_smooth', C.byref(lv), ptr(p), ptr(rhs), omega, ptr(mid), D.s)
        D.call('ffx_graph_smooth', C.byref(lv), ptr(mid), ptr(rhs), omega, ptr(two), D.s)
        D.call('ffx_graph_smooth2', C.byref(lv), ptr(p), ptr(rhs), omega, None, ptr(fused), D.s)
        assert np.array_equal(_bits(two), _bits(fused)), (shape, omega)
        if nx % 2 or ny % 2 or nz % 2:
            continue     # the prolongation needs even extents
        mid, two, fused = (t(np.full(cell, np.nan)) for _ in range(3))
        D.call('ffx_graph_prolong_smooth', C.byref(lv), ptr(p), ptr(coarse), ptr(rhs), omega, ptr(mid), D.s)
        D.call('ffx_graph_smooth', C.byref(lv), ptr(mid), ptr(rhs), omega, ptr(two), D.s)
        D.call('ffx_graph_prolong_smooth2', C.byref(lv), ptr(p), ptr(coarse), ptr(rhs), omega, None, ptr(fused),
               D.s)
        assert np.array_equal(_bits(two), _bits(fused)), (shape, omega, 'prolonged')
    # the convergence test with the speculative sweep: the residual maximum and the sweep
    m1, m2 = torch.full((1,), -1.0, device='cuda'), torch.full((1,), -1.0, device='cuda')
    one, both = t(np.full(cell, np.nan)), t(np.full(cell, np.nan))
    D.call('ffx_graph_residual_max', C.byref(lv), ptr(p), ptr(rhs), ptr(m1), D.s)
    D.call('ffx_graph_smooth', C.byref(lv), ptr(p), ptr(rhs), 2 / 3, ptr(one), D.s)
    D.call('ffx_graph_residual_max_smooth', C.byref(lv), ptr(p), ptr(rhs), 2 / 3, ptr(m2), ptr(both), D.s)
    assert float(m1[0]) == float(m2[0]) > 0 and np.array_equal(_bits(one), _bits(both))
    # without the link field the level takes the one-cell kernels, two launches through tmp
    scalar = N.FfxGraphLevel(*shape, None, ptr(solid_t), N.f3(*w))
    tmp, fused = t(np.full(cell, np.nan)), t(np.full(cell, np.nan))
    D.call('ffx_graph_smooth2', C.byref(scalar), ptr(p), ptr(rhs), 2 / 3, ptr(tmp), ptr(fused), D.s)
    mid, two = t(np.full(cell, np.nan)), t(np.full(cell, np.nan))
    D.call('ffx_graph_smooth', C.byref(lv), ptr(p), ptr(rhs), 2 / 3, ptr(mid), D.s)
    D.call('ffx_graph_smooth', C.byref(lv), ptr(mid), ptr(rhs), 2 / 3, ptr(two), D.s)
    assert np.array_equal(_bits(two), _bits(fused))


@pytest.mark.parametrize('variant, sweeps', [('fast', 4), ('plain', 4), ('fast', 3)])
def test_solve_with_fused_sweeps_equals_sweep_by_sweep(variant, sweeps):
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    D = dev()
    runs = []
    for fuse in (True, False):
        grid, s, colliders, emitters, noise = bench.scene(64, 'FP32', 6, mg_pre_sweeps=sweeps,
                                                          mg_post_sweeps=sweeps, **bench.VARIANTS[variant])
        sv = DenseProjectedSmoke(grid, s, D, colliders=colliders)
        sv.projector.fuse_sweeps = fuse
        sv.upload(torch.zeros(grid.cells))
        sv.upload_temperature(torch.zeros(grid.cells))
        sv.upload_velocity([torch.as_tensor(v * 300) for v in noise])
        runs.append((sv, emitters))
    for k in range(4):
        for sv, em in runs:
            sv.step_cfl(0.5, 0.02, sources=em)
        (a, _), (b, _) = runs
        assert a.projector.last_cycles == b.projector.last_cycles > 0, k
        torch.cuda.synchronize()
        for x, y in zip([a.density, a.temperature, a.projector.pressure, *a._velocity],
                        [b.density, b.temperature, b.projector.pressure, *b._velocity]):
            assert torch.equal(x, y), (variant, sweeps, k)
    for sv, _ in runs:
        sv.close()


@pytest.mark.parametrize('variant, storage', [('fast', 'BF16'), ('plain', 'FP32'), ('learned', 'FP32')])
def test_speculative_sweep_in_the_solve_loop(variant, storage):
    """The device loop whose convergence test also makes the next cycle's first
    pre-sweep (ffx_graph_residual_max_smooth) gives the cycle counts and fields
    of the loop without it, bit for bit."""
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    D = dev()
    runs = []
    for speculate in (True, False):
        grid, s, colliders, emitters, noise = bench.scene(64, storage, 7, **bench.VARIANTS[variant])
        sv = DenseProjectedSmoke(grid, s, D, colliders=colliders)
        if s.learned_warm_start:
            from fluxfx_b200.learned import attach
            attach(sv, colliders)
        sv.projector.speculate = speculate
        sv.upload(torch.zeros(grid.cells))
        sv.upload_temperature(torch.zeros(grid.cells))
        sv.upload_velocity([torch.as_tensor(v * 300) for v in noise])
        runs.append((sv, emitters))
    for k in range(4):
        for sv, em in runs:
            sv.step_cfl(0.5, 0.02, sources=em)
        (a, _), (b, _) = runs
        assert a.projector.last_cycles == b.projector.last_cycles > 0, k
        torch.cuda.synchronize()
        for x, y in zip([a.density, a.temperature, a.projector.pressure, *a._velocity],
                        [b.density, b.temperature, b.projector.pressure, *b._velocity]):
            assert torch.equal(x, y), (variant, k)
    for sv, _ in runs:
        sv.close()
