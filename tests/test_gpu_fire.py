"""Fire-configuration passes on the CUDA path: vorticity confinement,
combustion and moving colliders, per pass against the FP32 oracle and as full
steps against the reference backend's own runs (reference_fire_steps.npz)."""
import ctypes as C

import numpy as np
import pytest
import torch

from fluxfx_b200 import _native as N
from oracle import fire as F
from oracle import smoke as S
from tests import reference_cases as R
from tests.gpu_helpers import assert_close, dev, grid_ptr, n, t

pytestmark = pytest.mark.gpu


def ptr(x):
    return C.c_void_p(0 if x is None else x.data_ptr())


@pytest.fixture(scope='module')
def D():
    return dev()


def host(x):
    torch.cuda.synchronize()
    return x.detach().to(torch.float64).cpu().numpy()


@pytest.mark.parametrize('shape,extent', [((16, 12, 10), (1.0, 1.0, 1.0)), ((12, 10, 8), (1.3, 0.8, 1.7))])
def test_curl_and_confinement_match_oracle(D, shape, extent):
    g = S.Grid(shape, extent)
    gs, gp = grid_ptr(shape, extent)
    rng = np.random.default_rng(3)
    vel = [rng.uniform(-1, 1, fs).astype(np.float32) for fs in g.face_shapes]
    nx, ny, nz = shape
    curl = torch.zeros((nz, ny, nx, 4), device='cuda')
    D.call('ffx_curl', gp, N.FFX_F32, *[ptr(t(v)) for v in vel], ptr(curl), D.s)
    want = F.curl(g, vel)
    assert_close(host(curl), want, rel=1e-6, what='curl')
    outs = [t(np.zeros(fs)) for fs in g.face_shapes]
    D.call('ffx_confine', gp, N.FFX_F32, ptr(t(want)), *[ptr(t(v)) for v in vel], 0.02, 0.3, 2.0,
           *[ptr(o) for o in outs], D.s)
    exp = F.confine(g, vel, want, 0.02, 0.3, 2.0)
    for a in range(3):
        assert_close(n(outs[a]), exp[a], rel=1e-6, what=f'confined face {a}')


def test_combustion_matches_oracle(D):
    shape = (16, 12, 10)
    g = S.Grid(shape)
    gs, gp = grid_ptr(shape, (1.0, 1.0, 1.0))
    rng = np.random.default_rng(4)
    fuel = rng.uniform(-0.1, 1, g.cell_shape).astype(np.float32)
    temp = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    rho = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    tf, tt, tr, fl = t(fuel), t(temp), t(rho), t(np.zeros(g.cell_shape))
    D.call('ffx_combustion', gp, N.FFX_F32, ptr(tf), ptr(tt), ptr(tr), 0.02, 0.3, 0.75, 0.5, 1.0, ptr(fl),
           ptr(tf), ptr(tr), ptr(tt), D.s)        # in place
    flame = F.burn(g, fuel, temp, 0.02, 0.3, 0.75)
    # exp(-rate dt) may differ by an ulp between CUDA and NumPy: the per-pass bar (1e-5 of the max)
    assert_close(n(fl), flame, what='flame')
    assert_close(n(tf), F.apply_burn(g, fuel, flame, 0.02, -1.0), what='fuel')
    assert_close(n(tr), F.apply_burn(g, rho, flame, 0.02, 0.5), what='density')
    assert_close(n(tt), F.apply_burn(g, temp, flame, 0.02, 1.0), what='temperature')
    assert (n(tf) >= 0).all() and float(np.abs(n(fl)).max()) > 0


def test_moving_collider_passes_match_oracle(D):
    from fluxfx_b200.physics.collider_motion import collider_rows12, velocity_rows
    from fluxfx_b200.physics.collision import primitive
    shape, extent = (20, 16, 12), (1.0, 0.8, 0.6)
    g = S.Grid(shape, extent)
    gs, gp = grid_ptr(shape, extent)
    old = (primitive('SPHERE', (0.4, 0.4, 0.3), (0.15,) * 3), primitive('BOX', (0.6, 0.35, 0.3), (0.1, 0.12, 0.08)))
    new = (primitive('SPHERE', (0.43, 0.41, 0.3), (0.15,) * 3), primitive('BOX', (0.62, 0.35, 0.31), (0.1, 0.12, 0.08)))
    owners = []
    for cols in (old, new):
        rows, box = collider_rows12(cols)
        o = torch.zeros(g.cell_shape, dtype=torch.uint8, device='cuda')
        D.call('ffx_moving_mask', gp, len(cols), (C.c_float * len(rows))(*rows), (C.c_int32 * len(box))(*box),
               ptr(o), D.s)
        want = F.moving_mask(g, [(c.shape, c.inverse_rows) for c in cols])
        assert np.array_equal(host(o), want), 'owner mask'
        owners.append(o)
    table = np.float32([v for a, b in zip(old, new) for row in velocity_rows(a, b, 0.02) for v in row])
    walls = [t(np.zeros(fs)) for fs in g.face_shapes]
    D.call('ffx_moving_walls', gp, ptr(owners[1]), 2, (C.c_float * len(table))(*table.tolist()),
           *[ptr(w) for w in walls], D.s)
    want_walls = F.moving_walls(g, host(owners[1]), table.reshape(2, 3, 4))
    for a in range(3):
        assert np.array_equal(n(walls[a]), want_walls[a]), f'wall velocity {a}'
    rng = np.random.default_rng(8)
    rho = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    vel = [rng.uniform(-1, 1, fs).astype(np.float32) for fs in g.face_shapes]
    tr, tv = t(rho), [t(v) for v in vel]
    D.call('ffx_moving_remap', gp, N.FFX_F32, ptr(owners[1]), ptr(owners[0]), ptr(tr), None, None,
           *[ptr(v) for v in tv], *[ptr(w) for w in walls], D.s)
    assert np.array_equal(n(tr), F.remap_scalar(g, rho, host(owners[1]), host(owners[0])))
    exp = F.remap_faces(g, vel, host(owners[1]), host(owners[0]), want_walls)
    for a in range(3):
        assert np.array_equal(n(tv[a]), exp[a]), f'remapped face {a}'


@pytest.mark.parametrize('name', R.fire_cases())
def test_cuda_path_matches_reference_fire_runs(D, name):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.physics.config import GridSpec
    c = R.case(name, R.FIRE)
    cols = c['moving'](0) if c['moving'] is not None else c['colliders']
    solver = DenseProjectedSmoke(GridSpec(c['shape']), c['settings'], D, colliders=cols)
    if c['mask'] is not None:
        assert np.array_equal(host(solver.solids.mask) > 0.5, c['mask'])
    R.compare(host(solver.density), c['init_density'], R.TOL, 'seeded density')
    R.compare(host(solver.temperature), c['init_temperature'], R.TOL, 'seeded temperature')
    solver.upload_velocity([torch.as_tensor(v) for v in c['velocity']])
    for k, dt in enumerate(c['dts']):
        if c['moving'] is not None:
            solver.move_colliders(c['moving'](k + 1), dt)
        solver.step(dt, sources=c['sources'])
        if k not in c['steps']:
            continue
        want = c['steps'][k]
        R.compare(host(solver.density), want['density'], R.TOL, f'step {k} density')
        R.compare(host(solver.temperature), want['temperature'], R.TOL, f'step {k} temperature')
        for a in range(3):
            R.compare(host(solver._velocity[a]), want['velocity'][a], R.TOL, f'step {k} velocity {a}')
        R.compare_after(host(solver.projector.after), want, f'step {k} divergence after')
        if 'fuel' in want:
            R.compare(host(solver.combustion.fuel), want['fuel'], R.TOL, f'step {k} fuel')
            R.compare(host(solver.combustion.flame), want['flame'], R.TOL, f'step {k} flame')
        if 'mask' in want:
            assert np.array_equal(host(solver.solids.mask), want['mask']), f'step {k} owner mask'
    solver.close()


@pytest.mark.parametrize('alpha,warm', [(1.0, False), (1.9, True)])
def test_moving_collider_multigrid_matches_oracle(D, alpha, warm):
    """Multigrid with a moving collider (an extension of the fire configuration:
    the reference projects moving-collider scenes with masked Jacobi): after each
    move the aggregation hierarchy follows the new owner mask, and the steps
    match the oracle's, for the reference cycle and for the fast form
    (over-corrected, warm-started)."""
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.backend.solid_multigrid import SolidMultigridProjector
    from fluxfx_b200.physics.collision import primitive
    from fluxfx_b200.physics.config import GridSpec
    from fluxfx_b200.physics.pressure import PressureSettings
    from oracle.solver import OracleSmoke
    shape = (32, 24, 40)
    grid = GridSpec(shape)
    hx = 1.0 / shape[0]
    s = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', moving_colliders=True,
                         thermal_lift=1.0, density_weight=0.05, source_center=(0.5, 0.5, 0.2), source_radius=0.12,
                         pressure_tolerance=1e-4, pressure_max_cycles=100, mg_coarse_scale=alpha,
                         solid_warm_start=warm)
    pose = lambda k: (primitive('SPHERE', (0.3 + 0.5 * hx * k, 0.5, 0.6), (0.15, 0.15, 0.15)),)
    solver = DenseProjectedSmoke(grid, s, D, projector_class=SolidMultigridProjector, colliders=pose(0))
    ref = OracleSmoke(grid.shape, grid.extent, s, np.float32, kind='SOLID_MULTIGRID',
                      colliders=[(c.shape, c.inverse_rows) for c in pose(0)])
    rng = np.random.default_rng(21)
    vel = tuple((rng.uniform(-1, 1, fs) * 0.2).astype(np.float32) for fs in ref.g.face_shapes)
    solver.upload_velocity([torch.as_tensor(v) for v in vel])
    ref.upload(velocity=vel)
    levels0 = len(solver.projector.levels)
    for k, dt in enumerate((0.02, 0.02, 0.015, 0.02)):
        solver.move_colliders(pose(k + 1), dt)
        ref.move_colliders([(c.shape, c.inverse_rows) for c in pose(k + 1)], dt)
        solver.step(dt)
        ref.step(dt)
        assert np.array_equal(host(solver.solids.mask) > 0.5, ref.owners > 0.5), f'step {k} mask'
        assert solver.projector.last_cycles == ref.projector.last_cycles, (k, solver.projector.last_cycles,
                                                                          ref.projector.last_cycles)
        assert_close(n(solver.density), ref.density, rel=1e-5, what=f'step {k} density')
        for a in range(3):
            assert_close(n(solver._velocity[a]), ref.velocity[a], rel=1e-5, what=f'step {k} velocity {a}')
        assert solver.measure_projection()['rel_div_inf'] <= 1e-4
    assert len(solver.projector.levels) >= 2 and levels0 >= 2
    solver.close()
