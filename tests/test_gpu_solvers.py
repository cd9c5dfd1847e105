"""Solver-level parity: projectors and the full smoke step against the CPU oracle,
plus the behaviour checks of the reference's GPU validation scripts
(scripts/collision_validate.py, multigrid_operators_validate.py,
pressure_validate.py, mac_validate.py) run through the drop-in API."""
import math
from dataclasses import replace

import numpy as np
import pytest
import torch

from fluxfx_b200.physics.config import GridSpec
from fluxfx_b200.physics.pressure import PressureSettings
from oracle import smoke as S
from oracle import solver as O
from tests.gpu_helpers import assert_close, dev, n, sphere_box_mask

pytestmark = pytest.mark.gpu

# Full-step parity bar (per step, per field): max abs error <= STEP_REL * max|field|.
STEP_REL = 1e-5


@pytest.fixture(scope='module')
def D():
    return dev()


def _faces_from(g, vel):
    return [v.ravel().tolist() for v in vel]


def test_jacobi_projector_matches_oracle(D):
    from fluxfx_b200.backend.pressure import PressureProjector
    grid = GridSpec((12, 10, 8), (1.3, .8, 1.7))
    s = PressureSettings(pressure_iterations=30)
    g = S.Grid(grid.shape, grid.extent)
    rng = np.random.default_rng(10)
    vel = tuple(rng.uniform(-1, 1, fs).astype(np.float32) for fs in g.face_shapes)
    proj = PressureProjector(grid, s, D)
    ref = O.OracleProjector(g, s, 'JACOBI')
    fields = [D.texture(fs, v.ravel(), nonnegative=False) for fs, v in zip(grid.face_shapes, vel)]
    outs = [D.texture(fs) for fs in grid.face_shapes]
    for dt in (0.04, 0.04, 0.02):
        proj.project(fields, outs, dt)
        eo, eb, ea = ref.project(vel, dt)
        assert proj.last_iterations == ref.last_iterations
        assert_close(n(proj.before), eb, what='before')
        for a in range(3):
            assert_close(n(outs[a]), eo[a], what=f'velocity {a}')
        assert_close(n(proj.pressure), ref.pressure, what='pressure')
    m = proj.metrics()
    assert m['solver'] == 'JACOBI' and m['pressure_storage'] == 'LEGACY'


@pytest.mark.parametrize('warm', ['AUTO', 'LEGACY'])
def test_multigrid_projector_matches_oracle(D, warm):
    from fluxfx_b200.backend.multigrid import MultigridPressureProjector
    grid = GridSpec((16, 16, 16))
    s = PressureSettings(pressure_cycles=3, pressure_warm_start=warm)
    g = S.Grid(grid.shape, grid.extent)
    rng = np.random.default_rng(11)
    vel = tuple(rng.uniform(-1, 1, fs).astype(np.float32) for fs in g.face_shapes)
    proj = MultigridPressureProjector(grid, s, D)
    ref = O.OracleProjector(g, s, 'MULTIGRID')
    assert [lv['shape'] for lv in proj.levels] == list(ref.levels)
    fields = [D.texture(fs, v.ravel(), nonnegative=False) for fs, v in zip(grid.face_shapes, vel)]
    outs = [D.texture(fs) for fs in grid.face_shapes]
    for dt in (0.04, 0.04, 0.025):
        proj.project(fields, outs, dt)
        eo, eb, ea = ref.project(vel, dt)
        for a in range(3):
            assert_close(n(outs[a]), eo[a], what=f'velocity {a}')
        assert float(np.abs(n(proj.after) - ea).max()) <= 1e-5 * float(np.abs(eb).max()), 'after'
    m = proj.metrics()
    assert m['v_cycles'] == 3 and m['levels'][-1] == (4, 4, 4) and m['ratio'] < 0.05


def test_multigrid_tolerance_mode_reaches_target(D):
    from fluxfx_b200.backend.multigrid import MultigridPressureProjector
    grid = GridSpec((32, 32, 32))
    s = PressureSettings(pressure_tolerance=1e-4, pressure_max_cycles=40)
    g = S.Grid(grid.shape, grid.extent)
    rng = np.random.default_rng(12)
    vel = tuple(rng.uniform(-1, 1, fs).astype(np.float32) for fs in g.face_shapes)
    proj = MultigridPressureProjector(grid, s, D)
    ref = O.OracleProjector(g, s, 'MULTIGRID')
    fields = [D.texture(fs, v.ravel(), nonnegative=False) for fs, v in zip(grid.face_shapes, vel)]
    outs = [D.texture(fs) for fs in grid.face_shapes]
    proj.project(fields, outs, 0.04)
    ref.project(vel, 0.04)
    m = proj.metrics()
    assert m['rel_div_inf'] <= 1.2e-4, m
    assert abs(proj.last_cycles - ref.last_cycles) <= 1


def test_solid_multigrid_projector_matches_oracle(D):
    from fluxfx_b200.backend.collision import SolidDevice
    from fluxfx_b200.backend.solid_multigrid import SolidMultigridProjector
    grid = GridSpec((24, 20, 16))
    cols = sphere_box_mask(grid.shape, grid.extent)
    sd = SolidDevice(grid, cols, D)
    s = PressureSettings(pressure_cycles=2)
    mask = n(sd.mask).astype(bool)
    g = S.Grid(grid.shape, grid.extent, mask=mask)
    proj = SolidMultigridProjector(grid, s, sd)
    ref = O.OracleProjector(g, s, 'SOLID_MULTIGRID')
    assert [lv['shape'] for lv in proj.levels] == list(ref.levels)
    for i in range(len(proj.levels)):
        assert np.array_equal(proj.level_edges(i), ref.mg.levels[i][1])
    rng = np.random.default_rng(13)
    vel = S.walls(g, tuple(rng.uniform(-1, 1, fs).astype(np.float32) for fs in g.face_shapes))
    fields = [D.texture(fs, v.ravel(), nonnegative=False) for fs, v in zip(grid.face_shapes, vel)]
    outs = [D.texture(fs) for fs in grid.face_shapes]
    for dt in (0.02, 0.02):
        proj.project(fields, outs, dt)
        eo, eb, ea = ref.project(vel, dt)
        assert proj.last_cycles == ref.last_cycles
        for a in range(3):
            assert_close(n(outs[a]), eo[a], what=f'velocity {a}')
            # zero normal velocity on solid faces (collision_validate.py:47-59)
            x, y, z = g.coords(g.face_shapes[a])
            blocked = S.solid_face(g, x, y, z, a)
            assert np.abs(n(outs[a])[blocked]).max(initial=0) == 0
    m = proj.metrics()
    assert m['solver'] == 'SOLID_MULTIGRID' and m['ratio'] < 0.2


SMOKE_CASES = {
    'mg_maccormack_target': dict(shape=(16, 16, 16), colliders=False, sources=False,
                                 settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK',
                                               density_mode='TARGET', heat_mode='TARGET', source_rate=1.0,
                                               heat_source_rate=1.0, source_profile='SOLID', thermal_lift=1.0,
                                               density_weight=0.05, source_radius=0.2,
                                               source_center=(.5, .5, .2), pressure_cycles=4)),
    'colliders_maccormack': dict(shape=(24, 20, 16), colliders=True, sources=False,
                                 settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK',
                                               thermal_lift=0.5, density_weight=0.1, source_radius=0.15,
                                               source_center=(.3, .5, .2), heat_source_rate=10.0)),
    'table_semi_lagrangian': dict(shape=(20, 16, 12), colliders=False, sources=True,
                                  settings=dict(thermal_lift=0.2, pressure_iterations=40)),
}


@pytest.mark.parametrize('case', sorted(SMOKE_CASES))
def test_smoke_step_matches_oracle(D, case):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.physics.emission import Emission, Source, pack_sources
    spec = SMOKE_CASES[case]
    grid = GridSpec(spec['shape'])
    s = PressureSettings(**spec['settings'])
    cols = sphere_box_mask(grid.shape, grid.extent) if spec['colliders'] else ()
    solver = DenseProjectedSmoke(grid, s, D, colliders=cols)
    mask = n(solver.solids.mask).astype(bool) if cols else None
    ref = O.OracleSmoke(grid.shape, grid.extent, s, np.float32, mask=mask)
    assert ref.kind == {'mg_maccormack_target': 'MULTIGRID', 'colliders_maccormack': 'SOLID_MULTIGRID',
                        'table_semi_lagrangian': 'JACOBI'}[case]
    rng = np.random.default_rng(14)
    vel = tuple((rng.uniform(-1, 1, fs) * 0.3).astype(np.float32) for fs in ref.g.face_shapes)
    solver.upload_velocity(_faces_from(ref.g, vel))
    ref.upload(velocity=vel)
    srcs = None
    table = None
    if spec['sources']:
        srcs = [Source((.3, .5, .25), .15, 1.0, 2.0, Emission((.3, .5, .25)), 'TARGET', 'SOFT'),
                Source((.7, .4, .3), .12, .5, 1.0, Emission((.68, .4, .3), (0, 0, 1), 1.5))]
        table = (pack_sources(srcs), 2)
    for k, dt in enumerate((0.02, 0.02, 0.015)):
        solver.step(dt, sources=srcs)
        ref.step(dt, sources=table)
        for name, got, exp in (('density', solver.density, ref.density), ('temperature', solver.temperature,
                                                                           ref.temperature)):
            assert_close(n(got), exp, rel=STEP_REL, what=f'step {k} {name}')
        for a in range(3):
            assert_close(n(solver._velocity[a]), ref.velocity[a], rel=STEP_REL, what=f'step {k} velocity {a}')
        # the divergence after projection is a residual near zero: bound its
        # error by the scale of the divergence before projection
        err = float(np.abs(n(solver.projector.after) - ref.after).max())
        assert err <= 1e-5 * float(np.abs(ref.before).max()), f'step {k} divergence after: {err:.3e}'
    m = solver.measure_projection()
    assert m['step'] == 3 and math.isfinite(m['rms_after'])
    if cols:
        d = n(solver.density)
        assert (d[mask] == 0).all() and (n(solver.temperature)[mask] == 0).all()


def test_collision_api_behaviour(D):
    """scripts/collision_validate.py: mask parity, upload clears solids, slab leak, degenerate masks."""
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.physics.collision import Collider, primitive, raster_reference
    grid = GridSpec((24, 20, 16))
    c = math.sqrt(.5)
    rotated = Collider('BOX', ((c / .18, c / .18, 0, -c / .18), (-c / .1, c / .1, 0, 0), (0, 0, 1 / .2, -.5 / .2)))
    shapes = (primitive('SPHERE', (.35, .5, .5), (.17,) * 3), rotated)
    s = PressureSettings(velocity=(0, 0, .5), angular_speed=0, source_rate=2, heat_source_rate=100,
                         initial_temperature=50, pressure_iterations=240, thermal_lift=0, density_weight=0)
    solver = DenseProjectedSmoke(grid, s, D, colliders=shapes)
    mask = D.read(solver.solids.mask, grid.shape)
    assert mask == raster_reference(grid, shapes)
    assert solver.projector.uses_impulse
    solver.upload([1.0] * grid.cells)
    solver.upload_temperature([-4.0] * grid.cells)
    assert all(v == 0 for m, v in zip(mask, solver.read_density()) if m)
    assert all(v == 0 for m, v in zip(mask, solver.read_temperature()) if m)
    solver.step(.01)
    first = solver.measure_projection()
    assert first['ratio'] < .1
    for _ in range(19):
        solver.step(.01)
    dens, heat = solver.read_density(), solver.read_temperature()
    assert all(d == 0 and h == 0 for m, d, h in zip(mask, dens, heat) if m)
    assert all(math.isfinite(v) for v in dens + heat) and min(dens) >= 0
    solver.close()
    # a full slab separates two chambers; a trace longer than one cell must not leak through
    grid = GridSpec((32,) * 3)
    slab = primitive('BOX', (.5, .5, .5), (.6, .6, .025))
    s2 = replace(s, source_rate=0, heat_source_rate=0, initial_temperature=0, dissipation=0,
                 scalar_advection='MACCORMACK')
    solver = DenseProjectedSmoke(grid, s2, D, colliders=(slab,))
    solver.upload([float(z < 15) for z in range(32) for y in range(32) for x in range(32)])
    vel = [[1.0 if a == 2 else 0.0] * math.prod(sh) for a, sh in enumerate(grid.face_shapes)]
    solver.upload_velocity(vel)
    for _ in range(3):
        solver.step(.1)
    values = solver.read_density()
    assert max(values[17 * 32 * 32:]) == 0
    solver.close()
    # all-solid domain and one isolated fluid cell stay finite
    solver = DenseProjectedSmoke(GridSpec((8,) * 3), s2, D, colliders=(primitive('BOX', (.5,) * 3, (1,) * 3),))
    solver.step(.01)
    assert all(v == 0 for v in solver.read_density())
    assert all(v == 0 for v in D.read(solver.projector.pressure))
    solver.close()


def test_multigrid_operator_dispatch(D):
    """scripts/multigrid_operators_validate.py through device.dispatch."""
    from fluxfx_b200.backend.multigrid import MultigridPressureProjector
    from oracle.smoke import Grid, residual
    grid = GridSpec((8, 8, 8), (1.3, .8, 1.7))
    mg = MultigridPressureProjector(grid, PressureSettings(pressure_warm_start="LEGACY", pressure_cycles=4), D)
    pressure = [math.sin(i * .21) for i in range(512)]
    rhs = [math.sin(i * .13) for i in range(512)]
    p = D.texture(grid.shape, pressure, nonnegative=False)
    b = D.texture(grid.shape, rhs, nonnegative=False)
    out = D.texture(grid.shape)
    D.dispatch(mg.residual_kernel, out, grid.shape, {'invCell': mg.inv_cell, 'dt': .04}, p,
               sources={'divergenceField': b})
    g64 = Grid(grid.shape, grid.extent, np.float64)
    exp = residual(g64, np.array(pressure).reshape(8, 8, 8), np.array(rhs).reshape(8, 8, 8), .04, g64.inv)
    assert np.abs(np.array(D.read(out)) - exp.ravel()).max() < 1e-4 * max(1, np.abs(exp).max())
    coarse = D.texture((4, 4, 4))
    D.dispatch(mg.restrict_kernel, coarse, (4, 4, 4), input_field=p)
    P = np.array(pressure).reshape(8, 8, 8)
    assert np.abs(np.array(D.read(coarse)) - S.restrict(P).ravel()).max() < 1e-6
    coarse.fill_(2.0)
    D.dispatch(mg.prolong_kernel, out, grid.shape, input_field=p, sources={'coarseField': coarse})
    assert np.abs(np.array(D.read(out)) - np.array(pressure) - 2).max() < 1e-6
    lin = D.texture((4, 4, 4), [(x + .5) / 4 for z in range(4) for y in range(4) for x in range(4)])
    D.dispatch(mg.prolong_kernel, out, grid.shape, input_field=p, sources={'coarseField': lin})
    expected = [min(.875, max(.125, (x + .5) / 8)) for z in range(8) for y in range(8) for x in range(8)]
    assert max(abs(a - b - c) for a, b, c in zip(D.read(out), pressure, expected)) < 1e-6
    fields = [D.texture(s) for s in grid.face_shapes]
    outputs = [D.texture(s) for s in grid.face_shapes]
    mg.project(fields, outputs, .04)
    assert mg.metrics()['ratio'] == 0
    velocity = [[math.sin(i * .63) * .5 for i in range(math.prod(s))] for s in grid.face_shapes]
    fields = [D.texture(s, v, nonnegative=False) for s, v in zip(grid.face_shapes, velocity)]
    mg.project(fields, outputs, .04)
    assert mg.metrics()['ratio'] < .01
    mg.project(fields, outputs, .02)
    dt_changed = [D.read(f) for f in outputs]
    mg.reset()
    assert not mg.ready and mg.last_dt is None
    mg.project(fields, outputs, .02)
    again = [D.read(f) for f in outputs]
    assert max(abs(a - b) for aa, bb in zip(dt_changed, again) for a, b in zip(aa, bb)) < 1e-6
    mg.settings = replace(mg.settings, pressure_cycles=2)
    mg.project(fields, outputs, .02)
    assert mg.last_cycles == 2


def test_thermal_and_mac_solvers_match_oracle(D):
    """P0.3/P0.4 solver classes step like the oracle (mac_validate.py, thermal_validate.py)."""
    from fluxfx_b200.backend.thermal import DenseThermalAdvection
    from fluxfx_b200.physics.thermal import ThermalSettings
    grid = GridSpec((7, 5, 3))
    s = ThermalSettings(source_center=(.5, .5, .2), source_radius=.3, thermal_lift=.01)
    solver = DenseThermalAdvection(grid, s, D)
    g = S.Grid(grid.shape, grid.extent)
    rng = np.random.default_rng(15)
    vel = tuple(rng.uniform(-.5, .5, fs).astype(np.float32) for fs in g.face_shapes)
    dens = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    temp = rng.uniform(0, 50, g.cell_shape).astype(np.float32)
    solver.upload_velocity([v.ravel() for v in vel])
    solver.upload(dens.ravel())
    solver.upload_temperature(temp.ravel())
    for _ in range(4):
        solver.step(.02)
        adv = [S.mac_advect_velocity_face(g, vel, a, .02) for a in range(3)]
        adv[2] = S.buoyancy(g, adv[2], dens, temp, .02, s.thermal_lift, s.density_weight)
        dens2 = S.mac_advect_density(g, adv, dens, .02, s.source_center, s.source_radius, s.source_rate, s.dissipation)
        temp = S.mac_advect_density(g, adv, temp, .02, s.source_center, s.source_radius, s.heat_source_rate, s.cooling)
        dens, vel = dens2, tuple(adv)
    assert_close(n(solver.density), dens, rel=2e-5)
    assert_close(n(solver.temperature), temp, rel=5e-4)
    for a in range(3):
        assert_close(n(solver._velocity[a]), vel[a], rel=2e-5)
    assert solver.steps == 4 and abs(solver.time - .08) < 1e-12
    with pytest.raises(ValueError):
        solver.upload([-1.0] * grid.cells)
    with pytest.raises(ValueError):
        solver.step(0.2)


@pytest.mark.parametrize('warm', [False, True])
def test_pcg_reaches_the_vcycle_solution_in_fewer_cycles(D, warm):
    """MG-PCG (extension) solves the same collider system as the reference's
    V-cycles: to the same tolerance it gives the same projected velocity."""
    from fluxfx_b200.backend.collision import SolidDevice
    from fluxfx_b200.backend.solid_multigrid import SolidMultigridProjector
    grid = GridSpec((32, 32, 32))
    cols = sphere_box_mask(grid.shape, grid.extent)
    sd = SolidDevice(grid, cols, D)
    base = PressureSettings(pressure_tolerance=1e-6, pressure_max_cycles=200)
    vproj = SolidMultigridProjector(grid, base, sd)
    pproj = SolidMultigridProjector(grid, replace(base, pressure_method='PCG', solid_warm_start=warm), sd)
    g = S.Grid(grid.shape, grid.extent, mask=n(sd.mask).astype(bool))
    rng = np.random.default_rng(31)
    vel = tuple(rng.uniform(-1, 1, fs).astype(np.float32) for fs in g.face_shapes)
    fields = [D.texture(fs, v.ravel(), nonnegative=False) for fs, v in zip(grid.face_shapes, vel)]
    outs_v = [D.texture(fs) for fs in grid.face_shapes]
    outs_p = [D.texture(fs) for fs in grid.face_shapes]
    for dt in (0.02, 0.02, 0.015):
        vproj.project(fields, outs_v, dt)
        pproj.project(fields, outs_p, dt)
        mv, mp = vproj.metrics(), pproj.metrics()
        assert mv['rel_div_inf'] <= 1.5e-6 and mp['rel_div_inf'] <= 1.5e-6, (mv['rel_div_inf'], mp['rel_div_inf'])
        assert pproj.last_cycles < vproj.last_cycles, (pproj.last_cycles, vproj.last_cycles)
        # Two solutions with residuals <= 1e-6 max|div| can differ by low modes of
        # size ~ tol * max|div| * L / pi in velocity (~4e-5 here): bound at 1e-4.
        for a in range(3):
            scale = float(np.abs(n(outs_v[a])).max())
            assert float(np.abs(n(outs_v[a]) - n(outs_p[a])).max()) <= 1e-4 * scale


@pytest.mark.parametrize('sweeps', [(1, 1), (2, 2)])
def test_pcg_with_short_preconditioner_reaches_tolerance(D, sweeps):
    """PCG preconditioned by V(1,1) / V(2,2) aggregation cycles (the last
    sweep fused with the FP64 dot) converges to the tolerance and to the same
    projected velocity as the reference's V(4,4) cycles."""
    from fluxfx_b200.backend.collision import SolidDevice
    from fluxfx_b200.backend.solid_multigrid import SolidMultigridProjector
    grid = GridSpec((32, 32, 32))
    sd = SolidDevice(grid, sphere_box_mask(grid.shape, grid.extent), D)
    base = PressureSettings(pressure_tolerance=1e-6, pressure_max_cycles=200)
    vproj = SolidMultigridProjector(grid, base, sd)
    pproj = SolidMultigridProjector(grid, replace(base, pressure_method='PCG', solid_warm_start=True,
                                                  mg_pre_sweeps=sweeps[0], mg_post_sweeps=sweeps[1]), sd)
    rng = np.random.default_rng(5)
    outs_v = [D.texture(fs) for fs in grid.face_shapes]
    outs_p = [D.texture(fs) for fs in grid.face_shapes]
    for dt in (0.02, 0.015):
        fields = [D.texture(fs, rng.uniform(-1, 1, fs[0] * fs[1] * fs[2]), nonnegative=False)
                  for fs in grid.face_shapes]
        vproj.project(fields, outs_v, dt)
        pproj.project(fields, outs_p, dt)
        assert pproj.metrics()['rel_div_inf'] <= 1.5e-6 and pproj.last_cycles < 200
        for a in range(3):
            scale = float(np.abs(n(outs_v[a])).max())
            assert float(np.abs(n(outs_v[a]) - n(outs_p[a])).max()) <= 1e-4 * scale


@pytest.mark.parametrize('method', ['VCYCLE', 'PCG'])
def test_graph_replay_matches_eager_launches(D, method):
    """The pressure solve replayed from captured CUDA graphs runs the same
    kernels on the same buffers as eager launches: results are bit-identical,
    and so are the cycle counts."""
    from fluxfx_b200.backend.collision import SolidDevice
    from fluxfx_b200.backend.solid_multigrid import SolidMultigridProjector
    grid = GridSpec((32, 24, 16))
    sd = SolidDevice(grid, sphere_box_mask(grid.shape, grid.extent), D)
    s = PressureSettings(pressure_tolerance=1e-5, pressure_max_cycles=60, pressure_method=method,
                         solid_warm_start=method == 'PCG')
    graphed, eager = SolidMultigridProjector(grid, s, sd), SolidMultigridProjector(grid, s, sd)
    eager.use_graphs = False
    rng = np.random.default_rng(7)
    out_g = [D.texture(fs) for fs in grid.face_shapes]
    out_e = [D.texture(fs) for fs in grid.face_shapes]
    for dt in (0.02, 0.02, 0.01):
        # fresh velocities each call, so a warm-started solve still has work to do
        fields = [D.texture(fs, rng.uniform(-1, 1, fs[0] * fs[1] * fs[2]), nonnegative=False)
                  for fs in grid.face_shapes]
        graphed.project(fields, out_g, dt)
        eager.project(fields, out_e, dt)
        assert graphed.last_cycles == eager.last_cycles > 1
        assert graphed.last_iterations == eager.last_iterations
        for a in range(3):
            assert np.array_equal(n(out_g[a]), n(out_e[a])), a
    # V-cycle tolerance solves replay one device-loop graph; PCG iterations replay captured iterations
    assert (graphed._graphs or graphed._loops) and not eager._graphs and not eager._loops
    graphed.close()
    eager.close()


@pytest.mark.parametrize('method,coarse', [('VCYCLE', 'DIRECT'), ('PCG', 'DIRECT'), ('VCYCLE', 'SMOOTH')])
def test_coarse_tail_matches_per_level_launches(D, method, coarse):
    """The small coarse levels run as one single-block launch (ffx_graph_tail);
    the solve is bit-identical to launching every pass of those levels."""
    from fluxfx_b200.backend.collision import SolidDevice
    from fluxfx_b200.backend.solid_multigrid import SolidMultigridProjector
    grid = GridSpec((32, 32, 32))
    sd = SolidDevice(grid, sphere_box_mask(grid.shape, grid.extent), D)
    s = PressureSettings(pressure_tolerance=1e-5, pressure_max_cycles=40, pressure_method=method,
                         coarse_solver=coarse)
    tail, plain = SolidMultigridProjector(grid, s, sd), SolidMultigridProjector(grid, s, sd)
    plain.use_tail = False
    assert [lv['shape'] for lv in tail.levels] == [(32, 32, 32), (16, 16, 16), (8, 8, 8), (4, 4, 4)]
    assert tail.tail_start == 2
    assert (tail.coarse_matrix is not None) == (coarse == 'DIRECT')
    rng = np.random.default_rng(11)
    out_t = [D.texture(fs) for fs in grid.face_shapes]
    out_p = [D.texture(fs) for fs in grid.face_shapes]
    for dt in (0.02, 0.01):
        fields = [D.texture(fs, rng.uniform(-1, 1, fs[0] * fs[1] * fs[2]), nonnegative=False)
                  for fs in grid.face_shapes]
        tail.project(fields, out_t, dt)
        plain.project(fields, out_p, dt)
        assert tail.last_cycles == plain.last_cycles > 1
        assert tail.last_iterations == plain.last_iterations
        for a in range(3):
            assert np.array_equal(n(out_t[a]), n(out_p[a])), a
    tail.close()
    plain.close()
