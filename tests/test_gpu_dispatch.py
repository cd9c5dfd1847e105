"""Single-pass dispatch by reference shader name, as the reference's scripts
drive it (``device.dispatch(kernel, output, shape, uniforms, input_field,
sources)`` with the reference's uniform and sampler names, on a solver's own
device, handles and uniform helpers: ``_face_uniforms``, ``_source_uniforms``,
``_emitting_velocity``, ``_closed_scalar``). Every pass matches the oracle's
pass, with and without colliders (the collider device's mask)."""
import numpy as np
import pytest
import torch

from fluxfx_b200.backend.mac import VELOCITY_NAMES
from oracle import smoke as S
from tests.gpu_helpers import assert_close, dev, n, random_faces, sphere_box_mask, t

pytestmark = pytest.mark.gpu

SHAPE, EXTENT = (12, 10, 8), (1.3, 0.8, 1.7)


def _solver(masked):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.physics.config import GridSpec
    from fluxfx_b200.physics.pressure import PressureSettings
    grid = GridSpec(SHAPE, EXTENT)
    settings = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK',
                                source_center=(.5 * EXTENT[0], .45 * EXTENT[1], .3 * EXTENT[2]),
                                source_radius=.2 * min(EXTENT))
    colliders = sphere_box_mask(SHAPE, EXTENT) if masked else ()
    solver = DenseProjectedSmoke(grid, settings, dev(), colliders=colliders)
    mask = n(solver.solids.mask).astype(bool) if masked else None
    return solver, grid, S.Grid(SHAPE, EXTENT, mask=mask)


def _zeros(shape_zyx):
    return t(np.zeros(shape_zyx, dtype=np.float32))


@pytest.mark.parametrize('masked', [False, True])
def test_pressure_passes_by_shader_name(masked):
    solver, grid, g = _solver(masked)
    d = solver.device
    rng = np.random.default_rng(11)
    vel = random_faces(g, rng, 0.6)
    vel_t = [t(v) for v in vel]
    inv = tuple(float(v) for v in g.inv)
    walls = d.kernel('pressure_walls.glsl')
    bounded = [_zeros(fs) for fs in g.face_shapes]
    for a, shape in enumerate(grid.face_shapes):
        d.dispatch(walls, bounded[a], shape, {'componentAxis': float(a)}, vel_t[a])
    exp_b = S.walls(g, vel)
    for a in range(3):
        assert_close(n(bounded[a]), exp_b[a], what=f'walls {a}')
    div = _zeros(g.cell_shape)
    d.dispatch(d.kernel('pressure_divergence.glsl'), div, grid.shape, {'invCell': inv},
               sources=dict(zip(VELOCITY_NAMES, bounded)))
    assert_close(n(div), S.divergence(g, exp_b), rel=1e-6, what='divergence')
    p = rng.uniform(-1, 1, g.cell_shape).astype(np.float32)
    p_t = t(p)
    grad = d.kernel('pressure_gradient.glsl')
    outs = [_zeros(fs) for fs in g.face_shapes]
    for a, shape in enumerate(grid.face_shapes):
        d.dispatch(grad, outs[a], shape, {'invCell': inv, 'dt': 1.0, 'componentAxis': float(a)}, bounded[a],
                   sources={'pressureField': p_t})
    exp_g = S.gradient(g, exp_b, p, 1.0)
    for a in range(3):
        assert_close(n(outs[a]), exp_g[a], rel=1e-6, what=f'gradient {a}')
    solver.close()


@pytest.mark.parametrize('masked', [False, True])
def test_transport_passes_by_shader_name(masked):
    solver, grid, g = _solver(masked)
    d = solver.device
    s = solver.settings
    rng = np.random.default_rng(12)
    vel = random_faces(g, rng, 0.6)
    vel_t = [t(v) for v in vel]
    velocities = dict(zip(VELOCITY_NAMES, vel_t))
    dt = 0.04
    # face predictors (detail.transport_velocity's passes)
    face = d.kernel('transport_face.glsl')
    preds = [_zeros(fs) for fs in g.face_shapes]
    for a, shape in enumerate(grid.face_shapes):
        d.dispatch(face, preds[a], shape, solver._face_uniforms(a) | {'dt': dt}, vel_t[a], sources=velocities)
    exp_p = [S.face_predictor(g, vel, a, dt) for a in range(3)]
    for a in range(3):
        assert_close(n(preds[a]), exp_p[a], what=f'face predictor {a}')
    # the emitting velocity pass, MacCormack, single swept emitter with a jet
    start = (.45 * EXTENT[0], .4 * EXTENT[1], .28 * EXTENT[2])
    outs = [_zeros(fs) for fs in g.face_shapes]
    for a, shape in enumerate(grid.face_shapes):
        d.dispatch(solver._emitting_velocity, outs[a], shape,
                   solver._face_uniforms(a) | {'dt': dt, 'correctedVelocity': 1.0, 'sourceCenter': s.source_center,
                                               'sourceStart': start, 'sourceRadius': s.source_radius,
                                               'sourceProfile': 0.0, 'emissionVelocity': (0.1, -0.2, 0.7),
                                               'emissionCoupling': 3.0},
                   sources=velocities | {'originalFaceField': vel_t[a], 'facePredictor': preds[a]})
    em = dict(center=s.source_center, start=start, radius=s.source_radius, solid=False, jet=(0.1, -0.2, 0.7),
              coupling=3.0)
    for a in range(3):
        exp = S.advect_velocity_face(g, vel, exp_p[a], a, dt, True, 0.5, emitter=em)
        assert_close(n(outs[a]), exp, what=f'emitting velocity {a}')
    # buoyancy on W
    dens = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    temp = rng.uniform(0, 2, g.cell_shape).astype(np.float32)
    if masked:
        dens = np.where(g.mask, 0, dens).astype(np.float32)
        temp = np.where(g.mask, 0, temp).astype(np.float32)
    dens_t, temp_t = t(dens), t(temp)
    w_out = _zeros(g.face_shapes[2])
    d.dispatch(d.kernel('buoyancy.glsl'), w_out, grid.face_shapes[2],
               {'dt': dt, 'thermalLift': 0.4, 'densityWeight': 0.1}, vel_t[2],
               sources={'densityField': dens_t, 'temperatureField': temp_t})
    assert_close(n(w_out), S.buoyancy(g, vel[2], dens, temp, dt, 0.4, 0.1), what='buoyancy')
    # the scalar passes: detail.transport (transport_scalar.glsl twice) and the closed scalar pass
    corr = solver.detail.transport(dens_t, velocities, dt)
    ep = S.scalar_transport(g, vel, dens, dt)
    er = S.scalar_transport(g, vel, ep, -dt)
    assert_close(n(corr['predictorField']), ep, what='scalar predictor')
    assert_close(n(corr['reverseField']), er, what='scalar reverse')
    out = _zeros(g.cell_shape)
    uniforms = solver._source_uniforms() | {'cellCount': grid.shape, 'dt': dt, 'sourceStart': s.source_center,
                                            'sourceRate': 1.0, 'dissipation': 0.1, 'correctedTransport': 1.0,
                                            'sourceProfile': 1.0, 'targetDensity': 1.0}
    d.dispatch(solver._closed_scalar, out, grid.shape, uniforms, dens_t, sources=velocities | corr)
    em = dict(center=s.source_center, start=s.source_center, radius=s.source_radius, solid=True)
    exp = S.advect_scalar(g, vel, dens, ep, er, dt, True, 1.0, 0.1, 1.0, emitter=em)
    assert_close(n(out), exp, what='closed scalar')
    solver.close()


def test_table_passes_and_fence_by_shader_name():
    from fluxfx_b200.physics.emission import Emission, Source, pack_sources
    solver, grid, g = _solver(False)
    d = solver.device
    rng = np.random.default_rng(13)
    vel = random_faces(g, rng, 0.5)
    vel_t = [t(v) for v in vel]
    velocities = dict(zip(VELOCITY_NAMES, vel_t))
    dt = 0.04
    srcs = [Source((.3 * EXTENT[0], .5 * EXTENT[1], .3 * EXTENT[2]), .15 * min(EXTENT), 1, 2,
                   Emission((.32 * EXTENT[0], .5 * EXTENT[1], .3 * EXTENT[2]), (0, 0, 1), 2.0), 'TARGET', 'SOLID'),
            Source((.6 * EXTENT[0], .4 * EXTENT[1], .5 * EXTENT[2]), .2 * min(EXTENT), .5, 1,
                   Emission((.6 * EXTENT[0], .4 * EXTENT[1], .5 * EXTENT[2]), (0.5, 0, 0), 1.0))]
    solver._prepare_sources(srcs)
    table = pack_sources(srcs)
    outs = [_zeros(fs) for fs in g.face_shapes]
    for a, shape in enumerate(grid.face_shapes):
        d.dispatch(solver._multi_velocity, outs[a], shape,
                   solver._face_uniforms(a) | {'dt': dt, 'sourceCount': 2.0, 'correctedVelocity': 0.0},
                   sources=velocities | {'sourceTable': solver._source_table, 'originalFaceField': vel_t[a],
                                         'facePredictor': vel_t[a]})
    for a in range(3):
        exp = S.advect_velocity_face(g, vel, vel[a], a, dt, False, 0.5, sources=(table, 2))
        assert_close(n(outs[a]), exp, what=f'table velocity {a}')
    dens = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    dens_t = t(dens)
    out = _zeros(g.cell_shape)
    d.dispatch(solver._multi_scalar, out, grid.shape,
               {'domainExtent': grid.extent, 'cellCount': grid.shape, 'dt': dt, 'sourceCount': 2.0,
                'scalarChannel': 0.0, 'correctedTransport': 0.0, 'dissipation': 0.0},
               dens_t, sources=velocities | {'sourceTable': solver._source_table})
    exp = S.advect_scalar(g, vel, dens, dens, dens, dt, False, 0.0, 0.0, -1.0, sources=(table, 2), channel=0)
    assert_close(n(out), exp, what='table scalar')
    pixel = _zeros((1, 1, 1))
    d.dispatch(d.kernel('benchmark_fence.glsl'), pixel, (1, 1, 1),
               sources={'densityField': dens_t, 'velocityU': vel_t[0], 'velocityV': vel_t[1],
                        'velocityW': vel_t[2]})
    want = np.float32(dens.flat[0]) + np.float32(vel[0].flat[0]) + np.float32(vel[1].flat[0]) + \
        np.float32(vel[2].flat[0])
    assert abs(float(n(pixel).ravel()[0]) - float(want)) <= 1e-6 * max(1.0, abs(float(want)))
    solver.close()
