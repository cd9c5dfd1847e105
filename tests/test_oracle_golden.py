"""Pin the NumPy oracle (FP64) to golden vectors produced by the reference's own
pure-Python CPU code (tests/golden/make_golden.py). CPU only."""
from pathlib import Path

import numpy as np
import pytest

from oracle import smoke as S
from oracle import solver as O

GOLD = Path(__file__).resolve().parent / 'golden'
TOL = 1e-12


def load(name):
    return np.load(GOLD / f'{name}.npz')


def faces(g, d, keys):
    return tuple(np.asarray(d[k], dtype=np.float64).reshape(fs) for k, fs in zip(keys, g.face_shapes))


def cells(g, arr):
    return np.asarray(arr, dtype=np.float64).reshape(g.cell_shape)


def test_open_advection_matches_reference():
    d = load('advect_open')
    g = S.Grid(tuple(d['shape']), tuple(d['extent']), np.float64)
    out = S.advect_open(g, cells(g, d['field']), float(d['dt']), tuple(d['velocity']), float(d['angular']),
                        tuple(d['center']), float(d['radius']), float(d['rate']), float(d['decay']))
    assert np.abs(out.ravel() - d['result']).max() < TOL
    moved = S.advect_open(g, cells(g, d['impulse']), 0.1, (1.25, 0, 0), 0.0, tuple(d['center']),
                          float(d['radius']), 0.0, 0.0)
    assert np.abs(moved.ravel() - d['moved']).max() < TOL
    assert abs(moved.ravel()[3 + 8 * (2 + 6 * 1)] - 1.0) < 1e-12


def test_mac_self_advection_and_density_match_reference():
    d = load('mac')
    g = S.Grid(tuple(d['shape']), tuple(d['extent']), np.float64)
    vel = faces(g, d, ('u', 'v', 'w'))
    for axis, key in enumerate(('au', 'av', 'aw')):
        out = S.mac_advect_velocity_face(g, vel, axis, float(d['dt']))
        assert np.abs(out.ravel() - d[key]).max() < TOL
    res = S.mac_advect_density(g, vel, cells(g, d['density']), float(d['dt']), tuple(d['center']),
                               float(d['radius']), float(d['rate']), float(d['decay']))
    assert np.abs(res.ravel() - d['dresult']).max() < TOL
    seeded = S.seed_faces(g, tuple(d['seed_velocity']), float(d['seed_angular']))
    for axis, key in enumerate(('su', 'sv', 'sw')):
        assert np.abs(seeded[axis].ravel() - d[key]).max() < TOL


def test_thermal_step_matches_reference():
    d = load('thermal')
    g = S.Grid(tuple(d['shape']), tuple(d['extent']), np.float64)
    dt = float(d['dt'])
    vel = faces(g, d, ('u', 'v', 'w'))
    adv = tuple(S.mac_advect_velocity_face(g, vel, a, dt) for a in range(3))
    w = S.buoyancy(g, adv[2], cells(g, d['density']), cells(g, d['temperature']), dt,
                   float(d['lift']), float(d['weight']))
    new = (adv[0], adv[1], w)
    for axis, key in enumerate(('u2', 'v2', 'w2')):
        assert np.abs(new[axis].ravel() - d[key]).max() < TOL
    dens = S.mac_advect_density(g, new, cells(g, d['density']), dt, tuple(d['center']), float(d['radius']),
                                float(d['rate']), float(d['decay']))
    temp = S.mac_advect_density(g, new, cells(g, d['temperature']), dt, tuple(d['center']), float(d['radius']),
                                float(d['heat_rate']), float(d['cooling']))
    assert np.abs(dens.ravel() - d['d2']).max() < TOL
    assert np.abs(temp.ravel() - d['t2']).max() < 1e-10


def test_projection_pieces_match_reference():
    d = load('pressure')
    g = S.Grid(tuple(d['shape']), tuple(d['extent']), np.float64)
    vel = faces(g, d, ('u', 'v', 'w'))
    bounded = S.walls(g, vel)
    for a, k in enumerate(('bu', 'bv', 'bw')):
        assert np.array_equal(bounded[a].ravel(), d[k])
    div = S.divergence(g, bounded)
    assert np.abs(div.ravel() - d['div']).max() < 1e-11
    p = cells(g, d['p'])
    lap = S.residual(g, p, np.zeros_like(p), 1.0, g.inv)
    assert np.abs(-lap.ravel() - d['lap']).max() < 1e-10
    grad = S.gradient(g, tuple(np.zeros(fs) for fs in g.face_shapes), p, -1.0)
    for a, k in enumerate(('gu', 'gv', 'gw')):
        assert np.abs(grad[a].ravel() - d[k]).max() < 1e-11
    dt = float(d['dt'])
    q = np.zeros_like(div)
    for _ in range(int(d['iterations'])):
        q = S.jacobi(g, q, div, dt, 2 / 3)
    assert np.abs(q.ravel() - d['solved']).max() < 1e-9
    corrected = S.gradient(g, bounded, q, dt)
    for a, k in enumerate(('cu', 'cv', 'cw')):
        assert np.abs(corrected[a].ravel() - d[k]).max() < 1e-10


def test_coarse_inverse_matches_reference():
    from fluxfx_b200.physics.coarse_pressure import coarse_inverse, neumann_inverse
    d = load('coarse_inverse')
    assert np.abs(np.array(coarse_inverse((1., 1., 1.))) - d['unit']).max() < 1e-15
    assert np.abs(np.array(coarse_inverse((1.3, .8, 1.7))) - d['skew']).max() < 1e-15
    # the generalised closed form is a true Neumann pseudoinverse at 8^3 as well
    inv = neumann_inverse((8, 4, 6), (1., .5, 2.))
    g = S.Grid((8, 4, 6), (1., .5, 2.), np.float64)
    rhs = np.sin(np.arange(8 * 4 * 6) * .37)
    rhs -= rhs.mean()
    p = (inv @ rhs).reshape(g.cell_shape)
    lap = -S.residual(g, p, np.zeros_like(p), 1.0, g.inv)
    assert abs(p.sum()) < 1e-10
    assert np.abs(lap.ravel() - rhs).max() < 1e-10


@pytest.mark.parametrize('name', ['cube', 'slab', 'disconnected', 'sphere'])
def test_aggregation_hierarchy_matches_reference(name):
    d = load('solid_hierarchy')
    shape = tuple(int(v) for v in d[f'{name}_shape'])
    extent = tuple(float(v) for v in d[f'{name}_extent'])
    mask = np.asarray(d[f'{name}_mask']).reshape(shape[2], shape[1], shape[0]) > 0.5
    levels = S.build_hierarchy(shape, extent, mask)
    assert len(levels) == int(d[f'{name}_levels'])
    for i, (sh, edges) in enumerate(levels):
        assert tuple(sh) == tuple(int(v) for v in d[f'{name}_level{i}_shape'])
        assert np.array_equal(edges.ravel(), d[f'{name}_level{i}_edges'])     # bit-exact
    if f'{name}_inverse' in d:
        inv = S.graph_inverse(*levels[-1])
        assert np.abs(inv.astype(np.float32).ravel() - d[f'{name}_inverse']).max() < 1e-6


def test_raster_matches_reference_bit_exact():
    d = load('raster')
    g = S.Grid(tuple(d['shape']), tuple(d['extent']), np.float64)
    m = S.raster_mask(g, [('BOX', d['rows_a']), ('SPHERE', d['rows_b'])])
    assert np.array_equal(m.ravel().astype(np.float64), d['union'])
    g2 = S.Grid(tuple(d['shape2']), tuple(d['extent2']), np.float64)
    m2 = S.raster_mask(g2, [('SPHERE', d['rows_sphere']), ('BOX', d['rows_rotated'])])
    assert np.array_equal(m2.ravel().astype(np.float64), d['scene'])
    assert m2.sum() > 0


def test_emitter_table_and_timestep_policy_match_reference():
    from fluxfx_b200.physics.emission import Source, Emission, pack_sources
    from fluxfx_b200.physics.timestep import choose_timestep
    d = load('emission_timestep')
    srcs = [Source((.5, .4, .3), .1, 1, -10, Emission((.45, .4, .3), (0, 0, 1), 2.5), 'TARGET', 'SOLID', .25),
            Source((.2, .6, .7), .2, .5, 3, Emission((.2, .6, .7)))]
    assert np.array_equal(np.array(pack_sources(srcs)), d['table'])
    dts = [choose_timestep(0.05, 0.8, r, a, quantized=q)
           for r in (0.0, 3.0, 40.0) for a in (0.0, 50.0) for q in (True, False)]
    assert np.array_equal(np.array(dts), d['dts'])


def test_fp32_oracle_tracks_fp64():
    """The FP32 mirror of the kernels stays within FP32 rounding of the FP64 run."""
    d = load('mac')
    for dtype in (np.float32, np.float64):
        g = S.Grid(tuple(d['shape']), tuple(d['extent']), dtype)
        vel = tuple(np.asarray(d[k], dtype=dtype).reshape(fs) for k, fs in zip(('u', 'v', 'w'), g.face_shapes))
        out = S.mac_advect_velocity_face(g, vel, 0, float(d['dt']))
        if dtype is np.float32:
            assert out.dtype == np.float32
            o32 = out
        else:
            assert np.abs(o32 - out).max() < 1e-5


def test_solver_oracle_projection_removes_divergence():
    from fluxfx_b200.physics.pressure import PressureSettings
    s = PressureSettings(pressure_cycles=6, pressure_warm_start='LEGACY')
    g = S.Grid((16, 16, 16), (1., 1., 1.), np.float64)
    rng = np.random.default_rng(0)
    vel = tuple(rng.uniform(-1, 1, fs) for fs in g.face_shapes)
    proj = O.OracleProjector(g, s, 'MULTIGRID')
    out, before, after = proj.project(vel, 0.04)
    assert np.abs(after).max() < 0.05 * np.abs(before).max()
    # tolerance mode reaches the stated relative max-norm divergence
    s2 = PressureSettings(pressure_tolerance=1e-6, pressure_max_cycles=40)
    proj2 = O.OracleProjector(g, s2, 'MULTIGRID')
    out, before, after = proj2.project(vel, 0.04)
    assert np.abs(after).max() <= 1.01e-6 * np.abs(before).max()
