"""Per-pass parity: every native entry point against the CPU oracle (FP32 mirror)
on the same seeded inputs, through the C ABI."""
import ctypes as C

import numpy as np
import pytest
import torch

from fluxfx_b200 import _native as N
from oracle import smoke as S
from tests.gpu_helpers import assert_close, dev, grid_ptr, n, random_faces, solids, sphere_box_mask, t

pytestmark = pytest.mark.gpu

SHAPES = [((7, 5, 3), (1.0, 1.0, 1.0)), ((12, 10, 8), (1.3, 0.8, 1.7)), ((16, 16, 16), (1.0, 1.0, 1.0))]


def ptr(x):
    return C.c_void_p(0 if x is None else x.data_ptr())


@pytest.fixture(scope='module')
def D():
    return dev()


def test_probe_and_device_info(D):
    report = D.probe_3d()
    assert report['status'] == 'PASS'
    assert D.sm_count >= 1


def test_seeds_match_oracle(D):
    shape, extent = (12, 10, 8), (1.3, 0.8, 1.7)
    g = S.Grid(shape, extent)
    gs, gp = grid_ptr(shape, extent)
    out = t(np.zeros(g.cell_shape))
    D.call('ffx_seed_scalar', gp, 0, N.f3(.6, .4, .9), 0.5, 3.0, ptr(out), D.s)
    assert_close(n(out), S.seed_scalar(g, (.6, .4, .9), 0.5, 3.0), rel=1e-6)
    faces = [t(np.zeros(fs)) for fs in g.face_shapes]
    D.call('ffx_seed_faces', gp, 0, N.f3(.2, -.3, .4), 0.7, *map(ptr, faces), D.s)
    for a, o in zip(faces, S.seed_faces(g, (.2, -.3, .4), 0.7)):
        assert_close(n(a), o, rel=1e-6)


def test_raster_and_halo_bit_exact(D):
    from fluxfx_b200.backend.collision import collider_rows
    from fluxfx_b200.physics.collision import raster_reference
    from fluxfx_b200.physics.config import GridSpec
    from pathlib import Path
    gold = np.load(Path(__file__).parent / 'golden' / 'raster.npz')
    for shape, extent, rows, key in (((8, 6, 4), (2., 1., 1.), [('BOX', gold['rows_a']), ('SPHERE', gold['rows_b'])],
                                      'union'),
                                     ((24, 20, 16), (1., 1., 1.), [('SPHERE', gold['rows_sphere']),
                                                                   ('BOX', gold['rows_rotated'])], 'scene')):
        from fluxfx_b200.physics.collision import Collider
        cols = [Collider(sh, tuple(tuple(float(v) for v in r) for r in rr)) for sh, rr in rows]
        nx, ny, nz = shape
        mask = torch.zeros((nz, ny, nx), dtype=torch.uint8, device='cuda')
        rows_t = torch.tensor(collider_rows(cols), dtype=torch.float64, device='cuda')
        gs, gp = grid_ptr(shape, extent)
        D.call('ffx_raster_colliders', gp, (C.c_double * 3)(*extent), len(cols), ptr(rows_t), ptr(mask), D.s)
        got = n(mask).ravel()
        assert np.array_equal(got, gold[key]), key
        assert np.array_equal(got, np.array(raster_reference(GridSpec(shape, extent), cols)))
        halo = torch.zeros_like(mask)
        D.call('ffx_dilate_mask', gp, ptr(mask), ptr(halo), D.s)
        g = S.Grid(shape, extent, mask=n(mask).astype(bool))
        assert np.array_equal(n(halo).astype(bool), g.halo)


@pytest.mark.parametrize('shape,extent', SHAPES)
def test_legacy_transport_matches_oracle(D, shape, extent):
    rng = np.random.default_rng(1)
    g = S.Grid(shape, extent)
    gs, gp = grid_ptr(shape, extent)
    field = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    out = t(np.zeros(g.cell_shape))
    D.call('ffx_advect_open', gp, 0, ptr(t(field)), 0.07, N.f3(.3, -.2, .1), 1.0, N.f3(.5, .5, .4), 0.3, 2.0, 0.1,
           ptr(out), D.s)
    exp = S.advect_open(g, field, 0.07, (.3, -.2, .1), 1.0, (.5, .5, .4), 0.3, 2.0, 0.1)
    assert_close(n(out), exp, rel=2e-6)
    vel = random_faces(g, rng, 0.8)
    outs = [t(np.zeros(fs)) for fs in g.face_shapes]
    D.call('ffx_mac_advect_velocity', gp, 0, *[ptr(t(v)) for v in vel], 0.05, *map(ptr, outs), D.s)
    for a in range(3):
        assert_close(n(outs[a]), S.mac_advect_velocity_face(g, vel, a, 0.05), rel=2e-6)
    D.call('ffx_mac_advect_density', gp, 0, *[ptr(t(v)) for v in vel], ptr(t(field)), 0.05, N.f3(.5, .5, .4), 0.3,
           2.0, 0.1, ptr(out), D.s)
    assert_close(n(out), S.mac_advect_density(g, vel, field, 0.05, (.5, .5, .4), 0.3, 2.0, 0.1), rel=2e-6)
    dens = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    temp = rng.uniform(-5, 5, g.cell_shape).astype(np.float32)
    w_out = t(np.zeros(g.face_shapes[2]))
    D.call('ffx_buoyancy', gp, 0, ptr(t(vel[2])), ptr(t(dens)), ptr(t(temp)), 0.05, 0.3, 0.2, ptr(w_out), D.s)
    assert_close(n(w_out), S.buoyancy(g, vel[2], dens, temp, 0.05, 0.3, 0.2), rel=1e-6)


def _mask_setup(D, shape, extent):
    from fluxfx_b200.backend.collision import collider_rows
    cols = sphere_box_mask(shape, extent)
    nx, ny, nz = shape
    mask = torch.zeros((nz, ny, nx), dtype=torch.uint8, device='cuda')
    halo = torch.zeros_like(mask)
    rows = torch.tensor(collider_rows(cols), dtype=torch.float64, device='cuda')
    gs, gp = grid_ptr(shape, extent)
    D.call('ffx_raster_colliders', gp, (C.c_double * 3)(*extent), len(cols), ptr(rows), ptr(mask), D.s)
    D.call('ffx_dilate_mask', gp, ptr(mask), ptr(halo), D.s)
    return mask, halo


@pytest.mark.parametrize('masked', [False, True])
@pytest.mark.parametrize('shape,extent', SHAPES[1:])
def test_velocity_passes_match_oracle(D, shape, extent, masked):
    rng = np.random.default_rng(2)
    mask_t = halo_t = None
    if masked:
        mask_t, halo_t = _mask_setup(D, shape, extent)
    g = S.Grid(shape, extent, mask=n(mask_t).astype(bool) if masked else None)
    gs, gp = grid_ptr(shape, extent)
    so = solids(mask_t, halo_t)
    vel = random_faces(g, rng, 0.6)
    vel_t = [t(v) for v in vel]
    dt = 0.04
    preds = [t(np.zeros(fs)) for fs in g.face_shapes]
    D.call('ffx_face_predictor', gp, C.byref(so), 0, *map(ptr, vel_t), dt, *map(ptr, preds), D.s)
    exp_pred = [S.face_predictor(g, vel, a, dt) for a in range(3)]
    for a in range(3):
        assert_close(n(preds[a]), exp_pred[a], what=f'predictor {a}')
    dens = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    temp = rng.uniform(0, 2, g.cell_shape).astype(np.float32)
    # single swept emitter with a jet, MacCormack, buoyancy, walls
    src = N.FfxSources()
    src.count = -1
    src.single_solid_profile = 0
    src.single_center = N.f3(.5 * extent[0], .45 * extent[1], .3 * extent[2])
    src.single_start = N.f3(.45 * extent[0], .4 * extent[1], .28 * extent[2])
    src.single_radius = .2 * min(extent)
    src.single_jet = N.f3(0.1, -0.2, 0.7)
    src.single_coupling = 3.0
    outs = [t(np.zeros(fs)) for fs in g.face_shapes]
    D.call('ffx_advect_velocity', gp, C.byref(so), 0, *map(ptr, vel_t), *map(ptr, preds), dt, 1, 0.5,
           C.byref(src), ptr(t(dens)), ptr(t(temp)), 0.4, 0.1, 1, *map(ptr, outs), D.s)
    em = dict(center=tuple(src.single_center), start=tuple(src.single_start), radius=src.single_radius, solid=False,
              jet=(0.1, -0.2, 0.7), coupling=3.0)
    new = [S.advect_velocity_face(g, vel, exp_pred[a], a, dt, True, 0.5, emitter=em) for a in range(3)]
    new[2] = S.buoyancy(g, new[2], dens, temp, dt, 0.4, 0.1)
    new = S.walls(g, tuple(new))
    for a in range(3):
        assert_close(n(outs[a]), new[a], what=f'velocity {a}')
    # source-table form, semi-Lagrangian, no buoyancy, no walls
    from fluxfx_b200.physics.emission import Emission, Source, pack_sources
    srcs = [Source((.3 * extent[0], .5 * extent[1], .3 * extent[2]), .15 * min(extent), 1, 2,
                   Emission((.32 * extent[0], .5 * extent[1], .3 * extent[2]), (0, 0, 1), 2.0), 'TARGET', 'SOLID'),
            Source((.6 * extent[0], .4 * extent[1], .5 * extent[2]), .2 * min(extent), .5, 1,
                   Emission((.6 * extent[0], .4 * extent[1], .5 * extent[2]), (0.5, 0, 0), 1.0))]
    table = pack_sources(srcs)
    src2 = N.FfxSources()
    src2.count = 2
    for i, v in enumerate(table):
        src2.table[i] = v
    D.call('ffx_advect_velocity', gp, C.byref(so), 0, *map(ptr, vel_t), None, None, None, dt, 0, 0.5,
           C.byref(src2), None, None, 0.0, 0.0, 0, *map(ptr, outs), D.s)
    for a in range(3):
        exp = S.advect_velocity_face(g, vel, vel[a], a, dt, False, 0.5, sources=(table, 2))
        assert_close(n(outs[a]), exp, what=f'table velocity {a}')


@pytest.mark.parametrize('masked', [False, True])
@pytest.mark.parametrize('shape,extent', SHAPES[1:])
def test_scalar_passes_match_oracle(D, shape, extent, masked):
    rng = np.random.default_rng(3)
    mask_t = halo_t = None
    if masked:
        mask_t, halo_t = _mask_setup(D, shape, extent)
    g = S.Grid(shape, extent, mask=n(mask_t).astype(bool) if masked else None)
    gs, gp = grid_ptr(shape, extent)
    so = solids(mask_t, halo_t)
    vel = random_faces(g, rng, 0.5)
    vel_t = [t(v) for v in vel]
    dens = rng.uniform(0, 1, g.cell_shape).astype(np.float32)
    temp = rng.uniform(-1, 2, g.cell_shape).astype(np.float32)
    if masked:
        dens = np.where(g.mask, 0, dens).astype(np.float32)
        temp = np.where(g.mask, 0, temp).astype(np.float32)
    fields = [t(dens), t(temp)]
    dt = 0.05
    preds = [t(np.zeros(g.cell_shape)) for _ in range(2)]
    revs = [t(np.zeros(g.cell_shape)) for _ in range(2)]
    ins = (C.c_void_p * 2)(*[f.data_ptr() for f in fields])
    pp = (C.c_void_p * 2)(*[p.data_ptr() for p in preds])
    rr = (C.c_void_p * 2)(*[r.data_ptr() for r in revs])
    D.call('ffx_scalar_transport', gp, C.byref(so), 0, *map(ptr, vel_t), dt, 2, ins, pp, D.s)
    D.call('ffx_scalar_transport', gp, C.byref(so), 0, *map(ptr, vel_t), -dt, 2, pp, rr, D.s)
    ep = [S.scalar_transport(g, vel, f, dt) for f in (dens, temp)]
    er = [S.scalar_transport(g, vel, p, -dt) for p in ep]
    for k in range(2):
        assert_close(n(preds[k]), ep[k], what=f'predictor {k}')
        assert_close(n(revs[k]), er[k], what=f'reverse {k}')
    src = N.FfxSources()
    src.count = -1
    src.single_solid_profile = 1
    src.single_center = N.f3(.5 * extent[0], .5 * extent[1], .25 * extent[2])
    src.single_start = N.f3(.5 * extent[0], .5 * extent[1], .25 * extent[2])
    src.single_radius = .2 * min(extent)
    outs = [t(np.zeros(g.cell_shape)) for _ in range(2)]
    maxima = torch.zeros(2, device='cuda')
    chans = (N.FfxScalarChannel * 2)(
        N.FfxScalarChannel(ptr(fields[0]), ptr(preds[0]), ptr(revs[0]), ptr(outs[0]), 1.0, 0.1, 1.0, 0, 0),
        N.FfxScalarChannel(ptr(fields[1]), ptr(preds[1]), ptr(revs[1]), ptr(outs[1]), 2.0, 0.3, -1.0, 1, 0))
    D.call('ffx_advect_scalars', gp, C.byref(so), 0, *map(ptr, vel_t), dt, 1, C.byref(src), 2, chans, ptr(maxima),
           D.s)
    em = dict(center=tuple(src.single_center), start=tuple(src.single_start), radius=src.single_radius, solid=True)
    e0 = S.advect_scalar(g, vel, dens, ep[0], er[0], dt, True, 1.0, 0.1, 1.0, emitter=em)
    e1 = S.advect_scalar(g, vel, temp, ep[1], er[1], dt, True, 2.0, 0.3, -1.0, emitter=em)
    assert_close(n(outs[0]), e0, what='density')
    assert_close(n(outs[1]), e1, what='temperature')
    assert abs(float(maxima[0]) - np.abs(e0).max()) <= 1e-5 * np.abs(e0).max()
    if masked:
        assert (n(outs[0])[g.mask] == 0).all() and (n(outs[1])[g.mask] == 0).all()


@pytest.mark.parametrize('masked', [False, True])
def test_projection_passes_match_oracle(D, masked):
    shape, extent = (12, 10, 8), (1.3, 0.8, 1.7)
    rng = np.random.default_rng(4)
    mask_t = halo_t = None
    if masked:
        mask_t, halo_t = _mask_setup(D, shape, extent)
    g = S.Grid(shape, extent, mask=n(mask_t).astype(bool) if masked else None)
    gs, gp = grid_ptr(shape, extent)
    so = solids(mask_t, halo_t)
    vel = random_faces(g, rng)
    bounded = [t(np.zeros(fs)) for fs in g.face_shapes]
    div = t(np.zeros(g.cell_shape))
    D.call('ffx_walls_divergence', gp, C.byref(so), 0, *[ptr(t(v)) for v in vel], *map(ptr, bounded), ptr(div), D.s)
    eb = S.walls(g, vel)
    for a in range(3):
        assert np.array_equal(n(bounded[a]), eb[a])
    ed = S.divergence(g, eb)
    assert_close(n(div), ed, rel=1e-6)
    D.call('ffx_divergence', gp, C.byref(so), 0, *map(ptr, bounded), ptr(div), D.s)
    assert_close(n(div), ed, rel=1e-6)
    p = rng.uniform(-1, 1, g.cell_shape).astype(np.float32)
    outs = [t(np.zeros(fs)) for fs in g.face_shapes]
    after = t(np.zeros(g.cell_shape))
    maxima = torch.zeros(3, device='cuda')
    D.call('ffx_gradient', gp, C.byref(so), 0, *map(ptr, bounded), ptr(t(p)), 0.04, *map(ptr, outs), ptr(after),
           ptr(maxima), D.s)
    eg = S.gradient(g, eb, p, 0.04)
    for a in range(3):
        assert_close(n(outs[a]), eg[a], rel=1e-6)
        assert abs(float(maxima[a]) - np.abs(eg[a]).max()) <= 1e-6 * np.abs(eg[a]).max()
    assert_close(n(after), S.divergence(g, eg), rel=1e-6)
    # masked / unmasked Jacobi
    q = t(np.zeros(g.cell_shape))
    D.call('ffx_jacobi', N.n3(*shape), N.f3(*g.inv), ptr(mask_t), ptr(t(p)), ptr(div), 0.04, 2 / 3, ptr(q), D.s)
    assert_close(n(q), S.jacobi(g, p, ed, 0.04, 2 / 3, mask=g.mask), rel=1e-6)


def test_geometric_mg_operators_match_oracle(D):
    shape, extent = (16, 12, 8), (1.3, 0.8, 1.7)
    rng = np.random.default_rng(5)
    g = S.Grid(shape, extent)
    inv = tuple(g.f(c / e) for c, e in zip(shape, extent))
    p = rng.uniform(-1, 1, g.cell_shape).astype(np.float32)
    rhs = rng.uniform(-1, 1, g.cell_shape).astype(np.float32)
    r = t(np.zeros(g.cell_shape))
    D.call('ffx_mg_residual', N.n3(*shape), N.f3(*inv), ptr(t(p)), ptr(t(rhs)), 0.04, ptr(r), D.s)
    er = S.residual(g, p, rhs, 0.04, inv)
    assert_close(n(r), er, rel=1e-6)
    cs = (6, 8, 4)
    coarse = t(np.zeros((4, 6, 8)))
    D.call('ffx_mg_restrict', N.n3(*shape), ptr(t(er)), ptr(coarse), D.s)
    assert_close(n(coarse), S.restrict(er.astype(np.float32)), rel=1e-6)
    D.call('ffx_mg_residual_restrict', N.n3(*shape), N.f3(*inv), ptr(t(p)), ptr(t(rhs)), 0.04, ptr(coarse), D.s)
    assert_close(n(coarse), S.restrict(er), rel=1e-6)
    c = rng.uniform(-1, 1, (4, 6, 8)).astype(np.float32)
    out = t(np.zeros(g.cell_shape))
    D.call('ffx_mg_prolong', N.n3(*shape), ptr(t(p)), ptr(t(c)), ptr(out), D.s)
    assert_close(n(out), S.prolong(g, p, c), rel=1e-6)
    rmax = torch.zeros(1, device='cuda')
    D.call('ffx_mg_residual_max', N.n3(*shape), N.f3(*inv), ptr(t(p)), ptr(t(rhs)), 0.04, ptr(rmax), D.s)
    assert abs(float(rmax[0]) - np.abs(er).max()) <= 1e-6 * np.abs(er).max()
    # direct 4^3 solve with the reference's closed-form inverse
    from fluxfx_b200.physics.coarse_pressure import neumann_inverse
    inv4 = neumann_inverse((4, 4, 4), extent)
    rhs4 = np.sin(np.arange(64) * .73).astype(np.float32).reshape(4, 4, 4)
    rhs4 -= rhs4.mean()
    p4 = t(np.zeros((4, 4, 4)))
    D.call('ffx_direct_solve', 64, ptr(t(inv4, torch.float64)), ptr(t(rhs4)), 1.0, ptr(p4), D.s)
    g4 = S.Grid((4, 4, 4), extent, np.float64)
    lap = -S.residual(g4, n(p4), np.zeros((4, 4, 4)), 1.0, g4.inv)
    assert np.abs(lap - rhs4).max() < 2e-6


def test_graph_operators_and_hierarchy_match_oracle(D):
    from pathlib import Path
    gold = np.load(Path(__file__).parent / 'golden' / 'solid_hierarchy.npz')
    from fluxfx_b200.physics.solid_hierarchy import build_hierarchy
    for name in ('cube', 'slab', 'disconnected', 'sphere'):
        shape = tuple(int(v) for v in gold[f'{name}_shape'])
        extent = tuple(float(v) for v in gold[f'{name}_extent'])
        mask = gold[f'{name}_mask']
        levels = build_hierarchy(shape, extent, mask, device=D)
        assert len(levels) == int(gold[f'{name}_levels']), name
        for i, (sh, edges) in enumerate(levels):
            assert np.array_equal(edges.ravel(), gold[f'{name}_level{i}_edges']), (name, i)   # bit-exact
    # operators on the sphere case, level 0 (mask-derived) and level 1 (records)
    shape = tuple(int(v) for v in gold['sphere_shape'])
    extent = tuple(float(v) for v in gold['sphere_extent'])
    nx, ny, nz = shape
    maskb = gold['sphere_mask'].reshape(nz, ny, nx) > .5
    hier = S.build_hierarchy(shape, extent, maskb)
    rng = np.random.default_rng(6)
    solid_t = t(maskb, torch.uint8)
    w = [float(np.float32((c / e) ** 2)) for c, e in zip(shape, extent)]
    lv0 = N.FfxGraphLevel(*shape, None, ptr(solid_t), N.f3(*w))
    e1 = t(hier[1][1])
    lv1 = N.FfxGraphLevel(*hier[1][0], ptr(e1), None, N.f3(0, 0, 0))
    for lv, (sh, edges) in ((lv0, hier[0]), (lv1, hier[1])):
        cell = (sh[2], sh[1], sh[0])
        p = rng.uniform(-1, 1, cell).astype(np.float32)
        rhs = rng.uniform(-1, 1, cell).astype(np.float32)
        out = t(np.zeros(cell))
        D.call('ffx_graph_smooth', C.byref(lv), ptr(t(p)), ptr(t(rhs)), 2 / 3, ptr(out), D.s)
        assert_close(n(out), S.graph_smooth(p, rhs, edges), rel=1e-6)
        D.call('ffx_graph_residual', C.byref(lv), ptr(t(p)), ptr(t(rhs)), ptr(out), D.s)
        er = S.graph_residual(p, rhs, edges)
        assert_close(n(out), er, rel=1e-6)
        cc = (sh[2] // 2, sh[1] // 2, sh[0] // 2)
        cout = t(np.zeros(cc))
        D.call('ffx_graph_residual_restrict', C.byref(lv), ptr(t(p)), ptr(t(rhs)), ptr(cout), D.s)
        assert_close(n(cout), S.restrict(er), rel=1e-6)
        c = rng.uniform(-1, 1, cc).astype(np.float32)
        D.call('ffx_graph_prolong', C.byref(lv), ptr(t(p)), ptr(t(c)), ptr(out), D.s)
        ep = S.graph_prolong(p, c, edges)
        assert_close(n(out), ep, rel=1e-6)
        D.call('ffx_graph_prolong_smooth', C.byref(lv), ptr(t(p)), ptr(t(c)), ptr(t(rhs)), 2 / 3, ptr(out), D.s)
        assert_close(n(out), S.graph_smooth(ep, rhs, edges), rel=1e-6)


def test_reductions(D):
    rng = np.random.default_rng(7)
    x = rng.normal(size=100003).astype(np.float32)
    x[77] = -9.5
    out = torch.zeros(1, device='cuda')
    D.call('ffx_max_abs', x.size, 0, ptr(t(x)), ptr(out), D.s)
    assert float(out[0]) == 9.5
    x[5] = np.nan
    D.call('ffx_max_abs', x.size, 0, ptr(t(x)), ptr(out), D.s)
    assert float(out[0]) == pytest.approx(3.4e38, rel=1e-6)
    b = rng.normal(size=300001).astype(np.float32)
    a = (b * 1e-3).astype(np.float32)
    need = D.lib.ffx_divergence_stats_workspace(b.size)
    ws = torch.zeros(need // 8 + 1, dtype=torch.float64, device='cuda')
    res = torch.zeros(8, dtype=torch.float64, device='cuda')
    D.call('ffx_divergence_stats', b.size, ptr(t(b)), ptr(t(a)), ptr(res), ptr(ws), ws.numel() * 8, D.s)
    r = n(res)
    bd, ad = b.astype(np.float64), a.astype(np.float64)
    assert r[0] == pytest.approx((bd * bd).sum(), rel=1e-12)
    assert r[1] == pytest.approx((ad * ad).sum(), rel=1e-12)
    assert r[2] == np.abs(bd).max() and r[3] == np.abs(ad).max()
    assert r[4] == pytest.approx(bd.sum(), rel=1e-9, abs=1e-9)
    assert r[6] == b.size
    # workspace too small is refused with a clear status, nothing launched
    st = D.lib.ffx_divergence_stats(b.size, ptr(t(b)), ptr(t(a)), ptr(res), ptr(ws), 8, D.s)
    assert st == N.FFX_ERR_INVALID and b'workspace' in D.lib.ffx_last_error()


def test_invalid_arguments_are_rejected_without_launch(D):
    gs, gp = grid_ptr((8, 8, 8), (1., 1., 1.))
    x = t(np.zeros((8, 8, 9)))
    st = D.lib.ffx_walls(gp, None, 0, ptr(x), ptr(x), ptr(x), ptr(x), ptr(x), ptr(x), D.s)
    assert st == N.FFX_ERR_INVALID
    assert b'alias' in D.lib.ffx_last_error()
    bad = N.FfxGrid(0, 8, 8, 1, 1, 1, 0, 0, 0)
    assert D.lib.ffx_divergence(C.byref(bad), None, 0, ptr(x), ptr(x), ptr(x), ptr(x), D.s) == N.FFX_ERR_INVALID
    assert D.lib.ffx_direct_solve(2000, ptr(x), ptr(x), 1.0, ptr(x), D.s) == N.FFX_ERR_INVALID


def test_krylov_kernels_match_numpy(D):
    """MG-PCG building blocks: zero-start sweep, sweep + dot, direction + apply, update."""
    from pathlib import Path
    gold = np.load(Path(__file__).parent / 'golden' / 'solid_hierarchy.npz')
    shape = tuple(int(v) for v in gold['sphere_shape'])
    extent = tuple(float(v) for v in gold['sphere_extent'])
    nx, ny, nz = shape
    maskb = gold['sphere_mask'].reshape(nz, ny, nx) > .5
    edges = S.level0_edges(shape, extent, maskb)
    solid_t = t(maskb, torch.uint8)
    w = [float(np.float32((c / e) ** 2)) for c, e in zip(shape, extent)]
    lv = N.FfxGraphLevel(*shape, None, ptr(solid_t), N.f3(*w))
    rng = np.random.default_rng(21)
    cell = (nz, ny, nx)
    rhs = rng.uniform(-1, 1, cell).astype(np.float32)
    p = rng.uniform(-1, 1, cell).astype(np.float32)
    out = t(np.zeros(cell))
    D.call('ffx_graph_smooth_zero', C.byref(lv), ptr(t(rhs)), 2 / 3, ptr(out), D.s)
    assert_close(n(out), S.graph_smooth(np.zeros_like(p), rhs, edges), rel=1e-6)
    dot = torch.zeros(1, dtype=torch.float64, device='cuda')
    D.call('ffx_graph_smooth_dot', C.byref(lv), ptr(t(p)), ptr(t(rhs)), 2 / 3, ptr(out), ptr(dot), -1.0, D.s)
    sm = S.graph_smooth(p, rhs, edges)
    assert_close(n(out), sm, rel=1e-6)
    assert float(dot[0]) == pytest.approx(-(rhs.astype(np.float64) * sm).sum(), rel=1e-9)
    # direction + apply: q = A p with A = -L = diag p - nb
    z = rng.uniform(-1, 1, cell).astype(np.float32)
    pold = rng.uniform(-1, 1, cell).astype(np.float32)
    rz = torch.tensor([2.0, 4.0], dtype=torch.float64, device='cuda')   # beta = 2/4
    pn, q = t(np.zeros(cell)), t(np.zeros(cell))
    pq = torch.zeros(1, dtype=torch.float64, device='cuda')
    D.call('ffx_pcg_direction_apply', C.byref(lv), ptr(t(z)), ptr(t(pold)), ptr(rz[0:1]), ptr(rz[1:2]), ptr(pn),
           ptr(q), ptr(pq), D.s)
    dirn = (z + np.float32(0.5) * pold).astype(np.float32)
    diag, nb = S.graph_terms(dirn, edges)
    qe = np.where(diag > 0, diag * dirn - nb, 0)
    assert_close(n(pn), dirn, rel=1e-6)
    assert_close(n(q), qe, rel=1e-5)
    assert float(pq[0]) == pytest.approx((dirn.astype(np.float64) * qe).sum(), rel=1e-5)
    # update: alpha = rz/pq
    x0 = rng.uniform(-1, 1, cell).astype(np.float32)
    r0 = rng.uniform(-1, 1, cell).astype(np.float32)
    xs, rs = t(x0), t(r0)
    rmax = torch.zeros(1, device='cuda')
    D.call('ffx_pcg_update', x0.size, ptr(rz[0:1]), ptr(pq), ptr(xs), ptr(pn), ptr(rs), ptr(q), ptr(rmax), D.s)
    alpha = np.float32(2.0 / float(pq[0]))
    assert_close(n(xs), x0 + alpha * n(pn), rel=1e-6)
    re = r0 + alpha * n(q)
    assert_close(n(rs), re, rel=1e-6)
    assert float(rmax[0]) == pytest.approx(np.abs(re).max(), rel=1e-6)


def _links_numpy(mask):
    """Link bytes of a (nz, ny, nx) solid mask: bit 2a / 2a+1 = open face to the
    lower / upper neighbour along axis a (x, y, z), bit 6 = fluid."""
    fluid = ~mask
    out = np.where(fluid, 64, 0).astype(np.uint8)
    for a, ax in enumerate((2, 1, 0)):
        lo = np.zeros_like(fluid)
        hi = np.zeros_like(fluid)
        sl_a = [slice(None)] * 3
        sl_b = [slice(None)] * 3
        sl_a[ax], sl_b[ax] = slice(1, None), slice(None, -1)
        lo[tuple(sl_a)] = fluid[tuple(sl_a)] & fluid[tuple(sl_b)]
        hi[tuple(sl_b)] = fluid[tuple(sl_b)] & fluid[tuple(sl_a)]
        out |= np.where(lo, 1 << (2 * a), 0).astype(np.uint8)
        out |= np.where(hi, 1 << (2 * a + 1), 0).astype(np.uint8)
    return out


def _bits(x):
    torch.cuda.synchronize()
    return x.detach().cpu().numpy().view(np.uint32)


@pytest.mark.parametrize('shape', [(64, 20, 12), (256, 10, 10), (40, 18, 8)])
def test_level0_four_cell_kernels_equal_scalar_kernels(D, shape):
    """With link bytes and nx % 4 == 0 the level-0 passes run four cells per
    thread; every field they write is bit-identical to the one-cell kernels
    (the dot products, summed in another order, agree to 1e-12)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(nx + ny + nz)
    from fluxfx_b200.physics.collision import raster_reference
    from fluxfx_b200.physics.config import GridSpec
    grid = GridSpec(shape, axis_limit=256)
    mask = np.asarray(raster_reference(grid, sphere_box_mask(shape))).reshape(nz, ny, nx) > 0.5
    assert 0 < mask.sum() < mask.size
    mask |= rng.uniform(size=mask.shape) < 0.15
    solid_t = t(mask, torch.uint8)
    w = [float(np.float32(c ** 2)) for c in shape]
    scalar = N.FfxGraphLevel(*shape, None, ptr(solid_t), N.f3(*w))
    four = N.FfxGraphLevel(*shape, None, ptr(solid_t), N.f3(*w))
    links = torch.zeros((nz, ny, nx), dtype=torch.uint8, device='cuda')
    D.call('ffx_graph_links', C.byref(four), ptr(links), D.s)
    torch.cuda.synchronize()
    assert np.array_equal(links.cpu().numpy(), _links_numpy(mask))
    four.links = links.data_ptr()
    cell = (nz, ny, nx)
    p, rhs, z, pold = (t(rng.uniform(-1, 1, cell)) for _ in range(4))
    coarse = t(rng.uniform(-1, 1, (nz // 2, ny // 2, nx // 2)))
    rz = torch.tensor([3.0, 5.0], dtype=torch.float64, device='cuda')

    def both(fn):
        outs = []
        for lv in (scalar, four):
            outs.append(fn(lv))
        return outs

    def smooth(lv):
        o = t(np.full(cell, np.nan))
        D.call('ffx_graph_smooth', C.byref(lv), ptr(p), ptr(rhs), 2 / 3, ptr(o), D.s)
        return o
    a, b = both(smooth)
    assert np.array_equal(_bits(a), _bits(b))

    def zero(lv):
        o = t(np.full(cell, np.nan))
        D.call('ffx_graph_smooth_zero', C.byref(lv), ptr(rhs), 2 / 3, ptr(o), D.s)
        return o
    a, b = both(zero)
    assert np.array_equal(_bits(a), _bits(b))

    def smooth_dot(lv):
        o = t(np.full(cell, np.nan))
        d = torch.zeros(1, dtype=torch.float64, device='cuda')
        D.call('ffx_graph_smooth_dot', C.byref(lv), ptr(p), ptr(rhs), 2 / 3, ptr(o), ptr(d), -1.0, D.s)
        return o, d
    (a, da), (b, db) = both(smooth_dot)
    assert np.array_equal(_bits(a), _bits(b))
    assert float(db[0]) == pytest.approx(float(da[0]), rel=1e-12)

    def prolong_smooth(lv):
        o = t(np.full(cell, np.nan))
        D.call('ffx_graph_prolong_smooth', C.byref(lv), ptr(p), ptr(coarse), ptr(rhs), 2 / 3, ptr(o), D.s)
        return o
    a, b = both(prolong_smooth)
    assert np.array_equal(_bits(a), _bits(b))

    def prolong_smooth_dot(lv):
        o = t(np.full(cell, np.nan))
        d = torch.zeros(1, dtype=torch.float64, device='cuda')
        D.call('ffx_graph_prolong_smooth_dot', C.byref(lv), ptr(p), ptr(coarse), ptr(rhs), 2 / 3, ptr(o), ptr(d),
               -1.0, D.s)
        return o, d
    (a, da), (b, db) = both(prolong_smooth_dot)
    assert np.array_equal(_bits(a), _bits(b))
    assert np.array_equal(_bits(a), _bits(both(prolong_smooth)[0]))
    expect = -(n(rhs).astype(np.float64) * n(a)).sum()
    assert float(da[0]) == pytest.approx(expect, rel=1e-9) and float(db[0]) == pytest.approx(expect, rel=1e-9)

    def residual(lv):
        o = t(np.full(cell, np.nan))
        D.call('ffx_graph_residual', C.byref(lv), ptr(p), ptr(rhs), ptr(o), D.s)
        return o
    a, b = both(residual)
    assert np.array_equal(_bits(a), _bits(b))

    def residual_max(lv):
        o = torch.full((1,), -1.0, device='cuda')
        D.call('ffx_graph_residual_max', C.byref(lv), ptr(p), ptr(rhs), ptr(o), D.s)
        return o
    a, b = both(residual_max)
    assert float(a[0]) == float(b[0]) > 0

    def restrict(lv):
        o = t(np.full((nz // 2, ny // 2, nx // 2), np.nan))
        D.call('ffx_graph_residual_restrict', C.byref(lv), ptr(p), ptr(rhs), ptr(o), D.s)
        return o
    a, b = both(restrict)
    assert np.array_equal(_bits(a), _bits(b))

    for first in (True, False):
        def direction(lv):
            pn, q = t(np.full(cell, np.nan)), t(np.full(cell, np.nan))
            pq = torch.zeros(1, dtype=torch.float64, device='cuda')
            D.call('ffx_pcg_direction_apply', C.byref(lv), ptr(z), None if first else ptr(pold), ptr(rz[0:1]),
                   None if first else ptr(rz[1:2]), ptr(pn), ptr(q), ptr(pq), D.s)
            return pn, q, pq
        (pa, qa, sa), (pb, qb, sb) = both(direction)
        assert np.array_equal(_bits(pa), _bits(pb)) and np.array_equal(_bits(qa), _bits(qb))
        assert float(sb[0]) == pytest.approx(float(sa[0]), rel=1e-12)
