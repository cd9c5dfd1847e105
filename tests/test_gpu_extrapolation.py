"""Warm start extrapolated in time (warm_start_extrapolation and
warm_start_order, extensions of the solver).

The linear and quadratic passes (ffx_extrapolate_pressure, _pressure2) against
their formulas, bit for bit (the library is built without FMA contraction, so
the products and sums round like NumPy's FP32 ones); the solver with the
extrapolated start against the same solver started from the previous
pressure: every step meets the tolerance, the extrapolated start needs fewer
V-cycles, and the two runs stay within what the solve tolerance allows of
each other; and the extended solver (linear or quadratic start, optionally
fewer coarse-level sweeps) against the CPU oracle restating the same
extensions, step by step on the 64^3 collider scene."""
import ctypes as C

import numpy as np
import pytest
import torch

from fluxfx_b200 import _native as N
from tests.gpu_helpers import dev, n

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def D():
    return dev()


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _expected(p, hist, dt, prev, beta, first):
    d0, d1 = float(np.float32(dt)), float(np.float32(prev))
    r = d0 / d1
    inv = np.float32(1.0 / d1)
    if first:
        c1 = np.float32(r) if abs(r - 1.0) > 1e-6 else np.float32(1.0)
        return p * c1, p * inv
    c1 = np.float32(d0 * (1.0 + beta * r) / d1)
    c2 = np.float32(d0 * beta * r)
    return c1 * p - c2 * hist, p * inv


@pytest.mark.parametrize('count', [4096, 1001])
@pytest.mark.parametrize('first', [0, 1])
@pytest.mark.parametrize('clock', [(0.0019, 0.0021), (0.02, 0.02), (0.02, 0.02 * (1 + 1e-7))])
def test_extrapolate_kernel_matches_its_formula(D, count, first, clock):
    lib = N.load()
    rng = np.random.default_rng(count + first)
    p0 = rng.normal(size=count).astype(np.float32) * 3e-3
    h0 = rng.normal(size=count).astype(np.float32)
    beta = 1.0
    p, h = torch.as_tensor(p0).cuda(), torch.as_tensor(h0).cuda()
    ck = torch.tensor(clock, dtype=torch.float32, device='cuda')
    N.check(lib.ffx_extrapolate_pressure(count, _ptr(p), _ptr(h), _ptr(ck), beta, first, None))
    torch.cuda.synchronize()
    want_p, want_h = _expected(p0, h0, clock[0], clock[1], beta, first)
    assert np.array_equal(p.cpu().numpy(), want_p)
    assert np.array_equal(h.cpu().numpy(), want_h)


def test_extrapolate_kernel_without_previous_step_and_invalid_arguments(D):
    lib = N.load()
    p = torch.ones(64, device='cuda')
    h = torch.full((64,), 2.0, device='cuda')
    ck = torch.tensor([0.02, 0.0], dtype=torch.float32, device='cuda')   # no previous dt
    N.check(lib.ffx_extrapolate_pressure(64, _ptr(p), _ptr(h), _ptr(ck), 1.0, 0, None))
    torch.cuda.synchronize()
    assert (p.cpu() == 1).all() and (h.cpu() == 2).all()
    bad = [(64, p, h, 1.5, 0), (64, p, h, -0.1, 0), (64, p, p, 1.0, 0), (0, p, h, 1.0, 0), (64, p, h, 1.0, 2)]
    for count, a, b, beta, first in bad:
        rc = lib.ffx_extrapolate_pressure(count, _ptr(a), _ptr(b), _ptr(ck), beta, first, None)
        assert rc == N.FFX_ERR_INVALID
    # a pointer off the 16-byte grid is rejected before any launch
    rc = lib.ffx_extrapolate_pressure(60, C.c_void_p(p.data_ptr() + 4), _ptr(h), _ptr(ck), 1.0, 0, None)
    assert rc == N.FFX_ERR_INVALID
    assert b'16-byte' in lib.ffx_last_error()


def _solver(D, size, beta):
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    grid, s, colliders, emitters, noise = bench.scene(size, 'FP32', 0, **bench.VARIANTS['fast'],
                                                      warm_start_extrapolation=beta)
    solver = DenseProjectedSmoke(grid, s, D, colliders=colliders)
    zeros = torch.zeros(grid.cells)
    solver.upload(zeros)
    solver.upload_temperature(zeros)
    solver.upload_velocity([torch.as_tensor(v) for v in noise])
    return solver, emitters


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize('device_steps', [True, False])
def test_extrapolated_warm_start_meets_tolerance_with_fewer_cycles(D, device_steps):
    """Both runs solve the same systems to relative max-norm divergence
    <= 1e-4 every step; they start each solve from different guesses, so
    their fields separate only by the accumulated solve error (the bounds of
    the headline-solver test: 1e-3 relative L2 for the scalars, 1e-2 for the
    velocity)."""
    size, steps = 64, 12
    runs = {beta: _solver(D, size, beta) for beta in (0.0, 1.0)}
    cycles = {beta: [] for beta in runs}
    for k in range(steps):
        for beta, (solver, emitters) in runs.items():
            if device_steps:
                solver.step_cfl(0.5, 0.02, sources=emitters)
            else:
                solver.step(0.02 if k == 0 else min(0.02, 0.5 / size / max(solver.projector.velocity_maxima())),
                            sources=emitters)
            assert solver.measure_projection()['rel_div_inf'] <= 1e-4, (beta, k)
            cycles[beta].append(solver.projector.last_cycles)
    print('cycles per step: previous pressure %s, extrapolated %s' % (cycles[0.0], cycles[1.0]))
    assert sum(cycles[1.0][3:]) < sum(cycles[0.0][3:])
    A, B = runs[1.0][0], runs[0.0][0]
    assert _rel_l2(n(A.density), n(B.density)) <= 1e-3
    assert _rel_l2(n(A.temperature), n(B.temperature)) <= 1e-3
    for a in range(3):
        assert _rel_l2(n(A._velocity[a]), n(B._velocity[a])) <= 1e-2, a
    for solver, _ in runs.values():
        solver.close()


@pytest.mark.parametrize('count', [3001, 4096])
@pytest.mark.parametrize('have', [0, 1, 2])
@pytest.mark.parametrize('clock', [(0.0019, 0.0021), (0.02, 0.02)])
def test_quadratic_extrapolate_kernel_matches_its_formula(D, have, clock, count):
    from oracle.solver import extrapolate2
    lib = N.load()
    rng = np.random.default_rng(7 + have)
    d2 = 0.0023
    p0 = rng.normal(size=count).astype(np.float32) * 3e-3
    h = [rng.normal(size=count).astype(np.float32) for _ in range(2)]
    p, newest, oldest = (torch.as_tensor(a).cuda() for a in (p0, h[0], h[1]))
    ck = torch.tensor(clock, dtype=torch.float32, device='cuda')
    slots = torch.tensor([d2, -1.0], dtype=torch.float32, device='cuda')
    N.check(lib.ffx_extrapolate_pressure2(count, _ptr(p), _ptr(newest), _ptr(oldest), _ptr(ck), _ptr(slots[0:1]),
                                          _ptr(slots[1:2]), 0.75, have, None))
    torch.cuda.synchronize()
    history = [(h[0], float(np.float32(d2))), (h[1], 0.0)][:have]
    want_p, want_h = extrapolate2(p0, history, clock[0], clock[1], 0.75)
    assert np.array_equal(p.cpu().numpy(), want_p)
    assert np.array_equal(oldest.cpu().numpy(), want_h)          # the last solve, written over the oldest
    assert np.array_equal(newest.cpu().numpy(), h[0])
    assert slots.cpu().tolist() == [pytest.approx(d2), float(np.float32(clock[1]))]


@pytest.mark.parametrize('coarse_sweeps, order', [(0, 1), (2, 1), (0, 2)])
def test_extended_solver_matches_oracle_on_collider_scene(D, coarse_sweeps, order):
    """The collider scene at 64^3 with the extrapolated start (beta = 1) and,
    optionally, two pre- and post-sweeps on the levels below level 0, against
    the CPU oracle with the same settings: per step and field within 1e-5 of
    the field's maximum, the same V-cycle counts. Host steps (dt from the
    device's face maxima on both sides), six steps: the extrapolation starts
    at the third (the quadratic at the fourth)."""
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.physics.emission import pack_sources
    from oracle import solver as O
    from tests.test_gpu_configs import cfl_dt, compare_step
    settings = dict(bench.VARIANTS['extrapolated'], mg_coarse_sweeps=coarse_sweeps, warm_start_order=order)
    grid, s, colliders, emitters, noise = bench.scene(64, 'FP32', 0, **settings)
    solver = DenseProjectedSmoke(grid, s, D, colliders=colliders)
    if coarse_sweeps:
        assert solver.projector.coarse_pre == solver.projector.coarse_post == coarse_sweeps
    mask = n(solver.solids.mask).astype(bool)
    ref = O.OracleSmoke(grid.shape, grid.extent, s, np.float32, mask=mask)
    zeros = np.zeros(grid.cells, np.float32)
    solver.upload(torch.as_tensor(zeros))
    solver.upload_temperature(torch.as_tensor(zeros))
    solver.upload_velocity([torch.as_tensor(v) for v in noise])
    ref.upload(density=zeros, temperature=zeros, velocity=noise)
    table = (pack_sources(emitters), len(emitters))
    dt, cycles = 0.02, []
    for k in range(6):
        solver.step(dt, sources=emitters)
        ref.step(dt, sources=table)
        assert solver.projector.last_cycles == ref.projector.last_cycles, k
        cycles.append(ref.projector.last_cycles)
        compare_step(solver, ref, k)
        assert solver.measure_projection()['rel_div_inf'] <= 1e-4
        dt = cfl_dt(max(solver.projector.velocity_maxima()), 1.0 / 64)
    print(f'coarse sweeps {coarse_sweeps}, order {order}: cycles {cycles}')
    solver.close()
