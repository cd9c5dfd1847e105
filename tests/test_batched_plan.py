"""Host side of the batched uneven domains: the seeded scene generator
(domain sizes, emitters, colliders) and the plan builder's argument checks
and workspace sizing, through the C ABI with placeholder pointers (the plan
builder only reads them; nothing runs on a device)."""
import ctypes as C

import numpy as np
import pytest

from fluxfx_b200 import _native as N
from fluxfx_b200.backend.batched import batched_scenes


def test_scenes_follow_the_batched_configuration():
    scenes = batched_scenes(48, seed=3)
    assert len(scenes) == 48
    again = batched_scenes(48, seed=3)
    shapes = [s[0].shape for s in scenes]
    assert shapes == [s[0].shape for s in again]
    assert set(n for sh in shapes for n in sh) <= {32, 48, 64, 96, 128}
    assert len(set(shapes)) > 10                          # uneven, non-cubic
    cell = 1.0 / 64.0
    for grid, settings, colliders, emitters, noise in scenes:
        assert grid.cell_size == pytest.approx((cell,) * 3)
        assert 1 <= len(emitters) <= 3
        for e in emitters:
            assert 3 * cell <= e.radius <= 8 * cell
            assert 0.5 <= e.density_rate <= 1.0 and 0.5 <= e.heat_rate <= 1.0
            assert e.center[2] <= grid.extent[2] / 3 + 1e-12
        assert 1 <= len(colliders) <= 2
        assert settings.pressure_tolerance == 1e-4
        assert [a.shape for a in noise] == [(fs[2], fs[1], fs[0]) for fs in grid.face_shapes]
        assert max(float(np.abs(a).max()) for a in noise) <= 1e-3


def fake_domain(shape, tail=True, pre=4, post=4, base=0x10000):
    """A domain with distinct placeholder pointers and a consistent hierarchy."""
    counter = iter(range(base, base + 100000, 256))
    p = lambda: next(counter)
    D = N.FfxBatchDomain()
    D.grid = N.grid_struct(shape, tuple(n / 64 for n in shape))
    D.solid, D.halo = p(), p()
    D.u, D.v, D.w, D.pu, D.pv, D.pw, D.bu, D.bv, D.bw = [p() for _ in range(9)]
    D.density[0], D.density[1], D.temperature[0], D.temperature[1] = p(), p(), p(), p()
    D.predictor[0], D.predictor[1], D.reverse[0], D.reverse[1] = p(), p(), p(), p()
    D.after = p()
    D.velocity_corrected = D.scalar_corrected = 1
    D.blend = 0.5
    D.cell, D.cfl, D.dt_max, D.dt0 = 1 / 64, 0.5, 0.02, 0.02
    levels = []
    n = list(shape)
    while min(n) >= 8 and all(v % 2 == 0 for v in n):
        levels.append(tuple(n))
        n = [v // 2 for v in n]
    levels.append(tuple(n))
    D.levels = len(levels)
    for k, (nx, ny, nz) in enumerate(levels):
        lv = N.FfxGraphLevel(nx, ny, nz, None if k == 0 else p(), D.solid if k == 0 else None, N.f3(1, 1, 1))
        D.level[k].level = lv
        D.level[k].p, D.level[k].q, D.level[k].rhs = p(), p(), p()
    small = [k for k in range(1, len(levels)) if np.prod(levels[k]) <= 512]
    D.tail_start = small[0] if (tail and small and small[0] < len(levels) - 1) else -1
    D.inverse = p() if np.prod(levels[-1]) <= 256 else None
    D.pre, D.post, D.max_cycles, D.tolerance = pre, post, 200, 1e-4
    return D


def bytes_for(domains):
    arr = (N.FfxBatchDomain * len(domains))(*domains)
    out = C.c_int64(0)
    st = N.load().ffx_batch_workspace_bytes(arr, len(domains), C.byref(out))
    return st, out.value


def test_workspace_grows_with_the_domains():
    st1, one = bytes_for([fake_domain((32, 48, 64))])
    st2, three = bytes_for([fake_domain((32, 48, 64)), fake_domain((96, 32, 32), base=0x900000),
                            fake_domain((48, 48, 48), tail=False, base=0x1900000)])
    assert st1 == N.FFX_OK and st2 == N.FFX_OK
    assert 0 < one < three


@pytest.mark.parametrize('edit, message', [
    (lambda D: setattr(D, 'solid', None), b'missing mask'),
    (lambda D: setattr(D, 'levels', 1), b'multigrid levels'),
    (lambda D: setattr(D, 'pre', 3), b'even sum'),
    (lambda D: setattr(D, 'tolerance', 0.0), b'tolerance'),
    (lambda D: setattr(D, 'blend', 1.5), b'blend'),
    (lambda D: setattr(D, 'tail_start', 0), b'tail start'),
    (lambda D: D.density.__setitem__(1, D.density[0]), b'ping-pong'),
    (lambda D: setattr(D.level[1].level, 'nx', 7), b'coarsening'),
])
def test_plan_rejects_invalid_domains(edit, message):
    D = fake_domain((64, 32, 48))
    edit(D)
    st, _ = bytes_for([D])
    assert st == N.FFX_ERR_INVALID
    assert message in N.load().ffx_last_error()


def test_plan_rejects_mixed_sweeps_and_too_many_domains():
    st, _ = bytes_for([fake_domain((32, 32, 32)), fake_domain((32, 32, 32), pre=2, post=2, base=0x900000)])
    assert st == N.FFX_ERR_INVALID
    arr = (N.FfxBatchDomain * 65)()
    out = C.c_int64(0)
    assert N.load().ffx_batch_workspace_bytes(arr, 65, C.byref(out)) == N.FFX_ERR_INVALID
