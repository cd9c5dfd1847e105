"""Departure-point reuse in the velocity correction: where the predictor and
the correction form the same start point at every face (power-of-two grids,
and grids whose spacing extent / n is a power of two), the correction reads the
predictor's departure points and, in FP32, its sample, instead of tracing
again. The step's fields must be bit-identical to those of the same step with
reuse switched off; a grid whose start points differ must not reuse."""
import numpy as np
import pytest
import torch

from fluxfx_b200 import _native as N
from fluxfx_b200.physics.collision import primitive
from fluxfx_b200.physics.config import GridSpec
from fluxfx_b200.physics.pressure import PressureSettings
from tests.gpu_helpers import dev

pytestmark = pytest.mark.gpu


def _run(grid, reuse, steps=3, storage='FP32'):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    settings = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK',
                                thermal_lift=0.5, density_weight=0.1, source_center=(.3, .4, .25),
                                source_radius=.12, heat_source_rate=10.0, storage=storage)
    colliders = (primitive('SPHERE', (.55, .5, .5), (.2,) * 3),)
    s = DenseProjectedSmoke(grid, settings, dev(), colliders=colliders)
    s.detail.reuse_traces = reuse
    for _ in range(steps):
        s.step(0.02)
    torch.cuda.synchronize()
    out = [s.density.clone(), s.temperature.clone()] + [v.clone() for v in s._velocity]
    reused = s.detail.face_trace is not None
    s.close()
    return out, reused


@pytest.mark.parametrize('shape, extent, matches', [
    ((48, 40, 32), (48 / 64, 40 / 64, 32 / 64), True),     # spacing 1/64, counts not powers of two
    ((32, 32, 32), (1.0, 1.0, 1.0), True),                 # power-of-two grid
    ((24, 20, 16), (1.3, 0.8, 1.7), False),                # start points differ: no face reuse
])
@pytest.mark.parametrize('storage', ['FP32', 'BF16'])
def test_velocity_trace_reuse_is_bit_identical(shape, extent, matches, storage):
    # BF16: the correction reads the predictor's unrounded sample from the fourth trace plane
    assert N.face_starts_match(shape, extent) == matches
    grid = GridSpec(shape, extent)
    a, reused = _run(grid, True, storage=storage)
    b, _ = _run(grid, False, storage=storage)
    assert reused == matches
    for x, y in zip(a, b):
        assert torch.equal(x, y), float((x - y).abs().max())


@pytest.mark.parametrize('storage', ['FP32', 'BF16'])
@pytest.mark.parametrize('device_dt, amp', [(False, 0.3), (False, 2.0), (True, 0.3)])
def test_scalar_decisions_of_the_reverse_pass_are_bit_identical(storage, device_dt, amp):
    """The final scalar pass reading the reverse pass's correction decisions
    (ffx_scalar_reverse_ok, ffx_advect_scalars_ok) gives the fields of the final
    pass that traces forward again, bit for bit: the collider scene with traces
    of under half a cell and of about 2.5 cells (midpoints clipped at the
    colliders), host and device time steps, FP32 and BF16 storage."""
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    D = dev()
    runs = []
    for decide in (True, False):
        grid, s, colliders, emitters, noise = bench.scene(64, storage, 2, **bench.VARIANTS['fast'])
        sv = DenseProjectedSmoke(grid, s, D, colliders=colliders)
        if not decide:
            sv.detail.cell_decisions = lambda: None
        sv.upload(torch.zeros(grid.cells))
        sv.upload_temperature(torch.zeros(grid.cells))
        sv.upload_velocity([torch.as_tensor(v * (amp / 1e-3)) for v in noise])
        runs.append((sv, emitters))
    for k in range(4):
        for sv, em in runs:
            if device_dt:
                sv.step_cfl(0.5, 0.02, sources=em)
            else:
                sv.step(0.02, sources=em)
        torch.cuda.synchronize()
        (a, _), (b, _) = runs
        assert a.detail.cell_decisions() is not None
        for x, y in zip([a.density, a.temperature, *a._velocity], [b.density, b.temperature, *b._velocity]):
            assert torch.equal(x, y), (storage, device_dt, amp, k)
    for sv, _ in runs:
        sv.close()
