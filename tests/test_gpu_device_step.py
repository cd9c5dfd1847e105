"""Steps with no host round trip: the device-side time step (step_cfl,
ffx_next_dt) and the device-side V-cycle loop (ffx_loop_*, a CUDA graph with
a WHILE node).

* The loop: a tolerance solve run as one graph takes the same cycles and gives
  the same fields, bit for bit, as the host loop that reads the residual back
  after every cycle.
* The time step: stepping with dt = min(0.02, 0.5 h / max|u|) chosen on the
  device gives the fields of host steps that read the maxima back and choose
  the same dt (bit-identical for cold-started solves; the warm start's dt /
  previous dt ratio is formed from FP32 time steps on the device, so that
  variant agrees to the per-step tolerance of the other parity tests).
* No readback: after the first step (which captures the graphs), queuing a
  step never converts a device tensor to a host value.
"""
from unittest.mock import patch

import numpy as np
import pytest
import torch

from tests.gpu_helpers import dev

pytestmark = pytest.mark.gpu

H = 1.0 / 64


def _solver(D, variant, **overrides):
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    grid, s, colliders, emitters, noise = bench.scene(64, 'FP32', 3, **dict(bench.VARIANTS[variant], **overrides))
    sv = DenseProjectedSmoke(grid, s, D, colliders=colliders)
    if s.learned_warm_start:
        from fluxfx_b200.learned import attach
        attach(sv, colliders)
    sv.upload(torch.zeros(grid.cells))
    sv.upload_temperature(torch.zeros(grid.cells))
    sv.upload_velocity([torch.as_tensor(v) for v in noise])
    return sv, emitters


def _fields(sv):
    torch.cuda.synchronize()
    return [sv.density, sv.temperature, sv.projector.pressure, *sv._velocity]


def test_device_loop_equals_host_loop():
    D = dev()
    a, em = _solver(D, 'plain')
    b, _ = _solver(D, 'plain')
    b.projector.use_device_loop = False
    for k in range(4):
        a.step(0.02, sources=em)
        b.step(0.02, sources=em)
        assert a.projector.last_cycles == b.projector.last_cycles > 0, k
        for x, y in zip(_fields(a), _fields(b)):
            assert torch.equal(x, y), k
    assert a.projector.total_cycles() == b.projector.total_cycles()
    a.close()
    b.close()


@pytest.mark.parametrize('variant', ['plain', 'learned'])
def test_device_time_step_equals_host_time_step(variant):
    D = dev()
    a, em = _solver(D, variant)
    b, _ = _solver(D, variant)
    dt = 0.02
    for k in range(5):
        a.step_cfl(0.5, 0.02, sources=em)
        b.step(dt, sources=em)
        for x, y in zip(_fields(a), _fields(b)):
            assert torch.equal(x, y), (variant, k)
        umax = max(b.projector.velocity_maxima())
        dt = min(0.02, 0.5 * H / umax) if umax > 0 else 0.02
        assert a.current_dt() == np.float32(dt), (k, a.current_dt(), dt)
    assert abs(a.time - b.time) <= 1e-6 * b.time and a.steps == b.steps == 5
    a.close()
    b.close()


def test_warm_started_device_steps_agree_with_host_steps():
    D = dev()
    a, em = _solver(D, 'fast')
    b, _ = _solver(D, 'fast')
    dt = 0.02
    for k in range(5):
        a.step_cfl(0.5, 0.02, sources=em)
        b.step(dt, sources=em)
        for x, y in zip(_fields(a)[:2] + _fields(a)[3:], _fields(b)[:2] + _fields(b)[3:]):
            scale = float(y.abs().max())
            assert float((x - y).abs().max()) <= 1e-5 * max(scale, 1e-30), k
        umax = max(b.projector.velocity_maxima())
        dt = min(0.02, 0.5 * H / umax) if umax > 0 else 0.02
    a.close()
    b.close()


def test_device_steps_read_nothing_back():
    D = dev()
    a, em = _solver(D, 'learned')
    a.step_cfl(0.5, 0.02, sources=em)            # captures the solve graph
    torch.cuda.synchronize()

    def forbidden(*args, **kwargs):
        raise AssertionError('a device value was read back during a step')
    with patch.object(torch.Tensor, 'item', forbidden), patch.object(torch.Tensor, 'tolist', forbidden), \
            patch.object(torch.Tensor, 'cpu', forbidden), patch.object(torch.Tensor, '__float__', forbidden), \
            patch.object(torch.Tensor, '__int__', forbidden), patch.object(torch.Tensor, '__bool__', forbidden):
        for _ in range(3):
            a.step_cfl(0.5, 0.02, sources=em)
    torch.cuda.synchronize()
    assert a.steps == 4 and a.projector.last_cycles > 0
    assert a.measure_projection()['rel_div_inf'] <= 1e-4
    a.close()


@pytest.mark.parametrize('inner', [1, 2])
def test_iterative_refinement_reaches_the_tolerance(inner):
    """pressure_method='IR': every outer iteration recomputes the true FP32
    residual, decides in FP64, solves the correction equation from zero with
    `inner` V-cycles and adds the correction. It reaches the same tolerance as
    the V-cycle loop with about the same V-cycles, and the two solutions differ
    by what the tolerance allows (both corrected velocities have relative
    divergence <= 1e-4, their difference is a discrete gradient)."""
    D = dev()
    a, em = _solver(D, 'fast')
    b, _ = _solver(D, 'fast', pressure_method='IR', ir_inner_cycles=inner)
    for k in range(4):
        a.step(0.02, sources=em)
        b.step(0.02, sources=em)
        ma, mb = a.measure_projection(), b.measure_projection()
        assert ma['rel_div_inf'] <= 1e-4 and mb['rel_div_inf'] <= 1e-4, (k, ma, mb)
        ca, cb = a.projector.last_cycles, b.projector.last_cycles
        assert cb % inner == 0 and abs(cb - ca) <= inner + 1, (k, ca, cb)
        for x, y in zip(a._velocity, b._velocity):
            scale = float(y.abs().max())
            assert float((x - y).abs().max()) <= 2e-3 * scale, k
    a.close()
    b.close()
