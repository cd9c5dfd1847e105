"""Batched uneven domains on the GPU: every domain's fields after batched
steps (one persistent launch per pass, device-side convergence loop and time
step, CUDA graph) are bit-identical to stepping that domain alone through the
single-domain solver with the same time-step rule; autotuned tile shapes and
persistent grids change nothing but speed."""
import numpy as np
import pytest
import torch

from fluxfx_b200.backend.batched import BatchedSmoke, batched_scenes, build_solvers

pytestmark = pytest.mark.gpu

CELL = 1.0 / 64.0


def device():
    from fluxfx_b200.backend.device import CudaDevice
    return CudaDevice()


def stepped_alone(scenes, steps):
    solvers, sources = build_solvers(scenes, device())
    out = []
    for s, src in zip(solvers, sources):
        dt, cycles = 0.02, []
        for _ in range(steps):
            s.step(dt, sources=src)
            cycles.append(s.projector.last_cycles)
            umax = max(s.projector.velocity_maxima())
            dt = min(0.02, 0.5 * CELL / umax) if umax > 0 else 0.02
        torch.cuda.synchronize()
        out.append(dict(density=s._front.clone(), temperature=s._temperature.clone(),
                        velocity=[v.clone() for v in s._velocity], dt=dt, cycles=cycles))
        s.close()
    return out


def compare(batch, ref, steps):
    stats = batch.stats()
    for i, r in enumerate(ref):
        density, temperature, velocity = batch.fields(i)
        assert torch.equal(density, r['density']), i
        assert torch.equal(temperature, r['temperature']), i
        for a, b in zip(velocity, r['velocity']):
            assert torch.equal(a, b), i
        assert stats[i]['steps'] == steps
        assert stats[i]['dt'] == np.float32(r['dt']), (i, stats[i]['dt'], r['dt'])
        assert stats[i]['last_cycles'] == r['cycles'][-1], (i, stats[i], r['cycles'])
        assert stats[i]['total_cycles'] == sum(r['cycles'])
        assert 0 < r['cycles'][-1] < 200
        assert float(density.abs().max()) > 0


def test_batched_steps_match_single_domain_steps():
    scenes = batched_scenes(6, seed=11, sizes=(32, 48, 64))
    ref = stepped_alone(scenes, 3)
    solvers, sources = build_solvers(scenes, device())
    batch = BatchedSmoke(solvers, sources)
    for _ in range(3):
        batch.run(1)            # one-step graphs of both parities
    compare(batch, ref, 3)
    batch.close()


def test_multi_step_graph_with_tuned_passes(tmp_path):
    scenes = batched_scenes(5, seed=12, sizes=(32, 64, 96))
    ref = stepped_alone(scenes, 4)
    solvers, sources = build_solvers(scenes, device())
    batch = BatchedSmoke(solvers, sources)
    cache = str(tmp_path / 'tuning.json')
    best = batch.tune(repeats=1, cache=cache)
    assert set(best) >= {'velocity', 'smooth', 'gradient'}
    assert batch.tune(cache=cache) == {k: tuple(v) for k, v in best.items()}    # served from the cache
    batch.run(3)                # one graph of three steps
    batch.run(1)
    compare(batch, ref, 4)
    assert batch.launches_per_step(ref[0]['cycles'][-1] + 1) > 10
    batch.close()


def test_warm_started_batch_matches_single_domain_steps():
    """Solves from the previous pressure (rescaled by dt / previous dt) take
    the same cycles and give the same fields as the single-domain solver with
    solid_warm_start."""
    scenes = batched_scenes(4, seed=13, sizes=(32, 48, 64), warm_start=True)
    ref = stepped_alone(scenes, 5)
    solvers, sources = build_solvers(scenes, device())
    batch = BatchedSmoke(solvers, sources)
    batch.run(5)
    compare(batch, ref, 5)
    batch.close()
