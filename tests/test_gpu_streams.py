"""A solver on its own CUDA stream: every pass, torch op and readback of a
step is ordered on that stream, so fields, statistics and cycle counts equal
those of the same solver on torch's current stream, while the current stream
stays free (the fire workload runs four domains on four streams)."""
import pytest
import torch

from tests.gpu_helpers import dev

pytestmark = pytest.mark.gpu


def _solver(device, variant):
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    grid, s, colliders, emitters, noise = bench.scene(64, 'FP32', 5, **bench.VARIANTS[variant])
    sv = DenseProjectedSmoke(grid, s, device, colliders=colliders)
    sv.upload(torch.zeros(grid.cells))
    sv.upload_temperature(torch.zeros(grid.cells))
    sv.upload_velocity([torch.as_tensor(v) for v in noise])
    return sv, emitters


@pytest.mark.parametrize('variant', ['plain', 'fast'])
def test_side_stream_solver_equals_current_stream_solver(variant):
    from fluxfx_b200.backend.device import CudaDevice
    dev()
    a, em = _solver(CudaDevice(), variant)
    side = torch.cuda.Stream()
    b, _ = _solver(CudaDevice(stream=side), variant)
    torch.cuda.synchronize()
    for k in range(3):
        a.step(0.02, sources=em)
        b.step(0.02, sources=em)
        # no synchronisation here: the readbacks below must order themselves
        mb = b.measure_projection()
        ma = a.measure_projection()
        assert mb['rel_div_inf'] == ma['rel_div_inf'] and mb['v_cycles'] == ma['v_cycles'] > 0, (k, ma, mb)
        assert b.projector.velocity_maxima() == a.projector.velocity_maxima(), k
        assert b.scalar_maxima() == a.scalar_maxima(), k
    torch.cuda.synchronize()
    for x, y in zip([a.density, a.temperature, a.projector.pressure, *a._velocity],
                    [b.density, b.temperature, b.projector.pressure, *b._velocity]):
        assert torch.equal(x, y)
    a.close()
    b.close()
