"""The CUDA path, driven through the drop-in DenseProjectedSmoke API, replays
the reference backend's own runs (tests/golden/reference_steps.npz): same
seeded inputs, same settings, fields compared per recorded step."""
import numpy as np
import pytest
import torch

from tests import reference_cases as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def device():
    from fluxfx_b200.backend.device import CudaDevice
    return CudaDevice()


def host(t):
    torch.cuda.synchronize()
    return t.detach().to(torch.float64).cpu().numpy()


@pytest.mark.parametrize('name', R.cases())
def test_cuda_path_matches_reference_backend(device, name):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.physics.config import GridSpec
    c = R.case(name)
    solver = DenseProjectedSmoke(GridSpec(c['shape']), c['settings'], device, colliders=c['colliders'])
    if c['mask'] is not None:
        assert np.array_equal(host(solver.solids.mask) > 0.5, c['mask'])      # bit-exact raster
    R.compare(host(solver.density), c['init_density'], R.TOL, 'seeded density')
    R.compare(host(solver.temperature), c['init_temperature'], R.TOL, 'seeded temperature')
    solver.upload_velocity([torch.as_tensor(v) for v in c['velocity']])
    for k, dt in enumerate(c['dts']):
        solver.step(dt, emission=c['emission'], sources=c['sources'])
        if k not in c['steps']:
            continue
        want = c['steps'][k]
        R.compare(host(solver.density), want['density'], R.TOL, f'step {k} density')
        R.compare(host(solver.temperature), want['temperature'], R.TOL, f'step {k} temperature')
        for a in range(3):
            R.compare(host(solver._velocity[a]), want['velocity'][a], R.TOL, f'step {k} velocity {a}')
        R.compare_after(host(solver.projector.after), want, f'step {k} divergence after')
        m = solver.measure_projection()
        ref_m = want['metrics']
        for key in ('v_cycles', 'iterations', 'solver', 'pressure_storage'):
            if key in ref_m:
                assert m[key] == ref_m[key], (key, m[key], ref_m[key])
    solver.close()
