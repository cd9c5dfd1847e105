"""The shared-memory-tiled transport passes against the untiled gathers.

Every transport pass (face predictor, velocity, scalar predictor / reverse,
final scalars) has a tiled form, selected by ffx_set_transport_tiling(1), beside
the default untiled gathers. Both read the same values and do the same arithmetic, so the
fields after full steps must be bit-identical -- on ragged and power-of-two
grids, with colliders and emitters, in FP32 and BF16 storage, and with time
steps whose traces run past the staged window (the global fallback)."""
import numpy as np
import pytest
import torch

from fluxfx_b200 import _native as N
from fluxfx_b200.physics.config import GridSpec
from fluxfx_b200.physics.emission import Emission, Source
from fluxfx_b200.physics.pressure import PressureSettings
from tests.gpu_helpers import dev, sphere_box_mask

pytestmark = pytest.mark.gpu

CASES = {
    # ragged tiles (x not a multiple of 32, y not of 8), non-power-of-two spacing
    'ragged_colliders_fp32': dict(shape=(40, 20, 17), extent=(1.3, 0.8, 0.7), storage='FP32', colliders=True,
                                  speed=0.3, dts=(0.02, 0.02, 0.1)),
    # power-of-two grid (exact reciprocals, reused departure points), BF16 storage
    'pow2_colliders_bf16': dict(shape=(64, 32, 32), extent=(1.0, 0.5, 0.5), storage='BF16', colliders=True,
                                speed=0.5, dts=(0.02, 0.05)),
    # traces of several cells: most samples leave the window
    'fast_flow_no_colliders': dict(shape=(32, 32, 32), extent=(1.0, 1.0, 1.0), storage='FP32', colliders=False,
                                   speed=2.0, dts=(0.05, 0.1)),
}


@pytest.mark.parametrize('case', sorted(CASES))
def test_tiled_transport_is_bit_identical_to_untiled(case):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    spec = CASES[case]
    lib = N.load()
    D = dev()
    grid = GridSpec(spec['shape'], spec['extent'])
    s = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=1.0,
                         density_weight=0.05, heat_mode='TARGET', storage=spec['storage'], pressure_cycles=2)
    cols = sphere_box_mask(grid.shape, grid.extent) if spec['colliders'] else ()
    e = spec['extent']
    sources = [Source((.3 * e[0], .5 * e[1], .3 * e[2]), .15 * min(e), 1.0, 2.0, Emission((.3 * e[0], .5 * e[1], .3 * e[2])),
                      'TARGET', 'SOFT'),
               Source((.7 * e[0], .4 * e[1], .2 * e[2]), .1 * min(e), .5, 1.0,
                      Emission((.68 * e[0], .4 * e[1], .2 * e[2]), (0, 0, 1), 1.5))]
    rng = np.random.default_rng(7)
    vel = [torch.as_tensor((rng.uniform(-1, 1, (fs[2], fs[1], fs[0])) * spec['speed']).astype(np.float32))
           for fs in grid.face_shapes]
    dens = torch.as_tensor(rng.uniform(0, 1, grid.cells).astype(np.float32))
    previous = lib.ffx_set_transport_tiling(0)
    solvers = []
    for _ in range(2):
        sv = DenseProjectedSmoke(grid, s, D, colliders=cols)
        sv.upload(dens)
        sv.upload_temperature(dens * 2)
        sv.upload_velocity(vel)
        solvers.append(sv)
    try:
        for k, dt in enumerate(spec['dts']):
            for tiled, sv in zip((1, 0), solvers):
                lib.ffx_set_transport_tiling(tiled)
                sv.step(dt, sources=sources)
            torch.cuda.synchronize()
            a, b = solvers
            assert torch.equal(a.density, b.density), (k, 'density')
            assert torch.equal(a.temperature, b.temperature), (k, 'temperature')
            for axis in range(3):
                assert torch.equal(a._velocity[axis], b._velocity[axis]), (k, 'velocity', axis)
            assert a.projector.velocity_maxima() == b.projector.velocity_maxima()
            assert torch.equal(a._maxima, b._maxima)
    finally:
        lib.ffx_set_transport_tiling(previous)
        for sv in solvers:
            sv.close()
