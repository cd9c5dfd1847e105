"""Error of the FP32 and the mixed (BF16 storage, FP32 arithmetic) forms of
the collider smoke step against an FP64 run of the oracle, per field, on the
256^3 benchmark scene scaled to 48^3 (sphere and box colliders, two TARGET
emitters, MacCormack, projection to relative divergence 1e-4). Both GPU forms
use the fastest solver configuration (over-corrected V-cycles, warm start);
the oracle runs the reference's V(4,4) cycles: at the solve tolerance the
pressure, and so every field, agrees to about the tolerance."""
import numpy as np
import pytest
import torch

from oracle import solver as O
from tests.gpu_helpers import n

pytestmark = pytest.mark.gpu

N = 48
STEPS = 4
DT = 0.02


def scene():
    from fluxfx_b200.physics.collision import primitive
    from fluxfx_b200.physics.config import GridSpec
    from fluxfx_b200.physics.emission import Emission, Source
    from fluxfx_b200.physics.pressure import PressureSettings
    grid = GridSpec((N, N, N))
    h, c = 1.0 / N, N / 256.0
    sphere = primitive('SPHERE', (0.5, 0.5, 0.5), (40 * c * h,) * 3)
    box = primitive('BOX', (60 * c * h, 130 * c * h, 40 * c * h), (20 * c * h, 30 * c * h, 20 * c * h))
    emitters = [Source((0.3, 0.7, 0.2), 8 * c * h * 2, 0.8, 0.6, Emission((0.3, 0.7, 0.2)), 'TARGET', 'SOFT'),
                Source((0.7, 0.35, 0.15), 8 * c * h * 2, 0.7, 0.9, Emission((0.7, 0.35, 0.15)), 'TARGET', 'SOFT')]
    base = dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=1.0,
                density_weight=0.05, dissipation=0.0, cooling=0.0, heat_mode='TARGET', pressure_tolerance=1e-4,
                pressure_max_cycles=200)
    rng = np.random.default_rng(5)
    noise = [rng.uniform(-1e-3, 1e-3, (fs[2], fs[1], fs[0])).astype(np.float32) for fs in grid.face_shapes]
    return grid, base, (sphere, box), emitters, noise


def gpu_run(storage):
    from fluxfx_b200.backend.device import CudaDevice
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.physics.pressure import PressureSettings
    grid, base, colliders, emitters, noise = scene()
    s = PressureSettings(**base, storage=storage, solid_warm_start=True, mg_coarse_scale=1.6)
    solver = DenseProjectedSmoke(grid, s, CudaDevice(), colliders=colliders)
    solver.upload(torch.zeros(grid.cells))
    solver.upload_temperature(torch.zeros(grid.cells))
    solver.upload_velocity([torch.as_tensor(v) for v in noise])
    for _ in range(STEPS):
        solver.step(DT, sources=emitters)
    out = dict(density=n(solver.density), temperature=n(solver.temperature),
               u=n(solver._velocity[0]), v=n(solver._velocity[1]), w=n(solver._velocity[2]),
               mask=n(solver.solids.mask).astype(bool))
    solver.close()
    return out


def test_fp32_and_mixed_forms_against_fp64():
    from fluxfx_b200.physics.emission import pack_sources
    from fluxfx_b200.physics.pressure import PressureSettings
    fp32, mixed = gpu_run('FP32'), gpu_run('BF16')
    grid, base, colliders, emitters, noise = scene()
    ref = O.OracleSmoke(grid.shape, grid.extent, PressureSettings(**base), np.float64, mask=fp32['mask'])
    zeros = np.zeros(grid.shape[::-1])
    ref.upload(density=zeros, temperature=zeros, velocity=tuple(v.astype(np.float64) for v in noise))
    table = (pack_sources(emitters), len(emitters))
    for _ in range(STEPS):
        ref.step(DT, sources=table)
    exact = dict(density=ref.density, temperature=ref.temperature, u=ref.velocity[0], v=ref.velocity[1],
                 w=ref.velocity[2])
    report = {}
    for name, e in exact.items():
        scale = max(float(np.abs(e).max()), 1e-30)
        report[name] = (float(np.abs(fp32[name] - e).max()) / scale, float(np.abs(mixed[name] - e).max()) / scale)
    print('\nrelative max error vs FP64 (FP32, BF16 storage):',
          {k: (f'{a:.2e}', f'{b:.2e}') for k, (a, b) in report.items()})
    for name, (a, b) in report.items():
        assert a <= 2e-3, (name, report)
        assert b <= 3e-2, (name, report)
