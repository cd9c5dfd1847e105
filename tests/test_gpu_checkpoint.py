"""Checkpoint v1 round trips on the GPU: a run saved after some steps and
loaded into a new solver continues bit-identically to the run that was saved
(the reference's own check, ``scripts/combustion_validate.py:55-60``, allows
1e-4; resuming here is exact). Covers the collider-free geometric multigrid,
static colliders (the extension), BF16 storage and combustion; the atomic
write keeps the previous file when a save fails."""
import json

import numpy as np
import pytest
import torch

from fluxfx_b200.backend.checkpoint import FORMAT, FORMAT_COLLIDERS, advance_fixed, load_checkpoint, save_checkpoint
from fluxfx_b200.physics.config import GridSpec
from fluxfx_b200.physics.emission import Emission, Source
from fluxfx_b200.physics.pressure import PressureSettings
from tests.gpu_helpers import dev, sphere_box_mask

pytestmark = pytest.mark.gpu

CASES = {
    'multigrid_fp32': dict(shape=(32, 32, 32), colliders=False, settings=dict(pressure_cycles=3)),
    'colliders_bf16_warm': dict(shape=(24, 20, 16), colliders=True,
                                settings=dict(storage='BF16', pressure_tolerance=1e-4, solid_warm_start=True,
                                              mg_coarse_scale=1.9)),
    'combustion': dict(shape=(16, 16, 16), colliders=False,
                       settings=dict(combustion_enabled=True, fuel_source_rate=1.0, ignition_temperature=0.3,
                                     burn_rate=0.75, heat_yield=1.0, smoke_yield=0.5, heat_source_rate=0.4,
                                     heat_mode='TARGET', vorticity_strength=0.3)),
}


def _fields(s):
    torch.cuda.synchronize()
    out = [s.density.clone(), s.temperature.clone(), s.projector.pressure.clone()] + [v.clone() for v in s._velocity]
    if s.combustion is not None:
        out += [s.combustion.fuel.clone(), s.combustion.flame.clone()]
    return out


@pytest.mark.parametrize('case', sorted(CASES))
def test_resume_is_bit_identical(tmp_path, case):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    spec = CASES[case]
    D = dev()
    grid = GridSpec(spec['shape'])
    s = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=1.0,
                         density_weight=0.05, source_center=(.5, .5, .25), source_radius=.2, **spec['settings'])
    cols = sphere_box_mask(grid.shape, grid.extent) if spec['colliders'] else ()
    a = DenseProjectedSmoke(grid, s, D, colliders=cols)
    sources = [Source((.4, .5, .3), .15, 1.0, 0.8, Emission((.4, .5, .3)), 'TARGET', 'SOFT')]
    advance_fixed(a, 4, 0.02, sources=sources)
    path = tmp_path / 'run.npz'
    save_checkpoint(a, path)
    with np.load(path) as archive:
        meta = json.loads(str(archive['metadata']))
    assert meta['format'] == (FORMAT_COLLIDERS if cols else FORMAT)
    b = load_checkpoint(path, D)
    try:
        assert (b.time, b.steps) == (a.time, a.steps)
        assert b.projector.last_dt == a.projector.last_dt
        if cols:
            assert torch.equal(b.solids.mask, a.solids.mask) and torch.equal(b.solids.halo, a.solids.halo)
        for x, y in zip(_fields(a), _fields(b)):
            assert torch.equal(x, y)
        advance_fixed(a, 3, 0.02, sources=sources)
        advance_fixed(b, 3, 0.02, sources=sources)
        for k, (x, y) in enumerate(zip(_fields(a), _fields(b))):
            assert torch.equal(x, y), k
        assert a.projector.last_cycles == b.projector.last_cycles
    finally:
        a.close()
        b.close()


def test_failed_save_keeps_previous_file(tmp_path):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    D = dev()
    grid = GridSpec((8, 8, 8))
    a = DenseProjectedSmoke(grid, PressureSettings(pressure_iterations=10), D)
    advance_fixed(a, 1, 0.02)
    path = tmp_path / 'run.npz'
    save_checkpoint(a, path)
    before = path.read_bytes()
    a._front.fill_(float('nan'))
    with pytest.raises(ValueError, match='Nonfinite'):
        save_checkpoint(a, path)
    assert path.read_bytes() == before and not (tmp_path / 'run.npz.tmp').exists()
    a.faulted = True
    with pytest.raises(ValueError, match='healthy'):
        save_checkpoint(a, path)
    a.close()
