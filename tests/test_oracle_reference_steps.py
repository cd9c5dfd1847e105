"""The CPU oracle replays the reference backend's own runs (its Python
orchestration driving its compute shaders, compiled for the CPU). This pins
the shader-only parts of the oracle: MacCormack, closed/collider sampling,
trace clipping, emitters, geometric and aggregation multigrid. CPU only."""
import numpy as np
import pytest

from oracle.solver import OracleSmoke
from tests import reference_cases as R


@pytest.mark.parametrize('name', R.cases())
def test_oracle_matches_reference_backend(name):
    c = R.case(name)
    ref = OracleSmoke(c['shape'], (1.0, 1.0, 1.0), c['settings'], np.float32, mask=c['mask'])
    R.compare(ref.density, c['init_density'], R.TOL, 'seeded density')
    R.compare(ref.temperature, c['init_temperature'], R.TOL, 'seeded temperature')
    ref.upload(velocity=c['velocity'])
    table = None
    if c['sources'] is not None:
        from fluxfx_b200.physics.emission import pack_sources
        table = (pack_sources(c['sources']), len(c['sources']))
    for k, dt in enumerate(c['dts']):
        ref.step(dt, emission=c['emission'], sources=table)
        if k not in c['steps']:
            continue
        want = c['steps'][k]
        R.compare(ref.density, want['density'], R.TOL, f'step {k} density')
        R.compare(ref.temperature, want['temperature'], R.TOL, f'step {k} temperature')
        for a in range(3):
            R.compare(ref.velocity[a], want['velocity'][a], R.TOL, f'step {k} velocity {a}')
        R.compare_after(ref.after, want, f'step {k} divergence after')
