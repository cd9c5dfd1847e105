"""The CPU oracle replays the reference backend's own fire-configuration runs
(vorticity confinement, combustion, moving colliders; its Python
orchestration driving its compute shaders compiled for the CPU). CPU only."""
import numpy as np
import pytest

from oracle.solver import OracleSmoke
from tests import reference_cases as R


def replay(name):
    c = R.case(name, R.FIRE)
    cols = None
    if c['moving'] is not None:
        cols = [(m.shape, m.inverse_rows) for m in c['moving'](0)]
    ref = OracleSmoke(c['shape'], (1.0, 1.0, 1.0), c['settings'], np.float32,
                      mask=None if cols else c['mask'], colliders=cols)
    if cols:
        assert np.array_equal(ref.g.mask, c['mask'])
    R.compare(ref.density, c['init_density'], R.TOL, 'seeded density')
    R.compare(ref.temperature, c['init_temperature'], R.TOL, 'seeded temperature')
    ref.upload(velocity=c['velocity'])
    table = None
    if c['sources'] is not None:
        from fluxfx_b200.physics.emission import pack_sources
        table = (pack_sources(c['sources']), len(c['sources']))
    return c, ref, table


@pytest.mark.parametrize('name', R.fire_cases())
def test_oracle_matches_reference_fire_runs(name):
    c, ref, table = replay(name)
    for k, dt in enumerate(c['dts']):
        if c['moving'] is not None:
            ref.move_colliders([(m.shape, m.inverse_rows) for m in c['moving'](k + 1)], dt)
        ref.step(dt, sources=table)
        if k not in c['steps']:
            continue
        want = c['steps'][k]
        R.compare(ref.density, want['density'], R.TOL, f'step {k} density')
        R.compare(ref.temperature, want['temperature'], R.TOL, f'step {k} temperature')
        for a in range(3):
            R.compare(ref.velocity[a], want['velocity'][a], R.TOL, f'step {k} velocity {a}')
        R.compare_after(ref.after, want, f'step {k} divergence after')
        if 'fuel' in want:
            R.compare(ref.fuel, want['fuel'], R.TOL, f'step {k} fuel')
            R.compare(ref.flame, want['flame'], R.TOL, f'step {k} flame')
        if 'mask' in want:
            assert np.array_equal(ref.owners, want['mask']), f'step {k} owner mask'
