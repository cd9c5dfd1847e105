"""Checkpoint v1 format validation on the host (no GPU needed): the loader
rejects every malformed file before it builds a solver, as
``fluxfx/backend/checkpoint.py:41-58`` does."""
import json
from dataclasses import asdict

import numpy as np
import pytest

from fluxfx_b200.backend import checkpoint as K
from fluxfx_b200.physics.config import GridSpec
from fluxfx_b200.physics.pressure import PressureSettings


def _write(path, meta, arrays):
    with open(path, 'wb') as f:
        np.savez_compressed(f, metadata=json.dumps(meta), **arrays)


def _valid(shape=(4, 3, 2), **settings_kw):
    grid = GridSpec(shape)
    settings = asdict(PressureSettings(**settings_kw))
    ext = {k: settings.pop(k) for k in K.EXTENSION_SETTINGS}
    meta = {'format': K.FORMAT, 'settings': settings, 'grid': {'shape': list(shape), 'extent': [1.0, 1.0, 1.0]},
            'time': 0.5, 'steps': 3, 'last_dt': 0.02, 'extensions': ext}
    n = grid.cells
    arrays = {'density': np.full(n, 0.5, np.float32), 'temperature': np.zeros(n, np.float32),
              'pressure': np.zeros(n, np.float32)}
    for i, fs in enumerate(grid.face_shapes):
        arrays[f'velocity{i}'] = np.zeros(int(np.prod(fs)), np.float32)
    return meta, arrays


@pytest.mark.parametrize('mutate, message', [
    (lambda m, a: m.update(format='fluxfx-checkpoint-0'), 'Unsupported checkpoint format'),
    (lambda m, a: m.update(time=-1.0), 'Invalid checkpoint clock'),
    (lambda m, a: m.update(time=float('inf')), 'Invalid checkpoint clock'),
    (lambda m, a: m.update(steps=1.5), 'Invalid checkpoint clock'),
    (lambda m, a: m.update(last_dt=0.5), 'timestep must be finite'),
    (lambda m, a: a.update(density=np.zeros(5, np.float32)), 'Invalid field: density'),
    (lambda m, a: a.update(velocity1=np.full(a['velocity1'].size, np.nan, np.float32)), 'Invalid field: velocity1'),
    (lambda m, a: a.update(density=np.full(a['density'].size, -1.0, np.float32)), 'Negative field: density'),
    (lambda m, a: a.pop('pressure'), 'Missing field: pressure'),
    (lambda m, a: a.update(temperature=a['temperature'].astype(np.float64)), 'Invalid field: temperature'),
    (lambda m, a: m['settings'].update(not_a_setting=1), 'Unknown checkpoint settings'),
    (lambda m, a: m['settings'].update(pressure_cycles=0), 'Multigrid cycles'),
    (lambda m, a: m.update(format=K.FORMAT_COLLIDERS), 'without colliders'),
])
def test_loader_rejects_malformed_files(tmp_path, mutate, message):
    meta, arrays = _valid()
    mutate(meta, arrays)
    path = tmp_path / 'bad.npz'
    _write(path, meta, arrays)
    with pytest.raises(ValueError, match=message):
        K.load_checkpoint(path)


def test_combustion_checkpoint_needs_fuel_and_flame(tmp_path):
    meta, arrays = _valid(combustion_enabled=True)
    path = tmp_path / 'fire.npz'
    _write(path, meta, arrays)
    with pytest.raises(ValueError, match='Missing field: fuel'):
        K.load_checkpoint(path)
    n = arrays['density'].size
    arrays.update(fuel=np.zeros(n, np.float32), flame=np.full(n, -2.0, np.float32))
    _write(path, meta, arrays)
    with pytest.raises(ValueError, match='Negative field: flame'):
        K.load_checkpoint(path)


def test_reference_settings_and_extensions_are_split():
    """``settings`` carries only the reference's fields, so a reference reader
    can build its PressureSettings from it; the additions sit in ``extensions``."""
    meta, _ = _valid(pressure_tolerance=1e-4, storage='BF16')
    assert not set(meta['settings']) & set(K.EXTENSION_SETTINGS)
    assert meta['extensions']['storage'] == 'BF16'
    s = K._settings(meta)
    assert s.storage == 'BF16' and s.pressure_tolerance == 1e-4
