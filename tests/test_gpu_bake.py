"""Baking on the GPU: capture() and the asynchronous BakeRecorder.

The recorder snapshots each step's preview channels with one pack launch,
lets the solver run on, copies the snapshot to pinned memory on a copy stream
and writes the frame from a worker thread. The frames it bakes while steps
run back to back (no host synchronisation between them) must equal, bit for
bit, synchronous captures of an identical solver after the same steps."""
import numpy as np
import pytest
import torch

from fluxfx_b200.backend.cache import BakeRecorder, capture, channels_of
from fluxfx_b200.physics import cache
from fluxfx_b200.physics.config import GridSpec
from fluxfx_b200.physics.pressure import PressureSettings
from tests.gpu_helpers import dev, sphere_box_mask

pytestmark = pytest.mark.gpu


def _solver(D, storage, combustion):
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    grid = GridSpec((32, 24, 20))
    s = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=1.0,
                         source_center=(.5, .5, .2), source_radius=.2, storage=storage,
                         combustion_enabled=combustion, heat_source_rate=0.4 if combustion else 100.0,
                         ignition_temperature=0.3, burn_rate=0.75, heat_yield=1.0, smoke_yield=0.5)
    return DenseProjectedSmoke(grid, s, D, colliders=sphere_box_mask(grid.shape, grid.extent))


@pytest.mark.parametrize('storage, combustion, encoding', [('FP32', False, 'RAW'), ('BF16', True, 'AUTO_ZLIB')])
def test_async_bake_equals_synchronous_capture(tmp_path, storage, combustion, encoding):
    D = dev()
    a, b = _solver(D, storage, combustion), _solver(D, storage, combustion)
    names = channels_of(a)
    assert names == (['DENSITY', 'TEMPERATURE'] + (['FUEL', 'FLAME'] if combustion else []) + ['COLLISION'])
    frames = 6
    writer = cache.CacheWriter(tmp_path, a.grid, names, 1, frames, 24, cache.fingerprint({'bake': storage}),
                               encoding=encoding)
    rec = BakeRecorder(a, writer, depth=2)
    for f in range(1, frames + 1):
        a.step(0.02)
        rec.record(f)
    rec.finish()
    expected = []
    for _ in range(frames):
        b.step(0.02)
        expected.append(capture(b))
    r = cache.CacheReader(writer.path)
    assert r.meta['status'] == 'COMPLETE' and rec.d2h_bytes == frames * len(names) * a.grid.cells * 4
    for f in range(1, frames + 1):
        got = r.read(f)
        for name in names:
            assert got[name].tobytes() == expected[f - 1][name].tobytes(), (f, name)
    mask = expected[0]['COLLISION']
    assert set(np.unique(mask)) <= {0.0, 1.0} and mask.sum() > 0
    assert np.array_equal(mask, a.solids.mask.reshape(-1).cpu().numpy().astype(np.float32))
    want = b.density.float().reshape(-1).cpu().numpy()
    assert np.array_equal(expected[-1]['DENSITY'], want)
    a.close()
    b.close()


def test_failed_frame_marks_bake_failed(tmp_path):
    D = dev()
    a = _solver(D, 'FP32', False)
    writer = cache.CacheWriter(tmp_path, a.grid, channels_of(a), 1, 3, 24, cache.fingerprint({}))
    rec = BakeRecorder(a, writer, depth=1)
    a.step(0.02)
    rec.record(1)
    a._front.fill_(-1.0)          # a negative density is not a valid frame
    rec.record(2)
    with pytest.raises(ValueError, match='Invalid cache field'):
        rec.finish()
    r = cache.CacheReader(writer.path)
    assert r.meta['status'] == 'FAILED' and set(r.meta['frames']) == {'1'}
    a.close()
