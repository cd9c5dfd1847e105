"""The playback-cache format (fluxfx_b200.physics.cache) on the host.

Pinned to the reference's bytes: the fixtures under tests/golden/cache_raw and
cache_zlib were written by the reference's own CacheWriter
(tests/golden/make_golden_cache.py); this reader reads them and this writer
reproduces them byte for byte. The behaviour checks follow the reference's
tests/test_cache.py and tests/test_cache_compression.py."""
import json
import random
import shutil
from pathlib import Path
from unittest.mock import patch
from zlib import compress, crc32

import numpy as np
import pytest

from fluxfx_b200.physics import cache
from fluxfx_b200.physics.config import GridSpec

GOLDEN = Path(__file__).resolve().parent / 'golden'
GRID = GridSpec((2, 3, 4), (0.5, 0.75, 1.0))


def golden_fields(frame):
    n = 24
    return {'DENSITY': np.array([0.25 * frame + 0.01 * i for i in range(n)], np.float32),
            'TEMPERATURE': np.array([-2.0 + 0.5 * frame - 0.125 * i for i in range(n)], np.float32)}


@pytest.mark.parametrize('name, encoding', [('cache_raw', 'RAW'), ('cache_zlib', 'AUTO_ZLIB')])
def test_reads_and_reproduces_reference_bakes(tmp_path, name, encoding):
    ref = GOLDEN / name
    r = cache.CacheReader(ref)
    assert r.grid == GRID and r.meta['status'] == 'CANCELLED'
    for frame in (1, 2):
        got = r.read(frame)
        for ch, want in golden_fields(frame).items():
            assert got[ch].tobytes() == want.tobytes()
    with pytest.raises(ValueError, match='not baked'):
        r.read(3)
    w = cache.CacheWriter(tmp_path, GRID, ['DENSITY', 'TEMPERATURE'], 1, 3, 24, cache.fingerprint({'golden': 1}),
                          provenance={'mode': 'STATIC'}, encoding=encoding)
    w.write(1, golden_fields(1))
    w.write(2, golden_fields(2))
    w.finish('CANCELLED', 'golden fixture')
    assert (w.path / 'manifest.json').read_bytes() == (ref / 'manifest.json').read_bytes()
    for frame in (1, 2):
        assert (w.path / f'frame_{frame}.fxc').read_bytes() == (ref / f'frame_{frame}.fxc').read_bytes()


@pytest.fixture
def writer(tmp_path):
    def make(encoding='RAW', grid=GridSpec((2, 3, 4)), channels=('DENSITY', 'TEMPERATURE'), start=1, end=2):
        return cache.CacheWriter(tmp_path, grid, list(channels), start, end, 24, cache.fingerprint({'test': 1}),
                                 encoding=encoding)
    return make


def fields(n=24):
    return {'DENSITY': [.5] * n, 'TEMPERATURE': [-2.] * n}


def test_roundtrip_cancel_and_isolation(writer):
    w = writer()
    w.write(1, fields())
    w.write(2, fields())
    w.finish()
    r = cache.CacheReader(w.path)
    assert list(r.read(2)['TEMPERATURE']) == [-2.] * 24 and r.meta['status'] == 'COMPLETE'
    w2 = writer()
    assert w2.path != w.path
    w2.write(1, fields())
    w2.finish('CANCELLED')
    r2 = cache.CacheReader(w2.path)
    assert len(r2.read(1)['DENSITY']) == 24
    with pytest.raises(ValueError):
        r2.read(2)


def test_order_completion_and_closed_writer(writer):
    w = writer()
    with pytest.raises(ValueError):
        w.write(2, fields())
    with pytest.raises(ValueError):
        w.finish()
    w.write(1, fields())
    with pytest.raises(ValueError):
        w.write(1, fields())
    with pytest.raises(ValueError, match='channels'):
        w.write(2, {'DENSITY': [.5] * 24})
    w.finish('FAILED', 'stop')
    with pytest.raises(ValueError, match='closed'):
        w.write(2, fields())
    with pytest.raises(ValueError):
        w.finish('UNKNOWN')


def test_invalid_fields_do_not_publish(writer):
    w = writer()
    for data in ([float('nan')] * 24, [-1.] * 24, [1.]):
        with pytest.raises(ValueError):
            w.write(1, dict(fields(), DENSITY=data))
    assert cache.CacheReader(w.path).meta['frames'] == {}
    assert not (w.path / 'frame_1.fxc').exists()
    w.write(1, dict(fields(), TEMPERATURE=[-5.] * 24))     # negative heat is valid
    assert cache.CacheReader(w.path).read(1)['TEMPERATURE'][0] == -5.


def test_corruption_and_manifest_validation(writer):
    w = writer()
    w.write(1, fields())
    p = w.path / 'frame_1.fxc'
    raw = bytearray(p.read_bytes())
    raw[0] ^= 1
    p.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match='checksum'):
        cache.CacheReader(w.path).read(1)
    p.write_bytes(b'x')
    with pytest.raises(ValueError, match='size'):
        cache.CacheReader(w.path).read(1)
    m = dict(w.meta, frames={'../../bad': {}})
    (w.path / 'manifest.json').write_text(json.dumps(m))
    with pytest.raises(ValueError):
        cache.CacheReader(w.path)
    for bad in (dict(w.meta, signature='short'), dict(w.meta, status='WEIRD'), dict(w.meta, format='other')):
        (w.path / 'manifest.json').write_text(json.dumps(bad))
        with pytest.raises(ValueError):
            cache.CacheReader(w.path)


def test_estimate_range_and_fingerprint():
    assert cache.estimate_bytes((64,) * 3, ['DENSITY', 'TEMPERATURE'], 1, 120) > 64 ** 3 * 8 * 120
    for args in [(2, 1, 24), (1, 10001, 24), (1, 2, 0), (1, 2, float('nan'))]:
        with pytest.raises(ValueError):
            cache.validate_range(*args)
    with pytest.raises(ValueError):
        cache.estimate_bytes((8,) * 3, ['DENSITY', 'DENSITY'], 1, 2)
    with pytest.raises(ValueError):
        cache.estimate_bytes((8,) * 3, ['SMOKE'], 1, 2)
    assert cache.fingerprint(dict(a=1, b=2)) == cache.fingerprint(dict(b=2, a=1))
    assert cache.fingerprint(dict(a=1)) != cache.fingerprint(dict(a=2))


def test_animated_manifest_requires_inputs(writer):
    w = writer()
    w.write(1, fields())
    w.meta['provenance'] = {'mode': 'ANIMATED_INPUTS', 'inputs': {}}
    w.publish()
    with pytest.raises(ValueError):
        cache.CacheReader(w.path)
    w.meta['provenance']['inputs']['1'] = cache.fingerprint({'x': 1})
    w.publish()
    assert cache.CacheReader(w.path).read(1)['DENSITY'][0] == .5


# ---------------------------------------------------------------- compression
def big_fields():
    return {'DENSITY': np.full(512, .25, np.float32), 'TEMPERATURE': np.full(512, -2., np.float32)}


def test_zlib_lossless_and_raw_fallback(writer):
    w = writer('AUTO_ZLIB', grid=GridSpec((8, 8, 8)))
    w.write(1, big_fields())
    w.write(2, big_fields())
    w.finish()
    r = cache.CacheReader(w.path)
    assert r.meta['format'] == cache.COMPRESSED_FORMAT and r.meta['frames']['1']['codec'] == 'ZLIB'
    assert r.meta['frames']['1']['bytes'] < 4096
    for k, v in r.read(2).items():
        assert v.tobytes() == big_fields()[k].tobytes()
    rng = random.Random(27)
    small = {k: np.array([rng.random() * 100 for _ in range(8)], np.float32) for k in ('DENSITY', 'TEMPERATURE')}
    w2 = writer('AUTO_ZLIB', grid=GridSpec((2, 2, 2)))
    w2.write(1, small)
    assert w2.meta['frames']['1']['codec'] == 'RAW'
    assert cache.CacheReader(w2.path).read(1)['DENSITY'].tobytes() == small['DENSITY'].tobytes()
    w3 = writer('RAW', grid=GridSpec((8, 8, 8)))
    w3.write(1, big_fields())
    assert w3.meta['format'] == cache.FORMAT and 'encoding' not in w3.meta
    assert set(w3.meta['frames']['1']) == {'bytes', 'crc32'}
    with pytest.raises(ValueError):
        writer('UNKNOWN')


def _rewrite(w, payload, **record):
    (w.path / 'frame_1.fxc').write_bytes(payload)
    w.meta['frames']['1'].update(bytes=len(payload), **record)
    w.publish()


def test_bounded_rejection_of_bad_compressed_frames(writer):
    def encoded():
        w = writer('AUTO_ZLIB', grid=GridSpec((8, 8, 8)))
        w.write(1, big_fields())
        return w
    for change in (lambda b: b[:-1], lambda b: b + b'extra', lambda b: b + b):
        w = encoded()
        _rewrite(w, change((w.path / 'frame_1.fxc').read_bytes()))
        with pytest.raises(ValueError, match='compressed|size'):
            cache.CacheReader(w.path).read(1)
    w = encoded()
    _rewrite(w, compress(b'\0' * 8192))
    with pytest.raises(ValueError, match='compressed'):
        cache.CacheReader(w.path).read(1)
    w = encoded()
    w.meta['frames']['1']['crc32'] = '00000000'
    w.publish()
    with pytest.raises(ValueError, match='checksum'):
        cache.CacheReader(w.path).read(1)
    for invalid in (float('nan'), float('inf'), -1.):
        w = encoded()
        raw = np.array([invalid] * 512 + [-2.] * 512, np.float32).tobytes()
        _rewrite(w, compress(raw), crc32=f'{crc32(raw):08x}')
        with pytest.raises(ValueError, match='field'):
            cache.CacheReader(w.path).read(1)
    for record in ({'bytes': True}, {'bytes': 4097}, {'raw_bytes': 8192}, {'codec': 'UNKNOWN'}):
        w = encoded()
        w.meta['frames']['1'].update(record)
        w.publish()
        with pytest.raises(ValueError):
            cache.CacheReader(w.path).read(1)
    w = encoded()
    w.meta['encoding'] = 'UNKNOWN'
    w.publish()
    with pytest.raises(ValueError):
        cache.CacheReader(w.path)


def test_failed_write_preserves_published_prefix(writer):
    w = writer('AUTO_ZLIB', grid=GridSpec((8, 8, 8)))
    w.write(1, big_fields())
    with patch.object(cache.os, 'fsync', side_effect=OSError('disk full')):
        with pytest.raises(OSError):
            w.write(2, big_fields())
    r = cache.CacheReader(w.path)
    assert set(r.meta['frames']) == {'1'} and r.read(1)['DENSITY'][0] == .25
    assert not (w.path / 'frame_2.tmp').exists() and not (w.path / 'frame_2.fxc').exists()
    w.write(2, big_fields())
    assert cache.CacheReader(w.path).read(2)['TEMPERATURE'][0] == -2.
