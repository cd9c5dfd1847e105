"""Portable, bounded, atomic playback cache ("bake") -- the on-disk format.

Drop-in for FluxFX ``fluxfx/physics/cache.py:1-182``; the files it writes are
read by the reference's ``CacheReader`` and vice versa. A bake is a directory
``fluxfx-bake-<12 hex>`` holding ``manifest.json`` and one ``frame_<n>.fxc``
per frame:

* a frame file is the channels' little-endian float32 fields, x-fast, in the
  manifest's channel order (format ``fluxfx-playback-1``, encoding RAW), or,
  with encoding ``AUTO_ZLIB`` (format ``fluxfx-playback-2``), that byte string
  compressed with zlib level 1 when that is smaller (codec ``ZLIB``), else raw;
* the manifest (sorted keys, no NaN) records the grid, channels, frame range,
  fps, input signature, provenance, status (BAKING / COMPLETE / CANCELLED /
  FAILED) and per frame the stored size and the CRC-32 of the raw bytes
  (plus codec and raw size in format 2).

Frames are written once, in order; every file and the manifest are written to
a temporary name, fsynced and renamed, so a reader never sees a partial frame
and a failed write leaves the published prefix intact. Fields must be finite
and, except TEMPERATURE, non-negative. The reader bounds every size before it
allocates or decompresses.
"""
import json
import os
import sys
from hashlib import sha256
from math import isfinite, prod
from pathlib import Path
from uuid import uuid4
from zlib import compress, crc32, decompressobj, error as ZlibError

import numpy as np

from .config import GridSpec

FORMAT = 'fluxfx-playback-1'
COMPRESSED_FORMAT = 'fluxfx-playback-2'
ENCODINGS = ('RAW', 'AUTO_ZLIB')
CHANNELS = ('DENSITY', 'TEMPERATURE', 'FUEL', 'FLAME', 'COLLISION')
STATUSES = ('BAKING', 'COMPLETE', 'CANCELLED', 'FAILED')
MAX_FRAMES = 10000
MAX_MANIFEST_BYTES = 4 * 1024 * 1024


def valid_field(values, channel):
    """Finite, and non-negative unless the channel is TEMPERATURE."""
    v = np.asarray(values, dtype=np.float32)
    return bool(np.isfinite(v).all() and (channel == 'TEMPERATURE' or not (v < 0).any()))


def fingerprint(value):
    """SHA-256 of the canonical JSON of ``value`` (sorted keys, compact)."""
    text = json.dumps(value, sort_keys=True, separators=(',', ':'), allow_nan=False)
    return sha256(text.encode()).hexdigest()


def validate_range(start, end, fps):
    if type(start) is not int or type(end) is not int or not -1048574 <= start <= end <= 1048574 \
            or end - start >= MAX_FRAMES:
        raise ValueError('Use an ordered range of at most 10,000 frames')
    if not isfinite(fps) or not 0 < fps <= 1000:
        raise ValueError('Invalid cache frame rate')


def estimate_bytes(shape, channels, start, end):
    """Upper bound of a bake's size: raw fields plus manifest/filesystem slack."""
    GridSpec(tuple(shape))
    validate_range(start, end, 24)
    if not channels or len(set(channels)) != len(channels) or any(c not in CHANNELS for c in channels):
        raise ValueError('Invalid cache channels')
    return (prod(shape) * 4 * len(channels) + 4096) * (end - start + 1) + 65536


def _replace_atomically(path, payload):
    """Write ``payload`` (bytes) to ``path`` through a fsynced temporary file."""
    temp = path.with_name(path.name + '.tmp')
    try:
        with temp.open('wb') as stream:
            stream.write(payload)
            stream.flush()
            os.fsync(stream.fileno())
        temp.replace(path)
    finally:
        if temp.exists():
            temp.unlink()


def atomic_json(path, value):
    _replace_atomically(Path(path), json.dumps(value, sort_keys=True, allow_nan=False).encode())


def _le_bytes(values):
    a = np.ascontiguousarray(values, dtype=np.float32)
    if sys.byteorder != 'little':
        a = a.byteswap()
    return a.tobytes()


class CacheWriter:
    """Writes one bake under ``parent`` (``physics/cache.py:61-139``)."""

    def __init__(self, parent, grid, channels, start, end, fps, signature, provenance=None, encoding='RAW'):
        if encoding not in ENCODINGS:
            raise ValueError('Unsupported cache encoding')
        validate_range(start, end, fps)
        estimate_bytes(grid.shape, channels, start, end)
        self.path = Path(parent) / ('fluxfx-bake-' + uuid4().hex[:12])
        self.path.mkdir(parents=True, exist_ok=False)
        self.encoding = encoding
        self.meta = dict(format=FORMAT if encoding == 'RAW' else COMPRESSED_FORMAT, shape=list(grid.shape),
                         extent=list(grid.extent), channels=list(channels), start=start, end=end, fps=fps,
                         signature=signature, provenance=provenance or {}, status='BAKING', frames={})
        if encoding != 'RAW':
            self.meta['encoding'] = encoding
        self.publish()

    @property
    def cells(self):
        return prod(self.meta['shape'])

    def publish(self):
        atomic_json(self.path / 'manifest.json', self.meta)

    def next_frame(self):
        return self.meta['start'] + len(self.meta['frames'])

    def write(self, frame, fields):
        """Frame ``frame`` (the next in order) from {channel: values}."""
        if self.meta['status'] != 'BAKING':
            raise ValueError('Cache writer is closed')
        if type(frame) is not int or frame != self.next_frame() or frame > self.meta['end']:
            raise ValueError('Cache frames must be written once, in order')
        if set(fields) != set(self.meta['channels']):
            raise ValueError('Cache channels differ')
        parts = []
        for channel in self.meta['channels']:
            values = np.asarray(fields[channel])
            if values.size != self.cells:
                raise ValueError('Wrong field size')
            if not valid_field(values, channel):
                raise ValueError('Invalid cache field values')
            parts.append(_le_bytes(values.reshape(-1)))
        raw = b''.join(parts)
        payload, codec = raw, 'RAW'
        if self.encoding == 'AUTO_ZLIB':
            packed = compress(raw, 1)
            if len(packed) < len(raw):
                payload, codec = packed, 'ZLIB'
        target = self.path / f'frame_{frame}.fxc'
        temp = target.with_suffix('.tmp')
        try:
            with temp.open('xb') as stream:
                stream.write(payload)
                stream.flush()
                os.fsync(stream.fileno())
            temp.replace(target)
        finally:
            if temp.exists():
                temp.unlink()
        record = dict(bytes=target.stat().st_size, crc32=f'{crc32(raw):08x}')
        if self.encoding != 'RAW':
            record.update(codec=codec, raw_bytes=len(raw))
        self.meta['frames'][str(frame)] = record
        self.publish()

    def finish(self, status='COMPLETE', message=''):
        if status not in STATUSES[1:]:
            raise ValueError('Invalid cache status')
        if status == 'COMPLETE' and len(self.meta['frames']) != self.meta['end'] - self.meta['start'] + 1:
            raise ValueError('Cannot complete a partial cache')
        self.meta.update(status=status, message=message)
        self.publish()


class CacheReader:
    """Validating reader of a bake directory (``physics/cache.py:142-182``)."""

    def __init__(self, path):
        self.path = Path(path)
        manifest = self.path / 'manifest.json'
        if manifest.stat().st_size > MAX_MANIFEST_BYTES:
            raise ValueError('Cache manifest too large')
        m = self.meta = json.loads(manifest.read_text())
        if m['format'] not in (FORMAT, COMPRESSED_FORMAT):
            raise ValueError('Unsupported playback cache format')
        if m['format'] == COMPRESSED_FORMAT and m.get('encoding') != 'AUTO_ZLIB':
            raise ValueError('Unsupported cache encoding')
        self.grid = GridSpec(tuple(m['shape']), tuple(m['extent']))
        validate_range(m['start'], m['end'], m['fps'])
        estimate_bytes(self.grid.shape, m['channels'], m['start'], m['end'])
        if m['status'] not in STATUSES:
            raise ValueError('Invalid cache status')
        if not isinstance(m['signature'], str) or len(m['signature']) != 64:
            raise ValueError('Invalid cache signature')
        if not isinstance(m['frames'], dict) or len(m['frames']) > m['end'] - m['start'] + 1:
            raise ValueError('Invalid cache frame table')
        expected = {str(f) for f in range(m['start'], m['start'] + len(m['frames']))}
        if set(m['frames']) != expected:
            raise ValueError('Invalid cache frame sequence')
        if m['status'] == 'COMPLETE' and len(expected) != m['end'] - m['start'] + 1:
            raise ValueError('Incomplete cache marked complete')
        provenance = m.get('provenance', {})
        if provenance.get('mode') == 'ANIMATED_INPUTS':
            inputs = provenance.get('inputs', {})
            if not isinstance(inputs, dict) or not expected.issubset(inputs) or any(
                    not isinstance(inputs[f], str) or len(inputs[f]) != 64 for f in expected):
                raise ValueError('Animated cache lacks per-frame input signatures')

    def read(self, frame):
        """{channel: float32 array} of a baked frame, validated."""
        m = self.meta
        if type(frame) is not int or str(frame) not in m['frames']:
            raise ValueError(f'Frame {frame} is not baked')
        count = prod(self.grid.shape)
        size = count * 4 * len(m['channels'])
        record = m['frames'][str(frame)]
        path = self.path / f'frame_{frame}.fxc'
        codec = record.get('codec') if m['format'] == COMPRESSED_FORMAT else 'RAW'
        if codec not in ('RAW', 'ZLIB'):
            raise ValueError('Unsupported frame encoding')
        stored = record['bytes']
        if type(stored) is not int or not 0 < stored <= size or path.stat().st_size != stored:
            raise ValueError('Cache frame size mismatch')
        if m['format'] == COMPRESSED_FORMAT and record.get('raw_bytes') != size:
            raise ValueError('Cache decoded size mismatch')
        if codec == 'RAW' and stored != size:
            raise ValueError('Cache frame size mismatch')
        with path.open('rb') as stream:
            raw = stream.read(stored + 1)       # bounded: a file that grew is caught below
        if len(raw) != stored:
            raise ValueError('Cache frame size mismatch')
        if codec == 'ZLIB':
            try:
                decoder = decompressobj()
                raw = decoder.decompress(raw, size + 1)
                if len(raw) != size or not decoder.eof or decoder.unused_data or decoder.unconsumed_tail:
                    raise ValueError('Invalid compressed cache frame')
            except ZlibError as exc:
                raise ValueError('Invalid compressed cache frame') from exc
        if f'{crc32(raw):08x}' != record['crc32']:
            raise ValueError('Cache frame checksum mismatch')
        data = np.frombuffer(raw, dtype='<f4').astype(np.float32)
        fields = {}
        for i, channel in enumerate(m['channels']):
            values = data[i * count:(i + 1) * count]
            if not valid_field(values, channel):
                raise ValueError('Invalid cached field')
            fields[channel] = values
        return fields
