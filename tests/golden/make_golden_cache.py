"""Writes the playback-cache fixtures with the reference's own CacheWriter.

    FLUXFX_SOURCE=/path/to/FluxFX_Source python tests/golden/make_golden_cache.py

Two bakes of a 2 x 3 x 4 grid, channels DENSITY and TEMPERATURE, frames 1-2,
fps 24, signature fingerprint({'golden': 1}): one RAW (fluxfx-playback-1) and
one AUTO_ZLIB (fluxfx-playback-2), each with a cancelled third bake frame
range. They pin this repository's cache reader and writer to the reference's
bytes (``fluxfx/physics/cache.py``). Outputs: tests/golden/cache_raw/ and
tests/golden/cache_zlib/ (manifest.json + frame_*.fxc, bake directory renamed).
"""
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def fields(frame):
    n = 24
    return {'DENSITY': [0.25 * frame + 0.01 * i for i in range(n)],
            'TEMPERATURE': [-2.0 + 0.5 * frame - 0.125 * i for i in range(n)]}


def main():
    from oracle.glsl_ref.build import REFERENCE_CHECKOUT
    sys.path.insert(0, str(REFERENCE_CHECKOUT))
    from fluxfx.physics.cache import CacheWriter, fingerprint
    from fluxfx.physics.config import GridSpec
    grid = GridSpec((2, 3, 4), (0.5, 0.75, 1.0))
    for name, encoding in (('cache_raw', 'RAW'), ('cache_zlib', 'AUTO_ZLIB')):
        out = HERE / name
        if out.exists():
            shutil.rmtree(out)
        tmp = HERE / (name + '_tmp')
        tmp.mkdir()
        w = CacheWriter(tmp, grid, ['DENSITY', 'TEMPERATURE'], 1, 3, 24, fingerprint({'golden': 1}),
                        provenance={'mode': 'STATIC'}, encoding=encoding)
        w.write(1, fields(1))
        w.write(2, fields(2))
        w.finish('CANCELLED', 'golden fixture')
        w.path.rename(out)
        tmp.rmdir()
        print('wrote', out)


if __name__ == '__main__':
    main()
