"""Build recipe: the reference's compute shaders as a CPU library (checker only).

    python oracle/glsl_ref/build.py [/path/to/FluxFX_Source/fluxfx/shaders]

The reference checkout is the directory FLUXFX_SOURCE names (its
``FluxFX_Source`` folder); without it, the recipe looks in the checkout
location of the development container (``REFERENCE_CHECKOUT``).

Reads the shader sources where they lie in the reference checkout, writes
build inputs and the library only under ``oracle/_ref/``:

* ``oracle/_ref/gen/*.glsl`` -- the shader files, unchanged except that GLSL
  ``out`` parameters become C++ references (``out float x`` -> ``float& x``;
  used by solid_mg_operator.glsl) and the ``.xyz`` swizzle becomes a call
  ``.xyz()`` (used by confinement.glsl) -- the two constructs C++ cannot parse;
* ``oracle/_ref/libglsl_ref.so`` -- ``oracle/glsl_ref/kernels.cpp`` compiled
  with g++ -fsingle-precision-constant -ffp-contract=off -fopenmp.

Nothing here is part of the product; the library travels with the checkout so
the CPU reference leg can run where the reference sources are absent.
"""
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / '_ref'
GEN = OUT / 'gen'
LIB = OUT / 'libglsl_ref.so'
REFERENCE_CHECKOUT = Path(os.environ.get('FLUXFX_SOURCE', '/root/reference/FluxFX_Source'))
DEFAULT_SHADERS = REFERENCE_CHECKOUT / 'fluxfx' / 'shaders'
OUT_PARAM = re.compile(r'\bout\s+(float|int|vec2|vec3|vec4|ivec3)\s+(\w+)')
SWIZZLE_XYZ = re.compile(r'(?<!gl_GlobalInvocationID)\.xyz\b(?!\s*\()')


def build(shaders=DEFAULT_SHADERS, force=False):
    shaders = Path(shaders)
    if not shaders.is_dir():
        if LIB.exists():
            return LIB
        raise FileNotFoundError(f"reference shader directory {shaders} not found")
    GEN.mkdir(parents=True, exist_ok=True)
    sources = sorted(shaders.glob('*.glsl'))
    newest = max(p.stat().st_mtime for p in [*sources, HERE / 'kernels.cpp', HERE / 'glsl.hpp', Path(__file__)])
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest:
        return LIB
    for src in sources:
        text = SWIZZLE_XYZ.sub('.xyz()', OUT_PARAM.sub(r'\1& \2', src.read_text()))
        (GEN / src.name).write_text(text)
    cmd = ['g++', '-O2', '-std=c++17', '-fPIC', '-shared', '-fopenmp', '-fsingle-precision-constant',
           '-ffp-contract=off', '-fno-fast-math', '-w', '-I', str(HERE), '-I', str(GEN),
           str(HERE / 'kernels.cpp'), '-o', str(LIB)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"g++ failed:\n{res.stderr[-4000:]}")
    return LIB


if __name__ == '__main__':
    print(build(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SHADERS, force=True))
