"""Build recipe of libffx_core.so (nvcc, sm_100a).

``python -m fluxfx_b200.build`` compiles every ``csrc/*.cu`` into
``fluxfx_b200/_lib/libffx_core.so`` in place. The library is compiled without
FMA contraction (``--fmad=false``) so FP32 results match a strict IEEE
evaluation operation for operation.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / 'csrc'
OUT_DIR = HERE / '_lib'
LIB = OUT_DIR / 'libffx_core.so'
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '--fmad=false', '-std=c++17', '-Xcompiler', '-fPIC,-O2',
         '--expt-relaxed-constexpr', '-I', str(HERE.parent / 'include')]


def nvcc():
    cuda = os.environ.get('CUDA_HOME', '/usr/local/cuda')
    path = Path(cuda) / 'bin' / 'nvcc'
    return str(path) if path.exists() else 'nvcc'


def sources():
    return sorted(SRC.glob('*.cu'))


def _newer(target, deps):
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(d.stat().st_mtime <= t for d in deps)


def build(force=False, verbose=False, extra=()):
    """Compile objects in parallel, then link the shared library."""
    OUT_DIR.mkdir(exist_ok=True)
    headers = list(SRC.glob('*.cuh')) + [HERE.parent / 'include' / 'ffx.h']
    objs = []
    jobs = []
    for src in sources():
        obj = OUT_DIR / (src.stem + '.o')
        objs.append(obj)
        if force or not _newer(obj, [src, *headers, Path(__file__)]):
            jobs.append([nvcc(), *ARCH, *FLAGS, *extra, '-c', str(src), '-o', str(obj)])

    def run(cmd):
        if verbose:
            print(' '.join(cmd))
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        return res.stderr

    with ThreadPoolExecutor(max_workers=min(8, len(jobs) or 1)) as pool:
        logs = list(pool.map(run, jobs))
    if verbose:
        for log in logs:
            if log:
                print(log)
    if jobs or force or not LIB.exists():
        run([nvcc(), *ARCH, '-shared', '-cudart', 'static', *map(str, objs), '-o', str(LIB)])
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv,
          extra=('-Xptxas', '-v') if '--ptxas' in sys.argv else ())
    print(LIB)
