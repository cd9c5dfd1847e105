"""Per-field error of the CUDA path against an FP64 run of the oracle -- TEST
INFRASTRUCTURE (a checker run; nothing here is part of the product).

The scene is the 256^3 collider scene at 64^3 (bench.scene(64)): sphere and
box colliders, two emitters, MacCormack transport, projection to relative
max-norm divergence 1e-4. Every run starts from the same seeded fields and
takes the same fixed time step (dt = 0.008: a trace of at most half a cell for
velocities up to 1), so the runs differ only in arithmetic and solver:

    python oracle/precision_study.py gpu --steps 100 --out OUT.npz
        the CUDA path (needs a GPU): the reference algorithm in FP32 storage
        ('plain'), the headline solver in FP32 storage ('learned') and in BF16
        storage ('learned_bf16'); fields saved at steps 25, 50 and 100.
    python oracle/precision_study.py oracle --steps 100 --out REF.npz
        the oracle in FP64 with the reference algorithm solved to 1e-6 (the
        FP64 reference solution); same snapshots.
    python oracle/precision_study.py compare OUT.npz REF.npz
        relative max-norm and L2 errors per field, run and snapshot (JSON).
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

DT = 0.008
SNAPSHOTS = (25, 50, 100)
FIELDS = ('density', 'temperature', 'u', 'v', 'w')


def _snapshots(steps):
    return [s for s in SNAPSHOTS if s <= steps] or [steps]


def run_gpu(steps, out):
    import torch
    import bench
    from fluxfx_b200.backend.device import CudaDevice
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    device = CudaDevice()
    arrays = {}
    runs = {'plain': ('plain', 'FP32'), 'learned': ('learned', 'FP32'), 'learned_bf16': ('learned', 'BF16')}
    for name, (variant, storage) in runs.items():
        grid, s, colliders, emitters, noise = bench.scene(64, storage, 0, **bench.VARIANTS[variant])
        solver = DenseProjectedSmoke(grid, s, device, colliders=colliders)
        if s.learned_warm_start:
            from fluxfx_b200.learned import attach
            attach(solver, colliders)
        solver.upload(torch.zeros(grid.cells))
        solver.upload_temperature(torch.zeros(grid.cells))
        solver.upload_velocity([torch.as_tensor(v) for v in noise])
        for k in range(1, steps + 1):
            solver.step(DT, sources=emitters)
            if k in _snapshots(steps):
                torch.cuda.synchronize()
                fields = (solver.density, solver.temperature, *solver._velocity)
                for f, t in zip(FIELDS, fields):
                    arrays[f'{name}/{k}/{f}'] = t.float().cpu().numpy()
                m = solver.measure_projection()
                arrays[f'{name}/{k}/rel_div'] = np.array([m['rel_div_inf'], m.get('rel_div_inf_fp32', m['rel_div_inf'])])
        solver.close()
    np.savez_compressed(out, **arrays)
    print('wrote', out)


def run_oracle(steps, out):
    import bench
    from dataclasses import replace
    from fluxfx_b200.physics.emission import pack_sources
    from oracle import smoke as S
    from oracle.solver import OracleSmoke
    grid, s, colliders, emitters, noise = bench.scene(64, 'FP32', 0, **bench.VARIANTS['plain'])
    s = replace(s, pressure_tolerance=1e-6, pressure_max_cycles=256)
    g = S.Grid(grid.shape, grid.extent, np.float64)
    mask = S.raster_mask(g, [(c.shape, c.inverse_rows) for c in colliders])
    ref = OracleSmoke(grid.shape, grid.extent, s, np.float64, mask=mask)
    zeros = np.zeros(grid.cells)
    ref.upload(density=zeros, temperature=zeros, velocity=[np.asarray(v, np.float64) for v in noise])
    table = (pack_sources(emitters), len(emitters))
    arrays = {}
    for k in range(1, steps + 1):
        ref.step(DT, sources=table)
        if k in _snapshots(steps):
            for f, t in zip(FIELDS, (ref.density, ref.temperature, *ref.velocity)):
                arrays[f'fp64/{k}/{f}'] = t
            print('step', k, 'cycles', ref.projector.last_cycles, flush=True)
    np.savez_compressed(out, **arrays)
    print('wrote', out)


def compare(gpu_path, ref_path):
    gpu, ref = np.load(gpu_path), np.load(ref_path)
    report = {}
    for key in sorted(gpu.files):
        run, step, field = key.split('/')
        if field == 'rel_div':
            report.setdefault(run, {}).setdefault(step, {})['rel_div_inf'] = {
                'stored_faces': float(gpu[key][0]), 'before_rounding': float(gpu[key][1])}
            continue
        want = ref[f'fp64/{step}/{field}'].astype(np.float64)
        got = gpu[key].astype(np.float64)
        scale = float(np.abs(want).max())
        report.setdefault(run, {}).setdefault(step, {})[field] = {
            'rel_max': float(np.abs(got - want).max()) / scale if scale > 0 else 0.0,
            'rel_l2': float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300))}
    print(json.dumps(report, indent=1))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('mode', choices=('gpu', 'oracle', 'compare'))
    ap.add_argument('paths', nargs='*')
    ap.add_argument('--steps', type=int, default=100)
    ap.add_argument('--out', default='precision.npz')
    a = ap.parse_args()
    if a.mode == 'gpu':
        run_gpu(a.steps, a.out)
    elif a.mode == 'oracle':
        run_oracle(a.steps, a.out)
    else:
        compare(*a.paths)


if __name__ == '__main__':
    main()
