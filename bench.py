"""Benchmark: steps/s of the dense MAC smoke step at 256^3 with colliders.

Workload (the precision-form scene, plain FP32 unless --storage BF16):
256^3 cells, unit cube, closed free-slip walls; static colliders = a sphere of
radius 40 cells at the centre and a box over cells [40:80, 100:160, 20:60]
(uint8 mask, cell-centre inclusion); two seeded spherical emitters of radius
8 cells in the lower third that set density and temperature to values drawn
U(0.5, 1); buoyancy 1.0 T - 0.05 rho; MacCormack transport of U, V, W,
density and temperature; aggregation multigrid projection cycled until the
relative max-norm divergence is <= 1e-4; dt = min(0.02, 0.5 dx / max|u|).
Initial velocity: zero plus seeded uniform +-1e-3 noise on every face.

One "step" = one DenseProjectedSmoke.step plus the next-dt selection (one
readback of three floats). `value` is whole-job steps/s (N GPUs each run their
own replica domain: "weak" scaling, no collective on the step path). `e2e`
measures the same steps through the public API with each step's density field
read back into pinned host memory (the bake/preview readback) inside the
timed region. `--impl reference` times the CPU restatement of the reference
on a bounded sample of the same scene.

Inputs larger than L2 (every field of 256^3 is 64 MiB; the working set is
~1.5 GB), so no L2 flush is needed between steps.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "steps/s @256^3 to rel div 1e-4 (colliders, MacCormack, aggregation MG)"
UNIT = "steps/s"


def peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def scene(n, storage='FP32', seed=0):
    """Grid, settings, colliders, emitters and the seeded initial velocity."""
    import numpy as np
    from fluxfx_b200.physics.collision import primitive
    from fluxfx_b200.physics.config import GridSpec
    from fluxfx_b200.physics.emission import Emission, Source
    from fluxfx_b200.physics.pressure import PressureSettings
    grid = GridSpec((n, n, n), axis_limit=max(128, n))
    h = 1.0 / n
    c = n / 256.0   # scene geometry is specified in cells of the 256^3 grid
    sphere = primitive('SPHERE', (0.5, 0.5, 0.5), (40 * c * h,) * 3)
    box = primitive('BOX', (60 * c * h, 130 * c * h, 40 * c * h), (20 * c * h, 30 * c * h, 20 * c * h))
    rng = np.random.default_rng(seed)
    emitters = []
    for centre in ((0.3, 0.7), (0.7, 0.35)):
        cx, cy = centre
        cz = rng.uniform(0.12, 0.3)
        d, t = rng.uniform(0.5, 1.0, 2)
        pos = (cx + rng.uniform(-.05, .05), cy + rng.uniform(-.05, .05), cz)
        emitters.append(Source(pos, 8 * c * h, float(d), float(t), Emission(pos), 'TARGET', 'SOFT'))
    settings = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK',
                                thermal_lift=1.0, density_weight=0.05, dissipation=0.0, cooling=0.0,
                                heat_mode='TARGET', pressure_tolerance=1e-4, pressure_max_cycles=200,
                                storage=storage)
    noise = [rng.uniform(-1e-3, 1e-3, (fs[2], fs[1], fs[0])).astype(np.float32) for fs in grid.face_shapes]
    return grid, settings, (sphere, box), emitters, noise


def build_solver(n, storage, seed, device):
    import torch
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    grid, settings, colliders, emitters, noise = scene(n, storage, seed)
    solver = DenseProjectedSmoke(grid, settings, device, colliders=colliders)
    solver.upload(torch.zeros(grid.cells))
    solver.upload_temperature(torch.zeros(grid.cells))
    solver.upload_velocity([torch.as_tensor(v) for v in noise])
    return solver, emitters


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
              'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
              'clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(',')]
            if len(parts) == 7:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace('.', '', 1).isdigit()]
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[3 + k].lower() == 'active'})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(self.rows[0][1]) if self.rows[0][1].replace('.', '', 1).isdigit() else None,
                "reasons": reasons, "samples": len(self.rows)}


def run_b200(args):
    import torch
    import torch.distributed as dist
    from fluxfx_b200.backend.device import CudaDevice
    from fluxfx_b200.backend import solid_multigrid as SM

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group('nccl', timeout=__import__('datetime').timedelta(seconds=300))
    device = CudaDevice(local)
    n = args.size
    solver, emitters = build_solver(n, args.storage, args.seed + rank, device)
    stream = device.stream
    h = 1.0 / n

    def next_dt():
        umax = max(solver.projector.velocity_maxima())
        return min(0.02, 0.5 * h / umax) if umax > 0 else 0.02

    dt = 0.02
    for _ in range(args.warmup):
        solver.step(dt, sources=emitters)
        dt = next_dt()
    timer = SM.KernelTimer(stream)
    solver.projector.timer = timer
    cycles = []
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        solver.step(dt, sources=emitters)
        cycles.append(solver.projector.last_cycles)
        dt = next_dt()
    end.record(stream)
    torch.cuda.synchronize()
    elapsed = start.elapsed_time(end) / 1e3
    clock_info = clocks.stop()
    solver.projector.timer = None
    rel_div = solver.measure_projection()['rel_div_inf']
    # end to end: same steps through the public API, each step's density read back to pinned host memory
    host = torch.empty(solver.density.shape, dtype=solver.density.dtype, pin_memory=True)
    torch.cuda.synchronize()
    e2e_steps = max(1, args.steps // 2)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(e2e_steps):
        solver.step(dt, sources=emitters)
        with torch.cuda.stream(stream):
            host.copy_(solver.density, non_blocking=True)
        dt = next_dt()
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_time = t0.elapsed_time(t1) / 1e3
    times = torch.tensor([elapsed, e2e_time], dtype=torch.float64, device='cuda')
    if world > 1:
        dist.all_reduce(times, op=dist.ReduceOp.MAX)
    elapsed, e2e_time = float(times[0]), float(times[1])
    if rank == 0:
        hbm, peak_kind = peaks()
        cells = n ** 3
        avg_ms = timer.average_ms()
        bytes_per_launch = 13 * cells   # p in + rhs in + mask in + p out, 4+4+1+4 bytes per cell
        achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9 if avg_ms else None
        line = {
            "metric": METRIC, "value": world * args.steps / elapsed, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage == 'FP32' else "bf16-storage/f32-math",
            "data": "synthetic (seeded scene; no dataset)",
            "config": {"workload": f"dense smoke step {n}^3, sphere r=40 + box colliders, 2 emitters r=8, "
                                   f"MacCormack, aggregation MG to rel div<=1e-4, {args.storage} storage",
                       "cells": cells, "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}",
                       "v_cycles_mean": statistics.mean(cycles), "v_cycles_max": max(cycles),
                       "final_rel_div_inf": rel_div},
            "cell_updates_per_s": world * args.steps * cells / elapsed,
            "e2e": {"value": world * e2e_steps / e2e_time, "unit": UNIT, "h2d_bytes_per_step": 512,
                    "d2h_bytes_per_step": host.numel() * host.element_size()},
            "gpu_launches": None,
            "roofline": {"bound": "hbm", "kernel": "ffx graph_smooth_kernel (level-0 aggregation MG sweep)",
                         "achieved": achieved, "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None, "traffic": None,
                         "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg_ms,
                         "launches_timed": timer.count},
            "clocks": clock_info,
        }
        if args.cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(args, sample_n=None, sample_steps=1):
    """Time the NumPy restatement (one host thread) on a bounded sample of the
    scene and express it as steps/s of the full 256^3 grid via cell updates/s."""
    import numpy as np
    from oracle.smoke import Grid, raster_mask
    from oracle.solver import OracleSmoke
    from fluxfx_b200.physics.emission import pack_sources
    n = sample_n or args.cpu_sample
    grid, settings, colliders, emitters, noise = scene(n, 'FP32', args.seed)
    g = Grid(grid.shape, grid.extent, np.float32)
    mask = raster_mask(g, [(c.shape, c.inverse_rows) for c in colliders])
    ref = OracleSmoke(grid.shape, grid.extent, settings, np.float32, mask=mask)
    ref.upload(velocity=noise)
    table = (pack_sources(emitters), len(emitters))
    t0 = time.perf_counter()
    for _ in range(sample_steps):
        ref.step(0.02, sources=table)
    dt = time.perf_counter() - t0
    rate = sample_steps * n ** 3 / dt
    return {"value": rate / args.size ** 3, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{sample_steps} step(s) of the same scene at {n}^3 on the NumPy oracle "
                      f"({dt:.1f} s, {ref.projector.last_cycles} V-cycles); cell-update rate scaled to {args.size}^3"}


def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    samples = []
    for _ in range(args.warmup):
        cpu_baseline(args, args.cpu_sample, 1)
    for _ in range(args.steps):
        samples.append(cpu_baseline(args, args.cpu_sample, 1))
    value = statistics.mean(s['value'] for s in samples)
    base = samples[-1]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene)",
        "config": {"workload": f"dense smoke step {args.size}^3 scene, bounded CPU sample at {args.cpu_sample}^3"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": base['sample']},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='b200', choices=('b200', 'reference'))
    ap.add_argument('--size', type=int, default=256)
    ap.add_argument('--storage', default='FP32', choices=('FP32', 'BF16'))
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--cpu-sample', type=int, default=64)
    ap.add_argument('--no-cpu-baseline', dest='cpu_baseline', action='store_false')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
