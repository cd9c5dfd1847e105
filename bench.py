"""Benchmark: steps/s of the dense MAC smoke step at 256^3 with colliders.

Workload (the precision-form scene of the 256^3 configuration):
256^3 cells, unit cube, closed free-slip walls; static colliders = a sphere of
radius 40 cells at the centre and a box over cells [40:80, 100:160, 20:60]
(uint8 mask, cell-centre inclusion); two seeded spherical emitters of radius
8 cells in the lower third that set density and temperature to values drawn
U(0.5, 1); buoyancy 1.0 T - 0.05 rho; MacCormack transport of U, V, W,
density and temperature; aggregation multigrid projection until the relative
max-norm divergence is <= 1e-4; dt = min(0.02, 0.5 dx / max|u|). Initial
velocity: zero plus seeded uniform +-1e-3 noise on every face.

One "step" = one DenseProjectedSmoke.step_cfl: the step plus the next-dt
selection on the device (the pressure solve's V-cycle loop also runs on the
device), so a step is queued without any host readback. Solver variants, all
to the same tolerance from the same seeded start after the same warm-up:

* plain   -- the reference algorithm: stand-alone aggregation V-cycles (4/4
             Jacobi sweeps), pressure cold-started every step, FP32 storage;
* learned -- the same V(4,4) cycles started every step from the U-Net's
             prediction (network on the 128^3 restriction, trilinear
             prolongation), with the coarse correction over-corrected by 1.9
             at every prolongation (default: the learned-warm-start step);
* fast    -- the same over-corrected cycles started from the previous step's
             pressure (scaled by dt / previous dt) instead of the network;
* learned_plain -- the plain cycles from the network's prediction (the
             V-cycles the network alone saves);
* pcg     -- conjugate gradients preconditioned by a V(1,1) cycle, warm start;
* learned_warm -- fast, with the network correcting the previous pressure
             (p += net(rhs - L p)).
--storage selects BF16 (default: the mixed-precision form -- BF16 storage of
velocity, density and temperature, FP32 arithmetic, pressure and multigrid,
FP64 coarse solve and convergence decisions) or FP32 storage; --set overrides
any solver setting of the headline variant.

The JSON `value` is the `--variant` run (default learned, BF16 storage); the
plain FP32 run, the fast FP32 run, the plain-cycles-from-the-network run and
the headline solver with FP32 storage are reported beside it. `value` is whole-job steps/s (N GPUs each run their own
replica domain: "weak" scaling, no collective on the step path). `e2e`
measures the same steps through the public API with each step's density field
read back into pinned host memory (the bake/preview readback) inside the
timed region. Inputs are larger than L2 (each 256^3 field is 64 MiB; the
working set is ~1.6 GB), so no L2 flush is needed between steps.
`--impl reference` times the CPU restatement of the reference on a bounded
sample of the same scene.
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

METRIC = ("steps/s @256^3 to rel div 1e-4: warm-started mixed-precision MG (fastest form; learned+mixed beside it) "
          "vs plain FP32 MG (colliders, MacCormack)")
UNIT = "steps/s"

VARIANTS = {
    'plain': dict(pressure_method='VCYCLE', solid_warm_start=False),
    'learned': dict(pressure_method='VCYCLE', solid_warm_start=False, learned_warm_start=True, mg_coarse_scale=1.9),
    'fast': dict(pressure_method='VCYCLE', solid_warm_start=True, mg_coarse_scale=1.9),
    'extrapolated': dict(pressure_method='VCYCLE', solid_warm_start=True, mg_coarse_scale=1.9,
                         warm_start_extrapolation=1.0, warm_start_order=2),
    'learned_plain': dict(pressure_method='VCYCLE', solid_warm_start=False, learned_warm_start=True),
    'pcg': dict(pressure_method='PCG', solid_warm_start=True, mg_pre_sweeps=1, mg_post_sweeps=1),
    'learned_ir': dict(pressure_method='IR', solid_warm_start=False, learned_warm_start=True, mg_coarse_scale=1.9),
    'fast_ir': dict(pressure_method='IR', solid_warm_start=True, mg_coarse_scale=1.9),
    'learned_warm': dict(pressure_method='VCYCLE', solid_warm_start=True, learned_warm_start=True,
                         learned_correction=True, mg_coarse_scale=1.9),
}

# Algorithmic bytes per cell of each pass: the compulsory traffic of the
# passes as the scope table states it (inputs read once, outputs written once,
# face grids as 3 values per cell, one mask byte; s = bytes per stored
# velocity/scalar value): A1 predictor 6s + m, A2 velocity correction 9s + 2s
# + m (velocity, predictor and output faces, density and temperature), S1
# scalar predictor (+ reverse, per pass) 3s + 4s + m, S2 scalar correction
# 3s + 6s + m. The departure points that this design stores in the predictor
# passes and reads in the correction passes (3 FP32 values per face and per
# cell) are extra traffic of the design, reported separately.
def pass_bytes(s):
    m = 1
    return {
        'velocity_predictor': 6 * s + m,
        'velocity_transport': 9 * s + 2 * s + m,
        'scalar_predictor_reverse': 2 * (3 * s + 4 * s + m),
        'scalar_transport': 3 * s + 6 * s + m,
    }


def trace_bytes(face_trace=True, storage='BF16'):
    """Per cell, the traces written by the predictors and read by the
    corrections (faces only where both passes form the same start points): per
    face the departure point and the start velocity, and in BF16 storage the
    unrounded sample, 4 bytes each, for three faces per cell."""
    ft = 3 * 4 * (7 if storage == 'BF16' else 6) if face_trace else 0
    return {'velocity_predictor': ft, 'velocity_transport': ft, 'scalar_predictor_reverse': 12,
            'scalar_transport': 12}


def peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def scene(n, storage='FP32', seed=0, **overrides):
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
    cfg = dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=1.0,
               density_weight=0.05, dissipation=0.0, cooling=0.0, heat_mode='TARGET', pressure_tolerance=1e-4,
               pressure_max_cycles=200, storage=storage)
    cfg.update(overrides)
    settings = PressureSettings(**cfg)
    noise = [rng.uniform(-1e-3, 1e-3, (fs[2], fs[1], fs[0])).astype(np.float32) for fs in grid.face_shapes]
    return grid, settings, (sphere, box), emitters, noise


def replica_seed(seed, rank):
    """Seed of rank ``rank``'s domain: with --gpus N every rank advances its own
    independent replica of the scene (no data crosses ranks on the step path)."""
    return seed + rank


def build_solver(n, storage, seed, device, **overrides):
    import torch
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    grid, settings, colliders, emitters, noise = scene(n, storage, seed, **overrides)
    solver = DenseProjectedSmoke(grid, settings, device, colliders=colliders)
    if settings.learned_warm_start:
        from fluxfx_b200.learned import attach
        attach(solver, colliders)
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
                                          '--format=csv,noheader,nounits', '-lms', '50'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # the timed region starts once sampling runs (nvidia-smi takes a moment to start)
        deadline = time.time() + 3.0
        while not self.rows and time.time() < deadline and self.proc.poll() is None:
            time.sleep(0.01)

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

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [v for v in (num(r[0]) for r in self.rows) if v is not None]
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[3 + k].lower() == 'active'})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(self.rows[0][1]),
                "reasons": reasons, "samples": len(self.rows)}


def max_over_ranks(values, world):
    """Element-wise max of per-rank timings (every rank must call it)."""
    import torch
    import torch.distributed as dist
    if world <= 1:
        return [float(v) for v in values]
    backend = dist.get_backend()
    device = 'cuda' if backend == 'nccl' else 'cpu'
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_rate(world, steps, elapsed):
    """Whole-job steps/s: every rank advances its own domain `steps` times."""
    return world * steps / elapsed


class Run:
    """One solver variant on the bench scene: warm-up, timed steps, e2e steps."""

    def __init__(self, args, device, rank, variant, storage):
        self.args = args
        self.device = device
        self.variant = variant
        self.storage = storage
        overrides = dict(VARIANTS[variant])
        if variant == args.variant:
            if args.coarse_scale is not None:
                overrides['mg_coarse_scale'] = args.coarse_scale
            overrides.update(parse_settings(args.set))
        self.solver, self.emitters = build_solver(args.size, storage, replica_seed(args.seed, rank), device,
                                                  **overrides)
        if args.host_loop:
            # the V-cycle loop on the host (one residual readback per cycle): the same
            # kernels, launched from replayed graphs -- for profilers that do not list
            # the kernels inside a conditional graph node
            self.solver.projector.use_device_loop = False
        self.h = 1.0 / args.size
        self.dt = 0.02

    def step(self):
        """One step with dt = min(0.02, 0.5 dx / max|u|) chosen on the device
        from the previous step's velocity (first step 0.02): no host readback."""
        self.solver.step_cfl(0.5, 0.02, sources=self.emitters)

    def warm(self, count):
        for _ in range(count):
            self.step()

    def timed(self, count, passes=False):
        """``count`` steps as the solver runs them (CUDA graphs on). With
        ``passes`` an event is recorded between the passes of each step (a few
        events per step, none inside the pressure solve)."""
        import torch
        from fluxfx_b200.backend.device import PassTimer
        stream = self.device.stream
        solver = self.solver
        self.pass_timer = PassTimer(stream) if passes else None
        solver.pass_timer = self.pass_timer
        graphs0 = len(getattr(solver.projector, '_graphs', ()))
        calls0 = self.device.calls
        cycles0 = solver.projector.total_cycles()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(count):
            self.step()
        end.record(stream)
        torch.cuda.synchronize()
        # the solves count their cycles on the device: read once, after the timed region
        self.cycles = (solver.projector.total_cycles() - cycles0) / count
        self.launches = self.device.calls - calls0
        self.captures = len(getattr(solver.projector, '_graphs', ())) - graphs0
        solver.pass_timer = None
        return start.elapsed_time(end) / 1e3

    def e2e(self, count):
        """``count`` steps through the public API, each step's density read back
        into pinned host memory. The read of step k runs on a copy stream while
        step k + 1 computes; step k + 2, which overwrites that field (the density
        ping-pongs between two buffers), waits for it. The timed region ends
        when the last read has landed."""
        import torch
        stream = self.device.stream
        solver = self.solver
        copier = torch.cuda.Stream(device=stream.device)
        hosts = [torch.empty(solver.density.shape, dtype=solver.density.dtype, pin_memory=True) for _ in range(2)]
        landed = [None, None]
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for k in range(count):
            if landed[k % 2] is not None:
                stream.wait_event(landed[k % 2])      # the read of step k - 2 (this step's output buffer)
            self.step()
            ready = torch.cuda.Event()
            ready.record(stream)
            copier.wait_event(ready)
            with torch.cuda.stream(copier):
                hosts[k % 2].copy_(solver.density, non_blocking=True)
            landed[k % 2] = torch.cuda.Event()
            landed[k % 2].record(copier)
        for ev in landed:
            if ev is not None:
                stream.wait_event(ev)
        t1.record(stream)
        torch.cuda.synchronize()
        host = hosts[0]
        return t0.elapsed_time(t1) / 1e3, host.numel() * host.element_size()

    def close(self):
        self.solver.close()


def run_b200(args):
    import ctypes as C
    import torch
    import torch.distributed as dist
    from fluxfx_b200 import _native as N
    from fluxfx_b200.backend.device import CudaDevice

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group('nccl', timeout=__import__('datetime').timedelta(seconds=300))
    device = CudaDevice(local)
    n = args.size
    cells = n ** 3

    # --- headline variant -------------------------------------------------
    run = Run(args, device, rank, args.variant, args.storage)
    run.warm(args.warmup)
    if world > 1:
        torch.cuda.synchronize()
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    elapsed = run.timed(args.steps, passes=True)
    clock_info = clocks.stop()
    passes = run.pass_timer.totals_ms()
    head = dict(cycles=run.cycles, launches=run.launches, captures=run.captures)
    head_metrics = run.solver.measure_projection()
    rel_div = head_metrics['rel_div_inf']
    rel_div32 = head_metrics.get('rel_div_inf_fp32', rel_div)
    run.close()
    # end to end over the same steps: a fresh solver on the same scene, the same
    # warm-up, then the timed window again through the public call with every
    # step's density read back (the scene's later steps need more V-cycles, so
    # a window after the timed one would measure different work)
    e2e_steps = args.steps
    erun = Run(args, device, rank, args.variant, args.storage)
    erun.warm(args.warmup)
    e2e_time, d2h = erun.e2e(e2e_steps)
    erun.close()
    h2d = 2 * C.sizeof(N.FfxSources)   # the emitter table, passed with the two launches that emit

    # --- plain FP32 reference algorithm, same scene and warm-up ----------------
    plain = None
    if args.compare_plain and args.variant != 'plain':
        prun = Run(args, device, rank, 'plain', 'FP32')
        prun.warm(args.warmup)
        p_steps = max(2, args.steps // 2)
        p_elapsed = prun.timed(p_steps)
        plain = dict(elapsed=p_elapsed, steps=p_steps, cycles=prun.cycles,
                     rel_div=prun.solver.measure_projection()['rel_div_inf'])
        prun.close()

    # --- comparison variants: the previous pressure instead of the network, and
    # the plain cycles from the network's guess -----------------------------------
    def compare(variant, enabled, storage):
        if not enabled or (args.variant == variant and args.storage == storage):
            return None
        crun = Run(args, device, rank, variant, storage)
        crun.warm(args.warmup)
        c_steps = max(2, args.steps // 2)
        c_elapsed = crun.timed(c_steps)
        m = crun.solver.measure_projection()
        out = dict(elapsed=c_elapsed, steps=c_steps, cycles=crun.cycles, rel_div=m['rel_div_inf'],
                   rel_div32=m.get('rel_div_inf_fp32', m['rel_div_inf']), storage=storage)
        crun.close()
        return out

    # the other warm start at the headline's storage: the network every step
    # (beside the previous-pressure headline), or the previous pressure
    alt_variant = 'learned' if args.variant != 'learned' else 'fast'
    fast = compare(alt_variant, args.compare_fast, args.storage)
    # the extrapolated start against the previous pressure alone
    previous = compare('fast', args.compare_fast and args.variant == 'extrapolated', args.storage)
    learned = compare('learned_plain', args.compare_learned, args.storage)
    learned32 = compare(args.variant, args.compare_storage, 'FP32')

    elapsed, e2e_time, p_el, f_el, l_el, s_el, v_el = max_over_ranks(
        [elapsed, e2e_time, plain['elapsed'] if plain else 0.0, fast['elapsed'] if fast else 0.0,
         learned['elapsed'] if learned else 0.0, learned32['elapsed'] if learned32 else 0.0,
         previous['elapsed'] if previous else 0.0], world)
    if rank == 0:
        hbm, peak_kind = peaks()
        s = 4 if args.storage == 'FP32' else 2
        ft = N.grid_pow2((n, n, n), (1.0, 1.0, 1.0))
        pb, tb = pass_bytes(s), trace_bytes(ft, args.storage)
        pass_report = {}
        for name, ms in passes.items():
            per_step = ms / args.steps
            entry = {"ms_per_step": per_step}
            if name in pb:
                entry["algorithmic_bytes_per_cell"] = pb[name]
                entry["design_trace_bytes_per_cell"] = tb[name]
                entry["achieved_GBps"] = pb[name] * cells / (per_step / 1e3) / 1e9
                entry["frac_of_peak"] = entry["achieved_GBps"] / hbm
            pass_report[name] = entry
        line = {
            "metric": METRIC, "value": job_rate(world, args.steps, elapsed), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage == 'FP32' else "bf16-storage/f32-math",
            "data": "synthetic (seeded scene; no dataset)",
            "config": {"workload": f"dense smoke step {n}^3, sphere r=40 + box colliders, 2 emitters r=8, MacCormack, "
                                   f"projection to rel div<=1e-4; variant={args.variant} "
                                   f"({VARIANTS[args.variant]}"
                                   f"{'' if args.coarse_scale is None else f', mg_coarse_scale={args.coarse_scale}'}"
                                   f"{''.join(', ' + x for x in args.set)}), "
                                   f"{args.storage} storage",
                       "cells": cells, "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}",
                       "v_cycles_mean": head['cycles'],
                       "host_syncs_per_step": "one per V-cycle (--host-loop)" if args.host_loop else 0,
                       "graph_captures_in_timed_steps": head['captures'],
                       "final_rel_div_inf": rel_div,
                       "final_rel_div_inf_fp32": rel_div32,
                       "rel_div_note": "final_rel_div_inf is measured on the stored faces; with BF16 storage they "
                                       "cannot hold a velocity to 1e-4 (a BF16 value has ~3 digits), so the "
                                       "tolerance measure is final_rel_div_inf_fp32: the divergence of the "
                                       "projection's FP32 result in the gradient pass, before rounding to storage",
                       "plain_fp32_mg": None if plain is None else {
                           "steps_per_s": job_rate(world, plain['steps'], p_el), "steps": plain['steps'],
                           "v_cycles_mean": plain['cycles'],
                           "final_rel_div_inf": plain['rel_div']},
                       "speedup_vs_plain": None if plain is None else
                       job_rate(world, args.steps, elapsed) / job_rate(world, plain['steps'], p_el),
                       ("learned_every_step" if alt_variant == 'learned' else "fast_previous_pressure_mg"):
                           None if fast is None else {
                           "steps_per_s": job_rate(world, fast['steps'], f_el), "steps": fast['steps'],
                           "v_cycles_mean": fast['cycles'],
                           "final_rel_div_inf": fast['rel_div'], "final_rel_div_inf_fp32": fast['rel_div32'],
                           "storage": fast['storage'],
                           "speedup_vs_plain": None if plain is None else
                           job_rate(world, fast['steps'], f_el) / job_rate(world, plain['steps'], p_el),
                           "method": ("the U-Net's guess (net on the 128^3 restriction of the divergence and mask, "
                                      "trilinear prolongation) as the start of every solve, then over-corrected "
                                      "V(4,4) cycles" if alt_variant == 'learned' else
                                      "over-corrected V(4,4) cycles from the previous step's pressure (no network)")},
                       "previous_pressure_start": None if previous is None else {
                           "steps_per_s": job_rate(world, previous['steps'], v_el), "steps": previous['steps'],
                           "v_cycles_mean": previous['cycles'], "final_rel_div_inf": previous['rel_div'],
                           "final_rel_div_inf_fp32": previous['rel_div32'], "storage": previous['storage'],
                           "speedup_vs_plain": None if plain is None else
                           job_rate(world, previous['steps'], v_el) / job_rate(world, plain['steps'], p_el),
                           "method": "variant fast: the previous step's pressure times dt / previous dt alone "
                                     "starts every solve (no extrapolation)"},
                       "headline_note": ({
                           'fast': "variant fast: the previous step's pressure (times dt / previous dt) starts "
                                   "every solve, over-corrected V(4,4) cycles (alpha 1.9); measured beside it, "
                                   "the U-Net guess every step (learned_every_step) saves a fraction of a "
                                   "V-cycle against the previous pressure and costs more than it saves, so "
                                   "the faster form is the headline",
                           'extrapolated': "variant extrapolated: the last three solves' pressures, extrapolated "
                                           "in time by their quadratic, start every solve; over-corrected V(4,4) cycles "
                                           "(alpha 1.9); measured beside it, the previous pressure alone "
                                           "(previous_pressure_start) and the U-Net guess every step "
                                           "(learned_every_step), which saves a fraction of a V-cycle against the "
                                           "previous pressure and costs more than it saves"}.get(args.variant)),
                       "same_solver_fp32_storage": None if learned32 is None else {
                           "steps_per_s": job_rate(world, learned32['steps'], s_el), "steps": learned32['steps'],
                           "v_cycles_mean": learned32['cycles'], "final_rel_div_inf": learned32['rel_div'],
                           "storage": "FP32", "method": f"variant {args.variant} with FP32 storage"},
                       "plain_cycles_from_network": None if learned is None else {
                           "steps_per_s": job_rate(world, learned['steps'], l_el), "steps": learned['steps'],
                           "v_cycles_mean": learned['cycles'],
                           "final_rel_div_inf": learned['rel_div'], "storage": learned['storage'],
                           "final_rel_div_inf_fp32": learned['rel_div32'],
                           "method": "the reference's V(4,4) cycles from the U-Net's guess (net on the 128^3 "
                                     "restriction, trilinear prolongation)"}},
            "cell_updates_per_s": world * args.steps * cells / elapsed,
            "passes": pass_report,
            "e2e": {"value": job_rate(world, e2e_steps, e2e_time), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "path": "DenseProjectedSmoke.step with the emitter list each step (packed into the launch "
                            "parameters of the two emitting passes) + every step's density field read back into "
                            "pinned host memory on a copy stream, overlapped with the next step (the step after "
                            "that, which overwrites the field, waits for the read); a fresh solver on the same "
                            "scene and warm-up, so the same steps as the timed window"},
            "gpu_launches": head['launches'],
            "roofline": roofline(passes, args.steps, cells, s, hbm, peak_kind, ft, clock_info.get('sm_mhz')),
            "clocks": clock_info,
        }
        if args.cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# dram__bytes_read.sum + dram__bytes_write.sum of one advect_velocity_kernel
# launch (reading the stored departure points, start velocities and, in BF16
# storage, the predictor's unrounded samples), from an ncu capture of this
# bench's scene (BF16 storage; the kernel is the same for every solver variant).
MEASURED_TRAFFIC = {(256, 2): 1929255936 + 97080320}
# smsp__inst_executed.sum (warp instructions) of the same launch, same capture
MEASURED_WARP_INSTRUCTIONS = {(256, 2): 1.486e9}
B200_SMS, SCHEDULERS_PER_SM = 148, 4     # one warp instruction per scheduler per cycle


def issue_roofline(ms, cells, s, sm_mhz):
    """The instruction-issue roofline of the same kernel: its warp
    instructions per launch (ncu) over the GPU's issue rate at the clock seen
    in the timed region give the shortest launch that instruction count
    allows; frac = that floor / the measured launch time."""
    inst = MEASURED_WARP_INSTRUCTIONS.get((round(cells ** (1 / 3)), s))
    if not inst or not ms or not sm_mhz:
        return None
    rate = B200_SMS * SCHEDULERS_PER_SM * sm_mhz * 1e6      # warp instructions per second
    floor_ms = inst / rate * 1e3
    return {"bound": "issue", "warp_instructions_per_launch": inst,
            "peak_warp_instructions_per_s": rate, "floor_ms": floor_ms, "achieved_ms": ms, "frac": floor_ms / ms,
            "source": "ncu smsp__inst_executed.sum of one launch (profiles/transport_256_bf16.txt); clock from "
                      "this run's samples"}


def roofline(passes, steps, cells, s, hbm, peak_kind, face_trace=True, sm_mhz=None):
    """The dominant kernel of the step, advect_velocity_kernel (one launch per
    step; its time comes from the events bracketing that launch in the timed
    steps): algorithmic bytes per launch (the scope table's 9s + 2s + m per
    cell) / launch time against the measured copy bandwidth. The kernel is
    bound by instruction issue, not by HBM (about 940 instructions per face in
    the reference's FP32 evaluation order: three trilinear velocity samples for
    the forward trace, the predictor sample, the 8-corner clamp, the collider
    tests, emitters, buoyancy and walls), hence the low fraction."""
    ms = passes.get('velocity_transport', 0.0) / steps
    per_cell = pass_bytes(s)['velocity_transport']
    achieved = per_cell * cells / (ms / 1e3) / 1e9 if ms else None
    return {"bound": "hbm", "kernel": "advect_velocity_kernel (MacCormack velocity transport + emission + "
                                      "buoyancy + walls, one launch per step)",
            "achieved": achieved, "peak": hbm, "peak_kind": f"{peak_kind} (MEASURED_PEAKS hbm_gbs)", "unit": "GB/s",
            "frac": (achieved / hbm) if achieved else None,
            "traffic": MEASURED_TRAFFIC.get((round(cells ** (1 / 3)), s)),
            "traffic_source": "ncu dram read+write of one launch (same scene and storage), not measured in this run",
            "algorithmic_bytes_per_launch": per_cell * cells,
            "design_trace_bytes_per_launch": trace_bytes(face_trace, 'FP32' if s == 4 else 'BF16')['velocity_transport'] * cells,
            "avg_launch_ms": ms, "limiter": "instruction issue",
            "issue": issue_roofline(ms, cells, s, sm_mhz),
            "timing": "CUDA events bracketing the launch in every timed step"}


def cpu_baseline(args, sample_n=None, sample_steps=1):
    """Time the NumPy restatement (one host thread) on a bounded sample of the
    scene, the plain reference algorithm, and express it as steps/s of the
    full grid through the cell-update rate."""
    import numpy as np
    from oracle.smoke import Grid, raster_mask
    from oracle.solver import OracleSmoke
    from fluxfx_b200.physics.emission import pack_sources
    n = sample_n or args.cpu_sample
    grid, settings, colliders, emitters, noise = scene(n, 'FP32', args.seed, **VARIANTS['plain'])
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
    return {"value": rate / args.size ** 3, "unit": UNIT, "cores": 1, "host_cpu_count": os.cpu_count(),
            "threads_note": "NumPy element-wise passes run on one thread", "kind": "port",
            "sample": f"{sample_steps} step(s) of the same scene at {n}^3 on the NumPy restatement of the "
                      f"reference ({dt:.1f} s, {ref.projector.last_cycles} V-cycles); cell-update rate scaled "
                      f"to {args.size}^3"}


def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    for _ in range(args.warmup):
        cpu_baseline(args, args.cpu_sample, 1)
    samples = [cpu_baseline(args, args.cpu_sample, 1) for _ in range(args.steps)]
    value = statistics.mean(s['value'] for s in samples)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene)",
        "config": {"workload": f"dense smoke step {args.size}^3 scene, reference algorithm, "
                               f"bounded CPU sample at {args.cpu_sample}^3"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "host_cpu_count": os.cpu_count(), "kind": "port",
                         "sample": samples[-1]['sample']},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def run_batched(args):
    """48 uneven FP32 domains (axes from {32, 48, 64, 96, 128}, 1-3 emitters,
    0-2 sphere colliders), one persistent launch per pass, 32 steps per CUDA
    graph, autotuned passes; beside it the same domains stepped one solver at
    a time (each with its own V-cycle graphs and host time step)."""
    import torch
    from fluxfx_b200.backend.batched import BatchedSmoke, batched_scenes, build_solvers, cell_updates
    from fluxfx_b200.backend.device import CudaDevice
    device = CudaDevice()
    graph_steps = 32
    opts = parse_settings(args.set)
    warm = bool(opts.get('solid_warm_start', True))
    alpha = float(opts.get('mg_coarse_scale', 1.9))
    scenes = batched_scenes(48, seed=args.seed, warm_start=warm, coarse_scale=alpha)
    solvers, sources = build_solvers(scenes, device)
    cells = cell_updates(solvers)
    batch = BatchedSmoke(solvers, sources)
    tuned = batch.tune(repeats=3)
    stream = device.stream
    # warm-up: one graph of 32 steps (captures and instantiates it)
    batch.run(graph_steps)
    launches = max(1, args.steps // graph_steps)
    s0 = batch.stats()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(launches):
        batch.run(graph_steps)
    end.record(stream)
    torch.cuda.synchronize()
    clock_info = sampler.stop()
    seconds = start.elapsed_time(end) / 1e3
    s1 = batch.stats()
    steps = launches * graph_steps
    cycles = (sum(b['total_cycles'] for b in s1) - sum(a['total_cycles'] for a in s0)) / (steps * len(s1))
    iterations = s1[0]['loop_iterations'] - s0[0]['loop_iterations']
    per_step = batch.launches_per_step(0)
    loop_launches = batch.launches_per_step(1) - per_step
    gpu_launches = steps * per_step + iterations * loop_launches
    # the dominant pass alone: level-0 smoothing over every domain
    hbm, peak_kind = peaks()
    from fluxfx_b200 import _native as N
    reps = 20
    # the level-0 sweep over every domain: the four-cell kernel when the plan uses it
    # (its tuning launch is then the level-0 sweep), else the one-cell kernel
    four_cell = tuned.get('l0_smooth', (0, 0, 0.0))[2] > 1e-3
    sweep_kind = N.PASS_L0_SMOOTH if four_cell else N.PASS_SMOOTH
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(reps):
        N.check(batch.lib.ffx_batch_tune_pass(batch.plan, sweep_kind, batch.stream))
    t1.record(stream)
    t1.synchronize()
    smooth_ms = t0.elapsed_time(t1) / reps
    # p, rhs (FP32) in, q (FP32) out, one link (or mask) byte per cell
    smooth_gbs = 13.0 * cells / (smooth_ms * 1e-3) / 1e9
    # the same domains one solver at a time (sequential baseline)
    ref_solvers, ref_sources = build_solvers(scenes, device)
    seq_steps = 2
    h = 1.0 / 64.0
    dts = [0.02] * len(ref_solvers)

    def seq_step():
        for i, (sv, src) in enumerate(zip(ref_solvers, ref_sources)):
            sv.step(dts[i], sources=src)
            umax = max(sv.projector.velocity_maxima())
            dts[i] = min(0.02, 0.5 * h / umax) if umax > 0 else 0.02
    seq_step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(seq_steps):
        seq_step()
    b.record(stream)
    torch.cuda.synchronize()
    seq_seconds = a.elapsed_time(b) / 1e3
    for sv in ref_solvers:
        sv.close()
    rate = steps / seconds
    line = {
        "metric": "batched steps/s, 48 uneven domains (all domains advance one step)", "value": rate,
        "unit": "steps/s", "n_gpus": 1, "steps": steps, "warmup": graph_steps, "ms_per_step": 1e3 * seconds / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "48 uneven FP32 smoke domains, axes from {32,48,64,96,128}, 1-3 emitters, "
                               "0-2 sphere colliders, multigrid to rel div 1e-4, 32 steps per CUDA graph",
                   "solver": f"aggregation V(4,4) cycles, warm start {warm}, coarse-correction factor {alpha}",
                   "cells": cells, "domains": len(solvers), "l2": "working set > L2 (no flush)"},
        "cell_updates_per_s": cells * rate, "v_cycles_per_domain_step": cycles,
        "solve_loop_iterations_per_step": iterations / steps,
        "sequential": {"value": seq_steps / seq_seconds, "unit": "steps/s", "steps": seq_steps,
                       "speedup": rate / (seq_steps / seq_seconds)},
        "roofline": {"bound": "hbm", "kernel": ("batch_l0_smooth_kernel (level-0 sweep, four cells per thread, "
                                                "all domains)") if four_cell else
                     "batch_smooth_kernel (level-0 sweep, all domains)", "avg_launch_ms": smooth_ms,
                     "achieved": smooth_gbs, "peak": hbm, "unit": "GB/s", "frac": smooth_gbs / hbm,
                     "traffic": None, "peak_source": peak_kind, "bytes_per_cell": 13},
        "autotune": {k: {"shape": list(SHAPES_NAMES[v[0]]), "grid": v[1], "ms": v[2]} for k, v in tuned.items()},
        "gpu_launches": int(gpu_launches), "clocks": clock_info,
    }
    print(json.dumps(line), flush=True)
    batch.close()
    for sv in solvers:
        sv.close()


SHAPES_NAMES = ((32, 8), (64, 4), (128, 2), (16, 16))


def fire_scene(storage, seed, fast, **overrides):
    """The fire configuration: 192 x 192 x 320 cells (cells of 1/192, z up), a
    fuel emitter of radius 10 cells (fuel 1.0, temperature 0.4), combustion
    (burn rate 0.75, ignition 0.3, heat yield 1.0, smoke yield 0.5), vorticity
    confinement 0.3, a sphere collider of radius 20 cells moving +x by half a
    cell per step; multigrid to relative divergence 1e-4. ``fast``: BF16 or FP32
    storage as given, warm start, over-correction 1.9, the learned guess for
    cold starts; otherwise the plain FP32 multigrid (V(4,4) from zero)."""
    import numpy as np
    from fluxfx_b200.physics.collision import primitive
    from fluxfx_b200.physics.config import GridSpec
    from fluxfx_b200.physics.pressure import PressureSettings
    shape = (192, 192, 320)
    h = 1.0 / 192
    grid = GridSpec(shape, extent=(1.0, 1.0, 320 * h), axis_limit=320)
    rng = np.random.default_rng(seed)
    x0 = 0.25 + rng.uniform(-0.02, 0.02)
    pose = lambda k: (primitive('SPHERE', (x0 + 0.5 * h * k, 0.5, 0.9), (20 * h,) * 3),)
    cfg = dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', combustion_enabled=True,
               fuel_source_rate=1.0, heat_source_rate=0.4, heat_mode='TARGET', source_rate=0.0,
               source_radius=10 * h, source_center=(0.5 + rng.uniform(-0.02, 0.02), 0.5, 0.25),
               ignition_temperature=0.3, burn_rate=0.75, heat_yield=1.0, smoke_yield=0.5, vorticity_strength=0.3,
               thermal_lift=1.0, density_weight=0.05, moving_colliders=True, pressure_tolerance=1e-4,
               pressure_max_cycles=200, storage=storage if fast else 'FP32')
    if fast:
        cfg.update(solid_warm_start=True, mg_coarse_scale=1.9, learned_warm_start=True)
        cfg.update(overrides)
    noise = [rng.uniform(-1e-3, 1e-3, (fs[2], fs[1], fs[0])).astype(np.float32) for fs in grid.face_shapes]
    return grid, PressureSettings(**cfg), pose, noise


def run_fire(args):
    """Four fire domains on one GPU, each on its own CUDA stream so their
    passes overlap (the batched plan covers the static-collider step only),
    fast form against the plain FP32 multigrid form on the same dt sequence;
    error of the fast fields against the plain ones."""
    import torch
    from fluxfx_b200.backend.device import CudaDevice
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.backend.solid_multigrid import SolidMultigridProjector
    from fluxfx_b200.learned import attach
    domains, steps = 4, args.steps
    devices = [CudaDevice(stream=torch.cuda.Stream()) for _ in range(domains)]
    main = torch.cuda.current_stream()
    h = 1.0 / 192

    def build(fast):
        out = []
        for d in range(domains):
            grid, settings, pose, noise = fire_scene(args.storage, args.seed + d, fast,
                                                     **(parse_settings(args.set) if fast else {}))
            s = DenseProjectedSmoke(grid, settings, devices[d], projector_class=SolidMultigridProjector,
                                    colliders=pose(0))
            if fast:
                attach(s, pose(0))
                s.projector.defer_refresh_check = True
            s.upload(torch.zeros(grid.cells))
            s.upload_temperature(torch.zeros(grid.cells))
            s.upload_velocity([torch.as_tensor(v) for v in noise])
            out.append((s, pose))
        return out

    def run(solvers, dts=None):
        record = []
        totals = [s.projector.total_cycles() for s, _ in solvers]
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(main)
        for dev in devices:
            dev.stream.wait_event(a)
        for k in range(steps):
            row = []
            for d, (s, pose) in enumerate(solvers):
                dt = dts[k][d] if dts else (record[-1][d] if record else 0.02)
                s.move_colliders(pose(k + 1), dt)
                s.step(dt)
                if dts is None:
                    # the plain run chooses the time steps (one readback); the fast
                    # runs replay them and read nothing back
                    umax = max(s.projector.velocity_maxima())
                    row.append(min(0.02, 0.5 * h / umax) if umax > 0 else 0.02)
            record.append(row)
        for dev in devices:
            main.wait_stream(dev.stream)
        b.record(main)
        torch.cuda.synchronize()
        cycles = sum(s.projector.total_cycles() - t for (s, _), t in zip(solvers, totals))
        used = [[0.02] * domains] + record[:-1] if dts is None else dts
        return a.elapsed_time(b) / 1e3, cycles / (steps * domains), used

    plain = build(False)
    p_time, p_cycles, dts = run(plain)
    fields = [(s.density.float().clone(), s.temperature.float().clone(), s.combustion.fuel.float().clone(),
               [v.float().clone() for v in s._velocity]) for s, _ in plain]
    rel = [s.measure_projection()['rel_div_inf'] for s, _ in plain]
    for s, _ in plain:
        s.close()

    def errors(solvers):
        """Max-norm and L2 relative differences of every field from the plain run."""
        err = {}
        for (s, _), (rho, t, fuel, vel) in zip(solvers, fields):
            pairs = (('density', s.density, rho), ('temperature', s.temperature, t),
                     ('fuel', s.combustion.fuel, fuel), *[(f'velocity_{a}', s._velocity[a], vel[a]) for a in range(3)])
            for name, got, want in pairs:
                diff = got.float() - want
                e_max = float(diff.abs().max()) / max(float(want.abs().max()), 1e-30)
                e_l2 = float(diff.norm()) / max(float(want.norm()), 1e-30)
                prev = err.get(name, (0.0, 0.0))
                err[name] = (max(prev[0], e_max), max(prev[1], e_l2))
        return {k: {"max": v[0], "l2": v[1]} for k, v in err.items()}

    # the same fast solver with FP32 storage: the solver's own share of the difference
    storage = args.storage
    args.storage = 'FP32'
    fast32 = build(True)
    f32_time, f32_cycles, _ = run(fast32, dts)
    err32 = errors(fast32)
    for s, _ in fast32:
        s.close()
    args.storage = storage
    fast = build(True)
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    f_time, f_cycles, _ = run(fast, dts)
    clock_info = clocks.stop()
    err = errors(fast)
    f_metrics = [s.measure_projection() for s, _ in fast]
    f_rel = [m['rel_div_inf'] for m in f_metrics]
    f_rel32 = [m.get('rel_div_inf_fp32', m['rel_div_inf']) for m in f_metrics]
    for s, _ in fast:
        s.close()
    cells = 192 * 192 * 320 * domains
    line = {
        "metric": "fire steps/s, 4 domains of 192x192x320 (all domains advance one step)",
        "value": steps / f_time, "unit": "steps/s", "n_gpus": 1, "steps": steps, "warmup": 0,
        "ms_per_step": 1e3 * f_time / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16-storage/f32-math" if args.storage == 'BF16' else "f32", "data": "synthetic",
        "config": {"workload": "fire: fuel emitter r=10, combustion, confinement 0.3, moving sphere r=20 "
                               "(+0.5 cells/step), multigrid to rel div 1e-4 after every move, 4 domains in turn",
                   "fast": f"{args.storage} storage, warm start, over-correction 1.9, learned guess on cold starts",
                   "cells": cells},
        "cell_updates_per_s": cells * steps / f_time, "v_cycles_per_domain_step": f_cycles,
        "plain_fp32_mg": {"steps_per_s": steps / p_time, "v_cycles_per_domain_step": p_cycles,
                          "final_rel_div_inf_max": max(rel)},
        "fast_fp32_storage": {"steps_per_s": steps / f32_time, "v_cycles_per_domain_step": f32_cycles,
                              "rel_error_vs_plain_fp32": err32},
        "speedup_vs_plain": p_time / f_time,
        "final_rel_div_inf_max": max(f_rel),
        "final_rel_div_inf_fp32_max": max(f_rel32),
        "final_rel_div_note": "final_rel_div_inf_max is measured on the stored faces (BF16 storage rounds the "
                              "projected velocity); final_rel_div_inf_fp32_max on the projection's FP32 result "
                              "before rounding, the solve's own tolerance measure",
        "rel_error_vs_plain_fp32": err, "clocks": clock_info,
    }
    print(json.dumps(line), flush=True)


def parse_settings(items):
    """--set name=value pairs as PressureSettings overrides (ints, floats, booleans, strings)."""
    out = {}
    for item in items or ():
        name, _, text = item.partition('=')
        if text in ('True', 'False'):
            value = text == 'True'
        else:
            try:
                value = int(text)
            except ValueError:
                try:
                    value = float(text)
                except ValueError:
                    value = text
        out[name.strip()] = value
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='b200', choices=('b200', 'reference'))
    ap.add_argument('--size', type=int, default=256)
    ap.add_argument('--storage', default='BF16', choices=('FP32', 'BF16'),
                    help='field storage of the headline variant (default BF16: the mixed-precision form)')
    ap.add_argument('--host-loop', action='store_true',
                    help='run the V-cycle loop on the host (for kernel-listing profilers)')
    ap.add_argument('--no-compare-storage', dest='compare_storage', action='store_false',
                    help='skip the headline variant with FP32 storage')
    ap.add_argument('--variant', default='extrapolated', choices=tuple(VARIANTS))
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--cpu-sample', type=int, default=64)
    ap.add_argument('--no-cpu-baseline', dest='cpu_baseline', action='store_false')
    ap.add_argument('--no-compare-plain', dest='compare_plain', action='store_false')
    ap.add_argument('--no-compare-learned', dest='compare_learned', action='store_false')
    ap.add_argument('--no-compare-fast', dest='compare_fast', action='store_false')
    ap.add_argument('--set', action='append', default=[], metavar='NAME=VALUE',
                    help='settings override of the headline variant (repeatable)')
    ap.add_argument('--coarse-scale', type=float, default=None,
                    help='over-correction factor of the headline variant\'s prolongation (default: the variant\'s)')
    ap.add_argument('--workload', default='single256', choices=('single256', 'batched48', 'fire'),
                    help='single256: the 256^3 collider scene (default); batched48: 48 uneven domains; '
                         'fire: four 192x192x320 fire domains with a moving collider')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    elif args.workload == 'batched48':
        run_batched(args)
    elif args.workload == 'fire':
        run_fire(args)
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
