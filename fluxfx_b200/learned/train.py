"""Data, training and evaluation of the learned pressure warm start.

    python -m fluxfx_b200.learned.train --runs 64 --steps 256 --every 4 --size 128 \
        --epochs 3 --batch 8 --eval-runs 4 --out weights.pt --report report.json

Data: seeded collider scenes in the style of the 256^3 benchmark scene (a
sphere and a box at seeded positions, two emitters in the lower third,
MacCormack transport, buoyancy) at ``--size``^3; every ``--every``-th step of
each run records the projection's divergence, collider mask and converged
pressure (relative max-norm residual 1e-4; 64 runs x 256 steps / 4 = 4096
pairs by default). Pairs are normalised per sample: input divergence x s,
target (pressure x s minus its fluid mean) x w, s = 1 / max|div|, w = (n /
extent)^2 the Laplacian's conductance, so both are of order one. Training: Adam on
the mean-squared error over fluid cells. Evaluation: on held-out runs (other
seeds; 4 runs give 256 fields), the cycles that the aggregation V(4,4)
iteration and the V(1,1)-preconditioned conjugate gradients need to reach the
tolerance from zero, from the network's prediction and from the previous
step's pressure (the solver's own warm start).
"""
import argparse
import json
import time
from dataclasses import replace

import numpy as np
import torch

from .unet import UNet


def scene(n, seed):
    """Grid, settings, colliders, emitters and initial velocity of one seeded run."""
    from ..physics.collision import primitive
    from ..physics.config import GridSpec
    from ..physics.emission import Emission, Source
    from ..physics.pressure import PressureSettings
    rng = np.random.default_rng(seed)
    grid = GridSpec((n, n, n), axis_limit=max(128, n))
    r = rng.uniform(0.1, 0.18)
    sphere = primitive('SPHERE', tuple(rng.uniform(0.25, 0.75, 3)), (r, r, r))
    box = primitive('BOX', tuple(rng.uniform(0.2, 0.8, 3)), tuple(rng.uniform(0.04, 0.12, 3)))
    emitters = []
    for _ in range(2):
        pos = (rng.uniform(0.2, 0.8), rng.uniform(0.2, 0.8), rng.uniform(0.1, 0.3))
        d, t = rng.uniform(0.5, 1.0, 2)
        emitters.append(Source(pos, 8.0 / 256.0, float(d), float(t), Emission(pos), 'TARGET', 'SOFT'))
    settings = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=1.0,
                                density_weight=0.05, heat_mode='TARGET', pressure_tolerance=1e-4,
                                pressure_max_cycles=200)
    noise = [rng.uniform(-1e-3, 1e-3, (fs[2], fs[1], fs[0])).astype(np.float32) for fs in grid.face_shapes]
    return grid, settings, (sphere, box), emitters, noise


def weight_of(grid):
    """Largest Laplacian conductance (n / extent)^2: pressure x weight has the
    magnitude of the divergence."""
    return max((n / e) ** 2 for n, e in zip(grid.shape, grid.extent))


def normalise(div, pressure, mask, weight):
    """(div x s, (pressure x s minus its fluid mean) x weight, s) of one sample."""
    m = float(div.abs().max())
    s = 1.0 / m if m > 0 else 1.0
    fluid = mask == 0
    target = pressure * (s * weight)
    mean = target[fluid].mean() if bool(fluid.any()) else target.new_zeros(())
    return (div * s).contiguous(), (target - mean).contiguous(), s


def _fast_settings(settings):
    """The same scene solved by V(1,1)-preconditioned conjugate gradients with
    the previous pressure as the start (the converged pressure is the same to
    the tolerance; only the work to get there differs)."""
    return replace(settings, pressure_method='PCG', solid_warm_start=True, mg_pre_sweeps=1, mg_post_sweeps=1,
                   pressure_max_cycles=256)


def generate(device, n, runs, steps, every, seed0, previous=False):
    """Pairs (div, mask, pressure, scale) from `runs` seeded runs, kept on the
    device in preallocated stacks. With ``previous`` also the warm start the
    solver itself would use for each recorded solve: the previous step's
    pressure rescaled by dt / previous dt (impulse form)."""
    from ..backend.projected import DenseProjectedSmoke
    per_run = steps // every
    count = runs * per_run
    shape = (count, n, n, n)
    dev = device.device
    divs = torch.empty(shape, dtype=torch.float32, device=dev)
    targets = torch.empty(shape, dtype=torch.float32, device=dev)
    masks = torch.empty(shape, dtype=torch.uint8, device=dev)
    prevs = torch.empty(shape, dtype=torch.float32, device=dev) if previous else None
    scales = []
    i = 0
    for run in range(runs):
        grid, settings, colliders, emitters, noise = scene(n, seed0 + run)
        solver = DenseProjectedSmoke(grid, _fast_settings(settings), device, colliders=colliders)
        solver.upload(torch.zeros(grid.cells))
        solver.upload_temperature(torch.zeros(grid.cells))
        solver.upload_velocity([torch.as_tensor(v) for v in noise])
        dt, h, last_dt = 0.02, 1.0 / n, None
        for k in range(steps):
            record = (k + 1) % every == 0
            p = solver.projector
            if record and previous:
                prevs[i].copy_(p.pressure)
                if last_dt is not None and last_dt != dt:
                    prevs[i].mul_(dt / last_dt)
                elif last_dt is None:
                    prevs[i].zero_()
            solver.step(dt, sources=emitters)
            last_dt = dt
            umax = max(p.velocity_maxima())
            dt = min(0.02, 0.5 * h / umax) if umax > 0 else 0.02
            if not record:
                continue
            d, t, s = normalise(p.before, p.pressure, solver.solids.mask, weight_of(grid))
            divs[i].copy_(d)
            targets[i].copy_(t)
            masks[i].copy_(solver.solids.mask)
            scales.append(s)
            i += 1
        solver.close()
    return divs, masks, targets, scales, prevs


def train(net, data, epochs, batch, lr, stream, log=None):
    divs, masks, targets = data[:3]
    count = divs.shape[0]
    gen = torch.Generator().manual_seed(0)
    history = []
    for epoch in range(epochs):
        order = torch.randperm(count, generator=gen)
        total, nb = 0.0, 0
        t0 = time.perf_counter()
        for i in range(0, count - batch + 1, batch):
            idx = order[i:i + batch].to(divs.device)
            net.forward(divs[idx], masks[idx], 1.0, stream)
            loss = net.loss_backward(targets[idx], masks[idx], stream)
            net.adam_step(lr, stream)
            total += float(loss[0])
            nb += 1
        torch.cuda.synchronize()
        history.append({'epoch': epoch, 'loss': total / max(nb, 1), 'seconds': time.perf_counter() - t0,
                        'steps': nb})
        if log:
            log(history[-1])
    return history


def predict(net, div, mask, stream, weight):
    """Pressure guess for one divergence field (the network's scales undone)."""
    m = float(div.abs().max())
    s = 1.0 / m if m > 0 else 1.0
    pred = net.forward(div.unsqueeze(0).contiguous(), mask.unsqueeze(0).contiguous(), s, stream)
    return pred[0] / (s * weight)


def solve_count(projector, div, guess, budget=256):
    """Cycles the projector's method needs from ``guess`` (None = zero) to
    max|rhs - L p| <= tol max|rhs|: stand-alone V-cycles or preconditioned
    conjugate-gradient iterations (one V-cycle each)."""
    tol = projector.settings.pressure_tolerance
    projector.before.copy_(div)
    if guess is None:
        projector.pressure.zero_()
    else:
        projector.pressure.copy_(guess)
    projector.levels[0]['p'], projector.levels[0]['q'] = projector.pressure, projector.spare
    projector.last_cycles = 0
    projector.last_iterations = 0
    scale = float(div.abs().max())
    if projector.settings.pressure_method == 'PCG':
        projector._solve_krylov(scale, budget)
        projector.levels[0]['p'], projector.levels[0]['q'] = projector.pressure, projector.spare
        return projector.last_cycles
    cycles = 0
    while cycles < budget and projector._residual_max() > tol * scale:
        projector.cycle(0)
        cycles += 1
    projector.pressure, projector.spare = projector.levels[0]['p'], projector.levels[0]['q']
    return cycles


def forward_ms(net, n, stream, repeat=20):
    """Device time of one batch-1 forward pass at n^3 (CUDA events)."""
    div = torch.randn((1, n, n, n), device=net.device)
    mask = torch.zeros((1, n, n, n), dtype=torch.uint8, device=net.device)
    for _ in range(3):
        net.forward(div, mask, 1.0, stream)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cs = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
    start.record(cs)
    for _ in range(repeat):
        net.forward(div, mask, 1.0, stream)
    end.record(cs)
    end.synchronize()
    return start.elapsed_time(end) / repeat


def lowpass(field, levels, device):
    """Keep the smooth part of a cell field: ``levels`` 2x2x2 averages down,
    then trilinear prolongation back up (library multigrid transfers)."""
    from .. import _native as N
    from ..backend.device import ptr
    shapes = [tuple(field.shape[::-1])]
    for _ in range(levels):
        shapes.append(tuple(n // 2 for n in shapes[-1]))
    fields = [field.contiguous()]
    for k in range(levels):
        c = torch.empty(shapes[k + 1][::-1], dtype=torch.float32, device=field.device)
        device.call('ffx_mg_restrict', N.n3(*shapes[k]), ptr(fields[-1]), ptr(c), device.s)
        fields.append(c)
    up = fields[-1]
    for k in range(levels - 1, -1, -1):
        zero = torch.zeros(shapes[k][::-1], dtype=torch.float32, device=field.device)
        fine = torch.empty_like(zero)
        device.call('ffx_mg_prolong', N.n3(*shapes[k]), ptr(zero), ptr(up), ptr(fine), device.s)
        up = fine
    return up


def _initial_residual(projector, div, guess):
    projector.before.copy_(div)
    projector.pressure.copy_(guess)
    projector.levels[0]['p'], projector.levels[0]['q'] = projector.pressure, projector.spare
    return projector._residual_max() / max(float(div.abs().max()), 1e-30)


def _relative_error(guess, exact, fluid):
    g = guess[fluid] - guess[fluid].mean()
    e = exact[fluid] - exact[fluid].mean()
    return float((g - e).norm() / max(float(e.norm()), 1e-30))


def evaluate(net, device, n, runs, steps, every, seed0, stream, lowpass_levels=(1, 2)):
    """Cycles to the tolerance on held-out fields for the aggregation V(4,4)
    iteration and for the V(1,1)-preconditioned CG, each from zero, from the
    network's prediction (raw and low-passed) and from the previous step's
    pressure; with the guesses' relative error against the converged
    pressure and their initial relative residual."""
    from ..backend.collision import SolidDevice
    from ..backend.solid_multigrid import SolidMultigridProjector
    divs, masks, _, scales, prevs = generate(device, n, runs, steps, every, seed0, previous=True)
    per_run = steps // every
    guesses = ['zero', 'net'] + [f'net_lp{k}' for k in lowpass_levels] + ['previous']
    out = {m: {g: [] for g in guesses} for m in ('vcycle', 'pcg')}
    error = {g: [] for g in guesses[1:]}
    residual = {g: [] for g in guesses[1:]}
    for run in range(runs):
        grid, settings, colliders, _, _ = scene(n, seed0 + run)
        sd = SolidDevice(grid, colliders, device)
        projectors = {'vcycle': SolidMultigridProjector(grid, replace(settings, pressure_max_cycles=256), sd),
                      'pcg': SolidMultigridProjector(grid, _fast_settings(settings), sd)}
        for j in range(per_run):
            i = run * per_run + j
            div = divs[i] / scales[i]        # the recorded rhs (normalisation undone)
            fluid = masks[i] == 0
            net_guess = predict(net, div, masks[i], stream, weight_of(grid)).clone()
            cand = {'zero': None, 'net': net_guess, 'previous': prevs[i]}
            for k in lowpass_levels:
                cand[f'net_lp{k}'] = lowpass(net_guess, k, device)
            vc = projectors['vcycle']
            out['vcycle']['zero'].append(solve_count(vc, div, None))
            exact = vc.pressure.clone()
            for g in guesses[1:]:
                error[g].append(_relative_error(cand[g], exact, fluid))
                residual[g].append(_initial_residual(vc, div, cand[g]))
            for m, proj in projectors.items():
                for g in guesses:
                    if m == 'vcycle' and g == 'zero':
                        continue
                    out[m][g].append(solve_count(proj, div, cand[g]))
        for proj in projectors.values():
            proj.close()
        sd.close()
    summary = {'fields': len(out['pcg']['zero'])}
    for m, d in out.items():
        for g, v in d.items():
            summary[f'{m}_{g}_mean'] = float(np.mean(v))
        best_net = min((g for g in guesses if g.startswith('net')), key=lambda g: summary[f'{m}_{g}_mean'])
        summary[f'{m}_best_net'] = best_net
        summary[f'{m}_saved_vs_zero'] = summary[f'{m}_zero_mean'] - summary[f'{m}_{best_net}_mean']
        summary[f'{m}_saved_vs_previous'] = summary[f'{m}_previous_mean'] - summary[f'{m}_{best_net}_mean']
    for g in guesses[1:]:
        summary[f'error_{g}_median'] = float(np.median(error[g]))
        summary[f'residual_{g}_median'] = float(np.median(residual[g]))
    return summary, out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--size', type=int, default=128)
    ap.add_argument('--runs', type=int, default=64)
    ap.add_argument('--steps', type=int, default=256)
    ap.add_argument('--every', type=int, default=4)
    ap.add_argument('--epochs', type=int, default=3)
    ap.add_argument('--batch', type=int, default=8)
    ap.add_argument('--lr', type=float, default=1e-3)
    ap.add_argument('--eval-runs', type=int, default=4)
    ap.add_argument('--seed', type=int, default=1000)
    ap.add_argument('--out', default=None)
    ap.add_argument('--report', default=None)
    ap.add_argument('--load', default=None, help='evaluate these weights instead of training')
    args = ap.parse_args()
    from ..backend.device import CudaDevice
    dev = CudaDevice()
    stream = dev.stream.cuda_stream
    net = UNet(dev.device, seed=0)
    history, gen_s = [], 0.0
    if args.load:
        net.load_state_dict(torch.load(args.load))
    else:
        t0 = time.perf_counter()
        data = generate(dev, args.size, args.runs, args.steps, args.every, args.seed)
        gen_s = time.perf_counter() - t0
        t = data[2]
        print(json.dumps({'pairs': int(data[0].shape[0]), 'size': args.size, 'generate_seconds': gen_s,
                          'target_rms': float(t.pow(2).mean().sqrt()), 'target_max': float(t.abs().max()),
                          'input_rms': float(data[0].pow(2).mean().sqrt())}), flush=True)
        history = train(net, data, args.epochs, args.batch, args.lr, stream,
                        log=lambda h: print(json.dumps(h), flush=True))
        del data
        torch.cuda.empty_cache()
    if args.out:
        torch.save(net.state_dict(), args.out)
    t0 = time.perf_counter()
    summary, cycles = evaluate(net, dev, args.size, args.eval_runs, args.steps, args.every, args.seed + 100000, stream)
    report = {'config': vars(args), 'train': history, 'generate_seconds': gen_s,
              'evaluate_seconds': time.perf_counter() - t0, 'forward_ms': forward_ms(net, args.size, stream),
              'eval': summary}
    print(json.dumps(report), flush=True)
    if args.report:
        with open(args.report, 'w') as f:
            json.dump(report | {'eval_cycles': cycles}, f)


if __name__ == '__main__':
    main()
