"""Data, training and evaluation of the learned pressure warm start.

    python -m fluxfx_b200.learned.train --runs 64 --steps 256 --every 4 --size 128 \
        --epochs 3 --batch 8 --eval 256 --out weights.pt

Data: seeded collider scenes in the style of the 256^3 benchmark scene (a
sphere and a box at seeded positions, two emitters in the lower third,
MacCormack transport, buoyancy) at ``--size``^3; every ``--every``-th step of
each run records the projection's divergence, collider mask and converged
pressure (the plain aggregation solver to relative max-norm divergence 1e-4).
Pairs are normalised per sample: input divergence x s, target pressure x s
minus its fluid mean, s = 1 / max|div|. Training: Adam on mean-squared error
over fluid cells. Evaluation: on held-out runs (other seeds), the number of
V-cycles the reference's aggregation V(4,4) solver needs to reach the
tolerance from a zero initial guess and from the network's prediction.
"""
import argparse
import json
import math
import time

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


def normalise(div, pressure, mask):
    """(div x s, pressure x s minus its fluid mean, s) of one sample."""
    m = float(div.abs().max())
    s = 1.0 / m if m > 0 else 1.0
    fluid = mask == 0
    target = pressure * s
    mean = target[fluid].mean() if bool(fluid.any()) else target.new_zeros(())
    return (div * s).contiguous(), (target - mean).contiguous(), s


def generate(device, n, runs, steps, every, seed0):
    """Pairs (div, mask, pressure) from `runs` seeded runs, kept on the device."""
    from ..backend.projected import DenseProjectedSmoke
    divs, masks, targets, scales = [], [], [], []
    for run in range(runs):
        grid, settings, colliders, emitters, noise = scene(n, seed0 + run)
        solver = DenseProjectedSmoke(grid, settings, device, colliders=colliders)
        solver.upload(torch.zeros(grid.cells))
        solver.upload_temperature(torch.zeros(grid.cells))
        solver.upload_velocity([torch.as_tensor(v) for v in noise])
        dt, h = 0.02, 1.0 / n
        for k in range(steps):
            solver.step(dt, sources=emitters)
            umax = max(solver.projector.velocity_maxima())
            dt = min(0.02, 0.5 * h / umax) if umax > 0 else 0.02
            if (k + 1) % every:
                continue
            p = solver.projector
            d, t, s = normalise(p.before.clone(), p.pressure.clone(), solver.solids.mask)
            divs.append(d)
            targets.append(t)
            masks.append(solver.solids.mask.clone())
            scales.append(s)
        solver.close()
    return torch.stack(divs), torch.stack(masks), torch.stack(targets), scales


def train(net, data, epochs, batch, lr, stream, log=None):
    divs, masks, targets, _ = data
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


def predict(net, div, mask, stream):
    """Pressure guess for one divergence field (the network's scale undone)."""
    m = float(div.abs().max())
    s = 1.0 / m if m > 0 else 1.0
    pred = net.forward(div.unsqueeze(0).contiguous(), mask.unsqueeze(0).contiguous(), s, stream)
    return pred[0] / s


def cycles_to_tolerance(projector, div, guess, tol=1e-4, budget=200):
    """V-cycles of the reference aggregation solver from `guess` (None = 0) to
    max|rhs - L p| <= tol max|rhs|."""
    projector.before.copy_(div)
    if guess is None:
        projector.pressure.zero_()
    else:
        projector.pressure.copy_(guess)
    projector.levels[0]['p'], projector.levels[0]['q'] = projector.pressure, projector.spare
    scale = float(div.abs().max())
    cycles = 0
    while cycles < budget and projector._residual_max() > tol * scale:
        projector.cycle(0)
        cycles += 1
    projector.pressure, projector.spare = projector.levels[0]['p'], projector.levels[0]['q']
    return cycles


def evaluate(net, device, n, runs, steps, every, seed0, stream):
    from ..backend.collision import SolidDevice
    from ..backend.solid_multigrid import SolidMultigridProjector
    data = generate(device, n, runs, steps, every, seed0)
    divs, masks = data[0], data[1]
    results = []
    cache = {}
    for i in range(divs.shape[0]):
        run = i // max(1, steps // every)
        if run not in cache:
            grid, settings, colliders, _, _ = scene(n, seed0 + run)
            sd = SolidDevice(grid, colliders, device)
            cache.clear()
            cache[run] = SolidMultigridProjector(grid, settings, sd)
        proj = cache[run]
        div = divs[i]
        cold = cycles_to_tolerance(proj, div, None)
        guess = predict(net, div, masks[i], stream)
        warm = cycles_to_tolerance(proj, div, guess)
        results.append((cold, warm))
    cold = [c for c, _ in results]
    warm = [w for _, w in results]
    return {'fields': len(results), 'cycles_cold_mean': float(np.mean(cold)), 'cycles_warm_mean': float(np.mean(warm)),
            'cycles_saved_mean': float(np.mean(cold) - np.mean(warm)), 'cycles_cold': cold, 'cycles_warm': warm}


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
    args = ap.parse_args()
    from ..backend.device import CudaDevice
    dev = CudaDevice()
    stream = dev.stream.cuda_stream
    t0 = time.perf_counter()
    data = generate(dev, args.size, args.runs, args.steps, args.every, args.seed)
    gen_s = time.perf_counter() - t0
    print(json.dumps({'pairs': int(data[0].shape[0]), 'size': args.size, 'generate_seconds': gen_s}), flush=True)
    net = UNet(dev.device, seed=0)
    history = train(net, data, args.epochs, args.batch, args.lr, stream, log=lambda h: print(json.dumps(h), flush=True))
    del data
    torch.cuda.empty_cache()
    ev = evaluate(net, dev, args.size, args.eval_runs, args.steps, args.every, args.seed + 100000, stream)
    report = {'train': history, 'eval': {k: v for k, v in ev.items() if not k.startswith('cycles_') or k.endswith('mean')},
              'generate_seconds': gen_s}
    print(json.dumps(report), flush=True)
    if args.report:
        with open(args.report, 'w') as f:
            json.dump(report | {'eval_cycles': {'cold': ev['cycles_cold'], 'warm': ev['cycles_warm']}}, f)
    if args.out:
        torch.save(net.state_dict(), args.out)


if __name__ == '__main__':
    main()
