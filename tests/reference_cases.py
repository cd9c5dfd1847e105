"""Replay of the reference-backend golden runs (tests/golden/reference_steps.npz,
made by tests/golden/make_golden_glsl.py) on any solver with the drop-in API."""
import json
from pathlib import Path

import numpy as np

GOLD = Path(__file__).resolve().parent / 'golden' / 'reference_steps.npz'
FIRE = Path(__file__).resolve().parent / 'golden' / 'reference_fire_steps.npz'
# Parity bar against the reference run: max abs error <= TOL * max|field| per
# recorded step (the FP32 oracle sits at ~1e-6). The divergence after
# projection is a residual near zero, so it is compared against the scale of
# the divergence before projection: error <= AFTER_TOL * max|div before|.
TOL = 1e-5
AFTER_TOL = 1e-5


def load(path=GOLD):
    return np.load(path)


def cases(path=GOLD):
    return sorted(json.loads(str(load(path)['cases'])))


def fire_cases():
    """Vorticity confinement, combustion and moving-collider runs."""
    return cases(FIRE)


def case(name, path=GOLD):
    from fluxfx_b200.physics.collision import primitive
    from fluxfx_b200.physics.emission import Emission, Source
    from fluxfx_b200.physics.pressure import PressureSettings
    d = load(path)
    spec = json.loads(str(d['cases']))[name]
    shape = tuple(spec['shape'])
    settings = PressureSettings(**{k: (tuple(v) if isinstance(v, list) else v) for k, v in spec['settings'].items()})
    h = [1.0 / n for n in shape]
    colliders = ((primitive('SPHERE', (0.55, 0.5, 0.5), (0.22,) * 3),
                  primitive('BOX', (0.2, 0.3, 0.25), (3 * h[0], 4 * h[1], 2 * h[2]))) if spec['colliders'] else ())
    sources = None
    if spec['sources']:
        rates = [float(v) for v in d['fuel_rates']] if spec.get('fuel') else [0.0, 0.0]
        sources = [Source(tuple(c), r, dd, t, Emission(tuple(m[0]), tuple(m[1]), m[2]), mode, prof, fuel_rate=fr)
                   for (c, r, dd, t, m, mode, prof), fr in zip(json.loads(str(d['sources'])), rates)]
    moving = None
    if spec.get('moving'):
        (cx, cy, cz), r = json.loads(str(d['moving_start']))
        hx = 1.0 / shape[0]
        moving = lambda k: (primitive('SPHERE', (cx + 0.5 * hx * k, cy, cz), (r,) * 3),)
        colliders = moving(0)
    emission = None
    if spec.get('swept'):
        start, vel, coupling = json.loads(str(d['swept']))
        emission = Emission(tuple(start), tuple(vel), coupling)
    rng = np.random.default_rng(14)
    nx, ny, nz = shape
    face_shapes = ((nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx))
    velocity = [(rng.uniform(-1, 1, fs) * 0.3).astype(np.float32) for fs in face_shapes]
    mask = d[f'{name}/mask'].reshape(nz, ny, nx) > 0.5 if (spec['colliders'] or moving) else None
    steps = {}
    for k in d['recorded']:
        k = int(k)
        vel = d[f'{name}/step{k}/velocity']
        sizes = np.cumsum([0] + [int(np.prod(fs)) for fs in face_shapes])
        steps[k] = dict(density=d[f'{name}/step{k}/density'].reshape(nz, ny, nx),
                        temperature=d[f'{name}/step{k}/temperature'].reshape(nz, ny, nx),
                        velocity=[vel[sizes[i]:sizes[i + 1]].reshape(face_shapes[i]) for i in range(3)],
                        after=d[f'{name}/step{k}/after'].reshape(nz, ny, nx),
                        metrics=json.loads(str(d[f'{name}/step{k}/metrics'])))
        for extra in ('fuel', 'flame', 'mask'):
            key = f'{name}/step{k}/{extra}'
            if key in d.files:
                steps[k][extra] = d[key].reshape(nz, ny, nx)
    return dict(shape=shape, settings=settings, colliders=colliders, sources=sources, emission=emission,
                velocity=velocity, mask=mask, dts=tuple(float(v) for v in d['dts']), steps=steps, moving=moving,
                init_density=d[f'{name}/init_density'].reshape(nz, ny, nx),
                init_temperature=d[f'{name}/init_temperature'].reshape(nz, ny, nx))


def compare(got, want, tol, what):
    a = np.asarray(got, dtype=np.float64)
    e = np.asarray(want, dtype=np.float64)
    scale = max(float(np.abs(e).max()), 1e-30)
    err = float(np.abs(a - e).max())
    assert err <= tol * scale, f"{what}: max abs error {err:.3e} > {tol:.0e} * {scale:.3e}"
    return err / scale


def compare_after(got, want_step, what):
    a = np.asarray(got, dtype=np.float64)
    e = np.asarray(want_step['after'], dtype=np.float64)
    scale = max(float(want_step['metrics']['max_before']), 1e-30)
    err = float(np.abs(a - e).max())
    assert err <= AFTER_TOL * scale, f"{what}: max abs error {err:.3e} > {AFTER_TOL:.0e} * max|div before| {scale:.3e}"
    return err / scale
