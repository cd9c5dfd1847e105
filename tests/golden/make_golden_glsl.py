"""Golden vectors from the reference's own backend running its own shaders.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_glsl.py /path/to/FluxFX_Source [--fire-only]

Builds ``oracle/_ref/libglsl_ref.so`` (the reference's compute shaders compiled
for the CPU by ``oracle/glsl_ref/build.py``), then runs the reference's
unmodified Python backend (``fluxfx.backend.projected.DenseProjectedSmoke`` and
the projector classes it selects) on that CPU device, and records every step's
fields in ``tests/golden/reference_steps.npz``. These cover the shader-only
parts of the hot path that have no Python oracle in the reference: MacCormack
correction, closed and collider-renormalised sampling, trace clipping and
halo tests, swept and table emitters, TARGET emission, geometric and
aggregation multigrid V-cycles, and the impulse warm start.
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent

# Each case is run for three steps with dt = 0.02, 0.02, 0.015 from a seeded
# random velocity (numpy default_rng(14), uniform(-1, 1) * 0.3 per face, x-fast,
# float32) and the reference's seeded scalars; steps 0 and 2 are stored.
CASES = {
    'mg_maccormack_target': dict(
        shape=(16, 16, 16), colliders=False, sources=False,
        settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', density_mode='TARGET',
                      source_rate=1.0, heat_source_rate=1.0, source_profile='SOLID', thermal_lift=1.0,
                      density_weight=0.05, source_radius=0.2, source_center=(.5, .5, .2), pressure_cycles=4)),
    'colliders_maccormack': dict(
        shape=(24, 20, 16), colliders=True, sources=False,
        settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=0.5,
                      density_weight=0.1, source_radius=0.15, source_center=(.3, .5, .2), heat_source_rate=10.0)),
    'colliders_semi_lagrangian_jacobi': dict(
        shape=(12, 10, 8), colliders=True, sources=False,
        settings=dict(thermal_lift=0.5, density_weight=0.1, source_radius=0.2, source_center=(.3, .5, .2),
                      pressure_iterations=30)),
    'table_semi_lagrangian': dict(
        shape=(20, 16, 12), colliders=False, sources=True,
        settings=dict(thermal_lift=0.2, pressure_iterations=40)),
    'table_maccormack_colliders_swept': dict(
        shape=(16, 16, 16), colliders=True, sources=True,
        settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=0.3,
                      pressure_cycles=3)),
    'single_swept_jet_legacy_mg': dict(
        shape=(16, 16, 16), colliders=False, sources=False, swept=True,
        settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', pressure_warm_start='LEGACY',
                      source_radius=0.15, source_center=(.5, .5, .3), pressure_cycles=2)),
}
# Fire-config passes (vorticity confinement, combustion, moving colliders),
# recorded the same way into reference_fire_steps.npz.
FIRE_CASES = {
    'confinement_maccormack': dict(
        shape=(16, 16, 16), colliders=False, sources=False,
        settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', vorticity_strength=0.3,
                      vorticity_limit=2.0, thermal_lift=1.0, density_weight=0.05, source_radius=0.2,
                      source_center=(.5, .5, .2), pressure_cycles=3)),
    'combustion_single': dict(
        shape=(16, 16, 12), colliders=False, sources=False,
        settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', combustion_enabled=True,
                      fuel_source_rate=1.0, ignition_temperature=0.3, burn_rate=0.75, heat_yield=1.0,
                      smoke_yield=0.5, heat_source_rate=0.4, source_radius=0.2, source_center=(.5, .5, .3),
                      thermal_lift=1.0, density_weight=0.05, pressure_cycles=3)),
    'combustion_table_colliders_confined': dict(
        shape=(16, 16, 16), colliders=True, sources=True, fuel=True,
        settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', combustion_enabled=True,
                      ignition_temperature=0.3, burn_rate=0.75, heat_yield=1.0, smoke_yield=0.5,
                      vorticity_strength=0.3, thermal_lift=0.3, pressure_cycles=3)),
    'moving_sphere_jacobi': dict(
        shape=(16, 16, 16), colliders=False, sources=False, moving=True,
        settings=dict(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', moving_colliders=True,
                      thermal_lift=0.5, density_weight=0.1, source_radius=0.15, source_center=(.6, .5, .2),
                      pressure_iterations=30)),
}
MOVING_START = ((0.35, 0.5, 0.5), 0.2)   # sphere centre, radius; moves +x by half a cell per step
FUEL_RATES = (1.5, 0.0)                  # fuel_rate of SOURCES[0], SOURCES[1] in the fuel case
DTS = (0.02, 0.02, 0.015)
RECORDED = (0, 2)   # steps whose fields are stored


def colliders_for(shape, primitive):
    h = [1.0 / n for n in shape]
    return (primitive('SPHERE', (0.55, 0.5, 0.5), (0.22,) * 3),
            primitive('BOX', (0.2, 0.3, 0.25), (3 * h[0], 4 * h[1], 2 * h[2])))


SOURCES = [((.3, .5, .25), .15, 1.0, 2.0, ((.3, .5, .25), (0, 0, 0), 0.0), 'TARGET', 'SOFT'),
           ((.7, .4, .3), .12, .5, 1.0, ((.68, .4, .3), (0, 0, 1), 1.5), 'RATE', 'SOLID')]
SWEPT = ((.45, .5, .28), (0.0, 0.2, 0.8), 2.0)


def run_case(name, spec, arrays, dev, solver, srcs, emission, moving=None):
    shape = spec['shape']
    arrays[f'{name}/init_density'] = np.array(solver.read_density(), dtype=np.float32)
    arrays[f'{name}/init_temperature'] = np.array(solver.read_temperature(), dtype=np.float32)
    if solver.solids is not None:
        arrays[f'{name}/mask'] = np.array(dev.read(solver.solids.mask, shape), dtype=np.float32)
    for k, dt in enumerate(DTS):
        if moving is not None:
            solver.move_colliders(moving(k + 1), dt)
        solver.step(dt, emission=emission, sources=srcs)
        if k not in RECORDED:
            continue
        arrays[f'{name}/step{k}/density'] = np.array(solver.read_density(), dtype=np.float32)
        arrays[f'{name}/step{k}/temperature'] = np.array(solver.read_temperature(), dtype=np.float32)
        arrays[f'{name}/step{k}/velocity'] = np.concatenate(
            [np.array(v, dtype=np.float32) for v in solver.read_velocity()])
        arrays[f'{name}/step{k}/after'] = np.array(dev.read(solver.projector.after, shape), dtype=np.float32)
        if solver.combustion is not None:
            arrays[f'{name}/step{k}/fuel'] = np.array(dev.read(solver.combustion.fuel, shape), dtype=np.float32)
            arrays[f'{name}/step{k}/flame'] = np.array(dev.read(solver.combustion.flame, shape), dtype=np.float32)
        if moving is not None:
            arrays[f'{name}/step{k}/mask'] = np.array(dev.read(solver.solids.mask, shape), dtype=np.float32)
        m = solver.measure_projection()
        arrays[f'{name}/step{k}/metrics'] = np.array(json.dumps({k2: v for k2, v in m.items()
                                                                  if isinstance(v, (int, float, str))}))
    assert dev.out_of_range() == 0, name
    print(name, type(solver.projector).__name__, 'dispatches', dev.dispatches)


def main(ref_root):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ref_root))
    from oracle.glsl_ref.build import build
    build(Path(ref_root) / 'fluxfx' / 'shaders')
    from oracle.glsl_ref.device import GlslCpuDevice
    from fluxfx.backend.projected import DenseProjectedSmoke
    from fluxfx.physics.collision import primitive
    from fluxfx.physics.config import GridSpec
    from fluxfx.physics.emission import Emission, Source
    from fluxfx.physics.pressure import PressureSettings

    arrays = {}
    for name, spec in ({} if '--fire-only' in sys.argv else CASES).items():
        shape = spec['shape']
        dev = GlslCpuDevice()
        cols = colliders_for(shape, primitive) if spec['colliders'] else ()
        solver = DenseProjectedSmoke(GridSpec(shape), PressureSettings(**spec['settings']), dev, colliders=cols)
        rng = np.random.default_rng(14)
        vel = [(rng.uniform(-1, 1, (fs[2], fs[1], fs[0])) * 0.3).astype(np.float32) for fs in solver.grid.face_shapes]
        solver.upload_velocity([v.ravel().tolist() for v in vel])
        srcs = None
        if spec['sources']:
            srcs = [Source(c, r, d, t, Emission(*m), mode, prof) for c, r, d, t, m, mode, prof in SOURCES]
        emission = Emission(*SWEPT) if spec.get('swept') else None
        arrays[f'{name}/init_density'] = np.array(solver.read_density(), dtype=np.float32)
        arrays[f'{name}/init_temperature'] = np.array(solver.read_temperature(), dtype=np.float32)
        if cols:
            arrays[f'{name}/mask'] = np.array(dev.read(solver.solids.mask, shape), dtype=np.float32)
        for k, dt in enumerate(DTS):
            solver.step(dt, emission=emission, sources=srcs)
            if k not in RECORDED:
                continue
            arrays[f'{name}/step{k}/density'] = np.array(solver.read_density(), dtype=np.float32)
            arrays[f'{name}/step{k}/temperature'] = np.array(solver.read_temperature(), dtype=np.float32)
            arrays[f'{name}/step{k}/velocity'] = np.concatenate(
                [np.array(v, dtype=np.float32) for v in solver.read_velocity()])
            arrays[f'{name}/step{k}/after'] = np.array(dev.read(solver.projector.after, shape), dtype=np.float32)
            m = solver.measure_projection()
            arrays[f'{name}/step{k}/metrics'] = np.array(json.dumps({k2: v for k2, v in m.items()
                                                                      if isinstance(v, (int, float, str))}))
        assert dev.out_of_range() == 0, name
        print(name, type(solver.projector).__name__, 'dispatches', dev.dispatches)
    fire = {}
    for name, spec in FIRE_CASES.items():
        shape = spec['shape']
        dev = GlslCpuDevice()
        moving = None
        if spec.get('moving'):
            (cx, cy, cz), r = MOVING_START
            h = 1.0 / shape[0]
            moving = lambda k, cx=cx, cy=cy, cz=cz, r=r, h=h: (primitive('SPHERE', (cx + 0.5 * h * k, cy, cz), (r,) * 3),)
            cols = moving(0)
        else:
            cols = colliders_for(shape, primitive) if spec['colliders'] else ()
        solver = DenseProjectedSmoke(GridSpec(shape), PressureSettings(**spec['settings']), dev, colliders=cols)
        rng = np.random.default_rng(14)
        vel = [(rng.uniform(-1, 1, (fs[2], fs[1], fs[0])) * 0.3).astype(np.float32) for fs in solver.grid.face_shapes]
        solver.upload_velocity([v.ravel().tolist() for v in vel])
        srcs = None
        if spec['sources']:
            rates = FUEL_RATES if spec.get('fuel') else (0.0, 0.0)
            srcs = [Source(c, r, d, t, Emission(*m), mode, prof, fuel_rate=fr)
                    for (c, r, d, t, m, mode, prof), fr in zip(SOURCES, rates)]
        run_case(name, spec, fire, dev, solver, srcs, None, moving)
    fire['cases'] = np.array(json.dumps(FIRE_CASES))
    fire['dts'] = np.array(DTS)
    fire['recorded'] = np.array(RECORDED)
    fire['sources'] = np.array(json.dumps(SOURCES))
    fire['fuel_rates'] = np.array(FUEL_RATES)
    fire['moving_start'] = np.array(json.dumps(MOVING_START))
    np.savez_compressed(HERE / 'reference_fire_steps.npz', **fire)
    print('wrote', HERE / 'reference_fire_steps.npz')
    if '--fire-only' in sys.argv:
        return
    arrays['cases'] = np.array(json.dumps({n: {k: v for k, v in s.items()} for n, s in CASES.items()}))
    arrays['dts'] = np.array(DTS)
    arrays['recorded'] = np.array(RECORDED)
    arrays['sources'] = np.array(json.dumps(SOURCES))
    arrays['swept'] = np.array(json.dumps(SWEPT))
    np.savez_compressed(HERE / 'reference_steps.npz', **arrays)
    print('wrote', HERE / 'reference_steps.npz')


if __name__ == '__main__':
    from oracle.glsl_ref.build import REFERENCE_CHECKOUT
    args = [a for a in sys.argv[1:] if not a.startswith('--')]
    main(Path(args[0]) if args else REFERENCE_CHECKOUT)
