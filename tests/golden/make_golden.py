"""Generate golden vectors from the FluxFX reference's own CPU code.

Run once in a checkout that has the reference sources available:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py /path/to/FluxFX_Source

It imports the reference's pure-Python oracles (``fluxfx/physics/reference.py``,
``mac_reference.py``, ``pressure_reference.py``, ``thermal_reference.py``,
``coarse_pressure.py``, ``solid_hierarchy.py``, ``collision.py``,
``emission.py``, ``timestep.py``) and writes their outputs on small seeded
inputs to ``tests/golden/*.npz``. The test suite only reads the ``.npz`` files.
"""
import sys
from dataclasses import replace
from math import prod, sqrt
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def main(ref_root):
    sys.path.insert(0, str(ref_root))
    from fluxfx.physics.config import GridSpec, AdvectionSettings
    from fluxfx.physics.thermal import ThermalSettings
    from fluxfx.physics import reference, mac_reference, pressure_reference, thermal_reference
    from fluxfx.physics.coarse_pressure import coarse_inverse
    from fluxfx.physics.solid_hierarchy import build_hierarchy, graph_inverse
    from fluxfx.physics.collision import primitive, raster_reference, Collider
    from fluxfx.physics.emission import Source, Emission, pack_sources
    from fluxfx.physics.timestep import choose_timestep

    # -- P0.2 open-boundary advection in a prescribed flow -----------------------
    grid = GridSpec((8, 6, 4))
    field = [float((i * 7) % 13) for i in range(prod(grid.shape))]
    s = AdvectionSettings(velocity=(0.3, -0.2, 0.1), angular_speed=1.0, source_rate=2.0, dissipation=0.1)
    out = reference.advect(field, grid, s, 0.07)
    quiet = AdvectionSettings(velocity=(1.25, 0, 0), angular_speed=0, source_rate=0, dissipation=0)
    impulse = [0.0] * prod(grid.shape)
    impulse[2 + 8 * (2 + 6 * 1)] = 1.0
    moved = reference.advect(impulse, grid, quiet, 0.1)
    np.savez_compressed(OUT / 'advect_open.npz', shape=grid.shape, extent=grid.extent, field=field, result=out,
             velocity=s.velocity, angular=s.angular_speed, center=s.source_center, radius=s.source_radius,
             rate=s.source_rate, decay=s.dissipation, dt=0.07, impulse=impulse, moved=moved)

    # -- P0.3 MAC self-advection and density transport ---------------------------
    grid = GridSpec((6, 5, 4), (2.0, 3.0, 4.0))
    vel = tuple([((i * 7 + 3 * a) % 19 - 9) / 10 for i in range(prod(sh))] for a, sh in enumerate(grid.face_shapes))
    adv = mac_reference.advect_velocity(vel, grid, 0.07)
    dens = [((i * 5) % 11) / 11 for i in range(prod(grid.shape))]
    ds = AdvectionSettings(velocity=(0, 0, 0), angular_speed=0, source_center=(1.0, 1.5, 1.2),
                           source_radius=0.9, source_rate=3.0, dissipation=0.2)
    dres = mac_reference.advect_density(dens, vel, grid, ds, 0.07)
    seed = mac_reference.seed_velocity(grid, AdvectionSettings(velocity=(.2, -.3, .4), angular_speed=0.7))
    np.savez_compressed(OUT / 'mac.npz', shape=grid.shape, extent=grid.extent, u=vel[0], v=vel[1], w=vel[2],
             au=adv[0], av=adv[1], aw=adv[2], density=dens, dresult=dres, center=ds.source_center,
             radius=ds.source_radius, rate=ds.source_rate, decay=ds.dissipation, dt=0.07,
             su=seed[0], sv=seed[1], sw=seed[2], seed_velocity=(.2, -.3, .4), seed_angular=0.7)

    # -- P0.4 thermal step (SL velocity, buoyancy, SL scalars) -------------------
    grid = GridSpec((5, 4, 3), (1.0, 0.8, 0.6))
    ts = ThermalSettings(source_center=(0.5, 0.4, 0.1), source_radius=0.3, source_rate=1.5,
                         dissipation=0.1, heat_source_rate=20.0, cooling=0.3, thermal_lift=0.01,
                         density_weight=0.2)
    vel = tuple([((i * 3 + a) % 7 - 3) / 10 for i in range(prod(sh))] for a, sh in enumerate(grid.face_shapes))
    dens = [((i * 3) % 5) / 5 for i in range(60)]
    temp = [((i * 7) % 9) * 4.0 - 10 for i in range(60)]
    d2, t2, v2 = thermal_reference.step(dens, temp, vel, grid, ts, 0.05)
    np.savez_compressed(OUT / 'thermal.npz', shape=grid.shape, extent=grid.extent, u=vel[0], v=vel[1], w=vel[2],
             density=dens, temperature=temp, d2=d2, t2=t2, u2=v2[0], v2=v2[1], w2=v2[2], dt=0.05,
             center=ts.source_center, radius=ts.source_radius, rate=ts.source_rate, decay=ts.dissipation,
             heat_rate=ts.heat_source_rate, cooling=ts.cooling, lift=ts.thermal_lift, weight=ts.density_weight)

    # -- closed-box projection ----------------------------------------------------
    grid = GridSpec((6, 5, 4), (1.3, .8, 1.7))
    vel = tuple([((i * 7 + a * 3) % 19 - 9) / 13 for i in range(prod(sh))] for a, sh in enumerate(grid.face_shapes))
    bounded = pressure_reference.walls(vel, grid)
    div = pressure_reference.divergence(bounded, grid)
    p = [((i * 11) % 17) / 17 for i in range(prod(grid.shape))]
    lap = pressure_reference.laplacian(p, grid)
    grad = pressure_reference.pressure_gradient(p, grid)
    solved = pressure_reference.solve(div, grid, 0.04, iterations=37)
    corrected, pressure, stats = pressure_reference.project(vel, grid, 0.04, iterations=37)
    np.savez_compressed(OUT / 'pressure.npz', shape=grid.shape, extent=grid.extent, u=vel[0], v=vel[1], w=vel[2],
             bu=bounded[0], bv=bounded[1], bw=bounded[2], div=div, p=p, lap=lap,
             gu=grad[0], gv=grad[1], gw=grad[2], solved=solved, iterations=37, dt=0.04,
             cu=corrected[0], cv=corrected[1], cw=corrected[2], pressure=pressure,
             rms_after=stats['rms_after'], ratio=stats['ratio'])

    # -- 4^3 Neumann pseudoinverse --------------------------------------------------
    np.savez_compressed(OUT / 'coarse_inverse.npz', unit=coarse_inverse((1., 1., 1.)),
             skew=coarse_inverse((1.3, .8, 1.7)))

    # -- aggregation hierarchy ------------------------------------------------------
    cases = {}
    cube = [float(2 <= x < 4 and 2 <= y < 4 and 2 <= z < 4) for z in range(8) for y in range(8) for x in range(8)]
    cases['cube'] = ((8, 8, 8), (1., 2., 3.), cube)
    slab = [float(z in (3, 4)) for z in range(8) for y in range(8) for x in range(8)]
    cases['slab'] = ((8, 8, 8), (1., 1., 1.), slab)
    disc = [1.] * 512
    disc[0] = disc[1 + 8 + 64] = 0
    cases['disconnected'] = ((8, 8, 8), (1., 1., 1.), disc)
    sph = []
    for z in range(16):
        for y in range(16):
            for x in range(32):
                sph.append(float((x - 11.5) ** 2 + (y - 7.5) ** 2 + (z - 6.5) ** 2 <= 16))
    cases['sphere'] = ((32, 16, 16), (2., 1., 1.), sph)
    arrays = {}
    for name, (shape, extent, mask) in cases.items():
        levels = build_hierarchy(shape, extent, mask)
        arrays[f'{name}_shape'] = shape
        arrays[f'{name}_extent'] = extent
        arrays[f'{name}_mask'] = mask
        arrays[f'{name}_levels'] = len(levels)
        for i, (sh, edges) in enumerate(levels):
            arrays[f'{name}_level{i}_shape'] = sh
            arrays[f'{name}_level{i}_edges'] = np.array(edges, dtype=np.float32)
        sh, edges = levels[-1]
        if prod(sh) <= 256 and len(levels) > 1:
            arrays[f'{name}_inverse'] = np.array(graph_inverse(sh, edges), dtype=np.float32)
    np.savez_compressed(OUT / 'solid_hierarchy.npz', names=list(cases), **arrays)

    # -- collider raster --------------------------------------------------------------
    grid = GridSpec((8, 6, 4), (2, 1, 1))
    a = primitive('BOX', (.5, .5, .5), (.25, .2, .2))
    b = primitive('SPHERE', (1.5, .5, .5), (.25, .2, .2))
    union = raster_reference(grid, (a, b))
    c = sqrt(.5)
    rotated = Collider('BOX', ((c / .18, c / .18, 0, -c / .18), (-c / .1, c / .1, 0, 0), (0, 0, 1 / .2, -.5 / .2)))
    sphere = primitive('SPHERE', (.35, .5, .5), (.17,) * 3)
    grid2 = GridSpec((24, 20, 16))
    scene = raster_reference(grid2, (sphere, rotated))
    np.savez_compressed(OUT / 'raster.npz', shape=grid.shape, extent=grid.extent, union=union,
             rows_a=a.inverse_rows, rows_b=b.inverse_rows, shape2=grid2.shape, extent2=grid2.extent,
             scene=scene, rows_sphere=sphere.inverse_rows, rows_rotated=rotated.inverse_rows)

    # -- emitter table and timestep policy ---------------------------------------------
    srcs = [Source((.5, .4, .3), .1, 1, -10, Emission((.45, .4, .3), (0, 0, 1), 2.5), 'TARGET', 'SOLID', .25),
            Source((.2, .6, .7), .2, .5, 3, Emission((.2, .6, .7)))]
    table = pack_sources(srcs)
    dts = [choose_timestep(0.05, 0.8, r, a, quantized=q)
           for r in (0.0, 3.0, 40.0) for a in (0.0, 50.0) for q in (True, False)]
    np.savez_compressed(OUT / 'emission_timestep.npz', table=table, dts=dts)
    print('golden fixtures written to', OUT)


if __name__ == '__main__':
    sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
    from oracle.glsl_ref.build import REFERENCE_CHECKOUT
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else REFERENCE_CHECKOUT)
