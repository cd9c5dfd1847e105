"""Descriptor and policy behaviour of the drop-in API, following the reference's
own unit tests (tests/test_physics.py, test_mac.py, test_pressure.py,
test_multigrid.py, test_detail.py, test_collision.py, test_timestep.py,
test_combustion.py, test_emission.py in FluxFX). CPU only."""
import math
from dataclasses import replace

import pytest

from fluxfx_b200.physics.collision import Collider, primitive, raster_reference
from fluxfx_b200.physics.combustion import react
from fluxfx_b200.physics.config import AdvectionSettings, GridSpec, validate_dt, workgroups
from fluxfx_b200.physics.emission import Emission, Source, motion_velocity, pack_sources
from fluxfx_b200.physics.interaction import validate_live_update
from fluxfx_b200.physics.pressure import PressureSettings, divergence_stats
from fluxfx_b200.physics.thermal import ThermalSettings, acceleration
from fluxfx_b200.physics.timestep import cfl_timestep, choose_timestep


def test_grid_validation_and_memory():
    for shape in ((0, 8, 8), (129, 8, 8), (8.0, 8, 8), (8, 8)):
        with pytest.raises(ValueError):
            GridSpec(shape)
    for extent in ((1, 0, 1), (math.nan, 1, 1), (math.inf, 1, 1)):
        with pytest.raises(ValueError):
            GridSpec(extent=extent)
    assert workgroups((7, 5, 3)) == (2, 2, 1)
    assert GridSpec().density_bytes == 2 * 1024 * 1024
    g = GridSpec((6, 5, 4), (2.0, 3.0, 4.0))
    assert g.face_shapes == ((7, 5, 4), (6, 6, 4), (6, 5, 5))
    assert g.mac_bytes == 8 * (120 + 140 + 144 + 150)


def test_axis_cap_is_lifted_only_on_request():
    with pytest.raises(ValueError):
        GridSpec((256, 256, 256))
    g = GridSpec((256, 256, 256), axis_limit=256)
    assert g.cells == 256 ** 3
    with pytest.raises(ValueError):
        GridSpec((320, 8, 8), axis_limit=256)
    with pytest.raises(ValueError):
        GridSpec((8, 8, 8), axis_limit=64)


def test_timestep_and_advection_validation():
    for dt in (0, -1, math.nan, math.inf, 0.2):
        with pytest.raises(ValueError):
            validate_dt(dt)
    with pytest.raises(ValueError):
        AdvectionSettings(source_rate=-1)
    with pytest.raises(ValueError):
        AdvectionSettings(source_radius=0)
    with pytest.raises(ValueError):
        AdvectionSettings(velocity=(0, math.nan, 0))


def test_thermal_settings_and_force_sign():
    s = ThermalSettings(source_rate=0, heat_source_rate=0, dissipation=0, cooling=0)
    assert acceleration(100, 0, s) > 0 and acceleration(-100, 0, s) < 0 and acceleration(0, 1, s) < 0
    assert acceleration(10, 1, s) == pytest.approx(0)
    for kwargs in ({'cooling': -1}, {'thermal_lift': -1}, {'density_weight': -1},
                   {'heat_source_rate': math.nan}, {'initial_temperature': math.nan}):
        with pytest.raises(ValueError):
            ThermalSettings(**kwargs)


def test_pressure_settings_validation():
    for kwargs in ({'pressure_iterations': 0}, {'pressure_iterations': 1.5}, {'pressure_iterations': True},
                   {'pressure_relaxation': 1}, {'pressure_relaxation': float('nan')},
                   {'pressure_cycles': 0}, {'pressure_cycles': 17}, {'pressure_cycles': True},
                   {'pressure_solver': 'bad'}, {'scalar_advection': 'bogus'}, {'vorticity_strength': -1},
                   {'vorticity_limit': 0}, {'density_mode': 'bogus'}, {'source_profile': 'bogus'},
                   {'velocity_advection': 'bogus'}, {'pressure_warm_start': 'bogus'},
                   {'pressure_tolerance': -1e-4}, {'pressure_tolerance': 1.0}, {'velocity_blend': 1.5},
                   {'storage': 'FP16'}, {'heat_mode': 'SET'}, {'mg_max_levels': -1}):
        with pytest.raises(ValueError):
            PressureSettings(**kwargs)
    with pytest.raises(ValueError):
        divergence_stats([1], [float('nan')])
    st = divergence_stats([1.0, -1.0], [0.1, -0.1])
    assert st['ratio'] == pytest.approx(0.1) and st['max_before'] == 1.0 and st['mean_after'] == 0


def test_live_settings():
    a = PressureSettings()
    validate_live_update(a, replace(a, scalar_advection='MACCORMACK', density_mode='TARGET',
                                    source_profile='SOLID', pressure_cycles=8, velocity_advection='MACCORMACK'))
    validate_live_update(a, replace(a, pressure_tolerance=1e-4, pressure_max_cycles=40))
    for change in ({'pressure_warm_start': 'LEGACY'}, {'pressure_solver': 'MULTIGRID'}, {'storage': 'BF16'}):
        with pytest.raises(ValueError):
            validate_live_update(a, replace(a, **change))
    with pytest.raises(TypeError):
        validate_live_update(a, ThermalSettings())


def test_multigrid_policy():
    from fluxfx_b200.backend.multigrid import hierarchy_shapes, use_multigrid
    assert hierarchy_shapes((128, 64, 32)) == [(128, 64, 32), (64, 32, 16), (32, 16, 8), (16, 8, 4)]
    assert hierarchy_shapes((9, 7, 5)) == [(9, 7, 5)]
    assert hierarchy_shapes((64, 64, 64), max_levels=4)[-1] == (8, 8, 8)
    assert use_multigrid(GridSpec(), PressureSettings())
    assert not use_multigrid(GridSpec((128, 127, 128)), PressureSettings())
    assert not use_multigrid(GridSpec((128, 128, 128)), PressureSettings(pressure_solver='JACOBI'))
    assert use_multigrid(GridSpec(), PressureSettings(pressure_solver='MULTIGRID'))


def test_colliders():
    sphere = primitive('SPHERE', (.5, .5, .5), (.2,) * 3)
    box = primitive('BOX', (.5, .5, .5), (.2,) * 3)
    assert sphere.contains((.6, .5, .5)) and not sphere.contains((.69, .69, .5))
    assert box.contains((.69, .69, .5)) and not box.contains((.71, .5, .5))
    c = math.sqrt(.5)
    rotated = Collider('BOX', ((c / .3, c / .3, 0, 0), (-c / .1, c / .1, 0, 0), (0, 0, 10, 0)))
    assert rotated.contains((.2, .2, 0)) and not rotated.contains((.2, -.2, 0))
    grid = GridSpec((8, 6, 4), (2, 1, 1))
    a = primitive('BOX', (.5, .5, .5), (.25, .2, .2))
    b = primitive('SPHERE', (1.5, .5, .5), (.25, .2, .2))
    assert raster_reference(grid, (a, b)) == [max(x, y) for x, y in zip(raster_reference(grid, (a,)),
                                                                          raster_reference(grid, (b,)))]
    for args in [('MESH', ((1, 0, 0, 0), (0, 1, 0, 0), (0, 0, 1, 0))), ('BOX', ((0, 0, 0, 0),) * 3),
                 ('BOX', ((float('nan'), 0, 0, 0),) * 3)]:
        with pytest.raises(ValueError):
            Collider(*args)
    with pytest.raises(ValueError):
        primitive('BOX', (0, 0, 0), (1, 0, 1))


def test_emitters():
    data = pack_sources([Source((.5,) * 3, .1, 1, -10, Emission((.5,) * 3), 'TARGET', 'SOLID')])
    assert data[12:16] == (-10, 1, 1, 0) and len(data) == 128
    with pytest.raises(ValueError):
        pack_sources([Source((.5,) * 3, .1, 1, 1, Emission((.5,) * 3))] * 9)
    with pytest.raises(ValueError):
        Emission((0, 0))
    with pytest.raises(ValueError):
        Source((.5,) * 3, 0, 1, 1, Emission((.5,) * 3))
    v = motion_velocity((0, 0, 0), (3, 4, 0), 1.0, 1.0, (0, 0, 1), 2.5)
    assert v == pytest.approx((1.5, 2.0, 1.0))


def test_timestep_policies():
    assert choose_timestep(0.05, 0.8, 0.0) == 0.05
    q = choose_timestep(0.05, 0.8, 40.0, quantized=True)
    assert q == 0.0125
    c = choose_timestep(0.05, 0.8, 40.0, 50.0, quantized=False)
    assert 40 * c + 50 * c * c <= 0.8
    assert cfl_timestep(0.02, 0.5, (1 / 256,) * 3, 0.0) == 0.02
    assert cfl_timestep(0.02, 0.5, (1 / 256,) * 3, 1.0) == pytest.approx(0.5 / 256)
    with pytest.raises(RuntimeError):
        choose_timestep(0.05, 0.8, 1e9, quantized=False)


def test_combustion_kinetics():
    assert react(1.0, 200, 0.1, 150, 4.0) == pytest.approx(1 - math.exp(-0.4))
    assert react(1.0, 100, 0.1, 150, 4.0) == 0
    with pytest.raises(ValueError):
        react(-1.0, 200, 0.1, 150, 4.0)


def test_rigid_collider_motion_rows():
    """Wall velocity rows of a moved collider (physics/collider_motion.py:107-118):
    translation gives the linear velocity everywhere, a rotation about the
    centre gives omega x (p - c); shape or size changes are rejected."""
    from fluxfx_b200.physics.collider_motion import velocity_rows, validate_motion
    from fluxfx_b200.physics.collision import Collider
    a = primitive('BOX', (0.4, 0.5, 0.5), (0.1, 0.2, 0.1))
    b = primitive('BOX', (0.42, 0.49, 0.5), (0.1, 0.2, 0.1))
    rows = velocity_rows(a, b, 0.02)
    for p in ((0.1, 0.2, 0.3), (0.9, 0.4, 0.2)):
        v = [r[0] * p[0] + r[1] * p[1] + r[2] * p[2] + r[3] for r in rows]
        assert v == pytest.approx([1.0, -0.5, 0.0], abs=1e-12)
    theta, c = 0.1, (0.5, 0.5, 0.5)
    ct, st = math.cos(theta), math.sin(theta)
    rot = ((ct, -st, 0.0), (st, ct, 0.0), (0.0, 0.0, 1.0))       # columns = rotated axes
    size = (0.1, 0.2, 0.1)
    rrows = []
    for i in range(3):
        r = [rot[k][i] / size[i] for k in range(3)]
        rrows.append(tuple(r + [-sum(r[k] * c[k] for k in range(3))]))
    rows = velocity_rows(primitive('BOX', c, size), Collider('BOX', tuple(rrows)), 0.02)
    w = theta / 0.02
    p = (0.7, 0.45, 0.3)
    v = [r[0] * p[0] + r[1] * p[1] + r[2] * p[2] + r[3] for r in rows]
    assert v == pytest.approx([-w * (p[1] - c[1]), w * (p[0] - c[0]), 0.0], abs=1e-9)
    with pytest.raises(ValueError):
        validate_motion((a,), (primitive('BOX', (0.4, 0.5, 0.5), (0.1, 0.3, 0.1)),))
    with pytest.raises(ValueError):
        validate_motion((a,), (a, b))


def test_warm_start_extrapolation_setting():
    assert PressureSettings().warm_start_extrapolation == 0.0     # the reference's start by default
    assert PressureSettings(warm_start_extrapolation=1).warm_start_extrapolation == 1
    assert PressureSettings(warm_start_extrapolation=0.5, solid_warm_start=True).warm_start_extrapolation == 0.5
    for bad in (-0.1, 1.5, math.nan, math.inf, '1', True):
        with pytest.raises(ValueError):
            PressureSettings(warm_start_extrapolation=bad)


def test_coarse_sweeps_setting():
    assert PressureSettings().mg_coarse_sweeps == 0      # the reference: the same sweeps on every level
    assert PressureSettings(mg_coarse_sweeps=2).mg_coarse_sweeps == 2
    for bad in (-1, 17, 2.0, True):
        with pytest.raises(ValueError):
            PressureSettings(mg_coarse_sweeps=bad)


def test_warm_start_order_setting():
    assert PressureSettings().warm_start_order == 1
    assert PressureSettings(warm_start_order=2).warm_start_order == 2
    for bad in (0, 3, 2.0, True):
        with pytest.raises(ValueError):
            PressureSettings(warm_start_order=bad)
