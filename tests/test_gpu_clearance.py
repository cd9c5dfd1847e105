"""The clearance field (ffx_halo_clearance, ffx_clearance) and the transport
passes' clear forms.

* The field equals its definition computed on the host: 1 exactly where no
  solid cell and no cell outside the grid lies within Chebyshev distance 3, 2
  where no solid cell but a cell outside the grid does, 0 elsewhere.
* Steps that use the field give the fields of the same steps without it, bit
  for bit: power-of-two and other grids, FP32 and BF16 storage, emitters,
  static and moving colliders, and traces both within the clear form's 0.75
  cells and far beyond it (which take the full collider tests).
"""
import numpy as np
import pytest
import torch
from scipy.ndimage import maximum_filter

from tests.gpu_helpers import dev

pytestmark = pytest.mark.gpu


def _expected_clear(solid):
    inner = (slice(3, -3),) * 3
    walls = np.pad(solid.astype(np.uint8), 3, constant_values=1)       # outside counts as solid
    near_any = maximum_filter(walls, size=7, mode='constant', cval=1)[inner]
    mask = np.pad(solid.astype(np.uint8), 3, constant_values=0)        # solids only
    near_solid = maximum_filter(mask, size=7, mode='constant', cval=0)[inner]
    return np.where(near_solid != 0, 0, np.where(near_any != 0, 2, 1)).astype(np.uint8)


@pytest.mark.parametrize('n', [48, 64])
def test_clearance_matches_its_definition(n):
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    D = dev()
    grid, s, colliders, _, _ = bench.scene(n, 'FP32', 1)
    sv = DenseProjectedSmoke(grid, s, D, colliders=colliders)
    torch.cuda.synchronize()
    solid = sv.solids.mask.cpu().numpy() != 0
    clear = sv.solids.clear.cpu().numpy()
    assert np.array_equal(clear, _expected_clear(solid))
    assert set(np.unique(clear)) == {0, 1, 2}
    sv.close()


def _without_clear(sv):
    for owner in (sv, sv.detail, sv.projector):
        owner._solids.clear = None


def _pair(n, storage, variant, amp, seed=4):
    import bench
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    D = dev()
    out = []
    for use_clear in (True, False):
        grid, s, colliders, emitters, noise = bench.scene(n, storage, seed, **bench.VARIANTS[variant])
        sv = DenseProjectedSmoke(grid, s, D, colliders=colliders)
        if not use_clear:
            _without_clear(sv)
        sv.upload(torch.zeros(grid.cells))
        sv.upload_temperature(torch.zeros(grid.cells))
        sv.upload_velocity([torch.as_tensor(v * (amp / 1e-3)) for v in noise])
        out.append(sv)
    return out, emitters


def _fields(sv):
    torch.cuda.synchronize()
    return [sv.density, sv.temperature, sv.projector.pressure, *sv._velocity]


@pytest.mark.parametrize('n,storage,variant,amp', [
    (64, 'FP32', 'plain', 1e-3),     # power-of-two grid: traces well inside 0.75 cells
    (64, 'BF16', 'fast', 0.3),       # up to ~0.4 cells per step
    (64, 'FP32', 'fast', 2.0),       # ~2.5 cells: the full collider tests
    (48, 'FP32', 'plain', 0.3),      # h = 1/48: the clear form's rounding-exact fast values
    (48, 'BF16', 'fast', 2.0),
])
def test_clear_form_is_bit_identical(n, storage, variant, amp):
    (a, b), em = _pair(n, storage, variant, amp)
    for k in range(4):
        a.step(0.02, sources=em)
        b.step(0.02, sources=em)
        for x, y in zip(_fields(a), _fields(b)):
            assert torch.equal(x, y), (n, storage, variant, amp, k)
    a.close()
    b.close()


def test_clear_form_with_a_moving_collider():
    from fluxfx_b200.backend.projected import DenseProjectedSmoke
    from fluxfx_b200.backend.solid_multigrid import SolidMultigridProjector
    from fluxfx_b200.physics.collision import primitive
    from fluxfx_b200.physics.config import GridSpec
    from fluxfx_b200.physics.pressure import PressureSettings
    D = dev()
    shape = (48, 40, 56)
    grid = GridSpec(shape)
    hx = 1.0 / shape[0]
    s = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', moving_colliders=True,
                         thermal_lift=1.0, density_weight=0.05, source_center=(0.5, 0.5, 0.2), source_radius=0.1,
                         pressure_tolerance=1e-4, pressure_max_cycles=100, vorticity_strength=0.3)
    pose = lambda k: (primitive('SPHERE', (0.3 + 0.5 * hx * k, 0.5, 0.6), (0.15, 0.15, 0.15)),)
    rng = np.random.default_rng(8)
    vel = [torch.as_tensor((rng.uniform(-1, 1, (fs[2], fs[1], fs[0])) * 0.3).astype(np.float32))
           for fs in grid.face_shapes]
    solvers = []
    for use_clear in (True, False):
        sv = DenseProjectedSmoke(grid, s, D, projector_class=SolidMultigridProjector, colliders=pose(0))
        if not use_clear:
            _without_clear(sv)
        sv.upload_velocity(vel)
        solvers.append(sv)
    a, b = solvers
    for k in range(5):
        for sv in solvers:
            sv.move_colliders(pose(k + 1), 0.02)
            sv.step(0.02)
        torch.cuda.synchronize()
        assert torch.equal(a.solids.clear, torch.as_tensor(_expected_clear(a.solids.mask.cpu().numpy() != 0),
                                                           device=a.solids.clear.device)), k
        for x, y in zip([a.density, a.temperature, *a._velocity], [b.density, b.temperature, *b._velocity]):
            assert torch.equal(x, y), k
    a.close()
    b.close()


@pytest.mark.parametrize('shape', [(64, 64, 64), (37, 9, 21), (1, 1, 1), (33, 17, 40), (200, 3, 5)])
def test_one_pass_halo_and_clearance(shape):
    """ffx_halo_clearance's halo equals ffx_dilate_mask's bit for bit, its
    clearance is 1 exactly where ffx_dilate_mask followed by ffx_clearance gives
    1 and equals the three-valued definition everywhere, on grids whose extents
    are and are not multiples of its tile (32 x 8 x 16 cells), with empty,
    sparse and dense random masks."""
    import ctypes as C
    from fluxfx_b200 import _native as N
    D = dev()
    nx, ny, nz = shape
    g = N.grid_struct(shape, (1.0, 1.0, 1.0))
    rng = np.random.default_rng(nx + 5 * ny + 11 * nz)
    for density in (0.0, 0.002, 0.05):
        mask = torch.as_tensor((rng.uniform(size=(nz, ny, nx)) < density).astype(np.uint8), device='cuda')
        halo2, clear2, halo1, clear1 = (torch.full((nz, ny, nx), 7, dtype=torch.uint8, device='cuda')
                                        for _ in range(4))
        p = lambda x: C.c_void_p(x.data_ptr())
        D.call('ffx_dilate_mask', C.byref(g), p(mask), p(halo2), D.s)
        D.call('ffx_clearance', C.byref(g), p(halo2), p(clear2), D.s)
        D.call('ffx_halo_clearance', C.byref(g), p(mask), p(halo1), p(clear1), D.s)
        torch.cuda.synchronize()
        assert torch.equal(halo1, halo2), (shape, density)
        assert torch.equal(clear1 == 1, clear2 == 1) and int(clear2.max()) <= 1, (shape, density)
        assert np.array_equal(clear1.cpu().numpy(), _expected_clear(mask.cpu().numpy() != 0)), (shape, density)
