"""The sparse brick projection against its dense twin on the GPU
(FluxFX_Source/native/projection.mm compare_projection): the same seeded
velocity projected with Jacobi sweeps or V-cycles on active bricks only and on
dense arrays gives identical pressure, divergence and faces on the solve
region, reduces the divergence, and stores only the bricks the region needs."""
import pytest

from fluxfx_b200.backend.sparse import compare_projection

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('mode', [0, 1, 2])
@pytest.mark.parametrize('iterations, cycles', [(48, 0), (0, 3)])
@pytest.mark.parametrize('n, side', [(64, 8), (128, 16)])
def test_sparse_projection_equals_dense(mode, iterations, cycles, n, side):
    r = compare_projection(n, side, iterations, mode, cycles)
    assert r['pressure_error'] == 0.0 and r['divergence_error'] == 0.0, r
    assert r['before_error'] == 0.0 and r['face_error'] == 0.0, r
    # 48 damped Jacobi sweeps remove 20-50 % of the divergence RMS of this
    # seeded field (measured 0.52-0.81 of it left), three V-cycles about 90 %
    assert r['after_rms'] < (0.9 if cycles == 0 else 0.2) * r['before_rms'], r
    if mode:
        assert r['sparse_bytes'] < 0.7 * r['dense_bytes'], r
    else:
        assert r['active_bricks'] == (n // side) ** 3
