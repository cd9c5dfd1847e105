"""Division by a grid constant on grids that are not powers of two.

The transport kernels divide positions by the cell spacing h, the cell count n
and the extent e with a reciprocal and two remainder corrections (div_rn in
ffx_common.cuh) instead of the IEEE division. ffx_division_mismatches compares
the two over all 2^32 FP32 inputs for one divisor. Over the inputs the form is
exact for (+-0, +-inf, NaN and every finite a with 2^-96 <= |a| <= 2^96, which
holds every grid position) every divisor here must give zero mismatches: the
constants of the fire grid (192 x 192 x 320 cells of 1/192), of the batched
domains (1/64 cells, extents 0.5 to 2), of the test grids, the ends of the
divisor range [2^-30, 2^30] and seeded random divisors across it."""
import numpy as np
import pytest
import torch

from tests.gpu_helpers import dev

pytestmark = pytest.mark.gpu


def _grid_constants(shape, extent):
    out = []
    for n, e in zip(shape, extent):
        e32, n32 = np.float32(e), np.float32(n)
        out += [float(e32), float(n32), float(np.float32(e32 / n32))]
    return out


def _divisors():
    ds = []
    ds += _grid_constants((192, 192, 320), (1.0, 1.0, 320 / 192))           # fire
    ds += _grid_constants((48, 96, 64), (0.75, 1.5, 1.0))                    # batched extents
    ds += _grid_constants((12, 10, 8), (1.3, 0.8, 1.7))                      # dispatch test grid
    ds += _grid_constants((48, 40, 56), (1.0, 40 / 48, 56 / 48))             # moving-collider test grid
    ds += [3.0, 7.0, 0.1, 1 / 3, 1e-5, 1e5, 123.456, 2.0 ** -30, 2.0 ** 30, 1.5 * 2.0 ** -30, 0.75 * 2.0 ** 30]
    rng = np.random.default_rng(2024)
    ds += [float(np.float32(v)) for v in 2.0 ** rng.uniform(-29.5, 29.5, 12)]
    return sorted(set(float(np.float32(v)) for v in ds))


def test_division_by_grid_constants_is_exact():
    D = dev()
    count = torch.zeros(2, dtype=torch.int64, device='cuda')
    import ctypes as C
    bad, outside = {}, {}
    for b in _divisors():
        D.call('ffx_division_mismatches', b, C.c_void_p(count.data_ptr()), D.s)
        inside, other = (int(v) for v in count.cpu())
        if inside:
            bad[b] = inside
        outside[b] = other
    # +-0, +-inf, NaN and 2^-96 <= |a| <= 2^96: bit-identical to the IEEE division
    assert not bad, bad
    print('mismatches outside the exact class (nonzero |a| < 2^-96, finite |a| > 2^96):', outside)
