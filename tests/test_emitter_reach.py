"""The emitter reach box the CUDA passes use to skip emission_weight: every
point outside it must evaluate to exactly zero in the FP32 weight (here the
oracle's restatement of ``emission_weight.glsl:2-29``, same operation order).
The box is min/max(start, center) -/+ (r + 4e-3 M), M = max(|extent|,
|start|, |center|, r), rounded outwards to float. CPU only."""
import numpy as np
import pytest

from oracle import smoke as S


def reach(center, start, radius, extent):
    m = max([abs(radius)] + [abs(float(v)) for v in (*extent, *center, *start)])
    margin = abs(radius) + 4e-3 * m
    lo = np.minimum(np.float64(center), np.float64(start)) - margin
    hi = np.maximum(np.float64(center), np.float64(start)) + margin
    flo, fhi = lo.astype(np.float32), hi.astype(np.float32)
    flo = np.where(flo.astype(np.float64) > lo, np.nextafter(flo, np.float32(-np.inf)), flo)
    fhi = np.where(fhi.astype(np.float64) < hi, np.nextafter(fhi, np.float32(np.inf)), fhi)
    return flo, fhi


def just_outside(rng, lo, hi, extent, count):
    """Points in [0, extent] outside [lo, hi], most of them within a few ulps of a face."""
    pts = rng.uniform(0, 1, (count, 3)).astype(np.float32) * np.float32(extent)
    axis = rng.integers(0, 3, count)
    side = rng.integers(0, 2, count)
    steps = rng.integers(1, 4, count)
    for k in range(count):
        a = axis[k]
        v = np.float32(lo[a]) if side[k] == 0 else np.float32(hi[a])
        for _ in range(steps[k]):
            v = np.nextafter(v, np.float32(-np.inf) if side[k] == 0 else np.float32(np.inf))
        pts[k, a] = v
    keep = np.any((pts < lo) | (pts > hi), axis=1)
    return pts[keep]


@pytest.mark.parametrize('solid', [False, True])
def test_weight_is_zero_outside_the_reach_box(solid):
    rng = np.random.default_rng(5 + solid)
    g = S.Grid((8, 8, 8), (1.0, 1.0, 1.0), np.float32)
    checked = 0
    for trial in range(300):
        extent = rng.uniform(0.5, 4.0, 3)
        center = rng.uniform(0, 1, 3) * extent
        kind = trial % 3
        if kind == 0:
            start = center.copy()                                   # static sphere
        elif kind == 1:
            start = center + rng.normal(0, 1e-7, 3)                 # degenerate sweep (l2 < 1e-12)
        else:
            start = np.clip(center + rng.normal(0, 0.2, 3) * extent, 0, extent)
        radius = float(10 ** rng.uniform(-3, -0.5)) * float(extent.max())
        center, start = center.astype(np.float32), start.astype(np.float32)
        lo, hi = reach(center, start, radius, extent)
        pts = just_outside(rng, lo, hi, extent, 64)
        w = S.emission_weight(g, [pts[:, 0], pts[:, 1], pts[:, 2]], center, start, radius, solid)
        assert np.all(np.asarray(w) == 0), (trial, np.asarray(w).max())
        # and the box is not empty of emission: the segment's points inside weigh > 0
        mid = (center.astype(np.float64) + start) / 2
        inside = S.emission_weight(g, [np.float32([mid[0]]), np.float32([mid[1]]), np.float32([mid[2]])],
                                   center, start, radius, solid)
        assert float(np.asarray(inside).max()) > 0
        checked += len(pts)
    assert checked > 10000
