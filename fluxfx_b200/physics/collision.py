"""Static analytic colliders: unit sphere/box primitives under an affine inverse map.

Follows FluxFX ``fluxfx/physics/collision.py:6-37``. ``inverse_rows`` are three
rows (a, b, c, d) mapping a point p in metres to q = A p + d; the solid is
|q| <= 1 (sphere) or max|q_i| <= 1 (box), boundaries inclusive.

``raster_reference`` is the CPU statement of the voxelisation the device
raster kernel reproduces bit-for-bit (it evaluates in FP64 in the same
operation order).
"""
from dataclasses import dataclass
from math import isfinite

import numpy as np

SHAPES = ('SPHERE', 'BOX')


@dataclass(frozen=True)
class Collider:
    shape: str
    inverse_rows: tuple

    def __post_init__(self):
        if self.shape not in SHAPES:
            raise ValueError('Collider must be a sphere or box')
        rows = self.inverse_rows
        if len(rows) != 3 or any(len(r) != 4 for r in rows):
            raise ValueError('Collider requires three affine inverse rows')
        if not all(isfinite(v) for r in rows for v in r):
            raise ValueError('Collider transform must be finite')
        (a0, a1, a2), (b0, b1, b2), (c0, c1, c2) = (r[:3] for r in rows)
        det = a0 * (b1 * c2 - b2 * c1) - a1 * (b0 * c2 - b2 * c0) + a2 * (b0 * c1 - b1 * c0)
        if abs(det) < 1e-12:
            raise ValueError('Collider transform must be invertible')

    def local(self, point):
        return tuple(r[0] * point[0] + r[1] * point[1] + r[2] * point[2] + r[3] for r in self.inverse_rows)

    def contains(self, point):
        q = self.local(point)
        if self.shape == 'SPHERE':
            return q[0] * q[0] + q[1] * q[1] + q[2] * q[2] <= 1
        return max(abs(v) for v in q) <= 1

    @property
    def table_row(self):
        """12 FP64 coefficients + shape code, the layout the raster kernel reads."""
        return [float(v) for r in self.inverse_rows for v in r] + [float(self.shape == 'BOX')]


def primitive(shape, center, size):
    """Axis-aligned collider; ``size`` is the sphere radius or box half-size per axis."""
    if len(center) != 3 or len(size) != 3 or not all(isfinite(v) and v > 0 for v in size):
        raise ValueError('Three positive finite sizes required')
    rows = []
    for i in range(3):
        row = [0.0, 0.0, 0.0, -center[i] / size[i]]
        row[i] = 1 / size[i]
        rows.append(tuple(row))
    return Collider(shape, tuple(rows))


def raster_reference(grid, colliders):
    """Union of colliders sampled at cell centres; x-fast list of 0.0/1.0."""
    nx, ny, nz = grid.shape
    h = grid.cell_size
    x = (np.arange(nx, dtype=np.float64) + .5) * h[0]
    y = (np.arange(ny, dtype=np.float64) + .5) * h[1]
    z = (np.arange(nz, dtype=np.float64) + .5) * h[2]
    pz, py, px = np.meshgrid(z, y, x, indexing='ij')  # each (nz, ny, nx)
    solid = np.zeros((nz, ny, nx), dtype=bool)
    for c in colliders:
        q = [((0.0 + r[0] * px) + r[1] * py) + r[2] * pz + r[3] for r in c.inverse_rows]
        if c.shape == 'SPHERE':
            inside = ((0.0 + q[0] * q[0]) + q[1] * q[1]) + q[2] * q[2] <= 1
        else:
            inside = np.maximum(np.maximum(np.abs(q[0]), np.abs(q[1])), np.abs(q[2])) <= 1
        solid |= inside
    return solid.astype(np.float64).ravel().tolist()
