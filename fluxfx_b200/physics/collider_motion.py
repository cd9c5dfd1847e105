"""Rigid collider motion between two poses (host side, FP64).

Mirrors FluxFX ``fluxfx/physics/collider_motion.py``: a collider is an affine
inverse map q = A p + t with A = diag(1/size) R^T (rotation R, per-axis size);
``validate_motion`` accepts a new pose list only if every collider keeps its
shape and size (``collider_motion.py:81-89``), and ``velocity_rows`` gives the
rigid-body velocity field of the move, v(p) = (c1 - c0)/dt + omega x (p - c1)
with omega the rotation vector of R1 R0^T divided by dt, as three rows of
(p, 1) coefficients per collider (``collider_motion.py:107-118``).
"""
from math import acos, sqrt

from .collision import Collider

MAX_SURFACE_SPEED = 2.0


def _dot(a, b):
    return sum(x * y for x, y in zip(a, b))


def _solve3(a, b):
    """x with A x = b by Cramer's rule (A 3x3, non-singular)."""
    def det(m):
        return (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0])
                + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]))
    d = det(a)
    out = []
    for k in range(3):
        m = [list(r) for r in a]
        for i in range(3):
            m[i][k] = b[i]
        out.append(det(m) / d)
    return tuple(out)


class Pose:
    """Centre, per-axis size and rotation matrix (columns = collider axes)."""

    def __init__(self, shape, center, size, rotation):
        self.shape, self.center, self.size, self.rotation = shape, tuple(center), tuple(size), rotation

    @classmethod
    def from_collider(cls, collider):
        rows = collider.inverse_rows
        size = tuple(1.0 / sqrt(_dot(r[:3], r[:3])) for r in rows)
        axes = tuple(tuple(v * s for v in r[:3]) for r, s in zip(rows, size))
        if any(abs(_dot(axes[i], axes[j])) > 1e-5 for i in range(3) for j in range(i)):
            raise ValueError('Moving colliders do not support shear; use an unscaled or uniformly scaled domain')
        cross = (axes[1][1] * axes[2][2] - axes[1][2] * axes[2][1], axes[1][2] * axes[2][0] - axes[1][0] * axes[2][2],
                 axes[1][0] * axes[2][1] - axes[1][1] * axes[2][0])
        if _dot(axes[0], cross) < 0:
            raise ValueError('Moving colliders require positive scale')
        center = _solve3([list(r[:3]) for r in rows], [-r[3] for r in rows])
        rotation = tuple(tuple(axes[j][i] for j in range(3)) for i in range(3))   # R[i][j] = axis j, component i
        return cls(collider.shape, center, size, rotation)


def validate_motion(previous, current):
    if len(previous) != len(current):
        raise ValueError('Collider entries changed; press Reset')
    poses = []
    for old, new in zip(previous, current):
        a, b = Pose.from_collider(old), Pose.from_collider(new)
        if a.shape != b.shape or any(abs(x - y) > max(x, y) * 1e-5 for x, y in zip(a.size, b.size)):
            raise ValueError('Collider shape or size changed; press Reset')
        poses.append((a, b))
    return tuple(poses)


def _rotation_vector(m):
    """Axis * angle of a rotation matrix (angle in [0, pi])."""
    trace = m[0][0] + m[1][1] + m[2][2]
    angle = acos(max(-1.0, min(1.0, (trace - 1.0) / 2.0)))
    v = (m[2][1] - m[1][2], m[0][2] - m[2][0], m[1][0] - m[0][1])
    s = sqrt(_dot(v, v))
    if angle < 1e-12 or s < 1e-15:
        return (0.0, 0.0, 0.0)
    if angle > 3.14159:
        # near pi the skew part vanishes: take the axis from the symmetric part
        diag = [max(0.0, (m[i][i] + 1.0) / 2.0) for i in range(3)]
        k = max(range(3), key=lambda i: diag[i])
        axis = [0.0, 0.0, 0.0]
        axis[k] = sqrt(diag[k])
        for i in range(3):
            if i != k:
                axis[i] = (m[i][k] + m[k][i]) / (4.0 * axis[k])
        n = sqrt(_dot(axis, axis))
        return tuple(angle * a / n for a in axis)
    return tuple(angle * a / s for a in v)


def velocity_rows(old, new, dt):
    """Rows r_a with v_a(p) = r_a . (p, 1) for the rigid move old -> new in dt."""
    a, b = Pose.from_collider(old), Pose.from_collider(new)
    r0, r1 = a.rotation, b.rotation
    rel = tuple(tuple(sum(r1[i][k] * r0[j][k] for k in range(3)) for j in range(3)) for i in range(3))
    x, y, z = (w / dt for w in _rotation_vector(rel))
    skew = ((0.0, -z, y), (z, 0.0, -x), (-y, x, 0.0))
    linear = tuple((v - u) / dt for u, v in zip(a.center, b.center))
    return tuple(skew[i] + (linear[i] - _dot(skew[i], b.center),) for i in range(3))


def collider_rows12(colliders):
    """12 inverse-affine coefficients per collider (FP64) and the box flags."""
    return ([float(v) for c in colliders for r in c.inverse_rows for v in r],
            [int(c.shape == 'BOX') for c in colliders])


__all__ = ['Collider', 'MAX_SURFACE_SPEED', 'Pose', 'collider_rows12', 'validate_motion', 'velocity_rows']
