"""CPU restatement of the fire-configuration passes -- TEST INFRASTRUCTURE ONLY.

Vorticity confinement, combustion and moving colliders of FluxFX, vectorised
NumPy in the shaders' FP32 operation order (GLSL vector expressions evaluate
component-wise, left to right; ``dot`` sums x, y, z[, w] in order; ``cross``
and ``length`` as in the CPU build of the shaders). Pinned against the
reference's own backend running its own shaders on the CPU
(``tests/golden/reference_fire_steps.npz``). Only ``tests/``, ``smoke()`` and
the CPU-baseline leg of ``bench.py`` use this module.
"""
import numpy as np

from . import smoke as S


def _clampi(v, n):
    return np.clip(v, 0, n - 1)


# ----------------------------------------------------------------------------
# vorticity confinement (backend/detail.py:39-49, curl.glsl, confinement.glsl)
# ----------------------------------------------------------------------------
def _centered_velocity(g, vel, x, y, z):
    """``centeredVelocity`` (curl.glsl:1-7): face averages at the clamped cell."""
    U, V, W = vel
    nx, ny, nz = g.shape
    x, y, z = _clampi(x, nx), _clampi(y, ny), _clampi(z, nz)
    half = g.f(0.5)
    return (half * (U[z, y, x] + U[z, y, x + 1]),
            half * (V[z, y, x] + V[z, y + 1, x]),
            half * (W[z, y, x] + W[z + 1, y, x]))


def curl(g, vel):
    """(omega.xyz, |omega|) per cell (curl.glsl:8-17); returns an (nz, ny, nx, 4) array."""
    x, y, z = g.coords(g.cell_shape)
    half = g.f(0.5)

    def diff(dx, dy, dz, inv):
        a = _centered_velocity(g, vel, x + dx, y + dy, z + dz)
        b = _centered_velocity(g, vel, x - dx, y - dy, z - dz)
        return tuple(((ai - bi) * half) * inv for ai, bi in zip(a, b))

    ddx = diff(1, 0, 0, g.inv[0])
    ddy = diff(0, 1, 0, g.inv[1])
    ddz = diff(0, 0, 1, g.inv[2])
    om = (ddy[2] - ddz[1], ddz[0] - ddx[2], ddx[1] - ddy[0])
    mag = np.sqrt(S._dot(om, om))
    return np.stack([om[0], om[1], om[2], mag], axis=-1).astype(g.dt)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _force_at(g, c4, x, y, z, strength, limit):
    """``forceAt`` (confinement.glsl:5-15) at cells (x, y, z), clamped reads."""
    f = g.f
    nx, ny, nz = g.shape

    def at(xx, yy, zz):
        return c4[_clampi(zz, nz), _clampi(yy, ny), _clampi(xx, nx)]

    half = f(0.5)
    coef = [half * g.inv[a] for a in range(3)]
    grad = (coef[0] * (at(x + 1, y, z)[..., 3] - at(x - 1, y, z)[..., 3]),
            coef[1] * (at(x, y + 1, z)[..., 3] - at(x, y - 1, z)[..., 3]),
            coef[2] * (at(x, y, z + 1)[..., 3] - at(x, y, z - 1)[..., 3]))
    mag = np.sqrt(S._dot(grad, grad))
    h = f(1.0) / max(g.inv[0], max(g.inv[1], g.inv[2]))
    safe = np.where(mag < f(1e-8), f(1), mag)
    n = tuple(gi / safe for gi in grad)
    here = at(x, y, z)
    cr = _cross(n, (here[..., 0], here[..., 1], here[..., 2]))
    sh = f(strength) * h
    force = tuple(sh * ci for ci in cr)
    flen = np.sqrt(S._dot(force, force))
    scale = np.minimum(f(1.0), f(limit) / np.maximum(flen, f(1e-12)))
    force = tuple(fi * scale for fi in force)
    zero = mag < f(1e-8)
    return tuple(np.where(zero, f(0), fi) for fi in force)


def confine(g, vel, c4, dt, strength, limit):
    """Confinement acceleration added to every face (confinement.glsl:16-23)."""
    f = g.f
    out = []
    for axis in range(3):
        x, y, z = g.coords(g.face_shapes[axis])
        o = [0, 0, 0]
        o[axis] = 1
        fa = _force_at(g, c4, x, y, z, strength, limit)
        fb = _force_at(g, c4, x - o[0], y - o[1], z - o[2], strength, limit)
        force_axis = f(0.5) * (fa[axis] + fb[axis])
        out.append((vel[axis] + f(dt) * force_axis).astype(g.dt))
    return tuple(out)


# ----------------------------------------------------------------------------
# combustion (backend/combustion.py:21-31, combustion_burn.glsl, combustion_apply.glsl)
# ----------------------------------------------------------------------------
def burn(g, fuel, temperature, dt, ignition, rate):
    """Consumed fuel per second (combustion_burn.glsl:1-8)."""
    f = g.f
    fu = np.maximum(fuel, f(0))
    decay = (f(1) - np.exp(-f(rate) * f(dt))).astype(g.dt)
    burned = np.where(temperature >= f(ignition), fu * decay, f(0))
    return (burned / f(dt)).astype(g.dt)


def apply_burn(g, field, flame, dt, yield_value):
    """field + dt * yield * flame, clamped at 0 for negative yields (combustion_apply.glsl:1-7)."""
    f = g.f
    v = field + (f(dt) * f(yield_value)) * flame
    if yield_value < 0:
        v = np.maximum(v, f(0))
    return v.astype(g.dt)


# ----------------------------------------------------------------------------
# moving colliders (backend/moving_collision.py, moving_*.glsl)
# ----------------------------------------------------------------------------
def moving_mask(g, colliders):
    """Owner ids 0 (fluid), 1, 2, ... in collider order, first owner wins
    (moving_mask.glsl:1-11), cell-centre test in FP32."""
    f = g.f
    x, y, z = g.coords(g.cell_shape)
    p = [((c.astype(g.dt) + f(0.5)) * g.e[a]) / g.n[a] for a, c in enumerate((x, y, z))]
    value = g.zeros(g.cell_shape)
    for index, (shape, rows) in enumerate(colliders):
        rows = [tuple(f(v) for v in r) for r in rows]
        q = [((r[0] * p[0] + r[1] * p[1]) + r[2] * p[2]) + r[3] * f(1) for r in rows]
        if shape == 'SPHERE':
            inside = S._dot(q, q) <= f(1.0)
        else:
            inside = (np.abs(q[0]) <= f(1)) & (np.abs(q[1]) <= f(1)) & (np.abs(q[2]) <= f(1))
        value = np.where((value < f(0.5)) & inside, f(index + 1), value)
    return value


def moving_walls(g, owners, table):
    """Rigid wall velocity on every interior face next to a solid cell
    (moving_wall.glsl:1-19). ``table``: (n_colliders, 3, 4) FP32 rows
    v_a(p) = row . (p, 1)."""
    f = g.f
    own = owners.astype(np.int64)
    nx, ny, nz = g.shape
    out = []
    for axis in range(3):
        x, y, z = g.coords(g.face_shapes[axis])
        c = [x, y, z]
        n = g.face_shapes[axis][2 - axis]
        interior = (c[axis] > 0) & (c[axis] < n - 1)
        hi = [_clampi(x, nx), _clampi(y, ny), _clampi(z, nz)]
        lo = list(hi)
        lo[axis] = _clampi(c[axis] - 1, g.shape[axis])
        o_hi = own[hi[2], hi[1], hi[0]]
        o_lo = own[lo[2], lo[1], lo[0]]
        owner = np.where(o_lo > 0, o_lo, o_hi)
        off = [f(0.5)] * 3
        off[axis] = f(0)
        p = [((cc.astype(g.dt) + off[a]) * g.e[a]) / g.n[a] for a, cc in enumerate(c)]
        rows = np.asarray(table, dtype=g.dt).reshape(-1, 3, 4)
        r = rows[np.maximum(owner - 1, 0), axis]          # (..., 4)
        value = ((r[..., 0] * p[0] + r[..., 1] * p[1]) + r[..., 2] * p[2]) + r[..., 3] * f(1)
        out.append(np.where(interior & (owner > 0), value, f(0)).astype(g.dt))
    return tuple(out)


def remap_scalar(g, field, owners, old_owners):
    """Cells covered now or before start empty (moving_remap_scalar.glsl:1-7)."""
    blocked = (owners > 0.5) | (old_owners > 0.5)
    return np.where(blocked, g.f(0), field).astype(g.dt)


def remap_faces(g, vel, owners, old_owners, boundary):
    """Covered faces take the wall velocity, newly exposed ones start at 0
    (moving_remap_face.glsl:1-12)."""
    nx, ny, nz = g.shape
    out = []
    for axis in range(3):
        x, y, z = g.coords(g.face_shapes[axis])
        c = [x, y, z]
        n = g.face_shapes[axis][2 - axis]
        interior = (c[axis] > 0) & (c[axis] < n - 1)
        hi = [_clampi(x, nx), _clampi(y, ny), _clampi(z, nz)]
        lo = list(hi)
        lo[axis] = _clampi(c[axis] - 1, g.shape[axis])
        blocked = (owners[hi[2], hi[1], hi[0]] > 0.5) | (owners[lo[2], lo[1], lo[0]] > 0.5)
        prev = (old_owners[hi[2], hi[1], hi[0]] > 0.5) | (old_owners[lo[2], lo[1], lo[0]] > 0.5)
        v = np.where(blocked, boundary[axis], np.where(prev, g.f(0), vel[axis]))
        out.append(np.where(interior, v, g.f(0)).astype(g.dt))
    return tuple(out)


def _pose(rows):
    """(center, rotation matrix) of a collider from its inverse affine rows
    q = A p + t, A = diag(1/size) R^T."""
    rows = np.asarray(rows, dtype=np.float64)
    a, t = rows[:, :3], rows[:, 3]
    center = -np.linalg.solve(a, t)
    axes = a / np.linalg.norm(a, axis=1, keepdims=True)
    return center, axes.T


def velocity_table(old_rows, new_rows, dt):
    """Rigid-motion velocity rows v_a(p) = row_a . (p, 1) per collider: the
    translation velocity plus omega x (p - new centre), omega the rotation
    vector of the relative rotation divided by dt (the motion model of
    physics/collider_motion.py:107-118), FP64 -> FP32."""
    from scipy.spatial.transform import Rotation
    out = []
    for o, n in zip(old_rows, new_rows):
        c0, r0 = _pose(o)
        c1, r1 = _pose(n)
        omega = Rotation.from_matrix(r1 @ r0.T).as_rotvec() / dt
        x, y, z = omega
        skew = np.array([[0.0, -z, y], [z, 0.0, -x], [-y, x, 0.0]])
        linear = (c1 - c0) / dt
        out.append(np.concatenate([skew, (linear - skew @ c1)[:, None]], axis=1))
    return np.asarray(out, dtype=np.float32)
