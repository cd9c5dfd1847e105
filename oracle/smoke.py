"""CPU oracle of FluxFX's dense MAC smoke step -- TEST INFRASTRUCTURE ONLY.

This module is the checker. Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it; the product package
(``fluxfx_b200``) never does.

It restates, as vectorised NumPy, every per-cell formula of the reference's
hot path (GLSL compute shaders under ``fluxfx/shaders/``) and the host-side
orchestration that sequences them (``fluxfx/backend/*.py``). Each function
cites the reference file:line it follows. Arithmetic runs in the dtype of the
``Grid`` (float32 to mirror the device kernels operation-for-operation, or
float64 for the "error against an FP64 run" figures). Expressions keep the
GLSL evaluation order (``mix(x, y, a) = x*(1-a) + y*a``, dot products summed
x, y, z) so that FP32 results and every discrete decision (floor, clamps,
trace clipping, MacCormack fallbacks) agree with the CUDA kernels, which are
compiled without FMA contraction.

Layout: scalar fields are arrays of shape (nz, ny, nx) (x fastest); face
fields U, V, W have shapes (nz, ny, nx+1), (nz, ny+1, nx), (nz+1, ny, nx).
Vectors are tuples (x, y, z) of arrays. Masks are bool arrays of the cell
shape (True = solid).

Pinning: the pure-Python oracles of the reference (``fluxfx/physics/
reference.py``, ``mac_reference.py``, ``pressure_reference.py``,
``thermal_reference.py``, ``coarse_pressure.py``, ``solid_hierarchy.py``,
``collision.py``) are matched at 1e-12 on the golden fixtures in
``tests/golden``. The shader-only parts (MacCormack, closed sampling, trace
clipping, multigrid cycles, emission sweeps) have no Python counterpart in the
reference; they are pinned against the reference's GLSL sources compiled for
the CPU (``oracle/glsl_ref``) where that library has been built.
"""
from math import prod

import numpy as np

FACE_OFFSETS = ((0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0))
HUGE = 3.4e38
TRACE_LIMIT = 384


# ----------------------------------------------------------------------------
# grid context
# ----------------------------------------------------------------------------
class Grid:
    """Cell counts, extent, arithmetic dtype and (optional) solid mask."""

    def __init__(self, shape, extent=(1.0, 1.0, 1.0), dtype=np.float32, mask=None):
        self.shape = tuple(int(n) for n in shape)          # (nx, ny, nz)
        self.extent64 = tuple(float(e) for e in extent)
        self.dt = np.dtype(dtype)
        f = self.dt.type
        self.n = tuple(f(n) for n in self.shape)
        self.e = tuple(f(e) for e in self.extent64)
        self.h = tuple(e / n for e, n in zip(self.e, self.n))              # domainExtent / cellCount
        self.inv = tuple(f(1.0 / (e / n)) for e, n in zip(self.extent64, self.shape))  # host 1/h
        nx, ny, nz = self.shape
        self.cell_shape = (nz, ny, nx)
        self.face_shapes = ((nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx))
        self.mask = None
        self.halo = None
        self.boundary = None      # moving colliders: wall velocity per face grid (moving_wall.glsl)
        if mask is not None:
            self.set_mask(mask)

    def f(self, v):
        return self.dt.type(v)

    def set_mask(self, mask):
        m = np.asarray(mask)
        if m.dtype != bool:
            m = m.reshape(self.cell_shape) > 0.5
        self.mask = m.reshape(self.cell_shape)
        # Dilated mask: any solid (or out-of-domain) cell in the 3x3x3 block.
        pad = np.pad(self.mask, 1, constant_values=True)
        nz, ny, nx = self.cell_shape
        halo = np.zeros_like(self.mask)
        for dz in range(3):
            for dy in range(3):
                for dx in range(3):
                    halo |= pad[dz:dz + nz, dy:dy + ny, dx:dx + nx]
        self.halo = halo

    def zeros(self, shape):
        return np.zeros(shape, dtype=self.dt)

    def coords(self, shape):
        """Integer (x, y, z) coordinate arrays of a (z, y, x)-shaped grid."""
        z, y, x = np.meshgrid(*(np.arange(s) for s in shape), indexing='ij')
        return x, y, z


def _fetch(field, x, y, z):
    return field[z, y, x]


def _mix(x, y, a):
    return x * (1 - a) + y * a


def _dot(a, b):
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]


# ----------------------------------------------------------------------------
# sampling (mac_sample.glsl, closed_sample.glsl)
# ----------------------------------------------------------------------------
def sample_face(field, qx, qy, qz):
    """Clamped trilinear sample of one face grid (``mac_sample.glsl:2-19``)."""
    sz, sy, sx = field.shape
    qx = np.clip(qx, 0, sx - 1)
    qy = np.clip(qy, 0, sy - 1)
    qz = np.clip(qz, 0, sz - 1)
    bx, by, bz = np.floor(qx), np.floor(qy), np.floor(qz)
    fx, fy, fz = qx - bx, qy - by, qz - bz
    bx, by, bz = bx.astype(np.int64), by.astype(np.int64), bz.astype(np.int64)
    value = np.zeros_like(qx)
    for oz in (0, 1):
        wz = fz if oz else 1 - fz
        iz = np.minimum(bz + oz, sz - 1)
        for oy in (0, 1):
            wy = fy if oy else 1 - fy
            iy = np.minimum(by + oy, sy - 1)
            for ox in (0, 1):
                wx = fx if ox else 1 - fx
                ix = np.minimum(bx + ox, sx - 1)
                value = value + wx * wy * wz * field[iz, iy, ix]
    return value


def velocity_at(g, vel, p):
    """Staggered velocity at physical points p (``mac_sample.glsl:20-26``)."""
    qx = p[0] * g.n[0] / g.e[0]
    qy = p[1] * g.n[1] / g.e[1]
    qz = p[2] * g.n[2] / g.e[2]
    return (sample_face(vel[0], qx, qy - 0.5, qz - 0.5),
            sample_face(vel[1], qx - 0.5, qy, qz - 0.5),
            sample_face(vel[2], qx - 0.5, qy - 0.5, qz))


def _solid_cell(g, x, y, z):
    """Out-of-domain cells count as solid (``solid_boundary.glsl:2-6``)."""
    nx, ny, nz = g.shape
    out = (x < 0) | (y < 0) | (z < 0) | (x >= nx) | (y >= ny) | (z >= nz)
    res = out.copy()
    ok = ~out
    res[ok] = g.mask[z[ok], y[ok], x[ok]]
    return res


def fetch_closed(g, field, x, y, z):
    nx, ny, nz = g.shape
    return field[np.clip(z, 0, nz - 1), np.clip(y, 0, ny - 1), np.clip(x, 0, nx - 1)]


def sample_closed(g, field, qx, qy, qz):
    """Clamp-to-edge trilinear scalar sample; with colliders, renormalised over
    fluid corners (``closed_sample.glsl:7-29``)."""
    bx, by, bz = np.floor(qx), np.floor(qy), np.floor(qz)
    fx, fy, fz = qx - bx, qy - by, qz - bz
    bx, by, bz = bx.astype(np.int64), by.astype(np.int64), bz.astype(np.int64)
    if g.mask is not None:
        nx, ny, nz = g.shape
        value = np.zeros_like(qx)
        total = np.zeros_like(qx)
        for oz in (0, 1):
            wz = fz if oz else 1 - fz
            cz = np.clip(bz + oz, 0, nz - 1)
            for oy in (0, 1):
                wy = fy if oy else 1 - fy
                cy = np.clip(by + oy, 0, ny - 1)
                for ox in (0, 1):
                    wx = fx if ox else 1 - fx
                    cx = np.clip(bx + ox, 0, nx - 1)
                    fluid = ~g.mask[cz, cy, cx]
                    weight = wx * wy * wz
                    value = np.where(fluid, value + weight * field[cz, cy, cx], value)
                    total = np.where(fluid, total + weight, total)
        safe = np.where(total > 1e-8, total, 1)
        return np.where(total > 1e-8, value / safe, g.f(0))

    def fc(ox, oy, oz):
        return fetch_closed(g, field, bx + ox, by + oy, bz + oz)
    z0 = _mix(_mix(fc(0, 0, 0), fc(1, 0, 0), fx), _mix(fc(0, 1, 0), fc(1, 1, 0), fx), fy)
    z1 = _mix(_mix(fc(0, 0, 1), fc(1, 0, 1), fx), _mix(fc(0, 1, 1), fc(1, 1, 1), fx), fy)
    return _mix(z0, z1, fz)


def sample_zero(g, field, qx, qy, qz):
    """Zero-extended trilinear sample (``advect.glsl:8-23``)."""
    nx, ny, nz = g.shape
    bx, by, bz = np.floor(qx), np.floor(qy), np.floor(qz)
    fx, fy, fz = qx - bx, qy - by, qz - bz
    bx, by, bz = bx.astype(np.int64), by.astype(np.int64), bz.astype(np.int64)

    def fz_(ox, oy, oz):
        x, y, z = bx + ox, by + oy, bz + oz
        inside = (x >= 0) & (y >= 0) & (z >= 0) & (x < nx) & (y < ny) & (z < nz)
        v = field[np.clip(z, 0, nz - 1), np.clip(y, 0, ny - 1), np.clip(x, 0, nx - 1)]
        return np.where(inside, v, g.f(0))
    z0 = _mix(_mix(fz_(0, 0, 0), fz_(1, 0, 0), fx), _mix(fz_(0, 1, 0), fz_(1, 1, 0), fx), fy)
    z1 = _mix(_mix(fz_(0, 0, 1), fz_(1, 0, 1), fx), _mix(fz_(0, 1, 1), fz_(1, 1, 1), fx), fy)
    return _mix(z0, z1, fz)


# ----------------------------------------------------------------------------
# collider geometry (solid_boundary.glsl)
# ----------------------------------------------------------------------------
def solid_face(g, x, y, z, axis):
    """Face is blocked if either adjacent cell is solid (``solid_boundary.glsl:7-10``)."""
    d = [0, 0, 0]
    d[axis] = 1
    return _solid_cell(g, x, y, z) | _solid_cell(g, x - d[0], y - d[1], z - d[2])


def clip_solid_trace(g, origin, target):
    """Voxel DDA from origin to target; stops just before the first solid cell,
    at most 384 crossings (``solid_boundary.glsl:13-36``)."""
    f = g.f
    cnt = g.n
    a = [np.clip(origin[i] / g.e[i] * cnt[i], f(0.0001), cnt[i] - f(0.0001)) for i in range(3)]
    b = [np.clip(target[i] / g.e[i] * cnt[i], f(0.0001), cnt[i] - f(0.0001)) for i in range(3)]
    delta = [b[i] - a[i] for i in range(3)]
    cell = [np.floor(a[i]).astype(np.int64) for i in range(3)]
    direction = [np.sign(delta[i]).astype(np.int64) for i in range(3)]
    crossing = [np.full_like(a[0], 1e20) for _ in range(3)]
    stride = [np.full_like(a[0], 1e20) for _ in range(3)]
    for i in range(3):
        moving = np.abs(delta[i]) > 1e-10
        edge = (cell[i] + (direction[i] > 0)).astype(g.dt)
        safe_delta = np.where(moving, delta[i], 1)
        crossing[i] = np.where(moving, (edge - a[i]) / safe_delta, crossing[i])
        stride[i] = np.where(moving, 1 / np.abs(safe_delta), stride[i])
    length = np.sqrt(_dot(delta, delta))
    result = [origin[i].copy() for i in range(3)]
    done = _solid_cell(g, *cell)            # starting inside a solid: keep origin
    for _ in range(TRACE_LIMIT):
        active = ~done
        if not active.any():
            break
        cx, cy, cz = crossing
        axis = np.where((cx <= cy) & (cx <= cz), 0, np.where(cy <= cz, 1, 2))
        t = np.choose(axis, crossing)
        reached = active & (t >= 1)
        for i in range(3):
            result[i] = np.where(reached, b[i] / cnt[i] * g.e[i], result[i])
        done |= reached
        active = ~done
        for i in range(3):
            step = active & (axis == i)
            cell[i] = np.where(step, cell[i] + direction[i], cell[i])
        hit = active & _solid_cell(g, *cell)
        back = np.maximum(g.f(0), t - g.f(0.0001) / np.maximum(length, g.f(1)))
        for i in range(3):
            result[i] = np.where(hit, (a[i] + delta[i] * back) / cnt[i] * g.e[i], result[i])
        done |= hit
        active = ~done
        for i in range(3):
            step = active & (axis == i)
            crossing[i] = np.where(step, crossing[i] + stride[i], crossing[i])
    # Traces that exhausted the crossing budget keep their origin.
    return result


def solid_halo(g, p):
    """Any solid cell in the 3x3x3 block around p (``solid_boundary.glsl:39-44``)."""
    c = [np.floor(p[i] / g.e[i] * g.n[i]).astype(np.int64) for i in range(3)]
    nx, ny, nz = g.shape
    inside = (c[0] >= 0) & (c[1] >= 0) & (c[2] >= 0) & (c[0] < nx) & (c[1] < ny) & (c[2] < nz)
    res = np.ones(c[0].shape, dtype=bool)
    res[inside] = g.halo[c[2][inside], c[1][inside], c[0][inside]]
    return res


def _distance(a, b):
    d = [a[i] - b[i] for i in range(3)]
    return np.sqrt(_dot(d, d))


def safe_solid_correction(g, p, departure, midpoint, arrival):
    """``solid_boundary.glsl:45-50``."""
    ok = ~solid_halo(g, p) & ~solid_halo(g, departure) & ~solid_halo(g, arrival)
    for target in (departure, midpoint, arrival):
        ok &= _distance(clip_solid_trace(g, p, target), target) < 1e-7
    return ok


# ----------------------------------------------------------------------------
# emitters (emission_weight.glsl, source_table.glsl)
# ----------------------------------------------------------------------------
def emission_weight(g, p, center, start, radius, solid_profile):
    """Time-averaged compact-sphere weight along a swept segment
    (``emission_weight.glsl:2-29``)."""
    f = g.f
    center = [f(c) for c in center]
    start = [f(s) for s in start]
    radius = f(radius)
    seg = [center[i] - start[i] for i in range(3)]
    l2 = (seg[0] * seg[0] + seg[1] * seg[1]) + seg[2] * seg[2]
    r2 = radius * radius
    if l2 < 1e-12:
        d = [p[i] - center[i] for i in range(3)]
        dd = _dot(d, d)
        w = np.maximum(1 - dd / r2, f(0))
        if solid_profile:
            return np.where(dd < r2, f(1), f(0))
        return w * w
    lpath = np.sqrt(l2)
    axis = [seg[i] / lpath for i in range(3)]
    off = [p[i] - start[i] for i in range(3)]
    along = _dot(off, axis)
    perp = [off[i] - along * axis[i] for i in range(3)]
    a = 1 - _dot(perp, perp) / r2
    pos = a > 0
    half = radius * np.sqrt(np.where(pos, a, 0))
    lo = np.maximum(-along, -half)
    hi = np.minimum(lpath - along, half)
    good = pos & (hi > lo)
    if solid_profile:
        return np.where(good, (hi - lo) / lpath, f(0))
    sh = np.where(good, half, 1)
    u = lo / sh
    v = hi / sh
    integral = (v - u) - f(2.0 / 3.0) * (v * v * v - u * u * u) + f(0.2) * (v * v * v * v * v - u * u * u * u * u)
    val = np.clip(a * a * half / lpath * integral, f(0), f(1))
    return np.where(good, val, f(0))


def table_weight(g, p, row):
    """Weight of one 16-float source-table entry (``source_table.glsl:39-42``)."""
    return emission_weight(g, p, row[0:3], row[4:7], row[3], row[14] > 0.5)


# ----------------------------------------------------------------------------
# velocity transport (transport_face.glsl, emitting/multi_advect_velocity.glsl,
# correct_velocity_fused.glsl, mac_advect_velocity.glsl)
# ----------------------------------------------------------------------------
def _face_points(g, axis, form):
    """Face coordinates and physical positions; ``form`` selects the shader's
    expression order: 'h' -> (c+off)*h, 'en' -> (c+off)*e/n."""
    x, y, z = g.coords(g.face_shapes[axis])
    off = FACE_OFFSETS[axis]
    c = (x, y, z)
    if form == 'h':
        p = tuple((c[i].astype(g.dt) + g.f(off[i])) * g.h[i] for i in range(3))
    else:
        p = tuple((c[i].astype(g.dt) + g.f(off[i])) * g.e[i] / g.n[i] for i in range(3))
    return x, y, z, p


def _backtrace(g, vel, p, dt, clip):
    dt = g.f(dt)
    v = velocity_at(g, vel, p)
    s = g.f(0.5) * dt
    mid = tuple(p[i] - s * v[i] for i in range(3))
    if clip:
        mid = tuple(clip_solid_trace(g, p, mid))
    vm = velocity_at(g, vel, mid)
    dep = tuple(p[i] - dt * vm[i] for i in range(3))
    if clip:
        dep = tuple(clip_solid_trace(g, p, dep))
    return v, dep


def face_predictor(g, vel, axis, dt):
    """MacCormack predictor for one face component (``transport_face.glsl:1-20``)."""
    x, y, z, p = _face_points(g, axis, 'h')
    clip = g.mask is not None
    _, dep = _backtrace(g, vel, p, dt, clip)
    off = FACE_OFFSETS[axis]
    q = [dep[i] / g.h[i] - g.f(off[i]) for i in range(3)]
    value = sample_face(vel[axis], *q)
    if clip:
        value = np.where(solid_face(g, x, y, z, axis), g.f(0), value)
    return value


def advect_velocity_face(g, vel, predictor, axis, dt, corrected, blend=0.5,
                         emitter=None, sources=None):
    """Velocity transport + emitter coupling for one face component.

    ``emitting_advect_velocity.glsl:1-21`` / ``multi_advect_velocity.glsl:1-31``
    with ``correct_velocity_fused.glsl:5-27``. ``emitter`` = dict(center, start,
    radius, solid, jet, coupling) for the single-emitter form; ``sources`` = the
    packed 128-float table plus count for the multi-source form.
    """
    f = g.f
    dtf = f(dt)
    x, y, z, p = _face_points(g, axis, 'en')
    clip = g.mask is not None
    v0, dep = _backtrace(g, vel, p, dt, clip)
    off = [f(o) for o in FACE_OFFSETS[axis]]
    orig = vel[axis]
    h = g.h
    low = sample_face(orig, *[dep[i] / h[i] - off[i] for i in range(3)])
    value = low
    if corrected:
        fsz = orig.shape
        size = (fsz[2], fsz[1], fsz[0])
        lo_b = [off[i] * h[i] for i in range(3)]
        hi_b = [(f(size[i] - 1) + off[i]) * h[i] for i in range(3)]
        s = f(0.5) * dtf
        mid2 = tuple(p[i] + s * v0[i] for i in range(3))
        vm2 = velocity_at(g, vel, mid2)
        arr = tuple(p[i] + dtf * vm2[i] for i in range(3))
        ok = np.ones(x.shape, dtype=bool)
        if clip:
            ok &= safe_solid_correction(g, p, dep, mid2, arr)
        for i in range(3):
            ok &= ~((dep[i] < lo_b[i]) | (dep[i] > hi_b[i]) | (arr[i] < lo_b[i]) | (arr[i] > hi_b[i]))
        pa = sample_face(predictor, *[arr[i] / h[i] - off[i] for i in range(3)])
        val = predictor[z, y, x] + f(0.5) * (orig[z, y, x] - pa)
        q = [dep[i] / h[i] - off[i] for i in range(3)]
        b = [np.floor(q[i]).astype(np.int64) for i in range(3)]
        sx, sy, sz = size

        def fo(ox, oy, oz):
            return orig[np.clip(b[2] + oz, 0, sz - 1), np.clip(b[1] + oy, 0, sy - 1), np.clip(b[0] + ox, 0, sx - 1)]
        lo = fo(0, 0, 0)
        hi = lo
        for oz in (0, 1):
            for oy in (0, 1):
                for ox in (0, 1):
                    vv = fo(ox, oy, oz)
                    lo = np.minimum(lo, vv)
                    hi = np.maximum(hi, vv)
        clamped = np.minimum(np.maximum(val, lo), hi)
        value = np.where(ok, _mix(low, clamped, f(blend)), low)
    if emitter is not None:
        w = emission_weight(g, p, emitter['center'], emitter['start'], emitter['radius'], emitter['solid'])
        bl = 1 - np.exp(-f(emitter['coupling']) * dtf * w)
        value = _mix(value, f(emitter['jet'][axis]), bl)
    if sources is not None:
        table, count = sources
        table = [f(v) for v in table]
        total = np.zeros_like(value)
        target = np.zeros_like(value)
        for i in range(count):
            row = table[16 * i:16 * i + 16]
            rate = row[7] * table_weight(g, p, row)
            total = total + rate
            target = target + rate * row[8 + axis]
        pos = total > 0
        st = np.where(pos, total, 1)
        value = np.where(pos, _mix(value, target / st, 1 - np.exp(-dtf * total)), value)
    if clip:
        value = np.where(solid_face(g, x, y, z, axis), f(0), value)
    return value


def mac_advect_velocity_face(g, vel, axis, dt):
    """P0.3 plain semi-Lagrangian face self-advection (``mac_advect_velocity.glsl:1-10``)."""
    x, y, z, p = _face_points(g, axis, 'en')
    _, dep = _backtrace(g, vel, p, dt, False)
    return velocity_at(g, vel, dep)[axis]


def buoyancy(g, w, density, temperature, dt, lift, weight):
    """Face-averaged buoyancy on W with z-clamped extension (``buoyancy.glsl:1-14``)."""
    f = g.f
    nz = g.shape[2]
    zf = np.arange(nz + 1)
    below = np.clip(zf - 1, 0, nz - 1)
    above = np.clip(zf, 0, nz - 1)
    rho = f(0.5) * (density[below] + density[above])
    theta = f(0.5) * (temperature[below] + temperature[above])
    a = f(lift) * theta - f(weight) * rho
    return w + f(dt) * a


# ----------------------------------------------------------------------------
# scalar transport (transport_scalar.glsl, closed/multi_advect_scalar.glsl,
# correct_scalar.glsl, advect.glsl, mac_advect_density.glsl)
# ----------------------------------------------------------------------------
def _cell_points(g):
    x, y, z = g.coords(g.cell_shape)
    p = tuple((c.astype(g.dt) + g.f(0.5)) * g.h[i] for i, c in enumerate((x, y, z)))
    return x, y, z, p


def scalar_transport(g, vel, field, dt):
    """Closed semi-Lagrangian scalar pass; with -dt it is the MacCormack reverse
    (``transport_scalar.glsl:1-19``)."""
    x, y, z, p = _cell_points(g)
    clip = g.mask is not None
    _, dep = _backtrace(g, vel, p, dt, clip)
    q = [dep[i] / g.h[i] - g.f(0.5) for i in range(3)]
    value = sample_closed(g, field, *q)
    if clip:
        value = np.where(g.mask, g.f(0), value)
    return value


def _transported_scalar(g, vel, field, predictor, reverse, x, y, z, p, v0, dep, dt, corrected):
    """``correct_scalar.glsl:1-21``."""
    f = g.f
    h = g.h
    q = [dep[i] / h[i] - f(0.5) for i in range(3)]
    low = sample_closed(g, field, *q)
    if not corrected:
        return low
    dtf = f(dt)
    s = f(0.5) * dtf
    mid2 = tuple(p[i] + s * v0[i] for i in range(3))
    vm2 = velocity_at(g, vel, mid2)
    arr = tuple(p[i] + dtf * vm2[i] for i in range(3))
    ok = np.ones(x.shape, dtype=bool)
    if g.mask is not None:
        ok &= safe_solid_correction(g, p, dep, mid2, arr)
    for i in range(3):
        lo_b = f(0.5) * h[i]
        hi_b = g.e[i] - f(0.5) * h[i]
        ok &= ~((dep[i] < lo_b) | (dep[i] > hi_b) | (arr[i] < lo_b) | (arr[i] > hi_b))
    val = predictor[z, y, x] + f(0.5) * (field[z, y, x] - reverse[z, y, x])
    b = [np.floor(q[i]).astype(np.int64) for i in range(3)]
    lo = fetch_closed(g, field, *b)
    hi = lo
    for oz in (0, 1):
        for oy in (0, 1):
            for ox in (0, 1):
                vv = fetch_closed(g, field, b[0] + ox, b[1] + oy, b[2] + oz)
                lo = np.minimum(lo, vv)
                hi = np.maximum(hi, vv)
    return np.where(ok, np.minimum(np.maximum(val, lo), hi), low)


def advect_scalar(g, vel, field, predictor, reverse, dt, corrected, rate, decay, target,
                  emitter=None, sources=None, channel=0, target_heat=False):
    """Final scalar pass: corrected transport, decay and emission.

    Single emitter: ``closed_advect_scalar.glsl:1-22`` (``target`` >= 0 selects
    TARGET mode). Source table: ``multi_advect_scalar.glsl:1-29`` (channel 0
    density, 1 heat, 2 fuel). ``target_heat`` is the TARGET extension for
    temperature in the table form (the reference only has it for density).
    """
    f = g.f
    dtf = f(dt)
    x, y, z, p = _cell_points(g)
    clip = g.mask is not None
    v0, dep = _backtrace(g, vel, p, dt, clip)
    if predictor is None:
        predictor = reverse = field
    value = _transported_scalar(g, vel, field, predictor, reverse, x, y, z, p, v0, dep, dt, corrected)
    value = value * np.exp(-f(decay) * dtf)
    if sources is None:
        em = emitter
        w = emission_weight(g, p, em['center'], em['start'], em['radius'], em['solid'])
        if target >= 0:
            value = np.maximum(value, f(target) * w)
        else:
            value = value + dtf * f(rate) * w
    else:
        table, count = sources
        table = [f(v) for v in table]
        tgt = np.zeros_like(value)
        for i in range(count):
            row = table[16 * i:16 * i + 16]
            r = row[11] if channel == 0 else (row[12] if channel == 1 else row[15])
            w = table_weight(g, p, row)
            is_target = (channel == 0 and row[13] > 0.5) or (channel == 1 and target_heat)
            if is_target:
                tgt = np.maximum(tgt, r * w)
            else:
                value = value + dtf * r * w
        if channel == 0 or (channel == 1 and target_heat):
            value = np.maximum(value, tgt)
    if clip:
        value = np.where(g.mask, f(0), value)
    return value


def analytic_velocity(g, p, base, angular):
    """Prescribed rotation + translation (``advect.glsl:2-6``)."""
    f = g.f
    qx = p[0] - f(0.5) * g.e[0]
    qy = p[1] - f(0.5) * g.e[1]
    w = f(angular)
    return (f(base[0]) + (-w * qy), f(base[1]) + w * qx, f(base[2]) + qx * 0)


def advect_open(g, field, dt, base, angular, center, radius, rate, decay):
    """P0.2 open-boundary scalar advection in a prescribed flow (``advect.glsl:25-38``)."""
    f = g.f
    dtf = f(dt)
    x, y, z, p = _cell_points(g)
    v = analytic_velocity(g, p, base, angular)
    s = f(0.5) * dtf
    mid = tuple(p[i] - s * v[i] for i in range(3))
    vm = analytic_velocity(g, mid, base, angular)
    dep = tuple(p[i] - dtf * vm[i] for i in range(3))
    q = [dep[i] / g.h[i] - f(0.5) for i in range(3)]
    value = sample_zero(g, field, *q) * np.exp(-f(decay) * dtf)
    off = [p[i] - f(center[i]) for i in range(3)]
    w = np.maximum(1 - _dot(off, off) / (f(radius) * f(radius)), f(0))
    return value + dtf * f(rate) * w * w


def mac_advect_density(g, vel, field, dt, center, radius, rate, decay):
    """P0.3 open-boundary scalar advection by MAC velocity (``mac_advect_density.glsl:18-31``)."""
    f = g.f
    dtf = f(dt)
    x, y, z, p = _cell_points(g)
    _, dep = _backtrace(g, vel, p, dt, False)
    q = [dep[i] / g.h[i] - f(0.5) for i in range(3)]
    value = sample_zero(g, field, *q) * np.exp(-f(decay) * dtf)
    off = [p[i] - f(center[i]) for i in range(3)]
    w = np.maximum(1 - _dot(off, off) / (f(radius) * f(radius)), f(0))
    return value + dtf * f(rate) * w * w


def seed_scalar(g, center, radius, scale=1.0):
    """Soft-sphere seed (``seed.glsl``, ``temperature_seed.glsl``)."""
    f = g.f
    x, y, z = g.coords(g.cell_shape)
    p = tuple((c.astype(g.dt) + f(0.5)) * g.e[i] / g.n[i] for i, c in enumerate((x, y, z)))
    off = [p[i] - f(center[i]) for i in range(3)]
    w = np.maximum(1 - _dot(off, off) / (f(radius) * f(radius)), f(0))
    if scale == 1.0:
        return w * w
    return f(scale) * w * w


def seed_faces(g, base, angular):
    """Analytic rotation seed for the faces (``mac_seed.glsl``)."""
    out = []
    for axis in range(3):
        x, y, z, p = _face_points(g, axis, 'en')
        out.append(analytic_velocity(g, p, base, angular)[axis])
    return tuple(out)


# ----------------------------------------------------------------------------
# projection (pressure_*.glsl, backend/pressure.py)
# ----------------------------------------------------------------------------
def walls(g, vel):
    """Zero normal velocity on box walls and solid faces (``pressure_walls.glsl``)."""
    out = []
    for axis in range(3):
        x, y, z = g.coords(g.face_shapes[axis])
        c = (x, y, z)
        n = g.face_shapes[axis][2 - axis]
        wall = (c[axis] == 0) | (c[axis] == n - 1)
        if g.mask is not None:
            wall |= solid_face(g, x, y, z, axis)
        # moving colliders: walls take the wall velocity (FLUXFX_MOVING_COLLIDERS, pressure_walls.glsl:10-12)
        wall_value = g.f(0) if g.boundary is None else g.boundary[axis]
        out.append(np.where(wall, wall_value, vel[axis]))
    return tuple(out)


def divergence(g, vel):
    """Cell divergence, 0 in solids (``pressure_divergence.glsl``)."""
    U, V, W = vel
    d = (U[:, :, 1:] - U[:, :, :-1]) * g.inv[0] + (V[:, 1:, :] - V[:, :-1, :]) * g.inv[1] \
        + (W[1:, :, :] - W[:-1, :, :]) * g.inv[2]
    if g.mask is not None:
        d = np.where(g.mask, g.f(0), d)
    return d


def _shift(p, axis, sign):
    """Neighbour values along ``axis`` (array axis order z, y, x) and a validity mask."""
    ax = 2 - axis
    n = p.shape[ax]
    idx = np.arange(n) + sign
    valid = (idx >= 0) & (idx < n)
    taken = np.take(p, np.clip(idx, 0, n - 1), axis=ax)
    shape = [1, 1, 1]
    shape[ax] = n
    return taken, np.broadcast_to(valid.reshape(shape), p.shape)


def jacobi(g, p, rhs, dt, omega, inv=None, mask=None):
    """One weighted-Jacobi sweep on the Neumann (optionally masked) 7-point
    Laplacian (``pressure_jacobi.glsl:1-34``)."""
    f = g.f
    inv = inv or g.inv
    neighbor = np.zeros_like(p)
    diag = np.zeros_like(p)
    for axis in range(3):
        w = inv[axis] * inv[axis]
        for sign in (-1, 1):
            val, ok = _shift(p, axis, sign)
            if mask is not None:
                sm, _ = _shift(mask, axis, sign)
                ok = ok & ~sm
            neighbor = np.where(ok, neighbor + w * val, neighbor)
            diag = np.where(ok, diag + w, diag)
    safe = np.where(diag == 0, 1, diag)
    cand = (neighbor - rhs / f(dt)) / safe
    out = _mix(p, cand, f(omega))
    out = np.where(diag == 0, f(0), out)
    if mask is not None:
        out = np.where(mask, f(0), out)
    return out


def residual(g, p, rhs, dt, inv):
    """r = rhs/dt - L p (``mg_residual.glsl``)."""
    lap = np.zeros_like(p)
    for axis in range(3):
        w = inv[axis] * inv[axis]
        for sign in (-1, 1):
            val, ok = _shift(p, axis, sign)
            lap = np.where(ok, lap + w * (val - p), lap)
    return rhs / g.f(dt) - lap


def restrict(fine):
    """2x2x2 average in z, y, x order (``mg_restrict.glsl``)."""
    nz, ny, nx = fine.shape
    v = np.zeros((nz // 2, ny // 2, nx // 2), dtype=fine.dtype)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                v = v + fine[dz::2, dy::2, dx::2]
    return v / fine.dtype.type(8)


def prolong(g, p, coarse):
    """p + cell-centred trilinear interpolation of ``coarse`` (``mg_prolong.glsl``)."""
    f = g.f
    nz, ny, nx = p.shape
    cz, cy, cx = coarse.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing='ij')
    q = [(c.astype(p.dtype) + f(0.5)) * f(0.5) - f(0.5) for c in (x, y, z)]
    b = [np.floor(qq) for qq in q]
    fr = [q[i] - b[i] for i in range(3)]
    b = [bb.astype(np.int64) for bb in b]
    value = np.zeros_like(p)
    for oz in (0, 1):
        wz = fr[2] if oz else 1 - fr[2]
        iz = np.clip(b[2] + oz, 0, cz - 1)
        for oy in (0, 1):
            wy = fr[1] if oy else 1 - fr[1]
            iy = np.clip(b[1] + oy, 0, cy - 1)
            for ox in (0, 1):
                wx = fr[0] if ox else 1 - fr[0]
                ix = np.clip(b[0] + ox, 0, cx - 1)
                value = value + wx * wy * wz * coarse[iz, iy, ix]
    return p + value


def coarse_direct(g, rhs, dt, inverse):
    """Dense pseudoinverse mat-vec (``coarse_pressure.glsl``); FP64 accumulation."""
    r = rhs.astype(np.float64).ravel()
    return ((np.asarray(inverse, dtype=np.float64).reshape(r.size, r.size) @ r) / float(dt)).astype(g.dt).reshape(rhs.shape)


def gradient(g, bounded, p, dt):
    """u - dt grad p on open faces, 0 on walls and solid faces (``pressure_gradient.glsl``)."""
    f = g.f
    out = []
    dtf = f(dt)
    for axis in range(3):
        x, y, z = g.coords(g.face_shapes[axis])
        c = [x, y, z]
        n = g.face_shapes[axis][2 - axis]
        opened = (c[axis] > 0) & (c[axis] < n - 1)
        if g.mask is not None:
            opened &= ~solid_face(g, x, y, z, axis)
        nx, ny, nz = g.shape
        hi = [np.clip(x, 0, nx - 1), np.clip(y, 0, ny - 1), np.clip(z, 0, nz - 1)]
        lo = list(hi)
        lo[axis] = np.clip(c[axis] - 1, 0, g.shape[axis] - 1)
        grad = (p[hi[2], hi[1], hi[0]] - p[lo[2], lo[1], lo[0]]) * g.inv[axis]
        # moving colliders: closed faces take the wall velocity (pressure_gradient.glsl:11-13)
        closed = f(0) if g.boundary is None else g.boundary[axis]
        out.append(np.where(opened, bounded[axis] - dtf * grad, closed))
    return tuple(out)


def max_abs(field):
    """Max |v| with NaN/Inf mapped to 3.4e38 (``max_reduce.glsl``)."""
    a = np.abs(field.astype(np.float64))
    a = np.where(np.isfinite(a), a, HUGE)
    return float(a.max()) if a.size else 0.0


def hierarchy_shapes(shape, max_levels=0):
    """Halve while every axis is even and the smallest is >= 8 (``backend/multigrid.py:6-11``)."""
    out = [tuple(shape)]
    while min(shape) >= 8 and all(n % 2 == 0 for n in shape):
        if max_levels and len(out) >= max_levels:
            break
        shape = tuple(n // 2 for n in shape)
        out.append(shape)
    return out


class GeometricMG:
    """Plain V-cycle (``backend/multigrid.py:20-95``)."""

    def __init__(self, g, pre=3, post=3, max_levels=0, coarse_inverse=None, coarse_solver='DIRECT'):
        self.g = g
        self.pre, self.post = pre, post
        self.shapes = hierarchy_shapes(g.shape, max_levels)
        self.invs = [tuple(g.f(n / e) for n, e in zip(s, g.extent64)) for s in self.shapes]
        self.coarse_inverse = coarse_inverse
        self.coarse_solver = coarse_solver
        self.sweeps = 0

    def smooth(self, level, p, rhs, dt, count):
        for _ in range(count):
            p = jacobi(self.g, p, rhs, dt, 2.0 / 3.0, inv=self.invs[level])
            self.sweeps += 1
        return p

    def cycle(self, level, p, rhs, dt):
        g = self.g
        if level == len(self.shapes) - 1:
            if self.coarse_inverse is not None and self.coarse_solver == 'DIRECT':
                return coarse_direct(g, rhs, dt, self.coarse_inverse)
            return self.smooth(level, p, rhs, dt, 80)
        p = self.smooth(level, p, rhs, dt, self.pre)
        r = residual(g, p, rhs, dt, self.invs[level])
        crhs = restrict(r)
        cp = self.cycle(level + 1, np.zeros_like(crhs), crhs, 1.0)
        p = prolong(g, p, cp)
        return self.smooth(level, p, rhs, dt, self.post)


# ----------------------------------------------------------------------------
# collider multigrid (physics/solid_hierarchy.py, backend/solid_multigrid.py,
# solid_mg_*.glsl)
# ----------------------------------------------------------------------------
def level0_edges(shape, extent, mask):
    """Per-cell (+x, +y, +z, active) conductances (``solid_hierarchy.py:11-25``)."""
    nx, ny, nz = shape
    fluid = ~mask.reshape(nz, ny, nx)
    edges = np.zeros((nz, ny, nx, 4), dtype=np.float32)
    edges[..., 3] = fluid
    for a in range(3):
        w = np.float32((shape[a] / extent[a]) ** 2)
        ax = 2 - a
        nb, ok = _shift(fluid, a, 1)
        edges[..., a] = np.where(fluid & nb & ok, w, np.float32(0))
    return edges


def coarsen_edges(edges):
    """One Galerkin aggregation level; None when any aggregate would join
    disconnected children (``solid_hierarchy.py:27-53``)."""
    nz, ny, nx, _ = edges.shape
    cz, cy, cx = nz // 2, ny // 2, nx // 2
    child = {}
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                child[dx + 2 * dy + 4 * dz] = edges[dz::2, dy::2, dx::2].astype(np.float64)
    active = np.stack([child[j][..., 3] > 0 for j in range(8)], axis=-1)   # (cz,cy,cx,8)
    # Flood fill from the lowest active child over fine edges inside the aggregate.
    anyact = active.any(-1)
    first = np.argmax(active, axis=-1)
    seen = np.zeros_like(active)
    np.put_along_axis(seen, first[..., None], anyact[..., None], axis=-1)
    for _ in range(8):
        new = seen.copy()
        for j in range(8):
            for a in range(3):
                k = j ^ (1 << a)
                lower = k if j & (1 << a) else j
                link = child[lower][..., a] > 0
                new[..., k] |= seen[..., j] & active[..., k] & link
        if (new == seen).all():
            break
        seen = new
    if (seen != active).any():
        return None
    coarse = np.zeros((cz, cy, cx, 4), dtype=np.float32)
    coarse[..., 3] = anyact
    for a in range(3):
        total = np.zeros((cz, cy, cx), dtype=np.float64)
        for j in range(8):
            if j & (1 << a):
                total = total + child[j][..., a]
        coarse[..., a] = (total / 8).astype(np.float32)
    return coarse


def build_hierarchy(shape, extent, mask, max_levels=0):
    """List of (shape, edges (nz,ny,nx,4) float32) from fine to coarse."""
    edges = level0_edges(shape, extent, np.asarray(mask).reshape(shape[2], shape[1], shape[0]) > 0.5
                         if np.asarray(mask).dtype != bool else np.asarray(mask))
    levels = [(tuple(shape), edges)]
    while min(shape) >= 8 and all(n % 2 == 0 for n in shape):
        if max_levels and len(levels) >= max_levels:
            break
        coarse = coarsen_edges(edges)
        if coarse is None:
            break
        shape = tuple(n // 2 for n in shape)
        edges = coarse
        levels.append((shape, edges))
    return levels


def graph_matrix(shape, edges):
    n = prod(shape)
    e = edges.reshape(n, 4).astype(np.float64)
    m = np.zeros((n, n))
    strides = (1, shape[0], shape[0] * shape[1])
    for i in range(n):
        for a, s in enumerate(strides):
            w = e[i, a]
            if w:
                j = i + s
                m[i, i] -= w
                m[j, j] -= w
                m[i, j] += w
                m[j, i] += w
    return m


def graph_inverse(shape, edges):
    """FP64 pseudoinverse of the coarsest graph Laplacian (``solid_hierarchy.py:57-75``)."""
    return np.linalg.pinv(graph_matrix(shape, edges), rcond=1e-12, hermitian=True)


def graph_terms(p, edges):
    """Diagonal and neighbour sums of the graph Laplacian (``solid_mg_operator.glsl``)."""
    nz, ny, nx = p.shape
    diag = np.zeros_like(p)
    nb = np.zeros_like(p)
    for a in range(3):
        ax = 2 - a
        w_here = edges[..., a].astype(p.dtype)
        # lower neighbour: weight stored at c - o
        w_lo, ok_lo = _shift(w_here, a, -1)
        p_lo, _ = _shift(p, a, -1)
        diag = np.where(ok_lo, diag + w_lo, diag)
        nb = np.where(ok_lo, nb + w_lo * p_lo, nb)
        p_hi, ok_hi = _shift(p, a, 1)
        diag = np.where(ok_hi, diag + w_here, diag)
        nb = np.where(ok_hi, nb + w_here * p_hi, nb)
    return diag, nb


def graph_smooth(p, rhs, edges):
    """``solid_mg_smooth.glsl``."""
    diag, nb = graph_terms(p, edges)
    f = p.dtype.type
    safe = np.where(diag > 0, diag, 1)
    return np.where(diag > 0, _mix(p, (nb - rhs) / safe, f(2.0 / 3.0)), f(0))


def graph_residual(p, rhs, edges):
    """``solid_mg_residual.glsl``."""
    diag, nb = graph_terms(p, edges)
    return np.where(diag > 0, rhs - nb + diag * p, p.dtype.type(0))


def graph_prolong(p, coarse, edges, alpha=1.0):
    """Piecewise-constant injection on active cells (``solid_mg_prolong.glsl``);
    ``alpha`` over-corrects (an extension: p + alpha * coarse; 1 is the reference)."""
    up = coarse.repeat(2, 0).repeat(2, 1).repeat(2, 2)[:p.shape[0], :p.shape[1], :p.shape[2]]
    if alpha != 1.0:
        up = (p.dtype.type(alpha) * up).astype(p.dtype)
    return np.where(edges[..., 3] > 0, p + up, p.dtype.type(0))


class SolidMG:
    """Aggregation V-cycle (``backend/solid_multigrid.py:7-76``)."""

    def __init__(self, levels, pre=4, post=4, coarse_solver='DIRECT', dtype=np.float32, alpha=1.0, coarse_sweeps=0):
        self.levels = levels
        self.pre, self.post = pre, post
        # the coarse-sweeps extension: N pre- and post-sweeps below level 0 (0: the same as level 0)
        self.cpre, self.cpost = (coarse_sweeps, coarse_sweeps) if coarse_sweeps else (pre, post)
        self.alpha = alpha
        self.dtype = np.dtype(dtype)
        shape, edges = levels[-1]
        self.inverse = None
        if prod(shape) <= 256 and coarse_solver == 'DIRECT' and len(levels) > 1:
            self.inverse = graph_inverse(shape, edges)
        self.sweeps = 0

    def smooth(self, level, p, rhs, count):
        edges = self.levels[level][1]
        for _ in range(count):
            p = graph_smooth(p, rhs, edges)
            self.sweeps += 1
        return p

    def cycle(self, level, p, rhs):
        if level == len(self.levels) - 1:
            if self.inverse is not None:
                r = rhs.astype(np.float64).ravel()
                return (self.inverse @ r).astype(self.dtype).reshape(rhs.shape)
            return self.smooth(level, p, rhs, 80)
        edges = self.levels[level][1]
        pre, post = (self.pre, self.post) if level == 0 else (self.cpre, self.cpost)
        p = self.smooth(level, p, rhs, pre)
        r = graph_residual(p, rhs, edges)
        crhs = restrict(r)
        cp = self.cycle(level + 1, np.zeros_like(crhs), crhs)
        p = graph_prolong(p, cp, edges, self.alpha)
        return self.smooth(level, p, rhs, post)


def raster_mask(g, colliders):
    """Union of sphere/box colliders at cell centres, evaluated in FP64 in the
    order of ``physics/collision.py:23-37`` (the reference's GPU kernel
    ``solid_mask.glsl`` runs the same test in FP32)."""
    nx, ny, nz = g.shape
    h = tuple(e / n for e, n in zip(g.extent64, g.shape))
    z, y, x = np.meshgrid(*(np.arange(s) for s in (nz, ny, nx)), indexing='ij')
    px, py, pz = ((x + .5) * h[0], (y + .5) * h[1], (z + .5) * h[2])
    solid = np.zeros((nz, ny, nx), dtype=bool)
    for shape, rows in colliders:
        q = [((0.0 + r[0] * px) + r[1] * py) + r[2] * pz + r[3] for r in rows]
        if shape == 'SPHERE':
            inside = ((0.0 + q[0] * q[0]) + q[1] * q[1]) + q[2] * q[2] <= 1
        else:
            inside = np.maximum(np.maximum(np.abs(q[0]), np.abs(q[1])), np.abs(q[2])) <= 1
        solid |= inside
    return solid
