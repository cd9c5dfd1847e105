"""Sparse brick path: a brick pool and the pressure projection on active bricks.

Counterpart of FluxFX's native sparse prototype (``FluxFX_Source/native/
bricks.hpp:14-94`` -- the topology -- and ``projection.mm:15-120`` /
``compare_projection`` -- the sparse projection checked against a dense twin):

* ``BrickPool`` -- fixed-capacity brick topology (host, ``ffx_bricks_*``):
  activate / deactivate / lookup / neighbours / atomic box activation, slots
  reused in LIFO order, metadata reserved at creation.
* ``SparseProjection`` -- the projection of a velocity seeded on a solve region
  (the whole grid, a central box or two boxes) with weighted Jacobi sweeps or
  V-cycles, on a level hierarchy stored either as active bricks only (a brick
  is active when any cell within one cell of the region lies in it) or as
  dense arrays. The kernels (``ffx_sparse_*``) do the same arithmetic in both
  layouts, so ``compare_projection`` finds them equal on the region while the
  sparse layout holds only the bricks the region touches.

Units are cells and the pressure is the impulse, as in the prototype.
"""
import ctypes as C
from math import pi

import numpy as np
import torch

from .. import _native as N


class BrickPool:
    """Brick coordinates -> storage slots (``ffx_bricks_*``, host memory)."""

    def __init__(self, capacity):
        self.lib = N.load()
        self._pool = C.c_void_p()
        N.check(self.lib.ffx_bricks_create(int(capacity), C.byref(self._pool)))

    def _slot(self, fn, coord):
        out = C.c_int32()
        N.check(getattr(self.lib, fn)(self._pool, *[int(v) for v in coord], C.byref(out)))
        return out.value

    def activate(self, coord):
        return self._slot('ffx_bricks_activate', coord)

    def deactivate(self, coord):
        return bool(self._slot('ffx_bricks_deactivate', coord))

    def lookup(self, coord):
        return self._slot('ffx_bricks_lookup', coord)

    def neighbors(self, coord):
        out = (C.c_int32 * 6)()
        N.check(self.lib.ffx_bricks_neighbors(self._pool, *[int(v) for v in coord], out))
        return list(out)

    def activate_box(self, lo, extent):
        N.check(self.lib.ffx_bricks_activate_box(self._pool, (C.c_int32 * 3)(*lo), (C.c_int32 * 3)(*extent)))

    def stats(self):
        st = N.FfxBrickStats()
        N.check(self.lib.ffx_bricks_stats(self._pool, C.byref(st)))
        return {'capacity': st.capacity, 'active': st.active, 'metadata_bytes': st.metadata_bytes}

    def active(self):
        """(active slots in order, coordinates of every slot as an (capacity, 3) array)."""
        cap = self.stats()['capacity']
        slots = (C.c_int32 * cap)()
        coords = (C.c_int32 * (3 * cap))()
        N.check(self.lib.ffx_bricks_active(self._pool, slots, coords, cap))
        n = self.stats()['active']
        return list(slots[:n]), np.frombuffer(coords, dtype=np.int32).reshape(cap, 3).copy()

    def close(self):
        if self._pool:
            self.lib.ffx_bricks_destroy(self._pool)
            self._pool = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Arena:
    """Suballocator of one buffer (``ffx_arena_*``, host bookkeeping): offsets
    of 256-byte-aligned spans, first fit, merged on release."""

    def __init__(self, capacity):
        self.lib = N.load()
        self._arena = C.c_void_p()
        N.check(self.lib.ffx_arena_create(int(capacity), C.byref(self._arena)))

    def allocate(self, nbytes):
        out = C.c_uint64()
        N.check(self.lib.ffx_arena_allocate(self._arena, int(nbytes), C.byref(out)))
        return out.value

    def get(self, handle):
        """(offset, bytes, requested) of a live span."""
        o, b, r = C.c_uint64(), C.c_uint64(), C.c_uint64()
        N.check(self.lib.ffx_arena_get(self._arena, int(handle), C.byref(o), C.byref(b), C.byref(r)))
        return o.value, b.value, r.value

    def release(self, handle):
        N.check(self.lib.ffx_arena_release(self._arena, int(handle)))

    def stats(self):
        st = N.FfxArenaStats()
        N.check(self.lib.ffx_arena_stats(self._arena, C.byref(st)))
        return {k: getattr(st, k) for k, _ in N.FfxArenaStats._fields_}

    def close(self):
        if self._arena:
            self.lib.ffx_arena_destroy(self._arena)
            self._arena = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_mask(n, mode):
    """The solve region as an (n, n, n) boolean array, z-major."""
    r = np.arange(n)
    def box(lo, hi):
        m = (r >= lo) & (r < hi)
        return m[:, None, None] & m[None, :, None] & m[None, None, :]
    if mode == 1:
        return box(n // 4, 3 * n // 4)
    if mode == 2:
        return box(n // 8, 3 * n // 8) | box(5 * n // 8, 7 * n // 8)
    return np.ones((n, n, n), bool)


def seed_faces(n, mode):
    """A seeded divergent velocity on the faces beside the solve region, zero on
    the domain walls and elsewhere: (u, v, w) with shapes (n, n, n+1),
    (n, n+1, n), (n+1, n, n), z-major."""
    solve = solve_mask(n, mode)
    faces = []
    for a in range(3):
        shape = [n, n, n]
        shape[2 - a] += 1
        idx = np.indices(shape, dtype=np.float64)      # (z, y, x)
        pos = [idx[2] + 0.5, idx[1] + 0.5, idx[0] + 0.5]
        pos[a] -= 0.5
        value = 0.3 * np.sin(2 * pi * (a + 1) * pos[a] / n) * np.cos(2 * pi * pos[(a + 1) % 3] / n) + \
            0.1 * np.sin(4 * pi * pos[(a + 2) % 3] / n)
        # faces with a solve cell on either side, inside the domain
        pad = np.zeros([s + 2 for s in (n, n, n)], bool)
        pad[1:-1, 1:-1, 1:-1] = solve
        hi = [slice(1, s + 1) for s in shape]           # cell c (upper side of the face)
        lo = [slice(1, s + 1) for s in shape]
        lo[2 - a] = slice(0, shape[2 - a])              # cell c - e_a
        beside = pad[tuple(hi)] | pad[tuple(lo)]
        interior = np.ones(shape, bool)
        sl = [slice(None)] * 3
        sl[2 - a] = 0
        interior[tuple(sl)] = False
        sl[2 - a] = shape[2 - a] - 1
        interior[tuple(sl)] = False
        faces.append(np.where(beside & interior, value, 0.0).astype(np.float32))
    return faces


class _Level:
    def __init__(self, n, side, mode, sparse, device):
        self.n, self.side, self.mode, self.sparse = n, side, mode, sparse
        self.device = device
        if sparse:
            g = n // side
            solve = solve_mask(n, mode)
            # a brick is active when a cell within one cell of the region lies in it
            grown = solve.copy()
            for ax in range(3):
                grown |= np.roll(solve, 1, ax) & (np.arange(n) > 0).reshape([-1 if k == ax else 1 for k in range(3)])
                grown |= np.roll(solve, -1, ax) & (np.arange(n) < n - 1).reshape(
                    [-1 if k == ax else 1 for k in range(3)])
            bricks = grown.reshape(g, side, g, side, g, side).any(axis=(1, 3, 5))   # (bz, by, bx)
            self.pool = BrickPool(max(1, int(bricks.sum())))       # storage for the active bricks only
            for bz, by, bx in zip(*np.nonzero(bricks)):
                self.pool.activate((bx, by, bz))
            slots, coords = self.pool.active()
            self.count = len(slots)
            grid_map = np.full(g ** 3, -1, np.int32)
            for s in slots:
                x, y, z = coords[s]
                grid_map[(z * g + y) * g + x] = s
            self.map = torch.as_tensor(grid_map).to(device)
            self.active = torch.as_tensor(np.array(slots, np.int32)).to(device)
            self.coords = torch.as_tensor(coords.reshape(-1)).to(device)
            self.cells = self.pool.stats()['capacity'] * side ** 3
            self.faces = self.cells
        else:
            self.count = 1
            self.map = self.active = self.coords = None
            self.cells = n ** 3
            self.faces = (n + 1) * n * n
        self.struct = N.FfxSparseLevel(n, side, mode, int(sparse),
                                       self.map.data_ptr() if sparse else None,
                                       self.active.data_ptr() if sparse else None,
                                       self.coords.data_ptr() if sparse else None, self.count)
        zeros = lambda k: torch.zeros(k, dtype=torch.float32, device=device)
        self.q, self.spare, self.rhs, self.res = zeros(self.cells), zeros(self.cells), zeros(self.cells), zeros(self.cells)

    @property
    def bytes(self):
        b = 4 * (4 * self.cells)
        if self.sparse:
            b += self.map.numel() * 4 + self.active.numel() * 4 + self.coords.numel() * 4
        return b

    def cell_index(self):
        """Storage index of every cell (z-major (n, n, n) array, -1 where not stored)."""
        n, s = self.n, self.side
        idx = np.indices((n, n, n))
        z, y, x = idx[0], idx[1], idx[2]
        if not self.sparse:
            return (z * n + y) * n + x
        g = n // s
        slot = self.map.cpu().numpy()[((z // s) * g + y // s) * g + x // s]
        local = ((z % s) * s + y % s) * s + x % s
        return np.where(slot >= 0, slot * s ** 3 + local, -1)

    def face_index(self, a):
        n, s = self.n, self.side
        shape = [n, n, n]
        shape[2 - a] += 1
        idx = np.indices(shape)
        z, y, x = idx[0], idx[1], idx[2]
        if not self.sparse:
            dx, dy = n + (a == 0), n + (a == 1)
            return (z * dy + y) * dx + x
        inside = (x < n) & (y < n) & (z < n)
        g = n // s
        xc, yc, zc = np.minimum(x, n - 1), np.minimum(y, n - 1), np.minimum(z, n - 1)
        slot = self.map.cpu().numpy()[((zc // s) * g + yc // s) * g + xc // s]
        local = ((zc % s) * s + yc % s) * s + xc % s
        return np.where(inside & (slot >= 0), slot * s ** 3 + local, -1)

    def gather(self, field):
        """A stored cell field as a dense (n, n, n) array (0 where not stored)."""
        idx = self.cell_index()
        host = field.cpu().numpy()
        return np.where(idx >= 0, host[np.maximum(idx, 0)], 0.0).astype(np.float32)


class SparseProjection:
    """The projection of ``seed_faces(n, mode)`` on a sparse or dense hierarchy."""

    def __init__(self, n, side=8, mode=1, sparse=True, device=None, cycles=0):
        if n not in (32, 64, 128, 256) or side not in (8, 16) or mode not in (0, 1, 2):
            raise ValueError('SparseProjection: n 32/64/128/256, side 8/16, mode 0..2')
        self.device = device or torch.device('cuda')
        self.lib = N.load()
        self.stream = torch.cuda.current_stream(self.device)
        self.levels = [_Level(n, side, mode, sparse, self.device)]
        if cycles:
            cn = n // 2
            while cn >= 8:
                self.levels.append(_Level(cn, min(side, cn), mode, sparse, self.device))
                cn //= 2
        top = self.levels[0]
        self.u = torch.zeros(3 * top.faces, dtype=torch.float32, device=self.device)
        self.out = torch.zeros_like(self.u)
        self.after = torch.zeros(top.cells, dtype=torch.float32, device=self.device)
        host = np.zeros(3 * top.faces, np.float32)
        for a, f in enumerate(seed_faces(n, mode)):
            idx = top.face_index(a)
            keep = idx >= 0
            host[a * top.faces + idx[keep]] = f[keep]
        self.u.copy_(torch.as_tensor(host))
        self.seeded = seed_faces(n, mode)

    @property
    def bytes(self):
        return sum(l.bytes for l in self.levels) + 2 * 3 * self.levels[0].faces * 4 + self.levels[0].cells * 4

    def _call(self, name, *args):
        N.check(getattr(self.lib, name)(*args, C.c_void_p(self.stream.cuda_stream)))

    def _smooth(self, lv, count):
        for _ in range(count):
            self._call('ffx_sparse_jacobi', C.byref(lv.struct), C.c_void_p(lv.q.data_ptr()),
                       C.c_void_p(lv.rhs.data_ptr()), C.c_void_p(lv.spare.data_ptr()))
            lv.q, lv.spare = lv.spare, lv.q

    def _cycle(self, k):
        lv = self.levels[k]
        if k == len(self.levels) - 1:
            self._smooth(lv, 128)
            return
        self._smooth(lv, 4)
        self._call('ffx_sparse_residual', C.byref(lv.struct), C.c_void_p(lv.q.data_ptr()),
                   C.c_void_p(lv.rhs.data_ptr()), C.c_void_p(lv.res.data_ptr()))
        coarse = self.levels[k + 1]
        coarse.q.zero_()
        self._call('ffx_sparse_restrict', C.byref(lv.struct), C.c_void_p(lv.res.data_ptr()), C.byref(coarse.struct),
                   C.c_void_p(coarse.rhs.data_ptr()))
        self._cycle(k + 1)
        self._call('ffx_sparse_prolong', C.byref(coarse.struct), C.c_void_p(coarse.q.data_ptr()),
                   C.byref(lv.struct), C.c_void_p(lv.q.data_ptr()))
        self._smooth(lv, 4)

    def run(self, iterations=0, cycles=0):
        """Divergence, `cycles` V-cycles or `iterations` Jacobi sweeps, gradient,
        divergence after; returns the device time in ms."""
        top = self.levels[0]
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            top.q.zero_()
            start.record(self.stream)
            self._call('ffx_sparse_divergence', C.byref(top.struct), C.c_void_p(self.u.data_ptr()), top.faces,
                       C.c_void_p(top.rhs.data_ptr()))
            if cycles:
                for _ in range(cycles):
                    self._cycle(0)
            else:
                self._smooth(top, iterations)
            self._call('ffx_sparse_gradient', C.byref(top.struct), C.c_void_p(self.u.data_ptr()),
                       C.c_void_p(top.q.data_ptr()), top.faces, C.c_void_p(self.out.data_ptr()))
            self._call('ffx_sparse_divergence', C.byref(top.struct), C.c_void_p(self.out.data_ptr()), top.faces,
                       C.c_void_p(self.after.data_ptr()))
            end.record(self.stream)
        end.synchronize()
        return start.elapsed_time(end)

    def fields(self):
        """(pressure, divergence before, divergence after, faces after) as dense arrays."""
        top = self.levels[0]
        host = self.out.cpu().numpy()
        faces = []
        for a in range(3):
            idx = top.face_index(a)
            faces.append(np.where(idx >= 0, host[a * top.faces + np.maximum(idx, 0)], 0.0).astype(np.float32))
        return top.gather(top.q), top.gather(top.rhs), top.gather(self.after), faces


def compare_projection(n, side=8, iterations=64, mode=1, cycles=0, device=None):
    """The sparse and the dense projection of the same seeded velocity
    (``projection.mm`` ``compare_projection``): errors between them on the solve
    region, divergence before and after, storage of each."""
    sp = SparseProjection(n, side, mode, True, device, cycles)
    de = SparseProjection(n, side, mode, False, device, cycles)
    sp_ms = sp.run(iterations, cycles)
    de_ms = de.run(iterations, cycles)
    ps, bs, as_, fs = sp.fields()
    pd, bd, ad, fd = de.fields()
    solve = solve_mask(n, mode)
    rms = lambda x: float(np.sqrt(np.mean(np.square(x[solve], dtype=np.float64))))
    out = {'resolution': n, 'side': side, 'mode': mode, 'iterations': iterations, 'cycles': cycles,
           'active_bricks': sp.levels[0].count, 'levels': len(sp.levels), 'solve_cells': int(solve.sum()),
           'pressure_error': float(np.abs(ps - pd)[solve].max()),
           'divergence_error': float(np.abs(as_ - ad)[solve].max()),
           'before_error': float(np.abs(bs - bd)[solve].max()),
           'face_error': max(float(np.abs(a - b).max()) for a, b in zip(fs, fd)),
           'before_rms': rms(bd), 'after_rms': rms(ad),
           'sparse_bytes': sp.bytes, 'dense_bytes': de.bytes, 'sparse_ms': sp_ms, 'dense_ms': de_ms}
    return out
