"""Topology-preserving aggregation V-cycles for static voxel colliders.

Drop-in for FluxFX ``fluxfx/backend/solid_multigrid.py:7-93``. The Galerkin
hierarchy of ``fluxfx/physics/solid_hierarchy.py:11-54`` is built on the device
(``ffx_graph_coarsen`` per level, one flag readback per level at construction);
level 0 stores one link byte per cell (``ffx_graph_links``) instead of
conductances. The coarsest
level (<= 256 cells) is solved with an FP64 graph pseudoinverse. Residual +
restriction and prolongation + first post-smoothing sweep are fused passes
with results identical to the separate passes.
"""
import ctypes as C
from math import prod

import numpy as np
import torch

from .. import _native as N
from .collision import SolidPressureProjector
from .device import KernelHandle, ptr

DIRECT_LIMIT = 256
TAIL_CELLS = 512   # coarse levels at most this size run in one single-block launch


class KernelTimer:
    """CUDA events around every level-0 smoothing launch, on the solver's stream.

    Set ``projector.timer = KernelTimer(stream)`` to time the dominant kernel of
    the solve while the step runs; ``average_ms()`` synchronises and returns the
    mean launch duration."""

    def __init__(self, stream):
        self.stream = stream
        self.pairs = []

    def begin(self):
        e = torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        return e

    def end(self, start):
        e = torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        self.pairs.append((start, e))

    @property
    def count(self):
        return len(self.pairs)

    def average_ms(self):
        if not self.pairs:
            return None
        self.pairs[-1][1].synchronize()
        return sum(a.elapsed_time(b) for a, b in self.pairs) / len(self.pairs)


def graph_pseudoinverse(shape, edges):
    """FP64 pseudoinverse of the graph Laplacian with conductances ``edges``
    ((nz, ny, nx, 4) host array), as ``solid_hierarchy.graph_inverse`` forms it."""
    n = prod(shape)
    if n > DIRECT_LIMIT:
        raise ValueError('Direct coarse solve is limited to 256 cells')
    e = np.asarray(edges, dtype=np.float64).reshape(n, 4)
    m = np.zeros((n, n))
    strides = (1, shape[0], shape[0] * shape[1])
    for i in range(n):
        for a, st in enumerate(strides):
            w = e[i, a]
            if w:
                j = i + st
                m[i, i] -= w
                m[j, j] -= w
                m[i, j] += w
                m[j, i] += w
    return np.linalg.pinv(m, rcond=1e-12, hermitian=True)


class SolidMultigridProjector(SolidPressureProjector):
    def __init__(self, grid, settings=None, device=None):
        super().__init__(grid, settings, device)
        s = self.settings
        dev = self.device
        self.levels = []
        self.smooth_kernel = KernelHandle('solid_mg_smooth.glsl')
        self.residual_kernel = KernelHandle('solid_mg_residual.glsl')
        self.restrict_kernel = KernelHandle('mg_restrict.glsl')
        self.prolong_kernel = KernelHandle('solid_mg_prolong.glsl')
        self.pre_sweeps = s.mg_pre_sweeps or 4
        self.post_sweeps = s.mg_post_sweeps or 4
        # sweeps on the levels below level 0 (the same counts unless mg_coarse_sweeps is set)
        self.coarse_pre = s.mg_coarse_sweeps or self.pre_sweeps
        self.coarse_post = s.mg_coarse_sweeps or self.post_sweeps
        self.last_cycles = 0
        self.timer = None
        self.learned = None
        self.use_graphs = True
        self.use_tail = True
        # tolerance solves in V-cycle mode run as one graph with a device-side
        # WHILE loop (no host round trip per cycle); False keeps the host loop
        self.use_device_loop = True
        # moving colliders: check a refresh's coarsening flags at the next refresh
        # (read back asynchronously) instead of waiting for them (coarse direct
        # solves are refreshed at once, as they need the new records on the host)
        self.defer_refresh_check = False
        # level-0 sweeps in fused pairs (ffx_graph_smooth2; same results; off: measured slower)
        self.fuse_sweeps = False
        # the device loop's convergence test also makes the next cycle's first
        # pre-sweep (ffx_graph_residual_max_smooth; same results)
        self.speculate = True
        self._pending_refresh = None
        self._loops = {}
        # [cycles of the last solve, cycles of all device-loop solves, decisions]
        self._counters = torch.zeros(3, dtype=torch.int32, device=dev.device)
        self._host_total = 0
        self._sweeps_per_cycle = 0
        self._cycle_factor = s.ir_inner_cycles if s.pressure_method == 'IR' else 1
        self._build_hierarchy()
        self._rmax = torch.zeros(2, dtype=torch.float32, device=dev.device)

    # The cycle count of the last solve lives on the device after a device-loop
    # solve; reading it synchronises once.
    @property
    def last_cycles(self):
        if getattr(self, '_cycles_on_device', False):
            # iterative refinement counts outer iterations of ir_inner_cycles V-cycles each
            self._cycles_host = int(self.device.fetch(self._counters[0])) * self._cycle_factor
            self._cycles_on_device = False
            self._iterations_host = self._cycles_host // self._cycle_factor * self._sweeps_per_cycle
        return self._cycles_host

    @last_cycles.setter
    def last_cycles(self, value):
        self._cycles_on_device = False
        self._cycles_host = value

    @property
    def last_iterations(self):
        if getattr(self, '_cycles_on_device', False):
            return self.last_cycles // self._cycle_factor * self._sweeps_per_cycle
        return self._iterations_host

    @last_iterations.setter
    def last_iterations(self, value):
        self._iterations_host = value

    def total_cycles(self):
        """V-cycles (or PCG iterations) of every solve so far (one readback)."""
        return self._host_total + int(self.device.fetch(self._counters[1])) * self._cycle_factor

    def _shapes(self):
        """Level shapes the grid allows (halving while all dims are even and >= 8)."""
        s = self.settings
        shapes = [tuple(self.grid.shape)]
        while min(shapes[-1]) >= 8 and all(n % 2 == 0 for n in shapes[-1]):
            if s.mg_max_levels and len(shapes) >= s.mg_max_levels:
                break
            shapes.append(tuple(n // 2 for n in shapes[-1]))
        return shapes

    def _build_hierarchy(self):
        """Aggregation hierarchy of the current mask (``physics/solid_hierarchy.py:11-54``)
        built on the device: level-0 links, coarse records level by level (one
        flag readback each), the coarse pseudoinverse, the single-block tail."""
        s = self.settings
        dev = self.device
        self.levels = []
        shape = tuple(self.grid.shape)
        weights = [float(np.float32((n / e) ** 2)) for n, e in zip(shape, self.grid.extent)]
        level0 = N.FfxGraphLevel(*shape, None, ptr(self._mask), N.f3(*weights))
        level0.coarse_scale = s.mg_coarse_scale   # over-correction of the prolongation (1: the reference's)
        # one link byte per cell lets the level-0 passes run four cells per thread
        nx, ny, nz = shape
        if getattr(self, '_links', None) is None:
            self._links = torch.empty((nz, ny, nx), dtype=torch.uint8, device=dev.device)
        dev.call('ffx_graph_links', C.byref(level0), ptr(self._links), dev.s)
        level0.links = self._links.data_ptr()
        self.levels.append(dict(shape=shape, edges=None, graph=level0, p=self.pressure, q=self.spare,
                                rhs=self.before))
        flag = torch.zeros(1, dtype=torch.int32, device=dev.device)
        for coarse_shape in self._shapes()[1:]:
            cx, cy, cz = coarse_shape
            edges = torch.empty((cz, cy, cx, 4), dtype=torch.float32, device=dev.device)
            dev.call('ffx_graph_coarsen', C.byref(self.levels[-1]['graph']), ptr(edges), ptr(flag), dev.s)
            if int(self.device.fetch(flag)):
                break   # an aggregate would join disconnected children: stop here
            graph = N.FfxGraphLevel(*coarse_shape, ptr(edges), None, N.f3(0.0, 0.0, 0.0))
            graph.coarse_scale = s.mg_coarse_scale
            self.levels.append(dict(shape=coarse_shape, edges=edges, graph=graph, p=dev.texture(coarse_shape),
                                    q=dev.texture(coarse_shape), rhs=dev.texture(coarse_shape)))
        self.coarse_matrix = None
        self._coarse_solve()
        self._graphs = {}
        self._pending_refresh = None
        if getattr(self, '_loops', None):
            torch.cuda.synchronize(dev.device)
            self._free_loops()
        self._tail, self.tail_start = self._make_tail()

    def _coarse_solve(self):
        """FP64 pseudoinverse of the coarsest level. A matrix of the same size is
        updated in place, so captured graphs (which hold its address) stay valid."""
        s = self.settings
        last = self.levels[-1]
        if prod(last['shape']) <= DIRECT_LIMIT and s.coarse_solver == 'DIRECT' and len(self.levels) > 1:
            edges = self.device.fetch(last['edges']).numpy()
            inv = torch.as_tensor(graph_pseudoinverse(last['shape'], edges), dtype=torch.float64)
            old = getattr(self, 'coarse_matrix', None)
            if old is not None and old.shape == inv.shape:
                old.copy_(inv.to(old.device))
            else:
                self.coarse_matrix = inv.to(self.device.device)
            self.coarse_kernel = KernelHandle('solid_mg_direct.glsl')
        else:
            self.coarse_matrix = self.coarse_kernel = None

    def refresh_hierarchy(self):
        """Follow a collider mask that changed in place (moving colliders): the
        level-0 links and every coarse level's records are recomputed into the
        same buffers (one pass per level, one flag readback), so captured graphs
        stay valid; if the coarsening would now stop at another depth, the
        hierarchy is rebuilt. An extension: the reference keeps masked Jacobi
        for moving colliders."""
        dev = self.device
        if self.defer_refresh_check:
            # the previous refresh's flags, copied back while the steps ran: rebuild
            # now if they asked for it (a V-cycle on a stale hierarchy still reaches
            # the tolerance, only more slowly)
            pending = self._pending_refresh
            self._pending_refresh = None
            if pending is not None:
                event, host, n_then, probe_then = pending
                event.synchronize()
                f = host.tolist()
                if len(self.levels) == n_then and (any(f[1:n_then]) or (probe_then and not f[n_then])):
                    self._build_hierarchy()
        shapes = self._shapes()
        n = len(self.levels)
        probe = n < len(shapes)           # the hierarchy stopped early: could it go deeper now?
        flags = torch.zeros(n + 1, dtype=torch.int32, device=dev.device)
        dev.call('ffx_graph_links', C.byref(self.levels[0]['graph']), ptr(self._links), dev.s)
        for k in range(1, n):
            dev.call('ffx_graph_coarsen', C.byref(self.levels[k - 1]['graph']), ptr(self.levels[k]['edges']),
                     ptr(flags[k:k + 1]), dev.s)
        if probe:
            cx, cy, cz = shapes[n]
            scratch = torch.empty((cz, cy, cx, 4), dtype=torch.float32, device=dev.device)
            dev.call('ffx_graph_coarsen', C.byref(self.levels[n - 1]['graph']), ptr(scratch), ptr(flags[n:n + 1]),
                     dev.s)
        if self.defer_refresh_check and self.coarse_matrix is None:
            host = torch.empty(n + 1, dtype=torch.int32, pin_memory=True)
            with torch.cuda.stream(dev.stream):
                host.copy_(flags, non_blocking=True)
                event = torch.cuda.Event()
                event.record(dev.stream)
            self._pending_refresh = (event, host, n, probe)
            return
        f = dev.fetch(flags).tolist()
        if any(f[1:n]) or (probe and not f[n]):
            self._build_hierarchy()
        elif self.coarse_matrix is not None:
            self._coarse_solve()

    def _make_tail(self):
        """Descriptor of the coarse levels run as one ``ffx_graph_tail`` launch:
        the levels from the first one (below level 0) with at most TAIL_CELLS
        cells down to the coarsest, at most eight of them. Needs an even number
        of sweeps per level and cycle, so buffer roles repeat."""
        if (self.coarse_pre + self.coarse_post) % 2 or len(self.levels) < 3:
            return None, None
        start = next((k for k in range(1, len(self.levels)) if prod(self.levels[k]['shape']) <= TAIL_CELLS), None)
        if start is None or (start == len(self.levels) - 1 and self.coarse_matrix is not None):
            # (a coarsest level alone is worth a launch only for its 80 sweeps; a
            # direct solve is one launch already)
            return None, None
        start = max(start, len(self.levels) - N.TAIL_LEVELS)
        tail = N.FfxGraphTail()
        tail.count = len(self.levels) - start
        tail.pre, tail.post, tail.omega = self.coarse_pre, self.coarse_post, 2.0 / 3.0
        tail.inverse = self.coarse_matrix.data_ptr() if self.coarse_matrix is not None else None
        for k, level in enumerate(self.levels[start:]):
            slot = tail.levels[k]
            slot.level = level['graph']
            slot.p, slot.q, slot.rhs = level['p'].data_ptr(), level['q'].data_ptr(), level['rhs'].data_ptr()
        return tail, start

    @property
    def allocated_bytes(self):
        coarse = sum(4 * 7 * prod(v['shape']) for v in self.levels[1:])
        direct = 8 * self.coarse_matrix.numel() if self.coarse_matrix is not None else 0
        links = self._links.numel() if self._links is not None else 0
        return super().allocated_bytes + coarse + direct + links

    def _fuse_cycle(self, level, zero_init, dot):
        """Whether this cycle runs its level-0 sweeps in fused pairs
        (ffx_graph_smooth2, ffx_graph_prolong_smooth2; same results): level 0
        with its link field on rows of four cells, outside the Krylov cycles,
        when the fused cycle swaps the level's p/q roles as often, modulo 2, as
        the sweep-by-sweep one (a cycle then leaves the iterate in the same
        buffer either way)."""
        if (not self.fuse_sweeps or dot is not None or level is not self.levels[0] or self._links is None
                or level['shape'][0] % 4):
            return False
        pre, post = self.pre_sweeps, self.post_sweeps
        pairs = lambda n: n // 2 + n % 2
        fused = (1 + pairs(pre - 1) if zero_init and pre > 0 else pairs(pre)) + \
            (1 + pairs(post - 2) if post >= 2 else post)
        return (fused - pre - post) % 2 == 0

    def smooth(self, level, count, fused=False):
        timer = self.timer if level is self.levels[0] else None
        while count > 0:
            pair = fused and count >= 2
            started = timer.begin() if timer is not None else None
            if pair:
                # two sweeps in one pass, bit-identical to two ffx_graph_smooth launches
                self.device.call('ffx_graph_smooth2', C.byref(level['graph']), ptr(level['p']), ptr(level['rhs']),
                                 2.0 / 3.0, None, ptr(level['q']), self.device.s)
            else:
                self.device.call('ffx_graph_smooth', C.byref(level['graph']), ptr(level['p']), ptr(level['rhs']),
                                 2.0 / 3.0, ptr(level['q']), self.device.s)
            if timer is not None:
                timer.end(started)
            level['p'], level['q'] = level['q'], level['p']
            self.last_iterations += 2 if pair else 1
            count -= 2 if pair else 1

    def cycle(self, index, zero_init=False, dot=None, first_pre=False):
        """One V-cycle from ``index`` down (``backend/solid_multigrid.py:46-65``).

        ``zero_init``: the level's iterate is zero, so the first sweep reads none.
        ``dot``: FP64 device slot receiving -rhs . result from the last sweep
        (used by the Krylov solve). ``first_pre``: the first pre-sweep's result
        is already in the level's spare buffer (ffx_graph_residual_max_smooth,
        run with the convergence test before the cycle)."""
        level = self.levels[index]
        dev = self.device
        if index == len(self.levels) - 1:
            if self.coarse_matrix is not None:
                # written straight into p (the iterate is replaced, not updated),
                # so buffer roles repeat from one cycle to the next
                dev.call('ffx_direct_solve', prod(level['shape']), ptr(self.coarse_matrix), ptr(level['rhs']), 1.0,
                         ptr(level['p']), dev.s)
            else:
                if zero_init:
                    level['p'].zero_()
                self.smooth(level, 80)
            if dot is not None:
                dev.call('ffx_dot', level['p'].numel(), ptr(level['rhs']), ptr(level['p']), -1.0, ptr(dot), dev.s)
            return
        pre, post = (self.pre_sweeps, self.post_sweeps) if index == 0 else (self.coarse_pre, self.coarse_post)
        fuse = not first_pre and self._fuse_cycle(level, zero_init, dot)
        if first_pre and pre > 0:
            level['p'], level['q'] = level['q'], level['p']
            self.last_iterations += 1
            pre -= 1
        elif zero_init:
            if pre > 0:
                dev.call('ffx_graph_smooth_zero', C.byref(level['graph']), ptr(level['rhs']), 2.0 / 3.0,
                         ptr(level['q']), dev.s)
                level['p'], level['q'] = level['q'], level['p']
                self.last_iterations += 1
                pre -= 1
            else:
                level['p'].zero_()
        self.smooth(level, pre, fuse)
        coarse = self.levels[index + 1]
        tail = self.use_tail and index + 1 == self.tail_start
        # the coarse iterate starts from zero: the restriction pass clears it
        # (the tail clears its own levels)
        dev.call('ffx_graph_residual_restrict_zero', C.byref(level['graph']), ptr(level['p']), ptr(level['rhs']),
                 ptr(coarse['rhs']), None if tail else ptr(coarse['p']), dev.s)
        if tail:
            # every level below runs inside one launch
            dev.call('ffx_graph_tail', C.byref(self._tail), dev.s)
            self.last_iterations += self._tail_sweeps()
        else:
            self.cycle(index + 1)
        if post == 1 and dot is not None:
            dev.call('ffx_graph_prolong_smooth_dot', C.byref(level['graph']), ptr(level['p']), ptr(coarse['p']),
                     ptr(level['rhs']), 2.0 / 3.0, ptr(level['q']), ptr(dot), -1.0, dev.s)
            level['p'], level['q'] = level['q'], level['p']
            self.last_iterations += 1
            return
        if fuse and post > 1:
            # prolongation + the first two post-sweeps in one pass (ffx_graph_prolong_smooth2)
            dev.call('ffx_graph_prolong_smooth2', C.byref(level['graph']), ptr(level['p']), ptr(coarse['p']),
                     ptr(level['rhs']), 2.0 / 3.0, None, ptr(level['q']), dev.s)
            level['p'], level['q'] = level['q'], level['p']
            self.last_iterations += 2
            self.smooth(level, post - 2, fuse)
        elif post > 0:
            dev.call('ffx_graph_prolong_smooth', C.byref(level['graph']), ptr(level['p']), ptr(coarse['p']),
                     ptr(level['rhs']), 2.0 / 3.0, ptr(level['q']), dev.s)
            level['p'], level['q'] = level['q'], level['p']
            self.last_iterations += 1
            if dot is not None and post > 1:
                self.smooth(level, post - 2)
                dev.call('ffx_graph_smooth_dot', C.byref(level['graph']), ptr(level['p']), ptr(level['rhs']),
                         2.0 / 3.0, ptr(level['q']), ptr(dot), -1.0, dev.s)
                level['p'], level['q'] = level['q'], level['p']
                self.last_iterations += 1
                return
            self.smooth(level, post - 1)
        else:
            dev.call('ffx_graph_prolong', C.byref(level['graph']), ptr(level['p']), ptr(coarse['p']),
                     ptr(level['q']), dev.s)
            level['p'], level['q'] = level['q'], level['p']
        if dot is not None:
            dev.call('ffx_dot', level['p'].numel(), ptr(level['rhs']), ptr(level['p']), -1.0, ptr(dot), dev.s)

    def _tail_sweeps(self):
        n = len(self.levels) - self.tail_start - 1
        return n * (self.coarse_pre + self.coarse_post) + (0 if self.coarse_matrix is not None else 80)

    def _residual_max(self):
        level = self.levels[0]
        self.device.call('ffx_graph_residual_max', C.byref(level['graph']), ptr(level['p']), ptr(level['rhs']),
                         ptr(self._rmax[0:1]), self.device.s)
        return float(self.device.fetch(self._rmax[0]))

    # ------------------------------------------------------------ graph replay
    def _replayed(self, key, fn):
        """Run ``fn`` (a fixed sequence of passes over fixed buffers) through a
        CUDA graph captured on first use for this ``key``. Every level swaps its
        p/q roles an even number of times per cycle, so the buffers a cycle
        touches are the same every time it runs with the same level-0 roles."""
        if not self.use_graphs or self.timer is not None:
            fn()
            return
        dev = self.device
        entry = self._graphs.get(key)
        if entry is None:
            sweeps, calls = self.last_iterations, dev.calls
            graph = dev.capture(fn)
            entry = (graph, self.last_iterations - sweeps, dev.calls - calls)
            self.last_iterations, dev.calls = sweeps, calls
            self._graphs[key] = entry
        dev.replay(entry[0])
        self.last_iterations += entry[1]
        dev.calls += entry[2]   # the native passes the graph launches

    # ------------------------------------------------------------ Krylov solve
    def _krylov_buffers(self):
        if getattr(self, '_kry', None) is None:
            dev = self.device
            shape = self.levels[0]['shape']
            self._kry = dict(res=dev.texture(shape), z=dev.texture(shape), z2=dev.texture(shape),
                             p=[dev.texture(shape), dev.texture(shape)], q=dev.texture(shape),
                             rz=torch.zeros(2, dtype=torch.float64, device=dev.device),   # [current, previous]
                             pq=torch.zeros(1, dtype=torch.float64, device=dev.device),
                             rmax=torch.zeros(1, dtype=torch.float32, device=dev.device))
        return self._kry

    def _precondition(self, res, bufs, rz_slot):
        """z = V-cycle(res) from a zero iterate; rz_slot <- -res . z. Returns z."""
        L0 = self.levels[0]
        saved = (L0['p'], L0['q'], L0['rhs'])
        L0['p'], L0['q'], L0['rhs'] = bufs['z'], bufs['z2'], res
        self.cycle(0, zero_init=True, dot=rz_slot)
        z = L0['p']
        bufs['z'], bufs['z2'] = L0['p'], L0['q']
        L0['p'], L0['q'], L0['rhs'] = saved
        return z

    def _pcg_iteration(self, B, x, k):
        """z = M res; p = z + beta p_old; q = A p; x += alpha p; res += alpha q."""
        dev = self.device
        g = C.byref(self.levels[0]['graph'])
        z = self._precondition(B['res'], B, B['rz'][0:1])
        p_new, p_old = B['p'][k % 2], B['p'][(k + 1) % 2]
        first = k == 0
        dev.call('ffx_pcg_direction_apply', g, ptr(z), None if first else ptr(p_old), ptr(B['rz'][0:1]),
                 None if first else ptr(B['rz'][1:2]), ptr(p_new), ptr(B['q']), ptr(B['pq']), dev.s)
        dev.call('ffx_pcg_update', x.numel(), ptr(B['rz'][0:1]), ptr(B['pq']), ptr(x), ptr(p_new), ptr(B['res']),
                 ptr(B['q']), ptr(B['rmax']), dev.s)
        B['rz'][1:2].copy_(B['rz'][0:1])

    def _solve_krylov(self, scale, budget):
        """Conjugate gradients on A = -L preconditioned by the aggregation
        V-cycle, until max|rhs - L x| <= tol * max|rhs| (or ``budget`` cycles)."""
        s = self.settings
        dev = self.device
        B = self._krylov_buffers()
        g = C.byref(self.levels[0]['graph'])
        x = self.pressure
        n = x.numel()
        tol = s.pressure_tolerance * scale if s.pressure_tolerance > 0 else -1.0
        for _restart in range(2):
            dev.call('ffx_graph_residual', g, ptr(x), ptr(self.before), ptr(B['res']), dev.s)
            dev.call('ffx_max_abs', n, N.FFX_F32, ptr(B['res']), ptr(B['rmax']), dev.s)
            if float(self.device.fetch(B['rmax'])) <= tol:
                return
            k = 0
            while self.last_cycles < budget:
                if k == 0:
                    self._pcg_iteration(B, x, 0)
                else:
                    self._replayed(('pcg', x.data_ptr(), k % 2), lambda kk=k: self._pcg_iteration(B, x, kk))
                self.last_cycles += 1
                k += 1
                if float(self.device.fetch(B['rmax'])) <= tol:
                    break
            if tol < 0 or self.last_cycles >= budget:
                return
            # the recursively updated residual drifts in FP32: confirm on the true one
            dev.call('ffx_graph_residual_max', g, ptr(x), ptr(self.before), ptr(B['rmax']), dev.s)
            if float(self.device.fetch(B['rmax'])) <= tol:
                return

    def solve_pressure(self, dt, previous_dt):
        with torch.cuda.stream(self.device.stream):
            self._solve(dt, previous_dt)

    def _solve(self, dt, previous_dt):
        s = self.settings
        self.last_cycles = 0
        if len(self.levels) == 1:
            return super().solve_pressure(dt, previous_dt)
        warm = s.solid_warm_start and previous_dt is not None
        if warm and s.learned_warm_start and s.learned_correction and self.learned is not None:
            # learned correction of the warm start: p += N(rhs - L p)
            self._learned_correction()
        elif s.learned_warm_start and not warm:
            if self.learned is None:
                raise ValueError('learned_warm_start needs a model: projector.attach_learned(LearnedWarmStart(...))')
            self.learned.guess(self.before, self.pressure)
        elif not (s.solid_warm_start and previous_dt is not None):
            self.pressure.zero_()
        self.levels[0]['p'], self.levels[0]['q'] = self.pressure, self.spare
        self.last_iterations = 0
        budget = s.pressure_cycles * (s.pressure_cold_multiplier if previous_dt is None else 1)
        if s.pressure_method == 'PCG':
            scale = 0.0
            if s.pressure_tolerance > 0:
                self.device.call('ffx_max_abs', self.before.numel(), N.FFX_F32, ptr(self.before),
                                 ptr(self._rmax[1:2]), self.device.s)
                scale = float(self.device.fetch(self._rmax[1]))
                budget = s.pressure_max_cycles
            if s.pressure_tolerance > 0 and scale == 0:
                self.pressure.zero_()
            else:
                self._solve_krylov(scale, budget)
            self.levels[0]['p'], self.levels[0]['q'] = self.pressure, self.spare
            self._host_total += self.last_cycles
            return
        if s.pressure_method == 'IR':
            if not (s.pressure_tolerance > 0):
                raise ValueError("pressure_method 'IR' needs a pressure tolerance")
            self._device_solve(refine=True)
            return
        if s.pressure_tolerance > 0 and self.use_device_loop and self.use_graphs and self.timer is None:
            self._device_solve()
            return
        one_cycle = lambda: self._replayed(('vcycle', self.levels[0]['p'].data_ptr()), lambda: self.cycle(0))
        if s.pressure_tolerance <= 0:
            for _ in range(budget):
                one_cycle()
                self.last_cycles += 1
        else:
            self.device.call('ffx_max_abs', self.before.numel(), N.FFX_F32, ptr(self.before),
                             ptr(self._rmax[1:2]), self.device.s)
            scale = float(self.device.fetch(self._rmax[1]))
            if scale == 0:
                self.levels[0]['p'].zero_()
            else:
                while self.last_cycles < s.pressure_max_cycles and self._residual_max() > s.pressure_tolerance * scale:
                    one_cycle()
                    self.last_cycles += 1
        self.pressure, self.spare = self.levels[0]['p'], self.levels[0]['q']
        self._host_total += self.last_cycles

    # ------------------------------------------------------ device-side loop
    def _device_solve(self, refine=False):
        """The tolerance solve as one graph launch: max|rhs|, the residual
        maximum, and WHILE (cycles < max and max|r| > tol * max|rhs|) {V-cycle,
        residual maximum} decided on the device; the cycle count stays on the
        device until read. ``refine``: the iterative-refinement form, whose
        loop counts outer iterations (see ``_capture_loop``)."""
        dev = self.device
        key = ('refine' if refine else 'loop', self.levels[0]['p'].data_ptr(), self.levels[0]['q'].data_ptr())
        entry = self._loops.get(key)
        if entry is None:
            entry = self._capture_loop(refine)
            self._loops[key] = entry
        handle, per_cycle, calls = entry
        dev.call('ffx_loop_launch', handle, dev.s)
        dev.calls += calls - 1
        self._sweeps_per_cycle = per_cycle
        self._cycles_on_device = True
        self.pressure, self.spare = self.levels[0]['p'], self.levels[0]['q']

    def _capture_loop(self, refine=False):
        """Capture the solve loop (see ``_device_solve``) into a graph; returns
        (loop handle, sweeps per cycle, native passes per cycle).

        ``refine``: iterative refinement. The loop tests the true FP32 residual
        r = rhs - L p (kept in a buffer); each iteration solves L e = r from
        e = 0 with ``ir_inner_cycles`` V-cycles and sets p = p + e, so the
        pressure is only ever updated by whole corrections and every decision
        reads a freshly computed residual."""
        s = self.settings
        dev = self.device
        level = self.levels[0]
        n = self.before.numel()
        tol = float(s.pressure_tolerance)
        limit = int(s.pressure_max_cycles)
        counters = ptr(self._counters)
        loop = C.c_void_p()
        # the stream lives on the underlying CudaDevice (a SolidDevice delegates to it)
        root = dev.__dict__.get('base', dev)
        side = torch.cuda.Stream(root.device)
        side.wait_stream(root.stream)
        saved, saved_iters, saved_calls = root.stream, self._iterations_host, dev.calls
        p0, q0 = level['p'], level['q']

        def check_and_sweep():
            # max |rhs - L p| for the decision and, from the same pass, the sweep of p into q
            dev.call('ffx_graph_residual_max_smooth', C.byref(level['graph']), ptr(level['p']), ptr(level['rhs']),
                     2.0 / 3.0, ptr(self._rmax[0:1]), ptr(level['q']), dev.s)
        try:
            root.stream = side
            if refine:
                if getattr(self, '_ir', None) is None:
                    self._ir = tuple(dev.texture(level['shape']) for _ in range(3))   # r, e, e spare
                r, e, e2 = self._ir

                def true_residual():
                    dev.call('ffx_graph_residual', C.byref(level['graph']), ptr(p0), ptr(self.before), ptr(r), dev.s)
                    dev.call('ffx_max_abs', n, N.FFX_F32, ptr(r), ptr(self._rmax[0:1]), dev.s)
            with torch.cuda.stream(side):
                N.check(dev.lib.ffx_loop_begin(dev.s, C.byref(loop)))
                dev.call('ffx_loop_reset_counter', counters, dev.s)
                dev.call('ffx_max_abs', n, N.FFX_F32, ptr(self.before), ptr(self._rmax[1:2]), dev.s)
                dev.call('ffx_zero_if_unscaled', ptr(self._rmax[1:2]), ptr(level['p']), n, dev.s)
                speculate = not refine and self.speculate and self.pre_sweeps > 0
                if refine:
                    true_residual()
                elif speculate:
                    check_and_sweep()
                else:
                    dev.call('ffx_graph_residual_max', C.byref(level['graph']), ptr(level['p']), ptr(level['rhs']),
                             ptr(self._rmax[0:1]), dev.s)
                dev.call('ffx_loop_decide', loop, ptr(self._rmax[0:1]), ptr(self._rmax[1:2]), tol, limit, counters,
                         dev.s)
                body = C.c_void_p()
                N.check(dev.lib.ffx_loop_while(loop, C.byref(body)))
            inner = torch.cuda.ExternalStream(body.value, device=root.device)
            root.stream = inner
            calls0 = dev.calls
            self._iterations_host = 0
            with torch.cuda.stream(inner):
                if refine:
                    # the correction equation L e = r from e = 0, then p += e
                    level['p'], level['q'], level['rhs'] = e, e2, r
                    try:
                        for k in range(s.ir_inner_cycles):
                            self.cycle(0, zero_init=(k == 0))
                    finally:
                        corr = level['p']
                        level['p'], level['q'], level['rhs'] = p0, q0, self.before
                    dev.call('ffx_add', n, ptr(p0), ptr(corr), ptr(p0), dev.s)
                    true_residual()
                elif speculate:
                    # the cycle starts from the sweep the test made; the test after it
                    # makes the next cycle's (discarded when the loop stops)
                    self.cycle(0, first_pre=True)
                    check_and_sweep()
                else:
                    self.cycle(0)
                    dev.call('ffx_graph_residual_max', C.byref(level['graph']), ptr(level['p']), ptr(level['rhs']),
                             ptr(self._rmax[0:1]), dev.s)
                dev.call('ffx_loop_decide', loop, ptr(self._rmax[0:1]), ptr(self._rmax[1:2]), tol, limit, counters,
                         dev.s)
            per_cycle, calls = self._iterations_host, dev.calls - calls0
            if level['p'] is not p0 or level['q'] is not q0:
                raise RuntimeError('a V-cycle must leave the level-0 buffer roles unchanged')
            N.check(dev.lib.ffx_loop_end_while(loop))
            root.stream = side
            N.check(dev.lib.ffx_loop_end(loop))
        except Exception:
            if loop.value:
                dev.lib.ffx_loop_destroy(loop)
            raise
        finally:
            root.stream = saved
            self._iterations_host = saved_iters
            dev.calls = saved_calls
        return loop, per_cycle, calls

    def _free_loops(self):
        for handle, _, _ in self._loops.values():
            self.device.lib.ffx_loop_destroy(handle)
        self._loops = {}

    def gradient_links(self):
        # the link bytes follow the mask (recomputed on every collider move)
        if len(self.levels) > 1 and getattr(self, '_links', None) is not None and self.device.mask is not None:
            return self._links
        return None

    def _learned_correction(self):
        dev = self.device
        level = self.levels[0]
        if getattr(self, '_corr', None) is None:
            self._corr = (dev.texture(level['shape']), dev.texture(level['shape']))
        r, e = self._corr
        dev.call('ffx_graph_residual', C.byref(level['graph']), ptr(self.pressure), ptr(self.before), ptr(r), dev.s)
        self.learned.guess(r, e)
        dev.call('ffx_add', self.pressure.numel(), ptr(self.pressure), ptr(e), ptr(self.pressure), dev.s)

    def extrapolation_beta(self):
        s = self.settings
        # warm solves start from the extrapolation; a learned guess of cold solves is
        # compatible, a learned correction of warm ones is not
        learned_correction = s.learned_warm_start and s.learned_correction
        if s.warm_start_extrapolation > 0 and s.solid_warm_start and not learned_correction and len(self.levels) > 1:
            return s.warm_start_extrapolation
        return 0.0

    def attach_learned(self, model):
        """Pressure guess used when ``learned_warm_start`` is set
        (``fluxfx_b200.learned.LearnedWarmStart``)."""
        self.learned = model

    def reset(self):
        super().reset()
        self.last_cycles = 0
        for level in self.levels[1:]:
            for name in ('p', 'q', 'rhs'):
                level[name].zero_()

    def level_edges(self, index):
        """Host copy of a level's (+x, +y, +z, active) records, x-fast."""
        level = self.levels[index]
        if level['edges'] is not None:
            return self.device.fetch(level['edges']).numpy()
        nz, ny, nx = self.levels[0]['p'].shape
        out = torch.empty((nz, ny, nx, 4), dtype=torch.float32, device=self.device.device)
        self.device.call('ffx_graph_level0_edges', C.byref(level['graph']), ptr(out), self.device.s)
        return self.device.fetch(out).numpy()

    def metrics(self):
        return super().metrics() | {
            'solver': 'SOLID_MULTIGRID' if self.last_cycles else 'SOLID_JACOBI',
            'v_cycles': self.last_cycles, 'levels': [v['shape'] for v in self.levels],
            'coarse_solver': 'graph_pseudoinverse' if self.coarse_matrix is not None else 'masked_smoothing',
            'aggregation': 'connected_children_only'}

    def close(self):
        if getattr(self, '_loops', None):
            torch.cuda.synchronize(self.device.device)
            self._free_loops()
        self._graphs = {}
        self._kry = None
        if self.learned is not None:
            self.learned.close()
        self.learned = None
        self._links = None
        self._tail = None
        self.levels = []
        self.coarse_matrix = self.coarse_kernel = None
        super().close()
