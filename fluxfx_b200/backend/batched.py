"""Many independent smoke domains of uneven sizes advanced together.

No counterpart in the reference, whose solvers own one domain each
(``fluxfx/backend/projected.py:13-229``). ``BatchedSmoke`` takes fully set-up
``DenseProjectedSmoke`` solvers (collider path, FP32, stand-alone V-cycles to
a tolerance) and runs their steps through ``libffx_core``'s batched plan
(``ffx_batch_*``): one persistent launch per pass over every domain, the
pressure solve as a conditional WHILE node of a CUDA graph that stops when
every domain has converged, and each domain's next time step
``min(dt_max, cfl * cell / max|u|)`` computed on the device, so a run of many
steps is one graph launch with no host round trip. Each domain's fields after
a batched run are bit-identical to stepping that solver alone (from a reset)
with the same time-step rule. The solve starts from zero, or with
``solid_warm_start`` from the previous pressure times dt / previous dt.

A domain without colliders takes the collider path with an empty mask (the
reference's collider path with its collider outside the domain).

The tile shape and persistent grid of every pass kind come from ``tune()``,
an autotuner that times each pass alone on the plan's own buffers and keeps
the fastest configuration (cached by device and domain shapes when given a
cache file).
"""
import ctypes as C
import hashlib
import json
import os
from math import prod

import torch

from .. import _native as N
from .device import ptr
from .solid_multigrid import SolidMultigridProjector

SHAPES = ((32, 8), (64, 4), (128, 2), (16, 16))
GRIDS = (0, 1, 2, 4)
TUNABLE = (N.PASS_PREDICTOR, N.PASS_VELOCITY, N.PASS_DIVERGENCE, N.PASS_SCALE, N.PASS_GRADIENT,
           N.PASS_SCALAR_PREDICTOR, N.PASS_SCALAR_REVERSE, N.PASS_SCALAR_FINAL, N.PASS_RESIDUAL_MAX, N.PASS_SMOOTH,
           N.PASS_RESIDUAL_RESTRICT, N.PASS_PROLONG_SMOOTH) + N.FIXED_TILE_PASSES


def _check_solver(i, s):
    st = s.settings
    p = s.projector
    problems = []
    if s.solids is None:
        problems.append('no collider mask (give it a collider, e.g. one outside the domain)')
    if st.storage != 'FP32':
        problems.append('FP32 storage required')
    if not isinstance(p, SolidMultigridProjector) or len(p.levels) < 2:
        problems.append('needs the collider multigrid with at least two levels')
    elif not p.uses_impulse:
        problems.append('needs the impulse pressure form')
    if st.pressure_method != 'VCYCLE' or st.learned_warm_start or st.warm_start_extrapolation > 0:
        problems.append('stand-alone V-cycles required (from zero or the previous pressure)')
    if st.mg_coarse_sweeps and st.mg_coarse_sweeps != p.pre_sweeps or st.mg_coarse_sweeps and p.pre_sweeps != p.post_sweeps:
        problems.append('the same sweep counts on every level required')
    if not st.pressure_tolerance > 0:
        problems.append('a pressure tolerance is required')
    if st.moving_colliders or st.vorticity_strength > 0 or s.combustion is not None:
        problems.append('moving colliders, confinement and combustion are not batched')
    if problems:
        raise ValueError(f'domain {i}: ' + '; '.join(problems))


class BatchedSmoke:
    """Batched stepping of ``solvers`` (``DenseProjectedSmoke``), each with its
    ``sources`` (list of ``Source`` or None) and the time-step rule
    dt = min(dt_max, cfl * cell / max|u|), first dt = ``dt0``."""

    def __init__(self, solvers, sources, *, cfl=0.5, dt_max=0.02, dt0=0.02, cells=None):
        if not solvers or len(solvers) > N.BATCH_MAX:
            raise ValueError(f'1..{N.BATCH_MAX} domains required')
        self.lib = N.load()
        self.solvers = list(solvers)
        self.device = solvers[0].device
        self.stream = self.device.s
        self._domains = (N.FfxBatchDomain * len(solvers))()
        self._keep = []
        for i, (s, src) in enumerate(zip(self.solvers, sources)):
            _check_solver(i, s)
            cell = cells[i] if cells is not None else min(s.grid.cell_size)
            self._fill(self._domains[i], s, src, cell, cfl, dt_max, dt0)
        need = C.c_int64(0)
        N.check(self.lib.ffx_batch_workspace_bytes(self._domains, len(solvers), C.byref(need)))
        self.workspace = torch.zeros(int(need.value) + 256, dtype=torch.uint8, device=self.device.device)
        base = (self.workspace.data_ptr() + 255) & ~255
        plan = C.c_void_p()
        N.check(self.lib.ffx_batch_create(self._domains, len(solvers), C.c_void_p(base), int(need.value),
                                          C.byref(plan)))
        self.plan = plan
        self._graphs = {}
        self.config = {}
        self.steps = 0

    # ------------------------------------------------------------ setup
    def _fill(self, D, s, sources, cell, cfl, dt_max, dt0):
        st = s.settings
        p = s.projector
        det = s.detail
        if det.face_predictor is None:
            det.face_predictor = [s.device.texture(sh, dtype=det.dtype) for sh in s.grid.face_shapes]
        det._ensure_scalar(2)
        D.grid = s._g
        D.solid, D.halo = s.solids.mask.data_ptr(), s.solids.halo.data_ptr()
        clear = getattr(s.solids, 'clear', None)
        D.clear = clear.data_ptr() if clear is not None else None
        D.u, D.v, D.w = [f.data_ptr() for f in s._velocity]
        D.pu, D.pv, D.pw = [f.data_ptr() for f in det.face_predictor]
        D.bu, D.bv, D.bw = [f.data_ptr() for f in p.bounded]
        D.density[0], D.density[1] = s._front.data_ptr(), s._back.data_ptr()
        D.temperature[0], D.temperature[1] = s._temperature.data_ptr(), s._temperature_back.data_ptr()
        D.predictor[0], D.predictor[1] = det.predictors[0].data_ptr(), det.predictors[1].data_ptr()
        D.reverse[0], D.reverse[1] = det.reverses[0].data_ptr(), det.reverses[1].data_ptr()
        D.after = p.after.data_ptr()
        from ..physics.emission import Emission
        if sources is not None:
            s._prepare_sources(sources)
        D.sources = s._fill_sources(Emission(st.source_center), sources)
        D.velocity_corrected = int(st.velocity_advection == 'MACCORMACK')
        D.scalar_corrected = int(st.scalar_advection == 'MACCORMACK')
        D.blend, D.lift, D.weight = st.velocity_blend, st.thermal_lift, st.density_weight
        density_target = st.source_rate if st.density_mode == 'TARGET' else -1.0
        heat_target = st.heat_source_rate if st.heat_mode == 'TARGET' else -1.0
        D.density_channel = N.FfxScalarChannel(None, None, None, None, st.source_rate, st.dissipation, density_target,
                                               0, 0)
        D.heat_channel = N.FfxScalarChannel(None, None, None, None, st.heat_source_rate, st.cooling, heat_target, 1,
                                            int(st.heat_mode == 'TARGET'))
        D.cell, D.cfl, D.dt_max, D.dt0 = cell, cfl, dt_max, dt0
        D.levels = len(p.levels)
        if D.levels > N.BATCH_LEVELS:
            raise ValueError(f'at most {N.BATCH_LEVELS} multigrid levels')
        for k, lv in enumerate(p.levels):
            D.level[k].level = lv['graph']
            D.level[k].p, D.level[k].q, D.level[k].rhs = lv['p'].data_ptr(), lv['q'].data_ptr(), lv['rhs'].data_ptr()
        D.tail_start = p.tail_start if (p.use_tail and p._tail is not None) else -1
        D.inverse = p.coarse_matrix.data_ptr() if p.coarse_matrix is not None else None
        D.pre, D.post = p.pre_sweeps, p.post_sweeps
        D.max_cycles = st.pressure_max_cycles
        D.warm_start = int(st.solid_warm_start)
        D.tolerance = st.pressure_tolerance
        # departure points of the predictor passes, reused by the correction passes
        # (faces where both passes form the same start points), as the single-domain step does
        dev = s.device.device
        if D.velocity_corrected and det.reuse_traces and det._face_reuse:
            if det.face_trace is None:
                det.face_trace = [torch.empty(6 * prod(sh), dtype=torch.float32, device=dev)
                                  for sh in s.grid.face_shapes]
            for a in range(3):
                D.face_trace[a] = det.face_trace[a].data_ptr()
        if D.scalar_corrected and det.reuse_traces:
            if det.cell_trace is None:
                det.cell_trace = torch.empty(3 * prod(s.grid.shape), dtype=torch.float32, device=dev)
            D.cell_trace = det.cell_trace.data_ptr()
            # the reverse pass decides the final pass's corrections, as the single-domain step does
            if det.cell_ok is None:
                nx, ny, nz = s.grid.shape
                det.cell_ok = torch.empty((nz, ny, nx), dtype=torch.uint8, device=dev)
            D.cell_ok = det.cell_ok.data_ptr()

    # ------------------------------------------------------------ running
    @property
    def parity(self):
        return self.lib.ffx_batch_parity(self.plan)

    def graph(self, steps):
        """Instantiated graph of ``steps`` steps from the current parity (cached)."""
        key = (steps, self.parity)
        g = self._graphs.get(key)
        if g is None:
            h = C.c_void_p()
            N.check(self.lib.ffx_batch_graph(self.plan, steps, C.byref(h)))
            g = self._graphs[key] = h
        return g

    def run(self, steps=1):
        """Enqueue ``steps`` steps of every domain (one graph launch)."""
        g = self.graph(steps)
        N.check(self.lib.ffx_batch_launch(self.plan, g, steps, self.stream))
        self.steps += steps

    def stats(self):
        """Per domain: dt of the next step, dt and V-cycles of the last step,
        total V-cycles, steps, velocity maxima and simulated time."""
        out = (N.FfxBatchStats * len(self.solvers))()
        N.check(self.lib.ffx_batch_stats(self.plan, out, self.stream))
        return [dict(dt=o.dt, last_dt=o.last_dt, last_cycles=o.last_cycles, total_cycles=o.total_cycles,
                     steps=o.steps, maxima=tuple(o.maxima), time=o.time, loop_iterations=o.loop_iterations)
                for o in out]

    def fields(self, i):
        """(density, temperature, (u, v, w)) tensors of domain ``i`` now."""
        s = self.solvers[i]
        if self.parity:
            return s._back, s._temperature_back, tuple(s._velocity)
        return s._front, s._temperature, tuple(s._velocity)

    def launches_per_step(self, iterations):
        """Kernel launches of one step whose solve loop ran ``iterations`` times."""
        doms = [self._domains[i] for i in range(len(self.solvers))]
        tops = [d.tail_start if d.tail_start >= 0 else d.levels - 1 for d in doms]
        k = max(tops)
        pre, post = doms[0].pre, doms[0].post
        coarse = int(any(d.tail_start >= 0 for d in doms)) + int(any(d.tail_start < 0 and d.inverse for d in doms))
        coarse += 80 * int(any(d.tail_start < 0 and not d.inverse for d in doms))
        cycle = k * (pre + 1) + coarse + k * post
        vc = int(any(d.velocity_corrected for d in doms))
        sc = int(any(d.scalar_corrected for d in doms))
        return (vc + 3) + (1 + 2 * sc + 1) + 1 + iterations * (2 + cycle)

    # ------------------------------------------------------------ autotuning
    def signature(self):
        shapes = sorted(tuple(s.grid.shape) for s in self.solvers)
        return hashlib.sha1(json.dumps(shapes).encode()).hexdigest()[:16]

    def set_config(self, config):
        for name, (shape, grid) in config.items():
            kind = N.PASS_NAMES.index(name)
            N.check(self.lib.ffx_batch_set_config(self.plan, kind, shape, grid))
        self.config.update(config)
        self._free_graphs()

    def tune(self, repeats=5, cache=None):
        """Time every (tile shape, persistent grid) of each pass kind alone on
        the plan's buffers and keep the fastest; returns {pass: (shape, grid,
        ms)}. With ``cache`` (a JSON file) results are reused per device and
        domain shapes."""
        dev = torch.cuda.get_device_name(self.device.device)
        key = f'{dev}|{self.signature()}'
        table = {}
        if cache and os.path.exists(cache):
            with open(cache) as f:
                table = json.load(f)
            if key in table:
                self.set_config({k: tuple(v[:2]) for k, v in table[key].items()})
                return {k: tuple(v) for k, v in table[key].items()}
        stream = torch.cuda.ExternalStream(self.stream) if self.stream else torch.cuda.current_stream()
        best = {}
        for kind in TUNABLE:
            results = []
            for shape in ((0,) if kind in N.FIXED_TILE_PASSES else range(len(SHAPES))):
                for grid in GRIDS:
                    N.check(self.lib.ffx_batch_set_config(self.plan, kind, shape, grid))
                    N.check(self.lib.ffx_batch_tune_pass(self.plan, kind, self.stream))
                    start = torch.cuda.Event(enable_timing=True)
                    end = torch.cuda.Event(enable_timing=True)
                    start.record(stream)
                    for _ in range(repeats):
                        N.check(self.lib.ffx_batch_tune_pass(self.plan, kind, self.stream))
                    end.record(stream)
                    end.synchronize()
                    results.append((start.elapsed_time(end) / repeats, shape, grid))
            ms, shape, grid = min(results)
            best[N.PASS_NAMES[kind]] = (shape, grid, ms)
        self.set_config({k: v[:2] for k, v in best.items()})
        if cache:
            table[key] = best
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            with open(cache, 'w') as f:
                json.dump(table, f, indent=1)
        return best

    # ------------------------------------------------------------ teardown
    def _free_graphs(self):
        for g in self._graphs.values():
            self.lib.ffx_batch_graph_free(g)
        self._graphs = {}

    def close(self):
        self._free_graphs()
        if self.plan:
            self.lib.ffx_batch_destroy(self.plan)
            self.plan = None
        self.workspace = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batched_scenes(count=48, seed=0, sizes=(32, 48, 64, 96, 128), cell=1.0 / 64.0, warm_start=False,
                   coarse_scale=1.0):
    """Seeded uneven domains: each axis from ``sizes``; 1-3 spherical emitters
    (radius 3-8 cells, density and temperature U(0.5, 1), in the lower third);
    0-2 static sphere colliders (radius 4-16 cells, above the emitters). A
    domain without colliders gets one sphere outside the domain (an empty
    mask). ``warm_start`` and ``coarse_scale`` select the solver (previous
    pressure as the start; over-correction of the prolongation). Returns
    [(grid, settings, colliders, emitters, noise)]."""
    import numpy as np
    from ..physics.collision import primitive
    from ..physics.config import GridSpec
    from ..physics.emission import Emission, Source
    from ..physics.pressure import PressureSettings
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        shape = tuple(int(rng.choice(sizes)) for _ in range(3))
        extent = tuple(n * cell for n in shape)
        grid = GridSpec(shape, extent=extent, axis_limit=max(128, max(shape)))
        emitters = []
        for _ in range(int(rng.integers(1, 4))):
            r = float(rng.uniform(3, 8)) * cell
            pos = (float(rng.uniform(r, extent[0] - r)), float(rng.uniform(r, extent[1] - r)),
                   float(rng.uniform(r, extent[2] / 3)))
            d, t = rng.uniform(0.5, 1.0, 2)
            emitters.append(Source(pos, r, float(d), float(t), Emission(pos), 'TARGET', 'SOFT'))
        colliders = []
        for _ in range(int(rng.integers(0, 3))):
            r = float(rng.uniform(4, 16)) * cell
            c = (float(rng.uniform(0, extent[0])), float(rng.uniform(0, extent[1])),
                 float(rng.uniform(extent[2] / 2, extent[2])))
            colliders.append(primitive('SPHERE', c, (r, r, r)))
        if not colliders:
            colliders.append(primitive('SPHERE', (-1.0, -1.0, -1.0), (cell, cell, cell)))
        settings = PressureSettings(velocity_advection='MACCORMACK', scalar_advection='MACCORMACK', thermal_lift=1.0,
                                    density_weight=0.05, dissipation=0.0, cooling=0.0, heat_mode='TARGET',
                                    pressure_tolerance=1e-4, pressure_max_cycles=200, solid_warm_start=warm_start,
                                    mg_coarse_scale=coarse_scale)
        noise = [rng.uniform(-1e-3, 1e-3, (fs[2], fs[1], fs[0])).astype(np.float32) for fs in grid.face_shapes]
        out.append((grid, settings, tuple(colliders), emitters, noise))
    return out


def build_solvers(scenes, device):
    """One ``DenseProjectedSmoke`` per scene, fields uploaded (zero scalars,
    seeded face noise)."""
    from .projected import DenseProjectedSmoke
    solvers, sources = [], []
    for grid, settings, colliders, emitters, noise in scenes:
        s = DenseProjectedSmoke(grid, settings, device, colliders=colliders)
        s.upload(torch.zeros(grid.cells))
        s.upload_temperature(torch.zeros(grid.cells))
        s.upload_velocity([torch.as_tensor(v) for v in noise])
        solvers.append(s)
        sources.append(emitters)
    return solvers, sources


def cell_updates(solvers):
    return sum(prod(s.grid.shape) for s in solvers)
