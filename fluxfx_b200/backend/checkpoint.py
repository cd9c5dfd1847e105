"""Versioned checkpoints of a ``DenseProjectedSmoke`` run (save, load, resume).

Drop-in for FluxFX ``fluxfx/backend/checkpoint.py:14-77``: the
``fluxfx-checkpoint-1`` format is one compressed ``.npz`` holding a JSON
``metadata`` string (format, settings, grid, time, steps, last_dt) and the
fields as flat x-fast FP32 arrays -- ``density``, ``temperature``,
``pressure``, ``velocity0..2`` and, with combustion, ``fuel`` and ``flame``.
The write goes to ``<path>.tmp`` first and replaces ``path`` only when it
completed, so a failed write leaves the previous checkpoint intact. The load
validates the clock, ``last_dt``, every field's length and finiteness and the
non-negative fields, as the reference does.

Keeping the reference's readers working: ``settings`` holds only the
reference's setting fields; the settings this build adds (tolerance, storage,
solver variants, ...) and the grid's axis limit go under ``extensions``,
which a reference reader ignores.

Extension -- static colliders: the reference refuses to save a solver with
colliders. Here their descriptors (shape and affine inverse rows) are saved
under the format name ``fluxfx-checkpoint-1+colliders`` (so a reader of the
plain v1 format rejects the file instead of resuming without them) and the
mask is rasterised again on load, bit-identical. Moving colliders (whose wall
velocities depend on the last move) stay outside the format, as in the
reference.

A loaded solver resumes bit-identically: the next steps equal those of the
solver that was saved (FP32 arrays hold BF16 storage exactly; the projector's
pressure and previous dt are restored after the uploads that reset them).
"""
import json
from dataclasses import asdict, fields as dc_fields
from math import isfinite, prod
from pathlib import Path

import numpy as np
import torch

from ..physics.collision import Collider
from ..physics.config import REFERENCE_AXIS_LIMIT, GridSpec, validate_dt
from ..physics.pressure import PressureSettings
from .projected import DenseProjectedSmoke

FORMAT = 'fluxfx-checkpoint-1'
FORMAT_COLLIDERS = 'fluxfx-checkpoint-1+colliders'

# Settings this build adds to the reference's PressureSettings.
EXTENSION_SETTINGS = ('pressure_tolerance', 'pressure_max_cycles', 'mg_pre_sweeps', 'mg_post_sweeps',
                      'mg_max_levels', 'heat_mode', 'velocity_blend', 'storage', 'solid_warm_start',
                      'pressure_method', 'learned_warm_start', 'mg_coarse_scale', 'learned_correction',
                      'ir_inner_cycles', 'warm_start_extrapolation', 'mg_coarse_sweeps',
                      'warm_start_order')
_TUPLES = ('velocity', 'source_center')


def _host(t):
    return t.detach().to(torch.float32).reshape(-1).cpu().numpy()


def save_checkpoint(solver, path):
    """Write ``solver``'s state to ``path`` (``backend/checkpoint.py:14-38``)."""
    if solver.faulted:
        raise ValueError('Checkpoint v1 requires a healthy solver')
    if solver.solids is not None and solver.settings.moving_colliders:
        raise ValueError('Checkpoint v1 excludes moving colliders')
    settings = asdict(solver.settings)
    extensions = {name: settings.pop(name) for name in EXTENSION_SETTINGS}
    if solver.grid.axis_limit != REFERENCE_AXIS_LIMIT:
        extensions['axis_limit'] = solver.grid.axis_limit
    meta = {'format': FORMAT if solver.solids is None else FORMAT_COLLIDERS, 'settings': settings,
            'grid': {'shape': list(solver.grid.shape), 'extent': list(solver.grid.extent)},
            'time': solver.time, 'steps': solver.steps, 'last_dt': solver.projector.previous_dt(),
            'extensions': extensions}
    if solver.solids is not None:
        meta['colliders'] = [{'shape': c.shape, 'inverse_rows': [list(r) for r in c.inverse_rows]}
                             for c in solver.solids.colliders]
    torch.cuda.synchronize(solver.device.device)
    arrays = {'density': _host(solver.density), 'temperature': _host(solver.temperature),
              'pressure': _host(solver.projector.pressure)}
    arrays.update({f'velocity{i}': _host(v) for i, v in enumerate(solver._velocity)})
    if solver.combustion is not None:
        arrays.update(fuel=_host(solver.combustion.fuel), flame=_host(solver.combustion.flame))
    if any(not np.isfinite(a).all() for a in arrays.values()):
        raise ValueError('Nonfinite checkpoint state')
    path = Path(path)
    temporary = path.with_name(path.name + '.tmp')
    try:
        with temporary.open('wb') as stream:
            np.savez_compressed(stream, metadata=json.dumps(meta), **arrays)
        temporary.replace(path)
    finally:
        if temporary.exists():
            temporary.unlink()


def _settings(meta):
    options = dict(meta['settings'])
    options.update({k: v for k, v in meta.get('extensions', {}).items() if k in EXTENSION_SETTINGS})
    known = {f.name for f in dc_fields(PressureSettings)}
    unknown = sorted(set(options) - known)
    if unknown:
        raise ValueError('Unknown checkpoint settings: ' + ', '.join(unknown))
    for name in _TUPLES:
        if name in options:
            options[name] = tuple(options[name])
    return PressureSettings(**options)


def load_checkpoint(path, device=None):
    """A new solver resuming the checkpoint at ``path``
    (``backend/checkpoint.py:41-69``); ``device`` as ``DenseProjectedSmoke``'s."""
    with np.load(path, allow_pickle=False) as archive:
        meta = json.loads(str(archive['metadata']))
        if meta.get('format') not in (FORMAT, FORMAT_COLLIDERS):
            raise ValueError('Unsupported checkpoint format')
        ext = meta.get('extensions', {})
        grid = GridSpec(tuple(meta['grid']['shape']), tuple(meta['grid']['extent']),
                        axis_limit=int(ext.get('axis_limit', REFERENCE_AXIS_LIMIT)))
        settings = _settings(meta)
        if not isfinite(meta['time']) or meta['time'] < 0 or type(meta['steps']) is not int or meta['steps'] < 0:
            raise ValueError('Invalid checkpoint clock')
        if meta['last_dt'] is not None:
            validate_dt(meta['last_dt'])
        colliders = ()
        if meta['format'] == FORMAT_COLLIDERS:
            colliders = tuple(Collider(c['shape'], tuple(tuple(float(v) for v in r) for r in c['inverse_rows']))
                              for c in meta.get('colliders', ()))
            if not colliders:
                raise ValueError('Collider checkpoint without colliders')
            if settings.moving_colliders:
                raise ValueError('Checkpoint v1 excludes moving colliders')
        shapes = {k: grid.shape for k in ('density', 'temperature', 'pressure')}
        shapes.update({f'velocity{i}': s for i, s in enumerate(grid.face_shapes)})
        if settings.combustion_enabled:
            shapes.update(fuel=grid.shape, flame=grid.shape)
        arrays = {}
        for k in shapes:
            if k not in archive:
                raise ValueError('Missing field: ' + k)
            arrays[k] = archive[k].copy()
        for k, a in arrays.items():
            if a.dtype != np.float32 or a.shape != (prod(shapes[k]),) or not np.isfinite(a).all():
                raise ValueError('Invalid field: ' + k)
            if k in {'density', 'fuel', 'flame'} and (a < 0).any():
                raise ValueError('Negative field: ' + k)
    solver = DenseProjectedSmoke(grid, settings, device, colliders=colliders)
    try:
        if settings.learned_warm_start:
            from ..learned import attach
            attach(solver, colliders)
        solver.upload(torch.from_numpy(arrays['density']))
        solver.upload_temperature(torch.from_numpy(arrays['temperature']))
        solver.upload_velocity([torch.from_numpy(arrays[f'velocity{i}']) for i in range(3)])
        # the uploads reset the projector: restore its warm-start state afterwards
        p = solver.projector.pressure
        p.copy_(torch.from_numpy(arrays['pressure']).reshape(p.shape).to(p.device, p.dtype))
        solver.projector.last_dt = meta['last_dt']
        solver.projector.ready = False      # divergence diagnostics recomputed on the next step
        if solver.combustion is not None:
            for name in ('fuel', 'flame'):
                t = getattr(solver.combustion, name)
                t.copy_(torch.from_numpy(arrays[name]).reshape(t.shape).to(t.device, t.dtype))
        solver.time, solver.steps = meta['time'], meta['steps']
        return solver
    except Exception:
        solver.close()
        raise


def advance_fixed(solver, steps, dt, sources=None):
    """Offline reproducible input schedule: ``steps`` steps of ``dt``
    (``backend/checkpoint.py:72-77``; static colliders allowed here)."""
    validate_dt(dt)
    if type(steps) is not int or steps < 0:
        raise ValueError('Steps must be a nonnegative integer')
    if solver.solids is not None and solver.settings.moving_colliders:
        raise ValueError('Fixed checkpoint runner v1 excludes moving colliders')
    for _ in range(steps):
        solver.step(dt, sources=sources)
