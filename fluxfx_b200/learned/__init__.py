"""Learned pressure warm start (U-Net on the library's BF16 tensor-core convolutions)."""


def attach(solver, colliders, weights=None):
    """Give a collider solver (``DenseProjectedSmoke``) the trained network as
    its pressure guess; the solver uses it when its settings set
    ``learned_warm_start``. Returns the ``LearnedWarmStart``."""
    from .warm_start import LearnedWarmStart
    model = LearnedWarmStart(solver.grid, colliders, solver.device, weights=weights)
    solver.projector.attach_learned(model)
    return model
