"""The trained U-Net as the pressure solver's initial guess.

``LearnedWarmStart(grid, colliders, device)`` predicts the impulse pressure of
a projection from its divergence (``projector.before``) and the collider
mask. Grids up to 128 cells per axis run the network at their own
resolution; larger grids run it on 2x2x2 averages of the divergence, halving
the resolution until no axis exceeds 128 cells (dimensions divisible by 8 x
the factor), with the collider mask restricted alongside (a coarse cell is
solid when at least four of its children are, so moving colliders are followed
at every guess); the prediction is prolonged back trilinearly, one halving at a
time. Every pass is a library kernel
(``ffx_mg_restrict``, ``ffx_mask_restrict``, ``ffx_max_abs``,
``ffx_pack_input`` + the convolutions, ``ffx_unpack_channel``,
``ffx_mg_prolong``); torch only allocates.

Attach it with ``projector.attach_learned(model)`` and set
``learned_warm_start=True``: the solve then starts from the prediction when it
would otherwise start from zero (every step without ``solid_warm_start``; the
first step after a reset with it). The multigrid still iterates to the same
tolerance, so the plain method stays both the fallback and the arbiter.
"""
import ctypes as C
from pathlib import Path

import torch

from .. import _native as N
from ..backend.device import ptr
from .unet import HEAD_CHANNELS, UNet

WEIGHTS = Path(__file__).resolve().parent / 'weights' / 'unet128.pt'
MAX_NATIVE = 128


def weight_of(shape, extent):
    """Largest Laplacian conductance (n / extent)^2 of a grid."""
    return max((n / e) ** 2 for n, e in zip(shape, extent))


class LearnedWarmStart:
    """``device`` is the solver's device: a ``SolidDevice`` (its ``mask`` is
    read at every guess) or a plain device (no colliders)."""

    def __init__(self, grid, colliders, device, weights=None, net=None):
        base = getattr(device, 'base', device)
        self.device = base
        self.grid = grid
        # the network runs at most MAX_NATIVE cells per axis: on the grid itself, or on
        # restrictions by 2 per step (factor 2, 4, ...) with prolongations back
        self.factor = 1
        while max(grid.shape) // self.factor > MAX_NATIVE:
            self.factor *= 2
        shape = tuple(n // self.factor for n in grid.shape)
        if any(n % 8 for n in shape) or any(n % self.factor for n in grid.shape):
            raise ValueError('the network needs grid dimensions divisible by 8 x the restriction factor')
        self.shape = shape
        dev = base.device
        # shapes of the chain: the grid, then every restriction by 2 down to the network's
        self.shapes = [tuple(grid.shape)]
        while self.shapes[-1] != shape:
            self.shapes.append(tuple(n // 2 for n in self.shapes[-1]))
        self.fine_mask = getattr(device, 'mask', None) if colliders else None
        self.masks = [self.fine_mask] + [
            torch.zeros(sh[::-1], dtype=torch.uint8, device=dev) if self.fine_mask is not None else None
            for sh in self.shapes[1:]]
        self.mask = self.masks[-1] if self.fine_mask is not None else torch.zeros(shape[::-1], dtype=torch.uint8,
                                                                                  device=dev)
        self.weight = weight_of(shape, grid.extent)
        self.net = net or UNet(base.device, seed=0)
        if net is None:
            state = torch.load(weights or WEIGHTS)
            self.net.load_state_dict(state)
        # restricted divergences and prolonged predictions per coarse level, a zero field per fine level
        self.divs = [None] + [torch.empty(sh[::-1], dtype=torch.float32, device=dev) for sh in self.shapes[1:]]
        self.coarses = [None] + [torch.empty(sh[::-1], dtype=torch.float32, device=dev) for sh in self.shapes[1:]]
        self.zeros = [torch.zeros(sh[::-1], dtype=torch.float32, device=dev) for sh in self.shapes[:-1]]
        self._max = torch.zeros(1, dtype=torch.float32, device=dev)

    def guess(self, before, out):
        """Write the predicted pressure for the divergence ``before`` into ``out``."""
        dev = self.device
        s = dev.s
        src = before
        for k in range(1, len(self.shapes)):
            dev.call('ffx_mg_restrict', N.n3(*self.shapes[k - 1]), ptr(src), ptr(self.divs[k]), s)
            src = self.divs[k]
            if self.fine_mask is not None:
                dev.call('ffx_mask_restrict', N.n3(*self.shapes[k]), ptr(self.masks[k - 1]), 4, ptr(self.masks[k]), s)
        # the input scale 1 / max|div| stays on the device (no readback in the step);
        # a zero divergence gives a zero guess through the zero unpacking factor
        dev.call('ffx_max_abs', src.numel(), N.FFX_F32, ptr(src), ptr(self._max), s)
        calls = self.net.calls
        pred = self.net.forward(src.unsqueeze(0), self.mask.unsqueeze(0), None, s.value or 0, max_abs=self._max)
        dev.calls += self.net.calls - calls     # the network's launches count with the solver's
        last = len(self.shapes) - 1
        target = self.coarses[last] if last > 0 else out
        dev.call('ffx_unpack_channel_scaled', src.numel(), ptr(self.net.pred), HEAD_CHANNELS, ptr(self._max),
                 float(self.weight), ptr(target), s)
        for k in range(last, 0, -1):
            fine = out if k == 1 else self.coarses[k - 1]
            dev.call('ffx_mg_prolong', N.n3(*self.shapes[k - 1]), ptr(self.zeros[k - 1]), ptr(self.coarses[k]),
                     ptr(fine), s)
        return pred

    def close(self):
        self.net = None
        self.fine_mask = self.mask = None
        self.masks = self.divs = self.coarses = self.zeros = []
