"""Neumann pseudoinverse of the cell-centred 7-point Laplacian on a small box.

The 4^3 case is FluxFX ``fluxfx/physics/coarse_pressure.py:6-24`` (row-major
64x64 table, rows map a mean-free right-hand side to zero-mean pressure).
The same closed form -- the separable cosine eigenbasis of the Neumann
Laplacian, eigenvalue -4 (n/L)^2 sin^2(pi k / 2n) per axis -- is evaluated for
any small shape, so the coarsest multigrid level may be 8^3 (512 cells).
"""
from functools import lru_cache
from math import prod

import numpy as np

MAX_DIRECT_CELLS = 512


def _axis_basis(n, length):
    k = np.arange(n, dtype=np.float64)[:, None]          # mode
    c = np.arange(n, dtype=np.float64)[None, :]          # cell
    norm = np.where(k == 0, np.sqrt(1.0 / n), np.sqrt(2.0 / n))
    basis = norm * np.cos(np.pi * k * (c + .5) / n)      # (mode, cell), orthonormal
    eig = -4.0 * (n / length) ** 2 * np.sin(np.pi * k[:, 0] / (2 * n)) ** 2
    return basis, eig


@lru_cache(maxsize=16)
def _neumann_inverse_cached(shape, extent):
    if prod(shape) > MAX_DIRECT_CELLS:
        raise ValueError(f"Direct coarse solve is limited to {MAX_DIRECT_CELLS} cells")
    (bx, ex), (by, ey), (bz, ez) = (_axis_basis(n, e) for n, e in zip(shape, extent))
    # Eigenvalue of mode (kx, ky, kz), flattened x-fast like the cells.
    lam = (ez[:, None, None] + ey[None, :, None] + ex[None, None, :]).ravel()
    modes = np.einsum('ia,jb,kc->ijkabc', bz, by, bx).reshape(prod(shape), prod(shape))
    # modes[m, cell]: m = kx + nx*(ky + ny*kz), cell = x + nx*(y + ny*z)
    inv_lam = np.zeros_like(lam)
    inv_lam[1:] = 1.0 / lam[1:]  # drop the constant (null) mode
    return (modes.T * inv_lam) @ modes


def neumann_inverse(shape, extent):
    """(N, N) float64 pseudoinverse; N = prod(shape), x-fast cell order."""
    return _neumann_inverse_cached(tuple(int(n) for n in shape), tuple(float(e) for e in extent)).copy()


def coarse_inverse(extent):
    """The reference's 4^3 table: 4096 floats, row-major (row = output cell)."""
    return tuple(neumann_inverse((4, 4, 4), extent).ravel().tolist())
