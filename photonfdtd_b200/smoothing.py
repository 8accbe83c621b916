"""Diagonal anisotropic subpixel permittivity (host precompute).

Same tensor as src/photonfdtd/smoothing.py:119-172: per native cell, the
arithmetic mean eps_a and harmonic mean eps_h of the permittivity over
``factor`` sub-cells per active axis; the interface normal n is the
normalised gradient of eps_a; eps_ii = eps_a + (eps_h - eps_a) * n_i^2. The
means use numpy's block mean over the reshaped sub-cell axes, so the values
are bit-identical to the reference's. Box structures rasterise through index
ranges instead of full boolean masks.
"""
from __future__ import annotations

from types import SimpleNamespace
from typing import Tuple

import numpy as np

from .scene import Grid


def _fine_coords(grid, factor):
    """Coordinates of the grid refined ``factor`` times on each active axis
    (a Grid of the same size with cell/factor spacing, no PML)."""
    cs = tuple((c / factor) if c > 0 else 0.0 for c in grid.cell_size)
    return Grid(size=grid.size, cell_size=cs, pml_layers=(0, 0, 0)).coords


def _stamp_sub(structure, sub, duck):
    if hasattr(structure, "index_slices"):
        sl = structure.index_slices(duck)
        if sl is not None:
            sub[sl] = structure.medium.eps_r
    else:
        sub[structure.region_mask(duck)] = structure.medium.eps_r


def slab_means(grid, structures, background_eps: float, factor: int):
    """(eps_a, eps_h) float64 per native cell, built one x-slab at a time."""
    nx, ny, nz = grid.shape
    xf, yf, zf = _fine_coords(grid, factor)
    fx = factor if nx > 1 else 1
    fy = factor if ny > 1 else 1
    fz = factor if nz > 1 else 1
    eps_a = np.empty(grid.shape, dtype=np.float64)
    eps_h = np.empty(grid.shape, dtype=np.float64)
    for i in range(nx):
        xs = xf[i * fx:(i + 1) * fx]
        duck = SimpleNamespace(shape=(xs.size, yf.size, zf.size), coords=(xs, yf, zf))
        sub = np.full(duck.shape, float(background_eps), dtype=np.float64)
        for s in structures:
            _stamp_sub(s, sub, duck)
        r = sub.reshape(1, fx, ny, fy, nz, fz)
        eps_a[i] = r.mean(axis=(1, 3, 5))[0]
        eps_h[i] = (1.0 / (1.0 / r).mean(axis=(1, 3, 5)))[0]
    return eps_a, eps_h


def smooth_permittivity(grid, structures, background_eps: float = 1.0, factor: int = 3,
                        dtype=np.float64) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(eps_xx, eps_yy, eps_zz) for the Ex, Ey, Ez updates."""
    if factor < 1:
        raise ValueError("factor must be >= 1")
    shape = grid.shape
    eps_a, eps_h = slab_means(grid, structures, background_eps, factor)
    spacing = [grid.cell_size[a] if shape[a] > 1 else 1.0 for a in range(3)]
    grads = [np.gradient(eps_a, spacing[a], axis=a) if shape[a] > 1 else np.zeros_like(eps_a)
             for a in range(3)]
    gmag = np.sqrt(grads[0] ** 2 + grads[1] ** 2 + grads[2] ** 2)
    tiny = gmag.max() * 1e-9 if gmag.size else 0.0
    ok = gmag > max(tiny, np.finfo(np.float64).tiny)
    inv = np.where(ok, 1.0 / np.where(ok, gmag, 1.0), 0.0)
    normal = [g * inv for g in grads]
    delta = eps_h - eps_a
    return tuple((eps_a + delta * normal[a] ** 2).astype(dtype, copy=False) for a in range(3))
