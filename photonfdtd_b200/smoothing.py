"""Diagonal anisotropic subpixel permittivity (host precompute).

Same tensor as src/photonfdtd/smoothing.py:119-172: per native cell, the
arithmetic mean eps_a and harmonic mean eps_h of the permittivity over
``factor`` sub-cells per active axis; the interface normal n is the
normalised gradient of eps_a; eps_ii = eps_a + (eps_h - eps_a) * n_i^2. The
means use numpy's block mean over the reshaped sub-cell axes, so the values
are bit-identical to the reference's. Box structures rasterise through index
ranges instead of full boolean masks.

smooth_permittivity_device computes the same tensor on the GPU
(pf_smooth_boxes) for scenes made of boxes, bit for bit equal to
smooth_permittivity; Simulation uses it whenever a CUDA device is present.
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


def box_spans(grid, structures, factor: int):
    """(spans int32 (m, 6), eps float64 (m,)) of the boxes on the fine grid
    (half-open index ranges per axis), in stamping order; None when a
    structure is not a box (no index_slices)."""
    if not all(hasattr(s, "index_slices") for s in structures):
        return None
    xf, yf, zf = _fine_coords(grid, factor)
    nx = grid.shape[0]
    # slab_means stamps one x-slab of factor fine cells at a time; a slab one
    # cell thick (factor 1) takes the box rasterisation's collapsed-axis rule
    # (covered in full when the box's x extent straddles 0, else not at all),
    # so its x span is all or nothing, as on the host
    thin = nx > 1 and factor == 1
    xd = xf[:1] if thin else xf
    duck = SimpleNamespace(shape=(xd.size, yf.size, zf.size), coords=(xd, yf, zf))
    spans, eps = [], []
    for s in structures:
        sl = s.index_slices(duck)
        if sl is None:
            continue
        xs = (0, nx) if thin else (sl[0].start, sl[0].stop)
        spans.append([*xs, sl[1].start, sl[1].stop, sl[2].start, sl[2].stop])
        eps.append(float(s.medium.eps_r))
    return np.array(spans, np.int32).reshape(-1, 6), np.array(eps, np.float64)


def device_available() -> bool:
    try:
        import torch
        return bool(torch.cuda.is_available())
    except Exception:  # noqa: BLE001 - no CUDA runtime
        return False


def smooth_permittivity_device(grid, structures, background_eps: float = 1.0, factor: int = 3,
                               dtype=np.float64) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """smooth_permittivity for scenes made of boxes, on the GPU."""
    from . import _native as N
    if factor < 1:
        raise ValueError("factor must be >= 1")
    bs = box_spans(grid, structures, factor)
    if bs is None:
        raise NotImplementedError("GPU smoothing takes box structures only")
    spans, eps = bs
    dt = np.dtype(dtype)
    if dt not in (np.dtype(np.float32), np.dtype(np.float64)):
        raise ValueError("dtype must be float32 or float64")
    out = tuple(np.empty(grid.shape, dt) for _ in range(3))
    h = [grid.cell_size[a] if grid.shape[a] > 1 else 1.0 for a in range(3)]
    L = N.lib()
    rc = L.pf_smooth_boxes(*grid.shape, int(factor), float(background_eps), int(len(eps)),
                           spans.ctypes.data if len(eps) else None,
                           eps.ctypes.data if len(eps) else None, *[float(v) for v in h],
                           dt.itemsize, *[o.ctypes.data for o in out])
    if rc != N.PF_OK:
        raise N.NativeError(rc, L.pf_smooth_last_error().decode())
    return out
