"""NumPy restatement of the reference's density chain (test infrastructure).

The checker of csrc/design.cu; never imported by the product. Restates
src/photonfdtd/design.py: conic_filter (:40-58), which the reference computes
with jax.scipy.signal.convolve(mode="same") - the same-size, zero-padded full
convolution that scipy.signal.convolve computes here (JAX is not installed
where these tests run; its convolve mirrors scipy's semantics) - and
tanh_projection (:61-72). The reverse pass is written out as explicit
transposes, and tests/test_design_oracle.py pins it to central differences.
"""
from __future__ import annotations

import numpy as np
from scipy.signal import convolve


def cone(radius_cells: float) -> np.ndarray:
    """The filter kernel of design.py:50-54."""
    r = int(np.ceil(radius_cells))
    ax = np.arange(-r, r + 1)
    xx, yy = np.meshgrid(ax, ax, indexing="ij")
    return np.maximum(0.0, 1.0 - np.sqrt(xx ** 2 + yy ** 2) / radius_cells)


def conic_filter(rho: np.ndarray, radius_cells: float) -> np.ndarray:
    r = int(np.ceil(radius_cells))
    if r < 1:
        return np.asarray(rho, np.float64)
    k = cone(radius_cells)
    num = convolve(rho, k, mode="same", method="direct")
    den = convolve(np.ones_like(rho), k, mode="same", method="direct")
    return num / den


def tanh_projection(rho: np.ndarray, beta: float = 8.0, eta: float = 0.5) -> np.ndarray:
    if beta <= 0:
        return np.asarray(rho, np.float64)
    num = np.tanh(beta * eta) + np.tanh(beta * (rho - eta))
    den = np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta))
    return num / den


def forward(rho, radius_cells=0.0, beta=0.0, eta=0.5):
    return tanh_projection(conic_filter(np.asarray(rho, np.float64), radius_cells), beta, eta)


def backward(rho, grad_phys, radius_cells=0.0, beta=0.0, eta=0.5):
    """(d forward / d rho)^T grad_phys."""
    rho = np.asarray(rho, np.float64)
    g = np.asarray(grad_phys, np.float64)
    y = conic_filter(rho, radius_cells)
    if beta > 0:
        den = np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta))
        g = g * beta * (1.0 - np.tanh(beta * (y - eta)) ** 2) / den
    if int(np.ceil(radius_cells)) < 1:
        return g
    k = cone(radius_cells)
    den = convolve(np.ones_like(rho), k, mode="same", method="direct")
    # y = C rho / d with C a symmetric-kernel same-size convolution: C^T = C
    return convolve(g / den, k, mode="same", method="direct")


def etched_core_eps(grid, rho, eps_solid, eps_void, eps_sub, eps_clad, core_z,
                    filter_radius=0.0, beta=0.0, eta=0.5):
    """(eps_xx, eps_yy, eps_zz) of the reference's EtchedCore.eps_components
    (design.py:109-148) in NumPy: the physical density, the arithmetic and
    harmonic means, the in-plane normal from numpy.gradient, the blend along
    the normal, and the extrusion through the substrate / core / cladding
    stack."""
    nx, ny, nz = grid.shape
    dx = grid.cell_size[0]
    dy = grid.cell_size[1] if grid.shape[1] > 1 else dx
    rp = forward(np.asarray(rho, np.float64), filter_radius / dx, beta, eta)
    eps_a = eps_void + rp * (eps_solid - eps_void)
    eps_h = 1.0 / (rp / eps_solid + (1.0 - rp) / eps_void)
    gx = np.gradient(rp, dx, axis=0)
    gy = np.gradient(rp, dy, axis=1)
    gmag = np.sqrt(gx ** 2 + gy ** 2)
    safe = gmag > (gmag.max() * 1e-9 + 1e-30)
    inv = np.where(safe, 1.0 / np.where(safe, gmag, 1.0), 0.0)
    nxc, nyc = gx * inv, gy * inv
    delta = eps_h - eps_a
    comps = (eps_a + delta * nxc ** 2, eps_a + delta * nyc ** 2, eps_a)
    zc = np.asarray(grid.coords[2])
    core = ((zc >= core_z[0]) & (zc < core_z[1])).astype(float).reshape(1, 1, nz)
    bg = np.where(zc < core_z[0], eps_sub, eps_clad).reshape(1, 1, nz)
    return tuple(c[:, :, None] * core + bg * (1.0 - core) for c in comps)
