"""The density chain of topology optimisation, on the GPU.

Mirrors the reference's src/photonfdtd/design.py: ``conic_filter`` (:40-58),
``tanh_projection`` (:61-72) and ``value_and_grad_density`` (:164-175), which
the reference evaluates and differentiates with JAX. Here the filter and the
projection are CUDA kernels with a hand-written reverse pass
(csrc/design.cu, ``pfd_density_forward`` / ``pfd_density_backward``), over a
batch of n x n design windows in float64, and the gradient flows on through
the batched 2D TE adjoint (photonfdtd_b200.batch):

    rho --conic filter--> --tanh projection--> rho_phys
        --> eps = eps_lo + rho_phys (eps_hi - eps_lo) --> FDTD --> loss

The reference's EtchedCore builds an anisotropic subpixel tensor for a 3D
etched layer; the batched engine steps 2D TE instances with one coefficient
per cell, so the permittivity here is the linear interpolation of config 4.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional, Tuple

import numpy as np

from . import _native as N
from .workloads import EPS_CLAD, EPS_CORE


def _check(rc: int) -> None:
    if rc != N.PF_OK:
        msg = N.lib().pfd_last_error().decode(errors="replace")
        if rc == N.PF_ERR_INVALID:
            raise ValueError(msg)
        raise N.NativeError(rc, msg)


def _batch(rho) -> Tuple[np.ndarray, bool]:
    a = np.ascontiguousarray(rho, dtype=np.float64)
    single = a.ndim == 2
    if single:
        a = a[None]
    if a.ndim != 3 or a.shape[1] != a.shape[2]:
        raise ValueError("densities must be (n, n) or (n_inst, n, n)")
    return a, single


def density_forward(rho, radius_cells: float = 0.0, beta: float = 0.0,
                    eta: float = 0.5) -> np.ndarray:
    """tanh_projection(conic_filter(rho, radius_cells), beta, eta) of one
    (n, n) window or a batch (n_inst, n, n), on the GPU."""
    import torch
    a, single = _batch(rho)
    x = torch.from_numpy(a).cuda()
    y = torch.empty_like(x)
    _check(N.lib().pfd_density_forward(a.shape[0], a.shape[1], C.c_void_p(x.data_ptr()),
                                       float(radius_cells), float(beta), float(eta),
                                       C.c_void_p(y.data_ptr()), None))
    out = y.cpu().numpy()
    return out[0] if single else out


def density_backward(rho, grad_phys, radius_cells: float = 0.0, beta: float = 0.0,
                     eta: float = 0.5) -> np.ndarray:
    """The transpose of density_forward's Jacobian at rho applied to
    grad_phys = dL/d rho_phys: dL/d rho."""
    import torch
    a, single = _batch(rho)
    g, _ = _batch(grad_phys)
    if g.shape != a.shape:
        raise ValueError("grad_phys must have the shape of rho")
    x = torch.from_numpy(a).cuda()
    gp = torch.from_numpy(g).cuda()
    out = torch.empty_like(x)
    _check(N.lib().pfd_density_backward(a.shape[0], a.shape[1], C.c_void_p(x.data_ptr()),
                                        float(radius_cells), float(beta), float(eta),
                                        C.c_void_p(gp.data_ptr()), C.c_void_p(out.data_ptr()),
                                        None))
    r = out.cpu().numpy()
    return r[0] if single else r


def conic_filter(rho, radius_cells: float) -> np.ndarray:
    """design.py:40-58 on the GPU: the normalised cone-kernel filter."""
    return density_forward(rho, radius_cells, 0.0)


def tanh_projection(rho, beta: float = 8.0, eta: float = 0.5) -> np.ndarray:
    """design.py:61-72 on the GPU: smooth threshold toward 0 / 1."""
    return density_forward(rho, 0.0, beta, eta)


class DensityChain:
    """rho (n_inst, n, n) -> the batch's packed design permittivity and back.

    eps = eps_lo + rho_phys (eps_hi - eps_lo) with rho_phys the filtered and
    projected density; ``radius_cells`` / ``beta`` / ``eta`` as the reference's
    EtchedCore(filter_radius / dx, beta, eta)."""

    def __init__(self, radius_cells: float = 0.0, beta: float = 0.0, eta: float = 0.5,
                 eps_lo: float = EPS_CLAD, eps_hi: float = EPS_CORE):
        self.radius_cells = float(radius_cells)
        self.beta = float(beta)
        self.eta = float(eta)
        self.eps_lo = float(eps_lo)
        self.eps_hi = float(eps_hi)

    def rho_phys(self, rho) -> np.ndarray:
        return density_forward(rho, self.radius_cells, self.beta, self.eta)

    def eps(self, rho) -> np.ndarray:
        return self.eps_lo + self.rho_phys(rho) * (self.eps_hi - self.eps_lo)

    def grad_rho(self, rho, grad_eps) -> np.ndarray:
        g = np.asarray(grad_eps, np.float64) * (self.eps_hi - self.eps_lo)
        return density_backward(rho, g, self.radius_cells, self.beta, self.eta)


def value_and_grad_density(batch, rho, chain: Optional[DensityChain] = None,
                           loss: Optional[Callable] = None):
    """(values, dloss/drho) for every instance of a BatchTE whose design
    windows are n x n: rho (n_inst, n, n) raw densities through ``chain``
    (default: no filter, no projection), the batch's forward and adjoint, and
    the chain's reverse pass. Mirrors value_and_grad_density(sim,
    etched_core, rho, loss) (design.py:164-175), batched. ``loss`` as in
    batch.value_and_grad_eps (default: per-instance sum of |DFT|^2)."""
    from .batch import value_and_grad_eps
    chain = DensityChain() if chain is None else chain
    r, _ = _batch(rho)
    n = {w[2] for w in batch.windows}
    if len(n) != 1 or r.shape != (batch.n_inst, n.pop(), r.shape[2]):
        raise ValueError("rho must be (n_inst, n, n) with every window n x n")
    eps = chain.eps(r)
    vals, g_eps = value_and_grad_eps(batch, eps.reshape(-1), loss)
    return vals, chain.grad_rho(r, g_eps.reshape(r.shape))
