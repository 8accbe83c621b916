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

For the batched 2D TE engine (one coefficient per cell) the permittivity is
the linear interpolation of config 4. For a 3D scene, ``EtchedCore`` builds
the reference's substrate / etched core / cladding stack with its
anisotropic diagonal tensor in torch on top of the same kernels (wrapped as
a ``torch.autograd.Function``), and ``value_and_grad_density3d`` carries the
engine's per-component adjoint back to the density.
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


# --------------------------------------------------------------------------- #
# The etched-core layer stack for 3D scenes (design.py:75-175), in torch, so
# that its gradient flows into adjoint.value_and_grad_params.
# --------------------------------------------------------------------------- #
def _density_function():
    import torch

    class DensityFunction(torch.autograd.Function):
        """rho (n, n) CUDA float64 -> tanh_projection(conic_filter(rho)) by
        pfd_density_forward; the reverse pass by pfd_density_backward."""

        @staticmethod
        def forward(ctx, rho, radius_cells, beta, eta):
            x = rho.detach().contiguous()
            y = torch.empty_like(x)
            st = C.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
            _check(N.lib().pfd_density_forward(1, x.shape[0], C.c_void_p(x.data_ptr()),
                                               float(radius_cells), float(beta), float(eta),
                                               C.c_void_p(y.data_ptr()), st))
            ctx.save_for_backward(x)
            ctx.args = (float(radius_cells), float(beta), float(eta))
            return y

        @staticmethod
        def backward(ctx, g):
            (x,) = ctx.saved_tensors
            gp = g.detach().contiguous().to(torch.float64)
            out = torch.empty_like(x)
            st = C.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
            r, b, e = ctx.args
            _check(N.lib().pfd_density_backward(1, x.shape[0], C.c_void_p(x.data_ptr()), r, b, e,
                                                C.c_void_p(gp.data_ptr()),
                                                C.c_void_p(out.data_ptr()), st))
            return out, None, None, None

    return DensityFunction


def _gradient(f, h, axis):
    """numpy.gradient(f, h, axis) in torch: central differences inside,
    one-sided first-order differences at both ends."""
    import torch
    n = f.shape[axis]
    if n < 2:
        return torch.zeros_like(f)
    lo = f.narrow(axis, 0, 1)
    hi = f.narrow(axis, n - 1, 1)
    first = (f.narrow(axis, 1, 1) - lo) / h
    last = (hi - f.narrow(axis, n - 2, 1)) / h
    if n == 2:
        return torch.cat([first, last], dim=axis)
    mid = (f.narrow(axis, 2, n - 2) - f.narrow(axis, 0, n - 2)) / (2.0 * h)
    return torch.cat([first, mid, last], dim=axis)


class EtchedCore:
    """A substrate / patterned core / cladding stack driven by a 2D density
    (the reference's EtchedCore, design.py:75-161): ``eps_solid`` /
    ``eps_void`` in the core where material stays / is etched, ``eps_sub``
    below and ``eps_clad`` above the core layer ``core_z = (z0, z1)``;
    ``filter_radius`` (m), ``beta``, ``eta`` as conic_filter /
    tanh_projection. The core's diagonal permittivity blends the arithmetic
    and harmonic means of the two materials along the in-plane normal of the
    physical density (vertical sidewalls): eps_xx, eps_yy from the normal,
    eps_zz the arithmetic mean. The density is (nx, ny), square, at most
    96 x 96 (the filter kernels' window)."""

    def __init__(self, eps_solid: float, eps_void: float, eps_sub: float, eps_clad: float,
                 core_z: Tuple[float, float], filter_radius: float = 0.0, beta: float = 0.0,
                 eta: float = 0.5):
        self.eps_solid, self.eps_void = float(eps_solid), float(eps_void)
        self.eps_sub, self.eps_clad = float(eps_sub), float(eps_clad)
        self.core_z = (float(core_z[0]), float(core_z[1]))
        self.filter_radius, self.beta, self.eta = float(filter_radius), float(beta), float(eta)

    def rho_phys(self, rho, dx: float):
        """Filtered and projected density (a differentiable torch tensor)."""
        import torch
        rho = torch.as_tensor(rho, dtype=torch.float64)
        if rho.ndim != 2 or rho.shape[0] != rho.shape[1]:
            raise ValueError("the density must be square (n, n), n <= 96")
        rho = rho.cuda() if not rho.is_cuda else rho
        return _density_function().apply(rho, self.filter_radius / dx, self.beta, self.eta)

    def eps_components(self, grid, rho):
        """(eps_xx, eps_yy, eps_zz) of shape grid.shape for the raw density
        ``rho`` (nx, ny) (design.py:109-148), torch float64 on the device."""
        import torch
        nx, ny, nz = grid.shape
        dx = grid.cell_size[0]
        dy = grid.cell_size[1] if grid.shape[1] > 1 else dx
        rp = self.rho_phys(rho, dx)
        if tuple(rp.shape) != (nx, ny):
            raise ValueError(f"the density must be {(nx, ny)} for this grid")
        de = self.eps_solid - self.eps_void
        eps_a = self.eps_void + rp * de
        eps_h = 1.0 / (rp / self.eps_solid + (1.0 - rp) / self.eps_void)
        gx, gy = _gradient(rp, dx, 0), _gradient(rp, dy, 1)
        gmag = torch.sqrt(gx * gx + gy * gy)
        safe = gmag > (gmag.max() * 1e-9 + 1e-30)
        inv = torch.where(safe, 1.0 / torch.where(safe, gmag, torch.ones_like(gmag)),
                          torch.zeros_like(gmag))
        nxc, nyc = gx * inv, gy * inv
        delta = eps_h - eps_a
        exx = eps_a + delta * nxc * nxc
        eyy = eps_a + delta * nyc * nyc
        ezz = eps_a
        zc = np.asarray(grid.coords[2])
        core = torch.as_tensor(((zc >= self.core_z[0]) & (zc < self.core_z[1])).astype(float),
                               device=rp.device).reshape(1, 1, nz)
        bg = torch.as_tensor(np.where(zc < self.core_z[0], self.eps_sub, self.eps_clad),
                             device=rp.device).reshape(1, 1, nz)

        def extrude(e):
            return e[:, :, None] * core + bg * (1.0 - core)

        return extrude(exx), extrude(eyy), extrude(ezz)

    def ce_builder(self, sim):
        """rho -> {'Ex', 'Ey', 'Ez'} E coefficients dt / (eps0 eps_cc) for
        adjoint.value_and_grad_params (design.py:150-161)."""
        from .scene import EPS_0
        dt, grid = float(sim.dt), sim.grid

        def ce_of_rho(rho):
            exx, eyy, ezz = self.eps_components(grid, rho)
            return {"Ex": dt / (exx * EPS_0), "Ey": dt / (eyy * EPS_0), "Ez": dt / (ezz * EPS_0)}

        return ce_of_rho


def value_and_grad_density3d(sim, etched_core: EtchedCore, rho, loss, checkpoint_every=None):
    """(value, d loss / d rho) of a 3D scene whose core layer is set by the
    2D density ``rho`` through ``etched_core`` (design.py:164-175
    value_and_grad_density): the engine's adjoint per component, then torch
    through the stack and the GPU filter / projection kernels."""
    from .adjoint import value_and_grad_params
    return value_and_grad_params(sim, etched_core.ce_builder(sim), rho, loss, checkpoint_every)
