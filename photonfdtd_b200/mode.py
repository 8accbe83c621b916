"""Full-vectorial waveguide mode solver on the GPU: the counterpart of the
reference's ``ModeSolver`` / ``ModeResult`` (src/photonfdtd/mode.py:86-387),
same constructor, same ``solve()`` result.

The reference assembles the transverse-E operator P (Zhu & Brown 2002) as a
scipy sparse matrix and asks ARPACK, in shift-invert mode about
(k0 n_max)^2, for the eigenvalues beta^2 nearest that shift. Here P is
applied matrix-free on the device (``pfm_apply``, csrc/modesolver.cu) and
the top of its spectrum is found by Chebyshev-filtered subspace iteration
(Zhou & Saad, J. Comput. Phys. 219, 2006): the filter (``pfm_chebyshev``)
damps the part of the spectrum below the current Ritz cut-off and amplifies
the guided modes above it; a Rayleigh-Ritz step on the filtered block (QR on
the device, a small dense eigensolve on the host) refines the estimates until
every wanted eigenpair has a relative residual below ``tol``. The guided
modes are the largest beta^2 and lie just below the reference's shift, so
both select the same modes. Sorting, the polarisation filter, the max |E_t|
normalisation and the recovered Ex / H fields follow the reference.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .scene import C_0, MU_0


@dataclass
class ModeResult:
    """Result of a mode solve; the reference's ModeResult fields
    (mode.py:86-125): wavelength, n_eff (descending), psi = |E_t| normalised
    to unit maximum, y, z axes, complex Ey, Ez (the solved unknowns), Ex and
    H recovered for inspection, a component dict and the cross-section
    permittivity."""
    wavelength: float
    n_eff: np.ndarray
    psi: np.ndarray
    y: np.ndarray
    z: np.ndarray
    Ey: Optional[np.ndarray] = None
    Ez: Optional[np.ndarray] = None
    Ex: Optional[np.ndarray] = None
    Hx: Optional[np.ndarray] = None
    Hy: Optional[np.ndarray] = None
    Hz: Optional[np.ndarray] = None
    fields: Optional[dict] = None
    eps_r: Optional[np.ndarray] = None
    iterations: int = 0
    max_residual: float = 0.0


class ModeSolver:
    """Waveguide modes of a (y, z) cross-section, propagation along x
    (mode.py:128-195): ``size`` (Ly, Lz), ``cell_size`` scalar or (dy, dz),
    boxes stamped on the cross-section, ``wavelength``, ``background_eps``,
    ``num_modes`` (largest n_eff first), ``polarization`` None / "te"
    (Ey-dominant) / "tm" (Ez-dominant). ``tol`` bounds the relative residual
    |P x - beta^2 x| / |beta^2| of every returned eigenpair."""

    def __init__(self, size: Tuple[float, float], cell_size, structures: Sequence,
                 wavelength: float, background_eps: float = 1.0, num_modes: int = 1,
                 polarization: Optional[str] = None, tol: float = 1e-11,
                 max_iter: int = 400, degree: int = 60, seed: int = 0) -> None:
        if isinstance(cell_size, (int, float)):
            dy = dz = float(cell_size)
        else:
            dy, dz = float(cell_size[0]), float(cell_size[1])
        Ly, Lz = float(size[0]), float(size[1])
        ny, nz = int(round(Ly / dy)), int(round(Lz / dz))
        if ny < 4 or nz < 4:
            raise ValueError("Need at least 4 cells per axis")
        self.dy, self.dz, self.ny, self.nz = dy, dz, ny, nz
        self.y = (np.arange(ny) - (ny - 1) / 2) * dy
        self.z = (np.arange(nz) - (nz - 1) / 2) * dz
        self.wavelength = float(wavelength)
        self.num_modes = int(num_modes)
        if polarization is not None:
            polarization = polarization.lower()
            if polarization not in ("te", "tm"):
                raise ValueError("polarization must be None, 'te' or 'tm'")
        self.polarization = polarization
        self.tol, self.max_iter, self.degree, self.seed = float(tol), int(max_iter), int(degree), seed
        eps_r = np.full((ny, nz), float(background_eps))
        for s in structures:
            self._stamp(s, eps_r)
        self.eps_r = eps_r

    def _stamp(self, box, eps_r: np.ndarray) -> None:
        """A box on the cross-section (mode.py:196-226): a 2-vector centre /
        size is (y, z), a 3-vector one (x, y, z); closed bounds; a dispersive
        medium contributes its model's real permittivity at the wavelength."""
        c = list(box.center)
        s = list(box.size)
        if len(c) == 2:
            cy, cz, sy, sz = c[0], c[1], s[0], s[1]
        else:
            c += [0.0] * (3 - len(c))
            s += [0.0] * (3 - len(s))
            cy, cz, sy, sz = c[1], c[2], s[1], s[2]
        my = (self.y >= cy - sy / 2) & (self.y <= cy + sy / 2)
        mz = (self.z >= cz - sz / 2) & (self.z <= cz + sz / 2)
        if not my.any() or not mz.any():
            return
        med = box.medium
        if getattr(med, "is_dispersive", False):
            val = float(np.real(med.eps_model(C_0 / self.wavelength)))
        else:
            val = med.eps_r
        eps_r[np.ix_(np.flatnonzero(my), np.flatnonzero(mz))] = val

    # -- device operator ---------------------------------------------------- #
    def _ops(self, torch, dev, k2, nmax):
        L = N.lib()
        ny, nz, dy, dz = self.ny, self.nz, self.dy, self.dz
        eps = torch.tensor(self.eps_r.reshape(-1), dtype=torch.float64, device=dev)
        work = torch.empty(10 * ny * nz * nmax, dtype=torch.float64, device=dev)
        stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

        def chk(rc):
            if rc != N.PF_OK:
                raise N.NativeError(rc, L.pfm_last_error().decode(errors="replace"))

        def apply(X):  # X: (nvec, 2N) contiguous
            Y = torch.empty_like(X)
            chk(L.pfm_apply(ny, nz, dy, dz, k2, C.c_void_p(eps.data_ptr()),
                            C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), X.shape[0],
                            C.c_void_p(work.data_ptr()), stream))
            return Y

        def cheb(X, degree, lo, hi):
            chk(L.pfm_chebyshev(ny, nz, dy, dz, k2, C.c_void_p(eps.data_ptr()),
                                C.c_void_p(X.data_ptr()), X.shape[0], int(degree), float(lo),
                                float(hi), C.c_void_p(work.data_ptr()), stream))
            return X

        return apply, cheb

    def _top_eigs(self, k: int, k2: float):
        """The k largest eigenvalues beta^2 of P and their vectors."""
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("photonfdtd_b200.mode: the mode solver runs on a CUDA device")
        dev = torch.device("cuda", torch.cuda.current_device())
        n2 = 2 * self.ny * self.nz
        b = min(k + max(4, k), n2)
        apply, cheb = self._ops(torch, dev, k2, b)
        g = torch.Generator(device="cpu").manual_seed(self.seed)
        # the spectrum's far (negative) end by power iteration: |lambda|max
        z = torch.randn(1, n2, dtype=torch.float64, generator=g).to(dev)
        z /= z.norm()
        lam_abs = 0.0
        for _ in range(40):
            z = apply(z)
            lam_abs = float(z.norm())
            z /= lam_abs
        lo = -1.1 * lam_abs
        top = 1.02 * k2 * float(self.eps_r.max())  # above every guided beta^2
        cut = k2 * float(self.eps_r.min())
        X = torch.linalg.qr(torch.randn(n2, b, dtype=torch.float64, generator=g).to(dev))[0]
        X = X.T.contiguous()
        w = res = None
        for it in range(1, self.max_iter + 1):
            # keep T_m bounded: m acosh(t_top) <= 600 (cosh below 1e260)
            t_top = 1.0 + 2.0 * max(top - cut, 0.0) / max(cut - lo, 1e-300)
            deg = self.degree
            if t_top > 1.0:
                deg = max(4, min(deg, int(600.0 / math.acosh(t_top))))
            cheb(X, deg, lo, cut)
            Q = torch.linalg.qr(X.T)[0]                     # (n2, b) orthonormal
            PQ = apply(Q.T.contiguous())                    # (b, n2)
            H = (PQ @ Q).T.cpu().numpy()                    # Q^T P Q
            w, V = np.linalg.eig(H)
            o = np.argsort(-w.real)
            w, V = w[o], V[:, o]
            Xr = Q @ torch.from_numpy(np.ascontiguousarray(V.real)).to(dev)
            Xr /= Xr.norm(dim=0, keepdim=True)
            R = apply(Xr[:, :k].T.contiguous()).T - Xr[:, :k] * torch.from_numpy(
                np.ascontiguousarray(w.real[:k])).to(dev)
            res = (R.norm(dim=0).cpu().numpy() / np.abs(w.real[:k]))
            if w.real[b - 1] > lo:
                cut = float(w.real[b - 1])
            X = Xr.T.contiguous()
            if float(res.max()) < self.tol:
                break
        self.iterations, self.max_residual = it, float(res.max())
        return w.real[:k].copy(), Xr[:, :k].cpu().numpy()

    # -- solve ---------------------------------------------------------------- #
    def solve(self) -> ModeResult:
        """The num_modes highest-n_eff modes (mode.py:256-351)."""
        ny, nz = self.ny, self.nz
        n = ny * nz
        k0 = 2 * math.pi / self.wavelength
        want = self.num_modes if self.polarization is None else self.num_modes + 4
        k_solve = min(max(want, self.num_modes), 2 * n - 2)
        beta2, vecs = self._top_eigs(k_solve, k0 * k0)
        order = np.argsort(-beta2)
        beta2, vecs = beta2[order], vecs[:, order]
        n_eff_all = np.sqrt(np.clip(beta2, 0.0, None)) / k0
        Ez_all = vecs[:n, :].astype(np.complex128)
        Ey_all = vecs[n:, :].astype(np.complex128)
        selected = list(range(vecs.shape[1]))
        if self.polarization is not None:
            te, tm = [], []
            for i in selected:
                py = float(np.sum(np.abs(Ey_all[:, i]) ** 2))
                pz = float(np.sum(np.abs(Ez_all[:, i]) ** 2))
                (te if py >= pz else tm).append(i)
            selected = te if self.polarization == "te" else tm
        selected = selected[: self.num_modes]
        if not selected:
            selected = list(range(min(self.num_modes, vecs.shape[1])))
        m = len(selected)
        n_eff = n_eff_all[selected]
        Ez = Ez_all[:, selected].T.reshape(m, ny, nz)
        Ey = Ey_all[:, selected].T.reshape(m, ny, nz)
        Et = np.sqrt(np.abs(Ey) ** 2 + np.abs(Ez) ** 2)
        psi = np.empty((m, ny, nz), dtype=float)
        for i in range(m):
            mx = Et[i].max()
            if mx > 0:
                Ey[i] /= mx
                Ez[i] /= mx
                psi[i] = Et[i] / mx
            else:
                psi[i] = Et[i]
        Ex, Hx, Hy, Hz = self._recover_fields(Ey, Ez, n_eff, k0)
        fields = {"Ex": Ex, "Ey": Ey, "Ez": Ez, "Hx": Hx, "Hy": Hy, "Hz": Hz}
        return ModeResult(wavelength=self.wavelength, n_eff=n_eff, psi=psi, y=self.y, z=self.z,
                          Ex=Ex, Ey=Ey, Ez=Ez, Hx=Hx, Hy=Hy, Hz=Hz, fields=fields,
                          eps_r=self.eps_r.copy(), iterations=self.iterations,
                          max_residual=self.max_residual)

    def _recover_fields(self, Ey, Ez, n_eff, k0):
        """Ex from Gauss's law and H from Faraday's law with d/dx -> i beta,
        central differences on the collocated grid (mode.py:353-387):
        inspection fields, as in the reference."""
        m = Ey.shape[0]
        dy, dz = self.dy, self.dz
        omega = C_0 * k0
        eps = self.eps_r
        Ex, Hx, Hy, Hz = (np.zeros_like(Ey) for _ in range(4))
        for i in range(m):
            beta = n_eff[i] * k0
            if beta == 0:
                continue
            div = (np.gradient(eps * Ey[i], dy, axis=0) + np.gradient(eps * Ez[i], dz, axis=1))
            Ex[i] = -div / (1j * beta * eps)
            Hx[i] = (np.gradient(Ez[i], dy, axis=0)
                     - np.gradient(Ey[i], dz, axis=1)) / (1j * omega * MU_0)
            Hy[i] = (np.gradient(Ex[i], dz, axis=1) - 1j * beta * Ez[i]) / (1j * omega * MU_0)
            Hz[i] = (1j * beta * Ey[i] - np.gradient(Ex[i], dy, axis=0)) / (1j * omega * MU_0)
        return Ex, Hx, Hy, Hz
