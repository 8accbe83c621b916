"""2D TE forward run and its discrete adjoint, in NumPy (test infrastructure).

The checker for the batched 2D engine (``photonfdtd_b200.batch``). Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` may import it.

Forward: the reference's step (src/photonfdtd/simulation.py:1319-1406) for an
xy grid with nz = 1 and TE sources only, so of the six components only Ex, Ey
and Hz are ever non-zero. The curl and CPML updates restate
``OracleRun._apply`` (itself simulation.py:1252-1309) with the same array
expressions in the same order, so a float32 or float64 run reproduces the
reference bit for bit; ``tests/test_adjoint_oracle.py`` pins this against
``OracleRun`` (pinned in turn to the reference's golden runs). The output-line
DFT of Ey follows simulation.py:1116-1133: acc += (exp(i w t) * Ey) * dt with
t = (n+1) dt.

Adjoint: reverse mode of that step, one linear operation at a time, written
here as explicit scatter-adds (the CUDA engine gathers instead). For a real
loss L of the DFT F with cotangent G = dL/dRe F + i dL/dIm F it returns
dL/dK for every cell of the design window, K = dt / (eps eps0) being the E
coefficient (simulation.py:953-969). The reference differentiates the same
quantity by JAX autodiff (jaxbackend.py:666-722, value_and_grad_eps);
``tests/test_adjoint_oracle.py`` pins this adjoint against central finite
differences of the forward run in float64.
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np

from .fdtd_oracle import EPS0, gaussian_pulse, grid_of, scene_tables

_TE = {"Ex", "Ey", "Hz"}


class TEAdjointRun:
    """Forward + adjoint of one 2D TE simulation with a design window.

    ``window = (i0, j0, n)``: cells [i0, i0+n) x [j0, j0+n) whose coefficient
    gradient is returned. ``line_i`` is the x index of the Ey DFT line; by
    default the plane of the simulation's DFTMonitor.
    """

    def __init__(self, sim, window: Tuple[int, int, int], line_i: Optional[int] = None,
                 n_steps: Optional[int] = None):
        t = scene_tables(sim)
        g = grid_of(sim.grid)
        nx, ny, nz = g.shape
        if nz != 1 or nx < 2 or ny < 2:
            raise ValueError("TE oracle needs an xy grid with nz = 1")
        self.T = t["dtype"]
        self.dt = t["dt"]
        self.n_steps = t["n_steps"] if n_steps is None else int(n_steps)
        self.nx, self.ny = nx, ny
        self.dl = tuple(d if d > 0 else 1.0 for d in g.cell_size)
        self.K = np.ascontiguousarray(t["ce3"][0][:, :, 0])
        self.ch = t["ch"]
        cp = t["cpml"]
        T = self.T
        self.cpml = [tuple(np.asarray(a, dtype=T) for a in cp[ax]) for ax in range(2)]
        self.window = tuple(int(v) for v in window)
        dfts = [m for m in sim.monitors if type(m).__name__ == "DFTMonitor"]
        if line_i is None:
            m = dfts[0]
            line_i = int(np.argmin(np.abs(np.asarray(g.coords[0]) - float(m.plane_position))))
        self.line_i = int(line_i)
        self.omega = 2.0 * np.pi * np.asarray(dfts[0].freqs, dtype=np.float64)
        self.sources = []
        for s in sim.sources:
            if s.component not in _TE:
                raise ValueError("TE oracle: source component must be Ex, Ey or Hz")
            i, j, _ = g.index_at(s.position)
            self.sources.append((s, s.component, i, j))
        # CPML rows / columns carrying psi (simulation.py:1204-1221: where c != 0)
        bex, cex, bhx, chx = self.cpml[0]
        bey, cey, bhy, chy = self.cpml[1]
        self.ix_h = np.nonzero(chx[:nx - 1] != 0)[0]
        self.iy_h = np.nonzero(chy[:ny - 1] != 0)[0]
        self.ix_e = np.nonzero(cex[1:] != 0)[0]   # rows of the Ey region (i >= 1)
        self.iy_e = np.nonzero(cey[1:] != 0)[0]   # columns of the Ex region (j >= 1)

    # ---- forward ------------------------------------------------------- #
    def set_window_eps(self, eps_window: np.ndarray) -> None:
        """Replace the window's coefficients from a permittivity array, with
        the reference's expression dt / (eps * EPS_0) in the field type."""
        i0, j0, n = self.window
        eps = np.asarray(eps_window, dtype=self.T)
        self.K[i0:i0 + n, j0:j0 + n] = (self.dt / (eps * EPS0)).astype(self.T, copy=False)

    def _inject(self, F, family, t):
        for s, c, i, j in self.sources:
            if (c[0] == "H") != (family == "H"):
                continue
            val = s.amplitude * gaussian_pulse(s.waveform, np.array([t]))[0]
            F[c][i, j] += val

    def forward(self, record: bool = True) -> np.ndarray:
        """Run all steps from zero fields; returns the line DFT (n_freq, ny)
        and, with ``record``, keeps the window curls of every step."""
        T, nx, ny = self.T, self.nx, self.ny
        dx, dy = self.dl[0], self.dl[1]
        bex, cex, bhx, chx = self.cpml[0]
        bey, cey, bhy, chy = self.cpml[1]
        F = {c: np.zeros((nx, ny), dtype=T) for c in _TE}
        Ex, Ey, Hz = F["Ex"], F["Ey"], F["Hz"]
        ph_hx = np.zeros((self.ix_h.size, ny - 1), T)
        ph_hy = np.zeros((nx - 1, self.iy_h.size), T)
        ps_ey = np.zeros((nx, self.iy_e.size), T)    # Ex's psi along y
        ps_ex = np.zeros((self.ix_e.size, ny), T)    # Ey's psi along x
        mch = -self.ch
        Kx = self.K[:, 1:]
        Ky = self.K[1:, :]
        i0, j0, n = self.window
        acc = np.zeros((self.omega.size, ny), dtype=np.complex128)
        self.curls = np.zeros((self.n_steps if record else 0, n, n, 2), dtype=T)
        bhx_r, chx_r = bhx[self.ix_h][:, None], chx[self.ix_h][:, None]
        bhy_r, chy_r = bhy[self.iy_h][None, :], chy[self.iy_h][None, :]
        bey_r, cey_r = bey[1:][self.iy_e][None, :], cey[1:][self.iy_e][None, :]
        bex_r, cex_r = bex[1:][self.ix_e][:, None], cex[1:][self.ix_e][:, None]
        for s in range(self.n_steps):
            # Hz on [0, nx-1) x [0, ny-1): + dEy/dx - dEx/dy
            dA = ((Ey[1:, :] - Ey[:-1, :]) / dx)[:, :-1]
            dB = ((Ex[:, 1:] - Ex[:, :-1]) / dy)[:-1, :]
            curl = dA.copy()
            np.subtract(curl, dB, out=curl)
            np.multiply(curl, mch, out=curl)
            hreg = Hz[:-1, :-1]
            hreg += curl
            if self.ix_h.size:
                ph_hx[...] = bhx_r * ph_hx + chx_r * dA[self.ix_h]
                hreg[self.ix_h] += 1.0 * mch * ph_hx
            if self.iy_h.size:
                ph_hy[...] = bhy_r * ph_hy + chy_r * dB[:, self.iy_h]
                hreg[:, self.iy_h] += -1.0 * mch * ph_hy
            self._inject(F, "H", (s + 0.5) * self.dt)
            # Ex on j >= 1: + dHz/dy ; Ey on i >= 1: - dHz/dx
            dAe = (Hz[:, 1:] - Hz[:, :-1]) / dy
            dBe = (Hz[1:, :] - Hz[:-1, :]) / dx
            cx = dAe.copy()
            c1 = dAe.copy()
            np.multiply(c1, Kx, out=c1)
            xr = Ex[:, 1:]
            xr += c1
            cy = np.negative(dBe)
            c2 = np.negative(dBe)
            np.multiply(c2, Ky, out=c2)
            yr = Ey[1:, :]
            yr += c2
            if self.iy_e.size:
                ps_ey[...] = bey_r * ps_ey + cey_r * dAe[:, self.iy_e]
                xr[:, self.iy_e] += 1.0 * Kx[:, self.iy_e] * ps_ey
                cx[:, self.iy_e] = cx[:, self.iy_e] + ps_ey
            if self.ix_e.size:
                ps_ex[...] = bex_r * ps_ex + cex_r * dBe[self.ix_e]
                yr[self.ix_e] += -1.0 * Ky[self.ix_e] * ps_ex
                cy[self.ix_e] = cy[self.ix_e] - ps_ex
            self._inject(F, "E", (s + 1.0) * self.dt)
            if record:
                # window curls: cx lives on j >= 1, cy on i >= 1
                cxf = np.zeros((nx, ny), T)
                cyf = np.zeros((nx, ny), T)
                cxf[:, 1:] = cx
                cyf[1:, :] = cy
                self.curls[s, :, :, 0] = cxf[i0:i0 + n, j0:j0 + n]
                self.curls[s, :, :, 1] = cyf[i0:i0 + n, j0:j0 + n]
            ph = np.exp(1j * self.omega * ((s + 1.0) * self.dt)).reshape(-1, 1)
            acc += ph * Ey[self.line_i][None, :] * self.dt
        self.F = F
        self.dft = acc
        return acc

    # ---- adjoint ------------------------------------------------------- #
    def adjoint(self, G: np.ndarray) -> np.ndarray:
        """dL/dK over the design window for DFT cotangent G (n_freq, ny)."""
        if self.curls.shape[0] != self.n_steps:
            raise RuntimeError("adjoint needs a recorded forward run")
        nx, ny = self.nx, self.ny
        dx, dy = self.dl[0], self.dl[1]
        bex, cex, bhx, chx = [np.asarray(a, np.float64) for a in self.cpml[0]]
        bey, cey, bhy, chy = [np.asarray(a, np.float64) for a in self.cpml[1]]
        K = np.asarray(self.K, np.float64)
        ch = float(self.ch)
        aEx = np.zeros((nx, ny))
        aEy = np.zeros((nx, ny))
        aHz = np.zeros((nx, ny))
        a_hx = np.zeros((self.ix_h.size, ny - 1))
        a_hy = np.zeros((nx - 1, self.iy_h.size))
        a_ey = np.zeros((nx, self.iy_e.size))
        a_ex = np.zeros((self.ix_e.size, ny))
        i0, j0, n = self.window
        grad = np.zeros((n, n))
        G = np.asarray(G, np.complex128)
        for s in range(self.n_steps - 1, -1, -1):
            ph = np.exp(1j * self.omega * ((s + 1.0) * self.dt)).reshape(-1, 1)
            aEy[self.line_i] += self.dt * np.sum(G.real * ph.real + G.imag * ph.imag, axis=0)
            cur = np.asarray(self.curls[s], np.float64)
            grad += aEx[i0:i0 + n, j0:j0 + n] * cur[..., 0] + aEy[i0:i0 + n, j0:j0 + n] * cur[..., 1]
            # Ex' = Ex + K dAe + K psi', psi' = b psi + c dAe  (j >= 1)
            lx = aEx[:, 1:]
            Kx = K[:, 1:]
            a_dAe = Kx * lx
            if self.iy_e.size:
                a_psi = a_ey + Kx[:, self.iy_e] * lx[:, self.iy_e]
                a_dAe[:, self.iy_e] += cey[1:][self.iy_e][None, :] * a_psi
                a_ey = bey[1:][self.iy_e][None, :] * a_psi
            aHz[:, 1:] += a_dAe / dy
            aHz[:, :-1] -= a_dAe / dy
            # Ey' = Ey - K dBe - K psi', psi' = b psi + c dBe  (i >= 1)
            ly = aEy[1:, :]
            Ky = K[1:, :]
            a_dBe = -Ky * ly
            if self.ix_e.size:
                a_psi = a_ex - Ky[self.ix_e] * ly[self.ix_e]
                a_dBe[self.ix_e] += cex[1:][self.ix_e][:, None] * a_psi
                a_ex = bex[1:][self.ix_e][:, None] * a_psi
            aHz[1:, :] += a_dBe / dx
            aHz[:-1, :] -= a_dBe / dx
            # Hz' = Hz - ch (dA - dB) - ch psi_x' + ch psi_y' on [0, nx-1) x [0, ny-1)
            ah = aHz[:-1, :-1]
            a_dA = -ch * ah
            a_dB = ch * ah
            if self.ix_h.size:
                a_psi = a_hx - ch * ah[self.ix_h]
                a_dA[self.ix_h] += chx[self.ix_h][:, None] * a_psi
                a_hx = bhx[self.ix_h][:, None] * a_psi
            if self.iy_h.size:
                a_psi = a_hy + ch * ah[:, self.iy_h]
                a_dB[:, self.iy_h] += chy[self.iy_h][None, :] * a_psi
                a_hy = bhy[self.iy_h][None, :] * a_psi
            aEy[1:, :-1] += a_dA / dx
            aEy[:-1, :-1] -= a_dA / dx
            aEx[:-1, 1:] += a_dB / dy
            aEx[:-1, :-1] -= a_dB / dy
        return grad


def objective(dft: np.ndarray) -> float:
    """J = sum over frequencies and line cells of |F|^2."""
    return float(np.sum(np.abs(dft) ** 2))


def objective_cotangent(dft: np.ndarray) -> np.ndarray:
    """dJ/dRe F + i dJ/dIm F of ``objective``: 2 F."""
    return 2.0 * np.asarray(dft, np.complex128)
