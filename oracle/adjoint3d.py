"""NumPy restatement of the gradient value_and_grad_eps computes
(src/photonfdtd/jaxbackend.py:666-722: jax.grad of a monitor loss through
the whole time loop, with respect to eps_r).

TEST INFRASTRUCTURE: the checker the engine's adjoint (csrc/kernels_adj.cuh)
is compared against. It is never part of the product path.

The reference gets its gradient from JAX's reverse-mode differentiation of
its step, which JAX does not have to be installed for us to restate: the step
is linear in the fields for fixed coefficients, so reverse mode is the
transposed step run backwards in time. This file transposes the oracle's own
slab-structured step (fdtd_oracle.OracleRun._apply: per component, the curl
terms on the cropped region and the CPML psi slabs) update by update, keeping
the forward trajectory in memory (small scenes only). It shares no code with
the CUDA adjoint, which works per cell with quotient-adjoint arrays; the two
are checked against each other and this one against central differences of
the oracle's forward run.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Tuple

import numpy as np

from .fdtd_oracle import EPS0, OracleRun, _cls


_PLANE = {0: ("Ey", "Ez", "Hy", "Hz"), 1: ("Ez", "Ex", "Hz", "Hx"), 2: ("Ex", "Ey", "Hx", "Hy")}


def _flux_plane(run, m):
    """(axis, index, dA) of a flux monitor, as OracleRun._flux takes them."""
    g = run.grid
    ax = {"x": 0, "y": 1, "z": 2}[m.plane_axis]
    co = g.coords[ax]
    i = 0 if co.size == 1 else int(np.argmin(np.abs(co - m.plane_position)))
    w = [g.cell_size[a] if g.shape[a] > 1 else 1.0 for a in range(3)]
    return ax, i, float(np.prod([w[a] for a in range(3) if a != ax]))


class _RecordingRun(OracleRun):
    """An OracleRun that keeps, per step and E component, what the E
    coefficient multiplies: g = curl + sum(sign * psi') over the update's
    region (psi' the slab's value after the step), and per step each flux
    monitor's plane of E_t1, E_t2, H_t1, H_t2 (t1 = axis+1, t2 = axis+2)."""

    def __init__(self, sim, n_steps=None, ce3=None):
        super().__init__(sim, n_steps, ce3=ce3)
        self.g_hist: List[Dict[str, np.ndarray]] = []
        self.plane_hist: List[Dict[str, Tuple[np.ndarray, ...]]] = []

    def _record(self, step):
        planes = {}
        for m in self.monitors:
            if _cls(m) == "FluxMonitor":
                ax, i, _ = _flux_plane(self, m)
                sl = [slice(None)] * 3
                sl[ax] = i
                planes[m.name] = tuple(self.F[c][tuple(sl)].copy() for c in _PLANE[ax])
        self.plane_hist.append(planes)
        super()._record(step)

    def _apply(self, family):
        if family == "E":
            rec = {}
            F = self.F
            for name, reg, k_arr, k_sc, is_e, terms in self.updates:
                if not is_e or not terms:
                    continue
                g = None
                ds = []
                for ax, src, oax, sign, slabs in terms:
                    d = self._deriv(F[src], ax)
                    if self.shape[oax] > 1:
                        o = [slice(None)] * 3
                        o[oax] = self._crop(oax, True)
                        d = d[tuple(o)]
                    ds.append(d)
                    g = sign * d if g is None else g + sign * d
                for (ax, src, oax, sign, slabs), d in zip(terms, ds):
                    for sl, bb, cc, psi in slabs:
                        g[sl] = g[sl] + sign * (bb * psi + cc * d[sl])
                rec[name] = g
            self.g_hist.append(rec)
        super()._apply(family)


def _out_dict(res, torch):
    out = {"fields": {}, "dft": {}, "flux": {}}
    for name, comps in res["fields"].items():
        out["fields"][name] = {c: torch.tensor(np.asarray(a, np.float64), requires_grad=True)
                               for c, a in comps.items()}
    for name, comps in res["dft"].items():
        out["dft"][name] = {c: torch.tensor(np.asarray(a, np.complex128), requires_grad=True)
                            for c, a in comps.items()}
    for name, v in res["flux"].items():
        out["flux"][name] = torch.tensor(float(v), dtype=torch.float64, requires_grad=True)
    return out


def forward_value(sim, loss: Callable) -> float:
    """loss(out) of the oracle's forward run."""
    import torch
    r = OracleRun(sim)
    r.advance(r.n_steps)
    return float(loss(_out_dict(r.result(), torch)).detach())


def value_and_grad_eps(sim, loss: Callable) -> Tuple[float, np.ndarray]:
    """(J, dJ/deps_r) of a loss of the monitor outputs, in float64 numpy."""
    run, val, gk = _reverse(sim, loss, None)
    eps = np.asarray(run.t["eps"], np.float64)
    g = (gk["Ex"] + gk["Ey"]) + gk["Ez"]
    return val, g * (-run.dt / (EPS0 * eps * eps))


def value_and_grad_ce3(sim, ce3, loss: Callable) -> Tuple[float, np.ndarray]:
    """(J, dJ/dK_c) with the E coefficients of Ex, Ey, Ez given per cell
    (``ce3``, three grid-shaped arrays): the gradient value_and_grad_params
    chains to its parameters (jaxbackend.py:725-775), shaped (3, *grid)."""
    _, val, gk = _reverse(sim, loss, ce3)
    return val, np.stack([gk["Ex"], gk["Ey"], gk["Ez"]])


def _reverse(sim, loss: Callable, ce3):
    import torch
    run = _RecordingRun(sim, ce3=ce3)
    run.advance(run.n_steps)
    res = run.result()
    out = _out_dict(res, torch)
    val = loss(out)
    val.backward()
    shape, dt, dl = run.shape, run.dt, run.dl
    lam = {c: np.zeros(shape) for c in run.F}
    lpsi = [[[np.zeros(psi.shape) for (_, _, _, psi) in slabs]
             for (_, _, _, _, slabs) in terms] for (_, _, _, _, _, terms) in run.updates]
    gk = {c: np.zeros(shape) for c in ("Ex", "Ey", "Ez")}

    # the loss's sources per step: DFT samples, FieldMonitor frames and the
    # flux integrand S = E_t1 H_t2 - E_t2 H_t1 summed over the plane (x dA dt)
    def sources(n):
        for m in run.monitors:
            kind = _cls(m)
            if kind == "FluxMonitor":
                G = out["flux"][m.name].grad
                if G is None or float(G) == 0.0:
                    continue
                ax, i, da = _flux_plane(run, m)
                c = float(G) * da * dt
                e1, e2, h1, h2 = run.plane_hist[n][m.name]
                n1, n2, m1, m2 = _PLANE[ax]
                sl = [slice(None)] * 3
                sl[ax] = i
                sl = tuple(sl)
                lam[n1][sl] += c * h2
                lam[n2][sl] -= c * h1
                lam[m2][sl] += c * e1
                lam[m1][sl] -= c * e2
            elif kind == "DFTMonitor":
                st = run.dm[m.name]
                if n not in st["steps"]:
                    continue
                ds = m.downsample
                sl = [slice(None, None, ds) if ds > 1 else slice(None)] * 3
                if st["plane"] is not None:
                    ax, ci = st["plane"]
                    sl[ax] = slice(ci, ci + 1)
                for c in m.components:
                    G = out["dft"][m.name][c].grad
                    if G is None:
                        continue
                    G = G.detach().numpy()
                    t = (n + 1.0) * dt if c[0] == "E" else (n + 0.5) * dt
                    ph = np.exp(1j * st["omega"] * t).reshape((-1,) + (1,) * (G.ndim - 1))
                    lam[c][tuple(sl)] += (G.real * ph.real + G.imag * ph.imag).sum(0) * dt
            elif kind == "FieldMonitor":
                st = run.fm[m.name]
                steps = sorted(st["steps"])
                if n not in steps:
                    continue
                f = steps.index(n)
                for c in m.components:
                    G = out["fields"][m.name][c].grad
                    if G is None or f >= G.shape[0]:
                        continue
                    ds = m.downsample
                    if st["zsl"] != slice(None):
                        sl = (slice(None, None, ds), slice(None, None, ds), st["zsl"])
                    elif ds > 1:
                        sl = (slice(None, None, ds),) * 3
                    else:
                        sl = (slice(None),) * 3
                    lam[c][sl] += G[f].detach().numpy()

    def transpose(u, n):
        name, reg, k_arr, k_sc, is_e, terms = run.updates[u]
        if not terms:
            return
        lf = lam[name][reg]
        k = k_arr if is_e else k_sc
        if is_e:
            gk[name][reg] += lf * run.g_hist[n][name]
        for t, (ax, src, oax, sign, slabs) in enumerate(terms):
            ld = sign * k * lf
            for q, (sl, bb, cc, psi) in enumerate(slabs):
                kk = k[sl] if is_e else k
                lpn = sign * kk * lf[sl] + lpsi[u][t][q]
                ld[sl] = ld[sl] + cc * lpn
                lpsi[u][t][q] = bb * lpn
            # d = crop_oax(deriv(F[src], ax)), deriv = (hi - lo) / dl
            dshape = list(shape)
            dshape[ax] -= 1
            D = np.zeros(dshape)
            if shape[oax] > 1:
                o = [slice(None)] * 3
                o[oax] = run._crop(oax, is_e)
                D[tuple(o)] = ld
            else:
                D[...] = ld
            hi = [slice(None)] * 3
            lo = [slice(None)] * 3
            hi[ax] = slice(1, None)
            lo[ax] = slice(0, -1)
            lam[src][tuple(hi)] += D / dl[ax]
            lam[src][tuple(lo)] -= D / dl[ax]

    e_upd = [u for u, U in enumerate(run.updates) if U[4]]
    h_upd = [u for u, U in enumerate(run.updates) if not U[4]]
    for n in range(run.n_steps - 1, -1, -1):
        sources(n)
        for u in e_upd:
            transpose(u, n)
        for u in h_upd:
            transpose(u, n)
    return run, float(val.detach()), gk
