"""Gradient of a monitor loss with respect to the per-cell permittivity of
one simulation on the B200 engine: the counterpart of the reference's
``value_and_grad_eps`` (src/photonfdtd/jaxbackend.py:666-722).

The reference differentiates its JAX step with ``jax.grad`` under nested
checkpointing (jaxbackend.py:511-570). Here the forward run saves the
engine's state every ``checkpoint_every`` steps into device memory
(``pf_get_state``); the loss is evaluated on the Result's outputs with torch
autograd, which gives dJ/d(each output); the engine then walks the segments
backwards (``pf_adj_segment``): it restores a segment's checkpoint, replays
it recording H and the E-side CPML state per step, and runs the transposed
steps (``csrc/kernels_adj.cuh``) on adjoint fields driven by those
sensitivities, accumulating dJ/dK for K = dt / (eps0 eps_r) per cell.

The loss takes the reference's ``out`` dict with torch tensors instead of JAX
arrays: ``{'fields': {name: {comp: (n_rec, *snap) real}}, 'dft': {name:
{comp: (n_freq, *snap) complex128}}, 'flux': {name: scalar}}`` and returns a
scalar tensor, e.g. ``lambda out: (out['dft']['d']['Ez'].abs() ** 2).sum()``.
Dispersive media raise NotImplementedError, as in the reference, and so
does subpixel smoothing for value_and_grad_eps (value_and_grad_params takes
per-component coefficients instead).
"""
from __future__ import annotations

import math
from typing import Callable, Dict, Tuple

import numpy as np

from . import _native as N
from .engine import _COMP, B200Engine, build_tables, drive, field_plans, validate
from .scene import EPS_0


class _Checkpointing:
    """An engine proxy for ``drive``: ``advance`` stops at every multiple of
    ``every`` steps and saves the state there into a device buffer."""

    def __init__(self, eng: B200Engine, every: int, nbytes: int, device):
        self._eng = eng
        self.every = every
        self.nbytes = nbytes
        self.device = device
        self.ckpts: Dict[int, object] = {}

    def _save(self, step: int) -> None:
        import torch
        buf = torch.empty(self.nbytes, dtype=torch.uint8, device=self.device)
        self._eng.get_state_to(buf.data_ptr(), self.nbytes)
        self.ckpts[step] = buf

    def advance(self, step0: int, n_sub: int) -> None:
        pos, end = int(step0), int(step0) + int(n_sub)
        while pos < end:
            if pos % self.every == 0 and pos not in self.ckpts:
                self._save(pos)
            m = min(end - pos, self.every - pos % self.every)
            self._eng.advance(pos, m)
            pos += m

    def __getattr__(self, name):
        return getattr(self._eng, name)


def _out_dict(res, torch):
    """The loss-facing dict of torch leaves (requires_grad) from a Result."""
    leaves = {"fields": {}, "dft": {}, "flux": {}}
    for name, comps in res.fields.items():
        leaves["fields"][name] = {c: torch.tensor(np.asarray(a, np.float64), dtype=torch.float64,
                                                  requires_grad=True) for c, a in comps.items()}
    for name, comps in res.dft.items():
        leaves["dft"][name] = {c: torch.tensor(np.asarray(a, np.complex128),
                                               dtype=torch.complex128, requires_grad=True)
                               for c, a in comps.items()}
    for name, v in res.flux.items():
        leaves["flux"][name] = torch.tensor(float(v), dtype=torch.float64, requires_grad=True)
    return leaves


def _adjoint(sim, t: dict, loss: Callable, checkpoint_every) -> Tuple[float, np.ndarray]:
    """The forward run with checkpoints, the loss and its output
    sensitivities, and the reverse pass: (J, dJ/dK) shaped (3, *grid), the
    gradient per E coefficient K of Ex, Ey, Ez, when the tables give one
    coefficient per component (PF_CE_CELL3); else shaped (1, *grid), the
    sum over the components (all the reverse pass keeps then)."""
    import torch
    n_steps, dt = t["n_steps"], t["dt"]
    if n_steps < 1:
        raise ValueError("nothing to differentiate: the simulation has no steps")
    every = min(int(checkpoint_every or max(1, math.ceil(math.sqrt(n_steps)))), n_steps)
    eng = B200Engine(t)
    try:
        device = torch.device("cuda", torch.cuda.current_device())
        proxy = _Checkpointing(eng, every, eng.state_bytes(), device)
        res = drive(sim, proxy, t)

        out = _out_dict(res, torch)
        val = loss(out)
        if not torch.is_tensor(val):
            val = torch.as_tensor(val, dtype=torch.float64)
        value = float(val.detach())
        eng._chk(eng._L.pf_adj_init(eng.h, every))
        if val.requires_grad:
            val.backward()
        # dJ/d(flux integrals): sources on each plane's E and H
        for k, f in enumerate(t["flux"]):
            v = out["flux"].get(f["m"].name)
            if v is not None and v.grad is not None and float(v.grad) != 0.0:
                eng._chk(eng._L.pf_adj_set_flux_cotangent(eng.h, eng.flux_ids[k],
                                                          float(v.grad)))
        # dJ/d(DFT accumulators), per monitor in the engine's component order
        for k, d in enumerate(t["dft"]):
            m = d["m"]
            comps = sorted(m.components, key=lambda c: _COMP[c])
            grads = [out["dft"][m.name][c].grad for c in comps]
            if all(g is None for g in grads):
                continue
            cot = np.stack([np.zeros((d["omega"].size,) + tuple(d["counts"]), np.complex128)
                            if g is None else g.detach().numpy().reshape(
                                (d["omega"].size,) + tuple(d["counts"])) for g in grads])
            cot = np.ascontiguousarray(cot).view(np.float64)
            eng._chk(eng._L.pf_adj_set_dft_cotangent(eng.h, eng.dft_ids[k],
                                                     N.ptr(cot, N.C.c_double)))
        # dJ/d(FieldMonitor frames): a source on the snapshot taken after step s
        for name, p in field_plans(sim, n_steps, dt).items():
            steps = sorted(p["steps"])
            start, stop, stride = (np.asarray(v, np.int32) for v in p["region"])
            for c, leaf in out["fields"].get(name, {}).items():
                if leaf.grad is None:
                    continue
                g = leaf.grad.detach().numpy()
                for f, s in enumerate(steps[:g.shape[0]]):
                    vals = np.ascontiguousarray(g[f], np.float64).ravel()
                    if not vals.any():
                        continue
                    eng._chk(eng._L.pf_adj_add_field_source(
                        eng.h, int(s), _COMP[c], N.ptr(start, N.C.c_int32),
                        N.ptr(stop, N.C.c_int32), N.ptr(stride, N.C.c_int32),
                        N.ptr(vals, N.C.c_double)))
        # reverse pass over the checkpointed segments, last first
        for s0 in sorted(proxy.ckpts, reverse=True):
            n = min(every, n_steps - s0)
            buf = proxy.ckpts[s0]
            eng._chk(eng._L.pf_adj_segment(eng.h, int(s0), int(n), N.C.c_void_p(buf.data_ptr()),
                                           int(proxy.nbytes), 1))
        ncomp = 3 if t["ce_mode"] == N.PF_CE_CELL3 else 1
        grad_k = np.empty(ncomp * int(np.prod(t["shape"])), np.float64)
        read = (eng._L.pf_adj_read_grad_components if ncomp == 3 else eng._L.pf_adj_read_grad)
        eng._chk(read(eng.h, N.ptr(grad_k, N.C.c_double)))
    finally:
        eng.close()
    return value, grad_k.reshape((ncomp,) + tuple(t["shape"]))


def _no_dispersion(sim, what: str) -> None:
    if getattr(sim, "_has_dispersion", False):
        raise NotImplementedError(f"{what} does not support dispersive media (the pole state "
                                  "is not parameterized).")


def value_and_grad_eps(sim, loss: Callable, checkpoint_every: int = None
                       ) -> Tuple[float, np.ndarray]:
    """``(value, d value / d eps_r)`` for a scalar ``loss(out)`` of the
    simulation's monitor outputs (jaxbackend.py:666-722). ``checkpoint_every``
    is the segment length of the reverse pass (default ceil(sqrt(n_steps)));
    device memory holds n_steps / checkpoint_every states plus one segment of
    per-step records (three H fields and the E-side CPML state per step)."""
    validate(sim)
    _no_dispersion(sim, "value_and_grad_eps")
    if sim.subpixel:
        raise NotImplementedError(
            "value_and_grad_eps differentiates the scalar per-cell eps_r, which does not "
            "parameterize a subpixel-smoothed tensor; use value_and_grad_params.")
    t = build_tables(sim)
    value, g3 = _adjoint(sim, t, loss, checkpoint_every)
    dt = t["dt"]
    eps = np.asarray(sim.eps_r, dtype=np.float64).reshape(t["shape"])
    # K = dt / (eps0 eps_r) for all three components  =>  dK/deps_r = -dt / (eps0 eps_r^2)
    gk = g3[0] if g3.shape[0] == 1 else (g3[0] + g3[1]) + g3[2]
    grad = gk * (-dt / (EPS_0 * eps * eps))
    return value, grad.astype(np.dtype(sim.dtypes["eps_r"]))


def value_and_grad_params(sim, ce_of_params: Callable, params, loss: Callable,
                          checkpoint_every: int = None):
    """``(value, d value / d params)`` for design parameters that set the
    per-component E coefficients (jaxbackend.py:725-775): ``ce_of_params(p)``
    returns ``{'Ex', 'Ey', 'Ez'}`` grid-shaped torch tensors built from ``p``
    with torch operations (e.g. photonfdtd_b200.design.EtchedCore.ce_builder);
    the engine runs with exactly those coefficients, its adjoint gives dJ/dK
    per component, and torch carries them back to ``params``. ``params`` is a
    torch tensor (the gradient is returned as one of its dtype and device) or
    an array (returned as NumPy)."""
    import torch
    validate(sim)
    _no_dispersion(sim, "value_and_grad_params")
    as_numpy = not torch.is_tensor(params)
    p = (torch.as_tensor(np.asarray(params, np.float64)) if as_numpy else params).detach()
    p = p.clone().requires_grad_(True)
    with torch.enable_grad():
        ce = ce_of_params(p)
        comps = [ce[c] for c in ("Ex", "Ey", "Ez")]
        t = build_tables(sim, ce3=[c.detach().cpu().numpy() for c in comps])
        value, g3 = _adjoint(sim, t, loss, checkpoint_every)
        torch.autograd.backward(comps, [torch.as_tensor(g3[i], dtype=c.dtype, device=c.device)
                                        for i, c in enumerate(comps)])
    g = p.grad if p.grad is not None else torch.zeros_like(p)
    return value, (g.cpu().numpy() if as_numpy else g)
