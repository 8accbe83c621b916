"""Batched 2D TE simulations with a hand-written adjoint (the pf_batch ABI).

Many 2D inverse-design candidates of uneven size run as one batch on the GPU:
one pooled set of fields, each step one launch per kernel over every instance
(graph-captured in chunks), and a discrete adjoint that returns the gradient
of a loss of each instance's output-line DFT with respect to the permittivity
of its design window.

This is the batched counterpart of the reference's gradient path
``jaxbackend.value_and_grad_eps(sim, loss)`` (src/photonfdtd/
jaxbackend.py:666-722, memory bounded by remat checkpointing, :511-570) for
the TE problems of ``design.value_and_grad_density`` (src/photonfdtd/
design.py:164-175): the gradient flows through ce = dt / (eps_r * EPS_0) and
the whole time evolution. Here the adjoint is written out by hand
(``csrc/batch2d.cu``), the state is checkpointed every K steps and replayed
in between, and PyTorch appears only as the ``torch.autograd.Function`` that
exposes it.

    batch = BatchTE(sims, windows)                 # 2D TE Simulations
    eps = torch.tensor(batch.design_eps(), requires_grad=True)
    F = LineDFT.apply(eps, batch)                  # packed complex DFT
    J = batch.per_instance_sum(F.abs() ** 2)       # one objective per instance
    J.sum().backward()                             # eps.grad = dJ/deps

Every simulation must be an xy grid (nz = 1) with sources on Ex, Ey or Hz
only, non-dispersive, without subpixel smoothing, and exactly one monitor: a
``DFTMonitor(components=("Ey",), plane_axis="x")`` sampled every step. All
instances share cell size, dt, step count, precision and frequencies.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .engine import _eps_dtype, _nearest, material_words, validate
from .scene import EPS_0, MU_0

_TE_COMP = {"Ex": 0, "Ey": 1, "Hz": 2}


# --------------------------------------------------------------------------- #
# Per-instance tables
# --------------------------------------------------------------------------- #
def _wave_key(wave, family: str):
    if type(wave).__name__ == "GaussianPulse":
        return ("GaussianPulse", float(wave.freq0), float(wave.fwhm),
                float(getattr(wave, "delay", 0.0)), family)
    return (id(wave), family)


def instance_tables(sim, wave_cache: Dict, phase_cache: Dict) -> dict:
    """Coefficients, sources and DFT line of one 2D TE simulation, computed
    as the reference computes them (ce: simulation.py:953-969; CPML
    :794-808; source values one time at a time, :1367-1390; DFT phases
    exp(i w (n+1) dt), :1116-1133). Waveform rows and phase tables are shared
    through the caches across instances with equal parameters."""
    validate(sim)
    grid = sim.grid
    nx, ny, nz = (int(v) for v in grid.shape)
    if nz != 1 or nx < 2 or ny < 2:
        raise NotImplementedError("BatchTE needs xy grids (nz = 1, nx and ny >= 2)")
    if getattr(sim, "_has_dispersion", False):
        raise NotImplementedError("BatchTE does not support dispersive media")
    npdt = np.dtype(sim.dtypes["Ex"]).type
    edt = _eps_dtype(sim)
    dt, n_steps = float(sim.dt), int(sim.n_steps)
    custom = bool(getattr(sim, "_eps_r_custom", False))
    if custom:
        eps = np.asarray(sim.eps_r)[:, :, 0]
        ce = (dt / (eps * EPS_0)).astype(edt, copy=False).astype(npdt)
        eps64 = eps.astype(np.float64)
    elif getattr(sim, "subpixel", False):
        raise NotImplementedError("BatchTE does not support subpixel smoothing "
                                  "(one E coefficient per cell)")
    else:
        word, vals, _, _ = material_words(sim)
        table = (dt / (vals * EPS_0)).astype(edt, copy=False).astype(npdt)
        word = np.asarray(word).reshape(nx, ny)
        ce = table[word]
        eps64 = np.asarray(vals, np.float64)[word]
    coef = []
    for ax in (0, 1):
        for arr in (sim._b_e, sim._c_e, sim._b_h, sim._c_h):
            coef.append(np.ascontiguousarray(np.asarray(arr[ax]), dtype=npdt))
    # sources
    src = []
    for s in sim.sources:
        if s.component not in _TE_COMP:
            raise NotImplementedError(f"BatchTE: source component {s.component} is not TE "
                                      "(Ex, Ey, Hz)")
        i, j, _ = grid.index_at(s.position)
        fam = s.component[0]
        key = (_wave_key(s.waveform, fam), dt, n_steps)
        if key not in wave_cache:
            off = 0.5 if fam == "H" else 1.0
            vals_t = np.empty(n_steps, dtype=np.float64)
            for q in range(n_steps):
                vals_t[q] = s.waveform(np.array([(q + off) * dt]))[0]
            wave_cache[key] = (len(wave_cache), vals_t)
        src.append((_TE_COMP[s.component], int(i), int(j), wave_cache[key][0],
                    float(s.amplitude)))
    # the one DFT line
    mons = list(sim.monitors)
    if len(mons) != 1 or type(mons[0]).__name__ != "DFTMonitor":
        raise NotImplementedError("BatchTE needs exactly one monitor, a DFTMonitor")
    m = mons[0]
    if tuple(m.components) != ("Ey",) or getattr(m, "plane_axis", None) != "x":
        raise NotImplementedError("BatchTE: the DFTMonitor must record ('Ey',) on an x plane")
    if int(m.interval) != 1 or int(getattr(m, "downsample", 1)) > 1:
        raise NotImplementedError("BatchTE: the DFTMonitor must sample every step, "
                                  "without downsampling")
    line_i = _nearest(grid.coords[0], float(m.plane_position))
    omega = 2.0 * np.pi * np.asarray(m.freqs, dtype=np.float64)
    pkey = (tuple(omega.tolist()), dt, n_steps)
    if pkey not in phase_cache:
        ph = np.empty((n_steps, omega.size), dtype=np.complex128)
        for q in range(n_steps):
            ph[q] = np.exp(1j * omega * ((q + 1.0) * dt))
        phase_cache[pkey] = ph
    dl = tuple(float(d) for d in grid.cell_size[:2])
    return dict(nx=nx, ny=ny, npdt=npdt, edt=edt, dt=dt, n_steps=n_steps, dl=dl,
                ch=float(npdt(dt / MU_0)), ce=np.ascontiguousarray(ce, dtype=npdt), eps=eps64,
                coef=coef,
                sources=src, line_i=line_i, omega=omega, phase_key=pkey)


def psi_cells(tab) -> int:
    """CPML psi entries of one instance (where c != 0 along each axis)."""
    nx, ny = tab["nx"], tab["ny"]
    c = tab["coef"]
    npex, nphx = int(np.count_nonzero(c[1])), int(np.count_nonzero(c[3]))
    npey, nphy = int(np.count_nonzero(c[5])), int(np.count_nonzero(c[7]))
    return nphx * ny + nx * nphy + nx * npey + npex * ny


def default_checkpoint(n_steps: int, state_reals: int, design_cells: int) -> int:
    """K minimising stored reals: (N/K) states of `state_reals` plus a ring
    of K steps x 2 reals per design cell, i.e. K = sqrt(N * state / (2 D))."""
    k = math.sqrt(n_steps * state_reals / max(2.0 * design_cells, 1.0))
    return int(max(1, min(n_steps, round(k))))


def checkpoint_bytes(n_steps: int, k: int, state_reals: int, design_cells: int,
                     real_bytes: int) -> int:
    """Stored bytes of the adjoint at spacing K: ceil(N/K) - 1 states plus a
    ring of K steps x 2 reals per design cell."""
    return (((n_steps + k - 1) // k - 1) * state_reals + k * 2 * design_cells) * real_bytes


def choose_checkpoint(n_steps: int, state_reals: int, design_cells: int, real_bytes: int,
                      budget_bytes: float) -> int:
    """The largest K whose stored bytes fit `budget_bytes`: the fewest
    segments, hence the least forward replay (K >= N: none at all). When no
    K fits, the memory-minimising default_checkpoint."""
    k0 = default_checkpoint(n_steps, state_reals, design_cells)
    for segs in range(1, n_steps + 1):  # K = ceil(N / segs), largest first
        k = (n_steps + segs - 1) // segs
        if k < k0:
            break
        if checkpoint_bytes(n_steps, k, state_reals, design_cells, real_bytes) <= budget_bytes:
            return k
    return k0


def default_memory_budget() -> float:
    """Half of the device memory free now (0 without a CUDA device)."""
    try:
        import torch
        if torch.cuda.is_available():
            return 0.5 * float(torch.cuda.mem_get_info()[0])
    except Exception:  # noqa: BLE001 - no usable CUDA runtime: no budget
        pass
    return 0.0


# --------------------------------------------------------------------------- #
# The batch
# --------------------------------------------------------------------------- #
class BatchTE:
    """One GPU batch of 2D TE instances with forward and adjoint passes.

    ``windows[k] = (i0, j0, n)`` is instance k's design window. ``checkpoint_every``
    (K) trades memory for replay time only: the adjoint replays the forward
    once between checkpoints; K >= n_steps stores no state at all and skips
    the replay. Results do not depend on K. The default is the largest K
    whose stored bytes fit ``memory_budget`` (default: half of the device
    memory free at construction): on a B200 a config-4 batch keeps its whole
    33.5 GB ring and replays nothing; a batch that does not fit gets the
    memory-minimising K. ``tile_rows`` is the x height of a work tile (8, 16
    or 32 rows by 32 cells); "auto" (the default) lets the autotuner time a
    short forward chunk at each height on this batch and keep the fastest
    (``tile_ms_per_step`` records the three timings). Results do not depend
    on the tile height.
    """

    def __init__(self, sims: Sequence, windows: Sequence[Tuple[int, int, int]],
                 checkpoint_every: Optional[int] = None, tile_rows="auto",
                 memory_budget: Optional[float] = None, tune_steps: int = 64):
        if len(sims) == 0 or len(sims) != len(windows):
            raise ValueError("need one design window per simulation")
        wave_cache: Dict = {}
        phase_cache: Dict = {}
        tabs = [instance_tables(s, wave_cache, phase_cache) for s in sims]
        t0 = tabs[0]
        for t in tabs[1:]:
            for key in ("npdt", "dt", "n_steps", "dl", "ch", "phase_key"):
                if t[key] != t0[key]:
                    raise ValueError(f"BatchTE: instances differ in {key}")
        self.tabs = tabs
        self.n_inst = len(tabs)
        self.npdt, self.edt = t0["npdt"], t0["edt"]
        self.dt, self.n_steps = t0["dt"], t0["n_steps"]
        self.omega = t0["omega"]
        self.n_freq = int(self.omega.size)
        self.windows = [tuple(int(v) for v in w) for w in windows]
        self.ny = np.array([t["ny"] for t in tabs], np.int64)
        self.line_off = np.concatenate([[0], np.cumsum(self.ny)])
        dsz = np.array([w[2] * w[2] for w in self.windows], np.int64)
        self.design_off = np.concatenate([[0], np.cumsum(dsz)])
        self.n_line = int(self.line_off[-1])
        self.n_design = int(self.design_off[-1])
        self.ncell = int(sum(t["nx"] * t["ny"] for t in tabs))
        state = 3 * self.ncell + sum(psi_cells(t) for t in tabs)
        if checkpoint_every is None:
            budget = default_memory_budget() if memory_budget is None else memory_budget
            checkpoint_every = choose_checkpoint(self.n_steps, state, self.n_design,
                                                 np.dtype(self.npdt).itemsize, budget)
        self._L = N.lib()
        L = self._L
        h = C.c_void_p()
        rb = np.dtype(self.npdt).itemsize
        N.check(L.pfb_create(self.n_inst, rb, t0["dl"][0], t0["dl"][1], t0["ch"], self.dt,
                             self.n_steps, C.byref(h)), None, batch=True)
        self.h = h
        try:
            auto = tile_rows == "auto"
            self._setup(tabs, wave_cache, phase_cache, int(checkpoint_every),
                        32 if auto else int(tile_rows))
            self.tile_ms_per_step = None
            self.tile_rows = 32 if auto else int(tile_rows)
            if auto:
                ms = (C.c_float * 3)()
                best = C.c_int(0)
                self._chk(L.pfb_tune_tiles(h, int(tune_steps), ms, C.byref(best)))
                self.tile_rows = int(best.value)
                self.tile_ms_per_step = {r: float(m) for r, m in zip((8, 16, 32), ms)}
        except Exception:
            self.close()
            raise
        # the design permittivity each instance starts from
        self._eps = np.concatenate([t["eps"][w[0]:w[0] + w[2], w[1]:w[1] + w[2]].ravel()
                                    for t, w in zip(tabs, self.windows)])
        for t in tabs:
            del t["ce"], t["eps"]
        self._forward_eps: Optional[np.ndarray] = None

    def _chk(self, rc):
        N.check(rc, self.h, batch=True)

    def _setup(self, tabs, wave_cache, phase_cache, K, tile_rows):
        L, h = self._L, self.h
        for k, (t, w) in enumerate(zip(tabs, self.windows)):
            coef = (C.c_void_p * 8)(*[a.ctypes.data for a in t["coef"]])
            self._chk(L.pfb_set_instance(h, k, t["nx"], t["ny"], N.ptr(t["ce"]), coef,
                                         w[0], w[1], w[2], t["line_i"]))
        rows = sorted(wave_cache.values(), key=lambda v: v[0])
        wave = (np.ascontiguousarray(np.stack([r[1] for r in rows]))
                if rows else np.zeros((1, self.n_steps)))
        inst, comp, ii, jj, row, amp = [], [], [], [], [], []
        for k, t in enumerate(tabs):
            for c, i, j, r, a in t["sources"]:
                inst.append(k)
                comp.append(c)
                ii.append(i)
                jj.append(j)
                row.append(r)
                amp.append(a)
        arr = [np.array(v, np.int32) for v in (inst, comp, ii, jj, row)]
        amp_a = np.array(amp, np.float64)
        self._chk(L.pfb_set_sources(h, len(inst), *[N.ptr(a, C.c_int32) for a in arr],
                                    N.ptr(amp_a, C.c_double), int(wave.shape[0]),
                                    N.ptr(wave, C.c_double)))
        ph = np.ascontiguousarray(phase_cache[tabs[0]["phase_key"]]).view(np.float64)
        self._chk(L.pfb_set_dft(h, self.n_freq, N.ptr(ph, C.c_double)))
        self._chk(L.pfb_finalize(h, K, tile_rows))

    # ---- packed layouts ----------------------------------------------- #
    def line_slice(self, k: int) -> slice:
        return slice(int(self.line_off[k]), int(self.line_off[k + 1]))

    def design_slice(self, k: int) -> slice:
        return slice(int(self.design_off[k]), int(self.design_off[k + 1]))

    def dft_of(self, packed: np.ndarray, k: int) -> np.ndarray:
        """Instance k's line DFT as (n_freq, ny), from a packed (n_line, n_freq) array."""
        return np.asarray(packed)[self.line_slice(k)].T

    def window_of(self, packed: np.ndarray, k: int) -> np.ndarray:
        n = self.windows[k][2]
        return np.asarray(packed)[self.design_slice(k)].reshape(n, n)

    def pack_windows(self, arrays: Sequence[np.ndarray]) -> np.ndarray:
        return np.concatenate([np.asarray(a, np.float64).ravel() for a in arrays])

    def per_instance_sum(self, values):
        """Sum of a packed (n_line, ...) torch tensor over each instance's line
        cells and trailing axes: one value per instance."""
        import torch
        idx = torch.repeat_interleave(torch.arange(self.n_inst), torch.as_tensor(self.ny))
        v = values.reshape(values.shape[0], -1).sum(dim=1)
        out = torch.zeros(self.n_inst, dtype=v.dtype, device=v.device)
        return out.index_add(0, idx.to(v.device), v)

    # ---- passes -------------------------------------------------------- #
    def design_eps(self) -> np.ndarray:
        """Current packed design permittivity (float64)."""
        return self._eps.copy()

    def set_design_eps(self, eps_packed: np.ndarray) -> None:
        """New design permittivity (packed, n_design); the coefficients are
        dt / (eps * EPS_0) evaluated in the field type, as the reference does
        for an assigned eps_r grid."""
        eps = np.ascontiguousarray(eps_packed, dtype=np.float64).ravel()
        if eps.size != self.n_design:
            raise ValueError(f"expected {self.n_design} design values, got {eps.size}")
        ce = (self.dt / (eps.astype(self.npdt) * EPS_0)).astype(self.edt, copy=False)
        ce = np.ascontiguousarray(ce, dtype=self.npdt)
        self._chk(self._L.pfb_set_design_ce(self.h, N.ptr(ce)))
        self._eps = eps.copy()

    def forward(self) -> np.ndarray:
        """All steps from zero fields; the packed line DFT (n_line, n_freq)."""
        self._chk(self._L.pfb_forward(self.h))
        self._forward_eps = self._eps.copy()
        return self.read_dft()

    def read_dft(self) -> np.ndarray:
        out = np.empty((self.n_line, self.n_freq), np.complex128)
        self._chk(self._L.pfb_read_dft(self.h, N.ptr(out.view(np.float64), C.c_double)))
        return out

    def adjoint(self, cotangent: np.ndarray) -> np.ndarray:
        """dL/dK (packed over the design cells) for DFT cotangent
        G = dL/dRe F + i dL/dIm F (packed (n_line, n_freq) complex)."""
        g = np.ascontiguousarray(cotangent, dtype=np.complex128)
        if g.shape != (self.n_line, self.n_freq):
            raise ValueError(f"cotangent must be ({self.n_line}, {self.n_freq}) complex")
        self._chk(self._L.pfb_adjoint(self.h, N.ptr(g.view(np.float64), C.c_double)))
        out = np.empty(self.n_design, np.float64)
        self._chk(self._L.pfb_read_grad(self.h, N.ptr(out, C.c_double)))
        return out

    def grad_eps(self, grad_k: np.ndarray, eps: Optional[np.ndarray] = None) -> np.ndarray:
        """Chain rule through K = dt / (eps EPS_0): dL/deps = -dL/dK * dt / (EPS_0 eps^2)."""
        e = self._forward_eps if eps is None else np.asarray(eps, np.float64)
        return -np.asarray(grad_k) * self.dt / (EPS_0 * e * e)

    def read_field(self, k: int, comp: str) -> np.ndarray:
        t = self.tabs[k]
        out = np.empty((t["nx"], t["ny"]), dtype=self.npdt)
        self._chk(self._L.pfb_read_field(self.h, k, _TE_COMP[comp], N.ptr(out)))
        return out

    def info(self) -> dict:
        v = (C.c_int64 * 9)()
        self._chk(self._L.pfb_info(self.h, v, 9))
        keys = ("cells", "line_cells", "design_cells", "tiles", "checkpoint_every",
                "segments", "state_reals", "launches", "fused")
        return dict(zip(keys, list(v)))

    def stream(self) -> int:
        return int(self._L.pfb_stream(self.h) or 0)

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            self._L.pfb_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------- #
# Autograd
# --------------------------------------------------------------------------- #
def _line_dft_function():
    import torch

    class LineDFT(torch.autograd.Function):
        """eps (packed design permittivity, float64) -> packed line DFT
        (n_line, n_freq complex128); backward runs the batch's adjoint.

        ``batch`` is any object with ``set_design_eps``, ``forward``,
        ``adjoint`` and ``grad_eps`` (a ``BatchTE``)."""

        @staticmethod
        def forward(ctx, eps, batch):
            e = eps.detach().to("cpu", torch.float64).numpy()
            batch.set_design_eps(e)
            F = batch.forward()
            ctx.batch = batch
            ctx.eps_np = e
            ctx.eps_meta = (eps.dtype, eps.device)
            return torch.from_numpy(F).to(eps.device)

        @staticmethod
        def backward(ctx, grad_F):
            g = grad_F.detach().to("cpu", torch.complex128).numpy()
            gk = ctx.batch.adjoint(g)
            ge = ctx.batch.grad_eps(gk, ctx.eps_np)
            dtype, device = ctx.eps_meta
            return torch.from_numpy(ge).to(device=device, dtype=dtype), None

    return LineDFT


_LINE_DFT = None


def line_dft(eps, batch):
    """Differentiable packed line DFT of the batch for design permittivity
    ``eps`` (a torch tensor); see LineDFT."""
    global _LINE_DFT
    if _LINE_DFT is None:
        _LINE_DFT = _line_dft_function()
    return _LINE_DFT.apply(eps, batch)


def value_and_grad_eps(batch, eps: np.ndarray, loss=None):
    """(values, dloss/deps) for every instance of the batch.

    ``loss(F)`` maps the packed line DFT (torch complex128, (n_line, n_freq))
    to one value per instance (torch, (n_inst,)); the default is the
    per-instance sum of |F|^2. Mirrors the reference's
    ``value_and_grad_eps(sim, loss)`` (jaxbackend.py:666-722), batched, with
    the gradient restricted to each instance's design window (packed)."""
    import torch
    e = torch.tensor(np.asarray(eps, np.float64), requires_grad=True)
    F = line_dft(e, batch)
    if loss is None:
        vals = batch.per_instance_sum(F.real ** 2 + F.imag ** 2)
    else:
        vals = loss(F)
    vals.sum().backward()
    return vals.detach().numpy(), e.grad.detach().numpy()
