"""Host driver of the B200 stepping engine: tables, C-ABI calls, Result.

``run_b200(sim)`` is the backend entry point. It accepts any object with the
reference ``Simulation``'s attributes (this package's ``Simulation`` or the
reference's own, through ``photonfdtd_b200.plugin.install()``), builds the
tables the engine consumes, steps the engine, and assembles a ``Result``.

It mirrors the reference's Rust/CUDA driver (src/photonfdtd/rustbackend.py:
85-120 validation, :135-166 tables, :310-447 chunked loop) with one
difference: DFT and flux monitors accumulate on the device, so the host stops
the engine only at FieldMonitor steps (and for progress callbacks).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Tuple

import ctypes

import numpy as np

from . import _native as N
from .scene import EPS_0, MU_0

_COMP = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5}
_FIELD_KEYS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_COMPUTE_KEYS = _FIELD_KEYS + ("eps_r", "psi")


# --------------------------------------------------------------------------- #
# Validation (rustbackend.py:85-120 for the shared rules)
# --------------------------------------------------------------------------- #
def validate(sim) -> None:
    dts = {np.dtype(sim.dtypes[k]) for k in _COMPUTE_KEYS}
    if dts not in ({np.dtype(np.float64)}, {np.dtype(np.float32)}):
        raise NotImplementedError(
            "backend='b200' needs one uniform compute precision ('float32' or "
            "'float64'; monitor storage may differ).")
    if getattr(sim, "particle_sources", None):
        raise NotImplementedError(
            "ChargedParticle sources are not supported on the b200 backend.")
    for m in sim.monitors:
        kind = type(m).__name__
        if kind == "FieldMonitor" and getattr(m, "compression", None) is not None:
            raise NotImplementedError(
                "FieldMonitor(compression=) is a host-side store not wired to the "
                "b200 backend; drop compression.")
        if kind not in ("FieldMonitor", "DFTMonitor", "FluxMonitor"):
            raise NotImplementedError(f"unsupported monitor type {kind}")
    if getattr(sim, "subpixel", False) and getattr(sim, "_has_dispersion", False):
        raise NotImplementedError(
            "Subpixel smoothing combined with dispersive media is not yet supported.")


# --------------------------------------------------------------------------- #
# Rasterisation helpers
# --------------------------------------------------------------------------- #
def _cells(structure, grid):
    """Index selector of a structure's cells: slices for boxes, else a mask."""
    if hasattr(structure, "index_slices"):
        return structure.index_slices(grid)
    return structure.region_mask(grid)


def _stamp(arr, sel, value) -> None:
    """arr[sel] = value; a boolean mask goes through copyto(where=), which
    numpy runs about twice as fast as masked assignment."""
    if isinstance(sel, np.ndarray) and sel.dtype == np.bool_:
        np.copyto(arr, arr.dtype.type(value), where=sel)
    else:
        arr[sel] = value


def _medium_eps(med) -> float:
    return float(med.eps_r)


def _eps_dtype(sim):
    return np.dtype(sim.dtypes["eps_r"]).type


_MAX_MEDIA = 16  # dispersive media one engine takes (4 bits of the ADE word)


def material_words(sim, edt=None, disp_bits=False):
    """Per-cell uint32 word in table mode, the table values, and ADE cells.

    Stamps value indices instead of permittivities in structure order
    (later overwrites earlier, simulation.py:539-544) and, in the same pass,
    the dispersive medium id (simulation.py:579-590). Returns
    (word, eps_values, med_ids, media) where med_ids is an int16 grid
    (-1 = not dispersive) and media the dispersive media in first-use order.
    With ``disp_bits`` a dispersive structure stamps 0x80000000 | m << 27
    (m its medium's first-use index) in place of a value index and med_ids
    is None: pf_rank_dispersive_words then numbers each medium's cells.
    """
    grid = sim.grid
    shape = tuple(grid.shape)
    vals: List[float] = [1.0]
    lookup: Dict[float, int] = {1.0: 0}
    word = np.zeros(shape, dtype=np.uint32)
    med_ids = None if disp_bits else np.full(shape, -1, dtype=np.int16)
    media, med_index = [], {}
    edt = _eps_dtype(sim) if edt is None else edt
    for s in sim.structures:
        sel = _cells(s, grid)
        if sel is None:
            continue
        med = s.medium
        v = float(edt(_medium_eps(med)))
        if v not in lookup:
            lookup[v] = len(vals)
            vals.append(v)
        disp = getattr(med, "is_dispersive", False)
        if disp and id(med) not in med_index:
            med_index[id(med)] = len(media)
            media.append(med)
        if disp_bits:
            if disp:
                m = med_index[id(med)]
                if m >= _MAX_MEDIA:
                    raise NotImplementedError(
                        f"at most {_MAX_MEDIA} dispersive media, the scene has more")
                _stamp(word, sel, 0x80000000 | (m << 27))
            else:
                _stamp(word, sel, lookup[v])
            continue
        _stamp(word, sel, lookup[v])
        _stamp(med_ids, sel, med_index[id(med)] if disp else -1)
    return word, np.array(vals, dtype=edt), med_ids, media


def ade_tables(sim, med_ids, media, dt, counts=None):
    """Compact dispersive-cell indexing and pole coefficients
    (simulation.py:592-636): a = (2 - w0^2 dt^2)/(1 + g dt),
    b = (g dt - 1)/(1 + g dt), c = eps0 S dt^2/(1 + g dt), per pole.
    ``counts`` (cells per medium, from pf_rank_dispersive_words) replaces
    the scan of med_ids: every medium is kept, cell lists are not built."""
    wmax = 0.0
    for med in media:
        wmax = max(wmax, med.max_pole_omega() * dt)
    if wmax >= 2.0:
        raise ValueError(
            f"A dispersive medium has a pole with omega0*dt = {wmax:.2f} >= 2, which "
            "makes the explicit ADE update unstable at this resolution. Use a finer "
            "grid, restrict the medium to poles inside the simulation band, or use "
            "DispersiveMedium.at_wavelength(lambda) for a fixed-index Medium.")
    flat = None if counts is not None else med_ids.ravel()
    kept, base, count, npole, coef, inv, cells = [], [], [], [], [], [], []
    g = 0
    for m, med in enumerate(media):
        n = int(counts[m]) if counts is not None else None
        idx = np.flatnonzero(flat == m) if counts is None else None
        if counts is None:
            if idx.size == 0:
                continue
            n = idx.size
        kept.append(med)
        base.append(g)
        count.append(n)
        npole.append(len(med.poles))
        for p in med.poles:
            den = 1.0 + p.gamma * dt
            coef += [(2.0 - p.omega0 ** 2 * dt ** 2) / den, (p.gamma * dt - 1.0) / den,
                     (EPS_0 * p.strength * dt ** 2) / den]
        inv.append(1.0 / (EPS_0 * med.eps_inf))
        cells.append(idx)
        g += n
    return dict(media=kept, base=np.array(base, np.int64), count=np.array(count, np.int64),
                npole=np.array(npole, np.int32), coef=np.array(coef, np.float64),
                inv=np.array(inv, np.float64), cells=cells)


# --------------------------------------------------------------------------- #
# Monitor geometry
# --------------------------------------------------------------------------- #
def _nearest(coord, pos) -> int:
    return int(np.argmin(np.abs(np.asarray(coord) - pos)))


def dft_region(m, grid):
    """start/stop/stride per axis of a DFTMonitor's snapshot
    (simulation.py:1072-1078: strided by downsample, one plane if set)."""
    ds = m.downsample
    start, stop, stride = [0, 0, 0], list(grid.shape), [ds if ds > 1 else 1] * 3
    pl = m.plane()
    if pl is not None:
        ax, pos = pl
        ci = _nearest(grid.coords[ax], pos)
        start[ax], stop[ax], stride[ax] = ci, ci + 1, 1
    counts = tuple(len(range(a, b, s)) for a, b, s in zip(start, stop, stride))
    return start, stop, stride, counts


def flux_plane(m, grid) -> Tuple[int, int, float]:
    """(axis, index, dA) of a FluxMonitor (simulation.py:1440-1459)."""
    ax = {"x": 0, "y": 1, "z": 2}[m.plane_axis]
    co = grid.coords[ax]
    idx = 0 if co.size == 1 else _nearest(co, m.plane_position)
    w = [grid.cell_size[a] if grid.shape[a] > 1 else 1.0 for a in range(3)]
    others = [a for a in range(3) if a != ax]
    return ax, idx, w[others[0]] * w[others[1]]


# --------------------------------------------------------------------------- #
# Tables
# --------------------------------------------------------------------------- #
def _smoothed_components(sim, dtype):
    """The subpixel tensor in `dtype`: the simulation's own components when
    that is its working type, else recomputed (on the GPU for box scenes)."""
    if np.dtype(dtype) == np.dtype(_eps_dtype(sim)):
        return sim._smoothed_eps_components()
    from .smoothing import device_available, smooth_permittivity, smooth_permittivity_device
    if device_available():
        try:
            return smooth_permittivity_device(sim.grid, sim.structures, background_eps=1.0,
                                              factor=sim.subpixel_factor, dtype=dtype)
        except NotImplementedError:
            pass
    return smooth_permittivity(sim.grid, sim.structures, background_eps=1.0,
                               factor=sim.subpixel_factor, dtype=dtype)


def build_tables(sim, dtype=None, ce3=None) -> dict:
    """Everything the engine consumes, in the forms the C ABI takes.

    dtype (np.float32 / np.float64) overrides the simulation's working
    precision: a float64 shadow of a float32 scene (the error statement of
    photonfdtd_b200.accuracy) evaluates every table as a float64 run of the
    same scene would. ``ce3`` (three grid-shaped arrays) replaces the E
    coefficients of Ex, Ey, Ez outright (PF_CE_CELL3), as the reference's
    value_and_grad_params does with its ce_of_params (jaxbackend.py:725-775)."""
    grid = sim.grid
    npdt = np.dtype(sim.dtypes["Ex"] if dtype is None else dtype).type
    dt, n_steps = float(sim.dt), int(sim.n_steps)
    t = dict(shape=tuple(grid.shape), npdt=npdt, dt=dt, n_steps=n_steps,
             dl=tuple(d if d > 0 else 1.0 for d in grid.cell_size),
             ch=float(npdt(dt / MU_0)))
    t["cpml"] = [tuple(np.ascontiguousarray(np.asarray(arr[a]), dtype=npdt)
                       for arr in (sim._b_e, sim._c_e, sim._b_h, sim._c_h)) for a in range(3)]
    edt = _eps_dtype(sim) if dtype is None else npdt
    custom = bool(getattr(sim, "_eps_r_custom", False))
    need_ids = getattr(sim, "_has_dispersion", False) or not (custom or sim.subpixel
                                                               or ce3 is not None)
    word = vals = None
    media: list = []
    if need_ids:
        word, vals, _, media = material_words(sim, edt, disp_bits=True)
    table_mode = ce3 is None and not (sim.subpixel and not custom) and not custom
    ade = None
    if media:
        # rank the dispersive cells per medium in one native pass: in place in
        # table mode (the ce word carries them), else in a copy whose plain
        # cells are zeroed (the separate ADE cell word)
        cw = word.reshape(-1) if table_mode else word.reshape(-1).copy()
        counts = np.zeros(len(media), np.int64)
        N.check(N.lib().pf_rank_dispersive_words(N.ptr(cw, ctypes.c_uint32), cw.size, len(media),
                                                 N.ptr(counts, ctypes.c_int64),
                                                 0 if table_mode else 1))
        if counts.sum() > 0:
            ade = ade_tables(sim, None, media, dt, counts=counts)
            ade["cell_word"] = None if table_mode else cw
    if ce3 is not None:
        if len(ce3) != 3 or any(np.shape(c) != tuple(grid.shape) for c in ce3):
            raise ValueError("ce3 must hold three arrays of the grid's shape")
        t["ce_mode"] = N.PF_CE_CELL3
        t["ce"] = [np.ascontiguousarray(np.asarray(c), dtype=npdt) for c in ce3]
    elif sim.subpixel and not custom:
        comps = _smoothed_components(sim, edt)
        t["ce_mode"] = N.PF_CE_CELL3
        t["ce"] = [np.ascontiguousarray((dt / (np.asarray(e) * EPS_0)).astype(edt, copy=False),
                                        dtype=npdt) for e in comps]
    elif custom:
        eps = np.asarray(sim.eps_r).astype(edt, copy=False)
        t["ce_mode"] = N.PF_CE_CELL1
        t["ce"] = [np.ascontiguousarray((dt / (eps * EPS_0)).astype(edt, copy=False),
                                        dtype=npdt)]
    else:
        t["ce_mode"] = N.PF_CE_TABLE
        t["table"] = (dt / (vals * EPS_0)).astype(edt, copy=False).astype(np.float64)
        t["word"] = word
    if ade is not None:
        # dispersive word: bit 31 | medium << 27 | rank of the cell among the
        # medium's cells in C order (pf_rank_dispersive_words above); the
        # coefficient a dispersive cell gets from its stamped eps_inf
        ade["ce_m"] = np.array([float((dt / (np.array([med.eps_r], dtype=edt) * EPS_0))
                                      .astype(edt)[0]) for med in ade["media"]], np.float64)
        del ade["cells"]
    t["ade"] = ade
    t["sources"] = source_tables(sim, n_steps, dt)
    t["dft"], t["flux"] = [], []
    for m in sim.monitors:
        kind = type(m).__name__
        if kind == "DFTMonitor":
            start, stop, stride, counts = dft_region(m, grid)
            omega = 2.0 * np.pi * np.asarray(m.freqs, dtype=np.float64)
            mask = 0
            for c in m.components:
                mask |= 1 << _COMP[c]
            steps = range(0, n_steps, m.interval)
            ph_e = np.empty((len(steps), omega.size), dtype=np.complex128)
            ph_h = np.empty_like(ph_e)
            for q, s in enumerate(steps):
                ph_e[q] = np.exp(1j * omega * ((s + 1.0) * dt))
                ph_h[q] = np.exp(1j * omega * ((s + 0.5) * dt))
            t["dft"].append(dict(m=m, start=start, stop=stop, stride=stride, counts=counts,
                                 mask=mask, omega=omega, ph_e=ph_e, ph_h=ph_h))
        elif kind == "FluxMonitor":
            ax, idx, da = flux_plane(m, grid)
            t["flux"].append(dict(m=m, axis=ax, idx=idx, dA=da))
    return t


def source_tables(sim, n_steps: int, dt: float) -> dict:
    """Per-source component, flat cell, waveform row and amplitude, plus the
    waveform rows: value of each distinct waveform at its family's Yee times
    ((s+1/2)dt for H, (s+1)dt for E; simulation.py:1322-1323), evaluated one
    time at a time exactly as the reference's loop calls it."""
    grid = sim.grid
    ny, nz = grid.shape[1], grid.shape[2]
    rows: Dict[tuple, int] = {}
    wave_rows: List[np.ndarray] = []
    comp, cell, row, amp = [], [], [], []
    for src in sim.sources:
        i, j, k = grid.index_at(src.position)
        fam = src.component[0]
        key = (id(src.waveform), fam)
        if key not in rows:
            off = 0.5 if fam == "H" else 1.0
            vals = np.empty(n_steps, dtype=np.float64)
            for s in range(n_steps):
                vals[s] = src.waveform(np.array([(s + off) * dt]))[0]
            rows[key] = len(wave_rows)
            wave_rows.append(vals)
        comp.append(_COMP[src.component])
        cell.append((i * ny + j) * nz + k)
        row.append(rows[key])
        amp.append(float(src.amplitude))
    wave = np.stack(wave_rows) if wave_rows else np.zeros((0, n_steps))
    return dict(comp=np.array(comp, np.int32), cell=np.array(cell, np.int64),
                row=np.array(row, np.int32), amp=np.array(amp, np.float64),
                wave=np.ascontiguousarray(wave, dtype=np.float64))


# --------------------------------------------------------------------------- #
# Native engine handle
# --------------------------------------------------------------------------- #
class B200Engine:
    """One device engine; ``advance(step0, n_sub)`` and ``get(comp)`` follow
    the reference engine protocol (rustbackend.py:222-234, 297-304)."""

    def __init__(self, t: dict, kernel: int = N.PF_KERNEL_AUTO):
        L = N.lib()
        nx, ny, nz = t["shape"]
        self.shape = t["shape"]
        self.npdt = t["npdt"]
        h = C_void()
        N.check(L.pf_create(nx, ny, nz, np.dtype(self.npdt).itemsize, t["dl"][0], t["dl"][1],
                            t["dl"][2], t["ch"], t["n_steps"], C_byref(h)), None)
        self.h = h
        self._L = L
        try:
            self._setup(t, kernel)
        except Exception:
            self.close()
            raise
        self._cache: Dict[str, np.ndarray] = {}

    def _chk(self, rc):
        N.check(rc, self.h)

    def _setup(self, t, kernel):
        L, h = self._L, self.h
        import ctypes as C
        keep = []  # arrays must outlive the calls that borrow them
        if t["ce_mode"] == N.PF_CE_TABLE:
            word = np.ascontiguousarray(t["word"], dtype=np.uint32)
            tab = np.ascontiguousarray(t["table"], dtype=np.float64)
            keep += [word, tab]
            self._chk(L.pf_set_ce(h, N.PF_CE_TABLE, None, None, None, N.ptr(word, C.c_uint32),
                                  tab.size, N.ptr(tab, C.c_double)))
        else:
            ce = t["ce"]
            arrs = [ce[0], ce[0], ce[0]] if len(ce) == 1 else ce
            self._chk(L.pf_set_ce(h, t["ce_mode"], N.ptr(arrs[0]), N.ptr(arrs[1]),
                                  N.ptr(arrs[2]), None, 0, None))
        for ax in range(3):
            be, ce, bh, ch = t["cpml"][ax]
            self._chk(L.pf_set_cpml(h, ax, N.ptr(be), N.ptr(ce), N.ptr(bh), N.ptr(ch)))
        ade = t["ade"]
        if ade is not None:
            cw = ade["cell_word"]
            self._chk(L.pf_set_ade(h, len(ade["media"]), N.ptr(ade["count"], C.c_int64),
                                   N.ptr(ade["npole"], C.c_int32),
                                   N.ptr(ade["coef"], C.c_double), N.ptr(ade["inv"], C.c_double),
                                   N.ptr(ade["ce_m"], C.c_double),
                                   None if cw is None else N.ptr(cw, C.c_uint32)))
        s = t["sources"]
        self._chk(L.pf_set_sources(h, int(s["comp"].size), N.ptr(s["comp"], C.c_int32),
                                   N.ptr(s["cell"], C.c_int64), N.ptr(s["row"], C.c_int32),
                                   N.ptr(s["amp"], C.c_double), int(s["wave"].shape[0]),
                                   N.ptr(s["wave"], C.c_double)))
        self.dft_ids = []
        for d in t["dft"]:
            st = np.array(d["start"], np.int32)
            sp = np.array(d["stop"], np.int32)
            sd = np.array(d["stride"], np.int32)
            pe = np.ascontiguousarray(d["ph_e"]).view(np.float64)
            ph = np.ascontiguousarray(d["ph_h"]).view(np.float64)
            mid = C.c_int()
            self._chk(L.pf_add_dft(h, N.ptr(st, C.c_int32), N.ptr(sp, C.c_int32),
                                   N.ptr(sd, C.c_int32), d["mask"], int(d["omega"].size),
                                   int(d["m"].interval), N.ptr(pe, C.c_double),
                                   N.ptr(ph, C.c_double), t["dt"], C.byref(mid)))
            self.dft_ids.append(mid.value)
        self.flux_ids = []
        for f in t["flux"]:
            mid = C.c_int()
            self._chk(L.pf_add_flux(h, f["axis"], f["idx"], f["dA"], t["dt"], C.byref(mid)))
            self.flux_ids.append(mid.value)
        self._chk(L.pf_set_kernel(h, kernel))
        self._chk(L.pf_finalize(h))
        del keep

    def advance(self, step0: int, n_sub: int) -> None:
        self._cache.clear()
        self._chk(self._L.pf_advance(self.h, int(step0), int(n_sub)))

    def get(self, comp: str) -> np.ndarray:
        if comp not in self._cache:
            out = np.empty(self.shape, dtype=self.npdt)
            self._chk(self._L.pf_read_field(self.h, _COMP[comp], N.ptr(out)))
            self._cache[comp] = out
        return self._cache[comp]

    def get_region(self, comp: str, start, stop, stride) -> np.ndarray:
        """f[start:stop:stride] per axis of one current field, gathered on
        the device (pf_read_region); only the snapshot is copied out."""
        import ctypes as C
        st = np.array(start, np.int32)
        sp = np.array(stop, np.int32)
        sd = np.array(stride, np.int32)
        shape = tuple(len(range(a, b, c)) for a, b, c in zip(st, sp, sd))
        out = np.empty(shape, dtype=self.npdt)
        self._chk(self._L.pf_read_region(self.h, _COMP[comp], N.ptr(st, C.c_int32),
                                         N.ptr(sp, C.c_int32), N.ptr(sd, C.c_int32),
                                         N.ptr(out)))
        return out

    def set_field(self, comp: str, arr: np.ndarray) -> None:
        """Overwrite one component of the current state (pf_write_field)."""
        src = np.ascontiguousarray(arr, dtype=self.npdt)
        if src.shape != tuple(self.shape):
            raise ValueError(f"field of shape {src.shape}, the grid is {self.shape}")
        self._cache.clear()
        self._chk(self._L.pf_write_field(self.h, _COMP[comp], N.ptr(src)))

    def state_bytes(self) -> int:
        import ctypes as C
        v = C.c_int64()
        self._chk(self._L.pf_state_bytes(self.h, C.byref(v)))
        return int(v.value)

    def get_state(self) -> np.ndarray:
        """The stepping state blob (fields, psi, polarisation) as bytes."""
        out = np.empty(self.state_bytes(), dtype=np.uint8)
        self._chk(self._L.pf_get_state(self.h, N.ptr(out), out.size, 0))
        return out

    def set_state(self, step: int, blob: np.ndarray) -> None:
        """Restore a blob from get_state and set the step counter."""
        b = np.ascontiguousarray(blob, dtype=np.uint8)
        self._cache.clear()
        self._chk(self._L.pf_set_state(self.h, int(step), N.ptr(b), b.size, 0))

    def get_state_to(self, dev_ptr: int, nbytes: int) -> None:
        """Copy the state blob into device memory at dev_ptr (nbytes long)."""
        import ctypes as C
        self._chk(self._L.pf_get_state(self.h, C.c_void_p(dev_ptr), int(nbytes), 1))

    def step(self) -> int:
        import ctypes as C
        v = C.c_int64()
        self._chk(self._L.pf_step(self.h, C.byref(v)))
        return int(v.value)

    def read_dft(self, k: int, comp: str, n_freq: int, counts) -> np.ndarray:
        import ctypes as C
        out = np.empty((n_freq,) + tuple(counts), dtype=np.complex128)
        self._chk(self._L.pf_read_dft(self.h, self.dft_ids[k], _COMP[comp],
                                      N.ptr(out.view(np.float64), C.c_double)))
        return out

    def read_flux(self, k: int) -> float:
        import ctypes as C
        v = C.c_double()
        self._chk(self._L.pf_read_flux(self.h, self.flux_ids[k], C.byref(v)))
        return float(v.value)

    def stream(self) -> int:
        """Address of the engine's cudaStream_t."""
        import ctypes as C
        v = C.c_void_p()
        self._chk(self._L.pf_stream(self.h, C.byref(v)))
        return int(v.value or 0)

    def set_profiling(self, on: bool) -> None:
        self._chk(self._L.pf_set_profiling(self.h, 1 if on else 0))

    def read_profile(self, reset: bool = False):
        """(launches[4], ms[4]) per kind: step passes, sources, sampling, flush."""
        import ctypes as C
        n = (C.c_int64 * 4)()
        ms = (C.c_double * 4)()
        self._chk(self._L.pf_read_profile(self.h, n, ms, 1 if reset else 0))
        return list(n), list(ms)

    def info(self) -> dict:
        """Engine configuration (kernel path, tiling, division mode, ...)."""
        import ctypes as C
        buf = C.create_string_buffer(512)
        self._chk(self._L.pf_info(self.h, buf, 512))
        return dict(kv.split("=", 1) for kv in buf.value.decode().split())

    def device_bytes(self) -> int:
        import ctypes as C
        v = C.c_int64()
        self._chk(self._L.pf_device_bytes(self.h, C.byref(v)))
        return int(v.value)

    def check_finite(self) -> None:
        self._chk(self._L.pf_check_finite(self.h))

    def set_check_every(self, k: int) -> None:
        """Scan for inf / nan every k steps while advancing (0: off)."""
        self._chk(self._L.pf_set_check_every(self.h, int(k)))

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            self._L.pf_destroy(self.h)
            self.h = C_void()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def C_void():
    import ctypes as C
    return C.c_void_p()


def C_byref(x):
    import ctypes as C
    return C.byref(x)


# --------------------------------------------------------------------------- #
# Driver loop (rustbackend.py:310-447)
# --------------------------------------------------------------------------- #
def _result_cls(sim):
    """The Result dataclass of the simulation's own package."""
    mod = type(sim).__module__
    import importlib
    try:
        return importlib.import_module(mod).Result
    except (ImportError, AttributeError):
        from .simulation import Result
        return Result


def run_b200(sim, kernel: int = N.PF_KERNEL_AUTO):
    """Run ``sim`` on the B200 engine and return a Result.

    With ``sim.b200_check_every = k``, the engine scans the fields every k
    steps and raises NativeError (PF_ERR_NONFINITE) at the first inf / nan,
    e.g. a scene stepped past its Courant limit.

    With ``sim.b200_error_vs_f64 = True`` on a float32 scene, the Result also
    carries ``error_vs_f64``: every output's error against a float64 run of
    the same scene on the engine (photonfdtd_b200.accuracy), whose float64
    arithmetic reproduces the reference's float64 NumPy run to 1e-12."""
    import time
    t0 = time.perf_counter()
    validate(sim)
    t = build_tables(sim)
    t1 = time.perf_counter()
    eng = B200Engine(t, kernel=kernel)
    t2 = time.perf_counter()
    check = int(getattr(sim, "b200_check_every", 0) or 0)
    if check:
        eng.set_check_every(check)
    try:
        res = drive(sim, eng, t)
    finally:
        eng.close()
    t3 = time.perf_counter()
    LAST_RUN.clear()
    LAST_RUN.update(tables_s=t1 - t0, create_s=t2 - t1, run_s=t3 - t2,
                    advance_s=LAST_STEPPING_S[0],
                    h2d_bytes=upload_bytes(t), n_steps=t["n_steps"],
                    d2h_bytes=result_bytes(res), cells=int(np.prod(t["shape"])))
    if getattr(sim, "b200_error_vs_f64", False) and np.dtype(t["npdt"]) != np.float64:
        from .accuracy import error_vs_f64, float64_shadow
        res.error_vs_f64 = error_vs_f64(res, float64_shadow(sim, kernel))
    return res


# Phase timings and transfer sizes of the last run_b200 call (seconds, bytes):
# building the tables on the host, creating the engine (device allocation and
# upload), stepping with monitor read-back.
LAST_RUN: Dict[str, float] = {}
LAST_STEPPING_S = [0.0]  # time inside pf_advance during the last drive()


def upload_bytes(t) -> int:
    """Host-to-device bytes of an engine's tables."""
    n = 0
    if t["ce_mode"] == N.PF_CE_TABLE:
        n += t["word"].nbytes + t["table"].nbytes
    else:
        n += sum(a.nbytes for a in t["ce"])
    for ax in t["cpml"]:
        n += sum(a.nbytes for a in ax)
    if t["ade"] is not None and t["ade"]["cell_word"] is not None:
        n += t["ade"]["cell_word"].nbytes
    s = t["sources"]
    n += s["wave"].nbytes + s["amp"].nbytes + s["cell"].nbytes
    for d in t["dft"]:
        n += d["ph_e"].nbytes + d["ph_h"].nbytes
    return int(n)


def result_bytes(res) -> int:
    """Device-to-host bytes of a Result's monitor data."""
    n = 0
    for comps in res.fields.values():
        n += sum(np.asarray(a).nbytes for a in comps.values())
    for comps in res.dft.values():
        n += sum(np.asarray(a).nbytes for a in comps.values())
    return int(n + 8 * len(res.flux))


def field_plans(sim, n_steps: int, dt: float) -> Dict[str, dict]:
    """Per FieldMonitor: the steps after which a frame is taken and the
    snapshot region (start, stop, stride) (simulation.py:1062-1067: one z
    plane with plane_z, else every downsample-th cell per axis)."""
    grid = sim.grid
    plans: Dict[str, dict] = {}
    for m in sim.monitors:
        if type(m).__name__ != "FieldMonitor":
            continue
        if m.times is not None:
            steps = {int(round(tt / dt)) for tt in m.times if 0 <= int(round(tt / dt)) < n_steps}
        else:
            steps = set(range(0, n_steps, m.interval))
        ds = max(int(m.downsample), 1)
        shape = tuple(grid.shape)
        if m.plane_z is not None:
            zi = _nearest(grid.coords[2], m.plane_z)
            region = ((0, 0, zi), (shape[0], shape[1], zi + 1), (ds, ds, 1))
        else:
            region = ((0, 0, 0), shape, (ds, ds, ds))
        plans[m.name] = dict(m=m, steps=steps, region=region)
    return plans


def drive(sim, eng: B200Engine, t: dict, mon_dtype=None):
    grid = sim.grid
    dt, n_steps = t["dt"], t["n_steps"]
    mon_dtype = sim.dtypes["monitors"] if mon_dtype is None else mon_dtype
    Result = _result_cls(sim)
    result = Result(times=np.arange(n_steps) * dt)
    rec: Dict[str, dict] = {}
    for name, p in field_plans(sim, n_steps, dt).items():
        m = p["m"]
        rec[name] = dict(m=m, steps=p["steps"], region=p["region"], n=len(p["steps"]),
                         count=0, store={c: None for c in m.components}, times=[])

    stop_steps = sorted(set().union(*(r["steps"] for r in rec.values()))) if rec else []
    cb = getattr(sim, "progress_callback", None)
    every = max(n_steps // 100, 1)
    pos = 0

    import time
    stepping = [0.0]

    def advance_to(end):
        nonlocal pos
        while pos < end:
            n = min(end - pos, every) if cb is not None else end - pos
            t0 = time.perf_counter()
            eng.advance(pos, n)
            stepping[0] += time.perf_counter() - t0
            pos += n
            if cb is not None:
                cb(min(pos, n_steps), n_steps)

    for s in stop_steps:
        advance_to(s + 1)
        for r in rec.values():
            if s not in r["steps"]:
                continue
            m = r["m"]
            for c in m.components:
                snap = eng.get_region(c, *r["region"])
                if r["store"][c] is None:
                    r["store"][c] = np.empty((r["n"],) + snap.shape, dtype=mon_dtype)
                r["store"][c][r["count"]] = snap
            r["times"].append(s * dt)
            r["count"] += 1
    advance_to(n_steps)
    if cb is not None:
        cb(n_steps, n_steps)

    for m in sim.monitors:
        kind = type(m).__name__
        if kind == "FieldMonitor":
            r = rec[m.name]
            if r["count"] > 0:
                result.fields[m.name] = {c: r["store"][c] for c in m.components}
                result.monitor_times[m.name] = np.array(r["times"])
            else:
                result.fields[m.name] = {c: np.zeros((0,) + tuple(grid.shape))
                                         for c in m.components}
                result.monitor_times[m.name] = np.array([])
    for k, d in enumerate(t["dft"]):
        m = d["m"]
        result.dft_freqs[m.name] = np.asarray(m.freqs, dtype=np.float64)
        result.dft[m.name] = {c: eng.read_dft(k, c, d["omega"].size, d["counts"])
                              for c in m.components}
    for k, f in enumerate(t["flux"]):
        result.flux[f["m"].name] = eng.read_flux(k)
    LAST_STEPPING_S[0] = stepping[0]
    return result
