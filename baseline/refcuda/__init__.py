"""The reference's own CUDA stepping kernels, run on this GPU as a bar.

`RefCuda(sim)` builds the tables the reference's rust-cuda backend builds
(rustbackend._build_tables, rustbackend.py:135-166: ce_field = dt/(eps_r
eps0) per cell, CPML b/c per axis cast to the field dtype, compact CPML maps
where c != 0, per-source value rows amplitude * waveform((s + 1/2) dt or
(s + 1) dt)) and steps them with the reference's kernels through the harness
in launch.cu, compiled by build.py into baseline/_ref/. Same restrictions as
the reference backend (rustbackend.py:85-120): no dispersion, no subpixel
smoothing; monitors are not part of the kernels and are not run.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict = {}
EPS_0 = 8.8541878128e-12
MU_0 = 1.25663706212e-6
_COMP = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5}


def lib_path(precision: str) -> str:
    tag = "f32" if precision == "float32" else "f64"
    return os.path.join(os.path.dirname(_HERE), "_ref", f"librefcuda_{tag}.so")


def available(precision: str = "float32") -> bool:
    return os.path.exists(lib_path(precision))


def _lib(precision: str):
    if precision not in _LIBS:
        L = C.CDLL(lib_path(precision))
        rp = C.POINTER(C.c_float if precision == "float32" else C.c_double)
        rt = C.c_float if precision == "float32" else C.c_double
        vp = C.c_void_p
        L.refcuda_last_error.restype = C.c_char_p
        L.refcuda_real_size.restype = C.c_int
        L.refcuda_create.argtypes = [C.c_int] * 3 + [vp] * 7 + [rt] * 4 + \
            [C.c_int, vp, vp, vp, C.c_longlong, C.POINTER(vp)]
        L.refcuda_create.restype = C.c_int
        L.refcuda_run.argtypes = [vp, C.c_longlong, C.c_longlong, C.POINTER(C.c_float)]
        L.refcuda_run.restype = C.c_int
        L.refcuda_read.argtypes = [vp, C.c_int, vp]
        L.refcuda_read.restype = C.c_int
        L.refcuda_destroy.argtypes = [vp]
        L.refcuda_destroy.restype = None
        want = 4 if precision == "float32" else 8
        if L.refcuda_real_size() != want:
            raise RuntimeError(f"{lib_path(precision)}: wrong precision")
        _LIBS[precision] = L
    return _LIBS[precision]


def _pml_map(c: np.ndarray) -> np.ndarray:
    m = np.full(c.size, -1, dtype=np.int32)
    idx = np.flatnonzero(c != 0.0)
    m[idx] = np.arange(idx.size, dtype=np.int32)
    return m


def tables(sim) -> dict:
    """The reference backend's tables for `sim` (rustbackend.py:135-166)."""
    if getattr(sim, "_has_dispersion", False) or getattr(sim, "subpixel", False):
        raise NotImplementedError("the reference CUDA kernels take scalar ce, no dispersion")
    npdt = np.dtype(sim.dtypes["Ex"]).type
    dt, n_steps = float(sim.dt), int(sim.n_steps)
    t = dict(npdt=npdt, shape=tuple(sim.grid.shape), n_steps=n_steps,
             ce_field=np.ascontiguousarray(dt / (np.asarray(sim.eps_r, np.float64) * EPS_0),
                                           dtype=npdt),
             ch_field=npdt(dt / MU_0),
             b_e=[np.ascontiguousarray(a, dtype=npdt) for a in sim._b_e],
             c_e=[np.ascontiguousarray(a, dtype=npdt) for a in sim._c_e],
             b_h=[np.ascontiguousarray(a, dtype=npdt) for a in sim._b_h],
             c_h=[np.ascontiguousarray(a, dtype=npdt) for a in sim._c_h],
             dl=[npdt(d if d > 0 else 1.0) for d in sim.grid.cell_size])
    t["maps_e"] = [_pml_map(a) for a in t["c_e"]]
    t["maps_h"] = [_pml_map(a) for a in t["c_h"]]
    n_src = max(len(sim.sources), 1)
    steps = np.arange(n_steps)
    comp = np.zeros(n_src, np.int32)
    idx = np.zeros((n_src, 3), np.int32)
    vals = np.zeros((n_src, max(n_steps, 1)), npdt)
    for s, src in enumerate(sim.sources):
        comp[s] = _COMP[src.component]
        idx[s] = sim.grid.index_at(src.position)
        tt = (steps + (0.5 if src.component[0] == "H" else 1.0)) * dt
        vals[s] = np.asarray(src.amplitude * src.waveform(tt), dtype=npdt)
    t.update(src_comp=comp, src_idx=idx, src_vals=vals)
    return t


class RefCuda:
    """One simulation on the reference's kernels (device state, own stream)."""

    def __init__(self, sim):
        t = tables(sim)
        prec = "float32" if t["npdt"] is np.float32 else "float64"
        self.L = _lib(prec)
        self.t = t
        nx, ny, nz = t["shape"]
        for a, n in enumerate((nx, ny, nz)):
            for k in ("b_e", "c_e", "b_h", "c_h", "maps_e", "maps_h"):
                assert t[k][a].shape == (n,), (k, a, t[k][a].shape, n)
        assert t["ce_field"].shape == (nx, ny, nz)
        assert np.all((t["src_idx"] >= 0) & (t["src_idx"] < np.array([nx, ny, nz])))

        def arr(lst):
            return (C.c_void_p * 3)(*[a.ctypes.data for a in lst])
        self._keep = [arr(t[k]) for k in ("b_e", "c_e", "b_h", "c_h", "maps_e", "maps_h")]
        h = C.c_void_p()
        rc = self.L.refcuda_create(nx, ny, nz, t["ce_field"].ctypes.data, *self._keep,
                                   float(t["ch_field"]), *[float(d) for d in t["dl"]],
                                   int(t["src_comp"].size),
                                   t["src_comp"].ctypes.data, t["src_idx"].ctypes.data,
                                   t["src_vals"].ctypes.data, t["n_steps"], C.byref(h))
        self.h = h
        if rc != 0:
            msg = self.L.refcuda_last_error().decode()
            self.close()
            raise RuntimeError(msg)

    def run(self, step0: int, n: int, timed: bool = False):
        ms = C.c_float(0.0)
        rc = self.L.refcuda_run(self.h, step0, n, C.byref(ms) if timed else None)
        if rc != 0:
            raise RuntimeError(self.L.refcuda_last_error().decode())
        return ms.value if timed else None

    def field(self, comp: str) -> np.ndarray:
        out = np.empty(self.t["shape"], self.t["npdt"])
        if self.L.refcuda_read(self.h, _COMP[comp], out.ctypes.data) != 0:
            raise RuntimeError(self.L.refcuda_last_error().decode())
        return out

    def close(self):
        if getattr(self, "h", None):
            self.L.refcuda_destroy(self.h)
            self.h = None
