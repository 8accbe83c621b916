"""Error statement of a float32 result against a float64 run of its scene.

A float32 run on the engine reproduces the reference's float32 NumPy run bit
for bit; its distance from the exact solution is therefore the reference's
own float32 round-off, which this module measures against a float64 run of
the same scene. The float64 run is the engine's float64 path (the same
tables evaluated in float64, ``build_tables(sim, np.float64)``), which
reproduces the reference's float64 NumPy run to 1e-12 of the largest value
(tests/test_parity_gpu.py), so the numbers are the error against the
reference's float64 oracle, obtained on the GPU at full size.

    error_vs_f64(result32, float64_shadow(sim)) -> {key: {"rel_max", "rel_l2"}}

Keys follow the Result layout: "fields/<monitor>/<comp>", "dft/<monitor>/
<comp>", "flux/<monitor>". rel_max = max |a - b| / max |b| (the reference's
float32 bar, tests/test_rust.py:119-135, is 1e-5 on this measure); rel_l2 =
||a - b|| / ||b||.
"""
from __future__ import annotations

from typing import Dict

import numpy as np

from . import _native as N


def float64_shadow(sim, kernel: int = N.PF_KERNEL_AUTO):
    """The scene run on the engine in float64; a Result whose FieldMonitor
    frames are kept in float64."""
    from .engine import B200Engine, build_tables, drive, validate
    validate(sim)
    t = build_tables(sim, np.float64)
    eng = B200Engine(t, kernel=kernel)
    try:
        return drive(sim, eng, t, mon_dtype=np.float64)
    finally:
        eng.close()


def _pair(a, b) -> Dict[str, float]:
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    d = a - b
    mx = float(np.abs(b).max()) if b.size else 0.0
    l2 = float(np.linalg.norm(b))
    return {"rel_max": float(np.abs(d).max() / mx) if mx > 0 else float(np.abs(d).max(initial=0.0)),
            "rel_l2": float(np.linalg.norm(d) / l2) if l2 > 0 else float(np.linalg.norm(d))}


def error_vs_f64(res, ref64) -> Dict[str, Dict[str, float]]:
    """Per-output error of `res` against the float64 Result `ref64`."""
    out: Dict[str, Dict[str, float]] = {}
    for mon, comps in ref64.fields.items():
        for c, b in comps.items():
            out[f"fields/{mon}/{c}"] = _pair(res.fields[mon][c], b)
    for mon, comps in ref64.dft.items():
        for c, b in comps.items():
            out[f"dft/{mon}/{c}"] = _pair(res.dft[mon][c], b)
    for mon, b in ref64.flux.items():
        out[f"flux/{mon}"] = _pair([res.flux[mon]], [b])
    return out


def worst(errors: Dict[str, Dict[str, float]]) -> Dict[str, float]:
    """The largest rel_max and rel_l2 over the field and DFT outputs."""
    keys = [k for k in errors if not k.startswith("flux/")] or list(errors)
    return {"rel_max": max((errors[k]["rel_max"] for k in keys), default=0.0),
            "rel_l2": max((errors[k]["rel_l2"] for k in keys), default=0.0)}
