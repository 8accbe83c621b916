"""Write the golden fixtures: outputs of the reference photonfdtd itself.

Run where the reference package is importable: installed in baseline/_ref
(python -m baseline.install_ref) or found as a source tree by
baseline.locate (PHOTONFDTD_REFERENCE, or a ``reference`` directory beside
the repository). The reference is read, never modified:

    python tests/golden/make_golden.py [names...]

Each scene of ``tests/scenes.py`` is built against the reference package,
run with ``backend="numpy"`` (the reference's vectorised float32/float64
path, src/photonfdtd/simulation.py:910-1436), and its Result is stored as
``tests/golden/<scene>.npz``. ``tables.npz`` stores host-side tables (CPML
coefficients, subpixel tensors, step counts, source waveforms) computed by the
reference's own functions. The GPU box never runs this script; it only reads
the .npz files.

Large results are thinned to keep the fixtures small; ``_keep`` records what
was kept (frame indices) so the tests slice their own runs the same way.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

from baseline.locate import import_reference  # noqa: E402
import scenes  # noqa: E402

ref = import_reference()
if ref is None:
    raise SystemExit("the reference photonfdtd package is not importable here")

# Frames kept per FieldMonitor when a scene records many.
MAX_FRAMES = 6


def _thin(n):
    if n <= MAX_FRAMES:
        return np.arange(n)
    return np.unique(np.linspace(0, n - 1, MAX_FRAMES).round().astype(int))


def run_scene(name):
    sim = scenes.build(name, ref)
    sim.backend = "numpy"
    t0 = time.perf_counter()
    res = sim.run()
    wall = time.perf_counter() - t0
    out = {}
    keep = {}
    for mon, comps in res.fields.items():
        n = len(res.monitor_times[mon])
        k = _thin(n)
        keep[mon] = k.tolist()
        for c, arr in comps.items():
            out[f"f/{mon}/{c}"] = np.asarray(arr)[k]
        out[f"ft/{mon}"] = np.asarray(res.monitor_times[mon])
    thin = scenes.THIN_DFT.get(name)
    for mon, comps in res.dft.items():
        for c, arr in comps.items():
            if thin is not None:
                if c not in thin["comps"]:
                    continue
                arr = np.asarray(arr)[list(thin["freqs"])]
            out[f"dft/{mon}/{c}"] = np.asarray(arr)
        out[f"dftf/{mon}"] = np.asarray(res.dft_freqs[mon])
    for mon, v in res.flux.items():
        out[f"flux/{mon}"] = np.float64(v)
    meta = dict(scene=name, dt=sim.dt, n_steps=sim.n_steps, wall_s=wall,
                keep=keep, thin_dft=thin, numpy=np.__version__, reference=ref.__version__,
                shape=list(sim.grid.shape))
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: {sim.grid.shape} x {sim.n_steps} steps, {wall:.1f} s", flush=True)


def make_tables():
    """Reference host tables: CPML, subpixel smoothing, dt/n_steps, waveforms."""
    from photonfdtd.boundaries import cpml_coeffs_1axis, CPMLParams
    from photonfdtd.smoothing import smooth_permittivity
    from photonfdtd_b200 import workloads as W
    out = {}
    cases = [(104, 50e-9, 12, 9.5e-17), (384, 10e-9, 12, 1.9e-17),
             (536, 20e-9, 12, 3.8e-17), (20, 40e-9, 12, 7.6e-17),
             (30, 1.0, 0, 1e-17), (64, 25e-9, 7, 4.1e-17)]
    for ci, (n, dl, npml, dt) in enumerate(cases):
        for nm, arr in zip(("be", "ce", "bh", "ch"), cpml_coeffs_1axis(n, dl, npml, dt)):
            out[f"cpml/{ci}/{nm}"] = arr
    out["cpml_cases"] = np.array(cases)
    # a custom CPML parameter set
    p = CPMLParams(poly_order=4, sigma_factor=1.1, alpha_max=0.1, R_target=1e-6)
    for nm, arr in zip(("be", "ce", "bh", "ch"), cpml_coeffs_1axis(50, 30e-9, 9, 5e-17, p)):
        out[f"cpml/custom/{nm}"] = arr
    # subpixel smoothing on small scenes (3D and 2D), factor 3 and 2
    g3 = ref.Grid(size=(0.8e-6, 0.72e-6, 0.64e-6), cell_size=40e-9, pml_layers=0)
    boxes3 = [ref.Box(center=(0.05e-6, -0.03e-6, 0.0), size=(0.37e-6, 0.29e-6, 0.41e-6),
                      medium=ref.Medium(permittivity=7.0)),
              ref.Box(center=(-0.2e-6, 0.1e-6, 0.07e-6), size=(0.21e-6, 0.33e-6, 0.19e-6),
                      medium=ref.Medium(permittivity=2.2))]
    for f in (3, 2):
        exx, eyy, ezz = smooth_permittivity(g3, boxes3, factor=f)
        out[f"smooth3d/{f}"] = np.stack([exx, eyy, ezz])
    g2 = ref.Grid(size=(1.0e-6, 0.8e-6), cell_size=50e-9, pml_layers=(0, 0, 0))
    boxes2 = [ref.Box(center=(0.13e-6, 0.07e-6), size=(0.43e-6, 0.31e-6),
                      medium=ref.Medium(permittivity=11.0))]
    exx, eyy, ezz = smooth_permittivity(g2, boxes2, factor=3, dtype=np.float32)
    out["smooth2d/3"] = np.stack([exx, eyy, ezz])
    # dt and n_steps of the named workloads, plus monitor plane indices at full size
    for nm, sim in (("config1", W.config1(ref)),):
        out[f"dt/{nm}"] = np.array([sim.dt, sim.n_steps])
    for n, d, nd in ((536, 20e-9, 3), (384, 10e-9, 3)):
        g = ref.Grid(size=(n * d,) * 3, cell_size=d, pml_layers=12)
        idx = [g.index_at((p, p, p)) for p in (-1.6e-6, 1.6e-6, 0.0)]
        out[f"index_at/{n}"] = np.array(idx)
    # waveform samples
    w = ref.GaussianPulse(freq0=ref.C_0 / 1.55e-6, fwhm=15e-15, delay=1e-15)
    t = np.arange(500) * 3.8e-17
    out["wave/t"] = t
    out["wave/v"] = w(t)
    out["wave/v1"] = np.array([w(np.array([tt]))[0] for tt in t])
    # mode source expansion (line profile) on a 2D grid
    g = ref.Grid(size=(2e-6, 1.6e-6), cell_size=40e-9, pml_layers=(8, 8, 0))
    yy = np.linspace(-0.5e-6, 0.5e-6, 41)
    prof = np.exp(-(yy / 0.25e-6) ** 2)
    ms = ref.ModeSource(center=(-0.6e-6, 0.02e-6, 0.0), size=(0.0, 0.8e-6, 0.0),
                        component="Ez", waveform=w, profile=prof, profile_coords=(yy,),
                        amplitude=2.0)
    dips = ms.expand(g)
    out["mode/pos"] = np.array([d.position for d in dips])
    out["mode/amp"] = np.array([d.amplitude for d in dips])
    np.savez_compressed(os.path.join(HERE, "tables.npz"), **out)
    print("tables written", flush=True)


if __name__ == "__main__":
    names = sys.argv[1:] or (["tables"] + list(scenes.SCENES))
    for nm in names:
        if nm == "tables":
            make_tables()
        else:
            run_scene(nm)
