"""The reference's own CPU stepping paths, timed on this machine's host cores.

The reference package runs unmodified from its copy in baseline/_ref
(installed by baseline.install_ref): ``photonfdtd.Simulation(...).run()``
steps the scene with the reference's vectorised NumPy loop
(src/photonfdtd/simulation.py:1319-1410), or with its Numba kernel
(``use_numba=True``, :70-205, parallel over x on every core) where the
reference allows that (no dispersion, no subpixel smoothing).

Per-step time comes from the reference's own progress hook: with fewer than
100 steps, ``progress_callback(step, n)`` is called at the top of every step
and once after the last (:1319-1321, :1412-1413), so consecutive calls bracket
one step each and the scene setup inside ``run()`` (coefficient arrays, ADE
index lists, CPML slabs) is outside the timed steps. The first step is a
warm-up (first-touch allocation; the Numba kernel compiles there).

The workload is the benchmark's config 3 (384^3, Drude / two-pole Lorentz /
eps 2.1 blocks, six flux planes, an Ex/Ey DFT), built by
photonfdtd_b200.workloads.config3 against the reference's own classes. Its
110,592 media blocks are given as one structure per medium
(workloads.BlockMedium): the same cells and media, without 110,592 passes of
the reference's full-grid rasteriser in the setup.
"""
from __future__ import annotations

import os
import time

import numpy as np

from baseline.locate import import_reference


def _ref():
    ref = import_reference()
    if ref is None:
        raise RuntimeError("the reference package is not installed in baseline/_ref "
                           "(python -m baseline.install_ref)")
    return ref


def _timed_run(sim, warm: int) -> dict:
    stamps = []
    sim.progress_callback = lambda s, n: stamps.append((s, time.perf_counter()))
    t0 = time.perf_counter()
    sim.run()
    wall = time.perf_counter() - t0
    t = dict(stamps)
    n = sim.n_steps
    per = [t[s + 1] - t[s] for s in range(warm, n)]
    return dict(step_s=per, setup_s=t[0] - t0, wall_s=wall, n_steps=n)


def numpy_config3(size: int = 384, steps: int = 3, warm: int = 1) -> dict:
    """The reference NumPy path on `steps` timed steps of config 3."""
    from photonfdtd_b200 import workloads as W
    ref = _ref()
    sim = W.config3(ref, n_total=size, n_steps=warm + steps, union_blocks=True,
                    backend="numpy")
    r = _timed_run(sim, warm)
    cells = size ** 3
    mean = float(np.mean(r["step_s"]))
    return dict(value=cells / mean / 1e6, unit="Mcell-updates/s", cores=1, kind="reference",
                sample=(f"reference photonfdtd {ref.__version__} Simulation.run() NumPy path, "
                        f"config 3 at {size}^3 (ADE, 6 flux planes, DFT), {steps} steps timed "
                        f"after {warm} warm-up step by its progress hook: "
                        f"{mean:.2f} s/step; setup {r['setup_s']:.1f} s not timed"),
                s_per_step=mean)


def numba_config3_plain(size: int = 384, steps: int = 3, warm: int = 1) -> dict:
    """The reference Numba path (every core) on the non-dispersive variant of
    config 3 (eps 1.0 / 4.0 / 2.1 blocks; the Numba kernel rejects ADE)."""
    from photonfdtd_b200 import workloads as W
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(
        os.path.dirname(os.path.abspath(__file__)), "_ref", "numba_cache"))
    ref = _ref()
    try:
        import numba
        threads = int(numba.get_num_threads())
    except ImportError:
        return {"unavailable": "numba is not installed"}
    sim = W.config3(ref, n_total=size, n_steps=warm + steps, union_blocks=True,
                    dispersive=False, use_numba=True)
    if not sim.use_numba:
        return {"unavailable": "the reference did not enable its Numba path"}
    r = _timed_run(sim, warm)
    cells = size ** 3
    mean = float(np.mean(r["step_s"]))
    return dict(value=cells / mean / 1e6, unit="Mcell-updates/s", cores=threads,
                kind="reference",
                sample=(f"reference Simulation(use_numba=True).run(), non-dispersive config-3 "
                        f"variant at {size}^3 (eps 1.0/4.0/2.1 blocks, same monitors), {steps} "
                        f"steps after {warm} warm-up (JIT) step, {threads} threads: "
                        f"{mean:.3f} s/step"),
                s_per_step=mean)
