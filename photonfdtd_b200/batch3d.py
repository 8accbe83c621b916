"""Many independent simulations on one GPU at once: uneven 1D / 2D / 3D
scenes, any mix, each on its own engine and CUDA stream, stepped
concurrently.

A small scene leaves most of a B200 idle (a 64^3 grid is 262k cells, a
fraction of one wave of the step kernels over 148 SMs), and a sequential loop
over many of them pays each one's host preparation, launch gaps and
read-backs in turn. Here every scene gets its own engine (own non-blocking
stream, own device state), and a pool of host threads takes the scenes
whole: each worker builds its scene's tables, creates the engine and drives
it (``engine.drive``: each thread's ``pf_advance`` waits only for its own
stream; NumPy and the C calls release the GIL), so one scene's host
preparation overlaps the others' stepping and their kernels overlap on the
GPU. Results are bit-identical to running each scene alone (the kernels are
deterministic and share nothing). PFB200_RUN_MANY_SERIAL_PREP=1 prepares
every scene first, one after another, and only drives them concurrently.

This complements the pooled 2D TE batch (``photonfdtd_b200.batch``), which
steps hundreds of 2D instances in one launch per step but only for its one
scene family.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from typing import List, Optional, Sequence

from . import _native as N
from .engine import B200Engine, build_tables, drive, validate


def run_many(sims: Sequence, workers: Optional[int] = None,
             kernel: int = N.PF_KERNEL_AUTO) -> List:
    """Run every simulation and return their Results in order. ``workers``
    bounds the scenes in flight at once (default: all of them, at most 32);
    device memory must hold that many scenes' state together."""
    sims = list(sims)
    if not sims:
        return []
    for s in sims:
        validate(s)
    if not os.environ.get("PFB200_RUN_MANY_SERIAL_PREP"):
        return _run_pipelined(sims, workers, kernel)
    tables = [build_tables(s) for s in sims]
    engines: List[B200Engine] = []
    try:
        for t in tables:
            engines.append(B200Engine(t, kernel=kernel))
        n = len(sims)
        with ThreadPoolExecutor(max_workers=max(1, min(workers or n, 32, n))) as pool:
            return list(pool.map(lambda i: drive(sims[i], engines[i], tables[i]), range(n)))
    finally:
        for e in engines:
            e.close()


def _run_pipelined(sims, workers, kernel) -> List:
    """run_many with each scene's preparation (tables, engine) inside its
    worker too, so that one scene's host preparation overlaps the others'
    stepping; each engine is closed as soon as its Result is read."""
    def one(i):
        t = build_tables(sims[i])
        eng = B200Engine(t, kernel=kernel)
        try:
            return drive(sims[i], eng, t)
        finally:
            eng.close()
    n = len(sims)
    with ThreadPoolExecutor(max_workers=max(1, min(workers or n, 32, n))) as pool:
        return list(pool.map(one, range(n)))
