"""The fused single-pass 3D kernel against the split H/E passes.

Both paths share the per-cell arithmetic (csrc/cell_update.cuh); the fused
kernel recomputes H on tile halos and marches x-chunks with a recomputed
first plane. Every tiling (tile height 8 or 16, 1..7 x-chunks, domain sizes
that are not multiples of the tile) must give identical fields, DFT sums
and flux integrals.
"""
import os

import numpy as np
import pytest

import photonfdtd_b200 as pf
import scenes
from photonfdtd_b200 import _native as N
from photonfdtd_b200 import workloads as W
from photonfdtd_b200.engine import run_b200

pytestmark = pytest.mark.gpu
ALL6 = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def odd3d(pf, precision="float32", nz=45):
    """37 x 29 x nz cells: partial tiles on every axis, PML of different
    widths, a dispersive and a plain box, DFT, flux and end-state fields."""
    drude = pf.DispersiveMedium.drude(1.0, f_plasma_Hz=200e12, f_collision_Hz=8e12)
    grid = pf.Grid(size=(37 * 40e-9, 29 * 40e-9, nz * 40e-9), cell_size=40e-9,
                   pml_layers=(7, 5, 9))
    boxes = [pf.Box(center=(0.1e-6, -0.05e-6, 0.1e-6), size=(0.4e-6, 0.3e-6, 0.5e-6),
                    medium=drude),
             pf.Box(center=(-0.2e-6, 0.1e-6, -0.2e-6), size=(0.3e-6, 0.4e-6, 0.3e-6),
                    medium=pf.Medium(permittivity=4.0))]
    src = pf.PointDipole(position=(-0.3e-6, 0.0, 0.05e-6), component="Ez",
                         waveform=pf.GaussianPulse(freq0=250e12, fwhm=4e-15))
    mons = [pf.DFTMonitor(name="d", components=("Ex", "Hy", "Ez"), freqs=[230e12, 260e12],
                          plane_axis="y", plane_position=0.1e-6),
            pf.FluxMonitor(name="f", plane_axis="z", plane_position=0.5e-6)]
    sim = pf.Simulation(grid, structures=boxes, sources=[src], monitors=mons, run_time=12e-15,
                        precision=precision)
    sim.add_monitor(pf.FieldMonitor(name="end", components=ALL6,
                                    times=[(sim.n_steps - 1) * sim.dt]))
    return sim


CASES = {
    "odd3d_f32": lambda: odd3d(pf, "float32"),
    "odd3d_f64": lambda: odd3d(pf, "float64"),
    "odd3d_nz44_f32": lambda: odd3d(pf, "float32", nz=44),
    "odd3d_nz44_f64": lambda: odd3d(pf, "float64", nz=44),
    "cube3d_f32": lambda: scenes.build("cube3d_f32", pf),
    "sub3d_f32": lambda: scenes.build("sub3d_f32", pf),
    "ade3d_f32": lambda: scenes.ade3d(pf, "float32", n_steps=400),
}


def _run(make, kernel, ty=None, chunks=None, tma=True):
    env = {} if tma else {"PFB200_NO_TMA": "1"}
    if ty is not None:
        env["PFB200_FUSED_TY"] = str(ty)
    if chunks is not None:
        env["PFB200_XCHUNKS"] = str(chunks)
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return run_b200(make(), kernel=kernel)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _same(a, b, tag):
    for mon, comps in a.fields.items():
        for c, arr in comps.items():
            np.testing.assert_array_equal(b.fields[mon][c], arr, err_msg=f"{tag} {mon} {c}")
    for mon, comps in a.dft.items():
        for c, arr in comps.items():
            np.testing.assert_array_equal(b.dft[mon][c], arr, err_msg=f"{tag} dft {mon} {c}")
    for mon, v in a.flux.items():
        assert b.flux[mon] == v, (tag, mon)


@pytest.mark.parametrize("case", list(CASES))
def test_fused_equals_split(case):
    """Plain fused kernel (no TMA) over tile heights and chunkings."""
    make = CASES[case]
    ref = _run(make, N.PF_KERNEL_SPLIT)
    for ty, chunks in ((8, 1), (16, 3), (8, 7)):
        got = _run(make, N.PF_KERNEL_FUSED, ty, chunks, tma=False)
        _same(ref, got, f"{case} ty={ty} chunks={chunks}")


@pytest.mark.parametrize("case", ["odd3d_nz44_f32", "odd3d_nz44_f64", "sub3d_f32", "ade3d_f32"])
def test_tma_fused_equals_split(case):
    """TMA-staged fused kernel (z rows a multiple of 16 bytes) over chunkings."""
    from photonfdtd_b200.engine import B200Engine, build_tables
    make = CASES[case]
    t = build_tables(make())
    eng = B200Engine(t, kernel=N.PF_KERNEL_FUSED)
    info = eng.info()
    eng.close()
    assert info["tma"] == "1", info
    ref = _run(make, N.PF_KERNEL_SPLIT)
    for chunks in (1, 2, 5):
        got = _run(make, N.PF_KERNEL_FUSED, None, chunks, tma=True)
        _same(ref, got, f"{case} tma chunks={chunks}")


def test_fused_rejects_2d():
    sim = scenes.build("tm2d_f32", pf)
    with pytest.raises(NotImplementedError):
        run_b200(sim, kernel=N.PF_KERNEL_FUSED)
