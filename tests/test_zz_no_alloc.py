"""Allocation-free flux entry point against the engine's flux monitor.

Some callers of this library cannot allocate device memory where they call
it: their device memory belongs to another allocator, they only borrow the
field buffers, or they run a time loop that must not pay for cudaMalloc.
pf_flux_plane_noalloc serves them: it computes one step's flux contribution
from caller-owned field buffers into a caller-owned device double, keeping
its partial sums in a fixed device array instead of allocating scratch.

Here the engine steps a small 3D scene with three flux monitors, one normal
to each axis, so every plane-indexing branch of the entry point runs. On each
of two consecutive steps the fields are copied into separate device buffers
and the entry point is called once per monitor on them, so it is called
twice in a row per monitor. Added onto the engine's integral from before
those steps, in the order the engine adds its own per-step terms, the
contributions must equal the engine's integral after them exactly: the
partial sums use the same block layout, roundings and fold order as the
engine's flux sampling, so no tolerance is needed. The file is named to run
after every other GPU test and depends on no state they leave.
"""
import ctypes as C

import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200 import _native as N
from photonfdtd_b200.engine import B200Engine, build_tables

pytestmark = pytest.mark.gpu

ALL6 = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _scene(precision):
    grid = pf.Grid(size=(40 * 40e-9, 36 * 40e-9, 32 * 40e-9), cell_size=40e-9, pml_layers=6)
    box = pf.Box(center=(0.2e-6, 0.0, 0.0), size=(0.3e-6, 0.4e-6, 0.3e-6),
                 medium=pf.Medium(permittivity=3.0))
    src = pf.PointDipole(position=(0.0, 0.0, 0.0), component="Ez",
                         waveform=pf.GaussianPulse(freq0=250e12, fwhm=4e-15))
    mons = [pf.FluxMonitor(name="fx", plane_axis="x", plane_position=0.0),
            pf.FluxMonitor(name="fy", plane_axis="y", plane_position=-0.08e-6),
            pf.FluxMonitor(name="fz", plane_axis="z", plane_position=0.1e-6)]
    return pf.Simulation(grid, structures=[box], sources=[src], monitors=mons,
                         run_time=60e-15, precision=precision)


@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_noalloc_flux_matches_engine(precision):
    import torch
    lib = N.lib()
    t = build_tables(_scene(precision))
    nx, ny, nz = t["shape"]
    itemsize = np.dtype(t["npdt"]).itemsize
    eng = B200Engine(t)
    try:
        warm = 25
        eng.advance(0, warm)
        acc = [eng.read_flux(k) for k in range(len(t["flux"]))]
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        for call in range(2):
            eng.advance(warm + call, 1)
            fields = [torch.from_numpy(np.ascontiguousarray(eng.get(c))).cuda() for c in ALL6]
            ptrs = (C.c_void_p * 6)(*[f.data_ptr() for f in fields])
            for k, f in enumerate(t["flux"]):
                rc = lib.pf_flux_plane_noalloc(itemsize, nx, ny, nz, ptrs, f["axis"], f["idx"],
                                               f["dA"], t["dt"], C.c_void_p(out.data_ptr()),
                                               None)
                assert rc == N.PF_OK, lib.pf_noalloc_last_error().decode()
                torch.cuda.synchronize()
                acc[k] = acc[k] + out.item()
        want = [eng.read_flux(k) for k in range(len(t["flux"]))]
    finally:
        eng.close()
    assert sorted(f["axis"] for f in t["flux"]) == [0, 1, 2]
    for got, ref in zip(acc, want):
        assert ref != 0.0
        assert got == ref, (got, ref)


def test_noalloc_rejects_oversized_plane():
    lib = N.lib()
    dummy = (C.c_void_p * 6)(*([16] * 6))
    rc = lib.pf_flux_plane_noalloc(4, 2, 4097, 4097, dummy, 0, 0, 1.0, 1.0, C.c_void_p(16), None)
    assert rc == N.PF_ERR_INVALID
    assert "16,777,216" in lib.pf_noalloc_last_error().decode()
