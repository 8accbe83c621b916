"""Concurrent independent scenes (photonfdtd_b200.batch3d.run_many): a mix
of 1D, 2D and 3D golden scenes in float32 and float64, with dispersion,
subpixel smoothing, DFT, flux and field monitors, stepped at once on their
own engines and streams. Every output equals the same scene run alone, bit
for bit (flux included: the same reductions in the same order)."""
import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200.batch3d import run_many
from photonfdtd_b200.engine import run_b200

import scenes

pytestmark = pytest.mark.gpu

NAMES = ["tm2d_f32", "cube3d_f64", "xz2d_f32", "line1d_f64", "disp2d_f32", "sub3d_f32",
         "cube3d_f32", "tm2d_f64"]


@pytest.mark.parametrize("pipelined", [False, True])
def test_concurrent_runs_equal_single_runs(pipelined, monkeypatch):
    """Both with the scenes' preparation in the workers (the default) and
    prepared one after another first (PFB200_RUN_MANY_SERIAL_PREP)."""
    if not pipelined:
        monkeypatch.setenv("PFB200_RUN_MANY_SERIAL_PREP", "1")
    together = run_many([scenes.build(n, pf) for n in NAMES], workers=4)
    for name, res in zip(NAMES, together):
        alone = run_b200(scenes.build(name, pf))
        for mon, comps in alone.fields.items():
            for c, arr in comps.items():
                np.testing.assert_array_equal(res.fields[mon][c], arr, err_msg=f"{name} {mon} {c}")
        for mon, comps in alone.dft.items():
            for c, arr in comps.items():
                np.testing.assert_array_equal(res.dft[mon][c], arr, err_msg=f"{name} {mon} {c}")
        for mon, v in alone.flux.items():
            assert res.flux[mon] == v, (name, mon)


def test_empty_batch():
    assert run_many([]) == []
