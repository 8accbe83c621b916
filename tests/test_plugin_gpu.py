"""Golden scenes run through the reference's own Simulation on the GPU.

The reference package (installed in baseline/_ref) builds each scene with its
own classes; photonfdtd_b200.plugin.install() lets its Simulation take
backend="b200", so run() steps the scene on this engine and returns the
reference's own Result type. Fields and DFT sums must equal the reference's
NumPy run (the fixtures) bit for bit; flux integrals to 1e-5 relative (the
plane sums are float64 here, pairwise float32 or float64 in NumPy).
"""
import numpy as np
import pytest

import scenes
from golden_util import load

pytestmark = pytest.mark.gpu

NAMES = ["tm2d_f32", "cube3d_f64", "xz2d_f32", "disp2d_f32", "sub3d_f32", "te2d_f32"]


def _reference():
    from baseline.locate import import_reference
    ref = import_reference()
    if ref is None:
        pytest.skip("the reference package is not installed in baseline/_ref")
    from photonfdtd_b200 import plugin
    plugin.install(ref)
    return ref


@pytest.mark.parametrize("name", NAMES)
def test_reference_simulation_runs_on_b200(name):
    ref = _reference()
    sim = scenes.build(name, ref)
    sim.backend = "b200"
    res = sim.run()
    assert type(res).__module__.startswith("photonfdtd.")
    g, meta = load(name)
    for k in g.files:
        if k.startswith("f/"):
            _, mon, c = k.split("/")
            np.testing.assert_array_equal(np.asarray(res.fields[mon][c])[meta["keep"][mon]],
                                          g[k], err_msg=f"{name} {k}")
        elif k.startswith("dft/"):
            _, mon, c = k.split("/")
            np.testing.assert_array_equal(res.dft[mon][c], g[k], err_msg=f"{name} {k}")
        elif k.startswith("flux/"):
            v, want = res.flux[k.split("/")[1]], float(g[k])
            assert abs(v - want) <= 1e-5 * max(abs(want), 1e-300), (name, k, v, want)
