"""The plugin registers backend="b200" on the reference photonfdtd package.

Runs where the reference is importable (its copy installed in baseline/_ref,
or its source tree); the engine call itself is replaced by a recorder, so no
GPU is needed.
"""
import os
import sys

import pytest


def _reference():
    from baseline.locate import import_reference
    ref = import_reference()
    if ref is None:
        pytest.skip("reference package not importable here")
    return ref


def test_install_routes_b200_runs(monkeypatch):
    ref = _reference()
    from photonfdtd_b200 import engine, plugin
    plugin.install(ref)
    seen = {}

    def fake_run(sim):
        seen["sim"] = sim
        return "ran"

    monkeypatch.setattr(engine, "run_b200", fake_run)
    grid = ref.Grid(size=(2e-6, 2e-6), cell_size=50e-9, pml_layers=(8, 8, 0))
    src = ref.PointDipole(position=(0, 0), component="Ez",
                          waveform=ref.GaussianPulse(freq0=ref.C_0 / 1e-6, fwhm=5e-15))
    sim = ref.Simulation(grid, sources=[src], run_time=5e-15, backend="b200")
    assert sim.backend == "b200"
    assert sim.run() == "ran" and seen["sim"] is sim
    # other backends are untouched
    sim2 = ref.Simulation(grid, sources=[src], run_time=2e-15, backend="numpy")
    assert sim2.run().times.size == sim2.n_steps
    with pytest.raises(ValueError):
        ref.Simulation(grid, sources=[src], run_time=2e-15, backend="nope")


def test_engine_tables_of_reference_simulation_match_own():
    """build_tables gives the same engine inputs for the reference's
    Simulation and for this package's, on the same scene."""
    ref = _reference()
    import numpy as np
    import photonfdtd_b200 as pf
    import scenes
    from photonfdtd_b200.engine import build_tables
    for name in ("disp2d_f32", "xz2d_f64", "cube3d_f32"):
        a = build_tables(scenes.build(name, ref))
        b = build_tables(scenes.build(name, pf))
        assert a["ce_mode"] == b["ce_mode"]
        for k in ("word", "table"):
            if k in a:
                np.testing.assert_array_equal(a[k], b[k])
        for ax in range(3):
            for q in range(4):
                np.testing.assert_array_equal(a["cpml"][ax][q], b["cpml"][ax][q])
        for k in ("comp", "cell", "row", "amp", "wave"):
            np.testing.assert_array_equal(a["sources"][k], b["sources"][k])
