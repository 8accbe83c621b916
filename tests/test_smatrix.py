"""photonfdtd_b200.smatrix against the reference's smatrix functions
(src/photonfdtd/smatrix.py:41-118) on random port fields, NumPy and torch
inputs, and its error for a port monitor missing a component. CPU only."""
import importlib

import numpy as np
import pytest
import torch

from photonfdtd_b200 import smatrix


def _reference_smatrix():
    from baseline.locate import import_reference
    ref = import_reference()
    if ref is None:
        pytest.skip("the reference package is not installed in baseline/_ref")
    return importlib.import_module(ref.__name__ + ".smatrix")


def _fields(rng, shape):
    return {c: rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
            for c in smatrix.PORT_COMPONENTS}


def test_amplitudes_match_the_reference_numpy_and_torch():
    ref = _reference_smatrix()
    rng = np.random.default_rng(7)
    sim, mode = _fields(rng, (3, 1, 12, 9)), _fields(rng, (12, 9))
    want = ref.mode_amplitudes(sim, mode, 2.5e-15)
    got = smatrix.mode_amplitudes(sim, mode, 2.5e-15)
    for g, w in zip(got, want):
        assert np.abs(g - w).max() <= 1e-13 * np.abs(w).max()
    ts = {c: torch.tensor(v) for c, v in sim.items()}
    tm = {c: torch.tensor(v) for c, v in mode.items()}
    got_t = smatrix.mode_amplitudes(ts, tm, 2.5e-15)
    for g, w in zip(got_t, want):
        assert np.abs(g.numpy() - w).max() <= 1e-13 * np.abs(w).max()


def test_missing_port_component_is_an_error():
    class R:
        dft = {"p": {"Ey": np.zeros((1, 2)), "Ez": np.zeros((1, 2)), "Hy": np.zeros((1, 2))}}
    with pytest.raises(ValueError, match="Hz"):
        smatrix.port_fields(R(), "p")
