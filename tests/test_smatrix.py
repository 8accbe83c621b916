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


def test_unimodesource_expands_like_the_reference():
    """The one-way mode source's dipoles (positions, components, amplitudes)
    against the reference's UniModeSource.expand on the same solved mode
    (the reference's own solver, on the CPU) and grid."""
    from baseline.locate import import_reference
    ref = import_reference()
    if ref is None:
        pytest.skip("the reference package is not installed in baseline/_ref")
    import photonfdtd_b200 as pf
    core = ref.Box(center=(0, 0), size=(0.45e-6, 0.22e-6), medium=ref.Medium.from_index(3.48))
    mr = ref.ModeSolver(size=(1.2e-6, 0.8e-6), cell_size=(40e-9, 40e-9), structures=[core],
                        wavelength=1.55e-6, background_eps=1.44 ** 2, num_modes=1).solve()
    f0 = pf.C_0 / 1.55e-6
    kw = dict(center=(0.1e-6, 0, 0), size=(0, 1.2e-6, 0.8e-6), mode=mr, direction="-x",
              amplitude=0.7)
    mine = pf.UniModeSource(waveform=pf.GaussianPulse(freq0=f0, fwhm=10e-15), **kw).expand(
        pf.Grid(size=(1.0e-6, 1.2e-6, 0.8e-6), cell_size=40e-9, pml_layers=(4, 4, 4)))
    theirs = ref.UniModeSource(waveform=ref.GaussianPulse(freq0=f0, fwhm=10e-15), **kw).expand(
        ref.Grid(size=(1.0e-6, 1.2e-6, 0.8e-6), cell_size=40e-9, pml_layers=(4, 4, 4)))
    assert len(mine) == len(theirs) > 0
    for a, b in zip(mine, theirs):
        assert a.component == b.component
        assert np.allclose(a.position, b.position, rtol=0, atol=1e-18)
        assert a.amplitude == b.amplitude
