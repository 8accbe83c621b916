"""Port S-parameters (photonfdtd_b200.smatrix, the reference's
src/photonfdtd/smatrix.py interface) from the GPU mode solver and an engine
run: a silicon strip waveguide along x in oxide, an Ey dipole in the core, a
port DFT plane (Ey, Ez, Hy, Hz) downstream, the fundamental mode solved on
the same (y, z) cells. The amplitudes equal the reference's own smatrix
functions applied to the same arrays (1e-12), and |alpha+|^2 at the first
frequency, as a loss of the engine run's DFT outputs, is differentiated with
respect to eps_r by the engine's adjoint and by the oracle's transposed step
(oracle/adjoint3d.py): the two gradients agree to 1e-10 relative L2
(float64). Then the reference's own end-to-end checks on the engine: |S21|
of a ModeSource-launched waveguide mode within 0.05 of 1, and the backward
amplitude of a UniModeSource below 0.3 of the forward one."""
import numpy as np
import pytest
import torch

import photonfdtd_b200 as pf
from photonfdtd_b200 import smatrix
from photonfdtd_b200.adjoint import value_and_grad_eps
from photonfdtd_b200.engine import run_b200
from photonfdtd_b200.mode import ModeSolver

pytestmark = pytest.mark.gpu

C_0 = 299_792_458.0
LAM = 1.55e-6
D = 40e-9
SIZE = (1.6e-6, 1.2e-6, 1.0e-6)
CLAD, CORE = 1.444 ** 2, 3.48


def scene():
    grid = pf.Grid(size=SIZE, cell_size=D, pml_layers=(8, 8, 8))
    clad = pf.Box(center=(0.0, 0.0, 0.0), size=(4e-6, 4e-6, 4e-6),
                  medium=pf.Medium(permittivity=CLAD))
    core = pf.Box(center=(0.0, 0.0, 0.0), size=(4e-6, 0.44e-6, 0.24e-6),
                  medium=pf.Medium.from_index(CORE))
    f0 = C_0 / LAM
    src = pf.PointDipole(position=(-0.36e-6, 0.0, 0.0), component="Ey",
                         waveform=pf.GaussianPulse(freq0=f0, fwhm=4e-15))
    port = pf.DFTMonitor(name="port", components=("Ey", "Ez", "Hy", "Hz"),
                         freqs=[f0, 1.1 * f0], plane_axis="x", plane_position=0.36e-6)
    return pf.Simulation(grid, structures=[clad, core], sources=[src], monitors=[port],
                         run_time=24e-15, precision="float64")


def mode():
    core = pf.Box(center=(0.0, 0.0, 0.0), size=(4e-6, 0.44e-6, 0.24e-6),
                  medium=pf.Medium.from_index(CORE))
    return ModeSolver(size=SIZE[1:], cell_size=D, structures=[core], wavelength=LAM,
                      background_eps=CLAD, num_modes=1, polarization="te").solve()


def _reference():
    from baseline.locate import import_reference
    ref = import_reference()
    if ref is None:
        pytest.skip("the reference package is not installed in baseline/_ref")
    return ref


def test_amplitudes_equal_the_reference_functions():
    ref = _reference()
    import importlib
    ref_sm = importlib.import_module(ref.__name__ + ".smatrix")
    m = mode()
    assert m.n_eff[0] > 1.444
    res = run_b200(scene())
    a_ours = smatrix.s_parameters(res, "port", m, 0, dA=D * D)
    a_ref = ref_sm.s_parameters(res, "port", m, 0, dA=D * D)
    for x, y in zip(a_ours, a_ref):
        assert np.abs(np.asarray(x) - y).max() <= 1e-12 * np.abs(y).max()
    assert np.abs(a_ours[0]).max() > 0
    # the same on CUDA tensors
    port = {c: torch.as_tensor(v, device="cuda") for c, v in smatrix.port_fields(res, "port").items()}
    t = smatrix.mode_amplitudes(port, smatrix.mode_port_fields(m, 0, like=port["Ey"]), D * D)
    assert t[0].is_cuda
    assert np.abs(t[0].cpu().numpy() - a_ref[0]).max() <= 1e-12 * np.abs(a_ref[0]).max()


def test_s_parameter_gradient_engine_against_oracle():
    from oracle.adjoint3d import value_and_grad_eps as oracle_value_and_grad
    m = mode()

    def loss(out):
        port = smatrix.port_fields(out, "port")
        ap, _ = smatrix.mode_amplitudes(port, smatrix.mode_port_fields(m, 0, like=port["Ey"]),
                                        D * D)
        return ap[0].abs() ** 2

    v, g = value_and_grad_eps(scene(), loss)
    vo, go = oracle_value_and_grad(scene(), loss)
    assert v == pytest.approx(vo, rel=1e-12)
    assert np.abs(g).max() > 0
    assert np.linalg.norm(g - go) <= 1e-10 * np.linalg.norm(go)


# The reference's end-to-end S-parameter checks (tests/test_smatrix.py:88-152,
# run there on its JAX backend), here on the engine with the GPU mode solver:
# a silicon strip waveguide (0.45 x 0.22 um, n = 3.48) in a 2 x 1.4 um
# cross-section at 40 nm, the mode solved with a 1.44^2 background.
def _wg_mode():
    core = pf.Box(center=(0, 0), size=(0.45e-6, 0.22e-6), medium=pf.Medium.from_index(3.48))
    ms = ModeSolver(size=(2.0e-6, 1.4e-6), cell_size=(40e-9, 40e-9), structures=[core],
                    wavelength=1.55e-6, background_eps=1.44 ** 2, num_modes=2)
    return ms, ms.solve()


def test_waveguide_s21_energy_conserving():
    """A mode launched down a straight lossless waveguide keeps |S21| ~= 1
    between two downstream ports (the reference's bound: within 0.05)."""
    f0 = C_0 / 1.55e-6
    ms, mr = _wg_mode()
    core = pf.Box(center=(0, 0, 0), size=(10e-6, 0.45e-6, 0.22e-6),
                  medium=pf.Medium.from_index(3.48))
    grid = pf.Grid(size=(6e-6, 2.0e-6, 1.4e-6), cell_size=40e-9, pml_layers=(10, 10, 10))
    src = pf.ModeSource(center=(-2e-6, 0, 0), size=(0, 2.0e-6, 1.4e-6), component="Ey",
                        waveform=pf.GaussianPulse(freq0=f0, fwhm=10e-15),
                        profile=np.real(mr.Ey[0]), profile_coords=(ms.y, ms.z))
    ports = [pf.DFTMonitor(name=n, components=("Ey", "Ez", "Hy", "Hz"), freqs=[f0],
                           plane_axis="x", plane_position=x) for n, x in (("p1", 0.0),
                                                                          ("p2", 2.0e-6))]
    res = run_b200(pf.Simulation(grid, structures=[core], sources=[src], monitors=ports,
                                 run_time=200e-15))
    dA = 40e-9 * 40e-9
    a1, _ = pf.s_parameters(res, "p1", mr, 0, dA)
    a2, _ = pf.s_parameters(res, "p2", mr, 0, dA)
    assert abs(a2[0] / a1[0]) == pytest.approx(1.0, abs=0.05)


def test_unidirectional_source_extinction():
    """UniModeSource launches one way: the backward amplitude upstream is
    below 0.3 of the forward one downstream (the reference's bound)."""
    f0 = C_0 / 1.55e-6
    _, mr = _wg_mode()
    core = pf.Box(center=(0, 0, 0), size=(12e-6, 0.45e-6, 0.22e-6),
                  medium=pf.Medium.from_index(3.48))
    grid = pf.Grid(size=(8e-6, 2.0e-6, 1.4e-6), cell_size=40e-9, pml_layers=(10, 10, 10))
    src = pf.UniModeSource(center=(0, 0, 0), size=(0, 2.0e-6, 1.4e-6),
                           waveform=pf.GaussianPulse(freq0=f0, fwhm=10e-15), mode=mr,
                           direction="+x")
    ports = [pf.DFTMonitor(name=n, components=("Ey", "Ez", "Hy", "Hz"), freqs=[f0],
                           plane_axis="x", plane_position=x) for n, x in (("up", -1.5e-6),
                                                                          ("dn", 1.5e-6))]
    res = run_b200(pf.Simulation(grid, structures=[core], sources=[src], monitors=ports,
                                 run_time=220e-15))
    dA = 40e-9 * 40e-9
    fwd, _ = pf.s_parameters(res, "dn", mr, 0, dA)
    _, back = pf.s_parameters(res, "up", mr, 0, dA)
    assert abs(fwd[0]) > 0
    assert abs(back[0]) / abs(fwd[0]) < 0.3
