"""The 3D engine's adjoint (photonfdtd_b200.adjoint.value_and_grad_eps, the
counterpart of jaxbackend.py:666-722) against central finite differences of
the forward engine in float64: a 3D scene with CPML on every face, a
dielectric cube, an Ey dipole, a DFT plane (E and H components) and a
downsampled FieldMonitor frame, J mixing |DFT|^2, a cross term and frame
terms; the same scene with flux planes across x and y in J (linear and
squared flux); and a 2D TM scene (z collapsed). Every term of J is scaled by its
value on the unperturbed scene so that each one counts. Each checked cell's
gradient must agree with (J(eps + h) - J(eps - h)) / 2h to 1e-6 of the
largest gradient magnitude; the whole gradient must match the oracle's
transposed step (oracle/adjoint3d.py) to 1e-10. The float32 gradient is
compared with the float64 one, and the checkpoint spacing must not change
the result."""
import numpy as np
import pytest
import torch

import photonfdtd_b200 as pf
from photonfdtd_b200.adjoint import _out_dict, value_and_grad_eps
from photonfdtd_b200.engine import run_b200

pytestmark = pytest.mark.gpu

C_0 = 299_792_458.0
F0 = C_0 / 1.0e-6


def scene3d(precision="float64", eps=None):
    grid = pf.Grid(size=(1.6e-6, 1.36e-6, 1.2e-6), cell_size=80e-9, pml_layers=(5, 5, 4))
    box = pf.Box(center=(0.16e-6, 0.0, 0.0), size=(0.48e-6, 0.4e-6, 0.4e-6),
                 medium=pf.Medium.from_index(1.5))
    src = pf.PointDipole(position=(-0.4e-6, 0.08e-6, 0.0), component="Ey",
                         waveform=pf.GaussianPulse(freq0=F0, fwhm=4e-15))
    mons = [pf.DFTMonitor(name="d", components=("Ey", "Ez", "Hx"), freqs=[F0, 1.2 * F0],
                          plane_axis="x", plane_position=0.48e-6),
            pf.FieldMonitor(name="f", components=("Ex", "Hz"), times=[12e-15], downsample=2)]
    sim = pf.Simulation(grid, structures=[box], sources=[src], monitors=mons, run_time=20e-15,
                        precision=precision)
    if eps is not None:
        sim.eps_r = eps
    return sim


def scene2d(precision="float64", eps=None):
    grid = pf.Grid(size=(2.0e-6, 1.6e-6), cell_size=50e-9, pml_layers=(8, 8, 0))
    box = pf.Box(center=(0.2e-6, 0.0), size=(0.5e-6, 0.5e-6), medium=pf.Medium.from_index(2.0))
    src = pf.PointDipole(position=(-0.5e-6, 0.1e-6, 0.0), component="Ez",
                         waveform=pf.GaussianPulse(freq0=F0, fwhm=5e-15))
    mons = [pf.DFTMonitor(name="d", components=("Ez", "Hy"), freqs=[F0],
                          plane_axis="x", plane_position=0.6e-6)]
    sim = pf.Simulation(grid, structures=[box], sources=[src], monitors=mons, run_time=25e-15,
                        precision=precision)
    if eps is not None:
        sim.eps_r = eps
    return sim


TERMS3D = [lambda o: (o["dft"]["d"]["Ey"].abs() ** 2).sum(),
           lambda o: (o["dft"]["d"]["Ez"].abs() ** 2).sum(),
           lambda o: (o["dft"]["d"]["Hx"].real * o["dft"]["d"]["Ey"].imag).sum(),
           lambda o: (o["fields"]["f"]["Ex"] ** 2).sum(),
           lambda o: o["fields"]["f"]["Hz"].sum()]
def scene3d_flux(precision="float64", eps=None):
    """scene3d with flux planes across x and y in the loss."""
    sim = scene3d(precision, eps)
    sim.add_monitor(pf.FluxMonitor(name="fx", plane_axis="x", plane_position=0.4e-6))
    sim.add_monitor(pf.FluxMonitor(name="fy", plane_axis="y", plane_position=-0.16e-6))
    return sim


TERMS3D_FLUX = [lambda o: (o["dft"]["d"]["Ey"].abs() ** 2).sum(),
                lambda o: o["flux"]["fx"],
                lambda o: o["flux"]["fy"] ** 2]
TERMS2D = [lambda o: (o["dft"]["d"]["Ez"].abs() ** 2).sum(),
           lambda o: (o["dft"]["d"]["Hy"].real * o["dft"]["d"]["Ez"].imag).sum()]


def forward_out(build, eps=None, precision="float64"):
    return _out_dict(run_b200(build(precision=precision, eps=eps)), torch)


def scaled_loss(build, terms):
    """J = sum_k term_k / |term_k(unperturbed)|, the scales fixed numbers."""
    base = forward_out(build)
    scales = [1.0 / abs(float(t(base).detach())) for t in terms]
    return lambda out: sum(s * t(out) for s, t in zip(scales, terms))


def check_fd(build, terms, n_cells, seed):
    loss = scaled_loss(build, terms)
    sim = build()
    eps0 = np.array(sim.eps_r, dtype=np.float64)
    val, g = value_and_grad_eps(sim, loss)
    assert np.isfinite(g).all()
    assert val == pytest.approx(float(loss(forward_out(build, eps0)).detach()), rel=1e-12)
    gmax = np.abs(g).max()
    assert gmax > 0
    # the cells of largest gradient and a random sample of the rest
    flat = np.abs(g).ravel()
    top = np.argsort(flat)[-(n_cells // 2):]
    rng = np.random.default_rng(seed)
    pool = np.setdiff1d(np.flatnonzero(flat > 1e-3 * gmax), top)
    rest = rng.choice(pool, n_cells - top.size, replace=False)
    h = 1e-5
    worst = 0.0
    for c in np.concatenate([top, rest]):
        idx = np.unravel_index(c, eps0.shape)
        j = []
        for sgn in (1.0, -1.0):
            e = eps0.copy()
            e[idx] += sgn * h
            j.append(float(loss(forward_out(build, e)).detach()))
        fd = (j[0] - j[1]) / (2 * h)
        worst = max(worst, abs(fd - g[idx]) / gmax)
    assert worst <= 1e-6, worst


def test_adjoint3d_matches_central_differences():
    check_fd(scene3d, TERMS3D, 12, 3)


def test_adjoint2d_tm_matches_central_differences():
    check_fd(scene2d, TERMS2D, 10, 4)


def test_flux_loss_matches_central_differences():
    check_fd(scene3d_flux, TERMS3D_FLUX, 10, 6)


def test_checkpoint_spacing_does_not_change_the_gradient():
    loss = scaled_loss(scene3d, TERMS3D)
    _, g1 = value_and_grad_eps(scene3d(), loss)
    _, g2 = value_and_grad_eps(scene3d(), loss, checkpoint_every=7)
    _, g3 = value_and_grad_eps(scene3d(), loss, checkpoint_every=10_000)
    np.testing.assert_array_equal(g1, g2)
    np.testing.assert_array_equal(g1, g3)


def test_float32_gradient_tracks_float64():
    loss = scaled_loss(scene3d, TERMS3D)
    _, g64 = value_and_grad_eps(scene3d("float64"), loss)
    _, g32 = value_and_grad_eps(scene3d("float32"), loss)
    assert g32.dtype == np.float32
    err = np.linalg.norm(g32.astype(np.float64) - g64) / np.linalg.norm(g64)
    assert err <= 1e-3, err


def test_unsupported_cases_raise():
    loss = lambda o: (o["dft"]["d"]["Ey"].abs() ** 2).sum()  # noqa: E731
    sim = scene3d()
    sim.subpixel = True
    with pytest.raises(NotImplementedError):
        value_and_grad_eps(sim, loss)


@pytest.mark.parametrize("build,terms", [(scene3d, TERMS3D), (scene2d, TERMS2D),
                                         (scene3d_flux, TERMS3D_FLUX)])
def test_engine_adjoint_matches_oracle_adjoint(build, terms):
    """The engine's per-cell adjoint kernels against the oracle's transposed
    slab step (oracle/adjoint3d.py), both float64: the values agree to the
    last bits (the forward runs are bit-identical) and the gradients to
    1e-10 relative L2 (the two transposes associate their sums differently)."""
    from oracle.adjoint3d import value_and_grad_eps as oracle_value_and_grad
    loss = scaled_loss(build, terms)
    v, g = value_and_grad_eps(build(), loss)
    vo, go = oracle_value_and_grad(build(), loss)
    assert v == pytest.approx(vo, rel=1e-12)
    err = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert err <= 1e-10, err
