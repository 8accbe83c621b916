"""The oracle's gradient (oracle/adjoint3d.py, a restatement of what
jaxbackend.py:666-722's jax.grad computes) against central differences of
the oracle's own forward run, float64, on tiny scenes: a 3D grid with CPML
on every face (DFT plane with E and H components, a downsampled FieldMonitor
frame; the same with flux planes across x and z in the loss) and a 2D TM
grid. Pins the transposed step before the engine's adjoint
is compared with it on the GPU."""
import numpy as np
import pytest
import torch  # noqa: F401  (the loss is written with torch ops)

import photonfdtd_b200 as pf
from oracle.adjoint3d import forward_value, value_and_grad_eps

C_0 = 299_792_458.0
F0 = C_0 / 1.0e-6


def tiny3d(eps=None):
    grid = pf.Grid(size=(0.8e-6, 0.72e-6, 0.64e-6), cell_size=80e-9, pml_layers=(3, 2, 2))
    box = pf.Box(center=(0.08e-6, 0.0, 0.0), size=(0.24e-6, 0.24e-6, 0.24e-6),
                 medium=pf.Medium.from_index(1.6))
    src = pf.PointDipole(position=(-0.16e-6, 0.08e-6, 0.0), component="Ez",
                         waveform=pf.GaussianPulse(freq0=F0, fwhm=2e-15))
    mons = [pf.DFTMonitor(name="d", components=("Ez", "Hy"), freqs=[F0, 1.3 * F0],
                          plane_axis="x", plane_position=0.24e-6),
            pf.FieldMonitor(name="f", components=("Ey",), times=[4e-15], downsample=2)]
    sim = pf.Simulation(grid, structures=[box], sources=[src], monitors=mons, run_time=7e-15,
                        precision="float64")
    if eps is not None:
        sim.eps_r = eps
    return sim


def tiny2d(eps=None):
    grid = pf.Grid(size=(1.2e-6, 1.0e-6), cell_size=50e-9, pml_layers=(5, 4, 0))
    box = pf.Box(center=(0.1e-6, 0.0), size=(0.3e-6, 0.3e-6), medium=pf.Medium.from_index(2.0))
    src = pf.PointDipole(position=(-0.3e-6, 0.05e-6, 0.0), component="Ez",
                         waveform=pf.GaussianPulse(freq0=F0, fwhm=3e-15))
    mons = [pf.DFTMonitor(name="d", components=("Ez", "Hx"), freqs=[F0],
                          plane_axis="x", plane_position=0.35e-6)]
    sim = pf.Simulation(grid, structures=[box], sources=[src], monitors=mons, run_time=12e-15,
                        precision="float64")
    if eps is not None:
        sim.eps_r = eps
    return sim


def loss3d_terms():
    return [lambda o: (o["dft"]["d"]["Ez"].abs() ** 2).sum(),
            lambda o: (o["dft"]["d"]["Hy"].real * o["dft"]["d"]["Ez"].imag).sum(),
            lambda o: (o["fields"]["f"]["Ey"] ** 2).sum()]


def tiny3d_flux(eps=None):
    """tiny3d with flux planes across x and z."""
    sim = tiny3d(eps)
    sim.add_monitor(pf.FluxMonitor(name="fx", plane_axis="x", plane_position=0.24e-6))
    sim.add_monitor(pf.FluxMonitor(name="fz", plane_axis="z", plane_position=-0.08e-6))
    return sim


def loss3d_flux_terms():
    return [lambda o: (o["dft"]["d"]["Ez"].abs() ** 2).sum(),
            lambda o: o["flux"]["fx"],
            lambda o: o["flux"]["fz"] ** 2]


def loss2d_terms():
    return [lambda o: (o["dft"]["d"]["Ez"].abs() ** 2).sum(),
            lambda o: (o["dft"]["d"]["Hx"].abs() ** 2).sum()]


def scaled(build, terms):
    from oracle.adjoint3d import _out_dict
    from oracle.fdtd_oracle import OracleRun
    r = OracleRun(build())
    r.advance(r.n_steps)
    base = _out_dict(r.result(), torch)
    s = [1.0 / abs(float(t(base).detach())) for t in terms]
    return lambda o: sum(w * t(o) for w, t in zip(s, terms))


@pytest.mark.parametrize("build,terms,seed", [(tiny3d, loss3d_terms, 1), (tiny2d, loss2d_terms, 2),
                                               (tiny3d_flux, loss3d_flux_terms, 5)])
def test_oracle_gradient_matches_central_differences(build, terms, seed):
    loss = scaled(build, terms())
    sim = build()
    val, g = value_and_grad_eps(sim, loss)
    eps0 = np.array(sim.eps_r, dtype=np.float64)
    assert val == pytest.approx(forward_value(build(eps0), loss), rel=1e-13)
    gmax = np.abs(g).max()
    flat = np.abs(g).ravel()
    top = np.argsort(flat)[-4:]
    rng = np.random.default_rng(seed)
    rest = rng.choice(np.setdiff1d(np.flatnonzero(flat > 1e-3 * gmax), top), 4, replace=False)
    h = 1e-5
    for c in np.concatenate([top, rest]):
        idx = np.unravel_index(c, eps0.shape)
        j = []
        for sgn in (1.0, -1.0):
            e = eps0.copy()
            e[idx] += sgn * h
            j.append(forward_value(build(e), loss))
        fd = (j[0] - j[1]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * gmax, (idx, fd, g[idx], gmax)


@pytest.mark.parametrize("build,terms", [(tiny3d, loss3d_terms), (tiny3d_flux, loss3d_flux_terms)])
def test_oracle_per_component_gradient_matches_central_differences(build, terms):
    """dJ/dK_c for per-component E coefficients (the quantity
    value_and_grad_params chains to its parameters, jaxbackend.py:725-775):
    an anisotropic coefficient set on the tiny 3D scene (also with flux
    terms in the loss), against central differences in single coefficients
    of each component."""
    from oracle.adjoint3d import value_and_grad_ce3
    from oracle.fdtd_oracle import EPS0, OracleRun
    base = build()
    eps = np.array(base.eps_r, dtype=np.float64)
    rng = np.random.default_rng(9)
    dt = OracleRun(base).dt
    ce3 = [dt / (EPS0 * eps * (1.0 + 0.2 * c) * (1.0 + 0.05 * rng.random(eps.shape)))
           for c in range(3)]
    loss = scaled(build, terms())

    def value(c3):
        r = OracleRun(build(), ce3=c3)
        r.advance(r.n_steps)
        from oracle.adjoint3d import _out_dict
        return float(loss(_out_dict(r.result(), torch)).detach())

    val, g3 = value_and_grad_ce3(build(), ce3, loss)
    assert val == pytest.approx(value(ce3), rel=1e-13)
    gmax = np.abs(g3).max()
    for comp in range(3):
        flat = np.abs(g3[comp]).ravel()
        for c in np.argsort(flat)[-2:]:
            idx = np.unravel_index(c, eps.shape)
            h = 1e-6 * ce3[comp][idx]
            j = []
            for sgn in (1.0, -1.0):
                c3 = [a.copy() for a in ce3]
                c3[comp][idx] += sgn * h
                j.append(value(c3))
            fd = (j[0] - j[1]) / (2 * h)
            assert abs(fd - g3[comp][idx]) <= 1e-6 * gmax, (comp, idx, fd, g3[comp][idx])
