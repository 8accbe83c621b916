"""Gradients through per-component E coefficients (the reference's
value_and_grad_params, jaxbackend.py:725-775, and the EtchedCore density
stack, design.py:75-175), float64:

* the engine's per-component adjoint gradient dJ/dK_c equals the oracle's
  transposed step (oracle/adjoint3d.py) to 1e-10 relative L2 on an
  anisotropic coefficient set;
* adjoint.value_and_grad_params through a two-parameter torch map to the
  coefficients matches central differences to 1e-6;
* EtchedCore.eps_components equals the NumPy restatement of the reference's
  stack (oracle/design_ref.py) to 1e-12, and value_and_grad_density3d
  (filter and projection on the GPU kernels, the stack in torch, the engine's
  adjoint) matches central differences in single density pixels to 1e-6 of
  the largest gradient entry."""
import numpy as np
import pytest
import torch

import photonfdtd_b200 as pf
from photonfdtd_b200 import design
from photonfdtd_b200.adjoint import _adjoint, _out_dict, value_and_grad_params
from photonfdtd_b200.engine import B200Engine, build_tables, drive
from photonfdtd_b200.scene import EPS_0

pytestmark = pytest.mark.gpu

C_0 = 299_792_458.0
F0 = C_0 / 1.0e-6


def scene(n=(24, 24, 16), d=60e-9, pml=4):
    grid = pf.Grid(size=tuple(v * d for v in n), cell_size=d, pml_layers=(pml, pml, pml))
    src = pf.PointDipole(position=(-0.3e-6, 0.06e-6, 0.0), component="Ey",
                         waveform=pf.GaussianPulse(freq0=F0, fwhm=4e-15))
    mon = pf.DFTMonitor(name="d", components=("Ex", "Ey", "Hz"), freqs=[F0, 1.15 * F0],
                        plane_axis="x", plane_position=0.36e-6)
    return pf.Simulation(grid, sources=[src], monitors=[mon], run_time=14e-15,
                         precision="float64")


def loss(out):
    d = out["dft"]["d"]
    return (d["Ey"].abs() ** 2).sum() + 0.5 * (d["Ex"].abs() ** 2).sum() + \
        1e5 * (d["Hz"].real * d["Ey"].imag).sum()


def forward_value(sim, ce3):
    t = build_tables(sim, ce3=ce3)
    eng = B200Engine(t)
    try:
        res = drive(sim, eng, t)
    finally:
        eng.close()
    return float(loss(_out_dict(res, torch)).detach())


def test_per_component_gradient_matches_oracle():
    from oracle.adjoint3d import value_and_grad_ce3
    sim = scene()
    rng = np.random.default_rng(1)
    shape = tuple(sim.grid.shape)
    eps = [1.0 + 2.0 * rng.random(shape) * (c + 1) / 3 for c in range(3)]
    ce3 = [sim.dt / (EPS_0 * e) for e in eps]
    v, g = _adjoint(sim, build_tables(sim, ce3=ce3), loss, None)
    vo, go = value_and_grad_ce3(scene(), ce3, loss)
    assert v == pytest.approx(vo, rel=1e-12)
    for c in range(3):
        assert np.linalg.norm(g[c] - go[c]) <= 1e-10 * np.linalg.norm(go[c]), c


def test_value_and_grad_params_matches_central_differences():
    sim = scene()
    shape = tuple(sim.grid.shape)
    mask = np.zeros(shape)
    mask[8:16, 6:18, 4:12] = 1.0
    m = torch.tensor(mask)
    dt = sim.dt

    def ce_of(p):
        exx = 1.0 + (p[0] * 2.0) * m.to(p.device)
        eyy = 1.0 + (p[1] * 2.0) * m.to(p.device)
        ezz = 1.0 + (p[0] + p[1]) * m.to(p.device)
        return {"Ex": dt / (exx * EPS_0), "Ey": dt / (eyy * EPS_0), "Ez": dt / (ezz * EPS_0)}

    p0 = np.array([0.8, 1.3])
    val, g = value_and_grad_params(sim, ce_of, p0, loss)
    assert g.shape == (2,)
    for k in range(2):
        h = 1e-6
        j = []
        for sgn in (1.0, -1.0):
            p = p0.copy()
            p[k] += sgn * h
            ce = ce_of(torch.tensor(p))
            j.append(forward_value(scene(), [ce[c].numpy() for c in ("Ex", "Ey", "Ez")]))
        fd = (j[0] - j[1]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * abs(fd), (k, fd, g[k])
    assert val == pytest.approx(forward_value(scene(), [ce_of(torch.tensor(p0))[c].numpy()
                                                        for c in ("Ex", "Ey", "Ez")]), rel=1e-12)


STACK = dict(eps_solid=3.48 ** 2, eps_void=1.44 ** 2, eps_sub=1.44 ** 2, eps_clad=1.0,
             core_z=(-0.12e-6, 0.12e-6), filter_radius=150e-9, beta=4.0, eta=0.5)


def test_etched_core_eps_matches_the_restated_stack():
    from oracle.design_ref import etched_core_eps
    sim = scene()
    rho = np.random.default_rng(3).random(sim.grid.shape[:2])
    core = design.EtchedCore(**STACK)
    got = [c.detach().cpu().numpy() for c in core.eps_components(sim.grid, rho)]
    want = etched_core_eps(sim.grid, rho, **STACK)
    for a, b in zip(got, want):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_density_gradient_3d_matches_central_differences():
    sim = scene()
    rng = np.random.default_rng(4)
    rho0 = 0.3 + 0.4 * rng.random(sim.grid.shape[:2])
    core = design.EtchedCore(**STACK)
    val, g = design.value_and_grad_density3d(sim, core, rho0, loss)
    build = core.ce_builder(sim)

    def J(r):
        ce = build(torch.tensor(r))
        return forward_value(scene(), [ce[c].detach().cpu().numpy() for c in ("Ex", "Ey", "Ez")])

    assert val == pytest.approx(J(rho0), rel=1e-12)
    gmax = np.abs(g).max()
    assert gmax > 0
    for idx in [tuple(int(v) for v in np.unravel_index(np.argmax(np.abs(g)), g.shape)),
                (10, 12), (14, 9)]:
        h = 1e-5
        rp, rm = rho0.copy(), rho0.copy()
        rp[idx] += h
        rm[idx] -= h
        fd = (J(rp) - J(rm)) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * gmax, (idx, fd, g[idx])
