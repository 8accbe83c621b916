"""The density chain on the GPU (csrc/design.cu) against the NumPy oracle of
the reference's conic_filter + tanh_projection (design.py:40-72), and the
whole chain rho -> filter -> projection -> eps -> batched FDTD -> loss
against central differences (the reference pins its JAX gradient the same
way, tests/test_jax.py:76-108)."""
import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200 import design as Dz
from photonfdtd_b200 import workloads as W
from photonfdtd_b200.batch import BatchTE
from oracle import design_ref as D
from oracle.adjoint2d import objective

pytestmark = pytest.mark.gpu

CASES = [(0.0, 0.0), (3.0, 0.0), (0.0, 8.0), (2.6, 6.0), (5.0, 16.0)]


@pytest.mark.parametrize("radius,beta", CASES)
def test_kernels_match_oracle(radius, beta):
    rng = np.random.default_rng(7)
    rho = rng.uniform(size=(5, 64, 64))
    g = rng.standard_normal((5, 64, 64))
    got = Dz.density_forward(rho, radius, beta, 0.45)
    gb = Dz.density_backward(rho, g, radius, beta, 0.45)
    for k in range(5):
        want = D.forward(rho[k], radius, beta, 0.45)
        assert np.max(np.abs(got[k] - want)) <= 1e-13 * max(1.0, np.max(np.abs(want)))
        wb = D.backward(rho[k], g[k], radius, beta, 0.45)
        assert np.max(np.abs(gb[k] - wb)) <= 1e-12 * np.max(np.abs(wb))


def test_rejects_windows_beyond_the_limit():
    with pytest.raises(ValueError):
        Dz.density_forward(np.zeros((97, 97)), 2.0)


def test_chain_gradient_matches_central_differences():
    """d J / d rho through filter (R = 2.5 cells), projection (beta 4, eta
    0.5), eps, a float64 batch of two instances and its adjoint, against
    (J(rho + h e) - J(rho - h e)) / 2h with h = 1e-4 on 8 pixels each."""
    sizes, d = [(80, 64), (96, 70)], 16
    rhos = [W.config4_density(k, d) for k in range(2)]
    sims = [W.config4_instance(pf, nx, ny, rho=r, n_steps=600, n_freqs=3,
                               precision="float64", design=d)
            for (nx, ny), r in zip(sizes, rhos)]
    wins = [W.design_window_box(nx, ny, d) for nx, ny in sizes]
    chain = Dz.DensityChain(radius_cells=2.5, beta=4.0, eta=0.5)
    b = BatchTE(sims, wins)
    try:
        rho = np.stack(rhos)
        vals, g = Dz.value_and_grad_density(b, rho, chain)
        assert vals.shape == (2,) and g.shape == rho.shape
        rng = np.random.default_rng(5)
        pix = [(int(rng.integers(0, d)), int(rng.integers(0, d))) for _ in range(8)]
        h = 1e-4
        errs = []
        for (i, j) in pix:
            Js = []
            for sgn in (1.0, -1.0):
                r = rho.copy()
                r[:, i, j] += sgn * h
                b.set_design_eps(chain.eps(r).reshape(-1))
                F = b.forward()
                Js.append([objective(b.dft_of(F, k)) for k in range(2)])
            for k in range(2):
                fd = (Js[0][k] - Js[1][k]) / (2 * h)
                errs.append(abs(fd - g[k, i, j]) / max(abs(fd), 1e-300))
        assert max(errs) <= 1e-3, max(errs)
    finally:
        b.close()
