"""The full inverse-design batch: 256 uneven 2D TE instances, 4000 steps,
64 x 64 design windows, J = sum over frequencies and output-line cells of
|DFT Ey|^2 per instance. The adjoint gradient dJ/drho is checked against
central finite differences (h = 1e-4 in rho, float64 runs) on 32 random
pixels drawn with default_rng(5), one pixel in each of 32 different
instances, so that the +h and -h perturbations of all 32 pixels run as two
batched forward passes. Each relative error must be at most 1e-3.
"""
import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200 import workloads as W
from photonfdtd_b200.batch import BatchTE
from oracle.adjoint2d import objective, objective_cotangent

pytestmark = pytest.mark.gpu


def test_config4_gradient_matches_central_differences():
    sizes = W.config4_sizes()
    rhos = [W.config4_density(k) for k in range(len(sizes))]
    sims = [W.config4_instance(pf, nx, ny, rho=r, i=k, precision="float64")
            for k, ((nx, ny), r) in enumerate(zip(sizes, rhos))]
    wins = [W.design_window_box(nx, ny, 64) for nx, ny in sizes]
    b = BatchTE(sims, wins)
    try:
        span = W.EPS_CORE - W.EPS_CLAD
        rho0 = b.pack_windows(rhos)
        eps0 = W.EPS_CLAD + rho0 * span
        assert np.array_equal(b.design_eps(), eps0.astype(np.float64))
        F = b.forward()
        g = b.grad_eps(b.adjoint(objective_cotangent(F)), eps0) * span
        rng = np.random.default_rng(5)
        inst = rng.choice(len(sizes), 32, replace=False)
        pix = rng.integers(0, 64 * 64, 32)
        h = 1e-4
        J = []
        for sgn in (1.0, -1.0):
            r = rho0.copy()
            for k, p in zip(inst, pix):
                r[b.design_slice(int(k))][int(p)] += sgn * h
            b.set_design_eps(W.EPS_CLAD + r * span)
            Fp = b.forward()
            J.append(np.array([objective(b.dft_of(Fp, int(k))) for k in inst]))
        fd = (J[0] - J[1]) / (2 * h)
        ad = np.array([g[b.design_slice(int(k))][int(p)] for k, p in zip(inst, pix)])
        rel = np.abs(fd - ad) / np.abs(fd)
        assert np.all(np.abs(fd) > 0)
        assert rel.max() <= 1e-3, (rel.max(), int(np.argmax(rel)))
    finally:
        b.close()
