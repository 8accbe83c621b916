"""The density-chain oracle (conic filter + tanh projection, design.py:40-72
of the reference) on CPU: its documented properties and its reverse pass
against central differences."""
import numpy as np
import pytest

from oracle import design_ref as D


def test_filter_keeps_constants_and_projection_keeps_endpoints():
    rho = np.full((20, 20), 0.37)
    assert np.allclose(D.conic_filter(rho, 3.5), 0.37, rtol=0, atol=1e-15)
    assert np.array_equal(D.conic_filter(rho, 0.0), rho)
    p = D.tanh_projection(np.array([0.0, 0.5, 1.0]), beta=8.0, eta=0.5)
    assert np.allclose(p, [0.0, 0.5, 1.0], atol=1e-15)
    assert np.array_equal(D.tanh_projection(rho, beta=0.0), rho)


def test_filter_is_a_normalised_cone_average():
    rng = np.random.default_rng(0)
    rho = rng.uniform(size=(9, 11))
    R = 2.5
    k = D.cone(R)
    want = np.empty_like(rho)
    for i in range(rho.shape[0]):
        for j in range(rho.shape[1]):
            num = den = 0.0
            for a in range(-3, 4):
                for b in range(-3, 4):
                    ii, jj = i + a, j + b
                    if 0 <= ii < rho.shape[0] and 0 <= jj < rho.shape[1]:
                        num += k[a + 3, b + 3] * rho[ii, jj]
                        den += k[a + 3, b + 3]
            want[i, j] = num / den
    assert k.shape == (7, 7)
    assert np.allclose(D.conic_filter(rho, R), want, rtol=1e-14, atol=0)


@pytest.mark.parametrize("radius,beta", [(0.0, 6.0), (3.0, 0.0), (2.6, 8.0)])
def test_backward_matches_central_differences(radius, beta):
    rng = np.random.default_rng(1)
    rho = rng.uniform(0.1, 0.9, size=(12, 12))
    w = rng.standard_normal((12, 12))
    g = D.backward(rho, w, radius, beta, 0.45)
    h = 1e-6
    for (i, j) in [(0, 0), (3, 7), (11, 5), (6, 6)]:
        e = np.zeros_like(rho)
        e[i, j] = h
        fd = (np.sum(w * D.forward(rho + e, radius, beta, 0.45)) -
              np.sum(w * D.forward(rho - e, radius, beta, 0.45))) / (2 * h)
        assert abs(fd - g[i, j]) <= 1e-7 * max(1.0, abs(fd)), (i, j, fd, g[i, j])
