"""The surrogate network's NumPy oracle: architecture bookkeeping and its
reverse pass against central finite differences (float64, CPU)."""
import numpy as np

from photonfdtd_b200.surrogate import init_params, n_params, plan
from oracle.surrogate_ref import RefNet, bf16, col2im, im2col


def test_architecture():
    layers = plan()
    assert n_params(layers) == 1_750_562
    assert [L.kind for L in layers].count("conv") == 8


def test_im2col_col2im_are_adjoint():
    rng = np.random.default_rng(0)
    for shape, k, s, p in [((2, 9, 7, 3), (3, 3), 2, (1, 1)), ((1, 1, 8, 4), (1, 3), 1, (0, 1))]:
        x = rng.standard_normal(shape)
        col, Ho, Wo = im2col(x, k[0], k[1], s, p[0], p[1])
        d = rng.standard_normal(col.shape)
        assert np.isclose(np.sum(col * d), np.sum(x * col2im(d, shape, k[0], k[1], s, p[0], p[1])))


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 1e-30], np.float64)
    r = bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7 and r[3] == -2.5
    assert abs(r[4] - 1e-30) <= 2 ** -8 * 1e-30


def test_reverse_pass_matches_central_differences():
    layers = plan()
    params = init_params(layers, seed=3)
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, (2, 64, 64))
    R = rng.standard_normal((2, 32, 2))
    net = RefNet(layers, params)
    net.forward(x)
    grads, dx = net.backward(R)

    def loss(ps, xx):
        return float(np.sum(RefNet(layers, ps).forward(xx) * R))

    h = 1e-6
    for li in (0, 3, 5, 7, 10):
        w = params[li][0]
        for _ in range(2):
            i, j = (int(rng.integers(0, n)) for n in w.shape)
            pp = [(None if a is None else a.copy(), None if b is None else b.copy())
                  for a, b in params]
            pm = [(None if a is None else a.copy(), None if b is None else b.copy())
                  for a, b in params]
            pp[li][0][i, j] += h
            pm[li][0][i, j] -= h
            fd = (loss(pp, x) - loss(pm, x)) / (2 * h)
            assert abs(fd - grads[li][0][i, j]) <= 1e-5 * max(abs(fd), 1e-3), (li, fd)
    for _ in range(4):
        b, i, j = int(rng.integers(0, 2)), int(rng.integers(0, 64)), int(rng.integers(0, 64))
        xp, xm = x.copy(), x.copy()
        xp[b, i, j] += h
        xm[b, i, j] -= h
        fd = (loss(params, xp) - loss(params, xm)) / (2 * h)
        assert abs(fd - dx[b, i, j]) <= 1e-5 * max(abs(fd), 1e-3), fd


def test_trained_network_rho_gradient_matches_central_differences():
    """The float64 oracle network with the trained config-5 weights: the
    design-objective gradient with respect to rho against central
    differences (the reference the GPU gradient is checked against)."""
    import os
    import photonfdtd_b200
    from photonfdtd_b200 import surrogate as S
    from surrogate_util import oracle_value_and_grad
    path = os.path.join(os.path.dirname(photonfdtd_b200.__file__), "data",
                        "surrogate_config5.npz")
    ref = RefNet(plan(), S.SurrogateNet.load_params(path))
    z = np.load(path)
    rho = S.densities(range(18100, 18102))
    v, g = oracle_value_and_grad(ref, z["t_mean"], z["t_std"], rho)
    rng = np.random.default_rng(9)
    h = 1e-6
    for _ in range(4):
        k, i, j = int(rng.integers(0, 2)), int(rng.integers(0, 64)), int(rng.integers(0, 64))
        rp, rm = rho.copy(), rho.copy()
        rp[k, i, j] += h
        rm[k, i, j] -= h
        vp, _ = oracle_value_and_grad(ref, z["t_mean"], z["t_std"], rp)
        vm, _ = oracle_value_and_grad(ref, z["t_mean"], z["t_std"], rm)
        fd = (vp[k] - vm[k]) / (2 * h)
        assert abs(fd - g[k, i, j]) <= 1e-4 * max(abs(fd), 1e-4), (fd, g[k, i, j])
