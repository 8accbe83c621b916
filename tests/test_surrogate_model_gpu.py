"""The trained config-5 surrogate (photonfdtd_b200/data/surrogate_config5.npz,
written by photonfdtd_b200.surrogate_run) against the float64 FDTD engine on
64 held-out densities (seeds 18000-18063, never seen in training), and what
it buys: spectra within a few percent, orders of magnitude faster than the
FDTD runs it replaces."""
import os
import time

import numpy as np
import pytest

import photonfdtd_b200
from photonfdtd_b200 import surrogate as S
from surrogate_util import oracle_value_and_grad

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(photonfdtd_b200.__file__), "data", "surrogate_config5.npz")


def test_trained_surrogate_against_fp64_fdtd():
    import torch
    rho = S.densities(range(18000, 18064))
    gen = S.SpectrumGenerator(64, precision="float64")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    T = gen.spectra(rho)
    torch.cuda.synchronize()
    t_fdtd = time.perf_counter() - t0
    gen.close()
    net = S.SurrogateNet.load(WEIGHTS, 64)
    net.predict(rho)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    P = net.predict(rho)
    torch.cuda.synchronize()
    t_net = time.perf_counter() - t0
    err = S.spectrum_errors(P, T)
    # 2000 held-out designs: mean 2.9 %, p95 4.9 % (complex T, relative L2)
    assert err["mean"] <= 0.04, err
    assert err["p95"] <= 0.07, err
    # the mean spectrum (no network) is four times worse
    mean_only = S.spectrum_errors(np.broadcast_to(T.mean(axis=0), T.shape), T)
    assert mean_only["mean"] >= 2.5 * err["mean"], (mean_only, err)
    assert t_fdtd / t_net >= 100.0, (t_fdtd, t_net)


def test_value_and_grad_through_the_network_matches_the_oracle():
    """d objective / d rho through the network's reverse pass on the GPU
    against the float64 NumPy network (oracle/surrogate_ref.py) with the same
    trained weights; the oracle's own gradient is pinned to finite
    differences in tests/test_surrogate_oracle.py. BF16 activations limit the
    agreement to a few percent."""
    import torch
    from oracle.surrogate_ref import RefNet
    net = S.SurrogateNet.load(WEIGHTS, 32)
    rho = S.densities(range(18100, 18104))
    v, g = net.value_and_grad(rho, S.band_objective)
    ref = RefNet(S.plan(), S.SurrogateNet.load_params(WEIGHTS))
    z = np.load(WEIGHTS)
    vr, gr = oracle_value_and_grad(ref, z["t_mean"], z["t_std"], rho)
    assert np.allclose(v, vr, rtol=0.02, atol=0.01), (v, vr)
    cos = np.sum(g * gr) / (np.linalg.norm(g) * np.linalg.norm(gr))
    assert cos >= 0.98, cos
    assert np.linalg.norm(g - gr) <= 0.2 * np.linalg.norm(gr)
