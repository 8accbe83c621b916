"""The GPU mode solver (photonfdtd_b200.mode, csrc/modesolver.cu) against the
reference's own solver (src/photonfdtd/mode.py, scipy ARPACK in shift-invert
mode, run here from baseline/_ref): the operator kernels against the
reference's sparse matrix (1e-12 of max), the Chebyshev filter kernel against
the restated recurrence, then whole solves: the effective indices to 1e-9
relative and the normalised transverse fields |Ey|, |Ez| to 1e-6 relative
L2 (eigenvectors are defined up to sign / phase), with and without the
polarisation filter; and the reference's own known-answer tests
(tests/test_mode_vectorial.py): the high- and low-contrast slabs' TE0 / TM0
effective indices against the analytic dispersion relation within 0.5%."""
import ctypes as C
import math

import numpy as np
import pytest
import torch

import photonfdtd_b200 as pf
from photonfdtd_b200 import _native as N
from photonfdtd_b200.mode import ModeSolver
from oracle import mode_ref

pytestmark = pytest.mark.gpu

LAM0 = 1.55e-6
K0 = 2 * math.pi / LAM0


def _reference():
    from baseline.locate import import_reference
    ref = import_reference()
    if ref is None:
        pytest.skip("the reference package is not installed in baseline/_ref")
    return ref


def strip(mod, num_modes=4, polarization=None):
    m = mod or pf
    core = m.Box(center=(0.0, 0.0), size=(0.5e-6, 0.22e-6), medium=m.Medium.from_index(3.48))
    kw = dict(size=(2.0e-6, 1.5e-6), cell_size=0.02e-6, structures=[core], wavelength=LAM0,
              background_eps=1.444 ** 2, num_modes=num_modes)
    if polarization:
        kw["polarization"] = polarization
    return mod.ModeSolver(**kw) if mod is not None else ModeSolver(**kw)


def test_operator_kernels_match_the_reference_matrix():
    ms = strip(_reference())
    P, k2 = mode_ref.reference_operator(ms)
    X = np.random.default_rng(4).standard_normal((5, P.shape[0]))
    ref = (P @ X.T).T
    L = N.lib()
    dev = torch.device("cuda")
    eps = torch.tensor(ms.eps_r.ravel(), dtype=torch.float64, device=dev)
    x = torch.tensor(X, device=dev)
    y = torch.empty_like(x)
    work = torch.empty(10 * ms.ny * ms.nz * 5, dtype=torch.float64, device=dev)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    assert L.pfm_apply(ms.ny, ms.nz, ms.dy, ms.dz, k2, p(eps), p(x), p(y), 5, p(work), st) == 0
    got = y.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    lo, hi = -3e16, k2 * 2.5
    want = mode_ref.chebyshev(ms.eps_r, ms.dy, ms.dz, k2, X, 12, lo, hi)
    assert L.pfm_chebyshev(ms.ny, ms.nz, ms.dy, ms.dz, k2, p(eps), p(x), 5, 12, lo, hi,
                           p(work), st) == 0
    got = x.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    assert L.pfm_apply(ms.ny, ms.nz, ms.dy, ms.dz, -1.0, p(eps), p(x), p(y), 5, p(work),
                       st) == N.PF_ERR_INVALID


def _compare(ref_res, res, n_modes):
    assert res.n_eff.shape == (n_modes,)
    np.testing.assert_allclose(res.n_eff, ref_res.n_eff, rtol=1e-9, atol=0)
    for i in range(n_modes):
        for c in ("Ey", "Ez"):
            a, b = np.abs(getattr(res, c)[i]), np.abs(getattr(ref_res, c)[i])
            assert np.linalg.norm(a - b) <= 1e-6 * max(np.linalg.norm(b), 1e-30), (i, c)
        assert np.isclose(res.psi[i].max(), 1.0)
    assert res.max_residual < 1e-10


@pytest.mark.parametrize("polarization", [None, "te", "tm"])
def test_strip_modes_match_the_reference_solver(polarization):
    ref = _reference()
    n = 4 if polarization is None else 2
    ref_res = strip(ref, n, polarization).solve()
    res = strip(None, n, polarization).solve()
    _compare(ref_res, res, n)


def _analytic_slab(n1, n2, d, kind):
    from scipy.optimize import brentq
    fac = 1.0 if kind == "te" else (n1 ** 2 / n2 ** 2)
    lim = (math.pi / (K0 * d)) ** 2
    neff_min = math.sqrt(n1 ** 2 - lim) if lim < n1 ** 2 - n2 ** 2 else n2
    lo, hi = max(n2, neff_min) + 1e-6, n1 - 1e-9

    def g(neff):
        kap = K0 * math.sqrt(n1 ** 2 - neff ** 2)
        gam = K0 * math.sqrt(neff ** 2 - n2 ** 2)
        return kap * math.tan(kap * d / 2.0) - fac * gam

    return brentq(g, lo, hi)


@pytest.mark.parametrize("n1,n2,d,Lz,num_modes", [(3.0, 1.0, 0.30e-6, 2.0e-6, 26),
                                                  (1.50, 1.45, 0.70e-6, 4.0e-6, 6)])
def test_slab_known_answers_and_reference(n1, n2, d, Lz, num_modes):
    """The reference's acceptance cases (tests/test_mode_vectorial.py:52-137):
    a slab invariant along y in an 8 um PEC box, 30 cells across the core."""
    ref = _reference()
    Ly, dy, dz = 8e-6, 0.1e-6, d / 30

    def build(mod):
        core = (mod or pf).Box(center=(0.0, 0.0), size=(3 * Ly, d),
                               medium=(mod or pf).Medium.from_index(n1))
        kw = dict(size=(Ly, Lz), cell_size=(dy, dz), structures=[core], wavelength=LAM0,
                  background_eps=n2 ** 2, num_modes=num_modes)
        return mod.ModeSolver(**kw) if mod is not None else ModeSolver(**kw)

    res = build(None).solve()
    te = tm = None
    for i in range(len(res.n_eff)):
        py = float(np.sum(np.abs(res.Ey[i]) ** 2))
        pz = float(np.sum(np.abs(res.Ez[i]) ** 2))
        if py >= pz and te is None:
            te = float(res.n_eff[i])
        if py < pz and tm is None:
            tm = float(res.n_eff[i])
    te0, tm0 = _analytic_slab(n1, n2, d, "te"), _analytic_slab(n1, n2, d, "tm")
    assert abs(te - te0) / te0 < 5e-3 and abs(tm - tm0) / tm0 < 5e-3, (te, te0, tm, tm0)
    np.testing.assert_allclose(res.n_eff, build(ref).solve().n_eff, rtol=1e-9, atol=0)
