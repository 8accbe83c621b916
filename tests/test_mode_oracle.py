"""The matrix-free restatement of the reference's waveguide mode operator
(oracle/mode_ref.py) against the reference's own sparse assembly
(src/photonfdtd/mode.py:256-286), on random blocks for a silicon strip
cross-section and a high-contrast slab, and its Chebyshev filter against the
three-term recurrence on the sparse matrix. CPU only."""
import math

import numpy as np
import pytest

from oracle import mode_ref


def _reference():
    from baseline.locate import import_reference
    ref = import_reference()
    if ref is None:
        pytest.skip("the reference package is not installed in baseline/_ref")
    return ref


def strip(pf):
    core = pf.Box(center=(0.0, 0.0), size=(0.5e-6, 0.22e-6), medium=pf.Medium.from_index(3.48))
    return pf.ModeSolver(size=(1.2e-6, 0.8e-6), cell_size=(0.03e-6, 0.025e-6), structures=[core],
                         wavelength=1.55e-6, background_eps=1.444 ** 2, num_modes=2)


def slab(pf):
    core = pf.Box(center=(0.0, 0.0), size=(3 * 4e-6, 0.3e-6), medium=pf.Medium.from_index(3.0))
    return pf.ModeSolver(size=(4e-6, 1.0e-6), cell_size=(0.1e-6, 0.02e-6), structures=[core],
                         wavelength=1.55e-6, background_eps=1.0, num_modes=4)


@pytest.mark.parametrize("build", [strip, slab])
def test_matrix_free_operator_is_the_reference_matrix(build):
    ms = build(_reference())
    P, k2 = mode_ref.reference_operator(ms)
    X = np.random.default_rng(2).standard_normal((3, P.shape[0]))
    ref = (P @ X.T).T
    got = mode_ref.apply(ms.eps_r, ms.dy, ms.dz, k2, X)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_chebyshev_filter_is_the_recurrence():
    ms = strip(_reference())
    P, k2 = mode_ref.reference_operator(ms)
    X = np.random.default_rng(3).standard_normal((2, P.shape[0]))
    lo, hi = -3e16, k2 * 2.0
    e, c = 0.5 * (hi - lo), 0.5 * (hi + lo)
    prev, cur = X.T, (P @ X.T - c * X.T) / e
    for _ in range(1, 9):
        prev, cur = cur, 2.0 * (P @ cur - c * cur) / e - prev
    got = mode_ref.chebyshev(ms.eps_r, ms.dy, ms.dz, k2, X, 9, lo, hi)
    assert np.abs(got - cur.T).max() <= 1e-10 * np.abs(cur).max()
