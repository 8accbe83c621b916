"""NumPy restatement of the reference's waveguide mode operator
(src/photonfdtd/mode.py:228-286), matrix-free.

TEST INFRASTRUCTURE: the checker of csrc/modesolver.cu; never part of the
product path.

The reference assembles P = [[Puu, Puv], [Pvu, Pvv]] from scipy sparse
difference matrices (Uu, Uv forward differences along z and y with a zero
neighbour past the last node, Vu = -Uu^T, Vv = -Uv^T). Expanding its four
blocks, with the y and z operators commuting, gives the four-pass form that
`apply` evaluates (and the CUDA kernels too):
    a = Uv u, b = Uu v, A = eps u + Vv a / k2, B = eps v + Vu b / k2,
    C = (Vu A + Vv B - Vu Vv (a + b) / k2) / eps,
    P [u; v] = [k2 A - Vv b + Uu C ; k2 B - Vu a + Uv C].
`reference_operator` rebuilds the reference's own sparse matrix (through the
reference's ModeSolver._difference_operators) for comparison.
"""
from __future__ import annotations

import math

import numpy as np


def _fz(f, dz):
    g = -f.copy()
    g[:, :-1] += f[:, 1:]
    return g / dz


def _fy(f, dy):
    g = -f.copy()
    g[:-1] += f[1:]
    return g / dy


def _bz(f, dz):
    g = f.copy()
    g[:, 1:] -= f[:, :-1]
    return g / dz


def _by(f, dy):
    g = f.copy()
    g[1:] -= f[:-1]
    return g / dy


def apply(eps, dy, dz, k2, X):
    """P X for a block X of shape (nvec, 2 ny nz), each row [u; v]."""
    ny, nz = eps.shape
    n = ny * nz
    out = np.empty_like(X)
    for c in range(X.shape[0]):
        u = X[c, :n].reshape(ny, nz)
        v = X[c, n:].reshape(ny, nz)
        a, b = _fy(u, dy), _fz(v, dz)
        A = eps * u + _by(a, dy) / k2
        B = eps * v + _bz(b, dz) / k2
        Cc = (_bz(A, dz) + _by(B, dy) - _bz(_by(a + b, dy), dz) / k2) / eps
        out[c, :n] = (k2 * A - _by(b, dy) + _fz(Cc, dz)).ravel()
        out[c, n:] = (k2 * B - _bz(a, dz) + _fy(Cc, dy)).ravel()
    return out


def chebyshev(eps, dy, dz, k2, X, degree, lo, hi):
    """T_degree((P - c) / e) X, [lo, hi] mapped to [-1, 1]."""
    e, c = 0.5 * (hi - lo), 0.5 * (hi + lo)
    prev, cur = X, (apply(eps, dy, dz, k2, X) - c * X) / e
    for _ in range(1, degree):
        prev, cur = cur, 2.0 * (apply(eps, dy, dz, k2, cur) - c * cur) / e - prev
    return cur


def reference_operator(ms):
    """The reference's sparse P for a reference ModeSolver `ms`, assembled
    exactly as its solve() does (mode.py:262-286)."""
    import scipy.sparse as sp
    n = ms.ny * ms.nz
    k0 = 2 * math.pi / ms.wavelength
    k2 = k0 * k0
    Uu, Uv, Vu, Vv = ms._difference_operators()
    er = ms.eps_r.reshape(n).astype(float)
    eps_u = sp.diags(er)
    eps_v = sp.diags(er)
    ezi = sp.diags(1.0 / er)
    I = sp.eye(n, format="csr")
    Puu = (-Uu @ ezi @ Vv @ Vu @ Uv / k2 + (k2 * I + Uu @ ezi @ Vu) @ (eps_u + Vv @ Uv / k2))
    Pvv = (-Uv @ ezi @ Vu @ Vv @ Uu / k2 + (k2 * I + Uv @ ezi @ Vv) @ (eps_v + Vu @ Uu / k2))
    Puv = (Uu @ ezi @ Vv @ (eps_v + Vu @ Uu / k2) - (k2 * I + Uu @ ezi @ Vu) @ Vv @ Uu / k2)
    Pvu = (Uv @ ezi @ Vu @ (eps_u + Vv @ Uv / k2) - (k2 * I + Uv @ ezi @ Vv) @ Vu @ Uv / k2)
    return sp.bmat([[Puu, Puv], [Pvu, Pvv]], format="csr"), k2
