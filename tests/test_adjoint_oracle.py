"""The 2D TE adjoint oracle: its forward run is the reference's step to the
bit (pinned through OracleRun, itself pinned to the reference's golden
runs), its adjoint agrees with central finite differences of that forward run
in float64, and the torch.autograd wrapper applies the chain rule
eps -> K -> DFT -> loss with PyTorch's complex-gradient convention. CPU only.
"""
import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200 import workloads as W
from photonfdtd_b200.batch import (checkpoint_bytes, choose_checkpoint, default_checkpoint,
                                   line_dft, value_and_grad_eps)
from oracle.adjoint2d import TEAdjointRun, objective, objective_cotangent
from oracle.fdtd_oracle import EPS0, OracleRun

NX, NY, D = 60, 50, 12


def _window(nx=NX, ny=NY, d=D):
    return (nx // 2 - d // 2, ny // 2 - d // 2, d)


def _sim(precision, n_steps, rho=None, nx=NX, ny=NY, n_freqs=3):
    return W.config4_instance(pf, nx, ny, rho=rho, n_steps=n_steps, n_freqs=n_freqs,
                              precision=precision, design=D)


@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_te_forward_is_the_reference_step(precision):
    sim = _sim(precision, 160)
    r = OracleRun(sim)
    r.advance(r.n_steps)
    ref = r.result()["dft"]["out"]["Ey"][:, 0, :, 0]
    te = TEAdjointRun(sim, _window())
    F = te.forward()
    assert np.array_equal(F, ref)
    for c in ("Ex", "Ey", "Hz"):
        assert np.array_equal(te.F[c], r.F[c][:, :, 0]), c
    assert np.abs(F).max() > 0


def _rho_grad(te, rho):
    eps = W.EPS_CLAD + rho * (W.EPS_CORE - W.EPS_CLAD)
    te.set_window_eps(eps)
    F = te.forward()
    gk = te.adjoint(objective_cotangent(F))
    return objective(F), gk * (-te.dt / (EPS0 * eps ** 2)) * (W.EPS_CORE - W.EPS_CLAD)


def test_adjoint_matches_central_differences_float64():
    rho = W.config4_density(0, D)
    te = TEAdjointRun(_sim("float64", 600, rho), _window())
    J0, g = _rho_grad(te, rho)
    assert J0 > 0

    def J(r):
        te.set_window_eps(W.EPS_CLAD + r * (W.EPS_CORE - W.EPS_CLAD))
        return objective(te.forward(record=False))

    rng = np.random.default_rng(5)
    h = 1e-4
    for _ in range(6):
        i, j = (int(v) for v in rng.integers(0, D, 2))
        rp, rm = rho.copy(), rho.copy()
        rp[i, j] += h
        rm[i, j] -= h
        fd = (J(rp) - J(rm)) / (2 * h)
        assert abs(fd - g[i, j]) <= 1e-6 * abs(fd), (i, j, fd, g[i, j])


def test_planted_adjoint_error_is_caught():
    """A wrong sign on one CPML psi term in the adjoint breaks the FD check."""
    rho = W.config4_density(1, D)
    te = TEAdjointRun(_sim("float64", 400, rho), _window())
    _, g = _rho_grad(te, rho)
    te.cpml = [tuple(a.copy() for a in te.cpml[0]), te.cpml[1]]
    te.cpml[0][1][:] *= -1.0        # c_e_x used only by the adjoint from here on
    gk_bad = te.adjoint(objective_cotangent(te.dft))
    eps = W.EPS_CLAD + rho * (W.EPS_CORE - W.EPS_CLAD)
    g_bad = gk_bad * (-te.dt / (EPS0 * eps ** 2)) * (W.EPS_CORE - W.EPS_CLAD)
    assert np.max(np.abs(g_bad - g)) > 1e-6 * np.max(np.abs(g))


class _OracleBatch:
    """The BatchTE surface the autograd wrapper uses, on the TE oracle."""

    def __init__(self, runs):
        self.runs = runs
        self.dt = runs[0].dt
        self.ny = np.array([r.ny for r in runs])
        self.n_inst = len(runs)
        self.off = np.concatenate([[0], np.cumsum([r.window[2] ** 2 for r in runs])])
        self.loff = np.concatenate([[0], np.cumsum(self.ny)])

    def set_design_eps(self, eps):
        for k, r in enumerate(self.runs):
            n = r.window[2]
            r.set_window_eps(eps[self.off[k]:self.off[k + 1]].reshape(n, n))
        self._eps = eps.copy()

    def forward(self):
        return np.concatenate([r.forward().T for r in self.runs])

    def adjoint(self, g):
        return np.concatenate([r.adjoint(g[self.loff[k]:self.loff[k + 1]].T).ravel()
                               for k, r in enumerate(self.runs)])

    def grad_eps(self, gk, eps):
        return -gk * self.dt / (EPS0 * eps * eps)

    def per_instance_sum(self, values):
        import torch
        idx = torch.repeat_interleave(torch.arange(self.n_inst), torch.as_tensor(self.ny))
        v = values.reshape(values.shape[0], -1).sum(dim=1)
        return torch.zeros(self.n_inst, dtype=v.dtype).index_add(0, idx, v)


def test_autograd_wrapper_chain_rule_and_complex_convention():
    torch = pytest.importorskip("torch")
    runs = [TEAdjointRun(_sim("float64", 300, W.config4_density(k, D), nx=nx, ny=ny),
                         _window(nx, ny)) for k, (nx, ny) in enumerate([(60, 50), (56, 44)])]
    b = _OracleBatch(runs)
    eps0 = np.concatenate([(W.EPS_CLAD + W.config4_density(k, D) * (W.EPS_CORE - W.EPS_CLAD))
                           .ravel() for k in range(2)])
    # a loss mixing |F|^2 and a linear term in Im F, per instance
    def loss(F):
        return b.per_instance_sum(F.real ** 2 + F.imag ** 2 + 1e-10 * F.imag)
    vals, grad = value_and_grad_eps(b, eps0, loss)
    # the same gradient by hand: cotangent 2F + i 1e-10
    b.set_design_eps(eps0)
    F = b.forward()
    gk = b.adjoint(2.0 * F + 1e-10j)
    assert np.allclose(grad, b.grad_eps(gk, eps0), rtol=1e-12, atol=0)
    assert vals.shape == (2,)
    # and by a directional finite difference in float64
    rng = np.random.default_rng(3)
    v = rng.standard_normal(eps0.size)
    h = 1e-6
    def total(e):
        b.set_design_eps(e)
        FF = torch.from_numpy(b.forward())
        return float(loss(FF).sum())
    fd = (total(eps0 + h * v) - total(eps0 - h * v)) / (2 * h)
    assert abs(fd - grad @ v) <= 1e-6 * abs(fd)


def test_default_checkpoint_balances_states_and_ring():
    # 35.2M-cell batch of 256 64x64 windows, 4000 steps: a few hundred steps
    k = default_checkpoint(4000, 110_000_000, 256 * 64 * 64)
    assert 300 < k < 700
    assert default_checkpoint(10, 10, 1_000_000) == 1
    assert default_checkpoint(10, 10 ** 9, 1) == 10


def test_checkpoint_spacing_spends_the_memory_budget():
    N, state, D, rb = 4000, 110_000_000, 256 * 64 * 64, 4
    ring_all = N * 2 * D * rb                      # 33.5 GB: no checkpoints at all
    assert checkpoint_bytes(N, N, state, D, rb) == ring_all
    assert choose_checkpoint(N, state, D, rb, 90e9) == N
    k0 = default_checkpoint(N, state, D)
    assert choose_checkpoint(N, state, D, rb, 0.0) == k0   # nothing fits: minimal memory
    for budget in (8e9, 12e9, 20e9, 30e9):
        k = choose_checkpoint(N, state, D, rb, budget)
        assert k0 <= k < N
        assert checkpoint_bytes(N, k, state, D, rb) <= budget
        # the next larger spacing (one segment fewer) would not fit
        segs = (N + k - 1) // k
        k_up = (N + segs - 2) // (segs - 1)
        assert checkpoint_bytes(N, k_up, state, D, rb) > budget
