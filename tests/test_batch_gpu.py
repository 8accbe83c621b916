"""Batched 2D TE engine on the GPU against the TE oracle.

Forward: every instance's line DFT and final fields equal the oracle's (the
reference's step) bit for bit, float32 and float64. Adjoint: the gradient
with respect to the design permittivity matches the oracle's adjoint
(float64 to 1e-9 of its scale, float32 within 1e-3 relative L2) and central
finite differences of the GPU forward run in float64 (h = 1e-4 in density, 32
pixels, within 1e-3). Checkpoint spacing changes nothing, not one bit.
"""
import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200 import _native as N
from photonfdtd_b200 import workloads as W
from photonfdtd_b200.batch import BatchTE, value_and_grad_eps
from oracle.adjoint2d import TEAdjointRun, objective, objective_cotangent
from oracle.fdtd_oracle import EPS0

pytestmark = pytest.mark.gpu

SIZES = [(60, 50), (72, 44), (52, 58)]
D = 12


def _window(nx, ny, d=D):
    return (nx // 2 - d // 2, ny // 2 - d // 2, d)


def _sims(precision, n_steps, sizes=SIZES, d=D, n_freqs=3, seed0=0):
    rhos = [W.config4_density(seed0 + k, d) for k in range(len(sizes))]
    sims = [W.config4_instance(pf, nx, ny, rho=r, n_steps=n_steps, n_freqs=n_freqs,
                               precision=precision, design=d)
            for (nx, ny), r in zip(sizes, rhos)]
    return sims, rhos, [_window(nx, ny, d) for nx, ny in sizes]


@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_forward_matches_oracle_bitwise(precision):
    sims, _, wins = _sims(precision, 240)
    b = BatchTE(sims, wins, checkpoint_every=50)
    try:
        F = b.forward()
        for k, (s, w) in enumerate(zip(sims, wins)):
            te = TEAdjointRun(s, w)
            ref = te.forward(record=False)
            assert np.array_equal(b.dft_of(F, k), ref), k
            for c in ("Ex", "Ey", "Hz"):
                assert np.array_equal(b.read_field(k, c), te.F[c]), (k, c)
    finally:
        b.close()


@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_adjoint_matches_oracle(precision):
    sims, rhos, wins = _sims(precision, 300)
    b = BatchTE(sims, wins, checkpoint_every=64)
    try:
        F = b.forward()
        gk = b.adjoint(objective_cotangent(F))
        for k, (s, w) in enumerate(zip(sims, wins)):
            te = TEAdjointRun(s, w)
            ref = te.adjoint(objective_cotangent(te.forward()))
            got = b.window_of(gk, k)
            scale = np.max(np.abs(ref))
            assert scale > 0
            if precision == "float64":
                assert np.max(np.abs(got - ref)) <= 1e-9 * scale, k
            else:
                assert np.linalg.norm(got - ref) <= 1e-3 * np.linalg.norm(ref), k
    finally:
        b.close()


def test_checkpoint_spacing_changes_nothing():
    sims, _, wins = _sims("float64", 200)
    outs = []
    for K in (1, 7, 64, 200, 1000):
        b = BatchTE(sims, wins, checkpoint_every=K, tile_rows=(8, 16, 32)[K % 3])
        try:
            F = b.forward()
            g1 = b.adjoint(objective_cotangent(F))
            g2 = b.adjoint(objective_cotangent(F))   # again after the same forward
            assert np.array_equal(g1, g2)
            outs.append((F, g1, b.info()))
        finally:
            b.close()
    for F, g, info in outs[1:]:
        assert np.array_equal(F, outs[0][0])
        assert np.array_equal(g, outs[0][1])
    assert outs[0][2]["segments"] == 200 and outs[-1][2]["segments"] == 1


def test_tile_autotuner_changes_nothing():
    """The default tile height comes from timing 8, 16 and 32 rows on the
    batch itself; whichever it keeps, and after an explicit retile, the DFT
    and the gradient equal a fixed-height batch's bit for bit."""
    sims, _, wins = _sims("float32", 150)
    fixed = BatchTE(sims, wins, tile_rows=32)
    auto = BatchTE(sims, wins)
    L = N.lib()
    try:
        assert auto.tile_rows in (8, 16, 32)
        assert set(auto.tile_ms_per_step) == {8, 16, 32}
        assert all(m > 0 for m in auto.tile_ms_per_step.values())
        assert auto.tile_ms_per_step[auto.tile_rows] == min(auto.tile_ms_per_step.values())
        F0 = fixed.forward()
        g0 = fixed.adjoint(objective_cotangent(F0))
        F1 = auto.forward()
        assert np.array_equal(F1, F0)
        assert np.array_equal(auto.adjoint(objective_cotangent(F1)), g0)
        for rows in (8, 16):
            assert L.pfb_set_tile_rows(auto.h, rows) == N.PF_OK
            F2 = auto.forward()
            assert np.array_equal(F2, F0)
            assert np.array_equal(auto.adjoint(objective_cotangent(F2)), g0)
        assert L.pfb_set_tile_rows(auto.h, 12) == N.PF_ERR_INVALID
    finally:
        fixed.close()
        auto.close()


def test_gradient_matches_central_differences():
    """dJ/drho against (J(rho + h) - J(rho - h)) / 2h, h = 1e-4, float64, on 32
    pixels (default_rng(5)); each forward perturbs one pixel per instance."""
    sizes = [(80, 64), (96, 70)]
    d = 16
    sims, rhos, wins = _sims("float64", 700, sizes=sizes, d=d)
    b = BatchTE(sims, wins)
    try:
        span = W.EPS_CORE - W.EPS_CLAD
        rho0 = b.pack_windows(rhos)
        F = b.forward()
        J0 = [objective(b.dft_of(F, k)) for k in range(2)]
        g = b.grad_eps(b.adjoint(objective_cotangent(F)), W.EPS_CLAD + rho0 * span) * span
        rng = np.random.default_rng(5)
        pix = [(k, int(rng.integers(0, d * d))) for k in (0, 1) for _ in range(16)]
        h = 1e-4
        errs = []
        for q in range(16):
            p0, p1 = pix[q], pix[16 + q]
            Js = []
            for sgn in (1.0, -1.0):
                r = rho0.copy()
                r[b.design_slice(0)][p0[1]] += sgn * h
                r[b.design_slice(1)][p1[1]] += sgn * h
                b.set_design_eps(W.EPS_CLAD + r * span)
                Fp = b.forward()
                Js.append([objective(b.dft_of(Fp, k)) for k in range(2)])
            for k, p in ((0, p0), (1, p1)):
                fd = (Js[0][k] - Js[1][k]) / (2 * h)
                ad = g[b.design_slice(k)][p[1]]
                errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
        assert min(J0) > 0
        assert max(errs) <= 1e-3, max(errs)
    finally:
        b.close()


def test_autograd_function_on_gpu_batch():
    torch = pytest.importorskip("torch")
    sims, rhos, wins = _sims("float64", 200)
    b = BatchTE(sims, wins)
    try:
        eps = b.design_eps()
        vals, grad = value_and_grad_eps(b, eps)
        b.set_design_eps(eps)
        F = b.forward()
        gk = b.adjoint(objective_cotangent(F))
        assert np.array_equal(grad, b.grad_eps(gk, eps))
        for k in range(len(sims)):
            assert vals[k] == pytest.approx(objective(b.dft_of(F, k)), rel=1e-12)
        del torch
    finally:
        b.close()


def test_adjoint_needs_a_forward_of_the_current_design():
    sims, _, wins = _sims("float32", 40)
    b = BatchTE(sims, wins)
    try:
        g = np.zeros((b.n_line, b.n_freq), np.complex128)
        with pytest.raises(N.NativeError):
            b.adjoint(g)
        b.forward()
        b.set_design_eps(b.design_eps())
        with pytest.raises(N.NativeError):
            b.adjoint(g)
        with pytest.raises(ValueError):
            b.adjoint(g[:-1])
    finally:
        b.close()


@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_fused_steps_equal_split_passes(precision, monkeypatch):
    """The fused forward step (one launch per step, double-buffered fields,
    recomputed Hz halo) and the fused reverse step (hA / hB recomputed on the
    halo in shared memory) against the split passes: line DFT, final fields
    and the adjoint gradient bit for bit, with an odd checkpoint spacing so
    that chunks start on both levels."""
    sims, _, wins = _sims(precision, 200)
    out = {}
    for split in (False, True):
        if split:
            monkeypatch.setenv("PFB200_BATCH_SPLIT", "1")
        else:
            monkeypatch.delenv("PFB200_BATCH_SPLIT", raising=False)
        b = BatchTE(sims, wins, checkpoint_every=37, tile_rows=(32, 16)[int(split)])
        try:
            assert b.info()["fused"] == (0 if split else 1)
            F = b.forward()
            fields = [b.read_field(k, c) for k in range(len(sims)) for c in ("Ex", "Ey", "Hz")]
            g = b.adjoint(objective_cotangent(F))
            out[split] = (F, fields, g)
        finally:
            b.close()
    (F0, f0, g0), (F1, f1, g1) = out[False], out[True]
    assert np.array_equal(F0, F1)
    for a, c in zip(f0, f1):
        assert np.array_equal(a, c)
    assert np.array_equal(g0, g1)
