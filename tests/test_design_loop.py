"""Host logic of the surrogate-assisted design loop (surrogate.surrogate_loop)
on CPU stand-ins for the FDTD problem and the network: a smooth concave
objective of the density with its exact gradient, and surrogates whose
gradient is exact, offset by a constant, or whose predictions are off."""
import numpy as np
import pytest

from photonfdtd_b200 import surrogate as S

RNG = np.random.default_rng(7)
W = RNG.standard_normal((64, 64))


def _obj(rho):
    return -np.mean((rho - 0.5 - 0.1 * W) ** 2, axis=(1, 2))


def _grad(rho):
    return -2.0 * (rho - 0.5 - 0.1 * W) / rho[0].size


def _spec(v):
    return np.ones((v.size, S.N_FREQ), complex) * (1.0 + v[:, None])


class Problem:
    n = 4

    def __init__(self):
        self.grads = 0

    def value_grad_spectra(self, rho):
        self.grads += 1
        v = _obj(rho)
        return v, _grad(rho), _spec(v)

    def value(self, rho):
        v = _obj(rho)
        return v, _spec(v)

    def value_and_grad(self, rho):
        v, g, _ = self.value_grad_spectra(rho)
        return v, g


class Net:
    def __init__(self, offset=0.0, pred_scale=1.0):
        self.offset, self.pred_scale = offset, pred_scale

    def value_and_grad(self, rho, objective):
        return _obj(rho), _grad(rho) + self.offset

    def predict(self, rho):
        return _spec(_obj(rho)) * self.pred_scale


@pytest.fixture(autouse=True)
def _no_cuda(monkeypatch):
    monkeypatch.setattr(S, "_sync", lambda: None)


def _run(net, **kw):
    param = S.SmoothDesign()
    prob = Problem()
    r = S.surrogate_loop(prob, net, param, param.start(range(4)), iters=120, **kw)
    return r, prob


def test_iterations_are_design_updates_and_best_never_drops():
    r, prob = _run(Net())
    assert r["fdtd_gradients"] == prob.grads
    assert r["fdtd_gradients"] + r["surrogate_steps_kept"] == 120
    best = [e["best"] for e in r["log"]]
    assert all(b1 >= b0 for b0, b1 in zip(best, best[1:]))
    assert r["final"] == max(best + [r["final"]])


def test_exact_surrogate_is_never_rolled_back():
    r, _ = _run(Net())
    assert r["surrogate_bursts_rejected"] == 0
    assert r["surrogate_steps_kept"] > r["fdtd_gradients"]


def test_correction_removes_a_constant_gradient_bias():
    exact, _ = _run(Net())
    biased, _ = _run(Net(offset=3e-4))
    assert biased["surrogate_bursts_rejected"] == 0
    assert biased["final"] == pytest.approx(exact["final"], rel=1e-9, abs=1e-12)


def test_above_the_error_threshold_the_loop_is_the_plain_loop():
    bad, prob = _run(Net(pred_scale=1.5), fallback_steps=3)  # 50% off on |T|: always above 2%
    assert all(e["next_fdtd_steps"] == 3 and e["bursts_kept"] == 0 for e in bad["log"])
    assert bad["surrogate_steps_kept"] == 0 and bad["fdtd_gradients"] == 120
    param = S.SmoothDesign()
    plain = S.plain_adjoint_loop(Problem(), param, param.start(range(4)), iters=120)
    # the same Adam steps on the same gradients: the plain loop's result
    assert bad["final"] == pytest.approx(plain["final"], rel=1e-12)


def test_target_time_is_recorded_once_reached():
    r, _ = _run(Net(), target=-1.0)  # any verified objective clears it
    assert r["reached_target_s"] is not None and r["reached_target_s"] >= 0.0
    r, _ = _run(Net(), target=1.0)   # unreachable (the objective is <= 0)
    assert r["reached_target_s"] is None
