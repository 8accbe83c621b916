"""What the trained surrogate gains over the plain adjoint loop (config 5),
measured rather than assumed: the same 8 designs (latent starts 30000-30007,
the band objective, float32 FDTD), the plain loop for 200 FDTD-gradient
iterations, then the surrogate-assisted loop (photonfdtd_b200.surrogate.
surrogate_loop: corrected-gradient bursts verified by FDTD forward runs,
online tuning) with the plain loop's wall clock as its budget.

Asserted: the plain loop raises the objective; the surrogate loop reaches the
plain loop's final objective within 1 % inside that budget. Reported (the
test prints one JSON line): the wall clock each loop needs to reach that
target and their ratio, and the objective each holds at the end. No speedup
is asserted: the measured ratio is near 1, far from a 5x gain."""
import json
import os
import time

import numpy as np
import pytest

import photonfdtd_b200
from photonfdtd_b200 import surrogate as S

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(photonfdtd_b200.__file__), "data", "surrogate_config5.npz")


def test_surrogate_loop_against_plain_loop():
    net0 = S.SurrogateNet.load(WEIGHTS, 32)
    param = S.SmoothDesign()
    z0 = param.start(range(30000, 30008))
    prob = S.FDTDDesignProblem(8)
    try:
        prob.value_and_grad(param.rho(z0))  # warm-up (graph capture)
        v0 = float(np.mean(prob.value(param.rho(z0))[0]))
        plain = S.plain_adjoint_loop(prob, param, z0, iters=200)
        assert plain["final"] > v0 + 0.3, (v0, plain["final"])
        target = plain["final"]
        goal = target - 0.01 * abs(target)
        plain_reach = next(t for t, _, v in plain["history"] if v >= goal)
        net = S.SurrogateNet(32, params=net0.params(), t_mean=net0.t_mean, t_std=net0.t_std)
        t0 = time.perf_counter()
        sur = S.surrogate_loop(prob, net, param, z0, iters=100_000, tuner=S.OnlineTuner(net),
                               target=target, wall_budget=plain["wall_s"])
        wall = time.perf_counter() - t0
    finally:
        prob.close()
    report = {"plain_final": round(target, 4), "plain_wall_s": round(plain["wall_s"], 2),
              "plain_reach_s": round(plain_reach, 2), "surrogate_final": round(sur["final"], 4),
              "surrogate_wall_s": round(wall, 2), "surrogate_reach_s": sur["reached_target_s"],
              "speedup_to_target": (round(plain_reach / sur["reached_target_s"], 2)
                                    if sur["reached_target_s"] else None),
              "surrogate_fdtd_gradients": sur["fdtd_gradients"],
              "surrogate_fdtd_verifications": sur["fdtd_verifications"],
              "surrogate_steps_kept": sur["surrogate_steps_kept"]}
    print("surrogate_vs_plain " + json.dumps(report))
    assert sur["reached_target_s"] is not None, report
