"""Build, train and evaluate the config-5 surrogate, and run the design loops.

    python -m photonfdtd_b200.surrogate_run --out DIR [--n-train 18000]
        [--n-heldout 2000] [--epochs 60] [--loops] [--weights PATH]

1. Densities rho from config-4's recipe with seeds 0 .. n_train-1 (training)
   and 18000 .. 18000+n_heldout-1 (held out).
2. Their transmission spectra from the FDTD engine: forward-only batches of
   the fixed 400 x 250 geometry, float32 for training, float64 for the
   held-out reference.
3. Training on the GPU with the library's own kernels (SurrogateNet).
4. Held-out error of the surrogate against the float64 FDTD spectra.
5. With --loops: the plain adjoint design loop and the surrogate-assisted one
   (verified by FDTD every 10th iteration, falling back to the adjoint when
   the surrogate's spectrum error exceeds 2 %) on 8 starting designs, and
   the wall-clock each needs to reach the plain loop's final objective.

Writes DIR/surrogate_weights.npz (BF16 weights) and DIR/surrogate_report.json.
With --weights, steps 1-3 are skipped and the given weights are used.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--out", required=True)
    p.add_argument("--n-train", type=int, default=18000)
    p.add_argument("--n-heldout", type=int, default=2000)
    p.add_argument("--epochs", type=int, default=60)
    p.add_argument("--batch", type=int, default=128)
    p.add_argument("--gen-batch", type=int, default=2000)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--loops", action="store_true")
    p.add_argument("--loop-iters", type=int, default=200)
    p.add_argument("--weights", default=None)
    p.add_argument("--wd", type=float, default=0.05)
    p.add_argument("--profile-steps", type=int, default=0,
                   help="only time this many training steps on random inputs (batch --batch)")
    p.add_argument("--gemm-engine", type=int, default=1, choices=(0, 1),
                   help="tensor-core GEMM engine: 1 tcgen05 (default), 0 mma.sync")
    p.add_argument("--gemm-shape", default=None,
                   help="M,N,K: only time pfs_gemm_bf16 at this shape (--reps calls)")
    p.add_argument("--reps", type=int, default=10)
    p.add_argument("--traj-designs", type=int, default=0,
                   help="add training pairs from plain adjoint trajectories of this many "
                        "designs (latent seeds 100000+)")
    p.add_argument("--traj-batch", type=int, default=64)
    p.add_argument("--traj-iters", type=int, default=100)
    p.add_argument("--traj-every", type=int, default=2)
    p.add_argument("--traj-heldout", type=int, default=0,
                   help="of the trajectory designs, this many (the last whole batches) are "
                        "held out for evaluation")
    p.add_argument("--loop-variants", default="1:1:1",
                   help="surrogate loops to run, comma-separated FALLBACK:BURST_LR_MULT:MAX_BURSTS")
    p.add_argument("--data", default=None,
                   help="npz of cached spectra (T_train, T_heldout); written if absent")
    a = p.parse_args(argv)
    import torch
    from . import surrogate as S
    os.makedirs(a.out, exist_ok=True)
    rep = {}
    from . import _native as N
    N.lib().pfs_gemm_engine(a.gemm_engine)
    if a.gemm_shape:
        M, Nn, K = (int(v) for v in a.gemm_shape.split(","))
        print(json.dumps({"gemm_engine": a.gemm_engine, "shape": [M, Nn, K],
                          "tflops": round(S.gemm_tflops(M, Nn, K, reps=a.reps), 1)}))
        return
    if a.profile_steps:
        out = {"batch": a.batch, "gemm_engine": a.gemm_engine,
               "train_step_ms": S.time_training_step(a.batch, a.profile_steps)}
        # the GEMM kernel alone: a square case and the largest forward layers
        for (M, Nn, K) in [(8192, 8192, 8192), (a.batch * 64, 256, 1152),
                           (a.batch * 16, 128, 2304)]:
            out[f"gemm_{M}x{Nn}x{K}_tflops"] = round(S.gemm_tflops(M, Nn, K), 1)
        print(json.dumps(out))
        return

    def say(msg):
        print(msg, flush=True)

    def gen_spectra(rho, precision):
        g = S.SpectrumGenerator(min(a.gen_batch, len(rho)), precision=precision)
        out = np.empty((len(rho), S.N_FREQ), np.complex128)
        t0 = time.perf_counter()
        for s0 in range(0, len(rho), g.n):
            out[s0:s0 + g.n] = g.spectra(rho[s0:s0 + g.n])
        wall = time.perf_counter() - t0
        cells = g.cells * ((len(rho) + g.n - 1) // g.n) + g.cells  # + the empty run
        g.close()
        return out, wall, cells

    t_all = time.perf_counter()
    rho_h = S.densities(range(18000, 18000 + a.n_heldout))
    rho_t = S.densities(range(a.n_train))
    if a.data and os.path.exists(a.data):
        z = np.load(a.data)
        T_t, T_h = z["T_train"][:a.n_train], z["T_heldout"][:a.n_heldout]
        rep["data"] = {"n_train": len(T_t), "n_heldout": len(T_h), "cached": True}
    else:
        T_t, wt, ct = gen_spectra(rho_t, "float32")
        say(f"training spectra: {len(rho_t)} designs float32 in {wt:.1f} s")
        T_h, wh, ch = gen_spectra(rho_h, "float64")
        say(f"held-out spectra: {len(rho_h)} designs float64 in {wh:.1f} s")
        rep["data"] = {"n_train": len(rho_t), "n_heldout": len(rho_h),
                       "train_gen_s": round(wt, 1), "heldout_gen_s": round(wh, 1),
                       "train_gcell_per_s": round(ct / wt / 1e9, 1),
                       "heldout_gcell_per_s_f64": round(ch / wh / 1e9, 1)}
        if a.data:
            np.savez_compressed(a.data, T_train=T_t, T_heldout=T_h)
    rho_jh = T_jh = None
    if a.traj_designs:
        B = a.traj_batch
        prob = S.FDTDDesignProblem(B)
        param = S.SmoothDesign()
        t0 = time.perf_counter()
        rj, Tj = S.trajectory_data(prob, param, list(range(100000, 100000 + a.traj_designs)),
                                   a.traj_iters, every=a.traj_every, log=say)
        prob.close()
        per_chunk = len(rj) // (a.traj_designs // B)
        nh = (a.traj_heldout // B) * per_chunk
        n_used = len(rj) - nh
        rho_jh, T_jh = rj[n_used:], Tj[n_used:]
        rho_t = np.concatenate([rho_t, rj[:n_used].astype(np.float64)])
        T_t = np.concatenate([T_t, Tj[:n_used]])
        rep["trajectories"] = {"designs": a.traj_designs, "batch": B, "iters": a.traj_iters,
                               "every": a.traj_every, "pairs_train": int(n_used),
                               "pairs_heldout": int(nh), "seeds": "100000+",
                               "wall_s": round(time.perf_counter() - t0, 1)}
        say("trajectory data: " + json.dumps(rep["trajectories"]))
    x = tg = None
    if a.weights is None:
        dev = "cuda"
        x = torch.from_numpy((2.0 * rho_t - 1.0).astype(np.float32)).to(dev)
        tri = np.stack([T_t.real, T_t.imag], axis=-1)
        t_mean, t_std = tri.mean(axis=0), tri.std(axis=0) + 1e-12
        rep["targets"] = {"std_over_designs_mean": float(t_std.mean()),
                          "mean_abs_T": float(np.abs(T_t).mean()),
                          "predict_mean_error": S.spectrum_errors(
                              np.broadcast_to(t_mean[:, 0] + 1j * t_mean[:, 1], T_h.shape), T_h)}
        tg = torch.from_numpy(((tri - t_mean) / t_std).astype(np.float32)).to(dev)
        net = S.SurrogateNet(a.batch, seed=0, t_mean=t_mean, t_std=t_std)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hist = S.train(net, x, tg, a.epochs, lr=a.lr, wd=a.wd, log=say)
        torch.cuda.synchronize()
        rep["training"] = {"epochs": a.epochs, "batch": a.batch, "lr": a.lr, "wd": a.wd,
                           "wall_s": round(time.perf_counter() - t0, 1),
                           "loss_first": hist[0], "loss_last": hist[-1]}
        net.save(os.path.join(a.out, "surrogate_weights.npz"))
        pred_t = net.predict(rho_t[:2000])
        rep["train_error_vs_f32"] = S.spectrum_errors(pred_t, T_t[:2000])
    else:
        net = S.SurrogateNet.load(a.weights, a.batch)
    pred_h = net.predict(rho_h)
    rep["heldout_error_vs_f64"] = S.spectrum_errors(pred_h, T_h)
    pe = S.power_error(pred_h, T_h)
    rep["heldout_power_error_vs_f64"] = {"mean": float(pe.mean()), "median": float(np.median(pe)),
                                         "p95": float(np.percentile(pe, 95)),
                                         "frac_below_2pct": float(np.mean(pe < 0.02))}
    say("held-out error: " + json.dumps(rep["heldout_error_vs_f64"]))
    if rho_jh is not None and len(rho_jh):
        pj = net.predict(rho_jh.astype(np.float64))
        rep["trajectory_heldout_error_vs_f32"] = S.spectrum_errors(pj, T_jh)
        pe = S.power_error(pj, T_jh)
        rep["trajectory_heldout_power_error"] = {"mean": float(pe.mean()),
                                                 "p95": float(np.percentile(pe, 95))}
        say("trajectory held-out error: " + json.dumps(rep["trajectory_heldout_error_vs_f32"]))
    say("held-out power error: " + json.dumps(rep["heldout_power_error_vs_f64"]))

    if a.loops:
        inf = S.SurrogateNet(32, params=net.params(), t_mean=net.t_mean, t_std=net.t_std)
        nd = 8
        param = S.SmoothDesign()
        z0 = param.start(range(30000, 30000 + nd))
        prob = S.FDTDDesignProblem(nd)
        prob.value_and_grad(param.rho(z0))  # warm-up (graph capture)
        plain = S.plain_adjoint_loop(prob, param, z0, iters=a.loop_iters)
        say(f"plain adjoint loop: objective {plain['final']:.4f} in {plain['wall_s']:.1f} s")
        goal = plain["final"] - 0.01 * abs(plain["final"])
        plain_reach = next((t for t, _, v in plain["history"] if v >= goal), plain["wall_s"])
        if x is None:
            x = torch.from_numpy((2.0 * rho_t - 1.0).astype(np.float32)).to("cuda")
            tri = np.stack([T_t.real, T_t.imag], axis=-1)
            tg = torch.from_numpy(((tri - net.t_mean) / net.t_std).astype(np.float32)).to("cuda")
        params0 = net.params()
        surs = []
        for spec in a.loop_variants.split(","):
            fb, mult, nb = spec.split(":")
            # every loop starts from the trained network (online tuning changes it)
            inf = S.SurrogateNet(32, params=params0, t_mean=net.t_mean, t_std=net.t_std)
            tuner = S.OnlineTuner(inf, x, tg)
            r = S.surrogate_loop(prob, inf, param, z0, iters=a.loop_iters, tuner=tuner,
                                 target=plain["final"], fallback_steps=int(fb),
                                 burst_lr=0.05 * float(mult), max_bursts=int(nb))
            r["variant"] = {"fallback_steps": int(fb), "burst_lr": 0.05 * float(mult),
                            "max_bursts": int(nb)}
            say(f"surrogate loop {spec}: objective {r['final']:.4f} in {r['wall_s']:.1f} s, "
                f"reached plain's objective (1 %) at {r['reached_target_s']}")
            surs.append(r)
        sur = min(surs, key=lambda r: (r["reached_target_s"] or float("inf"), -r["final"]))
        rep["design_loops"] = {
            "designs": nd, "iters": a.loop_iters, "objective": "band_objective",
            "plain": {"final": plain["final"], "wall_s": round(plain["wall_s"], 2),
                      "fdtd_gradients": plain["fdtd_gradients"],
                      "history": [(round(t, 3), i, v) for t, i, v in plain["history"][::10]]},
            "surrogate": {"final": sur["final"], "wall_s": round(sur["wall_s"], 2),
                          "reached_target_s": sur["reached_target_s"],
                          "fdtd_gradients": sur["fdtd_gradients"],
                          "fdtd_verifications": sur["fdtd_verifications"],
                          "bursts_rejected": sur["surrogate_bursts_rejected"],
                          "surrogate_steps_kept": sur["surrogate_steps_kept"],
                          "variant": sur["variant"], "log": sur["log"]},
            "surrogate_variants": [{**r["variant"], "final": r["final"],
                                    "wall_s": round(r["wall_s"], 2),
                                    "reached_target_s": r["reached_target_s"],
                                    "fdtd_gradients": r["fdtd_gradients"],
                                    "fdtd_verifications": r["fdtd_verifications"],
                                    "surrogate_steps_kept": r["surrogate_steps_kept"]}
                                   for r in surs],
            "plain_reached_target_s": plain_reach,
            "speedup_to_target": (round(plain_reach / sur["reached_target_s"], 2)
                                  if sur["reached_target_s"] and plain_reach else None)}
        prob.close()
    rep["total_s"] = round(time.perf_counter() - t_all, 1)
    with open(os.path.join(a.out, "surrogate_report.json"), "w") as f:
        json.dump(rep, f, indent=1)
    say(json.dumps({k: v for k, v in rep.items() if k != "design_loops"}))


if __name__ == "__main__":
    main()
