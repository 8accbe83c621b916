#!/usr/bin/env python
"""Benchmark of the B200 FDTD stepping engine.

Default workload (config 3): 384^3 cells at 10 nm with a 12-cell CPML, float32
fields, a Drude / two-pole Lorentz / eps 2.1 dielectric mix in 8^3 blocks
(ADE on about two thirds of the cells), an Ex Gaussian dipole, six
full-plane flux monitors and an Ex/Ey DFT monitor at 8 wavelengths, all
accumulated on the device every step. One step = one full Yee + CPML + ADE
time step of the whole domain with its sources and monitors. The stepping
state (about 6 GB) is far larger than L2, so no L2 flush is needed between
timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0). value = Mcell-updates/s of the whole job,
timed with CUDA events on the engine's stream (max over ranks). With N > 1
every rank steps its own replica of the workload (the single-domain path
does not shard; replicas only), so scaling is weak.

The line's "adjoint" object is the second half of the headline metric:
seconds per gradient iteration of the batched 2D TE inverse-design workload
(config 4: 256 uneven instances, 4000 steps, 64 x 64 design windows),
measured through photonfdtd_b200.batch.value_and_grad_eps (host design in,
host gradient out), with its forward / adjoint split and a CPU baseline of the
NumPy forward + adjoint restatement on one instance.

--impl reference times the reference's own CPU implementation of the same
workload: photonfdtd.Simulation(...).run() from the reference package
installed in baseline/_ref (baseline/refcpu.py), its vectorised NumPy path on
a bounded sample of full-domain steps, plus its Numba path (every core) on
the non-dispersive variant it accepts. Where the package is absent it falls
back to the NumPy restatement in oracle/ (kind "port").

Other objects of the line: "e2e" (config 3 run end to end through the
reference's own Simulation with backend="b200" from the plugin), "config2"
(the 536^3 subpixel workload, with its own roofline), "error_vs_f64" (the
float32 result against a float64 run of the same steps), "reference_gpu"
(the reference's CUDA kernels compiled for this GPU) and "surrogate".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-updates/s (3D Yee+CPML+ADE, fp32)"
UNIT = "Mcell-updates/s"
WORKLOAD = ("config3: 384^3 cells (12-cell CPML inside), dx 10 nm, float32, Drude / "
            "2-pole Lorentz / eps 2.1 media in 8^3 blocks, Ex dipole, 6 full-plane flux "
            "monitors + Ex/Ey DFT at 8 wavelengths accumulated every step")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=300)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=("b200", "reference"))
    p.add_argument("--kernel", default="auto", choices=("auto", "split", "fused"))
    p.add_argument("--size", type=int, default=384, help="cells per axis (default 384)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="skip timing the reference's own CUDA kernels on the plain variant")
    p.add_argument("--no-surrogate", action="store_true",
                   help="skip the surrogate tensor-core GEMM / training-step figures")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-adjoint3d", action="store_true",
                   help="skip the single-scene 3D gradient leg")
    p.add_argument("--no-mode", action="store_true", help="skip the mode-solver leg")
    p.add_argument("--no-batch3d", action="store_true", help="skip the concurrent-scenes leg")
    p.add_argument("--only-batch3d", action="store_true",
                   help="print only the concurrent-scenes leg")
    p.add_argument("--only-mode", action="store_true", help="print only the mode-solver leg")
    p.add_argument("--only-adjoint3d", action="store_true",
                   help="print only the single-scene 3D gradient leg")
    p.add_argument("--adjoint-iters", type=int, default=2)
    p.add_argument("--only-adjoint", action="store_true",
                   help="time the config-4 gradient iteration alone (profiling)")
    p.add_argument("--adjoint-instances", type=int, default=256)
    p.add_argument("--adjoint-steps", type=int, default=4000)
    p.add_argument("--no-numba", action="store_true",
                   help="reference arm: skip the reference's Numba point")
    p.add_argument("--no-config2", action="store_true",
                   help="skip the 536^3 subpixel workload leg")
    p.add_argument("--no-f64", action="store_true",
                   help="skip the float64 error statement")
    p.add_argument("--e2e-steps", type=int, default=3000,
                   help="steps of the end-to-end Simulation.run() (config 3 runs 3000)")
    return p.parse_args()


def make_sim(pf, size, n_steps):
    from photonfdtd_b200 import workloads as W
    return W.config3(pf, n_total=size, block=8, n_steps=n_steps)


# --------------------------------------------------------------------------- #
# Algorithmic bytes per cell-update (compulsory traffic of one unblocked step):
# 6 fields read + written, one ce per cell, 1 B material id, each CPML psi
# element read + written, each ADE pole's P^n, P^{n-1} (3 components) read
# and written: 48 B per pole in float32.
# --------------------------------------------------------------------------- #
def algorithmic_bytes(t) -> dict:
    s = np.dtype(t["npdt"]).itemsize
    shape = t["shape"]
    ncell = int(np.prod(shape))
    n_psi = 0
    curl = {"Hx": ((1, 2)), "Hy": ((2, 0)), "Hz": ((0, 1)),
            "Ex": ((1, 2)), "Ey": ((2, 0)), "Ez": ((0, 1))}
    for comp, axes in curl.items():
        is_e = comp[0] == "E"
        ext = []
        for a in range(3):
            n = shape[a]
            ext.append(n - 1 if (a in axes and n > 1) else n)
        for ax in axes:
            if shape[ax] <= 1:
                continue
            c = t["cpml"][ax][1] if is_e else t["cpml"][ax][3]
            c = c[1:] if is_e else c[:-1]
            others = [ext[a] for a in range(3) if a != ax]
            n_psi += int((c != 0).sum()) * others[0] * others[1]
    poles = 0.0
    if t["ade"] is not None:
        poles = float((t["ade"]["count"] * t["ade"]["npole"]).sum()) / ncell
    n_ce = 3 if t["ce_mode"] == 1 else 1
    per_cell = 6 * 2 * s + n_ce * s + n_psi / ncell * 2 * s
    if t["ade"] is not None:
        per_cell += 1 + poles * 3 * 2 * 2 * s
    return dict(per_cell=per_cell, n_psi=n_psi, poles_per_cell=poles, ncell=ncell)


# --------------------------------------------------------------------------- #
class ClockSampler:
    """nvidia-smi SM clock and throttle reasons while the timed region runs."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """The largest of every rank's x (every rank calls it, in the same order);
    x itself without a process group."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, cells: int, steps: int, ms: float) -> float:
    """Whole-job Mcell-updates/s: world replicas of `cells` cells advanced
    `steps` steps in `ms` milliseconds (the slowest rank's time)."""
    return world * cells * steps / (ms / 1e3) / 1e6


def bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured (burst)"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def surrogate_bench():
    """The surrogate's tensor-core GEMM (tcgen05, TMEM accumulator) against
    the measured bf16 peak, on a square case and on the network's largest
    layer (batch 128), plus one training step of the network."""
    from photonfdtd_b200 import surrogate as S
    peak, kind = bf16_peak()
    sq = S.gemm_tflops(8192, 8192, 8192, reps=10)
    layer = S.gemm_tflops(128 * 64, 256, 1152, reps=50)
    return {"kernel": "k_gemm_tc (tcgen05.mma kind::f16, TMA 128B-swizzle ring, TMEM accumulator)",
            "roofline": {"bound": "tensor", "achieved": round(sq, 1), "peak": peak,
                         "unit": "TFLOP/s", "frac": round(sq / peak, 4), "peak_source": kind,
                         "shape": "8192x8192x8192 bf16 -> f32"},
            "largest_layer_tflops": round(layer, 1),
            "largest_layer_shape": "8192x256x1152 (conv4 forward: 3x3 stride 2, 128 -> 256 channels, 8x8 output, batch 128)",
            "train_step_ms": round(S.time_training_step(128, 20), 3), "train_batch": 128}


def reference_gpu_bench(size: int, steps: int = 100, warmup: int = 5):
    """The reference's own CUDA stepping kernels (rust/src/cuda.rs:29-265,
    compiled for sm_100a by baseline/refcuda/build.py) against this engine on
    the workload they can both run: the config-3 grid and media blocks with
    non-dispersive media (eps 1.0 / 4.0 / 2.1), float32, no monitors. Both
    timed by CUDA events on their own streams; `agreement` is the relative L2
    difference of the final Ex."""
    import torch
    from baseline import refcuda
    if not refcuda.available("float32"):
        return {"unavailable": "baseline/_ref/librefcuda_f32.so not built"}
    import photonfdtd_b200 as pf
    from photonfdtd_b200 import workloads as W
    from photonfdtd_b200.engine import B200Engine, build_tables
    sim = W.config3(pf, n_total=size, n_steps=warmup + steps, flux=False, dft=False,
                    dispersive=False)
    cells = size ** 3
    eng = B200Engine(build_tables(sim))
    st = torch.cuda.ExternalStream(eng.stream())
    eng.advance(0, warmup)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    eng.advance(warmup, steps)
    e1.record(st)
    torch.cuda.synchronize()
    ours_ms = e0.elapsed_time(e1)
    ex = eng.get("Ex").astype(np.float64)
    eng.close()
    ref = refcuda.RefCuda(sim)
    try:
        ref.run(0, warmup)
        ref_ms = ref.run(warmup, steps, timed=True)
        rx = ref.field("Ex").astype(np.float64)
    finally:
        ref.close()
    return {"workload": f"config3 grid {size}^3, media eps 1.0/4.0/2.1 in 8^3 blocks "
                        "(no ADE), Yee+CPML float32, Ex dipole, no monitors",
            "steps": steps, "unit": "Mcell-updates/s",
            "reference_kernels": round(cells * steps / (ref_ms / 1e3) / 1e6, 1),
            "reference_kernels_ms_per_step": round(ref_ms / steps, 4),
            "b200_engine": round(cells * steps / (ours_ms / 1e3) / 1e6, 1),
            "b200_engine_ms_per_step": round(ours_ms / steps, 4),
            "agreement_ex_rel_l2": float(np.linalg.norm(ex - rx) / np.linalg.norm(rx)),
            "source": "reference rust/src/cuda.rs update_h / update_e / inject, nvcc "
                      "sm_100a, launched as Inner::run_steps (1024-thread blocks)"}


def traffic_record(kernel_kind):
    """DRAM bytes per step of the step kernels from a committed ncu summary,
    if one exists for this workload (profiles/traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel_kind)
    except (OSError, ValueError):
        return None


# --------------------------------------------------------------------------- #
def cpu_baseline(size, steps=2):
    """The reference's own NumPy path (baseline/refcpu.py) on `steps` timed
    full-domain steps of the workload, one core (NumPy ufuncs are
    single-threaded); the oracle port where the reference is not installed."""
    from baseline import locate
    if locate.installed():
        from baseline import refcpu
        out = refcpu.numpy_config3(size, steps=steps)
        out.pop("s_per_step", None)
        return out
    return cpu_baseline_port(size, steps)


def cpu_baseline_port(size, steps=2):
    """The oracle (NumPy restatement of the reference CPU path) on full-domain
    steps of the same workload; one core (NumPy ufuncs are single-threaded)."""
    import photonfdtd_b200 as pf
    from oracle import OracleRun
    sim = make_sim(pf, size, 3000)
    run = OracleRun(sim)
    run.advance(1)  # warm-up: first-touch allocations
    t0 = time.perf_counter()
    run.advance(steps)
    wall = time.perf_counter() - t0
    ncell = int(np.prod(run.shape))
    return {"value": ncell * steps / wall / 1e6, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{steps} full-domain steps of the {size}^3 workload after 1 warm-up step "
                      f"({wall:.1f} s), oracle/fdtd_oracle.py (NumPy)"}


def run_reference(args):
    """--impl reference: rank 0 times the reference's CPU implementation;
    other ranks idle. Each timed step is one full-domain step of the
    workload, bounded to 3 timed steps (about 9 s each on one core)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    k = max(1, min(args.steps, 3))
    base = cpu_baseline(args.size, steps=k)
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": k, "warmup": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": args.size ** 3},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    from baseline import locate
    if locate.installed() and not args.no_numba:
        from baseline import refcpu
        try:
            line["numba"] = refcpu.numba_config3_plain(args.size, steps=k)
        except Exception as exc:  # noqa: BLE001 - reported, not fatal
            line["numba"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- #
def e2e_bench(size: int, steps: int, world: int, dist) -> dict:
    """Config 3 end to end through the call a user makes: the reference's
    own photonfdtd.Simulation with backend="b200" (photonfdtd_b200.plugin),
    scene on the host, Result back on the host; wall clock around run(),
    which builds the tables, creates the engine (device memory, table upload),
    steps, and reads the DFT and flux back. Falls back to this package's own
    Simulation when the reference is not installed."""
    import torch
    import photonfdtd_b200 as pf
    from photonfdtd_b200 import engine as E, plugin, workloads as W
    from baseline.locate import import_reference
    ref = import_reference()
    if ref is not None:
        plugin.install(ref)
        sim = W.config3(ref, n_total=size, n_steps=steps, union_blocks=True, backend="b200")
        api = "photonfdtd.Simulation(..., backend='b200').run() (reference package + plugin)"
    else:
        sim = W.config3(pf, n_total=size, n_steps=steps, union_blocks=True)
        api = "photonfdtd_b200.Simulation(...).run()"
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        t0 = time.perf_counter()
        res = sim.run()
        wall = time.perf_counter() - t0
    st = dict(E.LAST_RUN)
    if not (len(res.flux) == 6 and "d" in res.dft and np.isfinite(list(res.flux.values())).all()):
        raise RuntimeError("e2e: Simulation.run() returned an incomplete Result")
    wall = max_over_ranks(wall, dist)
    return {"value": round(job_rate(world, size ** 3, steps, wall * 1e3), 2), "unit": UNIT,
            "h2d_bytes_per_step": int(st["h2d_bytes"] / steps),
            "d2h_bytes_per_step": int(st["d2h_bytes"] / steps),
            "steps": steps, "wall_s": round(wall, 3),
            "phases_s": {"tables": round(st["tables_s"], 3), "engine": round(st["create_s"], 3),
                         "steps": round(st["advance_s"], 3),
                         "steps_and_readback": round(st["run_s"], 3)},
            "clocks": clk.summary(),
            "what": f"{api}: config 3 at {size}^3 for {steps} steps, host scene in, "
                    "Result (DFT + flux) out, wall clock"}


def config2_bench(steps: int, warmup: int, world: int, dist) -> dict:
    """Config 2: 536^3 cells, 64 boxes with subpixel smoothing (three per-cell
    coefficient arrays), the Ex dipole and a 16-wavelength Ex/Ey/Hx/Hy DFT on
    the z = 0 plane every step. The subpixel precompute runs on the GPU and is
    timed separately."""
    import torch
    import photonfdtd_b200 as pf
    from photonfdtd_b200 import workloads as W
    from photonfdtd_b200.engine import B200Engine, build_tables
    from photonfdtd_b200.smoothing import smooth_permittivity_device
    sim = W.config2(pf, n_steps=warmup + 2 * steps + 8)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    smooth_permittivity_device(sim.grid, sim.structures, background_eps=1.0,
                               factor=sim.subpixel_factor, dtype=np.float32)
    smooth_s = time.perf_counter() - t0
    t = build_tables(sim)
    alg = algorithmic_bytes(t)
    eng = B200Engine(t)
    try:
        st = torch.cuda.ExternalStream(eng.stream())
        eng.advance(0, warmup)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        eng.advance(warmup, steps)
        e1.record(st)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), dist)
        eng.set_profiling(True)
        eng.advance(warmup + steps, steps)
        _, pms = eng.read_profile(reset=True)
        eng.set_profiling(False)
    finally:
        eng.close()
    step_ms = pms[0] / steps
    peak, kind = peaks()
    achieved = alg["per_cell"] * alg["ncell"] / (step_ms / 1e3) / 1e9
    return {"workload": "config2: 536^3 cells (512^3 interior + 12-cell CPML) at 20 nm, "
                        "float32, 64 seeded boxes eps U[1, 12.1], subpixel smoothing "
                        "(factor 3, diagonal tensor: 3 coefficient arrays), Ex dipole, "
                        "16-wavelength Ex/Ey/Hx/Hy DFT on the z = 0 plane every step",
            "cells": alg["ncell"], "steps": steps,
            "value": round(job_rate(world, alg["ncell"], steps, ms), 2), "unit": UNIT,
            "ms_per_step": round(ms / steps, 4),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_source": kind, "step_kernels_ms_per_step": round(step_ms, 4),
                         "algorithmic_bytes_per_cell": round(alg["per_cell"], 2)},
            "dft_ms_per_step": round((pms[2] + pms[3]) / steps, 4),
            "smoothing_s": round(smooth_s, 3)}


def f64_error_bench(sim, t, steps: int = 1000) -> dict:
    """The float32 step's error against float64, two ways:
    replica: the reduced config-3 scene (64^3, the full 3000 steps) against
    the reference's own float64 NumPy run (tests/golden/ade3d_f64.npz);
    full_size: the benchmark workload, `steps` steps in float32 against the
    same steps of the engine's float64 path (within 1e-12 of NumPy float64 on
    every golden scene)."""
    import photonfdtd_b200 as pf
    from photonfdtd_b200 import accuracy as A
    from photonfdtd_b200 import workloads as W
    from photonfdtd_b200.engine import B200Engine, build_tables
    out = {}
    gpath = os.path.join(ROOT, "tests", "golden", "ade3d_f64.npz")
    if os.path.exists(gpath):
        g = np.load(gpath)
        rsim = W.config3(pf, n_total=64, block=8, n_steps=3000)
        rsim.add_monitor(pf.FieldMonitor(name="mid", components=("Ex", "Ey", "Ez", "Hx", "Hy",
                                                                 "Hz"), plane_z=0.0,
                                         times=[1000 * rsim.dt, 2999 * rsim.dt]))
        res = rsim.run()
        worst = {"rel_max": 0.0, "rel_l2": 0.0}
        for k in g.files:
            if k.startswith("f/"):
                _, mon, c = k.split("/")
                a = np.asarray(res.fields[mon][c])
            elif k.startswith("dft/"):
                _, mon, c = k.split("/")
                a = np.asarray(res.dft[mon][c])
            else:
                continue
            e = A._pair(a, g[k])
            worst = {q: max(worst[q], e[q]) for q in worst}
        out["replica"] = {"scene": "config-3 recipe at 64^3, 3000 steps, float32, against the "
                                   "reference's float64 NumPy run (tests/golden/ade3d_f64.npz)",
                          **{q: float(f"{v:.3e}") for q, v in worst.items()}}
    e32 = B200Engine(t)
    e64 = B200Engine(build_tables(sim, np.float64))
    try:
        e32.advance(0, steps)
        e64.advance(0, steps)
        worst = {"rel_max": 0.0, "rel_l2": 0.0}
        for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            e = A._pair(e32.get(c), e64.get(c))
            worst = {q: max(worst[q], e[q]) for q in worst}
        for k, d in enumerate(t["dft"]):
            for c in d["m"].components:
                e = A._pair(e32.read_dft(k, c, d["omega"].size, d["counts"]),
                            e64.read_dft(k, c, d["omega"].size, d["counts"]))
                worst = {q: max(worst[q], e[q]) for q in worst}
        fl = max(A._pair([e32.read_flux(k)], [e64.read_flux(k)])["rel_max"]
                 for k in range(len(t["flux"])))
    finally:
        e32.close()
        e64.close()
    out["full_size"] = {"scene": f"the benchmark workload, {steps} steps, float32 against the "
                                 "engine's float64 path (fields and DFT)",
                        **{q: float(f"{v:.3e}") for q, v in worst.items()},
                        "flux_rel": float(f"{fl:.3e}")}
    return out


# --------------------------------------------------------------------------- #
ADJ_WORKLOAD = ("config4: 256 2D TE instances, nx ~U{200..800} x ny ~U{150..400} at 20 nm "
                "(12-cell CPML), float32, 64x64 design window each, Ey line source, Ey DFT at "
                "8 wavelengths on the output line, 4000 steps forward + discrete adjoint")


def adjoint_bench(iters: int, cpu: bool, n_inst: int = 256, n_steps: int = 4000):
    """Seconds per gradient iteration of the config-4 batch: set the design,
    forward, read the line DFT, cotangent of J = sum |F|^2, adjoint, read
    dJ/deps - one value_and_grad_eps call, wall clock on the host."""
    import photonfdtd_b200 as pf
    from photonfdtd_b200 import workloads as W
    from photonfdtd_b200.batch import BatchTE, value_and_grad_eps
    sizes = W.config4_sizes()[:n_inst]
    sims = [W.config4_instance(pf, nx, ny, i=k, n_steps=n_steps) for k, (nx, ny) in enumerate(sizes)]
    wins = [W.design_window_box(nx, ny, 64) for nx, ny in sizes]
    t0 = time.perf_counter()
    b = BatchTE(sims, wins)
    setup = time.perf_counter() - t0
    eps = b.design_eps()
    value_and_grad_eps(b, eps)  # warm-up: graph capture
    l0 = b.info()["launches"]
    times, fwd, adj = [], [], []
    for _ in range(iters):
        t0 = time.perf_counter()
        vals, grad = value_and_grad_eps(b, eps)
        times.append(time.perf_counter() - t0)
        t1 = time.perf_counter()
        F = b.forward()
        t2 = time.perf_counter()
        b.adjoint(2.0 * F)
        t3 = time.perf_counter()
        fwd.append(t2 - t1)
        adj.append(t3 - t2)
    info = b.info()
    launches = (info["launches"] - l0) // (2 * iters)
    cells = b.ncell * b.n_steps
    # algorithmic bytes per cell-step: Ex, Ey, Hz read + written and ce read
    # (28 B in float32) plus each CPML psi entry read + written; the adjoint
    # moves the same for its adjoint fields and psi, plus the stored
    # design-window curls (2 reals per design cell per step)
    from photonfdtd_b200.batch import psi_cells
    s_b = np.dtype(b.npdt).itemsize
    psi = sum(psi_cells(tb) for tb in b.tabs)
    fwd_bytes = (7 * s_b * b.ncell + 2 * s_b * psi) * b.n_steps
    adj_bytes = fwd_bytes + 2 * s_b * b.n_design * b.n_steps
    peak, pkind = peaks()
    out = {"metric": "adjoint grad s/iter (256-instance batch)", "value": round(min(times), 3),
           "unit": "s/iter", "higher_is_better": False, "iters": iters,
           "workload": ADJ_WORKLOAD, "cells": b.ncell, "steps": b.n_steps,
           "forward_s": round(min(fwd), 3), "adjoint_s": round(min(adj), 3),
           "forward_gcell_per_s": round(cells / min(fwd) / 1e9, 2),
           "roofline": {
               "bound": "hbm", "unit": "GB/s", "peak": peak, "peak_source": pkind,
               "forward": {"achieved": round(fwd_bytes / min(fwd) / 1e9, 1),
                           "frac": round(fwd_bytes / min(fwd) / 1e9 / peak, 4),
                           "bytes_per_cell_step": round(fwd_bytes / cells, 2)},
               "adjoint": {"achieved": round(adj_bytes / min(adj) / 1e9, 1),
                           "frac": round(adj_bytes / min(adj) / 1e9 / peak, 4),
                           "bytes_per_cell_step": round(adj_bytes / cells, 2)}},
           "checkpoint_every": info["checkpoint_every"], "segments": info["segments"],
           "fused_steps": bool(info["fused"]), "tile_rows": b.tile_rows,
           "tile_ms_per_step": b.tile_ms_per_step,
           "setup_s": round(setup, 2), "gpu_launches_per_iter": int(launches),
           "objective_sum": float(np.sum(vals)), "grad_max": float(np.max(np.abs(grad)))}
    b.close()
    if cpu:
        out["cpu_baseline"] = adjoint_cpu_baseline(sims[0], wins[0], cells)
    return out


def adjoint3d_bench(n: int = 192, n_steps: int = 2000) -> dict:
    """value_and_grad_eps of one 3D scene (photonfdtd_b200.adjoint): n^3
    cells at 20 nm with a 12-cell CPML, float32, four dielectric boxes, an Ex
    dipole, an Ex / Ey DFT on the z = 0 plane at 4 wavelengths, J = sum |DFT|^2.
    Times the forward run alone (the faster of two runs) and the full
    gradient (forward with checkpoints, then per segment a replay and the
    reverse steps), wall clock around synchronised calls, both from the
    host scene (tables and engine creation included)."""
    import time
    import torch
    import photonfdtd_b200 as pf
    from photonfdtd_b200.adjoint import value_and_grad_eps
    from photonfdtd_b200.engine import run_b200
    d = 20e-9
    L = n * d
    grid = pf.Grid(size=(L, L, L), cell_size=d, pml_layers=(12, 12, 12))
    boxes = [pf.Box(center=(cx * L, cy * L, 0.0), size=(0.12 * L, 0.1 * L, 0.3 * L),
                    medium=pf.Medium(permittivity=ep))
             for cx, cy, ep in ((0.1, 0.05, 4.0), (-0.12, 0.1, 2.25), (0.05, -0.15, 6.0),
                                (-0.05, -0.05, 3.0))]
    f0 = 299_792_458.0 / 0.8e-6
    src = pf.PointDipole(position=(-0.25 * L, 0.0, 0.0), component="Ex",
                         waveform=pf.GaussianPulse(freq0=f0, fwhm=4e-15))
    dft = pf.DFTMonitor(name="d", components=("Ex", "Ey"),
                        freqs=list(f0 * np.array([0.9, 1.0, 1.1, 1.2])),
                        plane_axis="z", plane_position=0.0)
    dt = pf.Simulation(grid, structures=boxes, sources=[src], monitors=[dft],
                       run_time=1e-15, precision="float32").dt
    sim = pf.Simulation(grid, structures=boxes, sources=[src], monitors=[dft],
                        run_time=(n_steps - 0.5) * dt, precision="float32")

    def loss(out):
        return sum((v.abs() ** 2).sum() for v in out["dft"]["d"].values())

    run_b200(sim)  # warm-up (tables, module load)
    t_fwd = float("inf")
    for _ in range(2):  # the faster of two forward runs
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run_b200(sim)
        torch.cuda.synchronize()
        t_fwd = min(t_fwd, time.perf_counter() - t0)
    t0 = time.perf_counter()
    val, g = value_and_grad_eps(sim, loss)
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    cells = n ** 3
    return {"workload": f"{n}^3 cells (12-cell CPML) at 20 nm, float32, 4 dielectric boxes, Ex "
                        f"dipole, Ex/Ey DFT on z = 0 at 4 wavelengths, {int(sim.n_steps)} steps, "
                        "J = sum |DFT|^2",
            "cells": cells, "steps": int(sim.n_steps),
            "checkpoint_every": int(np.ceil(np.sqrt(sim.n_steps))),
            "forward_s": round(t_fwd, 3), "value_and_grad_s": round(t_grad, 3),
            "grad_over_forward": round(t_grad / t_fwd, 2),
            "reverse_mcell_steps_per_s": round(cells * sim.n_steps / max(t_grad - t_fwd, 1e-9)
                                               / 1e6, 1),
            "finite": bool(np.isfinite(g).all()), "value": float(val)}


def mode_bench() -> dict:
    """The GPU mode solver (photonfdtd_b200.mode) against the reference's
    scipy ARPACK solver (baseline/_ref) on the reference's high-contrast
    acceptance case: a 0.3 um n = 3 slab in air, 8 um x 2 um cross-section at
    0.1 x 0.01 um (80 x 200 cells, 32,000 unknowns), 26 modes at 1.55 um."""
    import time
    import torch
    import photonfdtd_b200 as pf
    from photonfdtd_b200.mode import ModeSolver

    def build(mod):
        m = mod or pf
        core = m.Box(center=(0.0, 0.0), size=(24e-6, 0.3e-6), medium=m.Medium.from_index(3.0))
        kw = dict(size=(8e-6, 2e-6), cell_size=(0.1e-6, 0.01e-6), structures=[core],
                  wavelength=1.55e-6, background_eps=1.0, num_modes=26)
        return mod.ModeSolver(**kw) if mod is not None else ModeSolver(**kw)

    build(None).solve()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = build(None).solve()
    torch.cuda.synchronize()
    t_gpu = time.perf_counter() - t0
    out = {"workload": "26 modes of a 0.3 um n=3 slab, 80 x 200 cells (32,000 unknowns)",
           "gpu_s": round(t_gpu, 3), "iterations": int(res.iterations),
           "max_residual": float(res.max_residual)}
    try:
        from baseline.locate import import_reference
        ref = import_reference()
    except Exception:  # noqa: BLE001
        ref = None
    if ref is not None:
        t0 = time.perf_counter()
        rres = build(ref).solve()
        out["reference_cpu_s"] = round(time.perf_counter() - t0, 3)
        out["n_eff_max_rel_diff"] = float(np.max(np.abs(res.n_eff - rres.n_eff) / rres.n_eff))
    return out


def batch3d_bench(n_scenes: int = 24, n_steps: int = 600) -> dict:
    """Many small uneven 3D scenes on one GPU (photonfdtd_b200.batch3d):
    n_scenes grids of 40^3 to 96^3 cells (seeded sizes, 8-cell CPML, two
    dielectric boxes, an Ez dipole, an Ez DFT plane at 2 wavelengths),
    float32, n_steps steps each, from host scenes to Results: one after
    another (run_b200 each) against all at once (run_many), wall clock, the
    better of two runs of each."""
    import time
    import torch
    import photonfdtd_b200 as pf
    from photonfdtd_b200.batch3d import run_many
    from photonfdtd_b200.engine import run_b200
    rng = np.random.default_rng(11)
    d, f0 = 40e-9, 299_792_458.0 / 1.2e-6

    def scene(n):
        L = n * d
        grid = pf.Grid(size=(L, L, L), cell_size=d, pml_layers=(8, 8, 8))
        boxes = [pf.Box(center=(0.1 * L, 0.0, 0.0), size=(0.2 * L, 0.3 * L, 0.3 * L),
                        medium=pf.Medium(permittivity=4.0)),
                 pf.Box(center=(-0.1 * L, 0.1 * L, 0.0), size=(0.1 * L, 0.2 * L, 0.4 * L),
                        medium=pf.Medium(permittivity=2.25))]
        src = pf.PointDipole(position=(-0.25 * L, 0.0, 0.0), component="Ez",
                             waveform=pf.GaussianPulse(freq0=f0, fwhm=4e-15))
        mon = pf.DFTMonitor(name="d", components=("Ez",), freqs=[f0, 1.2 * f0],
                            plane_axis="z", plane_position=0.0)
        dt = pf.Simulation(grid, structures=boxes, sources=[src], monitors=[mon],
                           run_time=1e-15).dt
        return pf.Simulation(grid, structures=boxes, sources=[src], monitors=[mon],
                             run_time=(n_steps - 0.5) * dt)

    sizes = [int(v) for v in rng.integers(40, 97, n_scenes)]
    cells = sum(n ** 3 for n in sizes) * n_steps
    run_many([scene(n) for n in sizes[:2]])  # warm-up
    t_seq = t_con = float("inf")
    for _ in range(2):  # the better of two runs of each
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for n in sizes:
            run_b200(scene(n))
        torch.cuda.synchronize()
        t_seq = min(t_seq, time.perf_counter() - t0)
        t0 = time.perf_counter()
        run_many([scene(n) for n in sizes])
        torch.cuda.synchronize()
        t_con = min(t_con, time.perf_counter() - t0)
    return {"workload": f"{n_scenes} 3D scenes of 40^3-96^3 cells (seeded), float32, "
                        f"{n_steps} steps each, host scene to Result",
            "cell_steps": cells, "sequential_s": round(t_seq, 3),
            "concurrent_s": round(t_con, 3), "speedup": round(t_seq / t_con, 2),
            "concurrent_mcell_updates_per_s": round(cells / t_con / 1e6, 1)}


def adjoint_cpu_baseline(sim, win, cells_total, steps=60):
    """The NumPy forward + adjoint restatement (oracle/adjoint2d.py) on the
    first instance for `steps` steps, scaled by cell-steps to the batch."""
    from oracle.adjoint2d import TEAdjointRun, objective_cotangent
    run = TEAdjointRun(sim, win, n_steps=steps)
    t0 = time.perf_counter()
    F = run.forward()
    run.adjoint(objective_cotangent(F))
    wall = time.perf_counter() - t0
    rate = run.nx * run.ny * steps / wall
    return {"value": round(cells_total / rate, 1), "unit": "s/iter", "cores": 1, "kind": "port",
            "sample": f"instance 0 ({run.nx}x{run.ny}), {steps} steps forward + adjoint in "
                      f"{wall:.1f} s, scaled by cell-steps to the 256-instance, 4000-step batch"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.only_batch3d:
        print(json.dumps(batch3d_bench()), flush=True)
        return
    if args.only_mode:
        print(json.dumps(mode_bench()), flush=True)
        return
    if args.only_adjoint3d:
        print(json.dumps(adjoint3d_bench()), flush=True)
        return
    if args.only_adjoint:
        adj = adjoint_bench(max(1, args.adjoint_iters), False, args.adjoint_instances,
                            args.adjoint_steps)
        print(json.dumps(adj), flush=True)
        return
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import photonfdtd_b200 as pf
    from photonfdtd_b200 import _native as N
    from photonfdtd_b200.engine import B200Engine, build_tables

    kern = {"auto": N.PF_KERNEL_AUTO, "split": N.PF_KERNEL_SPLIT,
            "fused": N.PF_KERNEL_FUSED}[args.kernel]
    n_total = max(3000, args.warmup + 2 * args.steps + 8)
    sim = make_sim(pf, args.size, n_total)
    t = build_tables(sim)
    alg = algorithmic_bytes(t)
    eng = B200Engine(t, kernel=kern)
    stream = torch.cuda.ExternalStream(eng.stream())

    # warm-up, then K timed steps bracketed by barrier + synchronize
    eng.advance(0, args.warmup)
    pos = args.warmup
    eng.read_profile(reset=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        eng.advance(pos, args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    pos += args.steps
    ms = ev0.elapsed_time(ev1)
    launches, _ = eng.read_profile(reset=True)
    ms = max_over_ranks(ms, dist)
    if dist is not None:
        dist.barrier()
    value = job_rate(world, alg["ncell"], args.steps, ms)

    # roofline of the step kernels: a second pass with per-launch events
    eng.set_profiling(True)
    kp = min(args.steps, 100)
    eng.advance(pos, kp)
    pos += kp
    plaunch, pms = eng.read_profile(reset=True)
    eng.set_profiling(False)
    step_ms = pms[0] / kp
    peak, peak_kind = peaks()
    achieved = alg["per_cell"] * alg["ncell"] / (step_ms / 1e3) / 1e9
    kind = "fused" if t["shape"][2] > 1 and plaunch[0] == kp else "split_h+e"
    tr = traffic_record(f"config3_{args.size}_{kind}")
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": tr,
            "peak_source": peak_kind,
            "kernel": ("fused H+E step" if kind == "fused" else "split H and E passes") +
                      f", {plaunch[0] // kp} launch(es) per step",
            "step_kernels_ms_per_step": round(step_ms, 4),
            "algorithmic_bytes_per_cell": round(alg["per_cell"], 2),
            "monitor_ms_per_step": round((pms[1] + pms[2] + pms[3]) / kp, 4)}

    eng.close()
    err64 = None
    if not args.no_f64:
        err64 = f64_error_bench(sim, t)

    # end to end through the public API with host data: the reference's own
    # Simulation (backend="b200" through the plugin) for config 3's steps
    e2e = None
    if not args.no_e2e:
        e2e = e2e_bench(args.size, args.e2e_steps, world, dist)

    line = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": alg["ncell"], "grid": list(t["shape"]),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "state ~6 GB > 126 MB L2: inputs larger than L2, no flush"},
            "roofline": roof, "e2e": e2e, "gpu_launches": int(sum(launches)),
            "clocks": clk.summary()}
    if err64 is not None:
        line["error_vs_f64"] = err64
    if not args.no_config2:
        line["config2"] = config2_bench(min(args.steps, 20), 3, world, dist)
    if not args.no_adjoint:
        adj = adjoint_bench(max(1, args.adjoint_iters), rank == 0 and world == 1 and
                            not args.no_cpu_baseline)
        if dist is not None:
            adj["value"] = round(max_over_ranks(adj["value"], dist), 3)
            adj["scaling"] = "weak (one batch per rank)"
        line["adjoint"] = adj
    if rank == 0 and world == 1 and not args.no_adjoint3d:
        line["adjoint3d"] = adjoint3d_bench()
    if rank == 0 and world == 1 and not args.no_batch3d:
        line["batch3d"] = batch3d_bench()
    if rank == 0 and world == 1 and not args.no_mode:
        line["mode_solver"] = mode_bench()
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_bench(args.size)
    if rank == 0 and world == 1 and not args.no_surrogate:
        line["surrogate"] = surrogate_bench()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.size)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
