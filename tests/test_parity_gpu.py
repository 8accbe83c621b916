"""GPU engine parity: the b200 backend against the reference and the oracle.

For every golden scene the engine's Result is compared
  * against the reference's own run (tests/golden): float64 to 1e-12 of the
    largest value (the reference's Rust/CUDA bar, tests/test_rust.py:37-47),
    float32 to 1e-5 relative L2 (the engine's stated float32 tolerance);
  * against the CPU oracle run on this machine: fields and DFT bit for bit
    (the kernels keep the reference's rounding sequence), flux to 1e-6 of the
    scene's flux scale (the engine sums planes in float64, the reference in
    pairwise float32).
"""
import numpy as np
import pytest

import photonfdtd_b200 as pf
import scenes
from golden_util import compare

pytestmark = pytest.mark.gpu

# the engine-vs-oracle comparison reruns the scene in NumPy on the host:
# the 3000-step ADE scenes and the 120^3 config-2 replicas take minutes there
SLOW = ("ade3d_f32", "ade3d_f64", "c2rep_f32", "c2rep_f64")
FAST = [n for n in scenes.SCENES if n not in SLOW]


def _tol(name):
    return (1e-12, 1e-12) if name.endswith("f64") or name == "config1" else (None, 1e-5)


@pytest.mark.parametrize("name", list(scenes.SCENES))
def test_engine_matches_reference(name):
    sim = scenes.build(name, pf)
    res = sim.run()
    tmax, tl2 = _tol(name)
    worst = (0.0, 0.0)
    for k, (rmax, rl2) in compare(res, name).items():
        if k.startswith("flux/"):
            assert rl2 < 1e-5, f"{name} {k}: flux differs by {rl2:.3e}"
            continue
        if tmax is not None:
            assert rmax <= tmax, f"{name} {k}: max rel {rmax:.3e}"
        assert rl2 <= tl2, f"{name} {k}: rel L2 {rl2:.3e}"
        worst = max(worst, (rmax, rl2))
    print(f"{name}: worst field/DFT rel max {worst[0]:.2e}, rel L2 {worst[1]:.2e}")


@pytest.mark.parametrize("name", FAST)
def test_engine_bitwise_against_oracle(name):
    from oracle import run_oracle
    sim = scenes.build(name, pf)
    res = sim.run()
    ref = run_oracle(scenes.build(name, pf))
    for mon, comps in ref["fields"].items():
        for c, arr in comps.items():
            np.testing.assert_array_equal(res.fields[mon][c], arr, err_msg=f"{name} {mon} {c}")
    for mon, comps in ref["dft"].items():
        for c, arr in comps.items():
            np.testing.assert_array_equal(res.dft[mon][c], arr, err_msg=f"{name} dft {mon} {c}")
    scale = max([abs(v) for v in ref["flux"].values()] + [1e-300])
    for mon, v in ref["flux"].items():
        assert abs(res.flux[mon] - v) <= 1e-6 * scale, (name, mon, res.flux[mon], v)


@pytest.mark.parametrize("name", ["xz2d_f32", "tm2d_f64", "disp2d_f32", "sub3d_f32"])
def test_inline_sources_and_dft_equal_separate_launches(name, monkeypatch):
    """With PFB200_INLINE=1 the split E pass adds the E-family sources and
    writes the DFT samples itself; by default separate kernels do it after
    the pass. Fields, DFT sums and flux must be identical either way."""
    out = []
    for on in (True, False):
        if on:
            monkeypatch.setenv("PFB200_INLINE", "1")
        else:
            monkeypatch.delenv("PFB200_INLINE", raising=False)
        out.append(scenes.build(name, pf).run())
    a, b = out
    for mon, comps in a.fields.items():
        for c, arr in comps.items():
            np.testing.assert_array_equal(arr, b.fields[mon][c], err_msg=f"{name} {mon} {c}")
    for mon, comps in a.dft.items():
        for c, arr in comps.items():
            np.testing.assert_array_equal(arr, b.dft[mon][c], err_msg=f"{name} dft {mon} {c}")
    for mon, v in a.flux.items():
        assert v == b.flux[mon], (name, mon)
