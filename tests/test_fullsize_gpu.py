"""The stepping kernels at the named workloads' full sizes, bit for bit.

The golden scenes pin the engine at reduced sizes over thousands of steps.
These tests pin it at the sizes the benchmark runs: config 3 (384^3 cells,
Drude / two-pole Lorentz / dielectric blocks, six full-plane flux monitors,
an Ex/Ey DFT) and config 2 (536^3 cells, 64 boxes with subpixel smoothing, a
16-wavelength DFT on the z = 0 plane). A few steps from zero fields would
leave almost every cell at zero, so both sides start from the same seeded
random fields (pf_write_field on the engine, OracleRun.set_fields on the
oracle) spanning many decades of magnitude: every cell, every CPML slab and
every dispersive record is exercised, and numerators on both sides of the
fast exact division's range occur. After three steps the six fields, the DFT
sums and the flux integrals must equal the oracle's: fields and DFT bit for
bit; flux to 1e-4 of its scale, because the reference sums each plane in
float32 (pairwise) and the engine in float64, and random fields of mixed sign
spanning many decades cancel far more than physical ones (a wrong plane,
component or sign would still miss by order one).

The config-2 oracle takes its subpixel coefficients from the engine's tables
(the GPU smoothing, pinned bit for bit to the host smoothing and to the
reference's own tables by tests/test_smoothing_gpu.py and
tests/test_host_tables.py): the oracle's own host smoothing of 536^3 would
take minutes.
"""
import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200 import workloads as W
from photonfdtd_b200.engine import B200Engine, build_tables

pytestmark = pytest.mark.gpu

ALL6 = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
STEPS = 3


def _random_fields(shape, seed):
    rng = np.random.default_rng(seed)
    out = {}
    for q, c in enumerate(ALL6):
        mag = 10.0 ** rng.uniform(-20.0, 9.0, size=shape).astype(np.float32)
        f = (rng.standard_normal(shape, dtype=np.float32) * mag).astype(np.float32)
        if c[0] == "H":
            f *= np.float32(1.0 / 377.0)
        out[c] = f
    return out


def _case(name):
    if name == "config3_384":
        sim = W.config3(pf, n_total=384, n_steps=3000)
    else:
        sim = W.config2(pf, interior=512, n_steps=2000)
    return sim


@pytest.mark.parametrize("case", ["config3_192", "config2_160"])
def test_bulk_fast_path_bitwise_against_oracle(case):
    """Grids large enough that whole blocks lie in the bulk box (both
    difference terms, no CPML state) and take the straight-line path, which
    the small golden scenes never reach; random states down to 1e-40, so
    products and quotients fall into the subnormal range. Fields after two
    steps equal the oracle's bit for bit."""
    from oracle import OracleRun
    if case == "config3_192":
        def make():
            return W.config3(pf, n_total=192, n_steps=100, flux=False, dft=False)
    else:
        def make():
            return W.config2(pf, interior=136, n_boxes=8, n_freqs=4, n_steps=100)
    t = build_tables(make())
    rng = np.random.default_rng(23)
    fields = {}
    for c in ALL6:
        mag = 10.0 ** rng.uniform(-40.0, 3.0, size=t["shape"]).astype(np.float32)
        fields[c] = (rng.standard_normal(t["shape"], dtype=np.float32) * mag).astype(np.float32)
    eng = B200Engine(t)
    try:
        for c in ALL6:
            eng.set_field(c, fields[c])
        eng.advance(0, 2)
        got = {c: eng.get(c).copy() for c in ALL6}
    finally:
        eng.close()
    run = OracleRun(make(), ce3=t["ce"] if t["ce_mode"] == 1 else None)
    run.set_fields(fields)
    run.advance(2)
    for c in ALL6:
        np.testing.assert_array_equal(got[c], run.F[c], err_msg=f"{case} {c}")


@pytest.mark.parametrize("name", ["config3_384", "config2_536"])
def test_full_size_steps_bitwise_against_oracle(name):
    from oracle import OracleRun
    sim = _case(name)
    t = build_tables(sim)
    shape = t["shape"]
    fields = _random_fields(shape, seed=17)
    eng = B200Engine(t)
    try:
        for c in ALL6:
            eng.set_field(c, fields[c])
        eng.advance(0, STEPS)
        got = {c: eng.get(c).copy() for c in ALL6}
        dft = {}
        for k, d in enumerate(t["dft"]):
            for c in d["m"].components:
                dft[(d["m"].name, c)] = eng.read_dft(k, c, d["omega"].size, d["counts"])
        flux = {f["m"].name: eng.read_flux(k) for k, f in enumerate(t["flux"])}
    finally:
        eng.close()
    ce3 = t["ce"] if t["ce_mode"] == 1 else None
    run = OracleRun(_case(name), ce3=ce3)
    run.set_fields(fields)
    del fields
    run.advance(STEPS)
    ref = run.result()
    for c in ALL6:
        np.testing.assert_array_equal(got[c], run.F[c], err_msg=f"{name} {c}")
    for (mon, c), arr in dft.items():
        np.testing.assert_array_equal(arr, ref["dft"][mon][c], err_msg=f"{name} dft {mon} {c}")
    scale = max([abs(v) for v in ref["flux"].values()] + [1e-300])
    for mon, v in ref["flux"].items():
        assert abs(flux[mon] - v) <= 1e-4 * scale, (name, mon, flux[mon], v)
