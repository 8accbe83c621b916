"""Dispersive cell words from build_tables (one native ranking pass,
pf_rank_dispersive_words) against the direct numbering the reference's
_build_ade describes (src/photonfdtd/simulation.py:592-636): every
dispersive cell carries bit 31 | medium << 27 | its rank among that medium's
cells in C order. Checked on the config-3 block scene (table mode), on a
scene whose first dispersive medium is painted over completely (it keeps its
slot with zero cells), and on a custom-eps scene (per-cell coefficient mode,
separate ADE word with plain cells zero); plus the helper's own errors.
On the GPU, the painted-over scene runs bit for bit against the oracle."""
import ctypes

import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200 import _native as N
from photonfdtd_b200 import engine as E
from photonfdtd_b200 import workloads as W

C_0 = 299_792_458.0


def direct_words(sim):
    """Word and per-medium counts numbered cell by cell in C order."""
    word, _, med_ids, media = E.material_words(sim, disp_bits=False)
    w = word.ravel().copy()
    ids = med_ids.ravel()
    counts = np.zeros(len(media), np.int64)
    for q in np.flatnonzero(ids >= 0):
        m = int(ids[q])
        w[q] = 0x80000000 | (m << 27) | int(counts[m])
        counts[m] += 1
    return w, counts, ids


def drude():
    return pf.DispersiveMedium(eps_inf=1.0, poles=(pf.Pole(strength=1.37e16 ** 2, omega0=0.0,
                                                           gamma=1e14),))


def lorentz():
    return pf.DispersiveMedium(eps_inf=2.0, poles=(
        pf.Pole(strength=3e15 ** 2, omega0=3e15, gamma=1e13),))


def test_config3_table_words():
    sim = W.config3(pf, n_total=32, n_steps=4)
    t = E.build_tables(sim)
    w, counts, _ = direct_words(sim)
    assert t["ce_mode"] == N.PF_CE_TABLE
    np.testing.assert_array_equal(t["word"].ravel(), w)
    np.testing.assert_array_equal(t["ade"]["count"], counts)
    assert t["ade"]["cell_word"] is None


def painted_over(custom=False, precision="float64", monitors=()):
    grid = pf.Grid(size=(0.64e-6, 0.48e-6, 0.4e-6), cell_size=40e-9, pml_layers=2)
    boxes = [pf.Box(center=(0.0, 0.0, 0.0), size=(0.2e-6, 0.2e-6, 0.2e-6), medium=drude()),
             pf.Box(center=(0.0, 0.0, 0.0), size=(0.3e-6, 0.3e-6, 0.3e-6),
                    medium=pf.Medium(permittivity=3.0)),
             pf.Box(center=(0.1e-6, 0.05e-6, 0.0), size=(0.25e-6, 0.2e-6, 0.3e-6),
                    medium=lorentz())]
    src = pf.PointDipole(position=(-0.2e-6, 0.0, 0.0), component="Ez",
                         waveform=pf.GaussianPulse(freq0=C_0 / 1e-6, fwhm=4e-15))
    sim = pf.Simulation(grid, structures=boxes, sources=[src], monitors=list(monitors),
                        run_time=12e-15, precision=precision)
    if custom:
        sim.eps_r = np.asarray(sim.eps_r) * 1.0
    return sim


def test_painted_over_medium_keeps_an_empty_slot():
    sim = painted_over()
    t = E.build_tables(sim)
    w, counts, _ = direct_words(sim)
    assert counts[0] == 0 and counts[1] > 0
    np.testing.assert_array_equal(t["word"].ravel(), w)
    np.testing.assert_array_equal(t["ade"]["count"], counts)
    assert len(t["ade"]["media"]) == 2 and t["ade"]["npole"].tolist() == [1, 1]


def test_cell1_mode_separate_ade_word():
    sim = painted_over(custom=True)
    assert getattr(sim, "_eps_r_custom", False)
    t = E.build_tables(sim)
    assert t["ce_mode"] == N.PF_CE_CELL1
    w, counts, ids = direct_words(sim)
    want = np.where(ids >= 0, w, 0).astype(np.uint32)
    np.testing.assert_array_equal(t["ade"]["cell_word"], want)
    np.testing.assert_array_equal(t["ade"]["count"], counts)


def painted_over_run(precision, custom):
    """painted_over with a field monitor, a DFT plane and a flux plane."""
    mons = [pf.FieldMonitor(name="f", components=("Ex", "Ez", "Hy"), interval=7),
            pf.DFTMonitor(name="d", components=("Ez",), freqs=[C_0 / 1e-6],
                          plane_axis="x", plane_position=0.12e-6),
            pf.FluxMonitor(name="fx", plane_axis="x", plane_position=0.12e-6)]
    return painted_over(custom, precision, mons)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,custom", [("float32", False), ("float64", False),
                                              ("float32", True)])
def test_painted_over_medium_runs_bitwise_against_oracle(precision, custom):
    """The engine takes a dispersive medium with zero cells (its slot kept,
    nothing allocated) and matches the oracle bit for bit, in table mode and
    in the per-cell coefficient mode (separate ADE word)."""
    from oracle import run_oracle
    sim = painted_over_run(precision, custom)
    assert np.dtype(sim.dtypes["Ex"]) == np.dtype(precision)
    res = sim.run()
    ref = run_oracle(painted_over_run(precision, custom))
    for c, arr in ref["fields"]["f"].items():
        assert np.abs(arr).max() > 0
        np.testing.assert_array_equal(res.fields["f"][c], arr, err_msg=c)
    np.testing.assert_array_equal(res.dft["d"]["Ez"], ref["dft"]["d"]["Ez"])
    assert abs(res.flux["fx"] - ref["flux"]["fx"]) <= 1e-6 * max(abs(ref["flux"]["fx"]), 1e-300)


def test_rank_helper_errors():
    L = N.lib()
    counts = np.zeros(2, np.int64)
    bad_medium = np.array([0x80000000 | (2 << 27)], np.uint32)
    with pytest.raises(ValueError, match="bad dispersive word"):
        N.check(L.pf_rank_dispersive_words(N.ptr(bad_medium, ctypes.c_uint32), 1, 2,
                                           N.ptr(counts, ctypes.c_int64), 0))
    low_bits = np.array([0x80000000 | 5], np.uint32)
    with pytest.raises(ValueError, match="bad dispersive word"):
        N.check(L.pf_rank_dispersive_words(N.ptr(low_bits, ctypes.c_uint32), 1, 2,
                                           N.ptr(counts, ctypes.c_int64), 0))
    with pytest.raises(NotImplementedError):
        N.check(L.pf_rank_dispersive_words(N.ptr(low_bits, ctypes.c_uint32), 1, 17,
                                           N.ptr(counts, ctypes.c_int64), 0))
    w = np.array([3, 0x80000000 | (1 << 27), 7, 0x80000000 | (1 << 27), 0x80000000], np.uint32)
    N.check(L.pf_rank_dispersive_words(N.ptr(w, ctypes.c_uint32), w.size, 2,
                                       N.ptr(counts, ctypes.c_int64), 1))
    assert w.tolist() == [0, 0x80000000 | (1 << 27), 0, 0x80000000 | (1 << 27) | 1, 0x80000000]
    assert counts.tolist() == [1, 2]
