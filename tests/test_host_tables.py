"""Host-side tables of the engine against the reference's own (tables.npz).

The engine's inputs - CPML coefficients, subpixel permittivity tensors,
source waveforms, mode-source dipoles, Courant step - are computed by this
package's host code; they must equal the reference's bit for bit, since the
float32 parity of the stepping depends on identical coefficients.
"""
import numpy as np
import pytest

import photonfdtd_b200 as pf
import scenes
from golden_util import GOLDEN
from oracle.fdtd_oracle import box_mask, box_slices, grid_of
from photonfdtd_b200 import workloads as W
from photonfdtd_b200.engine import build_tables

T = np.load(f"{GOLDEN}/tables.npz")


def test_cpml_coefficients_bitwise():
    for ci, (n, dl, npml, dt) in enumerate(T["cpml_cases"]):
        got = pf.cpml_coeffs_1axis(int(n), float(dl), int(npml), float(dt))
        for nm, arr in zip(("be", "ce", "bh", "ch"), got):
            np.testing.assert_array_equal(arr, T[f"cpml/{ci}/{nm}"], err_msg=f"case {ci} {nm}")
    p = pf.CPMLParams(poly_order=4, sigma_factor=1.1, alpha_max=0.1, R_target=1e-6)
    for nm, arr in zip(("be", "ce", "bh", "ch"), pf.cpml_coeffs_1axis(50, 30e-9, 9, 5e-17, p)):
        np.testing.assert_array_equal(arr, T[f"cpml/custom/{nm}"])


def test_subpixel_smoothing_bitwise():
    g3 = pf.Grid(size=(0.8e-6, 0.72e-6, 0.64e-6), cell_size=40e-9, pml_layers=0)
    boxes3 = [pf.Box(center=(0.05e-6, -0.03e-6, 0.0), size=(0.37e-6, 0.29e-6, 0.41e-6),
                     medium=pf.Medium(permittivity=7.0)),
              pf.Box(center=(-0.2e-6, 0.1e-6, 0.07e-6), size=(0.21e-6, 0.33e-6, 0.19e-6),
                     medium=pf.Medium(permittivity=2.2))]
    for f in (3, 2):
        got = np.stack(pf.smooth_permittivity(g3, boxes3, factor=f))
        np.testing.assert_array_equal(got, T[f"smooth3d/{f}"])
    g2 = pf.Grid(size=(1.0e-6, 0.8e-6), cell_size=50e-9, pml_layers=(0, 0, 0))
    boxes2 = [pf.Box(center=(0.13e-6, 0.07e-6), size=(0.43e-6, 0.31e-6),
                     medium=pf.Medium(permittivity=11.0))]
    got = np.stack(pf.smooth_permittivity(g2, boxes2, factor=3, dtype=np.float32))
    np.testing.assert_array_equal(got, T["smooth2d/3"])


def test_step_count_and_plane_indices():
    sim = W.config1(pf)
    assert (sim.dt, sim.n_steps) == tuple(T["dt/config1"])
    for n, d in ((536, 20e-9), (384, 10e-9)):
        g = pf.Grid(size=(n * d,) * 3, cell_size=d, pml_layers=12)
        idx = [g.index_at((p, p, p)) for p in (-1.6e-6, 1.6e-6, 0.0)]
        np.testing.assert_array_equal(np.array(idx), T[f"index_at/{n}"])


def test_waveform_bitwise():
    w = pf.GaussianPulse(freq0=pf.C_0 / 1.55e-6, fwhm=15e-15, delay=1e-15)
    np.testing.assert_array_equal(w(T["wave/t"]), T["wave/v"])
    np.testing.assert_array_equal(np.array([w(np.array([t]))[0] for t in T["wave/t"]]),
                                  T["wave/v1"])


def test_mode_source_expansion():
    w = pf.GaussianPulse(freq0=pf.C_0 / 1.55e-6, fwhm=15e-15, delay=1e-15)
    g = pf.Grid(size=(2e-6, 1.6e-6), cell_size=40e-9, pml_layers=(8, 8, 0))
    yy = np.linspace(-0.5e-6, 0.5e-6, 41)
    ms = pf.ModeSource(center=(-0.6e-6, 0.02e-6, 0.0), size=(0.0, 0.8e-6, 0.0), component="Ez",
                       waveform=w, profile=np.exp(-(yy / 0.25e-6) ** 2), profile_coords=(yy,),
                       amplitude=2.0)
    d = ms.expand(g)
    np.testing.assert_array_equal(np.array([x.position for x in d]), T["mode/pos"])
    np.testing.assert_array_equal(np.array([x.amplitude for x in d]), T["mode/amp"])


def test_box_ranges_equal_masks():
    """Index-range rasterisation (engine and oracle) equals the boolean mask."""
    rng = np.random.default_rng(0)
    grid = pf.Grid(size=(1e-6, 0.8e-6, 0.6e-6), cell_size=20e-9, pml_layers=0)
    g = grid_of(grid)
    for _ in range(200):
        b = pf.Box(center=tuple(rng.uniform(-0.6e-6, 0.6e-6, 3)),
                   size=tuple(rng.uniform(0, 0.8e-6, 3)), medium=pf.Medium(2.0))
        m = box_mask(b, g.coords, g.shape)
        m2 = np.zeros(g.shape, bool)
        sl = box_slices(b, g.coords)
        if sl is not None:
            m2[sl] = True
        assert (m == m2).all() and (b.region_mask(grid) == m).all()


@pytest.mark.parametrize("name", ["tm2d_f32", "disp2d_f64", "sub3d_f32", "te2d_f32", "xz2d_f64"])
def test_engine_coefficients_match_oracle(name):
    """Per-cell E coefficient the engine uploads (table lookup or arrays)
    equals the oracle's per-cell ce for every cell and component."""
    from oracle import scene_tables
    sim = scenes.build(name, pf)
    t = build_tables(sim)
    ref = scene_tables(scenes.build(name, pf))
    if t["ce_mode"] == 2:
        w = t["word"].ravel()
        ce = np.where(w & 0x80000000, 0.0, t["table"][np.minimum(w & 0x7fffffff, len(t["table"]) - 1)])
        disp = (w & 0x80000000) != 0
        if t["ade"] is not None:
            m = (w >> 27) & 15
            ce[disp] = t["ade"]["ce_m"][m[disp]]
        for c in range(3):
            np.testing.assert_array_equal(ce.reshape(t["shape"]).astype(t["npdt"]), ref["ce3"][c])
    else:
        arrs = t["ce"] * 3 if len(t["ce"]) == 1 else t["ce"]
        for c in range(3):
            np.testing.assert_array_equal(arrs[c], ref["ce3"][c])
    for ax in range(3):
        for q in range(4):
            np.testing.assert_array_equal(t["cpml"][ax][q], ref["cpml"][ax][q].astype(t["npdt"]))
