"""Small parity scenes, built against any photonfdtd-compatible module ``pf``.

The same builders produce the reference runs frozen in ``tests/golden`` (see
``make_golden.py``) and the engine runs compared against them, so a scene's
inputs are identical on both sides by construction. The first three follow
the reference's own parity tests (tests/test_rust.py:23-80 of
ngpaladi/photonfdtd); the rest cover the branches those do not reach
(collapsed-y 2D, H-family and coincident sources, downsampled and full-volume
monitors, flux on every axis, dispersion).
"""
from __future__ import annotations

import numpy as np

from photonfdtd_b200 import workloads as W

C_0 = 299_792_458.0
ALL6 = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def tm2d(pf, precision="float64"):
    """tests/test_rust.py:23-35: 2D TM dipole beside an n=2 box, DFT at f0."""
    freq0 = C_0 / 1.0e-6
    grid = pf.Grid(size=(4e-6, 3e-6), cell_size=50e-9, pml_layers=(10, 10, 0))
    box = pf.Box(center=(0.6e-6, 0.0), size=(1.0e-6, 1.0e-6),
                 medium=pf.Medium.from_index(2.0))
    src = pf.PointDipole(position=(-0.8e-6, 0.0, 0.0), component="Ez",
                         waveform=pf.GaussianPulse(freq0=freq0, fwhm=6e-15))
    mon = pf.FieldMonitor(name="s", components=("Ez", "Hx", "Hy"), interval=25)
    dft = pf.DFTMonitor(name="d", components=("Ez",), freqs=[freq0], interval=1)
    return pf.Simulation(grid, structures=[box], sources=[src], monitors=[mon, dft],
                         run_time=40e-15, precision=precision)


def cube3d(pf, precision="float64"):
    """tests/test_rust.py:50-61: 3D Ey dipole beside an n=1.8 cube."""
    freq0 = C_0 / 1.0e-6
    grid = pf.Grid(size=(2.5e-6, 2e-6, 2e-6), cell_size=80e-9, pml_layers=(8, 8, 8))
    box = pf.Box(center=(0.4e-6, 0, 0), size=(0.8e-6, 0.8e-6, 0.8e-6),
                 medium=pf.Medium.from_index(1.8))
    src = pf.PointDipole(position=(-0.5e-6, 0, 0), component="Ey",
                         waveform=pf.GaussianPulse(freq0=freq0, fwhm=5e-15))
    mon = pf.FieldMonitor(name="s", components=("Ey", "Hz"), times=[14e-15])
    full = pf.FieldMonitor(name="all", components=("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"),
                           times=[15e-15 - 1e-18])
    return pf.Simulation(grid, structures=[box], sources=[src], monitors=[mon, full],
                         run_time=15e-15, precision=precision)


def line1d(pf, precision="float64"):
    """tests/test_rust.py:72-79: 1D Ez dipole in vacuum."""
    freq0 = C_0 / 1.0e-6
    grid = pf.Grid(size=(8e-6,), cell_size=20e-9, pml_layers=(12,))
    src = pf.PointDipole(position=(0.0,), component="Ez",
                         waveform=pf.GaussianPulse(freq0=freq0, fwhm=5e-15))
    mon = pf.FieldMonitor(name="s", components=("Ez", "Hy"), times=[20e-15])
    return pf.Simulation(grid, sources=[src], monitors=[mon], run_time=22e-15,
                         precision=precision)


def xz2d(pf, precision="float64"):
    """2D in the xz plane (y collapsed): two boxes, an H-family source, two
    coincident E dipoles, flux normal to x and z, downsampled snapshot and
    full-volume DFT, plane_z snapshot."""
    freq0 = C_0 / 1.2e-6
    grid = pf.Grid(size=(3.2e-6, 0, 2.4e-6), cell_size=40e-9, pml_layers=(10, 0, 9))
    boxes = [pf.Box(center=(0.5e-6, 0.0, 0.2e-6), size=(0.9e-6, 0.0, 0.7e-6),
                    medium=pf.Medium(permittivity=5.0)),
             pf.Box(center=(0.2e-6, 0.0, -0.3e-6), size=(0.6e-6, 1.0, 0.5e-6),
                    medium=pf.Medium(permittivity=2.5))]
    w = pf.GaussianPulse(freq0=freq0, fwhm=5e-15, delay=2e-15)
    srcs = [pf.PointDipole(position=(-0.7e-6, 0.0, 0.1e-6), component="Ex", waveform=w),
            pf.PointDipole(position=(-0.7e-6, 0.0, 0.1e-6), component="Ex", waveform=w,
                           amplitude=-0.37),
            pf.PointDipole(position=(-0.5e-6, 0.0, -0.2e-6), component="Hy",
                           waveform=pf.GaussianPulse(freq0=freq0 * 1.1, fwhm=4e-15),
                           amplitude=250.0),
            pf.PointDipole(position=(0.1e-6, 0.0, 0.4e-6), component="Ez", waveform=w,
                           amplitude=0.5)]
    mons = [pf.FieldMonitor(name="ds", components=("Ex", "Ez", "Hy"), interval=17,
                            downsample=2),
            pf.FieldMonitor(name="pz", components=("Hy",), interval=40, plane_z=0.3e-6),
            pf.DFTMonitor(name="vol", components=("Ex", "Hy"), freqs=[0.9 * freq0, freq0],
                          interval=2, downsample=3),
            pf.DFTMonitor(name="px", components=("Ez", "Hy"), freqs=[freq0, 1.3 * freq0],
                          plane_axis="x", plane_position=0.9e-6),
            pf.FluxMonitor(name="fx", plane_axis="x", plane_position=0.95e-6),
            pf.FluxMonitor(name="fz", plane_axis="z", plane_position=-0.75e-6),
            pf.FluxMonitor(name="fy", plane_axis="y", plane_position=0.0)]
    return pf.Simulation(grid, structures=boxes, sources=srcs, monitors=mons,
                         run_time=35e-15, precision=precision)


def disp2d(pf, precision="float64"):
    """Drude + Lorentz + plain box in 2D TM, all dispersive paths (two poles,
    plain medium overriding a dispersive one), DFT and flux."""
    drude = pf.DispersiveMedium.drude(1.0, f_plasma_Hz=150e12, f_collision_Hz=5e12)
    lor = pf.DispersiveMedium.lorentz(2.0, [(1.2, 300e12, 4e12), (0.4, 500e12, 0.0)])
    grid = pf.Grid(size=(4e-6, 3.2e-6), cell_size=40e-9, pml_layers=(10, 10, 0))
    boxes = [pf.Box(center=(0.8e-6, 0.0), size=(1.2e-6, 1.2e-6), medium=drude),
             pf.Box(center=(-0.6e-6, 0.5e-6), size=(1.0e-6, 0.8e-6), medium=lor),
             pf.Box(center=(0.8e-6, 0.3e-6), size=(0.4e-6, 0.4e-6),
                    medium=pf.Medium(permittivity=3.0)),
             pf.Box(center=(-0.6e-6, -0.6e-6), size=(0.6e-6, 0.6e-6), medium=drude)]
    src = pf.PointDipole(position=(-1.2e-6, -0.1e-6), component="Ez",
                         waveform=pf.GaussianPulse(freq0=250e12, fwhm=6e-15))
    mons = [pf.FieldMonitor(name="s", components=("Ez", "Hx", "Hy"), interval=60),
            pf.DFTMonitor(name="d", components=("Ez",), freqs=[200e12, 260e12]),
            pf.FluxMonitor(name="f", plane_axis="x", plane_position=1.5e-6)]
    return pf.Simulation(grid, structures=boxes, sources=[src], monitors=mons,
                         run_time=50e-15, precision=precision)


def sub3d(pf, precision="float32"):
    """Reduced config-2 recipe: 40^3 interior + 12-cell CPML, 6 boxes,
    subpixel on, 4 DFT wavelengths, 600 steps."""
    sim = W.config2(pf, interior=40, n_boxes=6, n_freqs=4, n_steps=600,
                    subpixel=True, precision=precision)
    sim.add_monitor(pf.FieldMonitor(name="mid", components=ALL6, plane_z=0.0,
                                    times=[300 * sim.dt, 599 * sim.dt]))
    return sim


def ade3d(pf, precision="float32", n_steps=3000):
    """Reduced config-3 recipe: 64^3 total, 8^3 media blocks, 6 flux planes,
    Ex/Ey DFT at 8 wavelengths."""
    sim = W.config3(pf, n_total=64, block=8, n_steps=n_steps, precision=precision)
    sim.add_monitor(pf.FieldMonitor(name="mid", components=ALL6, plane_z=0.0,
                                    times=[(n_steps // 3) * sim.dt, (n_steps - 1) * sim.dt]))
    return sim


def c2rep(pf, precision="float32", n_steps=2000):
    """Config-2 replica at reduced size: a 96^3 interior (120^3 grid with the
    12-cell CPML) at 20 nm, 8 seeded boxes with centres and sides scaled by
    96/512, subpixel smoothing (factor 3), the Ex dipole and the 16-wavelength
    DFT on the z = 0 plane, over the full 2000 steps; plus the six fields on
    that plane at step 700 (pulse inside the domain) and at the last step (a
    residual of about 1e-8 of the peak, dominated by round-off)."""
    sim = W.config2(pf, interior=96, n_boxes=8, n_freqs=16, n_steps=n_steps,
                    subpixel=True, precision=precision)
    sim.add_monitor(pf.FieldMonitor(name="mid", components=ALL6, plane_z=0.0,
                                    times=[700 * sim.dt, (n_steps - 1) * sim.dt]))
    return sim


def te2d(pf, precision="float32", n_steps=2000):
    """Reduced config-4 recipe: one 120 x 90 instance, 32 x 32 design."""
    rho = W.config4_density(7, design=32)
    sim = W.config4_instance(pf, 120, 90, rho=rho, n_steps=n_steps, precision=precision,
                             design=32)
    sim.add_monitor(pf.FieldMonitor(name="end", components=("Ex", "Ey", "Hz"),
                                    times=[(n_steps - 1) * sim.dt]))
    return sim


SCENES = {
    "tm2d_f64": (tm2d, dict(precision="float64")),
    "tm2d_f32": (tm2d, dict(precision="float32")),
    "cube3d_f64": (cube3d, dict(precision="float64")),
    "cube3d_f32": (cube3d, dict(precision="float32")),
    "line1d_f64": (line1d, dict(precision="float64")),
    "xz2d_f64": (xz2d, dict(precision="float64")),
    "xz2d_f32": (xz2d, dict(precision="float32")),
    "disp2d_f64": (disp2d, dict(precision="float64")),
    "disp2d_f32": (disp2d, dict(precision="float32")),
    "config1": (W.config1, dict()),
    "sub3d_f32": (sub3d, dict(precision="float32")),
    "ade3d_f32": (ade3d, dict(precision="float32")),
    "te2d_f32": (te2d, dict(precision="float32")),
    # float64 runs of the reduced config-2/3/4 recipes: the float32 runs'
    # error against them is what every float32 result states
    "sub3d_f64": (sub3d, dict(precision="float64")),
    "ade3d_f64": (ade3d, dict(precision="float64")),
    "te2d_f64": (te2d, dict(precision="float64")),
    "c2rep_f32": (c2rep, dict(precision="float32")),
    "c2rep_f64": (c2rep, dict(precision="float64")),
}

# DFT results thinned in the fixtures (frequency indices and components
# kept), to keep them small; tests slice their own runs the same way.
THIN_DFT = {
    "c2rep_f32": dict(freqs=(0, 7, 15), comps=("Ex", "Hy")),
    "c2rep_f64": dict(freqs=(0, 7, 15), comps=("Ex", "Hy")),
}


def build(name, pf):
    fn, kw = SCENES[name]
    return fn(pf, **kw)
