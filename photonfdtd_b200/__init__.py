"""photonfdtd_b200 - B200-native FDTD stepping engine for photonfdtd.

A drop-in for photonfdtd's time-stepping hot path: the Yee + CPML (+ ADE
dispersion, + diagonal subpixel eps) step with soft sources and DFT / flux /
field monitors, executed by hand-written sm_100a CUDA kernels behind a C ABI
(include/pfb200.h, loaded with ctypes).

    import photonfdtd_b200 as pf
    sim = pf.Simulation(grid, structures, sources, monitors, run_time,
                        precision="float32", backend="b200")
    result = sim.run()

The scene classes mirror the reference package's (same names and
arguments), and ``photonfdtd_b200.plugin.install()`` registers
``backend="b200"`` on the reference ``photonfdtd.Simulation`` itself.
"""
from .scene import (C_0, EPS_0, ETA_0, MU_0, Q_E, VACUUM, Box, CPMLParams, DFTMonitor,
                    DispersiveMedium, FieldMonitor, FluxMonitor, GaussianPulse, Grid, Medium,
                    ModeSource, PointDipole, Pole, UniModeSource, cpml_coeffs_1axis)
from .mode import ModeResult, ModeSolver
from .smatrix import mode_amplitudes, s_parameters
from .simulation import Result, Simulation
from .smoothing import smooth_permittivity

__version__ = "0.1.0"

__all__ = [
    "C_0", "EPS_0", "ETA_0", "MU_0", "Q_E", "VACUUM", "Box", "CPMLParams", "DFTMonitor",
    "DispersiveMedium", "FieldMonitor", "FluxMonitor", "GaussianPulse", "Grid", "Medium",
    "ModeSource", "PointDipole", "Pole", "UniModeSource", "ModeResult", "ModeSolver",
    "cpml_coeffs_1axis", "Result", "Simulation", "mode_amplitudes", "s_parameters",
    "smooth_permittivity",
]
