"""Small subpixel scenes made of boxes: 3D (config-2 recipe) and 2D in the
xy and xz planes, for the smoothing tests."""
import numpy as np

import photonfdtd_b200 as pf
from photonfdtd_b200 import workloads as W


def scene_2d(size, seed=11, n_boxes=9, precision="float32"):
    grid = pf.Grid(size=size, cell_size=20e-9, pml_layers=12)
    rng = np.random.default_rng(seed)
    boxes = []
    for _ in range(n_boxes):
        c = tuple(float(rng.uniform(-0.6e-6, 0.6e-6)) if s > 0 else 0.0 for s in size)
        sz = tuple(float(rng.uniform(0.1e-6, 0.7e-6)) if s > 0 else 1.0 for s in size)
        boxes.append(pf.Box(center=c, size=sz,
                            medium=pf.Medium(permittivity=float(rng.uniform(1.5, 12.0)))))
    src = pf.PointDipole(position=(0.0, 0.0, 0.0), component="Ez",
                         waveform=pf.GaussianPulse(freq0=250e12, fwhm=6e-15))
    return pf.Simulation(grid, structures=boxes, sources=[src], run_time=5e-15, subpixel=True,
                         precision=precision)


def scenes():
    return [
        ("3d_f32_factor3", W.config2(pf, interior=40, n_boxes=20, n_steps=5)),
        ("3d_f64_factor2", W.config2(pf, interior=40, n_boxes=20, n_steps=5,
                                     precision="float64", subpixel_factor=2)),
        ("2d_xy", scene_2d((2.0e-6, 1.5e-6, 0.0))),
        ("2d_xz", scene_2d((2.0e-6, 0.0, 1.5e-6))),
        ("3d_factor1", W.config2(pf, interior=24, n_boxes=12, n_steps=5, subpixel_factor=1)),
        ("3d_factor4", W.config2(pf, interior=24, n_boxes=12, n_steps=5, subpixel_factor=4)),
    ]
