"""Named synthetic workloads of the stepping engine.

Each builder takes a photonfdtd-compatible module ``pf`` (this package, or the
reference ``photonfdtd`` itself) and returns a ready ``Simulation``. The same
recipe therefore builds the scene for the engine, for the CPU oracle and, in
``tests/golden/make_golden.py``, for the reference run that pins parity.

Workloads (full sizes are the defaults; the parity tests pass smaller ones):

* ``config1`` - plain 2D TM, float64: 104 x 104 cells at 50 nm (80 x 80
  interior + 12-cell CPML on x and y), Ez Gaussian dipole (lambda0 1 um,
  FWHM 10 fs), 200 fs, Ez FieldMonitor every 20 steps.
* ``config2`` - 3D non-dispersive, float32: (512 + 2*12)^3 cells at 20 nm, 64
  seeded random boxes (eps in [1, 12.1], sides in [0.2, 2] um), subpixel
  smoothing, Ex dipole (1.55 um, 15 fs), 2000 steps, DFTMonitor on the z = 0
  plane at 16 wavelengths in 1.4-1.7 um.
* ``config3`` - 3D dispersive ADE, float32: 384^3 cells at 10 nm (12-cell CPML
  inside the 384), one of three media per 8^3 block (Drude metal; two-pole
  Lorentz; eps 2.1 dielectric), Ex dipole (0.8 um, 10 fs), 3000 steps, six
  full-plane FluxMonitors at +-1.6 um, DFTMonitor (Ex, Ey) at 8 wavelengths.
* ``config4_instance`` - one 2D TE inverse-design instance, float32: nx x ny
  cells at 20 nm with 12-cell CPML, background eps 1.444^2, centred 64 x 64
  density design region, Ey line source, Ey DFT at 8 wavelengths on an output
  line. ``config4_sizes`` draws the 256 uneven (nx, ny).

All random draws are seeded (numpy default_rng), so a workload is the same
array on every machine. No public dataset is involved.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

C_0 = 299_792_458.0


def _dt(cell_size: float, ndim_for_courant: int, courant: float = 0.99) -> float:
    return courant / (C_0 * math.sqrt(ndim_for_courant / cell_size ** 2))


def _run_time_for(n_steps: int, dt: float) -> float:
    # ceil((n - 1/2) dt / dt) == n for any dt: pins the step count exactly.
    return (n_steps - 0.5) * dt


# --------------------------------------------------------------------------- #
def config1(pf, precision: str = "float64"):
    """Plain 2D TM float64 dipole (80^2 interior + 12-cell CPML, 50 nm)."""
    n = 104
    d = 50e-9
    grid = pf.Grid(size=(n * d, n * d), cell_size=d, pml_layers=(12, 12, 0))
    src = pf.PointDipole(position=(0.0, 0.0), component="Ez",
                         waveform=pf.GaussianPulse(freq0=C_0 / 1e-6, fwhm=10e-15))
    mon = pf.FieldMonitor(name="m", components=("Ez",), interval=20)
    return pf.Simulation(grid, sources=[src], monitors=[mon], run_time=200e-15,
                         precision=precision)


def config2_boxes(n_boxes: int = 64, scale: float = 1.0, seed: int = 2):
    """(centers, sizes, eps) of the seeded random boxes, metres."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-5.12e-6, 5.12e-6, size=(n_boxes, 3)) * scale
    sizes = rng.uniform(0.2e-6, 2.0e-6, size=(n_boxes, 3)) * scale
    eps = rng.uniform(1.0, 12.1, size=n_boxes)
    return centers, sizes, eps


def config2(pf, interior: int = 512, n_boxes: int = 64, n_freqs: int = 16,
            n_steps: int = 2000, subpixel: bool = True,
            precision: str = "float32", subpixel_factor: int = 3):
    """3D non-dispersive Yee + CPML with subpixel boxes and a z-plane DFT."""
    d = 20e-9
    pml = 12
    n = interior + 2 * pml
    grid = pf.Grid(size=(n * d,) * 3, cell_size=d, pml_layers=pml)
    centers, sizes, eps = config2_boxes(n_boxes, scale=interior / 512.0)
    boxes = [pf.Box(center=tuple(c), size=tuple(s), medium=pf.Medium(permittivity=float(e)))
             for c, s, e in zip(centers, sizes, eps)]
    src = pf.PointDipole(position=(0.0, 0.0, 0.0), component="Ex",
                         waveform=pf.GaussianPulse(freq0=C_0 / 1.55e-6, fwhm=15e-15))
    freqs = C_0 / np.linspace(1.4e-6, 1.7e-6, n_freqs)
    dft = pf.DFTMonitor(name="d", components=("Ex", "Ey", "Hx", "Hy"), freqs=freqs,
                        plane_axis="z", plane_position=0.0)
    dt = _dt(d, 3)
    return pf.Simulation(grid, structures=boxes, sources=[src], monitors=[dft],
                         run_time=_run_time_for(n_steps, dt), precision=precision,
                         subpixel=subpixel, subpixel_factor=subpixel_factor)


def config3_media(pf):
    """The three media of the dispersive workload, as shared objects."""
    drude = pf.DispersiveMedium(eps_inf=1.0, poles=(pf.Pole(strength=1.37e16 ** 2,
                                                            omega0=0.0, gamma=1.0e14),))
    lorentz = pf.DispersiveMedium(eps_inf=1.0, poles=(
        pf.Pole(strength=1.0 * 3e15 ** 2, omega0=3e15, gamma=1e13),
        pf.Pole(strength=0.5 * 6e15 ** 2, omega0=6e15, gamma=1e13)))
    dielectric = pf.Medium(permittivity=2.1)
    return drude, lorentz, dielectric


def config3_block_ids(n_blocks: int, seed: int = 3) -> np.ndarray:
    return np.random.default_rng(seed).integers(0, 3, size=(n_blocks,) * 3)


def config3_plain_media(pf):
    """Non-dispersive stand-ins for the three media (eps 1.0 / 4.0 / 2.1): the
    workload the reference's CUDA kernels can run (scalar ce, no ADE)."""
    return tuple(pf.Medium(permittivity=e) for e in (1.0, 4.0, 2.1))


class BlockMedium:
    """All blocks of one medium in a block-structured scene, as one structure.

    It follows the reference's structure protocol (src/photonfdtd/geometry.py
    Box.region_mask / Box.stamp): ``region_mask(grid)`` is the boolean grid
    of the medium's cells, ``stamp(grid, eps_r)`` writes its permittivity
    there, ``medium`` is the medium. The blocks of different media are
    disjoint, so one such structure per medium rasterises to exactly the
    cells (and ADE media) that one Box per block gives; it only spares a
    rasteriser that walks the full grid per structure (the reference's) one
    pass per block."""

    def __init__(self, medium, ids: np.ndarray, which: int, block: int):
        self.medium = medium
        self._ids = ids
        self._which = which
        self._block = block

    def region_mask(self, grid) -> np.ndarray:
        b = self._block
        sel = self._ids == self._which
        n0, n1, n2 = sel.shape
        m = np.broadcast_to(sel[:, None, :, None, :, None],
                            (n0, b, n1, b, n2, b)).reshape(n0 * b, n1 * b, n2 * b)
        shape = tuple(grid.shape)
        if m.shape == shape:
            return m
        out = np.zeros(shape, dtype=bool)
        n = [min(shape[a], m.shape[a]) for a in range(3)]
        out[:n[0], :n[1], :n[2]] = m[:n[0], :n[1], :n[2]]
        return out

    def stamp(self, grid, eps_r: np.ndarray) -> None:
        eps_r[self.region_mask(grid)] = self.medium.eps_r


def config3(pf, n_total: int = 384, block: int = 8, n_steps: int = 3000,
            flux: bool = True, dft: bool = True, precision: str = "float32",
            flux_pos: float = None, dispersive: bool = True, union_blocks: bool = False,
            **sim_kw):
    """3D dispersive ADE mix in 8^3 blocks, six flux planes, a z-plane DFT.
    dispersive=False swaps in config3_plain_media (same grid and blocks).
    union_blocks=True describes the blocks as one BlockMedium per medium
    instead of one Box per block (same cells, same media). sim_kw go to the
    Simulation (e.g. the reference's use_numba or backend)."""
    d = 10e-9
    grid = pf.Grid(size=(n_total * d,) * 3, cell_size=d, pml_layers=12)
    media = config3_media(pf) if dispersive else config3_plain_media(pf)
    nb = n_total // block
    ids = config3_block_ids(nb)
    x0 = -(n_total - 1) / 2 * d            # coordinate of cell 0
    boxes = []
    if union_blocks:
        boxes = [BlockMedium(media[q], ids, q, block) for q in range(3)]
    else:
        for bi in range(nb):
            for bj in range(nb):
                for bk in range(nb):
                    # box spanning cells [b*block, (b+1)*block) on each axis:
                    # its faces sit half a cell outside the first and last
                    # centres.
                    c = [x0 + (b * block + (block - 1) / 2) * d for b in (bi, bj, bk)]
                    boxes.append(pf.Box(center=tuple(c), size=(block * d,) * 3,
                                        medium=media[int(ids[bi, bj, bk])]))
    src = pf.PointDipole(position=(0.0, 0.0, 0.0), component="Ex",
                         waveform=pf.GaussianPulse(freq0=C_0 / 0.8e-6, fwhm=10e-15))
    mons = []
    if flux:
        fp = 1.6e-6 * n_total / 384 if flux_pos is None else flux_pos
        for ax in "xyz":
            for sgn, tag in ((-1, "lo"), (1, "hi")):
                mons.append(pf.FluxMonitor(name=f"flux_{ax}{tag}", plane_axis=ax,
                                           plane_position=sgn * fp))
    if dft:
        freqs = C_0 / np.linspace(0.7e-6, 0.9e-6, 8)
        mons.append(pf.DFTMonitor(name="d", components=("Ex", "Ey"), freqs=freqs,
                                  plane_axis="z", plane_position=0.0))
    dt = _dt(d, 3)
    return pf.Simulation(grid, structures=boxes, sources=[src], monitors=mons,
                         run_time=_run_time_for(n_steps, dt), precision=precision, **sim_kw)


# --------------------------------------------------------------------------- #
EPS_CLAD = 1.444 ** 2
EPS_CORE = 3.476 ** 2


def config4_sizes(n_instances: int = 256, seed: int = 4) -> List[Tuple[int, int]]:
    rng = np.random.default_rng(seed)
    nx = rng.integers(200, 801, size=n_instances)
    ny = rng.integers(150, 401, size=n_instances)
    return [(int(a), int(b)) for a, b in zip(nx, ny)]


def config4_density(i: int, design: int = 64, seed_base: int = 1000) -> np.ndarray:
    """Seeded Gaussian-filtered (sigma = 3 cells) field, unit-normalised,
    through a sigmoid: a smooth density in (0, 1)."""
    from scipy.ndimage import gaussian_filter
    g = gaussian_filter(np.random.default_rng(seed_base + i).standard_normal((design, design)),
                        sigma=3.0)
    g = g / g.std()
    return 1.0 / (1.0 + np.exp(-g))


def config4_eps(nx: int, ny: int, rho: np.ndarray, dtype=np.float32) -> np.ndarray:
    eps = np.full((nx, ny, 1), EPS_CLAD, dtype=np.float64)
    dsz = rho.shape[0]
    i0, j0 = nx // 2 - dsz // 2, ny // 2 - dsz // 2
    eps[i0:i0 + dsz, j0:j0 + dsz, 0] = EPS_CLAD + rho * (EPS_CORE - EPS_CLAD)
    return eps.astype(dtype)


def design_window_box(nx: int, ny: int, design: int) -> Tuple[int, int, int]:
    """(i0, j0, n) of the centred design window."""
    return nx // 2 - design // 2, ny // 2 - design // 2, design


def design_window(nx: int, ny: int, design: int) -> Tuple[slice, slice]:
    i0, j0 = nx // 2 - design // 2, ny // 2 - design // 2
    return slice(i0, i0 + design), slice(j0, j0 + design)


def config4_instance(pf, nx: int, ny: int, rho: np.ndarray = None, i: int = 0,
                     n_steps: int = 4000, n_freqs: int = 8, precision: str = "float32",
                     design: int = 64, band: Tuple[float, float] = (1.5e-6, 1.6e-6)):
    """One 2D TE instance: Ey line source at x index 20 over the interior, Ey
    DFT on the output line at x index nx - 21 at n_freqs wavelengths evenly
    spaced over `band`, custom eps from the density."""
    d = 20e-9
    pml = 12
    grid = pf.Grid(size=(nx * d, ny * d), cell_size=(d, d), pml_layers=(pml, pml, 0))
    pulse = pf.GaussianPulse(freq0=C_0 / 1.55e-6, fwhm=15e-15)
    xs = grid.coords[0]
    ys = grid.coords[1]
    srcs = [pf.PointDipole(position=(float(xs[20]), float(ys[j])), component="Ey",
                           waveform=pulse) for j in range(pml, ny - pml)]
    freqs = C_0 / np.linspace(band[0], band[1], n_freqs)
    mon = pf.DFTMonitor(name="out", components=("Ey",), freqs=freqs,
                        plane_axis="x", plane_position=float(xs[nx - 21]))
    dt = _dt(d, 2)
    sim = pf.Simulation(grid, sources=srcs, monitors=[mon],
                        run_time=_run_time_for(n_steps, dt), precision=precision)
    if rho is None:
        rho = config4_density(i, design)
    npdt = np.float32 if precision == "float32" else np.float64
    sim.eps_r = config4_eps(nx, ny, rho, dtype=npdt)
    return sim


# --------------------------------------------------------------------------- #
# config 5: the surrogate's design problem
# --------------------------------------------------------------------------- #
CONFIG5_SHAPE = (400, 250)
CONFIG5_BAND = (1.4e-6, 1.7e-6)
CONFIG5_FREQS = 32


def config5_instance(pf, rho: np.ndarray = None, n_steps: int = 4000,
                     precision: str = "float32"):
    """The fixed config-4-style geometry of the surrogate problem: 400 x 250
    cells, centred 64 x 64 design window, Ey DFT at 32 wavelengths evenly
    spaced over 1.4-1.7 um. rho = None is the empty design (cladding only)."""
    nx, ny = CONFIG5_SHAPE
    if rho is None:
        rho = np.zeros((64, 64))
    return config4_instance(pf, nx, ny, rho=rho, n_steps=n_steps, n_freqs=CONFIG5_FREQS,
                            precision=precision, design=64, band=CONFIG5_BAND)
