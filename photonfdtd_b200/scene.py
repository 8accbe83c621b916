"""Scene description: the photonfdtd API surface the stepping engine consumes.

Class names, constructor arguments, attribute names and error behaviour follow
the reference package (ngpaladi/photonfdtd v0.12.0) so a script written
against ``photonfdtd`` runs unchanged against ``photonfdtd_b200``:

* ``Grid`` - src/photonfdtd/grid.py:17-111
* ``Medium``, ``Pole``, ``DispersiveMedium`` - src/photonfdtd/materials.py:17-186
* ``Box`` - src/photonfdtd/geometry.py:22-53
* ``GaussianPulse``, ``PointDipole``, ``ModeSource`` - src/photonfdtd/sources.py:39-337
* ``FieldMonitor``, ``DFTMonitor``, ``FluxMonitor`` - src/photonfdtd/monitors.py:17-191
* ``CPMLParams``, ``cpml_coeffs_1axis`` - src/photonfdtd/boundaries.py:23-97

Numerical conventions that decide the engine's inputs are kept exactly:
cell coordinates ``(arange(n) - (n-1)/2) * d``, nearest-cell lookup with ties
to the lower index, closed-interval box rasterisation of cell centres, and
the CPML grading formulas (computed in float64 in the same expression order,
so the coefficient tables are bit-identical).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import ClassVar, List, Optional, Sequence, Tuple

import numpy as np

# SI constants (src/photonfdtd/constants.py:4-8).
C_0 = 299_792_458.0
EPS_0 = 8.854_187_8128e-12
MU_0 = 1.256_637_062_12e-6
ETA_0 = math.sqrt(MU_0 / EPS_0)
Q_E = 1.602_176_634e-19


# --------------------------------------------------------------------------- #
# Grid
# --------------------------------------------------------------------------- #
def _grid3(x, default=None):
    if x is None:
        return (default, default, default)
    if isinstance(x, (int, float)):
        return (x, x, x)
    x = tuple(x)
    if len(x) > 3 or len(x) == 0:
        raise ValueError(f"Expected 1/2/3-tuple or scalar, got length {len(x)}")
    return x + (default,) * (3 - len(x))


@dataclass
class Grid:
    """Uniform Cartesian Yee grid; PML cells lie inside ``size``.

    ``size``/``cell_size``/``pml_layers`` accept a scalar or a 1-3 tuple; a
    missing or zero size collapses that axis to one cell at coordinate 0.
    """
    size: Tuple[float, ...]
    cell_size: Tuple[float, ...]
    pml_layers: Tuple[int, ...] = (0, 0, 0)
    shape: Tuple[int, ...] = field(init=False)
    coords: Tuple[np.ndarray, ...] = field(init=False)
    ndim: int = field(init=False)

    def __post_init__(self) -> None:
        size = _grid3(self.size)
        cs = _grid3(self.cell_size)
        pml = _grid3(self.pml_layers, default=0)
        if not any(s is not None and s > 0 for s in size):
            raise ValueError("Grid must have at least one non-zero dimension")
        shape, coords, pml_on = [], [], []
        for i, (s, d, p) in enumerate(zip(size, cs, pml)):
            if s is None or s == 0:
                shape.append(1)
                coords.append(np.array([0.0]))
                pml_on.append(0)
                continue
            if d is None or d <= 0:
                raise ValueError(f"axis {i}: cell_size must be > 0")
            n = int(round(s / d))
            if n < 4:
                raise ValueError(f"axis {i}: need at least 4 cells, got {n}")
            shape.append(n)
            coords.append((np.arange(n) - (n - 1) / 2) * d)
            pml_on.append(int(p))
        self.size = tuple(0.0 if s is None else float(s) for s in size)
        self.cell_size = tuple(0.0 if d is None else float(d) for d in cs)
        self.pml_layers = tuple(pml_on)
        self.shape = tuple(shape)
        self.coords = tuple(coords)
        self.ndim = sum(1 for s in self.size if s > 0)

    @property
    def dx(self) -> float:
        return float(self.cell_size[0])

    @property
    def dy(self) -> float:
        return float(self.cell_size[1])

    @property
    def dz(self) -> float:
        return float(self.cell_size[2])

    @property
    def min_cell(self) -> float:
        return min(d for d in self.cell_size if d > 0)

    def index_at(self, point: Sequence[float]) -> Tuple[int, int, int]:
        """Cell nearest to ``point`` per axis, ties to the lower index."""
        pt = list(point) + [0.0] * (3 - len(point))
        out = []
        for a in range(3):
            c = self.coords[a]
            out.append(0 if c.size == 1 else int(np.argmin(np.abs(c - pt[a]))))
        return tuple(out)


# --------------------------------------------------------------------------- #
# Materials
# --------------------------------------------------------------------------- #
@dataclass(frozen=True)
class Medium:
    """Isotropic non-dispersive dielectric, relative permittivity ``permittivity``."""
    permittivity: float = 1.0
    name: str = ""
    is_dispersive: ClassVar[bool] = False

    @property
    def eps_r(self) -> float:
        return float(self.permittivity)

    @classmethod
    def from_index(cls, n: float, name: str = "") -> "Medium":
        return cls(permittivity=float(n) ** 2, name=name)


VACUUM = Medium(permittivity=1.0, name="vacuum")


@dataclass(frozen=True)
class Pole:
    """One susceptibility pole strength / (omega0^2 - omega^2 - 2i gamma omega)."""
    strength: float
    omega0: float
    gamma: float = 0.0


@dataclass(frozen=True)
class DispersiveMedium:
    """eps_inf plus a sum of Lorentz/Drude/Sellmeier poles (ADE stepped)."""
    eps_inf: float
    poles: Tuple[Pole, ...] = ()
    name: str = ""
    is_dispersive: ClassVar[bool] = True

    @property
    def eps_r(self) -> float:
        return float(self.eps_inf)

    def eps_model(self, freq_hz):
        """Complex permittivity at ``freq_hz`` (e^{-i omega t} convention)."""
        w = 2.0 * np.pi * np.asarray(freq_hz, dtype=float)
        eps = np.full(w.shape, complex(self.eps_inf)) if w.ndim else complex(self.eps_inf)
        for p in self.poles:
            eps = eps + p.strength / (p.omega0 ** 2 - w ** 2 - 2j * p.gamma * w)
        return eps

    def index(self, freq_hz):
        return np.sqrt(self.eps_model(freq_hz))

    def at_wavelength(self, wavelength_m: float, name: str = "") -> Medium:
        eps = float(np.real(self.eps_model(C_0 / float(wavelength_m))))
        return Medium(permittivity=eps, name=name or f"{self.name}@{wavelength_m * 1e9:.0f}nm")

    def max_pole_omega(self) -> float:
        return max((p.omega0 for p in self.poles), default=0.0)

    @classmethod
    def lorentz(cls, eps_inf, resonances, name=""):
        """From (delta_eps, f0_Hz, delta_f_Hz) resonances; gamma = pi*delta_f."""
        poles = []
        for de, f0, df in resonances:
            w0 = 2.0 * math.pi * f0
            poles.append(Pole(strength=de * w0 ** 2, omega0=w0, gamma=math.pi * df))
        return cls(eps_inf=float(eps_inf), poles=tuple(poles), name=name)

    @classmethod
    def drude(cls, eps_inf, f_plasma_Hz, f_collision_Hz, name=""):
        wp = 2.0 * math.pi * f_plasma_Hz
        return cls(eps_inf=float(eps_inf),
                   poles=(Pole(strength=wp ** 2, omega0=0.0, gamma=math.pi * f_collision_Hz),),
                   name=name)

    @classmethod
    def sellmeier(cls, terms, name=""):
        """From (B, C[um^2]) Sellmeier terms; each is a lossless Lorentz pole."""
        poles = []
        for b, c_um2 in terms:
            w0 = 2.0 * math.pi * C_0 / (math.sqrt(c_um2) * 1e-6)
            poles.append(Pole(strength=b * w0 ** 2, omega0=w0, gamma=0.0))
        return cls(eps_inf=1.0, poles=tuple(poles), name=name)


# --------------------------------------------------------------------------- #
# Geometry
# --------------------------------------------------------------------------- #
def _pos3(x) -> Tuple[float, float, float]:
    x = tuple(float(v) for v in x)
    if not 1 <= len(x) <= 3:
        raise ValueError(f"Expected 1/2/3-tuple, got length {len(x)}")
    return x + (0.0,) * (3 - len(x))


def axis_span(coord: np.ndarray, lo: float, hi: float) -> Optional[Tuple[int, int]]:
    """Index range [i0, i1) of the ascending ``coord`` inside [lo, hi], or None.

    Equal to the boolean test ``(coord >= lo) & (coord <= hi)`` because cell
    coordinates are strictly increasing, but O(log n) per axis.
    """
    i0 = int(np.searchsorted(coord, lo, side="left"))
    i1 = int(np.searchsorted(coord, hi, side="right"))
    return (i0, i1) if i1 > i0 else None


@dataclass(frozen=True)
class Box:
    """Axis-aligned box; rasterises onto cells whose centre lies inside
    (closed interval). Later structures overwrite earlier ones."""
    center: Tuple[float, ...]
    size: Tuple[float, ...]
    medium: object

    def _bounds(self):
        c, s = _pos3(self.center), _pos3(self.size)
        return tuple((ci - si / 2, ci + si / 2) for ci, si in zip(c, s))

    def index_slices(self, grid) -> Optional[Tuple[slice, slice, slice]]:
        """The box's cells as one slice per axis, or None when empty.

        A one-cell axis is collapsed: the box covers it when its extent
        straddles 0 (or is exactly the point 0)."""
        out = []
        for a, (lo, hi) in enumerate(self._bounds()):
            co = grid.coords[a]
            if co.size == 1:
                if not (lo <= 0.0 <= hi or (lo == hi == 0.0)):
                    return None
                out.append(slice(0, 1))
                continue
            span = axis_span(co, lo, hi)
            if span is None:
                return None
            out.append(slice(*span))
        return tuple(out)

    def region_mask(self, grid) -> np.ndarray:
        mask = np.zeros(tuple(c.size for c in grid.coords), dtype=bool)
        sl = self.index_slices(grid)
        if sl is not None:
            mask[sl] = True
        return mask

    def stamp(self, grid, eps_r: np.ndarray) -> None:
        sl = self.index_slices(grid)
        if sl is not None:
            eps_r[sl] = self.medium.eps_r


# --------------------------------------------------------------------------- #
# Sources
# --------------------------------------------------------------------------- #
@dataclass(frozen=True)
class GaussianPulse:
    """exp(-((t-t0)/sigma)^2) sin(2 pi f0 (t-t0)); sigma from the intensity
    FWHM, t0 = 4 sigma + delay."""
    freq0: float
    fwhm: float
    delay: float = 0.0

    @property
    def sigma(self) -> float:
        return float(self.fwhm) / (2.0 * math.sqrt(2.0 * math.log(2.0)))

    @property
    def t0(self) -> float:
        return 4.0 * self.sigma + float(self.delay)

    @property
    def envelope_l2(self) -> float:
        return float(self.sigma) * math.sqrt(math.pi / 2.0)

    def __call__(self, t):
        t = np.asarray(t)
        envelope = np.exp(-((t - self.t0) / self.sigma) ** 2)
        carrier = np.sin(2.0 * math.pi * self.freq0 * (t - self.t0))
        return envelope * carrier


@dataclass(frozen=True)
class PointDipole:
    """Soft additive point source on one E or H component."""
    position: Tuple[float, ...]
    component: str
    waveform: GaussianPulse
    amplitude: float = 1.0


@dataclass(frozen=True)
class ModeSource:
    """Distributed soft source on an injection plane, one dipole per cell,
    amplitude ``amplitude * profile`` (profile coordinates relative to
    ``center``); the zero (or smallest) ``size`` axis is the propagation axis.
    """
    center: Tuple[float, float, float]
    size: Tuple[float, float, float]
    component: str
    waveform: GaussianPulse
    profile: np.ndarray
    profile_coords: Tuple[np.ndarray, ...]
    amplitude: float = 1.0

    def _propagation_axis(self) -> int:
        sizes = list(self.size) + [0.0] * (3 - len(self.size))
        zeros = [i for i, s in enumerate(sizes) if s == 0]
        return zeros[0] if zeros else int(np.argmin(sizes))

    def expand(self, grid: Grid) -> List[PointDipole]:
        center = list(self.center) + [0.0] * (3 - len(self.center))
        size = list(self.size) + [0.0] * (3 - len(self.size))
        prop = self._propagation_axis()
        tan = [a for a in range(3) if a != prop]
        idxs, pcs = [], []
        for ax in tan:
            c = grid.coords[ax]
            if c.size == 1:
                idxs.append(np.array([0]))
                pcs.append(np.array([0.0]))
                continue
            m = (c >= center[ax] - size[ax] / 2.0) & (c <= center[ax] + size[ax] / 2.0)
            if not m.any():
                raise ValueError(f"ModeSource injection plane has zero overlap on axis {ax}")
            idxs.append(np.flatnonzero(m))
            pcs.append(c[m])
        cp = grid.coords[prop]
        ip = 0 if cp.size == 1 else int(np.argmin(np.abs(cp - center[prop])))
        prof = np.asarray(self.profile)
        rel0 = pcs[0] - center[tan[0]]
        rel1 = (pcs[1] - center[tan[1]]) if len(tan) > 1 else pcs[1]
        if prof.ndim == 1:
            if len(self.profile_coords) != 1:
                raise ValueError("1-D profile requires one profile_coords array")
            v = np.interp(rel0, self.profile_coords[0], prof, left=0.0, right=0.0)
            interp = v[:, None] if (len(pcs) == 2 and pcs[1].size == 1) else v
        elif prof.ndim == 2:
            if len(self.profile_coords) != 2:
                raise ValueError("2-D profile requires two profile_coords arrays")
            rows = np.empty((prof.shape[0], pcs[1].size))
            for r in range(prof.shape[0]):
                rows[r] = np.interp(rel1, self.profile_coords[1], prof[r], left=0.0, right=0.0)
            interp = np.empty((pcs[0].size, pcs[1].size))
            for col in range(pcs[1].size):
                interp[:, col] = np.interp(rel0, self.profile_coords[0], rows[:, col],
                                           left=0.0, right=0.0)
        else:
            raise ValueError("profile must be 1-D or 2-D")
        if interp.ndim == 1:
            interp = interp[:, None]
        out = []
        for a, i1 in enumerate(idxs[0]):
            for b, i2 in enumerate(idxs[1] if len(idxs) > 1 else [0]):
                w = float(interp[a, b]) * float(self.amplitude)
                if w == 0.0:
                    continue
                pos = [0.0, 0.0, 0.0]
                pos[prop] = float(cp[ip] if cp.size > 1 else center[prop])
                c0 = grid.coords[tan[0]]
                pos[tan[0]] = float(c0[i1] if c0.size > 1 else center[tan[0]])
                if len(tan) > 1:
                    c1 = grid.coords[tan[1]]
                    pos[tan[1]] = float(c1[i2] if c1.size > 1 else center[tan[1]])
                out.append(PointDipole(position=tuple(pos), component=self.component,
                                       waveform=self.waveform, amplitude=w))
        return out


@dataclass(frozen=True)
class UniModeSource:
    """One-way launch of a solved waveguide mode along x (sources.py:341-433):
    an electric and a magnetic current sheet on the same plane (the
    equivalence principle: J = x x H_m, M = -x x E_m), whose radiation adds
    in ``direction`` and cancels behind it. ``mode`` is a ModeResult solved
    on the plane's own (y, z) cells; each cell becomes four soft dipoles,
        Ey: C Hz / (eps0 eps_r),  Ez: -C Hy / (eps0 eps_r),
        Hy: -s C Ez / mu0,        Hz:  s C Ey / mu0,
    with s = +1 for "+x", -1 for "-x", C = ``amplitude``, the mode's fields
    first rotated so that its largest transverse E entry is real, then taken
    real. Each mode cell maps to the nearest grid cell of the plane."""
    center: Tuple[float, float, float]
    size: Tuple[float, float, float]
    waveform: GaussianPulse
    mode: object
    mode_index: int = 0
    direction: str = "+x"
    amplitude: float = 1.0

    def expand(self, grid: Grid) -> List[PointDipole]:
        if self.direction not in ("+x", "-x"):
            raise ValueError("UniModeSource supports direction '+x' or '-x'")
        sgn = 1.0 if self.direction == "+x" else -1.0
        cen = list(self.center) + [0.0] * (3 - len(self.center))
        m, q = self.mode, self.mode_index
        ey, ez = np.asarray(m.Ey[q]), np.asarray(m.Ez[q])
        hy, hz = np.asarray(m.Hy[q]), np.asarray(m.Hz[q])
        peak = int(np.argmax(np.abs(ey) + np.abs(ez)))
        rot = np.exp(-1j * np.angle((ey.ravel() + ez.ravel())[peak]))
        ey, ez, hy, hz = (np.real(f * rot) for f in (ey, ez, hy, hz))
        eps = np.asarray(m.eps_r)
        amp = float(self.amplitude)
        sheets = (("Ey", amp / (EPS_0 * eps) * hz), ("Ez", -amp / (EPS_0 * eps) * hy),
                  ("Hy", -sgn * amp / MU_0 * ez), ("Hz", sgn * amp / MU_0 * ey))
        xc, yc, zc = grid.coords
        x = float(xc[int(np.argmin(np.abs(xc - cen[0])))] if xc.size > 1 else cen[0])
        out = []
        for jy, yv in enumerate(np.asarray(m.y)):
            y = float(yc[int(np.argmin(np.abs(yc - (cen[1] + yv))))] if yc.size > 1 else cen[1])
            for jz, zv in enumerate(np.asarray(m.z)):
                z = float(zc[int(np.argmin(np.abs(zc - (cen[2] + zv))))]
                          if zc.size > 1 else cen[2])
                for comp, a in sheets:
                    v = float(a[jy, jz])
                    if v != 0.0:
                        out.append(PointDipole(position=(x, y, z), component=comp,
                                               waveform=self.waveform, amplitude=v))
        return out


# --------------------------------------------------------------------------- #
# Monitors
# --------------------------------------------------------------------------- #
@dataclass
class FieldMonitor:
    """Snapshots of components every ``interval`` steps or at ``times``;
    ``downsample`` strides every axis; ``plane_z`` keeps one z plane."""
    name: str
    components: Tuple[str, ...] = ("Ez",)
    interval: Optional[int] = None
    times: Optional[Sequence[float]] = None
    downsample: int = 1
    plane_z: Optional[float] = None
    compression: object = None
    compression_bits: int = 8

    def __post_init__(self):
        if self.interval is None and self.times is None:
            self.interval = 1
        if self.interval is not None and self.times is not None:
            raise ValueError("Specify only one of interval or times")
        if int(self.downsample) != self.downsample or self.downsample < 1:
            raise ValueError("downsample must be a positive integer")
        self.downsample = int(self.downsample)
        if self.compression is not None and self.compression not in (True, "auto", "zstd", "zlib"):
            raise ValueError("compression must be None, True, 'zstd', or 'zlib', "
                             f"got {self.compression!r}")
        if self.compression_bits not in (8, 16):
            raise ValueError("compression_bits must be 8 or 16")


@dataclass
class DFTMonitor:
    """Running DFT F(omega) = sum f(t_n) exp(+i omega t_n) dt in complex128,
    each component at its own Yee time; optional plane restriction."""
    name: str
    components: Tuple[str, ...] = ("Ez",)
    freqs: Sequence[float] = ()
    interval: int = 1
    downsample: int = 1
    plane_z: Optional[float] = None
    plane_axis: Optional[str] = None
    plane_position: Optional[float] = None

    def __post_init__(self):
        self.freqs = tuple(float(f) for f in self.freqs)
        if len(self.freqs) == 0:
            raise ValueError("DFTMonitor requires at least one frequency in `freqs`")
        if int(self.interval) != self.interval or self.interval < 1:
            raise ValueError("interval must be a positive integer")
        self.interval = int(self.interval)
        if int(self.downsample) != self.downsample or self.downsample < 1:
            raise ValueError("downsample must be a positive integer")
        self.downsample = int(self.downsample)
        if self.plane_z is not None and self.plane_axis is None:
            self.plane_axis = "z"
            self.plane_position = self.plane_z
        if self.plane_axis is not None:
            if self.plane_axis not in ("x", "y", "z"):
                raise ValueError("plane_axis must be 'x', 'y', or 'z'")
            if self.plane_position is None:
                raise ValueError("plane_axis requires plane_position")

    def plane(self):
        if self.plane_axis is None:
            return None
        return ({"x": 0, "y": 1, "z": 2}[self.plane_axis], float(self.plane_position))


@dataclass
class FluxMonitor:
    """Poynting flux through the full plane normal to ``plane_axis``,
    time-integrated over the run."""
    name: str
    plane_axis: str
    plane_position: float


# --------------------------------------------------------------------------- #
# CPML
# --------------------------------------------------------------------------- #
@dataclass(frozen=True)
class CPMLParams:
    poly_order: int = 3
    sigma_factor: float = 0.8
    alpha_max: float = 0.24
    R_target: float = 1e-7


def cpml_coeffs_1axis(n_cells: int, cell_size: float, n_pml: int, dt: float,
                      params: CPMLParams = CPMLParams()):
    """(b_e, c_e, b_h, c_h) float64 arrays of length ``n_cells``, kappa = 1.

    sigma(u) = sigma_max u^m, alpha(u) = alpha_max (1 - u), u in [0, 1] the
    normalised depth into the layer; b = exp(-(sigma+alpha) dt/eps0),
    c = sigma/(sigma+alpha) (b - 1). E samples sit at integer cells, H at +1/2.
    """
    zero = np.zeros(n_cells)
    if n_pml == 0:
        return zero.copy(), zero.copy(), zero.copy(), zero.copy()
    m = params.poly_order
    s_max = params.sigma_factor * (
        -(m + 1) * np.log(params.R_target) / (2.0 * ETA_0 * n_pml * cell_size))

    def coeffs(u):
        sg = s_max * u ** m
        al = params.alpha_max * (1.0 - u)
        tot = sg + al
        b = np.exp(-(sg + al) * dt / EPS_0)
        c = np.zeros_like(sg)
        pos = tot > 0
        c[pos] = sg[pos] / tot[pos] * (b[pos] - 1.0)
        return b, c

    depth = max(n_pml - 1, 1)
    tabs = []
    for offset in (0.0, 0.5):
        x = np.arange(n_cells) + offset if offset else np.arange(n_cells)
        b_arr, c_arr = np.zeros(n_cells), np.zeros(n_cells)
        b, c = coeffs(np.clip((n_pml - 1 - x[:n_pml]) / depth, 0.0, 1.0))
        b_arr[:n_pml], c_arr[:n_pml] = b, c
        b, c = coeffs(np.clip((x[-n_pml:] - (n_cells - n_pml)) / depth, 0.0, 1.0))
        b_arr[-n_pml:], c_arr[-n_pml:] = b, c
        tabs += [b_arr, c_arr]
    return tabs[0], tabs[1], tabs[2], tabs[3]
