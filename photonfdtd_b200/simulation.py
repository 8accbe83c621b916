"""``Simulation`` front end with ``backend="b200"``.

Same constructor, attributes and ``run()`` contract as the reference
``photonfdtd.Simulation`` (src/photonfdtd/simulation.py:361-530) for the
time-stepping path: precision resolution (:279-324), source expansion
(:474-488), permittivity stamping (:539-544), Courant dt and step count
(:522-528), CPML coefficients (:794-808). ``run()`` executes on the B200
engine (photonfdtd_b200.engine.run_b200); there is no CPU path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .scene import (C_0, CPMLParams, DFTMonitor, FieldMonitor, FluxMonitor, PointDipole,
                    cpml_coeffs_1axis)

_FIELD_KEYS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_E_KEYS = ("Ex", "Ey", "Ez")
_ARRAY_KEYS = _FIELD_KEYS + ("eps_r", "psi", "monitors")
_COMPUTE_KEYS = _FIELD_KEYS + ("eps_r", "psi")
_GROUP_ALIASES = ("default", "compute", "fields", "e_fields", "h_fields")
_VALID_DTYPES = {"float32": np.float32, "float64": np.float64}
BACKENDS = ("b200", "auto")


def resolve_precision(precision) -> Dict[str, type]:
    """{array key: dtype} from a dtype string or a per-array dict; the most
    specific key wins (array > e_fields/h_fields > fields > compute > default)."""
    if isinstance(precision, str):
        if precision not in _VALID_DTYPES:
            raise ValueError("precision must be 'float32' or 'float64'")
        d = _VALID_DTYPES[precision]
        return {k: d for k in _ARRAY_KEYS}
    if not isinstance(precision, dict):
        raise TypeError("precision must be a str ('float32'/'float64') or a dict mapping "
                        "array keys to dtype strings")
    allowed = set(_ARRAY_KEYS) | set(_GROUP_ALIASES)
    unknown = set(precision) - allowed
    if unknown:
        raise ValueError(f"unknown precision key(s) {sorted(unknown)}; "
                         f"allowed keys: {sorted(allowed)}")
    for k, v in precision.items():
        if v not in _VALID_DTYPES:
            raise ValueError(f"precision[{k!r}] must be 'float32' or 'float64', got {v!r}")

    def pick(*keys, fallback):
        for k in keys:
            if k in precision:
                return _VALID_DTYPES[precision[k]]
        return fallback

    default = _VALID_DTYPES[precision.get("default", "float64")]
    out = {}
    for k in _FIELD_KEYS:
        grp = "e_fields" if k in _E_KEYS else "h_fields"
        out[k] = pick(k, grp, "fields", "compute", fallback=default)
    out["eps_r"] = pick("eps_r", "compute", fallback=default)
    out["psi"] = pick("psi", "compute", fallback=default)
    out["monitors"] = pick("monitors", fallback=default)
    return out


@dataclass
class Result:
    times: np.ndarray
    fields: Dict[str, Dict[str, np.ndarray]] = field(default_factory=dict)
    monitor_times: Dict[str, np.ndarray] = field(default_factory=dict)
    flux: Dict[str, float] = field(default_factory=dict)
    dft: Dict[str, Dict[str, np.ndarray]] = field(default_factory=dict)
    dft_freqs: Dict[str, np.ndarray] = field(default_factory=dict)


class Simulation:
    """A photonfdtd simulation stepped on the B200 engine.

    Arguments as the reference's; ``backend`` is "b200" (or "auto", which
    means the same here). ``use_gpu``/``use_numba``/``use_jax`` select other
    engines in the reference and are rejected here.
    """

    def __init__(self, grid, structures: Sequence = (), sources: Sequence = (),
                 monitors: Sequence = (), run_time: float = 1e-12, courant: float = 0.99,
                 cpml_params: CPMLParams = CPMLParams(), verbose: bool = False,
                 use_gpu: bool = False, use_numba: bool = False, use_jax: bool = False,
                 precision="float64", subpixel: bool = False, subpixel_factor: int = 3,
                 backend: str = "b200") -> None:
        self.precision = precision
        self.dtypes = resolve_precision(precision)
        self.dtype = self.dtypes["Ex"]
        if use_gpu or use_numba or use_jax:
            raise NotImplementedError(
                "use_gpu / use_numba / use_jax select engines of the reference package; "
                "photonfdtd_b200 always steps on the B200 engine.")
        if backend not in BACKENDS:
            raise ValueError(f"backend must be one of {BACKENDS}")
        self.backend = backend
        self.use_gpu = self.use_numba = self.use_jax = False
        self.subpixel = bool(subpixel)
        self.subpixel_factor = int(subpixel_factor)
        self.grid = grid
        self.structures = list(structures)
        self._has_dispersion = any(getattr(getattr(s, "medium", None), "is_dispersive", False)
                                   for s in self.structures)
        if self._has_dispersion and self.subpixel:
            raise NotImplementedError("Subpixel smoothing combined with dispersive media is "
                                      "not yet supported. Use one or the other.")
        self.particle_sources: List = []
        self.sources: List[PointDipole] = []
        for s in sources:
            self.add_source(s)
        self.monitors = list(monitors)
        self.run_time = float(run_time)
        self.courant = float(courant)
        self.cpml_params = cpml_params
        self.verbose = verbose
        self.progress_callback: Optional[Callable[[int, int], None]] = None
        self._eps_r: Optional[np.ndarray] = None
        self._eps_r_custom = False
        inv_dl2 = 0.0
        for d in grid.cell_size:
            if d > 0:
                inv_dl2 += 1.0 / d ** 2
        self.dt = self.courant / (C_0 * math.sqrt(inv_dl2))
        self.n_steps = int(math.ceil(self.run_time / self.dt))
        self._build_cpml()

    # ---- sources / monitors ---- #
    def add_source(self, source) -> None:
        if isinstance(source, PointDipole) or type(source).__name__ == "PointDipole":
            self.sources.append(source)
        elif type(source).__name__ == "ChargedParticle":
            self.particle_sources.append(source)
        elif hasattr(source, "expand"):
            self.sources.extend(source.expand(self.grid))
        else:
            raise TypeError(f"Unsupported source type: {type(source).__name__}")

    def add_monitor(self, monitor) -> None:
        self.monitors.append(monitor)

    # ---- permittivity ---- #
    def _materialize_eps_r(self) -> np.ndarray:
        eps = np.ones(self.grid.shape, dtype=self.dtypes["eps_r"])
        for s in self.structures:
            s.stamp(self.grid, eps)
        self._eps_r = eps
        return eps

    @property
    def eps_r(self) -> np.ndarray:
        if self._eps_r is None:
            self._materialize_eps_r()
        return self._eps_r

    @eps_r.setter
    def eps_r(self, value) -> None:
        self._eps_r = value
        self._eps_r_custom = True

    def _smoothed_eps_components(self):
        from .smoothing import smooth_permittivity
        if self._eps_r_custom:
            eps = self.eps_r
            return (eps, eps, eps)
        from .smoothing import device_available, smooth_permittivity_device
        if device_available() and all(hasattr(st, "index_slices") for st in self.structures):
            # on the GPU, bit for bit the host result (boxes only)
            return smooth_permittivity_device(self.grid, self.structures, background_eps=1.0,
                                              factor=self.subpixel_factor,
                                              dtype=self.dtypes["eps_r"])
        return smooth_permittivity(self.grid, self.structures, background_eps=1.0,
                                   factor=self.subpixel_factor, dtype=self.dtypes["eps_r"])

    # ---- CPML (simulation.py:794-808) ---- #
    def _build_cpml(self) -> None:
        be, ce, bh, ch = [], [], [], []
        for ax in range(3):
            n = self.grid.shape[ax]
            dl = self.grid.cell_size[ax]
            npml = self.grid.pml_layers[ax] if n > 1 else 0
            b_e, c_e, b_h, c_h = cpml_coeffs_1axis(n, dl if n > 1 else 1.0, npml, self.dt,
                                                   self.cpml_params)
            be.append(b_e)
            ce.append(c_e)
            bh.append(b_h)
            ch.append(c_h)
        self._b_e, self._c_e, self._b_h, self._c_h = be, ce, bh, ch

    # ---- run ---- #
    def run(self, out_of_core: bool = False, tile_cells=None, ooc_workdir=None) -> Result:
        if out_of_core:
            raise NotImplementedError(
                "out_of_core is not needed on the b200 backend: the whole domain "
                "stays resident in device memory.")
        from .engine import run_b200
        return run_b200(self)
