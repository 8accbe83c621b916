"""NumPy restatement of photonfdtd's Yee + CPML + ADE time step (oracle).

TEST INFRASTRUCTURE: the checker the CUDA engine is compared against. It is
never part of the product path; see ``oracle/__init__.py`` for who may import
it.

Every function names the reference code it restates (paths relative to the
ngpaladi/photonfdtd v0.12.0 tree). The arithmetic keeps the reference's
expression order, so on the same inputs a float32 or float64 run of this
oracle reproduces the reference NumPy path to the last bit; the golden
fixtures in ``tests/golden`` (written by the reference itself) pin that.

The oracle reads scene objects by duck typing only: anything carrying the
reference's attribute names (``grid.size/cell_size/pml_layers``,
``structures[*].center/size/medium``, ``sources[*].position/component/
waveform/amplitude``, monitor fields) works, whether it came from the
reference package or from ``photonfdtd_b200``. No scene method is called:
grids, masks, coefficients and waveforms are all recomputed here.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# Physical constants (src/photonfdtd/constants.py:4-7).
C0 = 299_792_458.0
EPS0 = 8.854_187_8128e-12
MU0 = 1.256_637_062_12e-6
ETA0 = math.sqrt(MU0 / EPS0)

_COMP_INDEX = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5}


# --------------------------------------------------------------------------- #
# Grid geometry (src/photonfdtd/grid.py:28-64, 82-96)
# --------------------------------------------------------------------------- #
def _pad3(x, fill):
    if x is None:
        return (fill, fill, fill)
    if isinstance(x, (int, float)):
        return (x, x, x)
    x = tuple(x)
    return x + (fill,) * (3 - len(x))


class OGrid:
    """Shape, coordinates and spacing of a uniform Yee grid (grid.py:28-64).

    Axes whose size is 0/None collapse to one cell at coordinate 0. Cell
    coordinates are ``(arange(n) - (n-1)/2) * d``.
    """

    def __init__(self, size, cell_size, pml_layers):
        size3 = _pad3(size, None)
        cs3 = _pad3(cell_size, None)
        pml3 = _pad3(pml_layers, 0)
        shape, coords, pml, cell = [], [], [], []
        for s, d, p in zip(size3, cs3, pml3):
            cell.append(0.0 if d is None else float(d))
            if s is None or s == 0:
                shape.append(1)
                coords.append(np.array([0.0]))
                pml.append(0)
                continue
            n = int(round(s / d))
            shape.append(n)
            coords.append((np.arange(n) - (n - 1) / 2) * d)
            pml.append(int(p))
        self.shape = tuple(shape)
        self.coords = tuple(coords)
        self.pml_layers = tuple(pml)
        self.cell_size = tuple(cell)
        self.size = tuple(0.0 if s is None else float(s) for s in size3)

    def index_at(self, point) -> Tuple[int, int, int]:
        """Nearest cell per axis; ties resolve to the lower index (grid.py:82-96)."""
        pt = list(point) + [0.0] * (3 - len(point))
        out = []
        for a in range(3):
            c = self.coords[a]
            out.append(0 if c.size == 1 else int(np.argmin(np.abs(c - pt[a]))))
        return tuple(out)


def grid_of(g) -> OGrid:
    return OGrid(g.size, g.cell_size, g.pml_layers)


# --------------------------------------------------------------------------- #
# Box rasterisation (src/photonfdtd/geometry.py:38-53)
# --------------------------------------------------------------------------- #
def _geom3(x):
    x = tuple(float(v) for v in x)
    return x + (0.0,) * (3 - len(x))


def box_mask(box, coords, shape) -> np.ndarray:
    """Cells whose centre lies in the closed box (geometry.py:44-60).

    A one-element coordinate array takes the collapsed-axis branch (the box
    must straddle 0), exactly as the reference does, including on the
    one-cell-wide fine slabs the subpixel builder makes when factor == 1.
    """
    c = _geom3(box.center)
    s = _geom3(box.size)
    mask = np.ones(shape, dtype=bool)
    for a in range(3):
        lo, hi = c[a] - s[a] / 2, c[a] + s[a] / 2
        co = coords[a]
        if co.size == 1:
            if not (lo <= 0.0 <= hi or (lo == hi == 0.0)):
                return np.zeros(shape, dtype=bool)
            m = np.array([True])
        else:
            m = (co >= lo) & (co <= hi)
        sh = [1, 1, 1]
        sh[a] = m.size
        mask &= m.reshape(sh)
    return mask


def box_slices(box, coords):
    """The cells of box_mask as one index range per axis (None if empty).

    Same cells as the boolean test: coordinates are strictly increasing, so
    (co >= lo) & (co <= hi) is the run searchsorted(lo, left) ..
    searchsorted(hi, right). Lets the oracle stamp the 110,592 blocks of the
    full-size dispersive workload without a full-grid mask per block.
    """
    c = _geom3(box.center)
    s = _geom3(box.size)
    out = []
    for a in range(3):
        lo, hi = c[a] - s[a] / 2, c[a] + s[a] / 2
        co = coords[a]
        if co.size == 1:
            if not (lo <= 0.0 <= hi or (lo == hi == 0.0)):
                return None
            out.append(slice(0, 1))
            continue
        i0 = int(np.searchsorted(co, lo, side="left"))
        i1 = int(np.searchsorted(co, hi, side="right"))
        if i1 <= i0:
            return None
        out.append(slice(i0, i1))
    return tuple(out)


def _cells_of(s, grid):
    sl = box_slices(s, grid.coords)
    return sl


def _medium_eps(med) -> float:
    if getattr(med, "is_dispersive", False):
        return float(med.eps_inf)
    return float(med.eps_r) if hasattr(med, "eps_r") else float(med.permittivity)


def stamp_eps(grid: OGrid, structures, dtype) -> np.ndarray:
    """Permittivity grid, later structures overwrite (simulation.py:539-544)."""
    eps = np.ones(grid.shape, dtype=dtype)
    for s in structures:
        sl = _cells_of(s, grid)
        if sl is not None:
            eps[sl] = _medium_eps(s.medium)
    return eps


# --------------------------------------------------------------------------- #
# Subpixel smoothing (src/photonfdtd/smoothing.py:75-172)
# --------------------------------------------------------------------------- #
def smooth_eps(grid: OGrid, structures, factor: int, dtype):
    """Diagonal anisotropic subpixel permittivity (smoothing.py:119-172).

    Arithmetic and harmonic means over ``factor`` sub-cells per active axis,
    built one native x-slab at a time; normal from ``np.gradient`` of the
    arithmetic mean.
    """
    nx, ny, nz = grid.shape
    fine = OGrid(grid.size, tuple((c / factor) if c > 0 else 0.0
                                  for c in grid.cell_size), (0, 0, 0))
    xf, yf, zf = fine.coords
    fx = factor if nx > 1 else 1
    fy = factor if ny > 1 else 1
    fz = factor if nz > 1 else 1
    eps_a = np.empty(grid.shape, dtype=np.float64)
    eps_h = np.empty(grid.shape, dtype=np.float64)
    for i in range(nx):
        xs = xf[i * fx:(i + 1) * fx]
        sub_coords = (xs, yf, zf)
        sub_shape = (xs.size, yf.size, zf.size)
        sub = np.full(sub_shape, 1.0, dtype=np.float64)
        for s in structures:
            sub[box_mask(s, sub_coords, sub_shape)] = _medium_eps(s.medium)
        r = sub.reshape(1, fx, ny, fy, nz, fz)
        eps_a[i] = r.mean(axis=(1, 3, 5))[0]
        eps_h[i] = (1.0 / (1.0 / r).mean(axis=(1, 3, 5)))[0]
    spac = [grid.cell_size[a] if grid.shape[a] > 1 else 1.0 for a in range(3)]
    grads = [np.gradient(eps_a, spac[a], axis=a) if grid.shape[a] > 1
             else np.zeros_like(eps_a) for a in range(3)]
    gmag = np.sqrt(grads[0] ** 2 + grads[1] ** 2 + grads[2] ** 2)
    tiny = gmag.max() * 1e-9 if gmag.size else 0.0
    ok = gmag > max(tiny, np.finfo(np.float64).tiny)
    inv = np.where(ok, 1.0 / np.where(ok, gmag, 1.0), 0.0)
    nrm = [g * inv for g in grads]
    delta = eps_h - eps_a
    return tuple((eps_a + delta * nrm[a] ** 2).astype(dtype, copy=False)
                 for a in range(3))


# --------------------------------------------------------------------------- #
# CPML coefficients (src/photonfdtd/boundaries.py:31-97)
# --------------------------------------------------------------------------- #
def cpml_axis(n, dl, npml, dt, m=3, sigma_factor=0.8, alpha_max=0.24,
              r_target=1e-7):
    """(b_e, c_e, b_h, c_h) along one axis, kappa = 1 (boundaries.py:31-97).

    Polynomial sigma grade of order ``m``, linear alpha grade; E samples at
    integer cells, H at +1/2. Zero outside the two slabs.
    """
    if npml == 0:
        z = np.zeros(n)
        return z.copy(), z.copy(), z.copy(), z.copy()
    smax = sigma_factor * (-(m + 1) * np.log(r_target) / (2.0 * ETA0 * npml * dl))

    def bc(u):
        sig = smax * u ** m
        alp = alpha_max * (1.0 - u)
        den = sig + alp
        b = np.exp(-(sig + alp) * dt / EPS0)
        c = np.zeros_like(sig)
        ok = den > 0
        c[ok] = sig[ok] / den[ok] * (b[ok] - 1.0)
        return b, c

    out = [np.zeros(n) for _ in range(4)]
    ie = np.arange(n)
    ih = np.arange(n) + 0.5
    span = max(npml - 1, 1)
    for stag, pos in ((0, ie), (1, ih)):
        lo = np.clip((npml - 1 - pos[:npml]) / span, 0.0, 1.0)
        hi = np.clip((pos[-npml:] - (n - npml)) / span, 0.0, 1.0)
        b, c = bc(lo)
        out[2 * stag][:npml], out[2 * stag + 1][:npml] = b, c
        b, c = bc(hi)
        out[2 * stag][-npml:], out[2 * stag + 1][-npml:] = b, c
    return out[0], out[1], out[2], out[3]


# --------------------------------------------------------------------------- #
# Sources (src/photonfdtd/sources.py:39-78)
# --------------------------------------------------------------------------- #
def gaussian_pulse(wave, t):
    """exp(-((t-t0)/sigma)^2) * sin(2 pi f0 (t-t0)), t0 = 4 sigma + delay
    (sources.py:51-69)."""
    sigma = float(wave.fwhm) / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    t0 = 4.0 * sigma + float(getattr(wave, "delay", 0.0))
    t = np.asarray(t)
    env = np.exp(-((t - t0) / sigma) ** 2)
    car = np.sin(2.0 * math.pi * wave.freq0 * (t - t0))
    return env * car


# --------------------------------------------------------------------------- #
# Precision (src/photonfdtd/simulation.py:279-324), uniform compute only
# --------------------------------------------------------------------------- #
_DT = {"float32": np.float32, "float64": np.float64}


def resolve_precision(precision) -> Tuple[type, type]:
    """(compute dtype, monitor dtype). The oracle covers the uniform-compute
    case (every field, eps_r and psi in one dtype), which is what the engine
    accepts too."""
    if isinstance(precision, str):
        d = _DT[precision]
        return d, d
    default = precision.get("default", "float64")
    keys = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "eps_r", "psi")
    groups = {"Ex": "e_fields", "Ey": "e_fields", "Ez": "e_fields",
              "Hx": "h_fields", "Hy": "h_fields", "Hz": "h_fields"}
    seen = set()
    for k in keys:
        order = [k]
        if k in groups:
            order += [groups[k], "fields"]
        order += ["compute"]
        v = next((precision[o] for o in order if o in precision), default)
        seen.add(v)
    if len(seen) != 1:
        raise NotImplementedError("oracle covers uniform compute precision only")
    return _DT[seen.pop()], _DT[precision.get("monitors", default)]


# --------------------------------------------------------------------------- #
# Scene tables
# --------------------------------------------------------------------------- #
def _cls(o) -> str:
    return type(o).__name__


def scene_tables(sim, ce3=None) -> dict:
    """Everything the step loop consumes, rebuilt from the scene alone.

    Courant dt and step count (simulation.py:522-528), ce / per-component ce
    (:953-969), ch (:954), CPML (:794-808), ADE media (:572-636). ``ce3``, if
    given, replaces the subpixel per-component coefficients (a test that has
    them already, pinned elsewhere, skips the host smoothing of a large grid).
    """
    grid = grid_of(sim.grid)
    dtype, mon_dtype = resolve_precision(sim.precision)
    courant = float(getattr(sim, "courant", 0.99))
    inv = 0.0
    for d in grid.cell_size:
        if d > 0:
            inv += 1.0 / d ** 2
    dt = courant / (C0 * math.sqrt(inv))
    n_steps = int(math.ceil(float(sim.run_time) / dt))
    cp = getattr(sim, "cpml_params", None)
    cpkw = {}
    if cp is not None:
        cpkw = dict(m=cp.poly_order, sigma_factor=cp.sigma_factor,
                    alpha_max=cp.alpha_max, r_target=cp.R_target)
    cpml = []
    for a in range(3):
        n = grid.shape[a]
        cpml.append(cpml_axis(n, grid.cell_size[a] if n > 1 else 1.0,
                              grid.pml_layers[a] if n > 1 else 0, dt, **cpkw))
    structures = list(sim.structures)
    custom = bool(getattr(sim, "_eps_r_custom", False))
    # a caller-assigned permittivity grid replaces stamping and smoothing
    # (simulation.py:953, :508-518 of the reference's eps_r setter)
    eps = np.asarray(sim.eps_r) if custom else stamp_eps(grid, structures, dtype)
    ce = (dt / (eps * EPS0)).astype(dtype, copy=False)
    if ce3 is not None:
        ce3 = tuple(np.asarray(c, dtype=dtype) for c in ce3)
    elif custom:
        ce3 = (ce, ce, ce)
    elif getattr(sim, "subpixel", False):
        comps = smooth_eps(grid, structures, int(sim.subpixel_factor), dtype)
        ce3 = tuple((dt / (e * EPS0)).astype(dtype, copy=False) for e in comps)
    else:
        ce3 = (ce, ce, ce)
    return dict(grid=grid, dtype=dtype, mon_dtype=mon_dtype, dt=dt,
                n_steps=n_steps, cpml=cpml, ce=ce, ce3=ce3,
                ch=dtype(dt / MU0), eps=eps, structures=structures)


def ade_media(grid: OGrid, structures, dt):
    """Dispersive media, their cells and pole recursion coefficients
    (simulation.py:572-636). Returns a list of dicts, one per distinct medium
    object in first-use order."""
    ids = np.full(grid.shape, -1, dtype=np.int32)
    media, seen = [], {}
    for s in structures:
        med = s.medium
        mk = _cells_of(s, grid)
        if mk is None:
            continue
        if getattr(med, "is_dispersive", False):
            if id(med) not in seen:
                seen[id(med)] = len(media)
                media.append(med)
            ids[mk] = seen[id(med)]
        else:
            ids[mk] = -1
    wmax = 0.0
    for med in media:
        wmax = max(wmax, max((p.omega0 for p in med.poles), default=0.0) * dt)
    if wmax >= 2.0:
        raise ValueError(f"pole with omega0*dt = {wmax:.2f} >= 2 is unstable")
    out = []
    for mid, med in enumerate(media):
        idx = np.nonzero(ids == mid)
        if idx[0].size == 0:
            continue
        abc = []
        for p in med.poles:
            den = 1.0 + p.gamma * dt
            abc.append(((2.0 - p.omega0 ** 2 * dt ** 2) / den,
                        (p.gamma * dt - 1.0) / den,
                        (EPS0 * p.strength * dt ** 2) / den))
        out.append(dict(idx=idx, abc=abc, inv=1.0 / (EPS0 * med.eps_inf)))
    return out


# --------------------------------------------------------------------------- #
# The stepper
# --------------------------------------------------------------------------- #
# (field, aligned axis, (axis, source) of the + term, (axis, source) of the - term)
_CURL = (
    ("Hx", 0, (1, "Ez"), (2, "Ey")),
    ("Hy", 1, (2, "Ex"), (0, "Ez")),
    ("Hz", 2, (0, "Ey"), (1, "Ex")),
    ("Ex", 0, (1, "Hz"), (2, "Hy")),
    ("Ey", 1, (2, "Hx"), (0, "Hz")),
    ("Ez", 2, (0, "Hy"), (1, "Hx")),
)


def _runs(mask1d):
    """Maximal runs of True as (start, stop) (simulation.py:223-241)."""
    idx = np.flatnonzero(mask1d)
    if idx.size == 0:
        return []
    cuts = np.flatnonzero(np.diff(idx) != 1)
    starts = np.concatenate(([idx[0]], idx[cuts + 1]))
    stops = np.concatenate((idx[cuts] + 1, [idx[-1] + 1]))
    return list(zip(starts.tolist(), stops.tolist()))


class OracleRun:
    """Stateful oracle run; ``advance(n)`` steps, ``result()`` assembles.

    The per-step order is the reference's (simulation.py:1319-1406): H curl
    + CPML, H sources at (n+1/2)dt, capture E^n, E curl + CPML, ADE, E sources
    at (n+1)dt, then FieldMonitor / DFTMonitor / FluxMonitor in list order.
    """

    def __init__(self, sim, n_steps: Optional[int] = None, ce3=None):
        t = scene_tables(sim, ce3=ce3)
        self.t = t
        g: OGrid = t["grid"]
        self.grid = g
        self.dtype = t["dtype"]
        self.dt = t["dt"]
        self.n_steps = t["n_steps"] if n_steps is None else int(n_steps)
        self.shape = g.shape
        dt_ = self.dtype
        self.F = {c: np.zeros(g.shape, dtype=dt_) for c in _COMP_INDEX}
        self.dl = tuple(d if d > 0 else 1.0 for d in g.cell_size)
        self._build_updates()
        self.ade = ade_media(g, t["structures"], self.dt)
        for st in self.ade:
            npole = len(st["abc"])
            n = st["idx"][0].size
            st["cur"] = [[np.zeros(n, dt_) for _ in range(3)] for _ in range(npole)]
            st["prev"] = [[np.zeros(n, dt_) for _ in range(3)] for _ in range(npole)]
        self.sources = []
        for s in sim.sources:
            self.sources.append((s, _COMP_INDEX[s.component], g.index_at(s.position)))
        self.monitors = list(sim.monitors)
        self._init_monitors()
        self.step = 0

    # ---- update tables (simulation.py:1184-1232) ---- #
    def _crop(self, a, low):
        if self.shape[a] <= 1:
            return slice(None)
        return slice(1, None) if low else slice(0, -1)

    def _build_updates(self):
        t = self.t
        self.updates = []
        for name, al, (axa, sa), (axb, sb) in _CURL:
            is_e = name[0] == "E"
            reg = [slice(None)] * 3
            reg[axa] = self._crop(axa, is_e)
            reg[axb] = self._crop(axb, is_e)
            reg = tuple(reg)
            rshape = self.F[name][reg].shape
            k_arr = t["ce3"][al][reg] if is_e else None
            k_sc = None if is_e else -t["ch"]
            terms = []
            for ax, src, oax, sign in ((axa, sa, axb, 1.0), (axb, sb, axa, -1.0)):
                if self.shape[ax] <= 1:
                    continue
                b_all, c_all = (t["cpml"][ax][0], t["cpml"][ax][1]) if is_e else \
                    (t["cpml"][ax][2], t["cpml"][ax][3])
                cs = self._crop(ax, is_e)
                b1, c1 = b_all[cs], c_all[cs]
                slabs = []
                for s0, s1 in _runs(c1 != 0.0):
                    sl = [slice(None)] * 3
                    sl[ax] = slice(s0, s1)
                    rs = [1, 1, 1]
                    rs[ax] = s1 - s0
                    ps = list(rshape)
                    ps[ax] = s1 - s0
                    slabs.append((tuple(sl),
                                  np.asarray(b1[s0:s1], dtype=self.dtype).reshape(rs),
                                  np.asarray(c1[s0:s1], dtype=self.dtype).reshape(rs),
                                  np.zeros(ps, dtype=self.dtype)))
                terms.append((ax, src, oax, sign, slabs))
            self.updates.append((name, reg, k_arr, k_sc, is_e, terms))

    def _deriv(self, arr, ax):
        hi = [slice(None)] * 3
        lo = [slice(None)] * 3
        hi[ax] = slice(1, None)
        lo[ax] = slice(0, -1)
        return (arr[tuple(hi)] - arr[tuple(lo)]) / self.dl[ax]

    def _apply(self, family):
        F = self.F
        for name, reg, k_arr, k_sc, is_e, terms in self.updates:
            if (name[0] == "E") != (family == "E"):
                continue
            ds = []
            for ax, src, oax, sign, slabs in terms:
                d = self._deriv(F[src], ax)
                if self.shape[oax] > 1:
                    o = [slice(None)] * 3
                    o[oax] = self._crop(oax, is_e)
                    d = d[tuple(o)]
                ds.append(d)
            if not ds:
                continue
            curl = None
            for (ax, src, oax, sign, slabs), d in zip(terms, ds):
                if curl is None:
                    curl = d.copy() if sign > 0 else np.negative(d)
                elif sign > 0:
                    np.add(curl, d, out=curl)
                else:
                    np.subtract(curl, d, out=curl)
            np.multiply(curl, k_arr if is_e else k_sc, out=curl)
            freg = F[name][reg]
            freg += curl
            for (ax, src, oax, sign, slabs), d in zip(terms, ds):
                for sl, bb, cc, psi in slabs:
                    psi[...] = bb * psi + cc * d[sl]
                    k = k_arr[sl] if is_e else k_sc
                    freg[sl] += sign * k * psi

    # ---- ADE (simulation.py:638-669) ---- #
    def _ade_capture(self):
        for st in self.ade:
            st["En"] = [self.F[c][st["idx"]].copy() for c in ("Ex", "Ey", "Ez")]

    def _ade_apply(self):
        for st in self.ade:
            for c, name in enumerate(("Ex", "Ey", "Ez")):
                en = st["En"][c]
                delta = None
                for p, (a, b, cc) in enumerate(st["abc"]):
                    pc = st["cur"][p][c]
                    pp = st["prev"][p][c]
                    pn = a * pc + b * pp + cc * en
                    inc = pn - pc
                    delta = inc if delta is None else delta + inc
                    st["prev"][p][c] = pc
                    st["cur"][p][c] = pn
                if delta is not None:
                    self.F[name][st["idx"]] -= st["inv"] * delta

    # ---- sources (simulation.py:1367-1390) ---- #
    def _inject(self, family, t):
        for s, ci, (i, j, k) in self.sources:
            if s.component[0] != family:
                continue
            val = s.amplitude * gaussian_pulse(s.waveform, np.array([t]))[0]
            self.F[s.component][i, j, k] += val

    # ---- monitors (simulation.py:1001-1133, 1440-1459) ---- #
    def _init_monitors(self):
        g, n = self.grid, self.n_steps
        self.fm, self.dm, self.flux = {}, {}, {}
        for m in self.monitors:
            kind = _cls(m)
            if kind == "FieldMonitor":
                if m.times is not None:
                    steps = {int(round(tt / self.dt)) for tt in m.times}
                else:
                    steps = set(range(0, n, m.interval))
                zsl = slice(None)
                if m.plane_z is not None:
                    zi = int(np.argmin(np.abs(np.asarray(g.coords[2]) - m.plane_z)))
                    zsl = slice(zi, zi + 1)
                self.fm[m.name] = dict(m=m, steps=steps, zsl=zsl, frames={c: [] for c in m.components},
                                       times=[])
            elif kind == "DFTMonitor":
                pl = None
                if m.plane_axis is not None:
                    ax = {"x": 0, "y": 1, "z": 2}[m.plane_axis]
                    ci = int(np.argmin(np.abs(np.asarray(g.coords[ax]) - float(m.plane_position))))
                    pl = (ax, ci)
                self.dm[m.name] = dict(m=m, steps=set(range(0, n, m.interval)), plane=pl,
                                       omega=2.0 * np.pi * np.asarray(m.freqs, dtype=np.float64),
                                       acc={c: None for c in m.components})
            elif kind == "FluxMonitor":
                self.flux[m.name] = 0.0

    def _snap(self, arr, ds, zsl):
        if zsl != slice(None):
            return arr[::ds, ::ds, zsl]
        if ds > 1:
            return arr[::ds, ::ds, ::ds]
        return arr

    def _flux(self, m) -> float:
        F, g = self.F, self.grid
        ax = {"x": 0, "y": 1, "z": 2}[m.plane_axis]
        co = g.coords[ax]
        i = 0 if co.size == 1 else int(np.argmin(np.abs(co - m.plane_position)))
        w = [g.cell_size[a] if g.shape[a] > 1 else 1.0 for a in range(3)]
        if ax == 0:
            s = F["Ey"][i] * F["Hz"][i] - F["Ez"][i] * F["Hy"][i]
            da = w[1] * w[2]
        elif ax == 1:
            s = F["Ez"][:, i] * F["Hx"][:, i] - F["Ex"][:, i] * F["Hz"][:, i]
            da = w[0] * w[2]
        else:
            s = F["Ex"][:, :, i] * F["Hy"][:, :, i] - F["Ey"][:, :, i] * F["Hx"][:, :, i]
            da = w[0] * w[1]
        return float(np.sum(s) * da)

    def _record(self, step):
        t_e = (step + 1.0) * self.dt
        t_h = (step + 0.5) * self.dt
        for m in self.monitors:
            kind = _cls(m)
            if kind == "FieldMonitor":
                st = self.fm[m.name]
                if step in st["steps"]:
                    for c in m.components:
                        st["frames"][c].append(self._snap(self.F[c], m.downsample, st["zsl"]).copy())
                    st["times"].append(step * self.dt)
            elif kind == "DFTMonitor":
                st = self.dm[m.name]
                if step in st["steps"]:
                    ds = m.downsample
                    for c in m.components:
                        sl = [slice(None, None, ds) if ds > 1 else slice(None)] * 3
                        if st["plane"] is not None:
                            ax, ci = st["plane"]
                            sl[ax] = slice(ci, ci + 1)
                        snap = self.F[c][tuple(sl)]
                        t = t_e if c[0] == "E" else t_h
                        ph = np.exp(1j * st["omega"] * t).reshape((-1,) + (1,) * snap.ndim)
                        if st["acc"][c] is None:
                            st["acc"][c] = np.zeros((st["omega"].size,) + snap.shape,
                                                    dtype=np.complex128)
                        st["acc"][c] += ph * snap[None, ...] * self.dt
            elif kind == "FluxMonitor":
                self.flux[m.name] += self._flux(m) * self.dt

    # ---- driver ---- #
    def set_fields(self, fields: Dict[str, np.ndarray]) -> None:
        """Replace field components of the current state (the engine's
        pf_write_field); CPML psi and polarisation state are left as they are."""
        for c, arr in fields.items():
            self.F[c][...] = np.asarray(arr, dtype=self.dtype)

    def advance(self, n: int) -> None:
        for _ in range(int(n)):
            s = self.step
            self._apply("H")
            self._inject("H", (s + 0.5) * self.dt)
            if self.ade:
                self._ade_capture()
            self._apply("E")
            if self.ade:
                self._ade_apply()
            self._inject("E", (s + 1.0) * self.dt)
            self._record(s)
            self.step += 1

    def result(self) -> dict:
        mon_dt = self.t["mon_dtype"]
        out = dict(times=np.arange(self.n_steps) * self.dt, fields={}, monitor_times={},
                   flux=dict(self.flux), dft={}, dft_freqs={})
        for name, st in self.fm.items():
            m = st["m"]
            if st["times"]:
                out["fields"][name] = {c: np.stack(st["frames"][c]).astype(mon_dt)
                                       for c in m.components}
                out["monitor_times"][name] = np.array(st["times"])
            else:
                out["fields"][name] = {c: np.zeros((0,) + self.shape) for c in m.components}
                out["monitor_times"][name] = np.array([])
        for name, st in self.dm.items():
            m = st["m"]
            out["dft_freqs"][name] = np.asarray(m.freqs, dtype=np.float64)
            out["dft"][name] = {c: (st["acc"][c] if st["acc"][c] is not None else
                                    np.zeros((len(m.freqs),) + self.shape, dtype=np.complex128))
                                for c in m.components}
        return out


def run_oracle(sim, n_steps: Optional[int] = None) -> dict:
    """Run ``sim`` for its full step count (or ``n_steps``) and return a
    Result-shaped dict (simulation.py:327-336)."""
    r = OracleRun(sim, n_steps)
    r.advance(r.n_steps)
    return r.result()
