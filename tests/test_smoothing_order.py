"""The arithmetic of the GPU subpixel kernels (csrc/smoothing.cu), restated
in NumPy and checked bit for bit against the host smoothing (which equals
the reference's): sub-cells from the boxes' fine-grid spans, last box wins;
block means adding, for each outer sub-cell index in order, the sum of the
innermost resolved sub-cell axis started from 0; np.gradient's central and
one-sided differences; the normal and the tensor formula."""
import itertools

import numpy as np
import pytest

from photonfdtd_b200 import smoothing as SM
from smoothing_scenes import scenes


def restated(grid, structures, factor, dtype):
    nx, ny, nz = grid.shape
    f = [factor if n > 1 else 1 for n in (nx, ny, nz)]
    spans, eps = SM.box_spans(grid, structures, factor)
    sub = np.full((nx * f[0], ny * f[1], nz * f[2]), 1.0)
    for sp, e in zip(spans, eps):
        sub[sp[0]:sp[1], sp[2]:sp[3], sp[4]:sp[5]] = e
    r = sub.reshape(nx, f[0], ny, f[1], nz, f[2])
    act = [a for a in range(3) if f[a] > 1]
    inner = act[-1] if act else 2
    outer = [a for a in range(3) if a != inner]
    sa, sh = np.zeros((nx, ny, nz)), np.zeros((nx, ny, nz))
    for o in itertools.product(*[range(f[a]) for a in outer]):
        ta, th = np.zeros((nx, ny, nz)), np.zeros((nx, ny, nz))
        for q in range(f[inner]):
            idx = [0, 0, 0]
            for a, v in zip(outer, o):
                idx[a] = v
            idx[inner] = q
            v = r[:, idx[0], :, idx[1], :, idx[2]]
            ta, th = ta + v, th + 1.0 / v
        sa, sh = sa + ta, sh + th
    cnt = float(f[0] * f[1] * f[2])
    ea, eh = sa / cnt, 1.0 / (sh / cnt)
    g = []
    for a in range(3):
        if grid.shape[a] == 1:
            g.append(np.zeros_like(ea))
            continue
        h = grid.cell_size[a]
        x = np.moveaxis(ea, a, 0)
        out = np.empty_like(x)
        out[1:-1] = (x[2:] - x[:-2]) / (2.0 * h)
        out[0] = (x[1] - x[0]) / h
        out[-1] = (x[-1] - x[-2]) / h
        g.append(np.moveaxis(out, 0, a))
    gm = np.sqrt((g[0] * g[0] + g[1] * g[1]) + g[2] * g[2])
    thr = max(gm.max() * 1e-9, np.finfo(np.float64).tiny)
    inv = np.where(gm > thr, 1.0 / np.where(gm > thr, gm, 1.0), 0.0)
    return tuple((ea + (eh - ea) * ((g[a] * inv) * (g[a] * inv))).astype(dtype)
                 for a in range(3))


@pytest.mark.parametrize("name,sim", scenes(), ids=[n for n, _ in scenes()])
def test_restated_device_arithmetic_equals_host_smoothing(name, sim):
    want = SM.smooth_permittivity(sim.grid, sim.structures, 1.0, sim.subpixel_factor,
                                  sim.dtypes["eps_r"])
    got = restated(sim.grid, sim.structures, sim.subpixel_factor, sim.dtypes["eps_r"])
    for c in range(3):
        assert np.array_equal(got[c], want[c]), (name, c)


def test_box_spans_reject_non_boxes():
    class Blob:
        pass
    from smoothing_scenes import scene_2d
    sim = scene_2d((2.0e-6, 1.5e-6, 0.0))
    assert SM.box_spans(sim.grid, list(sim.structures) + [Blob()], 3) is None
