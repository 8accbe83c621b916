"""GPU subpixel permittivity (pf_smooth_boxes) equals the host smoothing,
hence the reference's numpy result, bit for bit."""
import numpy as np
import pytest

from photonfdtd_b200 import _native as N
from photonfdtd_b200 import smoothing as SM
from smoothing_scenes import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,sim", scenes(), ids=[n for n, _ in scenes()])
def test_device_smoothing_equals_host(name, sim):
    args = (sim.grid, sim.structures, 1.0, sim.subpixel_factor, sim.dtypes["eps_r"])
    want = SM.smooth_permittivity(*args)
    got = SM.smooth_permittivity_device(*args)
    for c in range(3):
        assert got[c].dtype == want[c].dtype
        assert np.array_equal(got[c], want[c]), (name, c)


def test_device_smoothing_without_boxes_is_the_background():
    sim = scenes()[2][1]
    xx, yy, zz = SM.smooth_permittivity_device(sim.grid, [], 2.5, 3, np.float32)
    assert np.all(xx == np.float32(2.5)) and np.all(yy == xx) and np.all(zz == xx)


def test_bad_arguments_are_rejected():
    L = N.lib()
    out = np.empty(8, np.float32)
    rc = L.pf_smooth_boxes(2, 2, 2, 3, 1.0, 0, None, None, 1.0, 1.0, 1.0, 3,
                           out.ctypes.data, out.ctypes.data, out.ctypes.data)
    assert rc == N.PF_ERR_INVALID
    assert "bad arguments" in L.pf_smooth_last_error().decode()
