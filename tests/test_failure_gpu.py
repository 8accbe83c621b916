"""Failure detection on the GPU, in the forms that fault nothing.

* A scene stepped past its Courant limit blows up; with a periodic finite
  check the engine stops at the first checked step holding an inf or nan and
  reports PF_ERR_NONFINITE (the host raises), and the process stays usable.
* Every mbarrier wait in the TMA-staged step and in the tcgen05 GEMM is
  bounded. A test hook makes one block wait on a barrier that nothing
  arrives on, with a short limit: the wait runs out, the block lets its own
  copies (and MMAs) finish, records the timeout and leaves. The call reports
  it (PF_ERR_TIMEOUT / pfs_gemm_timeouts), and the next call, hook off, is
  correct again: the context survived.
"""
import ctypes as C

import numpy as np
import pytest

import photonfdtd_b200 as pf
from photonfdtd_b200 import _native as N
from photonfdtd_b200.engine import B200Engine, build_tables

pytestmark = pytest.mark.gpu


def _scene(courant=0.99, n_steps=400):
    grid = pf.Grid(size=(32 * 40e-9,) * 3, cell_size=40e-9, pml_layers=6)
    box = pf.Box(center=(0.1e-6, 0.0, 0.0), size=(0.3e-6, 0.3e-6, 0.3e-6),
                 medium=pf.Medium(permittivity=2.5))
    src = pf.PointDipole(position=(0.0, 0.0, 0.0), component="Ex",
                         waveform=pf.GaussianPulse(freq0=250e12, fwhm=4e-15))
    probe = pf.Simulation(grid, structures=[box], sources=[src], run_time=1e-15,
                          precision="float32", courant=courant)
    return pf.Simulation(grid, structures=[box], sources=[src],
                         run_time=(n_steps - 0.5) * probe.dt, precision="float32",
                         courant=courant)


def test_unstable_run_is_stopped_as_nonfinite():
    sim = _scene(courant=1.6, n_steps=2000)
    sim.b200_check_every = 50
    with pytest.raises(N.NativeError) as ei:
        sim.run()
    assert ei.value.code == N.PF_ERR_NONFINITE
    assert "non-finite" in str(ei.value)
    # the same scene at a stable Courant number runs through, checks passing
    ok = _scene(courant=0.99, n_steps=300)
    ok.b200_check_every = 50
    res = ok.run()
    assert np.isfinite(res.times).all()


def test_tma_stage_wait_runs_out_and_is_reported():
    t = build_tables(_scene(n_steps=40))
    eng = B200Engine(t, kernel=N.PF_KERNEL_FUSED)
    try:
        assert eng.info()["tma"] == "1", eng.info()
        N.check(N.lib().pf_set_wait_test(eng.h, 1), eng.h)
        with pytest.raises(N.NativeError) as ei:
            eng.advance(0, 3)
        assert ei.value.code == N.PF_ERR_TIMEOUT
    finally:
        eng.close()
    # hook off: the fused TMA path equals the split passes bit for bit again
    a, b = B200Engine(t, kernel=N.PF_KERNEL_FUSED), B200Engine(t, kernel=N.PF_KERNEL_SPLIT)
    try:
        a.advance(0, 20)
        b.advance(0, 20)
        for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            assert np.array_equal(a.get(c), b.get(c)), c
    finally:
        a.close()
        b.close()


def test_gemm_wait_runs_out_and_is_counted():
    import torch
    L = N.lib()
    cnt = C.c_int()
    N.check(L.pfs_gemm_timeouts(C.byref(cnt), 1))
    g = torch.Generator(device="cpu").manual_seed(3)
    A = torch.randn(512, 256, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(384, 256, generator=g).to(torch.bfloat16).cuda()
    Cm = torch.zeros(512, 384, dtype=torch.float32, device="cuda")
    prev = L.pfs_gemm_engine(1)

    def gemm():
        N.check(L.pfs_gemm_bf16(512, 384, 256, C.c_void_p(A.data_ptr()), 256,
                                C.c_void_p(B.data_ptr()), 256, C.c_void_p(Cm.data_ptr()), 384,
                                1.0, 0.0, None))
        torch.cuda.synchronize()

    old = L.pfs_gemm_wait_test(1)
    try:
        gemm()
    finally:
        L.pfs_gemm_wait_test(old)
    N.check(L.pfs_gemm_timeouts(C.byref(cnt), 1))
    assert cnt.value >= 1
    # the timed-out block left its tile of the first 128 rows unwritten (zeros)
    assert torch.count_nonzero(Cm[:128]) < Cm[:128].numel()
    # hook off: the whole product is right and nothing timed out
    gemm()
    N.check(L.pfs_gemm_timeouts(C.byref(cnt), 1))
    L.pfs_gemm_engine(prev)
    assert cnt.value == 0
    want = A.float() @ B.float().T
    assert torch.allclose(Cm, want, rtol=1e-3, atol=1e-3)
