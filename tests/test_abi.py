"""The C ABI library: it loads, exports every symbol the header declares,
and rejects bad arguments with a status code and a message. No test here
launches a kernel, so the file runs without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import photonfdtd_b200._native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "pfb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pf[bsdm]?_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    syms = header_symbols()
    assert len(syms) >= 19 + 15
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/pfb200.h but not exported"
        assert s in N.SIGNATURES, f"{s} has no ctypes signature"


def test_version_string():
    assert N.lib().pf_version().decode().startswith("pfb200")


def test_create_rejects_bad_arguments():
    lib = N.lib()
    h = C.c_void_p()
    for args in ((0, 4, 4, 4), (4, 4, 4, 3), (4, -1, 4, 8)):
        rc = lib.pf_create(*args, 1.0, 1.0, 1.0, 1.0, 10, C.byref(h))
        assert rc == N.PF_ERR_INVALID
        assert h.value is None
        assert lib.pf_last_error(None).decode()
    rc = lib.pf_create(4, 4, 4, 4, 0.0, 1.0, 1.0, 1.0, 10, C.byref(h))
    assert rc == N.PF_ERR_INVALID


def test_null_handles_are_rejected():
    lib = N.lib()
    assert lib.pf_advance(None, 0, 1) == N.PF_ERR_INVALID
    assert lib.pf_finalize(None) == N.PF_ERR_INVALID
    assert lib.pf_read_field(None, 0, None) == N.PF_ERR_INVALID
    lib.pf_destroy(None)


def test_check_maps_codes_to_python_errors():
    with pytest.raises(ValueError):
        N.check(N.PF_ERR_INVALID, None)
    with pytest.raises(NotImplementedError):
        N.check(N.PF_ERR_UNSUPPORTED, None)
    with pytest.raises(N.NativeError):
        N.check(N.PF_ERR_CUDA, None)


def test_batch_rejects_bad_arguments_and_null_handles():
    lib = N.lib()
    h = C.c_void_p()
    for args in ((0, 4), (2, 3)):
        assert lib.pfb_create(*args, 1.0, 1.0, 1.0, 1.0, 10, C.byref(h)) == N.PF_ERR_INVALID
        assert h.value is None
    assert lib.pfb_create(2, 4, 1.0, 1.0, 1.0, 1.0, 0, C.byref(h)) == N.PF_ERR_INVALID
    assert lib.pfb_forward(None) == N.PF_ERR_INVALID
    assert lib.pfb_adjoint(None, None) == N.PF_ERR_INVALID
    assert lib.pfb_finalize(None, 8, 8) == N.PF_ERR_INVALID
    assert lib.pfb_read_dft(None, None) == N.PF_ERR_INVALID
    assert lib.pfb_last_error(None).decode()
    lib.pfb_destroy(None)
