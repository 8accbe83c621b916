"""ctypes binding of libpfb200.so (the C ABI in include/pfb200.h).

The library is built in-tree (``python -m photonfdtd_b200.build`` or
``__graft_entry__.build()``). There is no fallback: if the library is absent
or cannot be loaded, every engine call raises, naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

PF_OK = 0
PF_ERR_INVALID = -1
PF_ERR_CUDA = -2
PF_ERR_OOM = -3
PF_ERR_NONFINITE = -4
PF_ERR_TIMEOUT = -5
PF_ERR_UNSUPPORTED = -6
PF_ERR_STATE = -7

PF_CE_CELL1, PF_CE_CELL3, PF_CE_TABLE = 0, 1, 2
PF_KERNEL_AUTO, PF_KERNEL_SPLIT, PF_KERNEL_FUSED = 0, 1, 2

LIB_NAME = "libpfb200.so"
# PFB200_LIB names another build of the library (same ABI), e.g. one
# compiled with different tuning macros; default: the in-tree build.
LIB_PATH = os.environ.get("PFB200_LIB") or os.path.join(
    os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

_lib: Optional[C.CDLL] = None

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_dbl = C.c_double
_pi32 = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)
_pu32 = C.POINTER(C.c_uint32)
_pdbl = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol include/pfb200.h declares.
SIGNATURES = {
    "pf_version": (C.c_char_p, []),
    "pf_last_error": (C.c_char_p, [_vp]),
    "pf_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _dbl, _dbl, _dbl, _dbl, _i64,
                            C.POINTER(_vp)]),
    "pf_set_ce": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _pu32, C.c_int, _pdbl]),
    "pf_set_cpml": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp]),
    "pf_set_ade": (C.c_int, [_vp, C.c_int, _pi64, _pi32, _pdbl, _pdbl, _pdbl, _pu32]),
    "pf_rank_dispersive_words": (C.c_int, [_pu32, _i64, C.c_int, _pi64, C.c_int]),
    "pf_set_sources": (C.c_int, [_vp, C.c_int, _pi32, _pi64, _pi32, _pdbl, C.c_int, _pdbl]),
    "pf_add_dft": (C.c_int, [_vp, _pi32, _pi32, _pi32, C.c_int, C.c_int, C.c_int, _pdbl, _pdbl,
                             _dbl, C.POINTER(C.c_int)]),
    "pf_add_flux": (C.c_int, [_vp, C.c_int, C.c_int, _dbl, _dbl, C.POINTER(C.c_int)]),
    "pf_set_kernel": (C.c_int, [_vp, C.c_int]),
    "pf_finalize": (C.c_int, [_vp]),
    "pf_advance": (C.c_int, [_vp, _i64, _i64]),
    "pf_read_field": (C.c_int, [_vp, C.c_int, _vp]),
    "pf_read_dft": (C.c_int, [_vp, C.c_int, C.c_int, _pdbl]),
    "pf_read_flux": (C.c_int, [_vp, C.c_int, _pdbl]),
    "pf_step": (C.c_int, [_vp, _pi64]),
    "pf_adj_init": (C.c_int, [_vp, _i64]),
    "pf_adj_set_dft_cotangent": (C.c_int, [_vp, C.c_int, _pdbl]),
    "pf_adj_set_flux_cotangent": (C.c_int, [_vp, C.c_int, _dbl]),
    "pf_adj_add_field_source": (C.c_int, [_vp, _i64, C.c_int, _pi32, _pi32, _pi32, _pdbl]),
    "pf_adj_segment": (C.c_int, [_vp, _i64, _i64, _vp, _i64, C.c_int]),
    "pf_adj_read_grad": (C.c_int, [_vp, _pdbl]),
    "pf_adj_read_grad_components": (C.c_int, [_vp, _pdbl]),
    "pf_write_field": (C.c_int, [_vp, C.c_int, _vp]),
    "pf_set_check_every": (C.c_int, [_vp, _i64]),
    "pf_set_wait_test": (C.c_int, [_vp, C.c_int]),
    "pf_read_region": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32), _vp]),
    "pf_state_bytes": (C.c_int, [_vp, _pi64]),
    "pf_get_state": (C.c_int, [_vp, _vp, _i64, C.c_int]),
    "pf_set_state": (C.c_int, [_vp, _i64, _vp, _i64, C.c_int]),
    "pf_check_finite": (C.c_int, [_vp]),
    "pf_device_bytes": (C.c_int, [_vp, _pi64]),
    "pf_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "pf_set_profiling": (C.c_int, [_vp, C.c_int]),
    "pf_read_profile": (C.c_int, [_vp, _pi64, _pdbl, C.c_int]),
    "pf_info": (C.c_int, [_vp, C.c_char_p, C.c_int]),
    "pf_destroy": (None, [_vp]),
    "pf_flux_plane_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_vp),
                                        C.c_int, C.c_int, _dbl, _dbl, _vp, _vp]),
    "pf_noalloc_last_error": (C.c_char_p, []),
    # batched 2D TE engine with adjoint
    "pfb_create": (C.c_int, [C.c_int, C.c_int, _dbl, _dbl, _dbl, _dbl, _i64, C.POINTER(_vp)]),
    "pfb_set_instance": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.POINTER(_vp), C.c_int,
                                   C.c_int, C.c_int, C.c_int]),
    "pfb_set_sources": (C.c_int, [_vp, C.c_int, _pi32, _pi32, _pi32, _pi32, _pi32, _pdbl,
                                  C.c_int, _pdbl]),
    "pfb_set_dft": (C.c_int, [_vp, C.c_int, _pdbl]),
    "pfb_finalize": (C.c_int, [_vp, C.c_int, C.c_int]),
    "pf_smooth_boxes": (C.c_int, [C.c_int] * 4 + [C.c_double, C.c_int, _vp, _vp] +
                        [C.c_double] * 3 + [C.c_int, _vp, _vp, _vp]),
    "pf_smooth_last_error": (C.c_char_p, []),
    "pfb_set_tile_rows": (C.c_int, [_vp, C.c_int]),
    "pfb_tune_tiles": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    "pfb_set_design_ce": (C.c_int, [_vp, _vp]),
    "pfb_forward": (C.c_int, [_vp]),
    "pfb_adjoint": (C.c_int, [_vp, _pdbl]),
    "pfb_read_dft": (C.c_int, [_vp, _pdbl]),
    "pfb_read_grad": (C.c_int, [_vp, _pdbl]),
    "pfb_read_field": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "pfb_info": (C.c_int, [_vp, _pi64, C.c_int]),
    "pfb_stream": (_vp, [_vp]),
    "pfb_last_error": (C.c_char_p, [_vp]),
    "pfb_destroy": (None, [_vp]),
    # surrogate network kernels (device pointers as void*)
    "pfs_last_error": (C.c_char_p, []),
    "pfs_gemm_bf16": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp,
                                C.c_int, C.c_float, C.c_float, _vp]),
    "pfs_gemm_bf16_ex": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_int, _vp,
                                   C.c_int, C.c_int, _vp, C.c_int, C.c_float, C.c_float,
                                   C.c_int, _vp, _i64, _vp]),
    "pfs_gemm_bf16_bias_act": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int,
                                         _vp, C.c_int, _vp, _vp, C.c_int, _vp]),
    "pfs_gemm_bf16_splitk": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int,
                                       _vp, C.c_int, C.c_float, C.c_float, C.c_int, _vp, _i64,
                                       _vp]),
    "pfs_gemm_engine": (C.c_int, [C.c_int]),
    "pfs_gemm_timeouts": (C.c_int, [C.POINTER(C.c_int), C.c_int]),
    "pfs_gemm_wait_test": (C.c_int, [C.c_int]),
    "pfd_last_error": (C.c_char_p, []),
    "pfd_density_forward": (C.c_int, [C.c_int, C.c_int, _vp, _dbl, _dbl, _dbl, _vp, _vp]),
    "pfd_density_backward": (C.c_int, [C.c_int, C.c_int, _vp, _dbl, _dbl, _dbl, _vp, _vp,
                                       _vp]),
    "pfm_last_error": (C.c_char_p, []),
    "pfm_apply": (C.c_int, [C.c_int, C.c_int, _dbl, _dbl, _dbl, _vp, _vp, _vp, C.c_int, _vp,
                            _vp]),
    "pfm_chebyshev": (C.c_int, [C.c_int, C.c_int, _dbl, _dbl, _dbl, _vp, _vp, C.c_int, C.c_int,
                                _dbl, _dbl, _vp, _vp]),
    "pfs_im2col": (C.c_int, [C.c_int] * 9 + [_vp, _vp, C.c_int, _vp]),
    "pfs_col2im": (C.c_int, [C.c_int] * 9 + [_vp, C.c_int, _vp, _vp]),
    "pfs_bias_act": (C.c_int, [_i64, C.c_int, _vp, _vp, C.c_int, _vp, _vp, _vp]),
    "pfs_act_bwd": (C.c_int, [_i64, C.c_int, _vp, _vp, C.c_int, _vp, _vp, _vp, _vp, C.c_int,
                              _vp]),
    "pfs_transpose_bf16": (C.c_int, [C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp]),
    "pfs_to_bf16": (C.c_int, [_i64, _vp, _vp, _vp]),
    "pfs_upsample2": (C.c_int, [_i64, C.c_int, C.c_int, _vp, _vp, _vp]),
    "pfs_upsample2_bwd": (C.c_int, [_i64, C.c_int, C.c_int, _vp, _vp, _vp]),
    "pfs_mse": (C.c_int, [_i64, C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp]),
    "pfs_adam": (C.c_int, [_i64, _vp, _vp, _vp, _vp, C.c_float, C.c_float, C.c_float, C.c_float,
                           C.c_int, C.c_float, _vp, _vp]),
}


def lib() -> C.CDLL:
    """Load (once) and return the engine library; raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"photonfdtd_b200: {LIB_NAME} is not built. Build it with "
                "'python -m photonfdtd_b200.build' (nvcc, sm_100a).")
        try:
            h = C.CDLL(LIB_PATH)
        except OSError as e:
            raise RuntimeError(f"photonfdtd_b200: cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


class NativeError(RuntimeError):
    """A C ABI call failed; ``code`` is the PF_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def check(rc: int, handle=None, batch: bool = False) -> None:
    """Raise for a non-OK return code; ``batch`` selects the pf_batch error text."""
    if rc == PF_OK:
        return
    L = lib()
    msg = (L.pfb_last_error(handle) if batch else L.pf_last_error(handle)).decode(errors="replace")
    if rc == PF_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc == PF_ERR_INVALID:
        raise ValueError(msg)
    raise NativeError(rc, msg)


def ptr(a, ctype=None):
    """ctypes pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    if ctype is None:
        return a.ctypes.data_as(C.c_void_p)
    return a.ctypes.data_as(C.POINTER(ctype))
