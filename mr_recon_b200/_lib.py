"""ctypes binding of libmrnufft.so (the C ABI in include/mrnufft.h).

The library is built in-tree (``python -m mr_recon_b200.build``). There is no
CPU fallback: importing this module without the built library, or using it
without a CUDA device, raises.
"""

from __future__ import annotations

import ctypes as C
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmrnufft.so")

MRN_OK = 0
MRN_ERR_ARG = -1
MRN_ERR_WIDTH = -2
MRN_ERR_CUDA = -3
MRN_ERR_CUFFT = -4
MRN_ERR_NOMEM = -5
MRN_ERR_STATE = -6
MRN_ERR_UNSUPPORTED = -7
MRN_ERR_SCRATCH = -8

MRN_PLAN_RAW = 1
MRN_PLAN_NO_APOD = 2
MRN_OPT_FAST_KERNELS = 1
MRN_OPT_WARP_GRIDDING = 2
MRN_OPT_WEIGHT_TABLES = 3
MRN_OPT_INTERP_CHUNK = 4
MRN_OPT_GRID_CHUNK = 5
MRN_OPT_INTERP_TILE = 6
MRN_OPT_GRID_TILE = 7
MRN_OPT_REG_GRIDDING = 8
MRN_OPT_REG_INTERP = 9
MRN_OPT_GRID_LANES = 10
MRN_OPT_ENTRY_MAJOR = 11
MRN_OPT_NATIVE_FFT = 12

_vp = C.c_void_p
_i = C.c_int
_i64 = C.c_int64
_f = C.c_float
_d = C.c_double
_pi = C.POINTER(C.c_int)
_pi64 = C.POINTER(C.c_int64)
_pd = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol include/mrnufft.h declares
SIGNATURES = {
    "mrn_version": (C.c_char_p, []),
    "mrn_error_string": (C.c_char_p, [_i]),
    "mrn_last_cuda_error": (_i, []),
    "mrn_plan_create": (_i, [C.POINTER(_vp), _i, _i, _pi, _pi64, _pi, _d, _pd, _d, _i, _pi, _i, _i, _i]),
    "mrn_plan_destroy": (_i, [_vp]),
    "mrn_plan_offsets": (_i, [_vp, _pi64, _pi64, _pi64, _pi64]),
    "mrn_plan_sizes": (_i, [_vp, _pi64]),
    "mrn_plan_stats": (_i, [_vp, _pi64]),
    "mrn_plan_fft_kind": (_i, [_vp]),
    "mrn_plan_set_option": (_i, [_vp, _i, _i]),
    "mrn_plan_set_beta": (_i, [_vp, _pd]),
    "mrn_plan_enable_timing": (_i, [_vp, _i]),
    "mrn_plan_timing": (_i, [_vp, _pd, _pi64]),
    "mrn_plan_set_traj": (_i, [_vp, _vp, _vp]),
    "mrn_forward": (_i, [_vp, _vp, _vp, _vp]),
    "mrn_adjoint": (_i, [_vp, _vp, _vp, _vp]),
    "mrn_forward_ft": (_i, [_vp, _vp, _vp, _vp]),
    "mrn_interp": (_i, [_vp, _vp, _vp, _f, _vp]),
    "mrn_grid": (_i, [_vp, _vp, _vp, _f, _vp]),
    "mrn_adjoint_ift": (_i, [_vp, _vp, _vp, _vp]),
    "mrn_traj_grad": (_i, [_vp, _vp, _vp, _vp, _f, _vp]),
    "mrn_sense_forward": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "mrn_sense_adjoint": (_i, [_vp, _vp, _vp, _vp, _vp, _f, _vp]),
    "mrn_sense_normal": (_i, [_vp, _vp, _vp, _vp, _vp, _f, _f, _vp, _i, _vp]),
    "mrn_lr_forward": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "mrn_lr_adjoint": (_i, [_vp, _vp, _vp, _vp, _vp, _f, _vp]),
    "mrn_lr_normal": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _vp]),
    "mrn_plan_set_toeplitz": (_i, [_vp, _pi, _vp, _vp]),
    "mrn_toeplitz_normal": (_i, [_vp, _vp, _vp, _vp]),
    "mrn_sense_normal_toeplitz": (_i, [_vp, _vp, _vp, _vp, _f, _f, _vp, _i, _vp]),
    "mrn_cg_init": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _vp]),
    "mrn_cg_step": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mrn_cg_dir": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "mrn_cg_dot": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "mrn_interp_noalloc": (_i, [_i, _pi, _i, _i64, _pd, _d, _vp, _vp, _vp, _vp]),
}

_lib = None


def load() -> C.CDLL:
    """Load the library (once). Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m mr_recon_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MrnError(RuntimeError):
    pass


def check(rc: int, what: str = "") -> None:
    """Map a C-ABI status to the reference's Python exceptions: argument and
    width errors raise ValueError (as ungrid.py:138-141 does for too-wide
    kernels), everything else RuntimeError."""
    if rc == MRN_OK:
        return
    lib = load()
    msg = lib.mrn_error_string(rc).decode()
    if rc == MRN_ERR_CUDA:
        msg += f" (cudaError {lib.mrn_last_cuda_error()})"
    if what:
        msg = f"{what}: {msg}"
    if rc in (MRN_ERR_ARG, MRN_ERR_WIDTH, MRN_ERR_SCRATCH):
        raise ValueError(msg)
    if rc == MRN_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise MrnError(msg)


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise RuntimeError(
            f"{name} must be a CUDA tensor: mr_recon_b200 runs only on the GPU "
            "(no CPU fallback)")


def ptr(t) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream
