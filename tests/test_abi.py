"""The C-ABI library: loads, exports every symbol include/mrnufft.h declares,
and validates arguments on the host before touching the GPU. CPU only (no
compute calls)."""

import ctypes as C
import os
import re

import pytest

from mr_recon_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "mrnufft.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mrn_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_all_header_symbols():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/mrnufft.h but not exported"
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"
    assert lib.mrn_version().decode().startswith("mrnufft")


def test_error_strings():
    lib = _lib.load()
    for code in range(0, -8, -1):
        assert lib.mrn_error_string(code)
    with pytest.raises(ValueError):
        _lib.check(_lib.MRN_ERR_ARG)
    with pytest.raises(ValueError):
        _lib.check(_lib.MRN_ERR_WIDTH)
    with pytest.raises(NotImplementedError):
        _lib.check(_lib.MRN_ERR_UNSUPPORTED)
    with pytest.raises(RuntimeError):
        _lib.check(_lib.MRN_ERR_STATE)


def _create(ndim=2, im=(32, 32), M=100, C_=2, os_=1.25, width=(6.0, 6.0), flags=0, tile=None):
    lib = _lib.load()
    h = C.c_void_p()
    arr = lambda v, t: (t * len(v))(*v)  # noqa: E731
    rc = lib.mrn_plan_create(C.byref(h), ndim, 1, arr(list(im), C.c_int), arr([M], C.c_int64),
                             arr([C_], C.c_int), os_, arr(list(width), C.c_double), -1.0, flags,
                             arr(list(tile), C.c_int) if tile else None, 0, 0, 0)
    return rc, h


def test_plan_create_rejects_bad_arguments_on_host():
    # all of these fail argument validation before any CUDA call
    assert _create(ndim=0)[0] == _lib.MRN_ERR_ARG
    assert _create(ndim=4, im=(4, 4, 4, 4), width=(6.0,) * 4)[0] == _lib.MRN_ERR_ARG
    assert _create(width=(16.0, 6.0))[0] == _lib.MRN_ERR_WIDTH   # ungrid.py:138-141 analogue
    assert _create(width=(0.5, 6.0))[0] == _lib.MRN_ERR_WIDTH
    assert _create(os_=0.9)[0] == _lib.MRN_ERR_ARG
    assert _create(im=(0, 32))[0] == _lib.MRN_ERR_ARG
    assert _create(C_=0)[0] == _lib.MRN_ERR_ARG
    assert _create(tile=(0, 8))[0] == _lib.MRN_ERR_ARG
    # raw plans need an explicit beta
    assert _create(flags=_lib.MRN_PLAN_RAW)[0] == _lib.MRN_ERR_ARG


def test_null_plan_calls_fail_cleanly():
    lib = _lib.load()
    assert lib.mrn_forward(None, None, None, None) == _lib.MRN_ERR_ARG
    assert lib.mrn_adjoint(None, None, None, None) == _lib.MRN_ERR_ARG
    assert lib.mrn_plan_set_traj(None, None, None) == _lib.MRN_ERR_ARG
    assert lib.mrn_plan_destroy(None) == _lib.MRN_OK
    betas = (C.c_double * 3)(8.0, 7.0, 6.0)
    assert lib.mrn_plan_set_beta(None, betas) == _lib.MRN_ERR_ARG
    assert lib.mrn_cg_step(None, None, None, None, None, None, None) == _lib.MRN_ERR_ARG
    assert lib.mrn_cg_dir(None, None, None, None, None) == _lib.MRN_ERR_ARG


def test_per_axis_beta_arguments_on_host():
    """kernel_params beta: one value, or one per axis (sigpy's per-axis
    param); a wrong count is a ValueError before any device work."""
    import torch
    from mr_recon_b200.interp import _beta
    assert _beta(None, 2) == 1.0
    assert _beta({"beta": 7.5}, 3) == 7.5
    assert _beta({"beta": (7.5, 7.5)}, 2) == 7.5           # equal betas collapse to one
    assert _beta({"beta": (7.5, 6.0)}, 2) == (7.5, 6.0)
    assert _beta({"beta": torch.tensor([7.5, 6.0, 5.0])}, 3) == (7.5, 6.0, 5.0)
    with pytest.raises(ValueError):
        _beta({"beta": (7.5, 6.0)}, 3)


def test_type3_checks_bases_before_device_work():
    """type3_nufft takes 1-3 bases (the tile kernels' dimensions) and says so
    for more, as NotImplementedError, before any CUDA call."""
    import torch
    from mr_recon_b200.linops import type3_nufft
    with pytest.raises(NotImplementedError):
        type3_nufft(torch.zeros(4, 6, 6), torch.zeros(4, 10))
    with pytest.raises(AssertionError):
        type3_nufft(torch.zeros(2, 6, 6), torch.zeros(3, 10))
