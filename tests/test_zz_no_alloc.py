"""mrn_interp_noalloc: the interpolation entry point that allocates no device
memory (for callers that cannot call cudaMalloc at that point, e.g. while a
CUDA graph is being captured or when the host application owns all device
memory). Checked through the C ABI against the regular plan-based
interpolation (mrn_plan_create with MRN_PLAN_RAW + mrn_interp) on the same
inputs, on two calls in a row, at the same 1e-5 relative-L2 tolerance as the
other interpolation tests. This file is collected last on purpose.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from mr_recon_b200 import _lib

TOL = 1e-5


def _arr(vals, t):
    return (t * len(vals))(*vals)


def _regular_interp(grid_size, width, beta, grid, locs):
    """The existing entry point: raw plan + trajectory binning + mrn_interp."""
    lib = _lib.load()
    nd = len(grid_size)
    ncoil = grid.shape[0]
    npts = locs.shape[0]
    h = C.c_void_p()
    _lib.check(lib.mrn_plan_create(C.byref(h), nd, 1, _arr(list(grid_size), C.c_int),
                                   _arr([npts], C.c_int64), _arr([ncoil], C.c_int), 1.0,
                                   _arr(list(width), C.c_double), beta, _lib.MRN_PLAN_RAW, None, 0,
                                   0, torch.cuda.current_device()))
    try:
        st = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.mrn_plan_set_traj(h, locs.data_ptr(), st))
        out = torch.empty((ncoil, npts), dtype=torch.complex64, device="cuda")
        _lib.check(lib.mrn_interp(h, grid.data_ptr(), out.data_ptr(), 1.0, st))
        torch.cuda.synchronize()
    finally:
        lib.mrn_plan_destroy(h)
    return out


def _noalloc_interp(grid_size, width, beta, grid, locs):
    lib = _lib.load()
    nd = len(grid_size)
    out = torch.empty((grid.shape[0], locs.shape[0]), dtype=torch.complex64, device="cuda")
    rc = lib.mrn_interp_noalloc(nd, _arr(list(grid_size), C.c_int), grid.shape[0], locs.shape[0],
                                _arr(list(width), C.c_double), beta, grid.data_ptr(),
                                locs.data_ptr(), out.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "mrn_interp_noalloc")
    return out


def _case(rng, grid_size, ncoil, npts):
    g = torch.from_numpy((rng.randn(ncoil, *grid_size) + 1j * rng.randn(ncoil, *grid_size))
                         .astype(np.complex64)).cuda()
    locs = torch.from_numpy(((rng.rand(npts, len(grid_size)) * 1.2 - 0.1) * np.array(grid_size))
                            .astype(np.float32)).cuda()
    return g, locs


def _rel(a, b):
    return float((a - b).abs().norm() / b.abs().norm())


@pytest.mark.gpu
def test_noalloc_interp_matches_plan_interp_on_two_calls():
    rng = np.random.RandomState(2024)
    # call 1: 2D, width 6
    g1, l1 = _case(rng, (96, 80), 5, 20000)
    w1, b1 = (6.0, 6.0), 10.95
    out1 = _noalloc_interp((96, 80), w1, b1, g1, l1)
    ref1 = _regular_interp((96, 80), w1, b1, g1, l1)
    assert _rel(out1, ref1) < TOL
    # call 2 right after, different geometry and data (the scratch keeps call 1's
    # contents; nothing stale may leak into the result)
    g2, l2 = _case(rng, (20, 18, 22), 3, 7000)
    w2, b2 = (4.0, 4.0, 4.0), 7.0
    out2 = _noalloc_interp((20, 18, 22), w2, b2, g2, l2)
    ref2 = _regular_interp((20, 18, 22), w2, b2, g2, l2)
    assert _rel(out2, ref2) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("grid_size,width,beta,ncoil,npts", [
    ((300,), (6.0,), 10.95, 4, 3000),                # 1D
    ((64, 72), (5.5, 3.0), 9.0, 3, 8000),            # 2D, non-integer and unequal widths
    ((18, 20, 16), (4.0, 6.0, 5.0), 8.0, 2, 5000),   # 3D, a different width per axis
])
def test_noalloc_interp_per_axis_widths(grid_size, width, beta, ncoil, npts):
    # the per-axis tap count differs from the largest one (the scratch stride)
    # here, which is the layout-sensitive part of the weight and gather kernels
    rng = np.random.RandomState(sum(grid_size))
    g, locs = _case(rng, grid_size, ncoil, npts)
    for _ in range(2):
        out = _noalloc_interp(grid_size, width, beta, g, locs)
        ref = _regular_interp(grid_size, width, beta, g, locs)
        assert _rel(out, ref) < TOL


@pytest.mark.gpu
def test_noalloc_interp_rejects_oversized_problem():
    lib = _lib.load()
    # 4M samples of 2D width 6 need 256 MiB of scratch: refused before any launch
    rc = lib.mrn_interp_noalloc(2, _arr([64, 64], C.c_int), 1, 4_000_000, _arr([6.0, 6.0], C.c_double),
                                10.95, None, None, None, None)
    assert rc == _lib.MRN_ERR_SCRATCH
    with pytest.raises(ValueError):
        _lib.check(rc)
