"""Interpolation / gridding with the interface of mr_recon's triton_interp
package (``ungrid`` ungrid.py:34-63, ``grid`` grid.py:32-67, ``interpolate`` /
``interpolate_adjoint`` interp.py:77-177).

Supported: kernel='kaiser_bessel', norm='1', pad_mode='circular' (the
configuration every NUFFT call uses), 1-3 dimensions, per-dimension width
1 <= W < 16. Other kernels, norm='2' and pad_mode='zero' raise
NotImplementedError rather than falling back to another implementation.
Autograd: value gradients as the reference (ungrid <-> grid), plus location
gradients (the reference returns None for them).
"""

from __future__ import annotations

from typing import Optional

import torch

from . import _lib
from .plan import Plan, PlanCache, traj_key

__all__ = ["ungrid", "grid", "interpolate", "interpolate_adjoint"]

_cache = PlanCache(4)


def _check_opts(kernel, norm, pad_mode):
    if kernel != "kaiser_bessel":
        raise NotImplementedError(f"kernel {kernel!r}: only 'kaiser_bessel' is implemented")
    if str(norm) != "1":
        raise NotImplementedError(f"norm {norm!r}: only '1' (separable) is implemented")
    if pad_mode != "circular":
        raise NotImplementedError(f"pad_mode {pad_mode!r}: only 'circular' is implemented")


def _width_tuple(width, ndim):
    if isinstance(width, (int, float)):
        return (float(width),) * ndim
    width = tuple(float(w) for w in width)
    if len(width) != ndim:
        raise ValueError(f"If width specified as tuple it must be same length as grid size but got "
                         f"len(width) = {len(width)} and len(grid_size) = {ndim}")
    return width


def _raw_plan(grid_size, nbatch, locs, width, beta):
    npts = locs.numel() // locs.shape[-1]
    key = ("raw", tuple(grid_size), nbatch, width, beta, traj_key(locs))

    def make():
        p = Plan([tuple(grid_size)], [npts], [nbatch], 1.0, width, beta, raw=True, device=locs.device)
        if npts > 0:
            p.set_traj(locs.reshape(-1))
        return p

    return _cache.get(key, locs, make)


def _beta(kernel_params, ndim):
    """kernel_params['beta']: one value (kernels.py:258-265, default 1.0) or,
    as sigpy's per-axis ``param``, one per dimension."""
    kp = {} if kernel_params is None else kernel_params
    b = kp.get("beta", 1.0)
    if isinstance(b, torch.Tensor):
        b = b.tolist()
    if isinstance(b, (list, tuple)):
        b = tuple(float(v) for v in b)
        if len(b) != ndim:
            raise ValueError(f"kernel_params beta per dimension needs {ndim} values, got {len(b)}")
        return b[0] if len(set(b)) == 1 else b
    return float(b)


def _ungrid_impl(vals, locs, width, beta):
    ndim = locs.shape[-1]
    gshape = tuple(vals.shape[-ndim:])
    bshape = vals.shape[:-ndim]
    nb = 1
    for s in bshape:
        nb *= int(s)
    lshape = locs.shape[:-1]
    npts = locs.numel() // ndim
    out = torch.empty((*bshape, *lshape), dtype=torch.complex64, device=vals.device)
    if npts == 0 or nb == 0:
        return out
    plan = _raw_plan(gshape, nb, locs.detach(), width, beta)
    plan.interp(vals.detach().to(torch.complex64).contiguous(), out, 1.0)
    return out


def _grid_impl(vals, locs, grid_size, width, beta):
    ndim = len(grid_size)
    lshape = locs.shape[:-1]
    bshape = vals.shape[:vals.ndim - len(lshape)]
    nb = 1
    for s in bshape:
        nb *= int(s)
    npts = locs.numel() // ndim
    out = torch.empty((*bshape, *grid_size), dtype=torch.complex64, device=vals.device)
    if nb == 0:
        return out
    if npts == 0:
        return out.zero_()
    plan = _raw_plan(tuple(grid_size), nb, locs.detach(), width, beta)
    plan.grid(vals.detach().to(torch.complex64).contiguous(), out, 1.0)
    return out


def _locs_grad(grid_vals, samples, locs, width, beta):
    ndim = locs.shape[-1]
    gshape = tuple(grid_vals.shape[-ndim:])
    nb = grid_vals.numel() // max(1, int(torch.tensor(gshape).prod()))
    plan = _raw_plan(gshape, nb, locs.detach(), width, beta)
    out = torch.empty(locs.shape, dtype=torch.float32, device=locs.device)
    plan.traj_grad(grid_vals.to(torch.complex64).contiguous(), samples.to(torch.complex64).contiguous(), out, 1.0)
    return out.to(locs.dtype)


class _UngridFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, locs, width, beta):
        ctx.save_for_backward(vals if locs.requires_grad else None, locs)
        ctx.width, ctx.beta = width, beta
        ctx.gshape = tuple(vals.shape[-locs.shape[-1]:])
        return _ungrid_impl(vals, locs, width, beta)

    @staticmethod
    def backward(ctx, g):
        vals, locs = ctx.saved_tensors
        gv = gl = None
        if ctx.needs_input_grad[0]:
            gv = _grid_impl(g.contiguous(), locs, ctx.gshape, ctx.width, ctx.beta)
        if ctx.needs_input_grad[1]:
            gl = _locs_grad(vals.detach(), g.contiguous(), locs, ctx.width, ctx.beta)
        return gv, gl, None, None


class _GridFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, locs, grid_size, width, beta):
        ctx.save_for_backward(vals if locs.requires_grad else None, locs)
        ctx.width, ctx.beta = width, beta
        return _grid_impl(vals, locs, grid_size, width, beta)

    @staticmethod
    def backward(ctx, g):
        vals, locs = ctx.saved_tensors
        gv = gl = None
        if ctx.needs_input_grad[0]:
            gv = _ungrid_impl(g.contiguous(), locs, ctx.width, ctx.beta)
        if ctx.needs_input_grad[1]:
            gl = _locs_grad(g.contiguous(), vals.detach(), locs, ctx.width, ctx.beta)
        return gv, gl, None, None, None


def ungrid(vals: torch.Tensor, locs: torch.Tensor, width, kernel: str = "kaiser_bessel",
           norm: str = "1", pad_mode: str = "circular", kernel_params: Optional[dict] = None):
    """Grid -> off-grid samples: vals (*batch, *grid) complex, locs (*pts, d)
    grid coordinates (wrapped circularly) -> (*batch, *pts)."""
    _check_opts(kernel, norm, pad_mode)
    _lib.require_cuda(vals, "vals")
    _lib.require_cuda(locs, "locs")
    width = _width_tuple(width, locs.shape[-1])
    beta = _beta(kernel_params, locs.shape[-1])
    if torch.is_grad_enabled() and (vals.requires_grad or locs.requires_grad):
        return _UngridFn.apply(vals, locs, width, beta)
    return _ungrid_impl(vals, locs, width, beta)


def grid(vals: torch.Tensor, locs: torch.Tensor, grid_size, width, kernel: str = "kaiser_bessel",
         norm: str = "1", pad_mode: str = "circular", kernel_params: Optional[dict] = None):
    """Off-grid samples -> grid (scatter-add): vals (*batch, *pts) complex,
    locs (*pts, d) -> (*batch, *grid_size)."""
    _check_opts(kernel, norm, pad_mode)
    _lib.require_cuda(vals, "vals")
    _lib.require_cuda(locs, "locs")
    grid_size = tuple(int(g) for g in grid_size)
    if locs.shape[-1] != len(grid_size):
        raise ValueError(f"Expected last dim of locs: to equal ndim but got locs.shape[-1] "
                         f"{locs.shape[-1]} != ndim {len(grid_size)}")
    width = _width_tuple(width, len(grid_size))
    beta = _beta(kernel_params, len(grid_size))
    if torch.is_grad_enabled() and (vals.requires_grad or locs.requires_grad):
        return _GridFn.apply(vals, locs, grid_size, width, beta)
    return _grid_impl(vals, locs, grid_size, width, beta)


def interpolate(vals, locs, width, kernel="kaiser_bessel", norm: str = "1",
                pad_mode: str = "circular", kernel_params: dict = None):
    """Differentiable ungrid (interp.py:77-87)."""
    return ungrid(vals, locs, width, kernel, norm, pad_mode, kernel_params)


def interpolate_adjoint(vals, locs, grid_size, width, kernel: str = "kaiser_bessel",
                        norm: str = "1", pad_mode: str = "circular", kernel_params: dict = None):
    """Differentiable grid (interp.py:157-177)."""
    return grid(vals, locs, grid_size, width, kernel, norm, pad_mode, kernel_params)
