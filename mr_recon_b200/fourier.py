"""NUFFT operators with the interface of mr_recon's ``NUFFT`` / ``triton_nufft``
(src/mr_recon/fourier.py:107-582), backed by the sm_100a kernels of
libmrnufft.so.

``b200_nufft`` is a drop-in for ``triton_nufft``: same constructor
(im_size, oversamp=1.25, width=6, beta=None, apodize=True), same methods,
shapes, scaling and complex64 conventions. ``triton_nufft`` is exported as an
alias so existing call sites keep working. All tensors must live on a CUDA
device; there is no CPU path.
"""

from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch
import torch.nn as nn

from . import _lib
from .plan import Plan, PlanCache, traj_key
from .utils import PadLast, fft, ifft

__all__ = ["NUFFT", "b200_nufft", "triton_nufft", "calc_toep_kernel_helper", "fft", "ifft"]

complex_dtype = torch.complex64
real_dtype = torch.float32


def calc_toep_kernel_helper(nufft_adj_os, trj: torch.Tensor, weights: Optional[torch.Tensor] = None):
    """Toeplitz kernels from an adjoint NUFFT at the oversampled image size
    (fourier.py:63-105): adjoint of the weights, then a centred orthonormal FFT."""
    dev = trj.device
    if weights is None:
        weights = torch.ones(trj.shape[:-1], dtype=real_dtype, device=dev)
    trj_batch = trj.shape[1:-1]
    if trj.shape[0] == 1 and weights.shape[0] != 1:
        trj = trj.expand((weights.shape[0], *trj.shape[1:]))
    N = trj.shape[0]
    d = trj.shape[-1]
    ksp = torch.ones((N, 1, *trj_batch), device=dev, dtype=complex_dtype)
    ksp_weighted = ksp * weights[:, None, ...]
    img = nufft_adj_os(ksp_weighted, trj)[:, 0, ...]
    return fft(img, dim=tuple(range(-d, 0)))


class NUFFT(nn.Module):
    """NUFFT contract (fourier.py:107-352): forward = e^{-j 2 pi k.r} with
    k_i in [-N_i/2, N_i/2) and r_i in [-1/2, 1/2]."""

    def __init__(self, im_size: tuple):
        super().__init__()
        self.im_size = im_size

    def rescale_trajectory(self, trj: torch.Tensor) -> torch.Tensor:
        return trj

    def forward_FT_only(self, img):
        raise NotImplementedError

    def adjoint_iFT_only(self, ksp_os):
        raise NotImplementedError

    def adjoint_grid_only(self, ksp, trj):
        raise NotImplementedError

    def forward_interp_only(self, ksp_os, trj):
        raise NotImplementedError

    def forward(self, img: torch.Tensor, trj: torch.Tensor) -> torch.Tensor:
        return self.forward_interp_only(self.forward_FT_only(img), trj)

    def adjoint(self, ksp: torch.Tensor, trj: torch.Tensor) -> torch.Tensor:
        return self.adjoint_iFT_only(self.adjoint_grid_only(ksp, trj))

    def calc_teoplitz_kernels(self, trj, weights=None, os_factor=2.0):
        raise NotImplementedError

    def normal_toeplitz(self, img: torch.Tensor, toeplitz_kernels: torch.Tensor) -> torch.Tensor:
        """FFT-only normal operator with precomputed kernels (fourier.py:302-352)."""
        N = img.shape[0]
        im_size = tuple(self.im_size)
        im_size_os = toeplitz_kernels.shape[1:]
        d = len(im_size)
        img_batch = img.shape[1:-d]
        img_flt = img.reshape((N, -1, *im_size))
        padder = PadLast(im_size_os, im_size)
        x = padder.forward(img_flt)
        x = fft(x, dim=tuple(range(-d, 0)))
        x = x * toeplitz_kernels[:, None, ...]
        x = ifft(x, dim=tuple(range(-d, 0)))
        x = padder.adjoint(x)
        return x.reshape((N, *img_batch, *im_size))


class _ForwardFn(torch.autograd.Function):
    """ksp = NUFFT(img, trj). Backward: image gradient = adjoint NUFFT (as
    InterpolateFn.backward, interp.py:48-74); trajectory gradient from the
    derivative of the KB kernel (new; the reference returns None)."""

    @staticmethod
    def forward(ctx, img, trj, op):
        out = op._forward_impl(img, trj)
        ctx.op = op
        ctx.save_for_backward(img if trj.requires_grad else None, trj)
        return out

    @staticmethod
    def backward(ctx, g):
        img, trj = ctx.saved_tensors
        op = ctx.op
        g = g.contiguous()
        gi = gt = None
        if ctx.needs_input_grad[0]:
            gi = op._adjoint_impl(g, trj)
        if ctx.needs_input_grad[1]:
            gt = op._traj_grad(op.forward_FT_only(img.detach()), g, trj)
        return gi, gt, None


class _AdjointFn(torch.autograd.Function):
    """img = NUFFT^H(ksp, trj). Backward: ksp gradient = forward NUFFT
    (InterpolateAdjointFn.backward, interp.py:129-154); trajectory gradient
    from the KB derivative applied to the FT of the image gradient."""

    @staticmethod
    def forward(ctx, ksp, trj, op):
        out = op._adjoint_impl(ksp, trj)
        ctx.op = op
        ctx.save_for_backward(ksp if trj.requires_grad else None, trj)
        return out

    @staticmethod
    def backward(ctx, g):
        ksp, trj = ctx.saved_tensors
        op = ctx.op
        g = g.contiguous()
        gk = gt = None
        if ctx.needs_input_grad[0]:
            gk = op._forward_impl(g, trj)
        if ctx.needs_input_grad[1]:
            gt = op._traj_grad(op.forward_FT_only(g), ksp.detach(), trj)
        return gk, gt, None


class b200_nufft(NUFFT):
    """Kaiser-Bessel NUFFT on B200 -- drop-in for ``triton_nufft``
    (fourier.py:354-582): apodize, scale 1/sqrt(prod N), centred zero-pad,
    centred FFT (norm=None), KB interpolation, / W^d; the adjoint mirrors it."""

    def __init__(self, im_size: tuple, oversamp: Optional[float] = 1.25, width: Optional[int] = 6,
                 beta: Optional[float] = None, apodize: Optional[bool] = True,
                 tile: Optional[tuple] = None, coil_group: int = 0, max_chunk: int = 0,
                 fast: bool = True, warp_grid: bool = True, weight_tables: bool = False,
                 reg_grid: bool = True, reg_interp: bool = True, autotune: bool = False):
        super().__init__(im_size)
        self.autotune = autotune
        self.fast = fast
        self.reg_grid = reg_grid
        self.reg_interp = reg_interp
        self.warp_grid = warp_grid
        self.weight_tables = weight_tables
        self.oversamp = oversamp
        self.width = width
        self.apodize = apodize
        if beta is None:
            self.beta = np.pi * (((width / oversamp) * (oversamp - 0.5)) ** 2 - 0.8) ** 0.5
        else:
            self.beta = beta
        self.tile = tile
        self.coil_group = coil_group
        self.max_chunk = max_chunk
        self._plans = PlanCache(4)

    # ------------------------------------------------------------------ plans
    def _widths(self):
        w = self.width
        return tuple(float(v) for v in w) if isinstance(w, (tuple, list)) else (float(w),) * len(self.im_size)

    def _wd(self):
        return float(np.prod(self._widths()))

    def _plan(self, N, C, M, trj, device):
        key = ("nufft", N, C, M, traj_key(trj), str(device))

        def make():
            p = Plan([tuple(self.im_size)] * N, [M] * N, [C] * N, self.oversamp, self._widths(),
                     self.beta, apodize=self.apodize, tile=self.tile, coil_group=self.coil_group,
                     max_chunk=self.max_chunk, device=device, fast=self.fast,
                     warp_grid=self.warp_grid, weight_tables=self.weight_tables,
                     reg_grid=self.reg_grid, reg_interp=self.reg_interp)
            if trj is not None and M > 0:
                if self.autotune:
                    from .autotune import autotune
                    autotune(p, trj.detach().to(torch.float32).contiguous())
                else:
                    p.set_traj(trj)
            return p

        return self._plans.get(key, trj, make)

    def _check(self, x, trj=None):
        _lib.require_cuda(x, "input")
        if trj is not None:
            _lib.require_cuda(trj, "trajectory")
            if trj.shape[-1] != len(self.im_size):
                raise ValueError(f"trajectory last dim {trj.shape[-1]} != len(im_size) {len(self.im_size)}")

    # ------------------------------------------------------------------ impl
    def _forward_impl(self, img, trj):
        self._check(img, trj)
        d = len(self.im_size)
        N = trj.shape[0]
        if img.shape[0] != N:
            raise ValueError(f"batch dim mismatch: img {img.shape[0]} vs trj {N}")
        bshape = img.shape[1:-d]
        tshape = trj.shape[1:-1]
        C = int(np.prod(bshape)) if len(bshape) else 1
        M = int(np.prod(tshape)) if len(tshape) else 1
        x = img.detach().to(complex_dtype).contiguous()
        out = torch.empty((N, *bshape, *tshape), dtype=complex_dtype, device=img.device)
        if M == 0 or C == 0:
            return out.zero_()
        plan = self._plan(N, C, M, trj.detach(), img.device)
        plan.forward(x, out)
        return out

    def _adjoint_impl(self, ksp, trj):
        self._check(ksp, trj)
        d = len(self.im_size)
        N = trj.shape[0]
        tb = trj.ndim - 2
        bshape = ksp.shape[1:ksp.ndim - tb]
        tshape = trj.shape[1:-1]
        C = int(np.prod(bshape)) if len(bshape) else 1
        M = int(np.prod(tshape)) if len(tshape) else 1
        y = ksp.detach().to(complex_dtype).contiguous()
        out = torch.empty((N, *bshape, *self.im_size), dtype=complex_dtype, device=ksp.device)
        if C == 0:
            return out
        plan = self._plan(N, C, M, trj.detach(), ksp.device)
        if M == 0:
            return out.zero_()
        plan.adjoint(y, out)
        return out

    def _traj_grad(self, grid_c, samples, trj):
        """d/dk Re<samples, interp(grid_c)> / W^d for a centred grid."""
        d = len(self.im_size)
        N = trj.shape[0]
        tshape = trj.shape[1:-1]
        M = int(np.prod(tshape)) if len(tshape) else 1
        C = int(np.prod(grid_c.shape[1:-d])) if grid_c.ndim > d + 1 else 1
        plan = self._plan(N, C, M, trj.detach(), trj.device)
        out = torch.empty(trj.shape, dtype=real_dtype, device=trj.device)
        plan.traj_grad(grid_c.contiguous(), samples.to(complex_dtype).contiguous(), out, 1.0 / self._wd())
        return out.to(trj.dtype)

    # ------------------------------------------------------------------ API
    def forward(self, img: torch.Tensor, trj: torch.Tensor) -> torch.Tensor:
        """(N, *img_batch, *im_size) -> (N, *img_batch, *trj_batch); N=1 when unbatched."""
        if torch.is_grad_enabled() and (img.requires_grad or trj.requires_grad):
            return _ForwardFn.apply(img, trj, self)
        return self._forward_impl(img, trj)

    def adjoint(self, ksp: torch.Tensor, trj: torch.Tensor) -> torch.Tensor:
        """(N, *ksp_batch, *trj_batch) -> (N, *ksp_batch, *im_size)."""
        if torch.is_grad_enabled() and (ksp.requires_grad or trj.requires_grad):
            return _AdjointFn.apply(ksp, trj, self)
        return self._adjoint_impl(ksp, trj)

    def forward_FT_only(self, img: torch.Tensor) -> torch.Tensor:
        """Apodize, zero-pad, centred FFT (fourier.py:432-468): (N, *B, *im) -> (N, *B, *im_os)."""
        self._check(img)
        d = len(self.im_size)
        N = img.shape[0]
        bshape = img.shape[1:-d]
        C = int(np.prod(bshape)) if len(bshape) else 1
        plan = self._plan(N, C, 0, None, img.device)
        out = torch.empty((N, *bshape, *plan.os_sizes[0]), dtype=complex_dtype, device=img.device)
        plan.forward_ft(img.detach().to(complex_dtype).contiguous(), out)
        return out

    def forward_interp_only(self, ksp_os: torch.Tensor, trj: torch.Tensor) -> torch.Tensor:
        """KB interpolation and / W^d (fourier.py:470-503)."""
        self._check(ksp_os, trj)
        d = len(self.im_size)
        N = trj.shape[0]
        bshape = ksp_os.shape[1:-d]
        tshape = trj.shape[1:-1]
        C = int(np.prod(bshape)) if len(bshape) else 1
        M = int(np.prod(tshape)) if len(tshape) else 1
        out = torch.empty((N, *bshape, *tshape), dtype=complex_dtype, device=ksp_os.device)
        plan = self._plan(N, C, M, trj.detach(), ksp_os.device)
        plan.interp(ksp_os.detach().to(complex_dtype).contiguous(), out, 1.0 / self._wd())
        return out

    def adjoint_grid_only(self, ksp: torch.Tensor, trj: torch.Tensor) -> torch.Tensor:
        """KB gridding and / W^d (fourier.py:527-550)."""
        self._check(ksp, trj)
        d = len(self.im_size)
        N = trj.shape[0]
        tb = trj.ndim - 2
        bshape = ksp.shape[1:ksp.ndim - tb]
        C = int(np.prod(bshape)) if len(bshape) else 1
        M = int(np.prod(trj.shape[1:-1])) if trj.ndim > 2 else 1
        plan = self._plan(N, C, M, trj.detach(), ksp.device)
        out = torch.empty((N, *bshape, *plan.os_sizes[0]), dtype=complex_dtype, device=ksp.device)
        plan.grid(ksp.detach().to(complex_dtype).contiguous(), out, 1.0 / self._wd())
        return out

    def adjoint_iFT_only(self, ksp_os: torch.Tensor) -> torch.Tensor:
        """Centred iFFT, crop, scale, apodize (fourier.py:505-525)."""
        self._check(ksp_os)
        d = len(self.im_size)
        N = ksp_os.shape[0]
        bshape = ksp_os.shape[1:-d]
        C = int(np.prod(bshape)) if len(bshape) else 1
        plan = self._plan(N, C, 0, None, ksp_os.device)
        out = torch.empty((N, *bshape, *self.im_size), dtype=complex_dtype, device=ksp_os.device)
        plan.adjoint_ift(ksp_os.detach().to(complex_dtype).contiguous(), out)
        return out

    def normal_toeplitz(self, img: torch.Tensor, toeplitz_kernels: torch.Tensor) -> torch.Tensor:
        """FFT-only normal operator with precomputed kernels (fourier.py:302-352):
        centred pad, orthonormal FFT, x kernel, inverse FFT and crop in one plan
        call (mrn_toeplitz_normal). img (N, *B, *im), kernels (N, *im_os)."""
        _lib.require_cuda(img, "image")
        d = len(self.im_size)
        N = img.shape[0]
        bshape = tuple(img.shape[1:-d])
        if tuple(img.shape[-d:]) != tuple(self.im_size):
            raise ValueError(f"image size {tuple(img.shape[-d:])} != {tuple(self.im_size)}")
        im_os = tuple(int(v) for v in toeplitz_kernels.shape[-d:])
        if toeplitz_kernels.shape[0] != N:
            raise ValueError("one Toeplitz kernel per batch element is needed")
        C = int(np.prod(bshape)) if bshape else 1
        key = ("toeplitz", N, C, im_os, str(img.device))

        def make():
            return Plan([tuple(self.im_size)] * N, [0] * N, [C] * N, self.oversamp, self._widths(), self.beta,
                        apodize=self.apodize, device=img.device)

        plan = self._plans.get(key, None, make)
        # the kernels are copied into the plan on every call (a reorder pass the
        # size of one kernel per slice), so a caller's new kernels are never missed
        plan.set_toeplitz(toeplitz_kernels, [im_os] * N)
        out = torch.empty((N, *bshape, *self.im_size), dtype=complex_dtype, device=img.device)
        plan.toeplitz_normal(img.detach().to(complex_dtype).contiguous(), out)
        return out

    def calc_teoplitz_kernels(self, trj: torch.Tensor, weights: Optional[torch.Tensor] = None,
                              os_factor: Optional[float] = 2.0):
        """Toeplitz kernels (fourier.py:552-582)."""
        im_size_os = tuple(round(i * os_factor) for i in self.im_size)
        nufft_os = b200_nufft(im_size=im_size_os, oversamp=self.oversamp, width=self.width)
        return calc_toep_kernel_helper(nufft_os.adjoint, trj * os_factor, weights) * (
            os_factor ** len(self.im_size))


# Drop-in name used by mr_recon call sites.
triton_nufft = b200_nufft
