"""Reconstruction drivers with the interface of mr_recon's recons.py
(``CG_SENSE_recon`` recons.py:77-156, ``FISTA_recon`` :189-249,
``min_norm_recon`` :18-75, ``coil_combine``)."""

from __future__ import annotations

import time
from typing import Optional

import torch

from .algs import FISTA, SenseCG, conjugate_gradient, power_method_operator
from .linops import linop

complex_dtype = torch.complex64

__all__ = ["CG_SENSE_recon", "FISTA_recon", "min_norm_recon", "coil_combine"]


def _max_eigen(A, device, verbose):
    x0 = torch.randn(A.ishape, dtype=complex_dtype, device=device)
    _, me = power_method_operator(A.normal, x0, verbose=verbose)
    return me * 1.01


def _fused_solver(A, max_iter, lamda_l2, max_eigen, tolerance, graph, ksp):
    """The fused device CG of ``A`` for these solver settings. Solvers are kept
    on the linop, keyed by the settings and the identity of its plan, coil maps
    and density weights, so repeated calls (one per slice or frame) reuse the
    buffers and, with ``graph=True``, the CUDA graph captured on the first call."""
    toep = bool(getattr(A, "use_toeplitz", False)) and getattr(A.plan, "toeplitz_pad", None) is not None
    key = (int(max_iter), float(lamda_l2), float(max_eigen), float(tolerance), bool(graph),
           id(A.plan), id(A.mps), id(A.dcf), toep)
    cache = A.__dict__.setdefault("_fused_cg", {})
    cg = cache.get(key)
    if cg is None:
        cg = SenseCG(A.plan, A.mps, A.dcf, max_iter, lamda_l2, max_eigen, tolerance, toeplitz=toep)
        if graph:
            cg.ksp.copy_(ksp.reshape(-1))
            cg.capture()
        cache.clear()  # one solver per linop: a new setting replaces the old graph
        cache[key] = cg
    return cg


def CG_SENSE_recon(A: linop, ksp: torch.Tensor, max_iter: Optional[int] = 15,
                   lamda_l2: Optional[float] = 0.0, max_eigen: Optional[float] = None,
                   tolerance: Optional[float] = 1e-8, weights: Optional[torch.Tensor] = None,
                   ahb_init: Optional[torch.Tensor] = None, clear_gpu_mem: Optional[bool] = True,
                   verbose: Optional[bool] = True, graph: Optional[bool] = False) -> torch.Tensor:
    """recon = (A^H A + lamda_l2 I)^-1 A^H b, with A normalised by max_eigen.

    For a ``sense_linop`` on the B200 NUFFT (no time segmentation, no
    ``weights``, no ``ahb_init``) the solve runs on the fused device CG
    (``SenseCG``); ``graph=True`` records it in a CUDA graph first."""
    device = ksp.device
    if max_eigen is None:
        max_eigen = _max_eigen(A, device, verbose)
    fused = getattr(A, "plan", None) is not None and weights is None and ahb_init is None
    if fused:
        cg = _fused_solver(A, max_iter, lamda_l2, max_eigen, tolerance, graph, ksp)
        x = cg.solve(ksp.to(complex_dtype))
        return x.reshape(A.im_size).clone()
    start = time.perf_counter()
    if ahb_init is None:
        AHb = A.adjoint(ksp.type(complex_dtype)) / (max_eigen ** 0.5)
    else:
        AHb = ahb_init.type(complex_dtype) / (max_eigen ** 0.5)
    if verbose:
        print(f"AHb took {time.perf_counter() - start:.3f}(s)")
    if max_iter == 0:
        return AHb
    AHA = lambda x: A.normal(x) / max_eigen  # noqa: E731
    return conjugate_gradient(AHA=AHA, AHb=AHb, num_iters=max_iter, lamda_l2=lamda_l2,
                              tolerance=tolerance, weights=weights, verbose=verbose)


def min_norm_recon(A: linop, ksp: torch.Tensor, max_iter: int = 15,
                   lamda_l2: Optional[float] = 0.0, max_eigen: Optional[float] = None,
                   verbose: Optional[bool] = True) -> torch.Tensor:
    """recon = A^H (A A^H)^-1 b (recons.py:18-75)."""
    device = ksp.device
    if max_eigen is None:
        max_eigen = _max_eigen(A, device, verbose)
    AAH = lambda x: A.forward(A.adjoint(x)) / max_eigen  # noqa: E731
    y = conjugate_gradient(AHA=AAH, AHb=ksp.type(complex_dtype), lamda_l2=lamda_l2,
                           num_iters=max_iter, verbose=verbose)
    return A.adjoint(y) / (max_eigen ** 0.5)


def coil_combine(multi_chan_img: torch.Tensor, mps: Optional[torch.Tensor] = None,
                 walsh_kernel_size: Optional[int] = None) -> torch.Tensor:
    """SENSE / sum-of-squares coil combination (recons.py:158-187)."""
    if mps is not None:
        return (multi_chan_img * mps.conj()).sum(0) / (mps.abs().square().sum(0) + 1e-5)
    if walsh_kernel_size is not None:
        raise NotImplementedError
    return multi_chan_img.abs().square().sum(0).sqrt()


def FISTA_recon(A: linop, ksp: torch.Tensor, proxg, max_iter: int = 40,
                max_eigen: Optional[float] = None, verbose: Optional[bool] = True) -> torch.Tensor:
    """min_x ||Ax - b||^2 + g(x) by FISTA (recons.py:189-249)."""
    device = ksp.device
    if max_eigen is None:
        max_eigen = _max_eigen(A, device, verbose)
    AHb = A.adjoint(ksp.type(complex_dtype)) / (max_eigen ** 0.5)
    AHA = lambda x: A.normal(x) / max_eigen  # noqa: E731
    return FISTA(AHA, AHb, proxg, max_iter, verbose=verbose)
