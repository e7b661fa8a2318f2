"""Off-resonance (B0) time segmentation for the time-segmented SENSE model,
with the interface of mr_recon's imperfections/field.py.

    e^{-j 2 pi phi(r) alpha(t)} ~= sum_l b_l(r) h_l(t),  b_l(r) = e^{-j 2 pi phi(r) alpha_l}

``b0_to_phis_alphas`` writes a B0 map (Hz) and a readout time axis in that
form (field.py:58-96); ``alpha_segementation`` picks L segment centres alpha_l
and the temporal interpolators h_l (field.py:272-369). The resulting
``spatial_funcs`` (L, *im) and ``temporal_funcs`` (L, *trj) feed
``sense_linop(..., spatial_funcs=, temporal_funcs=)``, which runs all coils x
segments as one batched B200 NUFFT.
"""

from __future__ import annotations

import math
from typing import Optional, Tuple

import torch

__all__ = ["b0_to_phis_alphas", "alpha_segementation", "uniform_quantize"]

complex_dtype = torch.complex64
real_dtype = torch.float32


def b0_to_phis_alphas(b0_map: torch.Tensor, trj_size: tuple, ro_dim: int,
                      dt: float) -> Tuple[torch.Tensor, torch.Tensor]:
    """phi(r) = b0(r) / (2 max|b0|) in [-1/2, 1/2] with shape (1, *im), and
    alpha(t) = t_ro * dt * 2 max|b0| along the readout axis, size 1 along the
    other trajectory axes (broadcastable to trj_size): shape (1, ...)
    (field.py:58-96)."""
    scale = 2 * b0_map.abs().max()
    phis = b0_map / scale
    ts = torch.arange(trj_size[ro_dim], device=b0_map.device, dtype=real_dtype) * dt * scale
    shape = [1] * len(trj_size)
    shape[ro_dim] = trj_size[ro_dim]
    return phis[None], ts.reshape(shape)[None]


def uniform_quantize(data: torch.Tensor, K: int) -> Tuple[torch.Tensor, torch.Tensor]:
    """K centres at the midpoints of K equal bins over [min, max] of 1D data
    (shape (..., 1)), and each point's nearest-centre index, clamped to
    [0, K) (the 'uniform' method of mr_recon's utils.quantize_data,
    utils.py:137-157)."""
    flat = data.reshape(-1)
    lin = torch.linspace(float(flat.min()), float(flat.max()), K + 1, device=data.device)
    centers = ((lin[:-1] + lin[1:]) / 2).to(data.dtype)
    b = centers[0]
    m = (centers[1] - b) if K > 1 else torch.ones((), device=data.device, dtype=data.dtype)
    idx = torch.clamp(torch.round((flat - b) / m).to(torch.int64), 0, K - 1)
    return centers.reshape(K, 1), idx.reshape(data.shape[:-1])


def alpha_segementation(phis: torch.Tensor, alphas: torch.Tensor, L: int,
                        L_batch_size: Optional[int] = 1, interp_type: Optional[str] = "zero",
                        use_type3: Optional[bool] = True,
                        manual_spatial_funcs: Optional[torch.Tensor] = None,
                        verbose: Optional[bool] = True) -> Tuple[torch.Tensor, torch.Tensor]:
    """Spatial (L, *im) and temporal (L, *trj) basis functions of the
    segmented phase model for a single phase basis (phis (1, *im), alphas
    (1, *trj)), as field.py:272-369 with B = 1:

    * alpha_l: uniform quantisation of alpha into L bins;
    * b_l(r) = exp(-2 pi i phi(r) alpha_l);
    * interp_type 'zero': h_l(t) = 1 where alpha(t) is nearest alpha_l;
      'lstsq': h = pinv(B^H B / N) (B^H e(t) / N), the least-squares
      interpolator. The voxel sums (1/N) sum_r conj(b_l(r)) e^{-2 pi i
      phi(r) alpha(t)} come, with ``use_type3`` (the reference's default),
      from the Kaiser-Bessel type-3 NUFFT on the B200 kernels
      (type3_nufft(phis, alphas).forward, field.py:346-363), else exactly in
      float64, as type3_nufft_naive would (but once per distinct alpha
      value, alpha depending on the readout index only, as a chunked matrix
      product instead of a dense R x T matrix).
    ``L_batch_size`` and ``verbose`` are accepted for interface
    compatibility."""
    if phis.shape[0] != 1 or alphas.shape[0] != 1:
        raise NotImplementedError("alpha_segementation supports a single phase basis (B = 1)")
    dev = phis.device
    im_size = phis.shape[1:]
    trj_size = alphas.shape[1:]
    cents, inds = uniform_quantize(alphas.moveaxis(0, -1), L)
    a_l = cents[:, 0].to(real_dtype)
    ph = phis[0].to(real_dtype)
    spatial = torch.exp(-2j * math.pi * (ph[None] * a_l.reshape((L,) + (1,) * len(im_size))).to(torch.float32))
    spatial = spatial.to(complex_dtype)
    if manual_spatial_funcs is not None:
        spatial = manual_spatial_funcs
    if "zero" in interp_type:
        temporal = torch.stack([(inds == l).to(complex_dtype) for l in range(L)], 0)
    elif "lstsq" in interp_type:
        n = ph.numel()
        phr = ph.reshape(-1).to(torch.float64)
        sp = spatial.reshape(L, -1).to(torch.complex128)
        AHA = (sp.conj() @ sp.T) / n  # AHA[i, j] = mean(conj(b_i) b_j)
        if use_type3:
            # as the reference (field.py:352-367): Gram matrix, voxel sums and
            # pinv in complex64, whose default cut-off (L x float32 eps) keeps
            # the type-3 error (~1e-3) out of the Gram matrix's null space
            from .linops import type3_nufft
            t3n = type3_nufft(phis, alphas)
            s64 = spatial.reshape(L, -1).to(complex_dtype)
            AHA64 = (s64.conj() @ s64.T) / n
            AHy = t3n.forward(spatial.conj().to(complex_dtype)).reshape(L, -1) / n
            h = torch.linalg.pinv(AHA64) @ AHy
            return spatial, h.reshape((L,) + tuple(trj_size)).to(complex_dtype)
        else:
            ua, inv = torch.unique(alphas.reshape(-1).to(torch.float64), return_inverse=True)
            AHy = torch.zeros((L, ua.numel()), dtype=torch.complex128, device=dev)
            # (1/N) sum_r conj(b_l(r)) e^{-2 pi i phi(r) alpha}, exact, as a chunked matrix product
            chunk = max(1, (1 << 24) // max(n, 1))
            for c0 in range(0, ua.numel(), chunk):
                e = torch.exp(-2j * math.pi * phr[:, None] * ua[None, c0:c0 + chunk])  # (N, A)
                AHy[:, c0:c0 + chunk] = (sp.conj() @ e) / n
        h = torch.linalg.pinv(AHA) @ AHy
        if inv is not None:
            h = h[:, inv]
        temporal = h.reshape((L,) + tuple(trj_size)).to(complex_dtype)
    else:
        raise NotImplementedError(f"interp_type {interp_type!r}")
    return spatial, temporal
