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

__all__ = ["b0_to_phis_alphas", "alpha_segementation", "uniform_quantize", "kmeans_quantize",
           "isotropic_cluster_alphas"]

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


def kmeans_quantize(data: torch.Tensor, K: int, max_iter: int = 1000,
                    seed: int = 0) -> Tuple[torch.Tensor, torch.Tensor]:
    """K cluster centres of data (n, d) and each point's nearest centre, by
    Lloyd's k-means with euclidean distances (the 'cluster' method of
    mr_recon's utils.quantize_data, utils.py:117-135, which calls
    fast_pytorch_kmeans' KMeans(max_iter=1000, mode='euclidean')). The
    initial centres come from k-means++ seeding with a fixed generator, so
    the result is the same on every call (KMeans seeds from the global RNG);
    iterations stop when no assignment changes. A centre that loses all its
    points keeps its position."""
    x = data.reshape(data.shape[0], -1).to(torch.float64)
    n = x.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    first = int(torch.randint(n, (1,), generator=g))
    cents = [x[first]]
    d2 = ((x - cents[0]) ** 2).sum(1)
    for _ in range(1, K):
        p = (d2 / d2.sum()).cpu() if float(d2.sum()) > 0 else torch.full((n,), 1.0 / n, dtype=torch.float64)
        i = int(torch.multinomial(p, 1, generator=g))
        cents.append(x[i])
        d2 = torch.minimum(d2, ((x - x[i]) ** 2).sum(1))
    c = torch.stack(cents)
    idx = torch.cdist(x, c).argmin(1)
    for _ in range(max_iter):
        cnt = torch.bincount(idx, minlength=K).to(x.dtype)
        sums = torch.zeros_like(c).index_add_(0, idx, x)
        c = torch.where(cnt[:, None] > 0, sums / cnt.clamp(min=1)[:, None], c)
        new = torch.cdist(x, c).argmin(1)
        if torch.equal(new, idx):
            break
        idx = new
    return c.to(data.dtype), idx


def isotropic_cluster_alphas(alphas: torch.Tensor, phis: torch.Tensor,
                             L: int) -> Tuple[torch.Tensor, torch.Tensor]:
    """Segment centres (L, B) and per-sample indices (*trj_size) for several
    phase bases (field.py:216-269): phis and alphas are centred on their
    range midpoints, phis scaled to [-1/2, 1/2] per basis and alphas by the
    inverse, so the k-means distance in alpha space is the same phase error
    for every basis; the centres are scaled back."""
    B = alphas.shape[0]
    trj_size = alphas.shape[1:]
    ph = phis.reshape(B, -1).to(torch.float64)
    al = alphas.reshape(B, -1).to(torch.float64)
    ph_mp = (ph.min(1).values + ph.max(1).values) / 2
    al_mp = (al.min(1).values + al.max(1).values) / 2
    ph_c = ph - ph_mp[:, None]
    al_c = al - al_mp[:, None]
    scales = ph_c.abs().max(1).values * 2
    al_c = al_c * scales[:, None]
    cents, inds = kmeans_quantize(al_c.T.contiguous(), L)
    cents = cents / scales + al_mp
    return cents.reshape(L, B), inds.reshape(trj_size)


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
    B = phis.shape[0]
    if alphas.shape[0] != B:
        raise ValueError("phis and alphas need the same number of phase bases")
    dev = phis.device
    im_size = phis.shape[1:]
    trj_size = alphas.shape[1:]
    if B > 1:
        return _segment_multi(phis, alphas, L, interp_type, use_type3, manual_spatial_funcs)
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


def _segment_multi(phis, alphas, L, interp_type, use_type3, manual_spatial_funcs):
    """alpha_segementation for B > 1 phase bases (field.py:321-369): centres
    by isotropic k-means, b_l(r) = exp(-2 pi i sum_b phis_b(r) alpha_l,b),
    'zero' one-hot h_l or the 'lstsq' interpolator from the B-dimensional
    type-3 NUFFT (B <= 3 on the B200 kernels) or the exact sums."""
    B = phis.shape[0]
    im_size = phis.shape[1:]
    trj_size = alphas.shape[1:]
    cents, inds = isotropic_cluster_alphas(alphas, phis, L)
    ph = phis.reshape(B, -1).to(torch.float64)
    spatial = torch.exp(-2j * math.pi * (cents.to(torch.float64) @ ph)).to(complex_dtype)
    spatial = spatial.reshape((L, *im_size))
    if manual_spatial_funcs is not None:
        spatial = manual_spatial_funcs
    if "zero" in interp_type:
        temporal = torch.stack([(inds == l).to(complex_dtype) for l in range(L)], 0)
        return spatial, temporal
    if "lstsq" not in interp_type:
        raise NotImplementedError(f"interp_type {interp_type!r}")
    n = ph.shape[1]
    sp = spatial.reshape(L, -1)
    AHA = (sp.conj() @ sp.T) / n
    if use_type3:
        from .linops import type3_nufft
        t3n = type3_nufft(phis, alphas)
        AHy = t3n.forward(spatial.conj().to(complex_dtype)).reshape(L, -1) / n
    else:
        al = alphas.reshape(B, -1).to(torch.float64)
        AHy = torch.zeros((L, al.shape[1]), dtype=torch.complex128, device=phis.device)
        sp64 = sp.to(torch.complex128).conj()
        chunk = max(1, (1 << 24) // max(n, 1))
        for c0 in range(0, al.shape[1], chunk):
            e = torch.exp(-2j * math.pi * (ph.T @ al[:, c0:c0 + chunk]))  # (N, chunk)
            AHy[:, c0:c0 + chunk] = (sp64 @ e) / n
        AHA = AHA.to(torch.complex128)
    h = torch.linalg.pinv(AHA) @ AHy.to(AHA.dtype)
    return spatial, h.reshape((L, *trj_size)).to(complex_dtype)
