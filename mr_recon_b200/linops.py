"""Linear operators with the interface of mr_recon's linops.py (``linop``,
``batching_params``, ``sense_linop``, linops.py:22-47 and 1041-1308).

``sense_linop`` keeps the reference constructor and shapes. With the B200
NUFFT (the default here) and no time segmentation, forward / adjoint /
normal each run as one fused pass over all coils: coil maps are multiplied
inside the pre-FFT kernel, the density compensation inside the gridding
kernel, and conj(coil map) summation inside the post-iFFT kernel, where the
reference loops over coil and segment batches in Python
(linops.py:1160-1176, 1206-1226).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import torch
import torch.nn as nn
from einops import einsum, rearrange

from . import _lib
from .fourier import NUFFT, b200_nufft
from .plan import Plan
from .utils import PadLast, batch_iterator, fft, ifft, resize

complex_dtype = torch.complex64
real_dtype = torch.float32

__all__ = ["batching_params", "linop", "sense_linop", "subspace_linop", "subspace_linop_new", "type3_nufft",
           "type3_nufft_naive"]


@dataclass
class batching_params:
    """Batch sizes (linops.py:22-28). The fused B200 path ignores them: all
    coils and segments run in one launch."""
    coil_batch_size: Optional[int] = 1
    sub_batch_size: Optional[int] = 1
    field_batch_size: Optional[int] = 1
    toeplitz_batch_size: Optional[int] = 1
    img_batch_size: Optional[int] = 1


class linop(nn.Module):
    """Generic linop (linops.py:30-47)."""

    def __init__(self, ishape, oshape):
        super().__init__()
        self.ishape = ishape
        self.oshape = oshape

    def forward(self, *args):
        raise NotImplementedError

    def adjoint(self, *args):
        raise NotImplementedError

    def normal(self, *args):
        raise NotImplementedError


class type3_nufft_naive(linop):
    """y(t) = sum_r x(r) exp(-2 pi i phi(r) . alpha(t)) by explicit summation
    (linops.py:49-121): phis (B, *im_size), alphas (B, *trj_size). Forms the
    dense (R, T) encoding matrix as the reference does, so it is for small
    problems; type3_nufft is the fast transform."""

    def __init__(self, phis: torch.Tensor, alphas: torch.Tensor):
        super().__init__(phis.shape[1:], alphas.shape[1:])
        B = phis.shape[0]
        assert phis.shape[0] == alphas.shape[0], "phis and alphas must have same number of bases (B)"
        self.phis = phis.reshape((B, -1))
        self.alphas = alphas.reshape((B, -1))

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        N = x.shape[0]
        enc = torch.exp(-2j * torch.pi * (self.phis.T @ self.alphas))
        return (x.reshape((N, -1)) @ enc).reshape((N, *self.oshape))

    def adjoint(self, y: torch.Tensor) -> torch.Tensor:
        N = y.shape[0]
        enc = torch.exp(2j * torch.pi * (self.alphas.T @ self.phis))
        return (y.reshape((N, -1)) @ enc).reshape((N, *self.ishape))

    def normal(self, x: torch.Tensor) -> torch.Tensor:
        return self.adjoint(self.forward(x))


class type3_nufft(linop):
    """Kaiser-Bessel type-3 NUFFT y_k = sum_n x_n exp(-2 pi i phi_n . alpha_k)
    (linops.py:123-425, after Barnett et al.), on the B200 kernels:

    1. midpoint phase, then gridding of x at the rescaled phis onto a
       (2 S os + W)-point grid per basis with a width-W KB kernel whose beta
       differs per axis (the raw gridding plan, generic tile kernels);
    2. type-2 NUFFT of that grid at alphas * gamma (b200_nufft with the
       os 1.25 / W 6 defaults the reference's sigpy_nufft uses);
    3. deapodization by the KB transform, output midpoint phase.
    The adjoint runs the same steps transposed; normal() uses the Toeplitz
    embedding of step 2 when ``use_toep``. The constants follow the
    reference's float32 formulas (linops.py:170-205), including its choice
    of per-axis oversampling. Bases B = 1..3 (the reference allows up to 5)."""

    def __init__(self, phis: torch.Tensor, alphas: torch.Tensor, oversamp: float = 2.0,
                 width: float = 4.0, use_toep: Optional[bool] = False):
        B, *im_size = phis.shape
        B_, *trj_size = alphas.shape
        assert B == B_, "phis and alphas must have same number of bases (B)"
        assert phis.device == alphas.device, "phis and alphas must be on same device"
        if not 1 <= B <= 3:
            raise NotImplementedError(f"type3_nufft on B200 supports 1-3 bases, got {B}")
        super().__init__(tuple(im_size), tuple(trj_size))
        R = 1
        for n in im_size:
            R *= int(n)
        T = 1
        for n in trj_size:
            T *= int(n)
        ph = phis.reshape((B, R)).to(real_dtype)
        al = alphas.reshape((B, T)).to(real_dtype)
        ph_mp = (ph.min(dim=1).values + ph.max(dim=1).values) / 2
        al_mp = (al.min(dim=1).values + al.max(dim=1).values) / 2
        ph_c = ph - ph_mp[:, None]
        al_c = al - al_mp[:, None]
        scales = ph_c.abs().max(dim=1).values * 2
        ph_c = ph_c / scales[:, None]
        ph_mp = ph_mp / scales
        al_c = al_c * scales[:, None]
        al_mp = al_mp * scales
        self.phis, self.alphas, self.phis_mp, self.alphas_mp = ph_c, al_c, ph_mp, al_mp
        self.torch_dev = phis.device
        self.B = B
        self.grd_S = al_c.abs().max(dim=1).values
        self.grd_W = float(width)
        n_os = torch.ceil(2 * self.grd_S * oversamp + self.grd_W).long()
        self.grd_os = n_os / (n_os / oversamp).round()
        self.grd_N = n_os / self.grd_os
        self.grd_gamma = n_os / (2 * self.grd_os * self.grd_S)
        self.grd_beta = torch.pi * (((self.grd_W / self.grd_os) * (self.grd_os - 0.5)) ** 2 - 0.8) ** 0.5
        self.grd_N_os = tuple((self.grd_N * self.grd_os).ceil().long().tolist())
        self.nft = b200_nufft(self.grd_N_os, oversamp=1.25, width=6)
        up = (self.grd_os * self.grd_N).ceil()
        # image-domain gridding coordinates (R, B), in grid units
        self._trj = ((up / self.grd_N) * (self.phis.T * self.grd_N / self.grd_gamma) + up // 2).contiguous()
        self._kp = {"beta": tuple(float(b) for b in self.grd_beta.tolist())}
        self._apod_t = self.apod(self.alphas.T * self.grd_gamma / self.grd_N / self.grd_os,
                                 self.grd_beta, self.grd_W).prod(dim=-1)
        self._ktrj = (self.alphas.T * self.grd_gamma).contiguous()  # (T, B)
        self._ktrj_n = {}  # batch size -> (N, T, B) trajectory, kept so the NUFFT plan is reused
        self.kerns = None
        if use_toep:
            self.kerns = self.nft.calc_teoplitz_kernels(trj=self._ktrj[None], weights=self._apod_t[None] ** 2)

    @staticmethod
    def apod(x, beta, W):
        a = (beta ** 2 - (torch.pi * W * x) ** 2) ** 0.5
        return a / torch.sinh(a)

    def _grid(self, xv):
        from .interp import grid
        g = grid(xv.contiguous(), self._trj, self.grd_N_os, self.grd_W, kernel_params=self._kp)
        return g / self.grd_W ** self.B

    def _interp(self, g):
        from .interp import ungrid
        return ungrid(g.contiguous(), self._trj, self.grd_W, kernel_params=self._kp) / self.grd_W ** self.B

    def _trj_for(self, N):
        t = self._ktrj_n.get(N)
        if t is None:
            t = self._ktrj_n[N] = self._ktrj[None].expand(N, -1, -1).contiguous()
        return t

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        N = x.shape[0]
        phz = self.phis.T @ self.alphas_mp
        x_mp = x.reshape(N, -1) * torch.exp(-2j * torch.pi * phz)
        x_grid = self._grid(x_mp.to(complex_dtype))
        trj = self._trj_for(N)
        y = self.nft.forward(x_grid, trj) * float(torch.tensor(self.grd_N_os).prod()) ** 0.5
        y = y * self._apod_t
        phz = (self.alphas.T + self.alphas_mp) @ self.phis_mp
        y = y * torch.exp(-2j * torch.pi * phz)
        return y.reshape((N, *self.oshape))

    def adjoint(self, y: torch.Tensor) -> torch.Tensor:
        N = y.shape[0]
        phz = self.alphas.T @ self.phis_mp
        y_mp = y.reshape((N, -1)) * torch.exp(2j * torch.pi * phz)
        y_apod = (y_mp * self._apod_t).to(complex_dtype)
        trj = self._trj_for(N)
        x_grid = self.nft.adjoint(y_apod, trj) * float(torch.tensor(self.grd_N_os).prod()) ** 0.5
        x = self._interp(x_grid)
        phz = (self.phis.T + self.phis_mp) @ self.alphas_mp
        x = x * torch.exp(2j * torch.pi * phz)
        return x.reshape((N, *self.ishape))

    def normal(self, x: torch.Tensor) -> torch.Tensor:
        if self.kerns is None:
            return self.adjoint(self.forward(x))
        N = x.shape[0]
        B = self.B
        phz = (self.phis.T + self.phis_mp) @ self.alphas_mp
        x_mp = x.reshape(N, -1) * torch.exp(-2j * torch.pi * phz)
        x_grid = self._grid(x_mp.to(complex_dtype))
        x_zp = resize(x_grid, [N] + [2 * n for n in self.grd_N_os])
        x_ft = fft(x_zp, dim=tuple(range(-B, 0))) * self.kerns
        x_grid = resize(ifft(x_ft, dim=tuple(range(-B, 0))), (N, *self.grd_N_os))
        x_grid = x_grid * float(torch.tensor(self.grd_N_os).prod())
        xo = self._interp(x_grid.to(complex_dtype)) * torch.exp(2j * torch.pi * phz)
        return xo.reshape((N, *self.ishape))


class _LowRankPlan:
    """Components j = (k, l) of a low-rank SENSE model, k a subspace
    coefficient (image k) and l a segment (spatial function b_l), on one
    multi-slice plan whose slices share the trajectory (mrn_lr_forward /
    mrn_lr_adjoint / mrn_lr_normal). Components are ordered k-major, so
    the image-side sums over segments are one reshape and sum in a fixed
    order. ``weights`` (K, L, M) holds the temporal weight of each component
    (phi_k(t) h_l(t)); ``spatial`` (L, *im) the b_l."""

    def __init__(self, nufft: b200_nufft, trj, mps, dcf, spatial, weights):
        K, L, M = weights.shape
        im = tuple(mps.shape[1:])
        C = mps.shape[0]
        d = trj.shape[-1]
        J = K * L
        dev = trj.device
        self.K, self.L, self.J, self.im, self.C, self.M = K, L, J, im, C, M
        self.plan = Plan([im] * J, [M] * J, [C] * J, nufft.oversamp, nufft._widths(), nufft.beta,
                         apodize=nufft.apodize, tile=nufft.tile, coil_group=nufft.coil_group,
                         max_chunk=nufft.max_chunk, device=dev, fast=nufft.fast,
                         warp_grid=nufft.warp_grid, weight_tables=nufft.weight_tables,
                         reg_grid=nufft.reg_grid, reg_interp=nufft.reg_interp)
        # the low-rank calls never run the SENSE normal's entry-order samples
        self.plan.set_option(_lib.MRN_OPT_ENTRY_MAJOR, 0)
        self.plan.set_traj(trj.reshape(1, M, d).expand(J, M, d).contiguous().reshape(-1))
        self.mps = mps.to(complex_dtype).reshape(1, -1).expand(J, -1).contiguous().reshape(-1)
        self.w_fwd = weights.to(complex_dtype).reshape(J, M).contiguous()
        self.w_adj = (self.w_fwd * dcf.reshape(1, M).to(real_dtype)).contiguous()
        self.b = spatial.to(complex_dtype).reshape(L, -1).contiguous()

    def _components(self, alphas):
        """(K, *im) coefficient images -> (K*L, N) component images b_l alpha_k."""
        a = alphas.to(complex_dtype).reshape(self.K, 1, -1)
        return (a * self.b[None]).reshape(self.J, -1).contiguous()

    def _gather(self, xc):
        """(K*L, N) component images -> (K, N): sum_l conj(b_l) x_(k,l)."""
        return (xc.reshape(self.K, self.L, -1) * self.b.conj()[None]).sum(1)

    def forward(self, alphas):
        ksp = torch.empty((self.C, self.M), dtype=complex_dtype, device=alphas.device)
        self.plan.lr_forward(self._components(alphas), self.mps, self.w_fwd, ksp)
        return ksp

    def adjoint(self, ksp):
        xc = torch.empty((self.J, self.b.shape[1]), dtype=complex_dtype, device=ksp.device)
        self.plan.lr_adjoint(ksp.to(complex_dtype).contiguous(), self.w_adj, self.mps, xc)
        return self._gather(xc)

    def normal(self, alphas):
        xc = self._components(alphas)
        out = torch.empty_like(xc)
        self.plan.lr_normal(xc, self.mps, self.w_fwd, self.w_adj, out)
        return self._gather(out)


class sense_linop(linop):
    """SENSE model y_c = sum_l h_l * F(S_c * b_l * x) (linops.py:1041-1308)."""

    def __init__(self, trj: torch.Tensor, mps: torch.Tensor, dcf: Optional[torch.Tensor] = None,
                 nufft: Optional[NUFFT] = None, use_toeplitz: Optional[bool] = False,
                 spatial_funcs: Optional[torch.Tensor] = None,
                 temporal_funcs: Optional[torch.Tensor] = None,
                 bparams: Optional[batching_params] = batching_params()):
        im_size = tuple(mps.shape[1:])
        trj_size = tuple(trj.shape[:-1])
        ncoils = mps.shape[0]
        super().__init__(im_size, (ncoils, *trj_size))
        dev = trj.device
        assert mps.device == dev
        _lib.require_cuda(trj, "trajectory")
        if nufft is None:
            nufft = b200_nufft(im_size)
        self.segmented = spatial_funcs is not None or temporal_funcs is not None
        if dcf is None:
            dcf = torch.ones(trj_size, dtype=real_dtype, device=dev)
        if spatial_funcs is None:
            spatial_funcs = torch.ones((1,) * (len(im_size) + 1), dtype=complex_dtype, device=dev)
        if temporal_funcs is None:
            temporal_funcs = torch.ones((1,) * (len(trj_size) + 1), dtype=complex_dtype, device=dev)
        trj = nufft.rescale_trajectory(trj).type(real_dtype)
        dcf = dcf.type(real_dtype).contiguous()
        mps = mps.type(complex_dtype).contiguous()

        self.im_size = im_size
        self.trj_size = trj_size
        self.use_toeplitz = use_toeplitz
        self.trj = trj
        self.mps = mps
        self.dcf = dcf
        self.nufft = nufft
        self.bparams = bparams
        self.spatial_funcs = spatial_funcs
        self.temporal_funcs = temporal_funcs
        self.torch_dev = dev

        # fused single-pass plan (B200 NUFFT, no time segmentation)
        self.plan = None
        if isinstance(nufft, b200_nufft) and not self.segmented:
            M = 1
            for s in trj_size:
                M *= int(s)
            self.plan = Plan([im_size], [M], [ncoils], nufft.oversamp, nufft._widths(), nufft.beta,
                             apodize=nufft.apodize, tile=nufft.tile, coil_group=nufft.coil_group,
                             max_chunk=nufft.max_chunk, device=dev, fast=nufft.fast,
                             warp_grid=nufft.warp_grid, weight_tables=nufft.weight_tables,
                             reg_grid=nufft.reg_grid, reg_interp=nufft.reg_interp)
            if getattr(nufft, "autotune", False):
                from .autotune import autotune
                autotune(self.plan, trj.contiguous())
            else:
                self.plan.set_traj(trj.contiguous())

        # zero-order time segments (alpha_segementation's default): every sample
        # lies in exactly one segment, so A = sum_l P_l A_l B_l with disjoint
        # sample selections P_l and A^H A = sum_l conj(b_l) A_l^H A_l (b_l x):
        # one uneven multi-slice plan, slice l = segment l's samples, runs the
        # whole operator with each sample interpolated / gridded once
        self.seg = None
        if (isinstance(nufft, b200_nufft) and self.segmented and not use_toeplitz
                and not trj.requires_grad):
            self.seg = self._segment_plan(nufft, trj, mps, dcf, spatial_funcs, temporal_funcs)

        # any other segmentation (least-squares interpolators, linops.py:1151-1176,
        # 1196-1226): every segment is one component of a low-rank plan, the
        # temporal weights applied in the fused combine / gridding prologue
        self.lr = None
        if (isinstance(nufft, b200_nufft) and self.segmented and self.seg is None
                and not use_toeplitz and not trj.requires_grad):
            self.lr = self._lowrank_plan(nufft, trj, mps, dcf, spatial_funcs, temporal_funcs)

        if use_toeplitz:
            # linops.py:1102-1119: the spatial/temporal defaults are already in
            # place here, so the reference always builds (L, L, *im_os) kernels
            tf = temporal_funcs.to(complex_dtype)
            weights = einsum(tf.conj(), tf, "L1 ... , L2 ... -> L1 L2 ...")
            weights = rearrange(weights, "n1 n2 ... -> (n1 n2) ... ") * dcf[None, ...]
            kerns = []
            for b1 in range(0, weights.shape[0], bparams.toeplitz_batch_size):
                b2 = min(b1 + bparams.toeplitz_batch_size, weights.shape[0])
                kerns.append(nufft.calc_teoplitz_kernels(trj[None,], weights[b1:b2])[0])
            L = temporal_funcs.shape[0]
            self.toep_kerns = rearrange(torch.stack(kerns, dim=0), "(n1 n2) ... -> n1 n2 ...", n1=L, n2=L)
            if self.plan is not None and L == 1:
                # one image, no segments: the fused Toeplitz normal (mrn_sense_normal_toeplitz)
                self.plan.set_toeplitz(self.toep_kerns[0, 0], [tuple(self.toep_kerns.shape[-len(im_size):])])
        else:
            self.toep_kerns = None

    # ------------------------------------------------------------------
    def _segment_plan(self, nufft, trj, mps, dcf, spatial, temporal):
        """Multi-slice plan of a one-hot (zero-order) segmentation, or None
        when the temporal functions are not one-hot or the shapes differ."""
        L = temporal.shape[0]
        im, ts = self.im_size, self.trj_size
        if spatial.shape[0] != L or tuple(spatial.shape[1:]) != tuple(im):
            return None
        tf = temporal.expand((L, *ts))
        nz = tf != 0
        if not bool((nz.sum(0) == 1).all()) or not bool((tf[nz] == 1).all()):
            return None
        dev = trj.device
        M = int(nz[0].numel())
        d = trj.shape[-1]
        C = mps.shape[0]
        inds = nz.reshape(L, M).to(torch.int32).argmax(0)
        order = torch.argsort(inds, stable=True)
        counts = torch.bincount(inds, minlength=L)
        plan = Plan([tuple(im)] * L, [int(c) for c in counts.tolist()], [C] * L, nufft.oversamp,
                    nufft._widths(), nufft.beta, apodize=nufft.apodize, tile=nufft.tile,
                    coil_group=nufft.coil_group, max_chunk=nufft.max_chunk, device=dev,
                    fast=nufft.fast, warp_grid=nufft.warp_grid, weight_tables=nufft.weight_tables,
                    reg_grid=nufft.reg_grid, reg_interp=nufft.reg_interp)
        plan.set_traj(trj.reshape(M, d)[order].contiguous().reshape(-1))
        # plan k-space position of (coil c, sample t): ksp_off[l] + c * M_l + rank of t in l
        start = torch.cumsum(counts, 0) - counts
        pos = torch.empty(M, dtype=torch.int64, device=dev)
        pos[order] = torch.arange(M, device=dev)
        koff = torch.as_tensor(plan.ksp_off, dtype=torch.int64, device=dev)
        base = koff[inds] + (pos - start[inds])
        src = (base[None, :] + torch.arange(C, device=dev)[:, None] * counts[inds][None, :]).reshape(-1)
        return {"plan": plan, "src": src, "L": L,
                "mps": mps.reshape(1, -1).expand(L, -1).contiguous().reshape(-1),
                "dcf": dcf.reshape(M)[order].contiguous(),
                "b": spatial.to(complex_dtype).reshape(L, -1).contiguous()}

    def _lowrank_plan(self, nufft, trj, mps, dcf, spatial, temporal):
        """Low-rank plan of L segments (K = 1), or None when the shapes do
        not broadcast to one spatial function and one temporal weight per
        segment."""
        L = max(spatial.shape[0], temporal.shape[0])
        im, ts = self.im_size, self.trj_size
        try:
            sp = spatial.to(complex_dtype).expand((L, *im))
            tf = temporal.to(complex_dtype).expand((L, *ts))
        except RuntimeError:
            return None
        M = 1
        for v in ts:
            M *= int(v)
        return _LowRankPlan(nufft, trj.reshape(M, trj.shape[-1]), mps, dcf, sp,
                            tf.reshape(1, L, M))

    def _use_lr(self, *tensors):
        if self.lr is None:
            return False
        return not (torch.is_grad_enabled() and any(t.requires_grad for t in tensors))

    def _use_seg(self, *tensors):
        if self.seg is None:
            return False
        return not (torch.is_grad_enabled() and any(t.requires_grad for t in tensors))

    def forward(self, img: torch.Tensor) -> torch.Tensor:
        """(*im_size) -> (C, *trj_size)."""
        if self._use_seg(img):
            sg = self.seg
            xl = (sg["b"] * img.to(complex_dtype).reshape(1, -1)).reshape(-1)
            kp = torch.empty(sg["plan"].n_ksp, dtype=complex_dtype, device=img.device)
            sg["plan"].sense_forward(xl, sg["mps"], kp)
            return kp[sg["src"]].reshape((self.mps.shape[0], *self.trj_size))
        if self._use_lr(img):
            return self.lr.forward(img.reshape(1, *self.im_size)).reshape((self.mps.shape[0], *self.trj_size))
        if self.plan is not None:
            x = img.to(complex_dtype).contiguous()
            ksp = torch.empty((self.mps.shape[0], *self.trj_size), dtype=complex_dtype, device=x.device)
            self.plan.sense_forward(x, self.mps, ksp)
            return ksp
        L = self.spatial_funcs.shape[0]
        nc = self.mps.shape[0]
        ksp = torch.zeros((nc, *self.trj_size), dtype=complex_dtype, device=self.torch_dev)
        sxb = self.mps * img
        for l1, l2 in batch_iterator(L, L):
            SBx = sxb[:, None, ...] * self.spatial_funcs[l1:l2]
            FSBx = self.nufft.forward(SBx[None,], self.trj[None, ...])[0]
            ksp += (FSBx * self.temporal_funcs[l1:l2]).sum(dim=-len(self.trj_size) - 1)
        return ksp

    def adjoint(self, ksp: torch.Tensor) -> torch.Tensor:
        """(C, *trj_size) -> (*im_size)."""
        if self._use_seg(ksp):
            sg = self.seg
            kp = torch.empty(sg["plan"].n_ksp, dtype=complex_dtype, device=ksp.device)
            kp[sg["src"]] = ksp.to(complex_dtype).reshape(-1)
            xl = torch.empty_like(sg["b"])
            sg["plan"].sense_adjoint(kp, sg["dcf"], sg["mps"], xl)
            return (sg["b"].conj() * xl).sum(0).reshape(self.im_size)
        if self._use_lr(ksp):
            return self.lr.adjoint(ksp.reshape(self.mps.shape[0], -1)).reshape(self.im_size)
        if self.plan is not None:
            y = ksp.to(complex_dtype).contiguous()
            img = torch.empty(self.im_size, dtype=complex_dtype, device=y.device)
            self.plan.sense_adjoint(y, self.dcf, self.mps, img)
            return img
        L = self.temporal_funcs.shape[0]
        img = torch.zeros(self.im_size, dtype=complex_dtype, device=self.torch_dev)
        kw = ksp * self.dcf[None, ...]
        for l1, l2 in batch_iterator(L, L):
            HWy = kw[:, None, ...] * self.temporal_funcs[l1:l2].conj()
            FHWy = self.nufft.adjoint(HWy[None, ...], self.trj[None, ...])[0]
            SFHWy = einsum(FHWy, self.mps.conj(), "nc nseg ..., nc ... -> nseg ...")
            img += (SFHWy * self.spatial_funcs[l1:l2].conj()).sum(dim=-len(self.im_size) - 1)
        return img

    def normal(self, img: torch.Tensor) -> torch.Tensor:
        """A^H A x (linops.py:1230-1308)."""
        if not self.use_toeplitz:
            if self._use_seg(img):
                sg = self.seg
                xl = (sg["b"] * img.to(complex_dtype).reshape(1, -1)).contiguous()
                out = torch.empty_like(xl)
                sg["plan"].sense_normal(xl, sg["mps"], sg["dcf"], out)
                return (sg["b"].conj() * out).sum(0).reshape(self.im_size)
            if self._use_lr(img):
                return self.lr.normal(img.reshape(1, *self.im_size)).reshape(self.im_size)
            if self.plan is not None:
                x = img.to(complex_dtype).contiguous()
                out = torch.empty_like(x)
                self.plan.sense_normal(x, self.mps, self.dcf, out)
                return out
            return self.adjoint(self.forward(img))
        if self.plan is not None and getattr(self.plan, "toeplitz_pad", None) is not None:
            x = img.to(complex_dtype).contiguous()
            out = torch.empty_like(x)
            self.plan.sense_normal_toeplitz(x, self.mps, out)
            return out
        L = self.temporal_funcs.shape[0]
        dim = len(self.im_size)
        im_size_os = self.toep_kerns.shape[-dim:]
        padder = PadLast(im_size_os, self.im_size)
        img_hat = torch.zeros_like(img)
        kern = self.toep_kerns
        Sx = self.mps * img
        SBx = Sx[:, None, ...] * self.spatial_funcs  # C L *im
        FSBx = fft(padder.forward(SBx), dim=tuple(range(-dim, 0)))
        for m1, m2 in batch_iterator(L, 1 if dim == 3 else L):
            MF = einsum(kern[m1:m2], FSBx, "M L ..., C L ... -> C M ...")
            y = padder.adjoint(ifft(MF, dim=tuple(range(-dim, 0))))
            y = (y * self.spatial_funcs[m1:m2].conj()).sum(dim=-dim - 1)
            img_hat += (y * self.mps.conj()).sum(dim=0)
        return img_hat


def _subspace_weights(phi, temporal, trj_size):
    """(K, L, M) component weights phi_k(t) h_l(t); phi (K, T) runs along the
    last trajectory dimension (linops.py:1640, 'nsub ntr')."""
    K = phi.shape[0]
    L = temporal.shape[0]
    ts = tuple(trj_size)
    ph = phi.to(complex_dtype).reshape((K,) + (1,) * (len(ts) - 1) + (ts[-1],)).expand((K, *ts))
    tf = temporal.to(complex_dtype).expand((L, *ts))
    return (ph[:, None] * tf[None]).reshape(K, L, -1)


class subspace_linop(linop):
    """Subspace model y_c = sum_k phi_k(t) sum_l h_l(t) F(S_c b_l alpha_k)
    (linops.py:1496-1772): alphas (nsub, *im_size) -> ksp (C, *trj_size),
    phi (nsub, ntr) along the last trajectory dimension. With the B200 NUFFT
    every (coefficient, segment) pair is one component of a low-rank plan
    (mrn_lr_*): one pre / FFT / interpolation pass over all components with
    the phi_k h_l weights summed in a fused combine, and a gridding that
    reads the k-space once per component with conj(phi_k h_l) dcf applied
    in its prologue, where the reference loops over coil, segment and
    subspace batches (linops.py:1613-1700). The Toeplitz normal follows
    linops.py:1703-1772 on the B200 kernels' PSFs."""

    def __init__(self, im_size: tuple, trj: torch.Tensor, mps: torch.Tensor, phi: torch.Tensor,
                 dcf: Optional[torch.Tensor] = None, nufft: Optional[NUFFT] = None,
                 use_toeplitz: Optional[bool] = False, spatial_funcs: Optional[torch.Tensor] = None,
                 temporal_funcs: Optional[torch.Tensor] = None,
                 bparams: Optional[batching_params] = batching_params()):
        im_size = tuple(im_size)
        ishape = (phi.shape[0], *im_size)
        oshape = (mps.shape[0], *trj.shape[:-1])
        super().__init__(ishape, oshape)
        dev = trj.device
        assert phi.device == dev and mps.device == dev
        _lib.require_cuda(trj, "trajectory")
        if nufft is None:
            nufft = b200_nufft(im_size)
        trj_size = tuple(trj.shape[:-1])
        if dcf is None:
            dcf = torch.ones(trj_size, dtype=real_dtype, device=dev)
        if spatial_funcs is None:
            spatial_funcs = torch.ones((1,) * len(ishape), dtype=complex_dtype, device=dev)
        if temporal_funcs is None:
            temporal_funcs = torch.ones((1,) * len(oshape), dtype=complex_dtype, device=dev)
        trj = nufft.rescale_trajectory(trj).type(real_dtype)
        dcf = dcf.type(real_dtype)
        mps = mps.type(complex_dtype)
        phi = phi.type(complex_dtype)
        self.im_size = im_size
        self.trj_size = trj_size
        self.use_toeplitz = use_toeplitz
        self.trj, self.phi, self.mps, self.dcf = trj, phi, mps, dcf
        self.nufft = nufft
        self.bparams = bparams
        self.torch_dev = dev
        self.spatial_funcs = spatial_funcs
        self.temporal_funcs = temporal_funcs

        self.toep_kerns = None
        if use_toeplitz:
            # linops.py:1581-1601: kernels for every (nsub1, nsub2) pair of the
            # weights conj(phi_1) phi_2 dcf
            if spatial_funcs.numel() > 1:
                raise NotImplementedError("Toeplitz subspace model with spatial functions")
            K = phi.shape[0]
            phis = phi.conj()[:, None, :] * phi[None, ...]
            w = rearrange(phis, "k1 k2 ntr -> (k1 k2) ntr")
            w = w.reshape((K * K,) + (1,) * (len(trj_size) - 1) + (trj_size[-1],)) * dcf
            kerns = [nufft.calc_teoplitz_kernels(trj[None], w[a:a + 1]) for a in range(K * K)]
            self.toep_kerns = rearrange(torch.cat(kerns, 0), "(k1 k2) ... -> k1 k2 ...", k1=K, k2=K)

        self.lr = None
        if isinstance(nufft, b200_nufft) and not use_toeplitz and not trj.requires_grad:
            L = max(spatial_funcs.shape[0], temporal_funcs.shape[0])
            sp = spatial_funcs.to(complex_dtype).expand((L, *im_size))
            wts = _subspace_weights(phi, temporal_funcs.expand((L, *trj_size)), trj_size)
            self.lr = _LowRankPlan(nufft, trj.reshape(-1, trj.shape[-1]), mps, dcf, sp, wts)

    def _use_lr(self, *tensors):
        if self.lr is None:
            return False
        return not (torch.is_grad_enabled() and any(t.requires_grad for t in tensors))

    def forward(self, alphas: torch.Tensor) -> torch.Tensor:
        """(nsub, *im_size) -> (C, *trj_size) (linops.py:1613-1655)."""
        if self._use_lr(alphas):
            return self.lr.forward(alphas).reshape(self.oshape)
        nc = self.mps.shape[0]
        ksp = torch.zeros((nc, *self.trj_size), dtype=complex_dtype, device=self.torch_dev)
        L = self.spatial_funcs.shape[0]
        for l1, l2 in batch_iterator(L, L):
            mw = self.mps[:, None] * self.spatial_funcs[l1:l2]
            Sx = einsum(mw, alphas.to(complex_dtype), "nc nseg ..., nsub ... -> nc nsub nseg ...")
            FSx = self.nufft.forward(Sx[None], self.trj[None])[0]  # nc nsub nseg *trj
            ph = self.phi.reshape((self.phi.shape[0], 1) + (1,) * (len(self.trj_size) - 1) + (self.trj_size[-1],))
            PFSx = (FSx * ph[None]).sum(1)  # nc nseg *trj
            ksp += (PFSx * self.temporal_funcs[l1:l2]).sum(1)
        return ksp

    def adjoint(self, ksp: torch.Tensor) -> torch.Tensor:
        """(C, *trj_size) -> (nsub, *im_size) (linops.py:1657-1700)."""
        if self._use_lr(ksp):
            return self.lr.adjoint(ksp.reshape(self.mps.shape[0], -1)).reshape(self.ishape)
        L = self.spatial_funcs.shape[0]
        kw = ksp.to(complex_dtype) * self.dcf[None]
        alphas = torch.zeros(self.ishape, dtype=complex_dtype, device=self.torch_dev)
        ph = self.phi.conj().reshape((self.phi.shape[0], 1) + (1,) * (len(self.trj_size) - 1) + (self.trj_size[-1],))
        for l1, l2 in batch_iterator(L, L):
            Wy = kw[:, None] * self.temporal_funcs[l1:l2].conj()  # nc nseg *trj
            PWy = Wy[:, None] * ph[None]  # nc nsub nseg *trj
            FPWy = self.nufft.adjoint(PWy[None], self.trj[None])[0]  # nc nsub nseg *im
            SF = einsum(FPWy, self.mps.conj(), "nc nsub nseg ..., nc ... -> nsub nseg ...")
            alphas += (SF * self.spatial_funcs[l1:l2].conj()).sum(1)
        return alphas

    def normal(self, alphas: torch.Tensor) -> torch.Tensor:
        """A^H A alphas (linops.py:1702-1772)."""
        if not self.use_toeplitz:
            if self._use_lr(alphas):
                return self.lr.normal(alphas).reshape(self.ishape)
            return self.adjoint(self.forward(alphas))
        dim = len(self.im_size)
        K = self.phi.shape[0]
        padder = PadLast(self.toep_kerns.shape[-dim:], self.im_size)
        Sx = self.mps[:, None] * alphas.to(complex_dtype)[None]  # nc nsub *im
        FRSx = fft(padder.forward(Sx), dim=tuple(range(-dim, 0)))
        out = torch.zeros_like(alphas, dtype=complex_dtype)
        for i in range(K):
            MF = einsum(self.toep_kerns[i], FRSx, "nsub ..., nc nsub ... -> nc ...")
            y = padder.adjoint(ifft(MF, dim=tuple(range(-dim, 0))))
            out[i] = (y * self.mps.conj()).sum(0)
        return out


class subspace_linop_new(linop):
    """Subspace model over a (segmented) sense_linop (linops.py:1379-1495):
    trj (*trj_size, d) with trj_size = (..., T), phi (K, T), alphas (K,
    *im_size). Same operator as ``subspace_linop``; runs on its low-rank
    plan (one pass over every coefficient and segment)."""

    def __init__(self, trj: torch.Tensor, mps: torch.Tensor, phi: torch.Tensor,
                 dcf: Optional[torch.Tensor] = None, nufft: Optional[NUFFT] = None,
                 use_toeplitz: Optional[bool] = False, spatial_funcs: Optional[torch.Tensor] = None,
                 temporal_funcs: Optional[torch.Tensor] = None,
                 bparams: Optional[batching_params] = batching_params()):
        im_size = tuple(mps.shape[1:])
        super().__init__((phi.shape[0], *im_size), (mps.shape[0], *trj.shape[:-1]))
        if use_toeplitz is True:
            raise NotImplementedError("Toeplitz normal operator not implemented for subspace models")
        assert phi.shape[1] == trj.shape[-2]
        self.phi = phi
        self.A = subspace_linop(im_size, trj, mps, phi, dcf=dcf, nufft=nufft, use_toeplitz=False,
                                spatial_funcs=spatial_funcs, temporal_funcs=temporal_funcs,
                                bparams=bparams)

    def forward(self, alphas: torch.Tensor) -> torch.Tensor:
        return self.A.forward(alphas)

    def adjoint(self, ksp: torch.Tensor) -> torch.Tensor:
        return self.A.adjoint(ksp)

    def normal(self, alphas: torch.Tensor) -> torch.Tensor:
        return self.A.normal(alphas)
