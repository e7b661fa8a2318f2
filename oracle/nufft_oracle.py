"""CPU oracle for the Kaiser-Bessel NUFFT path of mr_recon -- TEST INFRASTRUCTURE.

This module is a numpy restatement of the reference algorithm. It is the
checker for the CUDA path and nothing else: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline and
``--impl reference`` legs) may import it. The product package
``mr_recon_b200`` never imports it and has no CPU fallback.

Pinning: ``tests/golden/make_golden.py`` runs the reference package itself
(its CPU torch fallback, ``ungrid_torch`` / ``grid_torch``) through import
shims and stores input/output vectors under ``tests/golden/``;
``tests/test_oracle_golden.py`` checks this module against every one of them.

Reference files (paths inside the mr_recon project):
  src/mr_recon/triton_interp/kernels.py   KB weight, separable weights
  src/mr_recon/triton_interp/ungrid.py    type-2 interpolation (grid -> samples)
  src/mr_recon/triton_interp/grid.py      type-1 gridding (samples -> grid)
  src/mr_recon/fourier.py                 triton_nufft, matrix_nufft, Toeplitz
  src/mr_recon/utils.py                   resize, gen_grd
  src/mr_recon/linops.py                  sense_linop
  src/mr_recon/algs.py, recons.py         conjugate_gradient, CG_SENSE_recon

Floating point: weights and coordinates are formed in float32 with the same
operation order as the reference (so tap masks agree bit for bit); gathers
and scatter-adds accumulate in float64 and are rounded to complex64 at the
end, which is at least as accurate as the reference's float32 sums.
"""

from __future__ import annotations

import math
from typing import Optional, Sequence

import numpy as np

try:  # multi-threaded FFT when available; numpy.fft otherwise
    import scipy.fft as _fft

    def _fftn(x, axes, workers):
        return _fft.fftn(x, axes=axes, workers=workers)

    def _ifftn(x, axes, workers):
        return _fft.ifftn(x, axes=axes, workers=workers)
except Exception:  # pragma: no cover
    def _fftn(x, axes, workers):
        return np.fft.fftn(x, axes=axes)

    def _ifftn(x, axes, workers):
        return np.fft.ifftn(x, axes=axes)

F32 = np.float32
C64 = np.complex64
FFT_WORKERS = 1
# False: FFTs in the input's precision (complex64, as the reference's torch.fft);
# True: FFTs in complex128, so the only float32 rounding left in the NUFFT is
# that of its stage outputs (used for the float64 CG-SENSE reference solution).
FFT_DOUBLE = False


def default_beta(width: float, oversamp: float) -> float:
    """KB shape parameter, fourier.py:371-372 (triton_nufft.__init__)."""
    return math.pi * (((width / oversamp) * (oversamp - 0.5)) ** 2 - 0.8) ** 0.5


def os_shape(im_size: Sequence[int], oversamp: float):
    """Oversampled grid size ceil(os*N), fourier.py:454."""
    return tuple(int(math.ceil(oversamp * n)) for n in im_size)


# --------------------------------------------------------------------------
# Kaiser-Bessel weight: kernels.py:21-82 (torch twin of the Triton
# ``kaiser_bessel`` at kernels.py:180-246). I0 by the Abramowitz & Stegun
# polynomial approximations 9.8.1 (|z| < 3.75) and 9.8.2 (z >= 3.75), p.378.
# --------------------------------------------------------------------------
_AS_SMALL = (3.5156229, 3.0899424, 1.2067492, 0.2659732, 0.0360768, 0.0045813)
_AS_LARGE = (0.39894228, 0.01328592, 0.00225319, -0.00157565, 0.00916281,
             -0.02057706, 0.02635537, -0.01647633, 0.00392377)


def kb_weight(x, beta, dtype=F32):
    """Unnormalised KB value I0(beta*sqrt(1-x^2)) for normalised distance x.

    NaN for |x| > 1 (the reference then zeroes non-finite weights,
    kernels.py:132). Evaluated in ``dtype`` (float32 by default, as the
    reference)."""
    x = np.asarray(x, dtype=dtype)
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        z = dtype(beta) * np.sqrt(dtype(1) - x * x)
        small_mask = z < 3.75
        t = z / dtype(3.75)
        t2 = t * t
        tp = [t2 * 0 + 1]
        for _ in range(6):
            tp.append(tp[-1] * t2)
        small = tp[0].copy()
        for c, p in zip(_AS_SMALL, tp[1:]):
            small = small + dtype(c) * p
        it = dtype(1) / t
        big_poly = dtype(_AS_LARGE[0]) + 0 * t
        ip = it
        for c in _AS_LARGE[1:]:
            big_poly = big_poly + dtype(c) * ip
            ip = ip * it
        big = np.exp(z) / np.sqrt(z) * big_poly
        return np.where(small_mask, small, big).astype(dtype)


def kb_weight_deriv(x, beta, dtype=np.float64):
    """d/dx of ``kb_weight`` (the derivative of the implemented polynomials).

    Used only by the trajectory-gradient checks. With z = beta*sqrt(1-x^2),
    dz/dx = -beta^2 x / z, so d/dx = -beta^2 x * (dI0/dz)/z; for the small
    branch (dI0/dz)/z is a polynomial in t^2 and stays finite at z = 0."""
    x = np.asarray(x, dtype=dtype)
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        z = dtype(beta) * np.sqrt(dtype(1) - x * x)
        t = z / dtype(3.75)
        t2 = t * t
        # small: I = 1 + sum_k a_k t^(2k); dI/dz / z = sum_k a_k 2k t^(2k-2) / 3.75^2
        acc = np.zeros_like(t2)
        p = np.ones_like(t2)
        for k, c in enumerate(_AS_SMALL, start=1):
            acc = acc + dtype(c) * dtype(2 * k) * p
            p = p * t2
        dsmall_over_z = acc / dtype(3.75 * 3.75)
        # big: I = e^z z^-1/2 P(s), s = 3.75/z
        s = dtype(3.75) / z
        P = np.zeros_like(z)
        dP = np.zeros_like(z)
        sp = np.ones_like(z)
        for k, c in enumerate(_AS_LARGE):
            P = P + dtype(c) * sp
            if k + 1 < len(_AS_LARGE):  # P'(s) = sum_k (k+1) c_{k+1} s^k
                dP = dP + dtype(_AS_LARGE[k + 1] * (k + 1)) * sp
            sp = sp * s
        # dP/dz = P'(s) * ds/dz = P'(s) * (-3.75/z^2)
        dPdz = dP * (-dtype(3.75) / (z * z))
        ez = np.exp(z) / np.sqrt(z)
        dbig = ez * (P - P / (2 * z) + dPdz)
        dbig_over_z = dbig / z
        d_over_z = np.where(z < 3.75, dsmall_over_z, dbig_over_z)
        return (-dtype(beta) ** 2 * x * d_over_z).astype(dtype)


# --------------------------------------------------------------------------
# Coordinates
# --------------------------------------------------------------------------
def remainder_f32(a, n):
    """torch.remainder for float32 by a positive modulus (ungrid.py:873,
    grid.py:525): fmod, then add n when the result is negative."""
    a = np.asarray(a, dtype=F32)
    n = F32(n)
    m = np.fmod(a, n).astype(F32)
    return np.where(m < 0, (m + n).astype(F32), m).astype(F32)


def scale_trj(trj, im_size, oversamp):
    """fourier.py:420-430: u_i = k_i * (ceil(os N_i)/N_i) + ceil(os N_i)//2,
    as two float32 operations (no fused multiply-add)."""
    trj = np.asarray(trj, dtype=F32)
    out = trj.copy()
    d = trj.shape[-1]
    for ax in range(d):
        n = im_size[ax - d] if len(im_size) >= d else im_size[ax]
        nos = int(math.ceil(oversamp * n))
        scale = F32(nos / n)
        shift = F32(nos // 2)
        out[..., ax] = (out[..., ax] * scale).astype(F32)
        out[..., ax] = (out[..., ax] + shift).astype(F32)
    return out


def _patch_offsets(width):
    rngs = [np.arange(int(math.floor(w)) + 1) for w in width]
    mesh = np.meshgrid(*rngs, indexing="ij")
    return np.stack([m.reshape(-1) for m in mesh], axis=-1)  # (npatch, d)


def _weights(locs, grid_locs, radius, beta):
    """kernels.py:101-140 for norm='1' with the KB kernel (the NUFFT path):
    separable product of 1D weights, non-finite weights set to zero."""
    dl = ((locs[:, None, :] - grid_locs.astype(F32)) / radius).astype(F32)
    w1 = kb_weight(dl, beta)
    w = np.prod(w1, axis=-1, dtype=F32)
    w[~np.isfinite(w)] = 0
    return w


def ungrid(vals, locs, width, beta, chunk=1 << 14):
    """Type-2 interpolation, grid -> samples (ungrid.py:34-63 + the torch
    fallback ungrid_torch, ungrid.py:897-957), circular padding, norm '1'.

    vals: (B, *G) complex; locs: (P, d) float32 in grid units (not yet
    wrapped). Returns (B, P) complex64."""
    vals = np.asarray(vals)
    locs = np.asarray(locs, dtype=F32).reshape(-1, np.shape(locs)[-1])
    d = locs.shape[-1]
    gshape = vals.shape[-d:]
    B = int(np.prod(vals.shape[:-d]))
    vflat = vals.reshape(B, -1).astype(np.complex128)
    locs = np.stack([remainder_f32(locs[:, i], gshape[i]) for i in range(d)], -1)
    width = tuple(float(w) for w in (width if np.ndim(width) else (width,) * d))
    radius = (np.array(width, dtype=F32) / F32(2)).astype(F32)
    lower = np.ceil((locs - radius).astype(F32)).astype(np.int64)
    diff = _patch_offsets(width)
    P = locs.shape[0]
    out = np.zeros((B, P), dtype=np.complex128)
    strides = np.array([int(np.prod(gshape[i + 1:])) for i in range(d)], dtype=np.int64)
    for p0 in range(0, P, chunk):
        p1 = min(P, p0 + chunk)
        gl = lower[p0:p1, None, :] + diff[None]
        w = _weights(locs[p0:p1], gl, radius, beta).astype(np.float64)
        glw = np.mod(gl, np.array(gshape, dtype=np.int64))
        lin = (glw * strides).sum(-1)
        out[:, p0:p1] = np.einsum("pk,bpk->bp", w, vflat[:, lin])
    return out.reshape(*vals.shape[:-d], P).astype(C64)


def grid(vals, locs, grid_size, width, beta, chunk=1 << 14):
    """Type-1 gridding, samples -> grid, a scatter-add (grid.py:32-67 + the
    torch fallback grid_torch, grid.py:556-624), circular padding, norm '1'.

    vals: (B, P) complex; locs: (P, d). Returns (B, *grid_size) complex64."""
    vals = np.asarray(vals)
    d = len(grid_size)
    locs = np.asarray(locs, dtype=F32).reshape(-1, d)
    P = locs.shape[0]
    B = int(np.prod(vals.shape[:-1])) if vals.ndim > 1 else 1
    vflat = vals.reshape(B, P).astype(np.complex128)
    locs = np.stack([remainder_f32(locs[:, i], grid_size[i]) for i in range(d)], -1)
    width = tuple(float(w) for w in (width if np.ndim(width) else (width,) * d))
    radius = (np.array(width, dtype=F32) / F32(2)).astype(F32)
    lower = np.ceil((locs - radius).astype(F32)).astype(np.int64)
    diff = _patch_offsets(width)
    G = int(np.prod(grid_size))
    strides = np.array([int(np.prod(grid_size[i + 1:])) for i in range(d)], dtype=np.int64)
    acc_re = np.zeros((B, G))
    acc_im = np.zeros((B, G))
    for p0 in range(0, P, chunk):
        p1 = min(P, p0 + chunk)
        gl = lower[p0:p1, None, :] + diff[None]
        w = _weights(locs[p0:p1], gl, radius, beta).astype(np.float64)
        glw = np.mod(gl, np.array(grid_size, dtype=np.int64))
        lin = (glw * strides).sum(-1).reshape(-1)
        for b in range(B):
            contrib = (w * vflat[b, p0:p1, None]).reshape(-1)
            acc_re[b] += np.bincount(lin, weights=contrib.real, minlength=G)
            acc_im[b] += np.bincount(lin, weights=contrib.imag, minlength=G)
    out = (acc_re + 1j * acc_im).astype(C64)
    return out.reshape(*vals.shape[:-1], *grid_size) if vals.ndim > 1 else out.reshape(grid_size)


def pipe_menon_dcf(trj, im_size, max_iter=30, beta=8.0, width=4.0):
    """Pipe-Menon density compensation as the reference's
    density_compensation(method='sigpy') computes it (algs.py:20-106): it
    calls sigpy.mri.pipe_menon_dcf(coord, img_shape, max_iter) -- sigpy is a
    third-party dependency, unpinned in the reference's environment.yml and
    absent here. Restated from that published routine (Pipe & Menon, MRM
    41:179-186, 1999): G = sigpy's Kaiser-Bessel gridding of the samples onto
    the img_shape grid (kernel 'kaiser_bessel', width 4, param beta 8, taps
    ceil(k - w/2) .. floor(k + w/2), the A&S I0 polynomial -- the same weight
    and tap rule as the reference's triton_interp, whose kernels.py says it
    follows sigpy), circular cells; w = 1, then w <- w / |G^H G w| for
    max_iter iterations; the reference then divides by the maximum. The grid
    origin (sigpy uses the coordinates as they are, this oracle shifts them
    by N // 2) only shifts the grid circularly, which G^H G does not see."""
    trj = np.asarray(trj, dtype=F32)
    d = trj.shape[-1]
    tshape = trj.shape[:-1]
    locs = (trj.reshape(-1, d) + np.array([n // 2 for n in im_size], dtype=F32)).astype(F32)
    w = np.ones(locs.shape[0], dtype=np.complex128)
    for _ in range(int(max_iter)):
        g = grid(w.astype(C64)[None], locs, tuple(im_size), width, beta)
        ghgw = ungrid(g, locs, width, beta)[0].astype(np.complex128)
        w = w / np.abs(ghgw)
    dcf = w.real.reshape(tshape)
    return (dcf / dcf.max()).astype(F32)


# --------------------------------------------------------------------------
# Centred FFT and resize: fourier.py:37-61, utils.py:41-84
# --------------------------------------------------------------------------
def resize(x, oshape):
    """Centred zero-pad / crop, utils.py:41-84 (offsets o//2 - i//2)."""
    x = np.asarray(x)
    ishape = x.shape
    oshape = tuple(oshape)
    if ishape == oshape:
        return x.copy()
    ishift = [max(i // 2 - o // 2, 0) for i, o in zip(ishape, oshape)]
    oshift = [max(o // 2 - i // 2, 0) for i, o in zip(ishape, oshape)]
    copy = [min(i - si, o - so) for i, si, o, so in zip(ishape, ishift, oshape, oshift)]
    out = np.zeros(oshape, dtype=x.dtype)
    isl = tuple(slice(s, s + c) for s, c in zip(ishift, copy))
    osl = tuple(slice(s, s + c) for s, c in zip(oshift, copy))
    out[osl] = x[isl]
    return out


def fft_c(x, axes, norm=None):
    """fft(): ifftshift -> fftn -> fftshift (fourier.py:37-48)."""
    y = np.fft.ifftshift(x, axes=axes)
    if FFT_DOUBLE:
        y = y.astype(np.complex128)
    y = _fftn(y, axes, FFT_WORKERS)
    if norm == "ortho":
        y = y / np.sqrt(np.prod([x.shape[a] for a in axes]))
    return np.fft.fftshift(y, axes=axes)


def ifft_c(x, axes, norm=None):
    """ifft(): ifftshift -> ifftn -> fftshift (fourier.py:50-61); norm=None
    includes the 1/prod(N) factor."""
    y = np.fft.ifftshift(x, axes=axes)
    if FFT_DOUBLE:
        y = y.astype(np.complex128)
    y = _ifftn(y, axes, FFT_WORKERS)
    if norm == "ortho":
        y = y * np.sqrt(np.prod([x.shape[a] for a in axes]))
    return np.fft.fftshift(y, axes=axes)


# --------------------------------------------------------------------------
# triton_nufft: fourier.py:354-582
# --------------------------------------------------------------------------
class KBNufftOracle:
    """Restatement of ``triton_nufft`` (fourier.py:354-582)."""

    def __init__(self, im_size, oversamp=1.25, width=6, beta=None, apodize=True):
        self.im_size = tuple(int(n) for n in im_size)
        self.oversamp = float(oversamp)
        self.width = width
        self.apodize = apodize
        self.beta = default_beta(width, oversamp) if beta is None else float(beta)
        self.d = len(self.im_size)
        self.os_size = os_shape(self.im_size, self.oversamp)

    # fourier.py:376-418
    def apod_1d(self, n):
        nos = int(math.ceil(self.oversamp * n))
        x = ((np.arange(n) - n // 2) / nos).astype(F32)
        with np.errstate(invalid="ignore"):
            a = np.sqrt(F32(self.beta) ** 2 - (F32(np.pi * self.width) * x) ** 2).astype(F32)
            return (a / np.sinh(a)).astype(F32)

    def apodize_img(self, img):
        img = img.copy()
        d = self.d
        for ax in range(-d, 0):
            a = self.apod_1d(img.shape[ax])
            shp = [1] * img.ndim
            shp[ax] = -1
            img = (img * a.reshape(shp)).astype(C64)
        return img

    # fourier.py:432-468
    def forward_FT_only(self, img):
        d = self.d
        img = np.asarray(img).astype(C64)
        oshape = img.shape[:-d] + self.os_size
        x = self.apodize_img(img) if self.apodize else img.copy()
        x = (x / np.sqrt(np.prod(img.shape[-d:]))).astype(C64)
        x = resize(x, oshape)
        return fft_c(x, axes=tuple(range(-d, 0))).astype(C64)

    # fourier.py:470-503
    def forward_interp_only(self, ksp_os, trj):
        d = self.d
        trj = np.asarray(trj, dtype=F32)
        N = trj.shape[0]
        u = scale_trj(trj, self.im_size, self.oversamp)
        out = []
        for i in range(N):
            out.append(ungrid(ksp_os[i], u[i].reshape(-1, d), (self.width,) * d, self.beta)
                       .reshape(*ksp_os.shape[1:-d], *trj.shape[1:-1]))
        return (np.stack(out) / F32(self.width ** d)).astype(C64)

    # fourier.py:505-525
    def adjoint_iFT_only(self, ksp_os):
        d = self.d
        img_os = ifft_c(ksp_os, axes=tuple(range(-d, 0)))
        oshape = ksp_os.shape[:-d] + self.im_size
        out = resize(img_os, oshape)
        out = out * (np.prod(self.os_size) / np.prod(self.im_size) ** 0.5)
        out = out.astype(C64)
        if self.apodize:
            out = self.apodize_img(out)
        return out

    # fourier.py:527-550
    def adjoint_grid_only(self, ksp, trj):
        d = self.d
        trj = np.asarray(trj, dtype=F32)
        N = trj.shape[0]
        tb = trj.ndim - 2
        u = scale_trj(trj, self.im_size, self.oversamp)
        out = []
        for i in range(N):
            kb = ksp[i]
            bshape = kb.shape[:kb.ndim - tb]
            vals = kb.reshape(*bshape, -1)
            g = grid(vals.reshape(-1, vals.shape[-1]), u[i].reshape(-1, d), self.os_size,
                     (self.width,) * d, self.beta)
            out.append(g.reshape(*bshape, *self.os_size))
        return (np.stack(out) / F32(self.width ** d)).astype(C64)

    def forward(self, img, trj):
        return self.forward_interp_only(self.forward_FT_only(img), trj)

    def adjoint(self, ksp, trj):
        return self.adjoint_iFT_only(self.adjoint_grid_only(ksp, trj))

    # fourier.py:552-582 with calc_toep_kernel_helper fourier.py:63-105
    def calc_toeplitz_kernels(self, trj, weights=None, os_factor=2.0):
        d = self.d
        trj = np.asarray(trj, dtype=F32)
        im_os = tuple(int(round(n * os_factor)) for n in self.im_size)
        nos = KBNufftOracle(im_os, self.oversamp, self.width)
        if weights is None:
            weights = np.ones(trj.shape[:-1], dtype=F32)
        N = trj.shape[0]
        ksp = np.ones((N, 1) + trj.shape[1:-1], dtype=C64) * weights[:, None]
        img = nos.adjoint(ksp.astype(C64), (trj * F32(os_factor)).astype(F32))[:, 0]
        # fourier.py:37 -- the helper's fft() defaults to norm='ortho'
        return (fft_c(img, axes=tuple(range(-d, 0)), norm="ortho") * (os_factor ** d)).astype(C64)

    # fourier.py:302-352 (NUFFT.normal_toeplitz)
    def normal_toeplitz(self, img, kerns):
        d = self.d
        im_os = kerns.shape[1:]
        N = img.shape[0]
        out = np.zeros_like(img)
        flat = img.reshape(N, -1, *self.im_size)
        oflat = out.reshape(N, -1, *self.im_size)
        for n in range(N):
            x = flat[n]
            xp = resize(x, x.shape[:-d] + tuple(im_os))
            y = fft_c(xp, axes=tuple(range(-d, 0)), norm="ortho") * kerns[n]
            y = ifft_c(y, axes=tuple(range(-d, 0)), norm="ortho")
            oflat[n] = resize(y, x.shape).astype(C64)
        return out


def nufft_forward_f64(img, trj, im_size, oversamp, width, beta, apodize=True):
    """The same KB NUFFT forward as KBNufftOracle.forward (fourier.py:432-503)
    evaluated entirely in float64: a smooth function of the trajectory, used as
    the finite-difference oracle for trajectory gradients.
    img: (N, C, *im) complex; trj: (N, M, d). Returns (N, C, M) complex128."""
    im_size = tuple(im_size)
    d = len(im_size)
    nf = KBNufftOracle(im_size, oversamp, width, beta, apodize)
    img = np.asarray(img, dtype=np.complex128)
    x = img.copy()
    if apodize:
        for ax in range(-d, 0):
            n = img.shape[ax]
            nos = int(math.ceil(oversamp * n))
            xx = (np.arange(n) - n // 2) / nos
            a = np.sqrt(beta ** 2 - (np.pi * width * xx) ** 2)
            a = a / np.sinh(a)
            shp = [1] * img.ndim
            shp[ax] = -1
            x = x * a.reshape(shp)
    x = x / np.sqrt(np.prod(im_size))
    x = resize(x, x.shape[:-d] + nf.os_size)
    G = fft_c(x, axes=tuple(range(-d, 0)))
    trj = np.asarray(trj, dtype=np.float64)
    N, M = trj.shape[0], trj.shape[1]
    C = img.shape[1]
    r = width / 2.0
    K = int(math.floor(width)) + 1
    out = np.zeros((N, C, M), dtype=np.complex128)
    nos = np.array(nf.os_size)
    strides = np.array([int(np.prod(nf.os_size[i + 1:])) for i in range(d)])
    for n in range(N):
        u = trj[n] * (nos / np.array(im_size)) + nos // 2
        u = np.mod(u, nos)
        lo = np.ceil(u - r).astype(np.int64)
        offs = _patch_offsets((K - 1,) * d)
        j = lo[:, None, :] + offs[None]
        dx = j - u[:, None, :]
        valid = np.abs(dx) <= r
        w1 = kb_weight(np.where(valid, np.abs(dx) / r, 0.0), beta, np.float64)
        w = np.prod(np.where(valid, w1, 0.0), axis=-1)
        lin = (np.mod(j, nos) * strides).sum(-1)
        Gf = G[n].reshape(C, -1)
        out[n] = np.einsum("mk,cmk->cm", w, Gf[:, lin])
    return out / width ** d


# --------------------------------------------------------------------------
# FP64 direct NDFT: matrix_nufft.forward / adjoint, fourier.py:593-695,
# with r from gen_grd (utils.py:166-200): r_i = (n_i - N_i//2) / N_i.
# --------------------------------------------------------------------------
def gen_grd(im_size):
    lins = [np.arange(-(n // 2), n // 2 + (n % 2)) / n for n in im_size]
    g = np.meshgrid(*lins, indexing="ij")
    return np.stack(g, -1)


def ndft_forward(img, trj, im_size, chunk=4096):
    d = len(im_size)
    img = np.asarray(img, dtype=np.complex128)
    trj = np.asarray(trj, dtype=np.float64)
    N = img.shape[0]
    R = int(np.prod(im_size))
    rs = gen_grd(im_size).reshape(-1, d)
    xb = img.reshape(N, -1, R)
    tf = trj.reshape(N, -1, d)
    out = np.zeros((N, xb.shape[1], tf.shape[1]), dtype=np.complex128)
    for n in range(N):
        for t0 in range(0, tf.shape[1], chunk):
            t1 = min(tf.shape[1], t0 + chunk)
            enc = np.exp(-2j * np.pi * (rs @ tf[n, t0:t1].T))  # (R, T)
            out[n, :, t0:t1] = xb[n] @ enc / np.sqrt(R)
    return out.reshape(N, *img.shape[1:-d], *trj.shape[1:-1])


def ndft_adjoint(ksp, trj, im_size, chunk=4096):
    d = len(im_size)
    trj = np.asarray(trj, dtype=np.float64)
    N = trj.shape[0]
    T = int(np.prod(trj.shape[1:-1]))
    R = int(np.prod(im_size))
    rs = gen_grd(im_size).reshape(-1, d)
    kb = np.asarray(ksp, dtype=np.complex128).reshape(N, -1, T)
    tf = trj.reshape(N, T, d)
    out = np.zeros((N, kb.shape[1], R), dtype=np.complex128)
    for n in range(N):
        for t0 in range(0, T, chunk):
            t1 = min(T, t0 + chunk)
            enc = np.exp(2j * np.pi * (tf[n, t0:t1] @ rs.T))  # (T, R)
            out[n] += kb[n, :, t0:t1] @ enc / np.sqrt(R)
    return out.reshape(N, *np.shape(ksp)[1:np.ndim(ksp) - (trj.ndim - 2)], *im_size)


# --------------------------------------------------------------------------
# SENSE linop (linops.py:1041-1308) and CG (algs.py:779-872,
# recons.py:77-156), without time segmentation unless given.
# --------------------------------------------------------------------------
class SenseOracle:
    def __init__(self, trj, mps, nufft: KBNufftOracle, dcf=None,
                 spatial_funcs=None, temporal_funcs=None):
        self.trj = np.asarray(trj, dtype=F32)  # (*T, d)
        self.mps = np.asarray(mps).astype(C64)  # (C, *im)
        self.nufft = nufft
        tshape = self.trj.shape[:-1]
        self.dcf = np.ones(tshape, F32) if dcf is None else np.asarray(dcf, F32)
        d = nufft.d
        self.spatial = (np.ones((1,) * (d + 1), C64) if spatial_funcs is None
                        else np.asarray(spatial_funcs).astype(C64))
        self.temporal = (np.ones((1,) * (len(tshape) + 1), C64) if temporal_funcs is None
                         else np.asarray(temporal_funcs).astype(C64))

    def forward(self, img):  # linops.py:1134-1178
        L = self.spatial.shape[0]
        out = 0
        for l in range(L):
            x = (self.mps * img * self.spatial[l]).astype(C64)
            k = self.nufft.forward(x[None], self.trj[None])[0]
            out = out + k * self.temporal[l]
        return np.asarray(out).astype(C64)

    def adjoint(self, ksp):  # linops.py:1180-1228
        L = self.temporal.shape[0]
        out = 0
        kw = ksp * self.dcf
        for l in range(L):
            y = (kw * np.conj(self.temporal[l])).astype(C64)
            x = self.nufft.adjoint(y[None], self.trj[None])[0]
            out = out + (x * np.conj(self.mps)).sum(0) * np.conj(self.spatial[l])
        return np.asarray(out).astype(C64)

    def normal(self, img):  # linops.py:1230-1247 (non-Toeplitz branch)
        return self.adjoint(self.forward(img))


class SubspaceOracle:
    """subspace_linop (linops.py:1496-1772): alphas (K, *im) -> ksp (C, *T),
    y_c = sum_k phi_k(t) sum_l h_l(t) F(S_c b_l alpha_k), phi (K, ntr) along
    the last trajectory dimension; adjoint alpha_k = sum_l conj(b_l) sum_c
    conj(S_c) F^H(conj(phi_k) conj(h_l) dcf y_c) (linops.py:1657-1700)."""

    def __init__(self, trj, mps, phi, nufft: KBNufftOracle, dcf=None,
                 spatial_funcs=None, temporal_funcs=None):
        self.sense = SenseOracle(trj, mps, nufft, dcf, spatial_funcs, temporal_funcs)
        tshape = self.sense.trj.shape[:-1]
        phi = np.asarray(phi).astype(C64)
        self.phi = phi.reshape((phi.shape[0],) + (1,) * (len(tshape) - 1) + (tshape[-1],))

    def forward(self, alphas):  # linops.py:1613-1655
        out = 0
        for k in range(self.phi.shape[0]):
            out = out + self.sense.forward(alphas[k]) * self.phi[k]
        return np.asarray(out).astype(C64)

    def adjoint(self, ksp):  # linops.py:1657-1700
        return np.stack([self.sense.adjoint((ksp * np.conj(self.phi[k])).astype(C64))
                         for k in range(self.phi.shape[0])]).astype(C64)


def subspace_toeplitz_normal(trj, mps, phi, alphas, nufft: KBNufftOracle, dcf=None, os_factor=2.0):
    """Toeplitz normal of subspace_linop: kernels K[k1][k2] of the weights
    conj(phi_k1(t)) phi_k2(t) dcf(t) (linops.py:1581-1601, phi along the last
    trajectory dimension) and out[i] = sum_c conj(S_c) crop(IFFT(sum_k
    K[i][k] FFT(pad(S_c alpha_k)))) with orthonormal centred FFTs
    (linops.py:1703-1772)."""
    trj = np.asarray(trj, dtype=F32)
    tshape = trj.shape[:-1]
    d = nufft.d
    phi = np.asarray(phi).astype(C64)
    K = phi.shape[0]
    ph = phi.reshape((K,) + (1,) * (len(tshape) - 1) + (tshape[-1],))
    dcf = np.ones(tshape, F32) if dcf is None else np.asarray(dcf, F32)
    kern = None
    for k1 in range(K):
        for k2 in range(K):
            w = np.broadcast_to(np.conj(ph[k1]) * ph[k2] * dcf, tshape).astype(C64)
            kk = nufft.calc_toeplitz_kernels(trj[None], w[None], os_factor)[0]
            if kern is None:
                kern = np.zeros((K, K) + kk.shape, dtype=C64)
            kern[k1, k2] = kk
    im_os = kern.shape[2:]
    mps = np.asarray(mps).astype(C64)
    axes = tuple(range(-d, 0))
    sx = mps[:, None] * np.asarray(alphas).astype(C64)[None]  # C K *im
    fx = fft_c(resize(sx, sx.shape[:2] + tuple(im_os)), axes=axes, norm="ortho")
    out = np.zeros_like(np.asarray(alphas), dtype=C64)
    for i in range(K):
        mf = np.einsum("k...,ck...->c...", kern[i], fx)
        y = resize(ifft_c(mf, axes=axes, norm="ortho"), mps.shape)
        out[i] = (y * np.conj(mps)).sum(0)
    return out.astype(C64)


def _vdot_real(a, b):
    return float(np.real(np.vdot(a.astype(np.complex128), b.astype(np.complex128))))


def conjugate_gradient(AHA, AHb, num_iters=10, lamda_l2=0.0, tolerance=1e-8):
    """algs.py:779-872 (no preconditioner); x0 = AHb."""
    op = lambda v: AHA(v) + lamda_l2 * v
    x = AHb.astype(np.complex128).copy()
    if num_iters == 0:
        return x.astype(C64)
    r = AHb - op(x)
    z = r
    p = z.copy()
    for _ in range(num_iters):
        Ap = op(p)
        pAp = _vdot_real(p, Ap)
        rz = _vdot_real(r, z)
        alpha = rz / pAp
        x = x + alpha * p
        r = r - alpha * Ap
        if np.linalg.norm(r) < tolerance:
            break
        z = r
        beta = _vdot_real(r, z) / rz
        p = z + beta * p
    return x.astype(C64)


def conjugate_gradient_f32(AHA, AHb, num_iters=10, lamda_l2=0.0, tolerance=1e-8):
    """algs.py:779-872 in the reference's own arithmetic: complex64 iterates,
    float32 sums for <p, Ap>, <r, z> and |r| (torch.sum on complex64), pAp
    taken to a Python float (.item(), :845), alpha and beta float32."""
    op = lambda v: (AHA(v) + np.complex64(lamda_l2) * v).astype(C64)
    x = AHb.astype(C64).copy()
    if num_iters == 0:
        return x
    r = (AHb.astype(C64) - op(x)).astype(C64)
    z = r
    p = z.copy()
    for _ in range(num_iters):
        Ap = op(p)
        pAp = float(np.real(np.sum(np.conj(p) * Ap, dtype=C64)))
        rz = np.float32(np.real(np.sum(np.conj(r) * z, dtype=C64)))
        alpha = np.float32(rz / np.float32(pAp))
        x = (x + alpha * p).astype(C64)
        r = (r - alpha * Ap).astype(C64)
        if np.linalg.norm(r) < tolerance:
            break
        z = r
        beta = np.float32(np.float32(np.real(np.sum(np.conj(r) * z, dtype=C64))) / rz)
        p = (z + beta * p).astype(C64)
    return x


def cg_sense(A: SenseOracle, ksp, max_iter, lamda_l2, max_eigen, tolerance=1e-8):
    """recons.py:77-156 with max_eigen given (no power method)."""
    AHb = A.adjoint(ksp.astype(C64)).astype(np.complex128) / max_eigen ** 0.5
    if max_iter == 0:
        return AHb.astype(C64)
    return conjugate_gradient(lambda v: A.normal(v.astype(C64)).astype(np.complex128) / max_eigen,
                              AHb, num_iters=max_iter, lamda_l2=lamda_l2, tolerance=tolerance)


# --------------------------------------------------------------------------
# Type-3 NUFFT y(t) = sum_r x(r) exp(-2 pi i phi(r) . alpha(t)):
# type3_nufft_naive (linops.py:49-121) exactly in float64, and the
# Kaiser-Bessel type-3 of type3_nufft (linops.py:123-425, after Barnett et
# al.): image-domain gridding of x at the rescaled phis, a type-2 NUFFT of
# that grid at the rescaled alphas, deapodization, midpoint phases.
# --------------------------------------------------------------------------
def type3_naive(x, phis, alphas, chunk=2048):
    """type3_nufft_naive.forward (linops.py:72-88) in float64: x (N, *im),
    phis (B, *im), alphas (B, *trj) -> (N, *trj)."""
    B = phis.shape[0]
    ph = np.asarray(phis, np.float64).reshape(B, -1)
    al = np.asarray(alphas, np.float64).reshape(B, -1)
    N = x.shape[0]
    xf = np.asarray(x).reshape(N, -1).astype(np.complex128)
    out = np.zeros((N, al.shape[1]), np.complex128)
    for t0 in range(0, al.shape[1], chunk):
        e = np.exp(-2j * np.pi * (ph.T @ al[:, t0:t0 + chunk]))
        out[:, t0:t0 + chunk] = xf @ e
    return out.reshape((N,) + alphas.shape[1:])


def type3_naive_adjoint(y, phis, alphas, chunk=2048):
    """type3_nufft_naive.adjoint (linops.py:90-106) in float64."""
    B = phis.shape[0]
    ph = np.asarray(phis, np.float64).reshape(B, -1)
    al = np.asarray(alphas, np.float64).reshape(B, -1)
    N = y.shape[0]
    yf = np.asarray(y).reshape(N, -1).astype(np.complex128)
    out = np.zeros((N, ph.shape[1]), np.complex128)
    for r0 in range(0, ph.shape[1], chunk):
        e = np.exp(2j * np.pi * (al.T @ ph[:, r0:r0 + chunk]))
        out[:, r0:r0 + chunk] = yf @ e
    return out.reshape((N,) + phis.shape[1:])


class Type3Oracle:
    """Restatement of type3_nufft (linops.py:123-425). Constants are formed
    in float32 with the reference's operation order (linops.py:170-205); the
    inner NUFFT is sigpy_nufft's defaults (os 1.25, W 6, fourier.py:730-748),
    which compute the same transform as triton_nufft, so KBNufftOracle
    stands in for it; the image-domain gridding/interpolation is sigpy's
    separable KB with one beta per axis (the same kernel as ``grid`` /
    ``ungrid`` above)."""

    def __init__(self, phis, alphas, oversamp=2.0, width=4.0, use_toep=False):
        B = phis.shape[0]
        self.B = B
        self.ishape = tuple(phis.shape[1:])
        self.oshape = tuple(alphas.shape[1:])
        ph = np.asarray(phis, F32).reshape(B, -1)
        al = np.asarray(alphas, F32).reshape(B, -1)
        ph_mp = ((ph.min(1) + ph.max(1)) / F32(2)).astype(F32)
        al_mp = ((al.min(1) + al.max(1)) / F32(2)).astype(F32)
        ph_c = (ph - ph_mp[:, None]).astype(F32)
        al_c = (al - al_mp[:, None]).astype(F32)
        scales = (np.abs(ph_c).max(1) * F32(2)).astype(F32)
        ph_c = (ph_c / scales[:, None]).astype(F32)
        ph_mp = (ph_mp / scales).astype(F32)
        al_c = (al_c * scales[:, None]).astype(F32)
        al_mp = (al_mp * scales).astype(F32)
        self.phis, self.alphas, self.phis_mp, self.alphas_mp = ph_c, al_c, ph_mp, al_mp
        S = np.abs(al_c).max(1).astype(F32)
        W = float(width)
        n_os = np.ceil((F32(2) * S * F32(oversamp) + F32(W)).astype(F32)).astype(np.int64)
        g_os = (n_os.astype(F32) / np.round((n_os.astype(F32) / F32(oversamp)).astype(F32))).astype(F32)
        g_N = (n_os.astype(F32) / g_os).astype(F32)
        self.gamma = (n_os.astype(F32) / (F32(2) * g_os * S)).astype(F32)
        self.beta = (F32(np.pi) * np.sqrt(((F32(W) / g_os) * (g_os - F32(0.5))) ** 2 - F32(0.8))).astype(F32)
        self.n_os = tuple(int(v) for v in np.ceil((g_N * g_os).astype(F32)))
        self.g_N, self.g_os, self.W = g_N, g_os, W
        self.nft = KBNufftOracle(self.n_os, 1.25, 6)
        up = np.ceil((g_os * g_N).astype(F32)).astype(F32)
        self.trj = ((up / g_N) * (ph_c.T * g_N / self.gamma) + np.floor(up / F32(2))).astype(F32)  # (R, B)
        self.kerns = None
        if use_toep:
            w = self._apod() ** 2
            self.kerns = self.nft.calc_toeplitz_kernels((al_c.T * self.gamma)[None].astype(F32),
                                                        weights=w[None].astype(F32))

    def _apod(self):
        x = (self.alphas.T * self.gamma / self.g_N / self.g_os).astype(F32)  # (T, B)
        a = np.sqrt(self.beta.astype(np.float64) ** 2 - (np.pi * self.W * x.astype(np.float64)) ** 2)
        return np.prod(a / np.sinh(a), axis=-1)

    def _grid(self, xv):
        g = grid(xv, self.trj, self.n_os, (self.W,) * self.B, self.beta)
        return (g / F32(self.W ** self.B)).astype(C64)

    def _interp(self, g):
        v = ungrid(g, self.trj, (self.W,) * self.B, self.beta)
        return (v / F32(self.W ** self.B)).astype(C64)

    def forward(self, x):
        N = x.shape[0]
        phz = self.phis.T.astype(np.float64) @ self.alphas_mp.astype(np.float64)
        xm = (np.asarray(x).reshape(N, -1) * np.exp(-2j * np.pi * phz)).astype(C64)
        xg = self._grid(xm)
        trj = np.repeat((self.alphas.T * self.gamma)[None].astype(F32), N, 0)
        y = self.nft.forward(xg, trj).astype(np.complex128) * np.sqrt(np.prod(self.n_os))
        y = y * self._apod()
        phz = (self.alphas.T.astype(np.float64) + self.alphas_mp) @ self.phis_mp.astype(np.float64)
        return (y * np.exp(-2j * np.pi * phz)).astype(C64).reshape((N,) + self.oshape)

    def adjoint(self, y):
        N = y.shape[0]
        phz = self.alphas.T.astype(np.float64) @ self.phis_mp.astype(np.float64)
        ym = np.asarray(y).reshape(N, -1) * np.exp(2j * np.pi * phz) * self._apod()
        trj = np.repeat((self.alphas.T * self.gamma)[None].astype(F32), N, 0)
        xg = self.nft.adjoint(ym.astype(C64), trj).astype(np.complex128) * np.sqrt(np.prod(self.n_os))
        x = self._interp(xg.astype(C64)).astype(np.complex128)
        phz = (self.phis.T.astype(np.float64) + self.phis_mp) @ self.alphas_mp.astype(np.float64)
        return (x * np.exp(2j * np.pi * phz)).astype(C64).reshape((N,) + self.ishape)

    def normal(self, x):
        if self.kerns is None:
            return self.adjoint(self.forward(x))
        N = x.shape[0]
        B = self.B
        phz = (self.phis.T.astype(np.float64) + self.phis_mp) @ self.alphas_mp.astype(np.float64)
        xm = (np.asarray(x).reshape(N, -1) * np.exp(-2j * np.pi * phz)).astype(C64)
        xg = self._grid(xm)
        ax = tuple(range(-B, 0))
        xz = resize(xg, (N,) + tuple(2 * n for n in self.n_os))
        xt = ifft_c(fft_c(xz, axes=ax, norm="ortho") * self.kerns, axes=ax, norm="ortho")
        xg = (resize(xt, (N,) + self.n_os) * np.prod(self.n_os)).astype(C64)
        out = self._interp(xg).astype(np.complex128) * np.exp(2j * np.pi * phz)
        return out.astype(C64).reshape((N,) + self.ishape)
