"""Small helpers with the semantics of mr_recon's utils.py / pad.py /
fourier.py:37-61, used around the NUFFT (Toeplitz path, tests, callers)."""

from __future__ import annotations

from typing import Optional

import torch
import torch.nn as nn
import torch.nn.functional as F
import torch.fft as tfft

real_dtype = torch.float32
complex_dtype = torch.complex64


def fft(x, dim=None, norm="ortho"):
    """Centred FFT: ifftshift -> fftn -> fftshift (fourier.py:37-48)."""
    x = tfft.ifftshift(x, dim=dim)
    x = tfft.fftn(x, dim=dim, norm=norm)
    return tfft.fftshift(x, dim=dim)


def ifft(x, dim=None, norm="ortho"):
    """Centred inverse FFT: ifftshift -> ifftn -> fftshift (fourier.py:50-61)."""
    x = tfft.ifftshift(x, dim=dim)
    x = tfft.ifftn(x, dim=dim, norm=norm)
    return tfft.fftshift(x, dim=dim)


def resize(input, oshape, ishift=None, oshift=None):
    """Centred zero-pad / crop (utils.py:41-84): offsets o//2 - i//2."""
    ishape = list(input.shape)
    oshape = list(oshape)
    if len(ishape) < len(oshape):
        ishape = [1] * (len(oshape) - len(ishape)) + ishape
    if ishape == oshape:
        return input.reshape(oshape)
    if ishift is None:
        ishift = [max(i // 2 - o // 2, 0) for i, o in zip(ishape, oshape)]
    if oshift is None:
        oshift = [max(o // 2 - i // 2, 0) for i, o in zip(ishape, oshape)]
    copy = [min(i - si, o - so) for i, si, o, so in zip(ishape, ishift, oshape, oshift)]
    islice = tuple(slice(si, si + c) for si, c in zip(ishift, copy))
    oslice = tuple(slice(so, so + c) for so, c in zip(oshift, copy))
    out = torch.zeros(oshape, dtype=input.dtype, device=input.device)
    out[oslice] = input.reshape(ishape)[islice]
    return out


def gen_grd(im_size, fovs: Optional[tuple] = None, balanced: bool = False) -> torch.Tensor:
    """Grid of image coordinates r_i = (n_i - N_i//2)/N_i (utils.py:166-200)."""
    if fovs is None:
        fovs = (1,) * len(im_size)
    if balanced:
        lins = [fovs[i] * torch.linspace(-1 / 2, 1 / 2, im_size[i]) for i in range(len(im_size))]
    else:
        lins = [fovs[i] * torch.arange(-(im_size[i] // 2), im_size[i] // 2 + (im_size[i] % 2)) / im_size[i]
                for i in range(len(im_size))]
    grds = torch.meshgrid(*lins, indexing="ij")
    return torch.cat([g[..., None] for g in grds], dim=-1).type(real_dtype)


def batch_iterator(total, batch_size):
    """(start, stop) pairs over range(total) (utils.py:364-382)."""
    assert total > 0, f"batch_iterator called with {total} elements"
    delim = list(range(0, total, batch_size)) + [total]
    return zip(delim[:-1], delim[1:])


class PadLast(nn.Module):
    """Centred pad / crop of the last dims (pad.py:5-37)."""

    def __init__(self, pad_im_size, im_size):
        super().__init__()
        assert len(pad_im_size) == len(im_size)
        self.im_dim = len(im_size)
        self.im_size = tuple(im_size)
        self.pad_im_size = tuple(pad_im_size)
        for psz in pad_im_size:
            assert not (psz % 2), "Pad sizes must be even"
        sizes = [[(psz - isz) // 2] * 2 for psz, isz in zip(pad_im_size, im_size)]
        self.pad = sum(sizes, start=[])
        self.pad.reverse()
        self.crop_slice = [slice(self.pad[2 * i], -self.pad[2 * i + 1]) for i in range(len(self.pad) // 2)]
        self.crop_slice.reverse()
        if tuple(pad_im_size) == tuple(im_size):
            self.crop_slice = [slice(None)] * self.im_dim

    def forward(self, x):
        assert tuple(x.shape[-self.im_dim:]) == self.im_size
        pad = self.pad + [0, 0] * (x.ndim - self.im_dim)
        return F.pad(x, pad)

    def adjoint(self, y):
        assert tuple(y.shape[-self.im_dim:]) == self.pad_im_size
        slc = [slice(None)] * (y.ndim - self.im_dim) + self.crop_slice
        return y[tuple(slc)]
