"""Seeded synthetic MRI workloads: trajectories (golden-angle radial,
variable-density spiral, 3D kooshball), a random-ellipse phantom, Gaussian
coil maps and complex noise. Trajectories are in grid units k_i in
[-N_i/2, N_i/2), the convention of the NUFFT. numpy generators, float32 /
complex64 outputs."""

from __future__ import annotations

import math

import numpy as np


def golden_angle_radial(n_spokes: int, n_ro: int, kmax: float) -> np.ndarray:
    """(n_spokes, n_ro, 2): readout linspace(-kmax, kmax, n_ro+1)[:-1] along
    angle n * pi * (3 - sqrt(5))."""
    r = np.linspace(-kmax, kmax, n_ro + 1)[:-1]
    ang = np.arange(n_spokes) * math.pi * (3 - math.sqrt(5))
    t = np.stack([r[None, :] * np.cos(ang)[:, None], r[None, :] * np.sin(ang)[:, None]], -1)
    return t.astype(np.float32)


def vd_spiral(n_interleaves: int, n_samples: int, kmax: float, alpha: float = 1.5,
              turns: float | None = None) -> np.ndarray:
    """(n_interleaves, n_samples, 2) variable-density Archimedean-type spiral:
    radius kmax * t^alpha (alpha > 1 oversamples the centre), angle
    2 pi turns t + 2 pi i / n_interleaves, clipped into [-kmax, kmax)."""
    if turns is None:
        turns = max(1.0, 2.0 * kmax / n_interleaves)
    t = np.linspace(0, 1, n_samples, endpoint=False)
    out = []
    for i in range(n_interleaves):
        r = kmax * t ** alpha
        th = 2 * math.pi * turns * t + 2 * math.pi * i / n_interleaves
        out.append(np.stack([r * np.cos(th), r * np.sin(th)], -1))
    tr = np.stack(out)
    return np.clip(tr, -kmax, np.nextafter(np.float32(kmax), np.float32(0))).astype(np.float32)


def kooshball(n_spokes: int, n_ro: int, kmax: float) -> np.ndarray:
    """(n_spokes, n_ro, 3) 3D radial: centre-out-and-back spokes through the
    origin along directions on a spiral-phyllotaxis sphere."""
    i = np.arange(n_spokes) + 0.5
    phi = np.arccos(1 - 2 * i / n_spokes / 2)  # upper hemisphere (spokes are diameters)
    theta = math.pi * (1 + 5 ** 0.5) * i
    d = np.stack([np.sin(phi) * np.cos(theta), np.sin(phi) * np.sin(theta), np.cos(phi)], -1)
    r = np.linspace(-kmax, kmax, n_ro + 1)[:-1]
    t = r[None, :, None] * d[:, None, :]
    return np.clip(t, -kmax, np.nextafter(np.float32(kmax), np.float32(0))).astype(np.float32)


def ellipse_phantom(im_size, n_ellipses: int = 20, rng=None) -> np.ndarray:
    """Sum of random ellipses (ellipsoids in 3D) with complex amplitudes."""
    rng = np.random.RandomState(0) if rng is None else rng
    d = len(im_size)
    grids = np.meshgrid(*[(np.arange(n) - n // 2) / (n / 2) for n in im_size], indexing="ij")
    img = np.zeros(im_size, dtype=np.complex128)
    for _ in range(n_ellipses):
        c = rng.uniform(-0.5, 0.5, d)
        ax = rng.uniform(0.05, 0.5, d)
        ang = rng.uniform(0, math.pi)
        amp = rng.uniform(0.2, 1.0) * np.exp(1j * rng.uniform(0, 2 * math.pi))
        x0 = grids[0] - c[0]
        x1 = grids[1] - c[1]
        xr = x0 * math.cos(ang) + x1 * math.sin(ang)
        yr = -x0 * math.sin(ang) + x1 * math.cos(ang)
        q = (xr / ax[0]) ** 2 + (yr / ax[1]) ** 2
        if d == 3:
            q = q + ((grids[2] - c[2]) / ax[2]) ** 2
        img[q <= 1] += amp
    return img.astype(np.complex64)


def gaussian_coil_maps(im_size, n_coils: int, width: float = 0.6, radius: float = 0.8) -> np.ndarray:
    """(C, *im_size) complex Gaussian bumps on a circle (2D) or sphere-ish
    spiral (3D), each with a linear phase, normalised to unit root-sum-of-squares."""
    d = len(im_size)
    grids = np.meshgrid(*[(np.arange(n) - n // 2) / (n / 2) for n in im_size], indexing="ij")
    maps = []
    for c in range(n_coils):
        a = 2 * math.pi * c / n_coils
        if d == 2:
            cen = (radius * math.cos(a), radius * math.sin(a))
        else:
            z = 1 - 2 * (c + 0.5) / n_coils
            rr = math.sqrt(max(0.0, 1 - z * z))
            cen = (radius * rr * math.cos(a * 2.4), radius * rr * math.sin(a * 2.4), radius * z)
        dist2 = sum((g - ci) ** 2 for g, ci in zip(grids, cen))
        ph = np.exp(1j * (a + 0.5 * grids[0] * math.cos(a) + 0.5 * grids[1] * math.sin(a)))
        maps.append(np.exp(-dist2 / (2 * width ** 2)) * ph)
    maps = np.stack(maps)
    rss = np.sqrt((np.abs(maps) ** 2).sum(0))
    return (maps / rss).astype(np.complex64)


def add_noise(ksp: np.ndarray, snr_db: float, rng=None) -> np.ndarray:
    """Complex Gaussian noise at the given SNR (signal power / noise power)."""
    rng = np.random.RandomState(1) if rng is None else rng
    p = np.mean(np.abs(ksp) ** 2)
    sigma = math.sqrt(p / (10 ** (snr_db / 10)) / 2)
    n = sigma * (rng.randn(*ksp.shape) + 1j * rng.randn(*ksp.shape))
    return (ksp + n).astype(np.complex64)


def randn_complex(shape, rng) -> np.ndarray:
    return (rng.randn(*shape) + 1j * rng.randn(*shape)).astype(np.complex64)
