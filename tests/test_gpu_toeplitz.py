"""GPU parity of the fused Toeplitz normal operator (mrn_toeplitz_normal,
mrn_sense_normal_toeplitz) against the oracle's restatement of
NUFFT.normal_toeplitz (fourier.py:302-352) and the Toeplitz branch of
sense_linop.normal (linops.py:1249-1308). Tolerance 1e-5 relative L2
(float32 FFTs on both sides)."""

import numpy as np
import pytest
import torch

from oracle import nufft_oracle as O
from mr_recon_b200 import synth
from mr_recon_b200.algs import SenseCG, conjugate_gradient
from mr_recon_b200.fourier import b200_nufft
from mr_recon_b200.linops import sense_linop
from mr_recon_b200.plan import Plan

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = 1e-5


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def Nn(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-30))


@pytest.mark.parametrize("im,W,C", [((48, 40), 6, 3), ((20, 18, 16), 4, 2), ((34, 30), 5, 1)])
def test_toeplitz_normal_matches_oracle(im, W, C):
    """Batched images (N = 2) with their own kernels, 2D and 3D, several coils."""
    rng = np.random.RandomState(sum(im) + C)
    d = len(im)
    trj = ((rng.rand(2, 700, d) - 0.5) * np.array(im)).astype(np.float32)
    wts = rng.rand(2, 700).astype(np.float32) + 0.5
    nf = b200_nufft(im, oversamp=1.25, width=W)
    on = O.KBNufftOracle(im, 1.25, W)
    kern = on.calc_toeplitz_kernels(trj, wts)
    x = synth.randn_complex((2, C, *im), rng)
    assert rel(Nn(nf.normal_toeplitz(T(x), T(kern))), on.normal_toeplitz(x, kern)) < TOL
    # the kernels from the B200 adjoint agree with the oracle's
    assert rel(Nn(nf.calc_teoplitz_kernels(T(trj), T(wts))), kern) < TOL


def test_toeplitz_odd_padding_is_refused():
    """PadLast pads (pad - N) / 2 cells on both sides (pad.py:5-37), so the
    reference cannot pad an odd difference; neither does the plan."""
    nf = b200_nufft((33, 30))
    kern = torch.ones((1, 66, 60), dtype=torch.complex64, device=DEV)
    with pytest.raises((ValueError, RuntimeError)):
        nf.normal_toeplitz(torch.ones((1, 1, 33, 30), dtype=torch.complex64, device=DEV), kern)


def test_toeplitz_uneven_multislice_plan():
    """Slices of different sizes (grouped padded grids, one FFT plan per size)."""
    rng = np.random.RandomState(3)
    sizes = [(24, 24), (30, 20), (24, 24)]
    coils = [2, 3, 1]
    plan = Plan(sizes, [0, 0, 0], coils, 1.25, (6.0, 6.0), device=DEV)
    pads = [tuple(2 * n for n in s) for s in sizes]
    kerns, imgs, refs = [], [], []
    for s, c in zip(sizes, coils):
        on = O.KBNufftOracle(s, 1.25, 6)
        trj = ((rng.rand(1, 400, 2) - 0.5) * np.array(s)).astype(np.float32)
        k = on.calc_toeplitz_kernels(trj)
        x = synth.randn_complex((1, c, *s), rng)
        kerns.append(k.reshape(-1))
        imgs.append(x.reshape(-1))
        refs.append(on.normal_toeplitz(x, k).reshape(-1))
    plan.set_toeplitz(T(np.concatenate(kerns)), pads)
    out = torch.empty(plan.n_img, dtype=torch.complex64, device=DEV)
    plan.toeplitz_normal(T(np.concatenate(imgs)), out)
    o = Nn(out)
    for s in range(3):
        a = o[plan.img_off[s]:plan.img_off[s] + refs[s].size]
        assert rel(a, refs[s]) < TOL


def _sense_problem(im=(40, 36), C=5, seed=5):
    rng = np.random.RandomState(seed)
    mps = synth.gaussian_coil_maps(im, C)
    trj = synth.vd_spiral(6, 400, im[0] / 2.0)
    dcf = (rng.rand(6, 400) + 0.5).astype(np.float32)
    x = synth.randn_complex(im, rng)
    return rng, mps, trj, dcf, x


def test_sense_linop_toeplitz_normal_matches_oracle():
    rng, mps, trj, dcf, x = _sense_problem()
    im = x.shape
    A = sense_linop(T(trj), T(mps), dcf=T(dcf), nufft=b200_nufft(im), use_toeplitz=True)
    on = O.KBNufftOracle(im, 1.25, 6)
    kern = on.calc_toeplitz_kernels(trj.reshape(1, -1, 2), dcf.reshape(1, -1))
    assert rel(Nn(A.toep_kerns[0, 0]), kern[0]) < TOL
    ref = (np.conj(mps) * on.normal_toeplitz((mps * x)[None], kern)[0]).sum(0)
    assert rel(Nn(A.normal(T(x))), ref) < TOL


def test_sense_cg_toeplitz_graph_eager_and_generic_cg():
    """CG-SENSE over the Toeplitz normal: graph replay == eager solve (same
    bits), and the device CG follows the generic CG over the same operator."""
    from mr_recon_b200.recons import CG_SENSE_recon
    rng, mps, trj, dcf, x = _sense_problem(seed=8)
    im = x.shape
    A = sense_linop(T(trj), T(mps), nufft=b200_nufft(im), use_toeplitz=True)
    y = A.forward(T(x))
    v = T(synth.randn_complex(im, rng))
    for _ in range(30):  # max eigenvalue of A^H A (recons.py:117-123)
        z = A.normal(v)
        lmax = float(torch.linalg.vector_norm(z))
        v = z / lmax
    me = 1.01 * lmax
    s = SenseCG(A.plan, A.mps, A.dcf, 10, 1e-2, me, toeplitz=True)
    x1 = s.solve(y.reshape(-1)).clone()
    s.capture()
    x2 = s.solve(y.reshape(-1)).clone()
    assert torch.equal(x1, x2)
    AHb = A.adjoint(y) / me ** 0.5
    xg = conjugate_gradient(lambda v: A.normal(v) / me, AHb, num_iters=10, lamda_l2=1e-2, verbose=False)
    assert rel(Nn(x1).reshape(im), Nn(xg)) < 1e-4
    xr = CG_SENSE_recon(A, y, max_iter=10, lamda_l2=1e-2, max_eigen=me, verbose=False)
    assert torch.equal(xr.reshape(-1), x1)
