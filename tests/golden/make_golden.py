"""Generate golden input/output vectors by running the reference itself.

Runs the unmodified mr_recon package (its CPU torch fallback path:
``ungrid_torch`` / ``grid_torch``, ungrid.py:897-957 / grid.py:556-624)
through the import shims in ``refshim.py``, and writes ``*.npz`` fixtures next
to this script. Needs the reference source tree; it is run once, by hand:

    python tests/golden/make_golden.py <reference>/src

The fixtures are small (a few hundred KB in total) and committed; the tests
never import the reference.
"""

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refshim  # noqa: E402


def golden_angle_radial(n_spokes, n_ro, kmax):
    """Golden-angle radial: coordinates linspace(-kmax, kmax, n_ro+1)[:-1]
    along angle n*pi*(3-sqrt(5))."""
    r = np.linspace(-kmax, kmax, n_ro + 1)[:-1]
    ang = np.arange(n_spokes) * math.pi * (3 - math.sqrt(5))
    t = np.stack([r[None, :] * np.cos(ang)[:, None], r[None, :] * np.sin(ang)[:, None]], -1)
    return t.astype(np.float32)


def main(ref_src):
    refshim.install(ref_src)
    import torch
    from mr_recon.fourier import triton_nufft, matrix_nufft
    from mr_recon.triton_interp.kernels import kaiser_bessel_torch
    from mr_recon.triton_interp.ungrid import ungrid
    from mr_recon.triton_interp.grid import grid
    from mr_recon.linops import sense_linop, batching_params
    from mr_recon.recons import CG_SENSE_recon

    torch.set_num_threads(8)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    N = lambda t: t.detach().cpu().numpy()  # noqa: E731

    # 1. KB weight on a dense x grid, several betas (kernels.py:21-82)
    xs = np.linspace(-1.05, 1.05, 4201).astype(np.float32)
    betas = np.array([1.0, 7.0, 10.95, 13.86], dtype=np.float64)
    kb = np.stack([N(kaiser_bessel_torch(T(xs), beta=float(b))) for b in betas])
    np.savez_compressed(os.path.join(HERE, "kb.npz"), x=xs, beta=betas, w=kb)

    # 2. ungrid / grid, 1D-3D, with edge coordinates (ungrid.py:34-63, grid.py:32-67)
    rng = np.random.RandomState(1234)
    cases = {}
    for d, gshape, width, beta, B, P in [
        (1, (37,), 6, 10.95, 3, 200),
        (2, (40, 36), 6, 10.95, 3, 500),
        (2, (33, 30), 5, 9.2, 2, 300),
        (3, (12, 10, 14), 4, 7.0, 2, 300),
    ]:
        locs = (rng.rand(P, d) * 1.2 - 0.1) * np.array(gshape)
        # exact half-integer/integer edges, negatives and out-of-range points
        locs[:8] = np.round(locs[:8])
        locs[8:16] = np.round(locs[8:16]) + width / 2.0
        locs[16:20] = -np.array(gshape) * 0.5 + 0.25
        locs[20] = 0.0
        locs[21] = np.array(gshape) - 1e-4
        locs = locs.astype(np.float32)
        vals = (rng.randn(B, *gshape) + 1j * rng.randn(B, *gshape)).astype(np.complex64)
        out_u = N(ungrid(T(vals), T(locs), (width,) * d, kernel_params={"beta": beta}))
        svals = (rng.randn(B, P) + 1j * rng.randn(B, P)).astype(np.complex64)
        out_g = N(grid(T(svals), T(locs), gshape, (width,) * d, kernel_params={"beta": beta}))
        key = f"d{d}_{'x'.join(map(str, gshape))}_w{width}"
        cases[key] = dict(locs=locs, vals=vals, ungrid=out_u, svals=svals, grid=out_g,
                          width=width, beta=beta, gshape=np.array(gshape))
    np.savez_compressed(os.path.join(HERE, "interp.npz"),
                        **{f"{k}__{f}": v for k, c in cases.items() for f, v in c.items()})

    # 3. triton_nufft forward/adjoint (fourier.py:354-550)
    out = {}
    # 3a. the 128^2 golden-angle radial case: os 2, W 6, C=1, N(0,1) image
    rng = np.random.RandomState(0)
    img = (rng.randn(1, 1, 128, 128) + 1j * rng.randn(1, 1, 128, 128)).astype(np.complex64)
    trj = golden_angle_radial(64, 256, 64.0)[None]
    nf = triton_nufft((128, 128), oversamp=2.0, width=6)
    ksp = N(nf.forward(T(img), T(trj)))
    adj = N(nf.adjoint(T(ksp), T(trj)))
    out.update(r128_img=img, r128_trj=trj, r128_ksp=ksp, r128_adj=adj, r128_beta=nf.beta)
    # 3b. odd grid and odd width, two trajectories, two coils
    rng = np.random.RandomState(1)
    im = (25, 22)
    img = (rng.randn(2, 2, *im) + 1j * rng.randn(2, 2, *im)).astype(np.complex64)
    trj = ((rng.rand(2, 7, 40, 2) - 0.5) * np.array(im)).astype(np.float32)
    nf = triton_nufft(im, oversamp=1.4, width=5)
    ksp = N(nf.forward(T(img), T(trj)))
    kin = (rng.randn(*ksp.shape) + 1j * rng.randn(*ksp.shape)).astype(np.complex64)
    adj = N(nf.adjoint(T(kin), T(trj)))
    ft = N(nf.forward_FT_only(T(img)))
    out.update(odd_img=img, odd_trj=trj, odd_ksp=ksp, odd_kin=kin, odd_adj=adj, odd_ft=ft)
    # 3c. 3D, os 1.25, W 4
    rng = np.random.RandomState(2)
    im = (16, 16, 16)
    img = (rng.randn(1, 2, *im) + 1j * rng.randn(1, 2, *im)).astype(np.complex64)
    trj = ((rng.rand(1, 400, 3) - 0.5) * 16).astype(np.float32)
    nf = triton_nufft(im, oversamp=1.25, width=4)
    ksp = N(nf.forward(T(img), T(trj)))
    adj = N(nf.adjoint(T(ksp), T(trj)))
    out.update(d3_img=img, d3_trj=trj, d3_ksp=ksp, d3_adj=adj)
    # 3d. image gradient of ||A x - y||^2 through the reference autograd (interp.py:48-74)
    rng = np.random.RandomState(3)
    im = (24, 24)
    nf = triton_nufft(im, oversamp=1.25, width=6)
    x0 = (rng.randn(1, 1, *im) + 1j * rng.randn(1, 1, *im)).astype(np.complex64)
    trj = ((rng.rand(1, 300, 2) - 0.5) * 24).astype(np.float32)
    y = (rng.randn(1, 1, 300) + 1j * rng.randn(1, 1, 300)).astype(np.complex64)
    xt = T(x0).requires_grad_(True)
    loss = (nf.forward(xt, T(trj)) - T(y)).abs().square().sum()
    loss.backward()
    out.update(ag_img=x0, ag_trj=trj, ag_y=y, ag_loss=N(loss), ag_grad=N(xt.grad))
    np.savez_compressed(os.path.join(HERE, "nufft.npz"), **out)

    # 4. Toeplitz kernels + normal_toeplitz (fourier.py:63-105, 302-352, 552-582)
    rng = np.random.RandomState(4)
    im = (20, 20)
    nf = triton_nufft(im, oversamp=1.25, width=6)
    trj = ((rng.rand(1, 250, 2) - 0.5) * 20).astype(np.float32)
    wts = rng.rand(1, 250).astype(np.float32)
    kern = nf.calc_teoplitz_kernels(T(trj), T(wts))
    x = (rng.randn(1, 2, *im) + 1j * rng.randn(1, 2, *im)).astype(np.complex64)
    xn = N(nf.normal_toeplitz(T(x), kern))
    np.savez_compressed(os.path.join(HERE, "toeplitz.npz"), trj=trj, wts=wts,
                        kern=N(kern), x=x, normal=xn)

    # 5. FP64-capable NDFT pin: matrix_nufft (fourier.py:593-695)
    rng = np.random.RandomState(5)
    im = (12, 10)
    mn = matrix_nufft(im)
    x = (rng.randn(1, 2, *im) + 1j * rng.randn(1, 2, *im)).astype(np.complex64)
    trj = ((rng.rand(1, 60, 2) - 0.5) * np.array(im)).astype(np.float32)
    k = N(mn.forward(T(x), T(trj)))
    ki = (rng.randn(1, 2, 60) + 1j * rng.randn(1, 2, 60)).astype(np.complex64)
    a = N(mn.adjoint(T(ki), T(trj)))
    np.savez_compressed(os.path.join(HERE, "ndft.npz"), x=x, trj=trj, fwd=k, kin=ki, adj=a)

    # 6. sense_linop + CG_SENSE_recon (linops.py:1041-1308, recons.py:77-156)
    rng = np.random.RandomState(6)
    im = (32, 32)
    C = 4
    yy, xx = np.meshgrid(np.arange(32) - 16, np.arange(32) - 16, indexing="ij")
    mps = []
    for c in range(C):
        a = 2 * math.pi * c / C
        cx, cy = 14 * math.cos(a), 14 * math.sin(a)
        mps.append(np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * 12.0 ** 2)) * np.exp(1j * a))
    mps = np.stack(mps)
    mps = (mps / np.sqrt((np.abs(mps) ** 2).sum(0))).astype(np.complex64)
    tt = np.linspace(0, 1, 256)
    trj = []
    for il in range(4):
        ph = 2 * math.pi * il / 4
        r = 16 * tt ** 1.3
        th = 2 * math.pi * 6 * tt + ph
        trj.append(np.stack([r * np.cos(th), r * np.sin(th)], -1))
    trj = np.clip(np.stack(trj), -16, 15.99).astype(np.float32)
    truth = (rng.randn(*im) + 1j * rng.randn(*im)).astype(np.complex64)
    nf = triton_nufft(im, oversamp=1.25, width=6)
    A = sense_linop(T(trj), T(mps), nufft=nf, bparams=batching_params(coil_batch_size=C))
    ksp = N(A.forward(T(truth)))
    ksp = ksp + 0.01 * (rng.randn(*ksp.shape) + 1j * rng.randn(*ksp.shape)).astype(np.complex64)
    ksp = ksp.astype(np.complex64)
    adj = N(A.adjoint(T(ksp)))
    nrm = N(A.normal(T(truth)))
    rec = N(CG_SENSE_recon(A, T(ksp), max_iter=5, lamda_l2=1e-3, max_eigen=2.0, verbose=False))
    np.savez_compressed(os.path.join(HERE, "sense.npz"), trj=trj, mps=mps, truth=truth, ksp=ksp,
                        adj=adj, normal=nrm, cg=rec, max_eigen=2.0, lamda=1e-3, iters=5)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference>/src  (the mr_recon source tree)" % sys.argv[0])
    main(sys.argv[1])
