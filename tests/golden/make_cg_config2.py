"""Oracle CG-SENSE solution of the 2D multi-coil configuration, for the GPU
parity test of the device CG at full size (tests/test_gpu_fullsize.py) and the
relative error the benchmark reports.

Problem: 256x256 random-ellipse phantom (20 ellipses, numpy seed 1234), 32
Gaussian coil maps, variable-density spiral 48 x 2048, KB NUFFT os 1.25 /
width 6, k-space = A x plus complex noise at 30 dB SNR (seed 99), max
eigenvalue of A^H A by 12 power iterations (seed 7) x 1.01, lambda 1e-3,
20 CG iterations from x0 = A^H b (recons.py:77-156, algs.py:779-872).

Stores the oracle's solution with float64 iterates (``x_cg64``), the max
eigenvalue used, and the distance of the reference's own float32 arithmetic
(``conjugate_gradient_f32``) from that solution. The oracle's FFTs run in
complex128 here (``FFT_DOUBLE``), so its operator carries only the complex64
rounding of each stage's output: a 20-iteration CG at lambda 1e-3 amplifies
rounding that differs from one operator application to the next by about
three orders of magnitude, so the reference solution must not carry more of
it than necessary. Runs on the CPU in about a
quarter of an hour (8 threads); no reference code is needed:

    python tests/golden/make_cg_config2.py
"""

import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import nufft_oracle as O  # noqa: E402
from mr_recon_b200 import synth  # noqa: E402

IM, C, LAM, ITERS = (256, 256), 32, 1e-3, 20


def problem():
    """The seeded inputs (also regenerated by the GPU test and the bench)."""
    x = synth.ellipse_phantom(IM, 20, np.random.RandomState(1234))
    mps = synth.gaussian_coil_maps(IM, C)
    trj = synth.vd_spiral(48, 2048, IM[0] / 2.0)
    return x, mps, trj


def main():
    O.FFT_WORKERS = 1
    O.FFT_DOUBLE = True
    x, mps, trj = problem()
    nf = O.KBNufftOracle(IM, 1.25, 6)
    pool = ThreadPoolExecutor(os.cpu_count() or 1)

    def fwd(img):  # (C, *IM) -> (C, 48, 2048)
        return np.stack(list(pool.map(lambda c: nf.forward(img[None, c:c + 1], trj[None])[0, 0], range(C))))

    def adj(ksp):  # (C, 48, 2048) -> (C, *IM)
        return np.stack(list(pool.map(lambda c: nf.adjoint(ksp[None, c:c + 1], trj[None])[0, 0], range(C))))

    def A(v):
        return fwd((mps * v).astype(np.complex64))

    def AH(k):
        return (adj(k.astype(np.complex64)) * np.conj(mps)).sum(0).astype(np.complex64)

    t0 = time.time()
    ksp = synth.add_noise(A(x), 30.0, np.random.RandomState(99))
    v = synth.randn_complex(IM, np.random.RandomState(7))
    lmax = 1.0
    for _ in range(12):
        z = AH(A(v))
        lmax = float(np.linalg.norm(z))
        v = (z / lmax).astype(np.complex64)
    me = 1.01 * lmax
    print(f"max eigen {me:.6g} ({time.time() - t0:.0f} s)", flush=True)
    AHb = AH(ksp) / np.float32(me ** 0.5)
    normal = lambda u: AH(A(u.astype(np.complex64))).astype(np.complex128) / me  # noqa: E731
    x64 = O.conjugate_gradient(normal, AHb.astype(np.complex128), ITERS, LAM)
    print(f"float64-iterate CG done ({time.time() - t0:.0f} s)", flush=True)
    normal32 = lambda u: (AH(A(u)) / np.float32(me)).astype(np.complex64)  # noqa: E731
    x32 = O.conjugate_gradient_f32(normal32, AHb.astype(np.complex64), ITERS, LAM)
    rel32 = float(np.linalg.norm(x32 - x64) / np.linalg.norm(x64))
    print(f"reference float32 arithmetic vs float64 iterates: {rel32:.3e} ({time.time() - t0:.0f} s)")
    np.savez_compressed(os.path.join(HERE, "cg_config2.npz"), x_cg64=x64.astype(np.complex64),
                        max_eigen=np.float64(me), rel_f32_arith=np.float64(rel32),
                        ksp_norm=np.float64(np.linalg.norm(ksp)), lam=np.float64(LAM), iters=np.int64(ITERS))


if __name__ == "__main__":
    main()
