"""Golden vectors for the naive type-3 transform, produced by the
reference's own ``type3_nufft_naive`` (src/mr_recon/linops.py:49-121)
through the import shims in ``refshim.py``. The reference's Kaiser-Bessel
``type3_nufft`` (linops.py:123-425) calls sigpy, which is absent, so it has
no fixture; its restatement is pinned to these exact sums instead. Run once,
by hand, where the reference source tree exists:

    python tests/golden/make_type3_golden.py <reference>/src

Writes ``type3.npz`` next to this script; the tests never import the reference.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refshim  # noqa: E402


def main(ref_src):
    refshim.install(ref_src)
    import torch
    from mr_recon.linops import type3_nufft_naive

    rng = np.random.RandomState(23)
    out = {}
    # B = 1: a B0-like phase map over a 2D image, alphas = readout time
    im = (18, 22)
    yy, xx = np.meshgrid(np.linspace(-1, 1, im[0]), np.linspace(-1, 1, im[1]), indexing="ij")
    phis1 = (40 * xx + 25 * yy ** 2 + 30 * np.exp(-((xx - 0.3) ** 2 + yy ** 2) / 0.1))[None].astype(np.float32)
    alphas1 = np.linspace(0, 0.6, 2 * 150).reshape(1, 2, 150).astype(np.float32)
    # B = 2: two spatial bases with different spans, so the per-axis grids differ
    phis2 = np.stack([20 * xx + 3 * yy, 7 * yy ** 2 - 2 * xx]).astype(np.float32)
    alphas2 = np.stack([np.linspace(-0.4, 0.9, 240), 0.6 * np.sin(np.linspace(0, 5, 240))]).astype(np.float32)
    for tag, phis, alphas in (("b1", phis1, alphas1), ("b2", phis2, alphas2)):
        x = (rng.randn(2, *im) + 1j * rng.randn(2, *im)).astype(np.complex64)
        y = (rng.randn(2, *alphas.shape[1:]) + 1j * rng.randn(2, *alphas.shape[1:])).astype(np.complex64)
        op = type3_nufft_naive(torch.from_numpy(phis), torch.from_numpy(alphas))
        out[f"{tag}_phis"] = phis
        out[f"{tag}_alphas"] = alphas
        out[f"{tag}_x"] = x
        out[f"{tag}_y"] = y
        out[f"{tag}_fwd"] = op.forward(torch.from_numpy(x)).numpy()
        out[f"{tag}_adj"] = op.adjoint(torch.from_numpy(y)).numpy()
    np.savez_compressed(os.path.join(HERE, "type3.npz"), **out)
    print("wrote type3.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference>/src  (the mr_recon source tree)" % sys.argv[0])
    main(sys.argv[1])
