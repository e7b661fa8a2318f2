"""Golden vectors for the off-resonance time segmentation, produced by the
reference's own ``b0_to_phis_alphas`` and ``alpha_segementation``
(src/mr_recon/imperfections/field.py:58-96, 272-369) through the import shims
in ``refshim.py``. Run once, by hand, where the reference source tree exists:

    python tests/golden/make_field_golden.py <reference>/src

Writes ``field.npz`` next to this script; the tests never import the reference.
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
    from mr_recon.imperfections.field import b0_to_phis_alphas, alpha_segementation

    rng = np.random.RandomState(11)
    im = (24, 28)
    yy, xx = np.meshgrid(np.linspace(-1, 1, im[0]), np.linspace(-1, 1, im[1]), indexing="ij")
    b0 = (60 * xx + 35 * yy ** 2 - 20 * xx * yy
          + 120 * np.exp(-((xx - 0.3) ** 2 + (yy + 0.2) ** 2) / 0.1)).astype(np.float32)
    b0 += rng.randn(*im).astype(np.float32)
    trj_size = (3, 200)
    dt = 25e-3 / trj_size[1]
    phis, alphas = b0_to_phis_alphas(torch.from_numpy(b0), trj_size, 1, dt)
    out = {"b0": b0, "dt": np.float64(dt), "trj_size": np.array(trj_size),
           "phis": phis.numpy(), "alphas": alphas.numpy()}
    for L in (4, 9):
        s, t = alpha_segementation(phis, alphas, L, interp_type="zero", verbose=False)
        out[f"zero{L}_spatial"] = s.numpy()
        out[f"zero{L}_temporal"] = t.numpy()
        s, t = alpha_segementation(phis, alphas, L, interp_type="lstsq", use_type3=False, verbose=False)
        out[f"lstsq{L}_spatial"] = s.numpy()
        out[f"lstsq{L}_temporal"] = t.numpy()
    np.savez_compressed(os.path.join(HERE, "field.npz"), **out)
    print("wrote field.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference>/src  (the mr_recon source tree)" % sys.argv[0])
    main(sys.argv[1])
