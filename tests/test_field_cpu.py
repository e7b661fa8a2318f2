"""Off-resonance time segmentation (mr_recon_b200.field) against vectors
produced by the reference's own b0_to_phis_alphas / alpha_segementation
(tests/golden/field.npz, made by tests/golden/make_field_golden.py). Host-side
torch code: runs on CPU."""

import os

import numpy as np
import torch

from mr_recon_b200.field import alpha_segementation, b0_to_phis_alphas

GOLD = os.path.join(os.path.dirname(__file__), "golden", "field.npz")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / max(np.linalg.norm(b), 1e-30))


def _inputs():
    g = np.load(GOLD)
    phis, alphas = b0_to_phis_alphas(torch.from_numpy(g["b0"]), tuple(int(v) for v in g["trj_size"]), 1,
                                     float(g["dt"]))
    return g, phis, alphas


def test_phis_alphas_match_reference():
    g, phis, alphas = _inputs()
    assert phis.shape == g["phis"].shape and alphas.shape == g["alphas"].shape
    assert rel(phis.numpy(), g["phis"]) < 1e-7
    assert rel(alphas.numpy(), g["alphas"]) < 1e-7


def test_zero_order_segmentation_matches_reference():
    g, phis, alphas = _inputs()
    for L in (4, 9):
        s, t = alpha_segementation(phis, alphas, L, interp_type="zero", verbose=False)
        assert rel(s.numpy(), g[f"zero{L}_spatial"]) < 1e-6
        assert np.array_equal(t.numpy(), g[f"zero{L}_temporal"])


def test_lstsq_segmentation_matches_reference():
    """The least-squares interpolator (reference run with its exact dense
    type-3 sum, use_type3=False). With L = 4 the Gram matrix is well
    conditioned and both agree to float32 accuracy. With L = 9 its condition
    number is ~2.5e3 and the reference, which solves in complex64, is off by
    ~3e-3; ours (float64) must fit the exact phase model at least as well."""
    g, phis, alphas = _inputs()
    ph = phis[0].double().numpy()
    al = alphas[0].double().numpy()
    exact = np.exp(-2j * np.pi * ph[..., None, None] * al[None, None])

    def model_err(s, t):
        ap = np.einsum("lxy,lat->xyat", s.astype(np.complex128), t.astype(np.complex128))
        return np.linalg.norm(ap - exact) / np.linalg.norm(exact)

    for L, tol in ((4, 1e-5), (9, 1e-2)):
        s, t = alpha_segementation(phis, alphas, L, interp_type="lstsq", use_type3=False, verbose=False)
        assert rel(s.numpy(), g[f"lstsq{L}_spatial"]) < 1e-6
        assert rel(t.numpy(), g[f"lstsq{L}_temporal"]) < tol
        assert model_err(s.numpy(), t.numpy()) <= model_err(g[f"lstsq{L}_spatial"], g[f"lstsq{L}_temporal"]) * (1 + 1e-6)


def test_segmented_phase_model_error_falls_with_L():
    g, phis, alphas = _inputs()
    exact = torch.exp(-2j * np.pi * phis[0][..., None, None] * alphas[0][None, None])  # (*im, 1, T)
    errs = []
    for L in (2, 4, 8, 16):
        s, t = alpha_segementation(phis, alphas, L, interp_type="lstsq", use_type3=False, verbose=False)
        approx = torch.einsum("lxy,lat->xyat", s, t)
        errs.append(rel(approx.numpy(), exact.numpy()))
    assert all(b < a for a, b in zip(errs, errs[1:])) and errs[-1] < 1e-3
