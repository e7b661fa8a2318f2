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


def test_two_phase_bases_kmeans_segmentation():
    """B = 2 phase bases (field.py:321-369 with isotropic_cluster_alphas,
    216-269): the k-means centres are a Lloyd fixed point (every point is
    assigned to its nearest centre, every centre is the mean of its points,
    in the isotropically scaled alpha space), the run is deterministic, and
    the zero-order and least-squares (exact sums) segmentations approximate
    the phase model better as L grows. The reference's k-means
    (fast_pytorch_kmeans) seeds from the global RNG, so its centres cannot
    be fixed as vectors; these properties are what it converges to too."""
    from mr_recon_b200.field import isotropic_cluster_alphas, kmeans_quantize
    rng = np.random.RandomState(3)
    im, T = (24, 20), 300
    yy, xx = np.meshgrid(np.linspace(-1, 1, im[0]), np.linspace(-1, 1, im[1]), indexing="ij")
    phis = torch.from_numpy(np.stack([0.4 * xx + 0.1 * yy ** 2, 0.5 * yy]).astype(np.float32))
    t = np.linspace(0, 1, T)
    alphas = torch.from_numpy(np.stack([30 * t, 12 * np.sin(3 * t) + rng.randn(T) * 0.2]).astype(np.float32))
    cents, inds = isotropic_cluster_alphas(alphas, phis, 8)
    c2, i2 = isotropic_cluster_alphas(alphas, phis, 8)
    assert torch.equal(cents, c2) and torch.equal(inds, i2)
    # Lloyd fixed point in the scaled space
    ph = phis.reshape(2, -1).double()
    al = alphas.reshape(2, -1).double()
    sc = (ph - ((ph.min(1).values + ph.max(1).values) / 2)[:, None]).abs().max(1).values * 2
    amp = (al.min(1).values + al.max(1).values) / 2
    x = ((al - amp[:, None]) * sc[:, None]).T
    cs = (cents.double() - amp) * sc
    assert torch.equal(torch.cdist(x, cs).argmin(1), inds.reshape(-1))
    for l in range(8):
        if (inds == l).any():
            assert torch.allclose(x[inds.reshape(-1) == l].mean(0), cs[l], atol=1e-9)
    # direct use of the k-means quantiser: a clean three-cluster case
    pts = torch.cat([torch.randn(50, 2, generator=torch.Generator().manual_seed(1)) * 0.05 + c
                     for c in (torch.tensor([0., 0.]), torch.tensor([3., 0.]), torch.tensor([0., 3.]))])
    cc, ii = kmeans_quantize(pts, 3)
    assert sorted(torch.bincount(ii).tolist()) == [50, 50, 50]
    # model error falls with L
    e_true = torch.exp(-2j * np.pi * (ph.T @ al))  # (N, T)

    def err(L, kind):
        s, tf = alpha_segementation(phis, alphas, L, interp_type=kind, use_type3=False, verbose=False)
        approx = s.reshape(L, -1).T.to(torch.complex128) @ tf.reshape(L, -1).to(torch.complex128)
        return float((approx - e_true).norm() / e_true.norm())
    for kind in ("zero", "lstsq"):
        errs = [err(L, kind) for L in (3, 6, 12)]
        assert errs[0] > errs[1] > errs[2]
    assert err(6, "lstsq") < err(6, "zero")
