"""The oracle (oracle/nufft_oracle.py) against the reference's own outputs
(tests/golden/*.npz, written by tests/golden/make_golden.py from the
unmodified mr_recon CPU path). CPU only."""

import os

import numpy as np
import pytest

from oracle import nufft_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_kb_weight_matches_reference():
    g = load("kb.npz")
    for i, b in enumerate(g["beta"]):
        w = O.kb_weight(g["x"], b)
        ref = g["w"][i]
        fin = np.isfinite(ref)
        assert np.array_equal(np.isfinite(w), fin)
        assert np.max(np.abs(w[fin] - ref[fin]) / np.abs(ref[fin])) < 5e-6


def test_kb_derivative_matches_finite_differences():
    x = np.linspace(-0.999, 0.999, 4001)
    for b in [1.0, 7.0, 10.95, 13.86]:
        h = 1e-6
        fd = (O.kb_weight(x + h, b, np.float64) - O.kb_weight(x - h, b, np.float64)) / (2 * h)
        an = O.kb_weight_deriv(x, b)
        assert np.max(np.abs(fd - an)) / np.max(np.abs(an)) < 1e-6


def _interp_cases():
    g = load("interp.npz")
    keys = sorted(set(k.split("__")[0] for k in g.files))
    return [(k, {f: g[k + "__" + f] for f in ["locs", "vals", "ungrid", "svals", "grid", "width", "beta", "gshape"]})
            for k in keys]


@pytest.mark.parametrize("case", _interp_cases(), ids=lambda c: c[0])
def test_ungrid_grid_match_reference(case):
    _, c = case
    d = len(c["gshape"])
    w = (int(c["width"]),) * d
    u = O.ungrid(c["vals"], c["locs"], w, float(c["beta"]))
    gg = O.grid(c["svals"], c["locs"], tuple(int(v) for v in c["gshape"]), w, float(c["beta"]))
    assert rel(u, c["ungrid"]) < 1e-6
    assert rel(gg, c["grid"]) < 1e-6


def test_nufft_radial_128_matches_reference():
    g = load("nufft.npz")
    nf = O.KBNufftOracle((128, 128), 2.0, 6)
    assert abs(nf.beta - float(g["r128_beta"])) < 1e-12
    assert rel(nf.forward(g["r128_img"], g["r128_trj"]), g["r128_ksp"]) < 1e-6
    assert rel(nf.adjoint(g["r128_ksp"], g["r128_trj"]), g["r128_adj"]) < 1e-6


def test_nufft_odd_sizes_match_reference():
    g = load("nufft.npz")
    nf = O.KBNufftOracle((25, 22), 1.4, 5)
    assert rel(nf.forward(g["odd_img"], g["odd_trj"]), g["odd_ksp"]) < 1e-6
    assert rel(nf.adjoint(g["odd_kin"], g["odd_trj"]), g["odd_adj"]) < 1e-6
    assert rel(nf.forward_FT_only(g["odd_img"]), g["odd_ft"]) < 1e-6


def test_nufft_3d_matches_reference():
    g = load("nufft.npz")
    nf = O.KBNufftOracle((16, 16, 16), 1.25, 4)
    assert rel(nf.forward(g["d3_img"], g["d3_trj"]), g["d3_ksp"]) < 2e-6
    assert rel(nf.adjoint(g["d3_ksp"], g["d3_trj"]), g["d3_adj"]) < 2e-6


def test_nufft_close_to_ndft_at_os2():
    g = load("nufft.npz")
    nd = O.ndft_forward(g["r128_img"][:, :, :, :], g["r128_trj"][:, :8], (128, 128))
    assert rel(g["r128_ksp"][:, :, :8], nd) < 5e-5


def test_toeplitz_matches_reference():
    g = load("toeplitz.npz")
    nf = O.KBNufftOracle((20, 20), 1.25, 6)
    assert rel(nf.calc_toeplitz_kernels(g["trj"], g["wts"]), g["kern"]) < 5e-6
    assert rel(nf.normal_toeplitz(g["x"], g["kern"]), g["normal"]) < 5e-6


def test_ndft_matches_reference():
    g = load("ndft.npz")
    assert rel(O.ndft_forward(g["x"], g["trj"], (12, 10)), g["fwd"]) < 2e-6
    assert rel(O.ndft_adjoint(g["kin"], g["trj"], (12, 10)), g["adj"]) < 2e-6


def test_sense_and_cg_match_reference():
    g = load("sense.npz")
    nf = O.KBNufftOracle((32, 32), 1.25, 6)
    A = O.SenseOracle(g["trj"], g["mps"], nf)
    assert rel(A.adjoint(g["ksp"]), g["adj"]) < 1e-5
    assert rel(A.normal(g["truth"]), g["normal"]) < 1e-5
    rec = O.cg_sense(A, g["ksp"], int(g["iters"]), float(g["lamda"]), float(g["max_eigen"]))
    # the reference runs CG in float32 (algs.py:841-867); the oracle uses float64
    # dot products, so the gap is the reference's own rounding, ~1e-4 after 5 iterations
    assert rel(rec, g["cg"]) < 3e-4


def test_image_gradient_matches_reference_autograd():
    g = load("nufft.npz")
    nf = O.KBNufftOracle((24, 24), 1.25, 6)
    r = nf.forward(g["ag_img"], g["ag_trj"]) - g["ag_y"]
    grad = 2 * nf.adjoint(r.astype(np.complex64), g["ag_trj"])
    assert rel(grad, g["ag_grad"]) < 1e-5


# ----------------------------------------------------------------- type-3
@pytest.mark.parametrize("tag", ["b1", "b2"])
def test_type3_naive_matches_reference(tag):
    """The float64 naive type-3 sum against the reference's own
    type3_nufft_naive (float32 there, so 1e-5)."""
    g = load("type3.npz")
    ph, al = g[f"{tag}_phis"], g[f"{tag}_alphas"]
    assert rel(O.type3_naive(g[f"{tag}_x"], ph, al), g[f"{tag}_fwd"]) < 1e-5
    assert rel(O.type3_naive_adjoint(g[f"{tag}_y"], ph, al), g[f"{tag}_adj"]) < 1e-5


@pytest.mark.parametrize("tag", ["b1", "b2"])
def test_type3_kb_restatement_against_reference_sums(tag):
    """The Kaiser-Bessel type-3 restatement (os 2, W 4) reproduces the
    reference's exact sums to the accuracy of the kernel (a wrong scale,
    shift or phase convention would give O(1) errors); B = 2 has a
    different oversampling, hence beta, per axis."""
    g = load("type3.npz")
    ph, al = g[f"{tag}_phis"], g[f"{tag}_alphas"]
    t3 = O.Type3Oracle(ph, al)
    if tag == "b2":
        assert t3.beta[0] != t3.beta[1]
    assert rel(t3.forward(g[f"{tag}_x"]), g[f"{tag}_fwd"]) < 3e-3
    assert rel(t3.adjoint(g[f"{tag}_y"]), g[f"{tag}_adj"]) < 3e-3
    exact = O.type3_naive_adjoint(g[f"{tag}_fwd"], ph, al)
    assert rel(O.Type3Oracle(ph, al, use_toep=True).normal(g[f"{tag}_x"]), exact) < 3e-3
