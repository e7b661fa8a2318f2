"""GPU parity of the sm_100a NUFFT path against the reference's golden vectors
(tests/golden, produced by the unmodified mr_recon) and against the CPU
oracle on the same seeded inputs.

Tolerances (relative L2): NUFFT forward/adjoint and split stages 1e-5
(float32 arithmetic on both sides; measured ~1e-7..1e-6), gradients 1e-4,
CG-SENSE 1e-4 against the float64-dot oracle CG."""

import os
import zlib

import numpy as np
import pytest
import torch

from oracle import nufft_oracle as O
from mr_recon_b200 import synth
from mr_recon_b200.fourier import b200_nufft, triton_nufft
from mr_recon_b200.interp import grid as mgrid, ungrid as mungrid
from mr_recon_b200.plan import Plan

pytestmark = pytest.mark.gpu
DEV = "cuda"
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-5


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def Nn(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def load(name):
    return np.load(os.path.join(GOLD, name))


# ----------------------------------------------------------------- golden
def test_golden_radial_128_os2_w6():
    g = load("nufft.npz")
    nf = triton_nufft((128, 128), oversamp=2.0, width=6)
    ksp = nf.forward(T(g["r128_img"]), T(g["r128_trj"]))
    assert ksp.shape == g["r128_ksp"].shape
    assert rel(Nn(ksp), g["r128_ksp"]) < TOL
    adj = nf.adjoint(T(g["r128_ksp"]), T(g["r128_trj"]))
    assert rel(Nn(adj), g["r128_adj"]) < TOL


def test_golden_odd_sizes_odd_width_batched():
    g = load("nufft.npz")
    nf = b200_nufft((25, 22), oversamp=1.4, width=5)
    assert rel(Nn(nf.forward(T(g["odd_img"]), T(g["odd_trj"]))), g["odd_ksp"]) < TOL
    assert rel(Nn(nf.adjoint(T(g["odd_kin"]), T(g["odd_trj"]))), g["odd_adj"]) < TOL
    assert rel(Nn(nf.forward_FT_only(T(g["odd_img"]))), g["odd_ft"]) < TOL


def test_golden_3d_os125_w4():
    g = load("nufft.npz")
    nf = b200_nufft((16, 16, 16), oversamp=1.25, width=4)
    assert rel(Nn(nf.forward(T(g["d3_img"]), T(g["d3_trj"]))), g["d3_ksp"]) < TOL
    assert rel(Nn(nf.adjoint(T(g["d3_ksp"]), T(g["d3_trj"]))), g["d3_adj"]) < TOL


def _interp_cases():
    g = load("interp.npz")
    keys = sorted(set(k.split("__")[0] for k in g.files))
    return [(k, {f: g[k + "__" + f] for f in ["locs", "vals", "ungrid", "svals", "grid", "width", "beta", "gshape"]})
            for k in keys]


@pytest.mark.parametrize("case", _interp_cases(), ids=lambda c: c[0])
def test_golden_ungrid_grid_with_edge_locations(case):
    _, c = case
    d = len(c["gshape"])
    w = (int(c["width"]),) * d
    kp = {"beta": float(c["beta"])}
    u = mungrid(T(c["vals"]), T(c["locs"]), w, kernel_params=kp)
    gg = mgrid(T(c["svals"]), T(c["locs"]), tuple(int(v) for v in c["gshape"]), w, kernel_params=kp)
    assert rel(Nn(u), c["ungrid"]) < TOL
    assert rel(Nn(gg), c["grid"]) < TOL


def test_golden_image_gradient():
    g = load("nufft.npz")
    nf = b200_nufft((24, 24), oversamp=1.25, width=6)
    x = T(g["ag_img"]).requires_grad_(True)
    loss = (nf.forward(x, T(g["ag_trj"])) - T(g["ag_y"])).abs().square().sum()
    loss.backward()
    assert abs(loss.item() - float(g["ag_loss"])) / float(g["ag_loss"]) < 1e-5
    assert rel(Nn(x.grad), g["ag_grad"]) < 1e-5


def test_golden_toeplitz():
    g = load("toeplitz.npz")
    nf = b200_nufft((20, 20), oversamp=1.25, width=6)
    k = nf.calc_teoplitz_kernels(T(g["trj"]), T(g["wts"]))
    assert rel(Nn(k), g["kern"]) < 1e-5
    assert rel(Nn(nf.normal_toeplitz(T(g["x"]), T(g["kern"]))), g["normal"]) < 1e-5


def test_golden_sense_linop_and_cg():
    from mr_recon_b200.linops import sense_linop
    from mr_recon_b200.recons import CG_SENSE_recon
    g = load("sense.npz")
    nf = triton_nufft((32, 32), oversamp=1.25, width=6)
    A = sense_linop(T(g["trj"]), T(g["mps"]), nufft=nf)
    assert rel(Nn(A.adjoint(T(g["ksp"]))), g["adj"]) < TOL
    assert rel(Nn(A.normal(T(g["truth"]))), g["normal"]) < TOL
    rec = CG_SENSE_recon(A, T(g["ksp"]), max_iter=int(g["iters"]), lamda_l2=float(g["lamda"]),
                         max_eigen=float(g["max_eigen"]), verbose=False)
    # reference CG runs in float32; ours accumulates dots in float64
    assert rel(Nn(rec), g["cg"]) < 3e-4
    on = O.KBNufftOracle((32, 32), 1.25, 6)
    ref64 = O.cg_sense(O.SenseOracle(g["trj"], g["mps"], on), g["ksp"], int(g["iters"]),
                       float(g["lamda"]), float(g["max_eigen"]))
    assert rel(Nn(rec), ref64) < 1e-4


# ----------------------------------------------------------------- oracle parity
CASES = [
    # name, im_size, os, W, C, trajectory kind, M
    ("2d_spiral_os125_w6", (96, 80), 1.25, 6, 5, "spiral", 6000),
    ("2d_random_os2_w4_c1", (64, 64), 2.0, 4, 1, "random", 5000),
    ("2d_radial_os2_w7_c3", (64, 48), 2.0, 7, 3, "radial", 4096),
    ("2d_spiral_os2_w5_c12", (64, 64), 2.0, 5, 12, "spiral", 3000),
    ("2d_radial_os125_w8_c40", (48, 56), 1.25, 8, 40, "radial", 2048),
    ("3d_random_os125_w4", (20, 18, 22), 1.25, 4, 3, "random", 3000),
    ("3d_koosh_os15_w5_c17", (16, 16, 16), 1.5, 5, 17, "koosh", 2048),
    ("1d_random_os2_w6", (100,), 2.0, 6, 2, "random", 300),
    ("2d_w10_os2", (40, 40), 2.0, 10, 2, "random", 800),
]


def _traj(kind, im, M, rng):
    d = len(im)
    if kind == "random":
        return ((rng.rand(1, M, d) - 0.5) * np.array(im)).astype(np.float32)
    if kind == "spiral":
        n = 8
        return synth.vd_spiral(n, M // n, min(im) / 2.0).reshape(1, -1, 2)
    if kind == "radial":
        n = 32
        return synth.golden_angle_radial(n, M // n, min(im) / 2.0).reshape(1, -1, 2)
    if kind == "koosh":
        n = 64
        return synth.kooshball(n, M // n, min(im) / 2.0).reshape(1, -1, 3)
    raise ValueError(kind)


# kernel paths (b200_nufft options; the default is lane-per-coil interpolation
# and register-tile gridding in 2D)
PATHS = {"default": {},
         "warp_smem": dict(reg_grid=False, reg_interp=False),
         "tables": dict(weight_tables=True, reg_grid=False, reg_interp=False),
         "fast_atomicgrid": dict(warp_grid=False, reg_interp=False),
         "general": dict(fast=False)}


@pytest.mark.parametrize("path", list(PATHS))
@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_oracle_parity_forward_adjoint_stages(case, path):
    name, im, os_, W, C, kind, M = case
    rng = np.random.RandomState(zlib.crc32(name.encode()) % (2 ** 31))
    trj = _traj(kind, im, M, rng)
    img = synth.randn_complex((1, C, *im), rng)
    ksp_in = synth.randn_complex((1, C, trj.shape[1]), rng)
    nf = b200_nufft(im, oversamp=os_, width=W, **PATHS[path])
    on = O.KBNufftOracle(im, os_, W)
    t = T(trj)
    assert rel(Nn(nf.forward(T(img), t)), on.forward(img, trj)) < TOL
    assert rel(Nn(nf.adjoint(T(ksp_in), t)), on.adjoint(ksp_in, trj)) < TOL
    ft = nf.forward_FT_only(T(img))
    assert rel(Nn(ft), on.forward_FT_only(img)) < TOL
    assert rel(Nn(nf.forward_interp_only(ft, t)), on.forward_interp_only(on.forward_FT_only(img), trj)) < TOL
    g = nf.adjoint_grid_only(T(ksp_in), t)
    assert rel(Nn(g), on.adjoint_grid_only(ksp_in, trj)) < TOL
    assert rel(Nn(nf.adjoint_iFT_only(g)), on.adjoint_iFT_only(on.adjoint_grid_only(ksp_in, trj))) < TOL


def test_split_heavy_tiles_match_oracle():
    """A dense cluster of samples with a tiny work-item size forces tiles to be
    split over many CTAs (partial tiles summed in item order in gridding)."""
    rng = np.random.RandomState(7)
    im = (48, 48)
    trj = np.concatenate([(rng.rand(1, 4000, 2) - 0.5) * 3.0, (rng.rand(1, 1000, 2) - 0.5) * 48], 1).astype(np.float32)
    img = synth.randn_complex((1, 4, *im), rng)
    y = synth.randn_complex((1, 4, trj.shape[1]), rng)
    nf = b200_nufft(im, oversamp=1.25, width=6, max_chunk=64)
    on = O.KBNufftOracle(im, 1.25, 6)
    assert rel(Nn(nf.forward(T(img), T(trj))), on.forward(img, trj)) < TOL
    assert rel(Nn(nf.adjoint(T(y), T(trj))), on.adjoint(y, trj)) < TOL
    plan = nf._plans.entries[-1][2]
    assert plan.stats()["split_tiles"] > 0


@pytest.mark.parametrize("opts", [dict(itile=12, gtile=6, ichunk=100, gchunk=40),
                                  dict(itile=32, gtile=5, ichunk=4096, gchunk=2000),
                                  dict(itile=9, gtile=20, ichunk=300, gchunk=64)])
def test_plan_decomposition_options_rebind(opts):
    """Changing tile edges and work-item sizes on a live plan re-bins the
    trajectory at the next set_traj; results stay at oracle parity (gtile 20
    leaves the register-tile kernel for the shared-memory one)."""
    from mr_recon_b200 import _lib
    rng = np.random.RandomState(5)
    im, C = (80, 64), 6
    trj = synth.vd_spiral(8, 900, 32.0).reshape(-1, 2)
    img = synth.randn_complex((C, *im), rng)
    y = synth.randn_complex((C, trj.shape[0]), rng)
    on = O.KBNufftOracle(im, 1.25, 6)
    p = Plan([im], [trj.shape[0]], [C], 1.25, (6.0, 6.0), device=DEV)
    tr = T(trj)
    p.set_traj(tr)
    for opt, key in ((_lib.MRN_OPT_INTERP_TILE, "itile"), (_lib.MRN_OPT_GRID_TILE, "gtile"),
                     (_lib.MRN_OPT_INTERP_CHUNK, "ichunk"), (_lib.MRN_OPT_GRID_CHUNK, "gchunk")):
        p.set_option(opt, opts[key])
    assert not p.traj_bound
    p.set_traj(tr)
    ksp = torch.empty(C * trj.shape[0], dtype=torch.complex64, device=DEV)
    out = torch.empty(C * im[0] * im[1], dtype=torch.complex64, device=DEV)
    p.forward(T(img).reshape(-1), ksp)
    p.adjoint(T(y).reshape(-1), out)
    assert rel(Nn(ksp).reshape(1, C, -1), on.forward(img[None], trj[None])) < TOL
    assert rel(Nn(out).reshape(1, C, *im), on.adjoint(y[None], trj[None])) < TOL


@pytest.mark.parametrize("itile", [3, 4, 5, 6, 8])
@pytest.mark.parametrize("C", [1, 5, 12, 16])
def test_3d_interp_regions_across_shared_memory_sizes(itile, C):
    """3D lane-per-coil interpolation over tile edges and coil counts whose staged regions span 10 KB to over 100 KB, around
    the 48 KB a launch gets without the shared-memory opt-in (static
    coordinate staging included)."""
    from mr_recon_b200 import _lib
    rng = np.random.RandomState(itile * 31 + C)
    im = (24, 20, 28)
    M = 1500
    trj = ((rng.rand(M, 3) - 0.5) * np.array(im)).astype(np.float32)
    img = synth.randn_complex((C, *im), rng)
    on = O.KBNufftOracle(im, 1.25, 4)
    p = Plan([im], [M], [C], 1.25, (4.0, 4.0, 4.0), device=DEV)
    p.set_option(_lib.MRN_OPT_INTERP_TILE, itile)
    p.set_traj(T(trj))
    ksp = torch.empty(C * M, dtype=torch.complex64, device=DEV)
    p.forward(T(img).reshape(-1), ksp)
    assert rel(Nn(ksp).reshape(1, C, -1), on.forward(img[None], trj[None])) < TOL


def test_autotune_keeps_parity_and_caches():
    """The autotuner times candidate decompositions on the bound trajectory,
    leaves the plan bound with the fastest, and reuses the choice for the
    same geometry without timing."""
    from mr_recon_b200 import autotune as AT
    AT.clear_cache()
    rng = np.random.RandomState(21)
    im, C = (72, 64), 7
    trj = synth.vd_spiral(6, 800, 32.0).reshape(1, -1, 2)
    img = synth.randn_complex((1, C, *im), rng)
    y = synth.randn_complex((1, C, trj.shape[1]), rng)
    on = O.KBNufftOracle(im, 1.25, 6)
    nf = b200_nufft(im, oversamp=1.25, width=6, autotune=True)
    assert rel(Nn(nf.forward(T(img), T(trj))), on.forward(img, trj)) < TOL
    assert rel(Nn(nf.adjoint(T(y), T(trj))), on.adjoint(y, trj)) < TOL
    plan = nf._plans.entries[-1][2]
    cand = AT.default_candidates(2)
    res = AT.autotune(plan, T(trj.reshape(-1, 2)))
    assert res["cached"]
    assert res["interp_tile"] in cand["interp_tile"] and res["grid_chunk"] in cand["grid_chunk"]
    ksp = torch.empty(C * trj.shape[1], dtype=torch.complex64, device=DEV)
    plan.forward(T(img).reshape(-1), ksp)
    assert rel(Nn(ksp).reshape(1, C, -1), on.forward(img, trj)) < TOL


@pytest.mark.parametrize("tile", [(8, 8), (16, 32), (64, 64), (5, 7)])
def test_tile_shapes_agree(tile):
    rng = np.random.RandomState(11)
    im = (64, 72)
    trj = synth.vd_spiral(6, 700, 32.0).reshape(1, -1, 2)
    img = synth.randn_complex((1, 9, *im), rng)
    y = synth.randn_complex((1, 9, trj.shape[1]), rng)
    on = O.KBNufftOracle(im, 1.25, 6)
    nf = b200_nufft(im, oversamp=1.25, width=6, tile=tile, coil_group=4)
    assert rel(Nn(nf.forward(T(img), T(trj))), on.forward(img, trj)) < TOL
    assert rel(Nn(nf.adjoint(T(y), T(trj))), on.adjoint(y, trj)) < TOL


def test_edge_cases():
    rng = np.random.RandomState(3)
    im = (32, 32)
    nf = b200_nufft(im, oversamp=1.25, width=6)
    on = O.KBNufftOracle(im, 1.25, 6)
    # exact grid points, exact kernel edges, k = -N/2, far out of range (wraps)
    pts = np.array([[0, 0], [-16, -16], [15.999, 15.999], [1.0, -2.0], [3.2, 0.0],
                    [40.0, -50.25], [-0.0, 7.5], [0.4, 0.4]], dtype=np.float32)[None]
    img = synth.randn_complex((1, 2, *im), rng)
    assert rel(Nn(nf.forward(T(img), T(pts))), on.forward(img, pts)) < TOL
    y = synth.randn_complex((1, 2, pts.shape[1]), rng)
    assert rel(Nn(nf.adjoint(T(y), T(pts))), on.adjoint(y, pts)) < TOL
    # a single sample, a single coil
    one = pts[:, :1]
    assert rel(Nn(nf.forward(T(img[:, :1]), T(one))), on.forward(img[:, :1], one)) < TOL
    # empty trajectory: adjoint is zero, forward is empty
    empty = np.zeros((1, 0, 2), np.float32)
    assert nf.forward(T(img), T(empty)).shape == (1, 2, 0)
    assert float(nf.adjoint(T(np.zeros((1, 2, 0), np.complex64)), T(empty)).abs().max()) == 0.0
    # grid smaller than the kernel (raw interpolation wraps several times)
    vals = synth.randn_complex((3, 4, 5), rng)
    locs = (rng.rand(50, 2) * 10 - 3).astype(np.float32)
    u = mungrid(T(vals), T(locs), (6, 6), kernel_params={"beta": 9.0})
    assert rel(Nn(u), O.ungrid(vals, locs, (6, 6), 9.0)) < TOL
    gg = mgrid(T(synth.randn_complex((3, 50), rng)), T(locs), (4, 5), (6, 6), kernel_params={"beta": 9.0})
    assert gg.shape == (3, 4, 5)


def test_errors_match_reference_behaviour():
    nf = b200_nufft((16, 16))
    with pytest.raises(RuntimeError):
        nf.forward(torch.zeros(1, 1, 16, 16, dtype=torch.complex64), torch.zeros(1, 4, 2))
    with pytest.raises(ValueError):
        mungrid(torch.zeros(1, 8, 8, dtype=torch.complex64, device=DEV), torch.zeros(3, 2, device=DEV), (20, 20))
    with pytest.raises(NotImplementedError):
        mungrid(torch.zeros(1, 8, 8, dtype=torch.complex64, device=DEV), torch.zeros(3, 2, device=DEV), (4, 4),
                kernel="spline")


# ----------------------------------------------------------------- properties at full size
def test_adjoint_consistency_and_linearity_config2_size():
    """<A x, y> = <x, A^H y> and A(a x1 + x2) = a A x1 + A x2 on the 256^2,
    32-coil, 48 x 2048 spiral geometry."""
    rng = np.random.RandomState(5)
    im = (256, 256)
    trj = T(synth.vd_spiral(48, 2048, 128.0)[None])
    x1 = torch.randn(1, 32, *im, dtype=torch.complex64, device=DEV)
    x2 = torch.randn(1, 32, *im, dtype=torch.complex64, device=DEV)
    y = torch.randn(1, 32, 48, 2048, dtype=torch.complex64, device=DEV)
    nf = b200_nufft(im)
    Ax = nf.forward(x1, trj)
    AHy = nf.adjoint(y, trj)
    lhs = torch.vdot(Ax.reshape(-1).to(torch.complex128), y.reshape(-1).to(torch.complex128))
    rhs = torch.vdot(x1.reshape(-1).to(torch.complex128), AHy.reshape(-1).to(torch.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    a = 0.7 - 0.2j
    lin = nf.forward(a * x1 + x2, trj)
    ref = a * Ax + nf.forward(x2, trj)
    assert float((lin - ref).abs().norm() / ref.abs().norm()) < 1e-5
    del rng


# ----------------------------------------------------------------- trajectory gradients
@pytest.mark.parametrize("d", [2, 3])
def test_trajectory_gradient_forward_vs_fp64_finite_differences(d):
    rng = np.random.RandomState(20 + d)
    im = (24, 20) if d == 2 else (12, 10, 14)
    W = 6 if d == 2 else 4
    os_ = 1.25
    M = 400
    trj = ((rng.rand(1, M, d) - 0.5) * np.array(im)).astype(np.float32)
    img = synth.randn_complex((1, 3, *im), rng)
    y = synth.randn_complex((1, 3, M), rng)
    nf = b200_nufft(im, oversamp=os_, width=W)
    t = T(trj).requires_grad_(True)
    loss = torch.sum(torch.view_as_real(nf.forward(T(img), t)) * torch.view_as_real(T(y)))
    loss.backward()
    g = Nn(t.grad)
    h = 1e-5
    idx = rng.choice(M, 12, replace=False)
    fds, ans = [], []
    for p in idx:
        for ax in range(d):
            tp = trj.astype(np.float64).copy()
            tm = tp.copy()
            tp[0, p, ax] += h
            tm[0, p, ax] -= h
            fp = np.sum(np.real(np.conj(y) * O.nufft_forward_f64(img, tp, im, os_, W, nf.beta)))
            fm = np.sum(np.real(np.conj(y) * O.nufft_forward_f64(img, tm, im, os_, W, nf.beta)))
            fds.append((fp - fm) / (2 * h))
            ans.append(g[0, p, ax])
    assert rel(ans, fds) < 1e-4


def test_trajectory_gradient_adjoint_and_interp_vs_fp64_fd():
    """Trajectory gradient through the adjoint NUFFT: d/dk Re<z, A^H(y; k)>
    equals d/dk Re<A(z; k), y>, checked by float64 central differences."""
    rng = np.random.RandomState(31)
    im = (20, 20)
    M = 300
    trj = ((rng.rand(1, M, 2) - 0.5) * 20).astype(np.float32)
    z = synth.randn_complex((1, 2, *im), rng)
    y = synth.randn_complex((1, 2, M), rng)
    nf = b200_nufft(im, oversamp=1.25, width=6)
    t = T(trj).requires_grad_(True)
    loss = torch.sum(torch.view_as_real(nf.adjoint(T(y), t)) * torch.view_as_real(T(z)))
    loss.backward()
    g = Nn(t.grad)
    h = 1e-5
    fds, ans = [], []
    for p in rng.choice(M, 10, replace=False):
        for ax in range(2):
            tp = trj.astype(np.float64).copy()
            tm = tp.copy()
            tp[0, p, ax] += h
            tm[0, p, ax] -= h
            fp = np.sum(np.real(np.conj(O.nufft_forward_f64(z, tp, im, 1.25, 6, nf.beta)) * y))
            fm = np.sum(np.real(np.conj(O.nufft_forward_f64(z, tm, im, 1.25, 6, nf.beta)) * y))
            fds.append((fp - fm) / (2 * h))
            ans.append(g[0, p, ax])
    assert rel(ans, fds) < 1e-4


# ----------------------------------------------------------------- uneven batches
def test_uneven_multislice_plan_matches_per_slice_oracle():
    rng = np.random.RandomState(9)
    sizes = [(40, 40), (48, 32), (40, 40), (56, 56)]
    coils = [3, 1, 5, 2]
    npts = [900, 400, 1300, 700]
    plan = Plan(sizes, npts, coils, 1.25, (6.0, 6.0), device=DEV)
    assert plan.fft_kind == 2  # 50 and 60 x 40 natively, 70 (= 2 x 5 x 7) on cuFFT
    trjs = [((rng.rand(m, 2) - 0.5) * np.array(s)).astype(np.float32) for s, m in zip(sizes, npts)]
    imgs = [synth.randn_complex((c, *s), rng) for s, c in zip(sizes, coils)]
    plan.set_traj(T(np.concatenate([t.reshape(-1) for t in trjs])))
    img_flat = T(np.concatenate([i.reshape(-1) for i in imgs]))
    ksp = torch.empty(plan.n_ksp, dtype=torch.complex64, device=DEV)
    plan.forward(img_flat, ksp)
    back = torch.empty(plan.n_img, dtype=torch.complex64, device=DEV)
    plan.adjoint(ksp, back)
    k = Nn(ksp)
    b = Nn(back)
    for s in range(4):
        on = O.KBNufftOracle(sizes[s], 1.25, 6)
        kr = on.forward(imgs[s][None], trjs[s][None])[0]
        ko = k[plan.ksp_off[s]:plan.ksp_off[s] + coils[s] * npts[s]].reshape(kr.shape)
        assert rel(ko, kr) < TOL
        br = on.adjoint(ko[None], trjs[s][None])[0]
        bo = b[plan.img_off[s]:plan.img_off[s] + br.size].reshape(br.shape)
        assert rel(bo, br) < TOL


def test_uneven_batched_cg_equals_per_slice_solves_bitwise():
    """CG-SENSE of an uneven batch (sizes, coil and sample counts differ, a
    dense spiral centre so gridding tiles split) in one plan against one plan
    and solve per slice with the batch's tiles, work-item sizes and gridding
    lane group: the same bits. The CG sums depend on each slice's own length
    and cuFFT does not depend on the batch count, so nothing else differs."""
    from mr_recon_b200 import _lib
    from mr_recon_b200.algs import SenseCG
    rng = np.random.RandomState(31)
    sizes = [(48, 48), (64, 64), (40, 40), (56, 56), (64, 64)]
    coils = [3, 12, 1, 7, 20]
    npts = [1600, 4800, 800, 3200, 4000]
    trjs = [synth.vd_spiral(8, m // 8, s[0] / 2.0).reshape(-1, 2) for s, m in zip(sizes, npts)]
    xs = [synth.ellipse_phantom(s, 6, rng).astype(np.complex64).reshape(-1) for s in sizes]
    mps = [synth.gaussian_coil_maps(s, c).astype(np.complex64).reshape(-1) for s, c in zip(sizes, coils)]
    opts = {_lib.MRN_OPT_INTERP_TILE: 10, _lib.MRN_OPT_INTERP_CHUNK: 128,
            _lib.MRN_OPT_GRID_TILE: 8, _lib.MRN_OPT_GRID_CHUNK: 96}

    def make(ims, ms, cs, trj):
        p = Plan(ims, ms, cs, 1.25, (6.0, 6.0), device=DEV)
        for k, v in opts.items():
            p.set_option(k, v)
        return p

    plan = make(sizes, npts, coils, np.concatenate(trjs))
    plan.set_traj(T(np.concatenate(trjs).reshape(-1)))
    assert plan.stats()["split_tiles"] > 0
    m_t = T(np.concatenate(mps))
    ksp = torch.empty(plan.n_ksp, dtype=torch.complex64, device=DEV)
    plan.sense_forward(T(np.concatenate(xs)), m_t, ksp)
    ksp += T(synth.randn_complex((plan.n_ksp,), rng)) * 0.01 * float(ksp.abs().max())
    cg = SenseCG(plan, m_t, None, 12, 1e-3, 40.0)
    cg.ksp.copy_(ksp)
    xb = cg.solve().clone()
    img_off = [int(o) for o in plan.img_off]
    ksp_off = [int(o) for o in plan.ksp_off]
    xo = 0
    for s in range(len(sizes)):
        p1 = make([sizes[s]], [npts[s]], [coils[s]], trjs[s])
        p1.set_option(_lib.MRN_OPT_GRID_LANES, 32)  # the batch's lane group (widest slice: 20 coils)
        p1.set_traj(T(trjs[s].reshape(-1)))
        n = coils[s] * sizes[s][0] * sizes[s][1]
        c1 = SenseCG(p1, m_t[img_off[s]:img_off[s] + n], None, 12, 1e-3, 40.0)
        c1.ksp.copy_(ksp[ksp_off[s]:ksp_off[s] + coils[s] * npts[s]])
        x1 = c1.solve()
        nx = sizes[s][0] * sizes[s][1]
        assert torch.equal(x1, xb[xo:xo + nx]), f"slice {s}"
        xo += nx


@pytest.mark.parametrize("coils", [40, 32, 12, 5])
def test_sense_normal_entry_major_equals_forward_then_adjoint(coils):
    """The 2D SENSE normal operator keeps its samples in gridding-entry order
    (the density weight applied by the interpolation): it must give exactly
    the bits of the sample-order forward followed by the adjoint, with split
    tiles and a density compensation, for full and partial coil groups."""
    from mr_recon_b200.linops import sense_linop
    rng = np.random.RandomState(40 + coils)
    im = (64, 56)
    trj = synth.vd_spiral(12, 900, 28.0)
    mps = synth.gaussian_coil_maps(im, coils).astype(np.complex64)
    dcf = (0.1 + np.linalg.norm(trj, axis=-1) / 28.0).astype(np.float32)
    A = sense_linop(T(trj), T(mps), dcf=T(dcf), nufft=b200_nufft(im, max_chunk=64))
    assert A.plan.stats()["split_tiles"] > 0
    x = T(synth.randn_complex(im, rng))
    n = A.normal(x)
    assert torch.equal(n, A.adjoint(A.forward(x)))
    # the same plan without the entry map runs the sample-order normal: same bits
    from mr_recon_b200 import _lib
    A.plan.set_option(_lib.MRN_OPT_ENTRY_MAJOR, 0)
    A.plan.set_traj(A.trj.contiguous())
    assert torch.equal(A.normal(x), n)
    on = O.KBNufftOracle(im, 1.25, 6)
    Ao = O.SenseOracle(trj, mps, on, dcf=dcf)
    assert rel(Nn(n), Ao.normal(Nn(x))) < TOL


def test_subspace_linop_toeplitz_normal_matches_oracle():
    """subspace_linop(use_toeplitz=True): the nsub x nsub kernels of the
    weights conj(phi_k1) phi_k2 dcf on the B200 adjoint and the FFT-only
    normal (linops.py:1581-1601, 1703-1772) against the oracle's restatement;
    close to the exact normal A^H A (the Toeplitz model error)."""
    from mr_recon_b200.linops import subspace_linop
    rng = np.random.RandomState(61)
    im, C, K = (24, 20), 3, 2
    trj = synth.vd_spiral(4, 240, 10.0).transpose(1, 0, 2).copy()  # (nro 240, ntr 4, 2)
    phi = synth.randn_complex((K, 4), rng)
    mps = synth.gaussian_coil_maps(im, C).astype(np.complex64)
    dcf = (0.5 + rng.rand(240, 4)).astype(np.float32)
    A = subspace_linop(im, T(trj), T(mps), T(phi), dcf=T(dcf), nufft=b200_nufft(im), use_toeplitz=True)
    a = synth.randn_complex((K, *im), rng)
    ref = O.subspace_toeplitz_normal(trj, mps, phi, a, O.KBNufftOracle(im, 1.25, 6), dcf=dcf)
    out = Nn(A.normal(T(a)))
    assert rel(out, ref) < 1e-4
    Ao = O.SubspaceOracle(trj, mps, phi, O.KBNufftOracle(im, 1.25, 6), dcf=dcf)
    assert rel(out, Ao.adjoint(Ao.forward(a))) < 5e-2


def test_sense_cg_graph_matches_oracle():
    from mr_recon_b200.linops import sense_linop
    from mr_recon_b200.recons import CG_SENSE_recon
    rng = np.random.RandomState(12)
    im = (48, 48)
    C = 6
    mps = synth.gaussian_coil_maps(im, C)
    trj = synth.vd_spiral(6, 500, 24.0)
    truth = synth.ellipse_phantom(im, 8, rng)
    on = O.KBNufftOracle(im, 1.25, 6)
    Ao = O.SenseOracle(trj, mps, on)
    ksp = synth.add_noise(Ao.forward(truth), 30.0, rng)
    # max eigenvalue of A^H A by the power method, x1.01 (recons.py:117-123)
    v = synth.randn_complex(im, rng)
    for _ in range(30):
        z = Ao.normal(v)
        lmax = float(np.linalg.norm(z))
        v = (z / lmax).astype(np.complex64)
    me = 1.01 * lmax
    ref = O.cg_sense(Ao, ksp, 8, 1e-3, me)
    A = sense_linop(T(trj), T(mps), nufft=b200_nufft(im))
    x_eager = CG_SENSE_recon(A, T(ksp), max_iter=8, lamda_l2=1e-3, max_eigen=me, verbose=False)
    x_graph = CG_SENSE_recon(A, T(ksp), max_iter=8, lamda_l2=1e-3, max_eigen=me, verbose=False, graph=True)
    assert rel(Nn(x_eager), ref) < 1e-4
    assert rel(Nn(x_graph), ref) < 1e-4


# ----------------------------------------------------------------- time segmentation
def test_time_segmented_sense_linop_matches_oracle():
    """sense_linop with B0 spatial / temporal basis functions from
    alpha_segementation (all coils x segments in one batched NUFFT) against
    the oracle's segmented SENSE model (linops.py:1134-1228)."""
    from mr_recon_b200.field import alpha_segementation, b0_to_phis_alphas
    from mr_recon_b200.linops import sense_linop
    rng = np.random.RandomState(17)
    im, C, L = (40, 36), 4, 6
    trj = synth.vd_spiral(3, 400, 18.0)  # (3, 400, 2)
    yy, xx = np.meshgrid(np.linspace(-1, 1, im[0]), np.linspace(-1, 1, im[1]), indexing="ij")
    b0 = (80 * xx - 50 * yy ** 2 + 100 * np.exp(-((xx - 0.2) ** 2 + yy ** 2) / 0.05)).astype(np.float32)
    phis, alphas = b0_to_phis_alphas(T(b0), (3, 400), 1, 10e-3 / 400)
    for kind in ("zero", "lstsq"):
        s, t = alpha_segementation(phis, alphas, L, interp_type=kind, verbose=False)
        mps = synth.gaussian_coil_maps(im, C).astype(np.complex64)
        A = sense_linop(T(trj), T(mps), nufft=b200_nufft(im), spatial_funcs=s, temporal_funcs=t)
        on = O.KBNufftOracle(im, 1.25, 6)
        Ao = O.SenseOracle(trj, mps, on, spatial_funcs=Nn(s), temporal_funcs=Nn(t))
        x = synth.randn_complex(im, rng)
        y = synth.randn_complex((C, 3, 400), rng)
        assert (A.seg is not None) == (kind == "zero")  # one-hot segments use the multi-slice plan
        assert rel(Nn(A.forward(T(x))), Ao.forward(x)) < TOL
        assert rel(Nn(A.adjoint(T(y))), Ao.adjoint(y)) < TOL
        assert rel(Nn(A.normal(T(x))), Ao.adjoint(Ao.forward(x))) < TOL


# ----------------------------------------------------------------- density compensation
def test_density_compensation_pipe_menon_properties():
    """Pipe-Menon DCF on the B200 kernels (the reference calls sigpy, absent
    here, so parity is pinned by the defining property): after the
    iterations G^H G w is flat over the samples, and for a radial trajectory
    the weights grow with |k| (the ramp), with a denser centre getting less
    weight."""
    from mr_recon_b200.algs import density_compensation
    from mr_recon_b200.interp import grid as mgrid, ungrid as mungrid
    im = (64, 64)
    trj = synth.golden_angle_radial(96, 128, 32.0)  # (96, 128, 2)
    t = T(trj)
    dcf = density_compensation(t, im, num_iters=30)
    assert dcf.shape == trj.shape[:-1] and float(dcf.max()) == pytest.approx(1.0)
    locs = (t + 32.0).reshape(-1, 2)
    w = dcf.reshape(-1).to(torch.complex64)
    kp = {"beta": 8.0}
    ghgw = mungrid(mgrid(w, locs, im, (4, 4), kernel_params=kp), locs, (4, 4), kernel_params=kp).abs()
    flat = ghgw / ghgw.mean()
    assert float((flat - 1).abs().quantile(0.9)) < 0.05
    r = torch.linalg.vector_norm(t, dim=-1).reshape(-1)
    d = dcf.reshape(-1)
    inner = d[(r > 2) & (r < 8)].mean()
    mid = d[(r > 14) & (r < 20)].mean()
    outer = d[(r > 24) & (r < 30)].mean()
    assert float(inner) < float(mid) < float(outer)


@pytest.mark.parametrize("case", ["radial2d", "spiral2d", "random3d"])
def test_density_compensation_matches_pipe_menon_oracle(case):
    """density_compensation (algs.py:20-106) against the oracle's restatement
    of sigpy.mri.pipe_menon_dcf (the routine the reference calls): the same
    30 iterations of w <- w / |G^H G w| on the same gridding operator."""
    from mr_recon_b200.algs import density_compensation
    rng = np.random.RandomState(11)
    if case == "radial2d":
        im, trj = (48, 48), synth.golden_angle_radial(40, 96, 24.0)
    elif case == "spiral2d":
        im, trj = (40, 44), synth.vd_spiral(5, 400, 20.0)
    else:
        im = (14, 16, 12)
        trj = ((rng.rand(3000, 3) - 0.5) * np.array(im)).astype(np.float32)
    dcf = density_compensation(T(trj), im, num_iters=30)
    ref = O.pipe_menon_dcf(trj, im, max_iter=30)
    assert rel(Nn(dcf), ref) < 1e-4


# ----------------------------------------------------------------- type-3 NUFFT
def test_raw_grid_per_axis_beta_matches_oracle():
    """Gridding / interpolation with one KB beta per axis (sigpy's per-axis
    kernel parameter, which type3_nufft passes) against the oracle."""
    rng = np.random.RandomState(41)
    gs, betas = (31, 24), (8.9, 7.3)
    locs = (rng.rand(1500, 2) * np.array(gs)).astype(np.float32)
    vals = synth.randn_complex((3, 1500), rng)
    gvals = synth.randn_complex((3, *gs), rng)
    kp = {"beta": betas}
    g = mgrid(T(vals), T(locs), gs, (4.0, 4.0), kernel_params=kp)
    u = mungrid(T(gvals), T(locs), (4.0, 4.0), kernel_params=kp)
    b = np.array(betas, np.float32)
    assert rel(Nn(g), O.grid(vals, locs, gs, (4.0, 4.0), b)) < TOL
    assert rel(Nn(u), O.ungrid(gvals, locs, (4.0, 4.0), b)) < TOL


@pytest.mark.parametrize("tag", ["b1", "b2"])
def test_type3_nufft_matches_oracle(tag):
    """type3_nufft on the B200 kernels against the oracle's restatement of
    the reference's KB type-3 (same algorithm: 1e-4, the midpoint phases
    being formed in float32 here and float64 there) and against the
    reference's exact sums (the kernel's accuracy, 3e-3)."""
    from mr_recon_b200.linops import type3_nufft
    g = load("type3.npz")
    ph, al = g[f"{tag}_phis"], g[f"{tag}_alphas"]
    x, y = g[f"{tag}_x"], g[f"{tag}_y"]
    op = type3_nufft(T(ph), T(al))
    on = O.Type3Oracle(ph, al)
    assert op.grd_N_os == on.n_os
    f = Nn(op.forward(T(x)))
    a = Nn(op.adjoint(T(y)))
    assert rel(f, on.forward(x)) < 1e-4
    assert rel(a, on.adjoint(y)) < 1e-4
    assert rel(f, g[f"{tag}_fwd"]) < 3e-3
    assert rel(a, g[f"{tag}_adj"]) < 3e-3
    assert rel(Nn(op.normal(T(x))), on.adjoint(on.forward(x))) < 1e-4
    opt = type3_nufft(T(ph), T(al), use_toep=True)
    ont = O.Type3Oracle(ph, al, use_toep=True)
    assert rel(Nn(opt.kerns), ont.kerns) < 1e-4
    assert rel(Nn(opt.normal(T(x))), ont.normal(x)) < 1e-4


def test_alpha_segmentation_lstsq_type3_vs_exact():
    """alpha_segementation's least-squares temporal functions through the
    type-3 NUFFT (the reference's default): with a well-conditioned Gram
    matrix (L = 4) they agree with the exact voxel sums; at larger L the
    phase model stays within the type-3 accuracy (the reference's own
    behaviour, its complex64 pinv cutting the null space)."""
    from mr_recon_b200.field import alpha_segementation, b0_to_phis_alphas
    im = (36, 32)
    yy, xx = np.meshgrid(np.linspace(-1, 1, im[0]), np.linspace(-1, 1, im[1]), indexing="ij")
    b0 = (70 * xx + 40 * yy ** 2 + 90 * np.exp(-((xx + 0.2) ** 2 + yy ** 2) / 0.08)).astype(np.float32)
    phis, alphas = b0_to_phis_alphas(T(b0), (2, 300), 1, 12e-3 / 300)
    exact = np.exp(-2j * np.pi * Nn(phis)[0][..., None, None].astype(np.float64) * Nn(alphas)[0][None, None])
    for L in (4, 8, 12):
        s3, t3 = alpha_segementation(phis, alphas, L, interp_type="lstsq", use_type3=True, verbose=False)
        se, te = alpha_segementation(phis, alphas, L, interp_type="lstsq", use_type3=False, verbose=False)
        if L == 4:
            assert rel(Nn(t3), Nn(te)) < 1e-3
        m3 = rel(np.einsum("lxy,lat->xyat", Nn(s3), Nn(t3)), exact)
        me = rel(np.einsum("lxy,lat->xyat", Nn(se), Nn(te)), exact)
        assert m3 < me * 1.05 + 2e-3


def test_two_basis_segmentation_lstsq_type3_vs_exact():
    """Two phase bases (field.py:321-369): the least-squares temporal
    functions through the 2-D type-3 NUFFT agree with the exact voxel sums
    for a well-conditioned segmentation, and the phase model error of both
    is within the type-3 accuracy of each other."""
    from mr_recon_b200.field import alpha_segementation
    im = (28, 24)
    yy, xx = np.meshgrid(np.linspace(-1, 1, im[0]), np.linspace(-1, 1, im[1]), indexing="ij")
    phis = T(np.stack([0.45 * xx + 0.05 * yy ** 2, 0.5 * yy]).astype(np.float32))
    tt = np.linspace(0, 1, 240)
    alphas = T(np.stack([25 * tt, 10 * np.sin(2.5 * tt)]).astype(np.float32))
    exact = np.exp(-2j * np.pi * np.einsum("bxy,bt->xyt", Nn(phis).astype(np.float64), Nn(alphas).astype(np.float64)))
    for L in (4, 8):
        s3, t3 = alpha_segementation(phis, alphas, L, interp_type="lstsq", use_type3=True, verbose=False)
        se, te = alpha_segementation(phis, alphas, L, interp_type="lstsq", use_type3=False, verbose=False)
        if L == 4:
            assert rel(Nn(t3), Nn(te)) < 1e-3
        m3 = rel(np.einsum("lxy,lt->xyt", Nn(s3), Nn(t3)), exact)
        me = rel(np.einsum("lxy,lt->xyt", Nn(se), Nn(te)), exact)
        assert m3 < me * 1.05 + 2e-3


# ----------------------------------------------------------------- low-rank operators
def test_lstsq_segments_use_lowrank_plan_and_match_oracle():
    """Least-squares segments (alpha_segementation interp_type='lstsq') on the
    low-rank plan (mrn_lr_*: all segments in one pass, the h_l weights in the
    fused combine and in the gridding prologue) against the oracle's
    segmented SENSE model, with a density compensation; forward, adjoint,
    normal, and two calls in a row give the same bits."""
    from mr_recon_b200.field import alpha_segementation, b0_to_phis_alphas
    from mr_recon_b200.linops import sense_linop
    rng = np.random.RandomState(23)
    im, C, L = (48, 40), 5, 5
    trj = synth.vd_spiral(4, 500, 20.0)  # (4, 500, 2)
    yy, xx = np.meshgrid(np.linspace(-1, 1, im[0]), np.linspace(-1, 1, im[1]), indexing="ij")
    b0 = (60 * xx + 40 * yy ** 2 + 90 * np.exp(-((xx + 0.3) ** 2 + yy ** 2) / 0.04)).astype(np.float32)
    phis, alphas = b0_to_phis_alphas(T(b0), (4, 500), 1, 12e-3 / 500)
    s, t = alpha_segementation(phis, alphas, L, interp_type="lstsq", use_type3=False, verbose=False)
    mps = synth.gaussian_coil_maps(im, C).astype(np.complex64)
    dcf = (0.2 + np.linalg.norm(trj, axis=-1) / 20.0).astype(np.float32)
    A = sense_linop(T(trj), T(mps), dcf=T(dcf), nufft=b200_nufft(im), spatial_funcs=s, temporal_funcs=t)
    assert A.seg is None and A.lr is not None
    Ao = O.SenseOracle(trj, mps, O.KBNufftOracle(im, 1.25, 6), dcf=dcf, spatial_funcs=Nn(s),
                       temporal_funcs=Nn(t))
    x = synth.randn_complex(im, rng)
    y = synth.randn_complex((C, 4, 500), rng)
    assert rel(Nn(A.forward(T(x))), Ao.forward(x)) < TOL
    a1 = A.adjoint(T(y))
    assert rel(Nn(a1), Ao.adjoint(y)) < TOL
    assert torch.equal(a1, A.adjoint(T(y)))
    assert rel(Nn(A.normal(T(x))), Ao.adjoint(Ao.forward(x))) < TOL


@pytest.mark.parametrize("nd", [2, 3])
def test_subspace_linop_matches_oracle(nd):
    """subspace_linop (linops.py:1496-1772) on the low-rank plan against the
    oracle's restatement, with subspace basis phi (K, ntr) along the last
    trajectory dimension and two segments (spatial / temporal functions);
    the autograd (loop) path must agree too."""
    from mr_recon_b200.linops import subspace_linop, subspace_linop_new
    rng = np.random.RandomState(5 + nd)
    if nd == 2:
        im, C, K, L = (40, 36), 3, 3, 2
        trj = synth.vd_spiral(6, 300, 18.0).transpose(1, 0, 2).copy()  # (nro 300, ntr 6, 2)
    else:
        im, C, K, L = (16, 18, 14), 2, 2, 2
        trj = ((rng.rand(200, 5, 3) - 0.5) * np.array(im)).astype(np.float32)  # (nro, ntr, 3)
    tsz = trj.shape[:-1]
    phi = synth.randn_complex((K, tsz[-1]), rng)
    mps = synth.gaussian_coil_maps(im, C).astype(np.complex64)
    sp = np.exp(1j * rng.rand(L, *im)).astype(np.complex64)
    tf = np.exp(1j * rng.rand(L, *tsz)).astype(np.complex64)
    dcf = (0.5 + rng.rand(*tsz)).astype(np.float32)
    A = subspace_linop(im, T(trj), T(mps), T(phi), dcf=T(dcf), nufft=b200_nufft(im, width=4 if nd == 3 else 6),
                       spatial_funcs=T(sp), temporal_funcs=T(tf))
    assert A.lr is not None
    Ao = O.SubspaceOracle(trj, mps, phi, O.KBNufftOracle(im, 1.25, 4 if nd == 3 else 6), dcf=dcf,
                          spatial_funcs=sp, temporal_funcs=tf)
    a = synth.randn_complex((K, *im), rng)
    y = synth.randn_complex((C, *tsz), rng)
    assert rel(Nn(A.forward(T(a))), Ao.forward(a)) < TOL
    assert rel(Nn(A.adjoint(T(y))), Ao.adjoint(y)) < TOL
    assert rel(Nn(A.normal(T(a))), Ao.adjoint(Ao.forward(a))) < TOL
    # the differentiable (loop) path computes the same operator
    at = T(a).requires_grad_(True)
    assert rel(Nn(A.forward(at).detach()), Ao.forward(a)) < TOL
    if nd == 2:
        B = subspace_linop_new(T(trj), T(mps), T(phi), dcf=T(dcf), nufft=b200_nufft(im),
                               spatial_funcs=T(sp), temporal_funcs=T(tf))
        assert rel(Nn(B.adjoint(T(y))), Ao.adjoint(y)) < TOL


@pytest.mark.parametrize("im,os_,native", [((80, 64), 1.25, True), ((25, 27), 2.0, True),
                                           ((45, 38), 2.0, False), ((24, 20, 16), 1.25, True),
                                           ((15, 12, 9), 2.0, True), ((24, 20, 18), 1.25, False)])
def test_native_fft_matches_cufft_and_oracle(im, os_, native):
    """The FFT stage as the library's own per-axis passes (pad / crop fused,
    zero-padded lines skipped) against the cuFFT path of the same plan and the
    oracle: plain forward / adjoint, forward_FT_only / adjoint_iFT_only and the
    SENSE forward / adjoint / normal. Grids with a prime factor above 5 (76,
    23) keep cuFFT, which the plan reports through its results only, so those
    cases check that the option is harmless."""
    from mr_recon_b200 import _lib
    rng = np.random.RandomState(len(im) * 100 + im[0])
    C, d = 5, len(im)
    W = 6 if d == 2 else 4
    if d == 2:
        trj = synth.vd_spiral(6, 700, im[0] / 2.0 - 1).reshape(-1, 2)
    else:
        trj = synth.kooshball(60, 2 * im[0], im[0] / 2.0).reshape(-1, 3)
    M = trj.shape[0]
    img = synth.randn_complex((C, *im), rng)
    y = synth.randn_complex((C, M), rng)
    mps = synth.randn_complex((C, *im), rng)
    x1 = synth.randn_complex(im, rng)
    dcf = (0.5 + rng.rand(M)).astype(np.float32)
    nimg = int(np.prod(im))

    def run(opt):
        p = Plan([im], [M], [C], os_, (float(W),) * d, device=DEV)
        p.set_option(_lib.MRN_OPT_NATIVE_FFT, opt)
        p.set_traj(T(trj))
        assert p.fft_kind == (1 if (opt and native) else 0)
        ksp = torch.empty(C * M, dtype=torch.complex64, device=DEV)
        out = torch.empty(C * nimg, dtype=torch.complex64, device=DEV)
        p.forward(T(img).reshape(-1), ksp)
        p.adjoint(T(y).reshape(-1), out)
        gos = int(np.prod([int(np.ceil(os_ * n)) for n in im]))
        g = torch.empty(C * gos, dtype=torch.complex64, device=DEV)
        back = torch.empty(C * nimg, dtype=torch.complex64, device=DEV)
        p.forward_ft(T(img).reshape(-1), g)
        p.adjoint_ift(g, back)
        sk = torch.empty(C * M, dtype=torch.complex64, device=DEV)
        sx = torch.empty(nimg, dtype=torch.complex64, device=DEV)
        sn = torch.empty(nimg, dtype=torch.complex64, device=DEV)
        p.sense_forward(T(x1).reshape(-1), T(mps).reshape(-1), sk)
        p.sense_adjoint(T(y).reshape(-1), T(dcf), T(mps).reshape(-1), sx)
        p.sense_normal(T(x1).reshape(-1), T(mps).reshape(-1), T(dcf), sn)
        torch.cuda.synchronize()
        return [Nn(t) for t in (ksp, out, g, back, sk, sx, sn)]

    nat, cuf = run(1), run(0)
    for a, b in zip(nat, cuf):
        assert rel(a, b) < 2e-6
    if native:  # the native passes really ran: float32 rounding differs from cuFFT's
        assert any(not np.array_equal(a, b) for a, b in zip(nat, cuf))
    on = O.KBNufftOracle(im, os_, W)
    assert rel(nat[0].reshape(1, C, -1), on.forward(img[None], trj[None])) < TOL
    assert rel(nat[1].reshape(1, C, *im), on.adjoint(y[None], trj[None])) < TOL
    Ao = O.SenseOracle(trj, mps, on, dcf=dcf)
    assert rel(nat[6], Ao.normal(x1).reshape(-1)) < TOL
