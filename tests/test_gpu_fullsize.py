"""GPU parity at the stated sizes of the benchmark configurations, and
run-to-run reproducibility of gridding and of the device CG.

Each configuration runs on the GPU at its full grid (and, where the oracle
allows, its full sample count and coil count); the CPU oracle checks a subset
it can finish in seconds: some coils, or a subset of the samples for the 3D
configuration, whose full 7.68 M-sample adjoint is checked through the adjoint
identity instead. Tolerances (relative L2): NUFFT stages 1e-5 (float32 on both
sides). The config-2 CG-SENSE solve is compared with the oracle's float64 CG
(fixture tests/golden/cg_config2.npz, made by tests/golden/make_cg_config2.py)
at twice the distance of the reference's own float32 arithmetic from it:
20 iterations at lambda 1e-3 stop far from convergence, and float32 rounding
that differs from one operator application to the next (~1e-6 here, mostly
the FFT) grows ~1000-fold over them, for the reference as for this code.
"""

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
import torch

from oracle import nufft_oracle as O
from mr_recon_b200 import synth
from mr_recon_b200.algs import SenseCG
from mr_recon_b200.fourier import b200_nufft
from mr_recon_b200.linops import sense_linop
from mr_recon_b200.plan import Plan

pytestmark = pytest.mark.gpu
DEV = "cuda"
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-5
POOL = ThreadPoolExecutor(os.cpu_count() or 1)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def Nn(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def crandn(shape, seed):
    g = torch.Generator(device=DEV).manual_seed(seed)
    return torch.randn(shape, dtype=torch.complex64, device=DEV, generator=g)


def config2_inputs():
    """256^2, 32 coils, 48 x 2048 VD spiral (the benchmark's NUFFT workload)."""
    im = (256, 256)
    x = synth.ellipse_phantom(im, 20, np.random.RandomState(1234))
    mps = synth.gaussian_coil_maps(im, 32)
    trj = synth.vd_spiral(48, 2048, 128.0)
    return im, x, mps, trj


# ----------------------------------------------------------------- reproducibility
def test_gridding_bitwise_reproducible_config2_split_tiles():
    """Tiles split over several work items used to add their parts with float
    atomics; their partial tiles are now summed in item order, so two adjoints
    of the same data are bit-identical (on another stream too)."""
    im, _, _, trj = config2_inputs()
    t = T(trj[None])
    nf = b200_nufft(im)
    y = crandn((1, 32, 48, 2048), 1)
    a = nf.adjoint(y, t)
    plan = nf._plans.entries[-1][2]
    assert plan.stats()["split_tiles"] > 0
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        nf.forward(crandn((1, 32, *im), 2), t)  # other work in between
        b = nf.adjoint(y, t)
    torch.cuda.current_stream().wait_stream(side)
    c = nf.adjoint(y, t)
    assert torch.equal(a, b) and torch.equal(a, c)


def test_gridding_bitwise_reproducible_3d_split_tiles():
    """3D register-tile gridding of a kooshball whose dense centre is cut into
    many work items (small gridding chunk)."""
    N = 48
    trj = T(synth.kooshball(600, 2 * N, N / 2.0).reshape(1, -1, 3))
    nf = b200_nufft((N, N, N), oversamp=1.25, width=4, max_chunk=128)
    y = crandn((1, 8, trj.shape[1]), 3)
    outs = [nf.adjoint(y, trj) for _ in range(3)]
    plan = nf._plans.entries[-1][2]
    assert plan.stats()["split_tiles"] > 10
    assert all(torch.equal(outs[0], o) for o in outs[1:])
    on = O.KBNufftOracle((N, N, N), 1.25, 4)
    assert rel(Nn(outs[0][:, :2]), on.adjoint(Nn(y[:, :2]), Nn(trj))) < TOL


def test_cg_graph_and_eager_bitwise_config2():
    """The device CG (fixed-order float64 sums, float64 iterates) replayed from
    a CUDA graph gives the same bits as the eager solve."""
    im, x, mps, trj = config2_inputs()
    A = sense_linop(T(trj), T(mps), nufft=b200_nufft(im))
    k = A.forward(T(x))
    solver = SenseCG(A.plan, A.mps, A.dcf, 20, 1e-3, 1551.7)
    solver.ksp.copy_(k.reshape(-1))
    x1 = solver.solve().clone()
    x2 = solver.solve().clone()
    solver.capture()
    x3 = solver.solve().clone()
    assert torch.equal(x1, x2) and torch.equal(x1, x3)


# ----------------------------------------------------------------- configuration 2
def test_config2_full_size_forward_adjoint_vs_oracle():
    """All 32 coils through the GPU at 256^2 on the full 98,304-sample spiral;
    the oracle checks 4 of the coils."""
    im, x, mps, trj = config2_inputs()
    imgs = (mps * x[None]).astype(np.complex64)[None]
    nf = b200_nufft(im)
    t = T(trj[None])
    k = Nn(nf.forward(T(imgs), t))
    y = crandn((1, 32, 48, 2048), 5)
    b = Nn(nf.adjoint(y, t))
    yn = Nn(y)
    on = O.KBNufftOracle(im, 1.25, 6)
    O.FFT_WORKERS = 1
    coils = [0, 11, 22, 31]
    kr = list(POOL.map(lambda c: on.forward(imgs[:, c:c + 1], trj[None])[0, 0], coils))
    br = list(POOL.map(lambda c: on.adjoint(yn[:, c:c + 1], trj[None])[0, 0], coils))
    for c, kc, bc in zip(coils, kr, br):
        assert rel(k[0, c], kc) < TOL
        assert rel(b[0, c], bc) < TOL


def test_config2_cg_sense_vs_oracle_float64_cg():
    """20 CG iterations, lambda 1e-3, on the full configuration against the
    oracle's float64 CG with float64 FFTs (fixture made on the CPU by
    make_cg_config2.py from the same seeded inputs). The fixture also records
    how far the reference's own float32 arithmetic lands from that solution
    (about 2e-3); the device CG (complex64 vectors, float64 dots) must stay
    within twice that."""
    g = np.load(os.path.join(GOLD, "cg_config2.npz"))
    im, x, mps, trj = config2_inputs()
    A = sense_linop(T(trj), T(mps), nufft=b200_nufft(im))
    k = synth.add_noise(Nn(A.forward(T(x))), 30.0, np.random.RandomState(99))
    assert abs(np.linalg.norm(k) / float(g["ksp_norm"]) - 1) < 1e-5
    solver = SenseCG(A.plan, A.mps, A.dcf, int(g["iters"]), float(g["lam"]), float(g["max_eigen"]))
    xg = Nn(solver.solve(T(k)))
    err = rel(xg.reshape(im), g["x_cg64"])
    assert err < 2.0 * float(g["rel_f32_arith"])


# ----------------------------------------------------------------- configuration 3
@pytest.fixture(scope="module")
def config3():
    N = 192
    trj = synth.kooshball(20000, 2 * N, N / 2.0).reshape(1, -1, 3)
    return N, trj


def test_config3_full_size_forward_vs_oracle(config3):
    """192^3, 16 coils, the full 7.68 M-sample kooshball, W 4, os 1.25 through
    the GPU; the oracle checks 2 coils at 50,000 samples spread over the
    whole trajectory (every 154th sample)."""
    N, trj = config3
    nf = b200_nufft((N, N, N), oversamp=1.25, width=4)
    img = crandn((1, 16, N, N, N), 7)
    k = nf.forward(img, T(trj))
    idx = np.arange(0, trj.shape[1], 154)[:50000]
    ks = Nn(k[0, :2, torch.as_tensor(idx, device=DEV)])
    on = O.KBNufftOracle((N, N, N), 1.25, 4)
    O.FFT_WORKERS = os.cpu_count() or 1
    ft = on.forward_FT_only(Nn(img[:, :2]))
    kr = on.forward_interp_only(ft, trj[:, idx])
    assert rel(ks, kr[0]) < TOL


def test_config3_full_grid_adjoint_vs_oracle(config3):
    """Adjoint onto the full 240^3 oversampled grid, 16 coils on the GPU, for
    50,000 of the kooshball's samples; the oracle checks 2 coils."""
    N, trj = config3
    idx = np.arange(0, trj.shape[1], 154)[:50000]
    ts = np.ascontiguousarray(trj[:, idx])
    nf = b200_nufft((N, N, N), oversamp=1.25, width=4)
    y = crandn((1, 16, ts.shape[1]), 8)
    b = Nn(nf.adjoint(y, T(ts))[:, :2])
    on = O.KBNufftOracle((N, N, N), 1.25, 4)
    O.FFT_WORKERS = os.cpu_count() or 1
    assert rel(b, on.adjoint(Nn(y[:, :2]), ts)) < TOL


def test_config3_full_size_adjoint_identity(config3):
    """<A x, y> = <x, A^H y> for the full configuration (16 coils, 7.68 M
    samples): the adjoint at full size, where the oracle would take minutes."""
    N, trj = config3
    nf = b200_nufft((N, N, N), oversamp=1.25, width=4)
    t = T(trj)
    x = crandn((1, 16, N, N, N), 9)
    y = crandn((1, 16, trj.shape[1]), 10)
    lhs = torch.vdot(nf.forward(x, t).reshape(-1).to(torch.complex128), y.reshape(-1).to(torch.complex128))
    rhs = torch.vdot(x.reshape(-1).to(torch.complex128), nf.adjoint(y, t).reshape(-1).to(torch.complex128))
    assert float(abs(lhs - rhs) / abs(lhs)) < 1e-5


# ----------------------------------------------------------------- configuration 4
def config4_geometry(seed=4, n_slices=64):
    rng = np.random.RandomState(seed)
    sizes = rng.choice([160, 192, 224, 256], n_slices)
    coils = rng.randint(8, 33, n_slices)
    npts = rng.randint(10000, 100001, n_slices) // 16 * 16
    return rng, sizes, coils, npts


def test_config4_all_64_slices_vs_oracle():
    """One uneven plan of all 64 slices (matrix 160..256, 8..32 coils, 10k..100k
    spiral samples) through the GPU; the oracle checks coil 0 of every slice,
    forward and adjoint."""
    rng, sizes, coils, npts = config4_geometry()
    ims = [(int(n), int(n)) for n in sizes]
    trjs = [synth.vd_spiral(16, int(m) // 16, n[0] / 2.0).reshape(-1, 2) for n, m in zip(ims, npts)]
    plan = Plan(ims, [int(m) for m in npts], [int(c) for c in coils], 1.25, (6.0, 6.0), device=DEV)
    plan.set_traj(T(np.concatenate(trjs)))
    img = crandn((plan.n_img,), 11)
    y = crandn((plan.n_ksp,), 12)
    k = torch.empty(plan.n_ksp, dtype=torch.complex64, device=DEV)
    b = torch.empty(plan.n_img, dtype=torch.complex64, device=DEV)
    plan.forward(img, k)
    plan.adjoint(y, b)
    k, b, img, y = Nn(k), Nn(b), Nn(img), Nn(y)
    O.FFT_WORKERS = 1

    def check(s):
        n, m = ims[s], int(npts[s])
        on = O.KBNufftOracle(n, 1.25, 6)
        io, ko = int(plan.img_off[s]), int(plan.ksp_off[s])
        x0 = img[io:io + n[0] * n[1]].reshape(1, 1, *n)
        y0 = y[ko:ko + m].reshape(1, 1, m)
        return (rel(k[ko:ko + m], on.forward(x0, trjs[s][None])[0, 0]),
                rel(b[io:io + n[0] * n[1]], on.adjoint(y0, trjs[s][None])[0, 0].reshape(-1)))

    errs = list(POOL.map(check, range(len(ims))))
    assert max(max(e) for e in errs) < TOL


# ----------------------------------------------------------------- configuration 5
def test_config5_time_segmented_sense_vs_oracle():
    """256^2, 16 coils, 4 x 16,384 spiral over 25 ms, B0 within +-200 Hz,
    L = 20 zero-order segments (one multi-slice plan on the GPU); the oracle's
    segmented SENSE model checks 2 coils of the forward and the adjoint of
    k-space that is zero on the other coils."""
    from mr_recon_b200.field import alpha_segementation, b0_to_phis_alphas
    N, C, nint, nro, L = 256, 16, 4, 16384, 20
    mps = synth.gaussian_coil_maps((N, N), C)
    trj = synth.vd_spiral(nint, nro, N / 2.0)
    yy, xx = np.meshgrid(np.linspace(-1, 1, N), np.linspace(-1, 1, N), indexing="ij")
    b0 = 0.6 * xx + 0.4 * yy - 0.5 * xx * yy + 0.3 * yy ** 2 + np.exp(-((xx - 0.25) ** 2 + (yy + 0.1) ** 2) / 0.08)
    b0 = (200.0 * b0 / np.abs(b0).max()).astype(np.float32)
    phis, alphas = b0_to_phis_alphas(T(b0), (nint, nro), 1, 25e-3 / nro)
    s, t = alpha_segementation(phis, alphas, L, interp_type="zero", verbose=False)
    A = sense_linop(T(trj), T(mps), nufft=b200_nufft((N, N)), spatial_funcs=s, temporal_funcs=t)
    assert A.seg is not None
    x = synth.randn_complex((N, N), np.random.RandomState(13))
    y = synth.randn_complex((C, nint, nro), np.random.RandomState(14))
    y[2:] = 0
    fwd = Nn(A.forward(T(x)))
    adj = Nn(A.adjoint(T(y)))
    on = O.KBNufftOracle((N, N), 1.25, 6)
    Ao = O.SenseOracle(trj, mps[:2], on, spatial_funcs=Nn(s), temporal_funcs=Nn(t))
    assert rel(fwd[:2], Ao.forward(x)) < TOL
    assert rel(adj, Ao.adjoint(y[:2])) < TOL
