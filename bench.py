#!/usr/bin/env python
"""Benchmark: Kaiser-Bessel NUFFT forward + adjoint throughput on B200.

Workload (one "step"): the 2D multi-coil CG-SENSE geometry -- 256x256
complex64 coil images (32 coils = Gaussian coil maps x random-ellipse
phantom), variable-density spiral of 48 interleaves x 2048 samples,
oversampling 1.25, kernel width 6 (the triton_nufft defaults) -- one forward
NUFFT of all coils followed by one adjoint NUFFT of all coils. Metric:
C * M / (t_fwd + t_adj) in Msample*coil/s. Inputs resident in HBM; L2 flushed
(256 MB write) between timed steps, outside the timed events.

Also reported on the same line: the gridding / interpolation kernel roofline
(stage times measured live with CUDA events inside the fused calls), the
end-to-end number through the public API with pinned host buffers, CG-SENSE
solves/s (20 iterations, lambda 1e-3, graph-captured vs eager), the CPU
oracle baseline, and SM clocks sampled during the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: one process per GPU (started by torchrun, or by this script with
--gpus N); the headline workload runs one independent replica per rank (weak
scaling, no data-path collective) and the batched configuration shards its
64 slices over the ranks; job time = max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "NUFFT fwd+adj Msamples·coil/s; batched CG-SENSE solves/s at ≤1e-4 rel err"
UNIT = "Msample·coil/s"
IM = (256, 256)
NCOIL = 32
NINTL, NSAMP = 48, 2048
OS, W = 1.25, 6
WORKLOAD = "2D multi-coil KB NUFFT fwd+adj: 256x256 c64, 32 coils, VD spiral 48x2048, os 1.25, W 6"
HOST_AHEAD_S = 0.4e-3  # device-side wait before each timed step: longer than the host's enqueue of one step
# DRAM bytes (read + write) per launch of each tile kernel on this workload,
# from one ncu capture of the kernels named in TRAFFIC_SOURCE (ncu cannot run
# inside the timed program, so the figure is carried here and labelled).
GRID_TRAFFIC_BYTES = 30_618_624 + 2_219_264
INTERP_TRAFFIC_BYTES = 26_141_440 + 982_272
TRAFFIC_SOURCE = ("ncu --set full capture of k_grid_reg<7,1> (write-back staged through shared memory) "
                  "and k_interp_reg<2,7,1> on this workload (dram__bytes_read.sum + dram__bytes_write.sum "
                  "per launch)")
CG_FIXTURE = os.path.join(ROOT, "tests", "golden", "cg_config2.npz")
# Speed of the oracle port relative to the reference's own CPU path
# (triton_nufft on CPU tensors, its torch fallback) on this workload: both
# timed on the same 8 host threads of the development machine (Intel Xeon,
# 2.7 GHz), 8 coils, forward + adjoint, median of 3 after a warm-up; their
# forward outputs agree to 6e-7. The reference cannot run where the benchmark
# runs, so the port stands in for it and is the slower of the two.
PORT_VS_REFERENCE = {"port_msample_coil_s": 0.44, "reference_msample_coil_s": 1.03, "threads": 8,
                     "ratio": 0.43}


def host_info():
    """Host CPU model and logical core count (for the CPU baselines)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "host_logical_cores": os.cpu_count()}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_inputs(seed):
    from mr_recon_b200 import synth
    rng = np.random.RandomState(seed)
    x = synth.ellipse_phantom(IM, 20, rng)
    mps = synth.gaussian_coil_maps(IM, NCOIL)
    imgs = (mps * x[None]).astype(np.complex64)[None]  # (1, C, 256, 256)
    trj = synth.vd_spiral(NINTL, NSAMP, IM[0] / 2.0)[None]  # (1, 48, 2048, 2)
    return x, mps, imgs, trj


class ClockSampler:
    """nvidia-smi SM clock / throttle sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [v.strip() for v in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(trj, imgs, coils, repeats=1, outputs=None):
    """The CPU oracle (a numpy restatement of the reference's CPU path) on
    `coils` coils, one coil per thread. Returns (Msample*coil/s, threads,
    seconds); with `outputs` (a dict) also stores the last repeat's forward
    k-space ("ksp", (1, coils, ...)) and adjoint images ("img")."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import nufft_oracle as O
    O.FFT_WORKERS = 1
    threads = min(coils, os.cpu_count() or 1)
    nf = O.KBNufftOracle(IM, OS, W)
    M = trj[0].reshape(-1, 2).shape[0]
    t_total = 0.0
    with ThreadPoolExecutor(threads) as ex:
        for _ in range(repeats):
            t0 = time.perf_counter()
            ks = list(ex.map(lambda c: nf.forward(imgs[:, c:c + 1], trj), range(coils)))
            bs = list(ex.map(lambda c: nf.adjoint(ks[c], trj), range(coils)))
            t_total += time.perf_counter() - t0
    if outputs is not None:
        outputs["ksp"] = np.concatenate(ks, 1)
        outputs["img"] = np.concatenate(bs, 1)
    return coils * M * repeats / t_total / 1e6, threads, t_total


REF_DIR = os.path.join(ROOT, "baseline", "_ref")


def reference_package():
    """Import the unmodified reference from baseline/_ref (the package's GPU and
    plotting dependencies, which the KB NUFFT path never calls, stubbed by
    tests/golden/refshim.py); None when it is not installed there."""
    if not os.path.isdir(os.path.join(REF_DIR, "mr_recon")):
        return None
    os.environ.setdefault("TORCH_COMPILE_DISABLE", "1")
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import refshim
    refshim.install(REF_DIR)
    import torch._dynamo
    torch._dynamo.config.disable = True  # the reference's @torch.compile (kernels.py:21,85) runs eagerly
    import mr_recon.fourier
    return mr_recon


def cpu_reference(trj, imgs, coils, repeats=1, threads=None):
    """The reference's own CPU path: its triton_nufft forward + adjoint on CPU
    tensors (the torch fallback of its Triton kernels), all coils in one call
    on `threads` host threads. Returns (Msample*coil/s, threads, seconds) or
    None when the reference is not installed."""
    ref = reference_package()
    if ref is None:
        return None
    import torch
    threads = threads or os.cpu_count() or 1
    torch.set_num_threads(threads)
    nf = ref.fourier.triton_nufft(IM, oversamp=OS, width=W)
    ti = torch.from_numpy(np.ascontiguousarray(imgs[:, :coils]))
    tt = torch.from_numpy(np.ascontiguousarray(trj))
    M = trj[0].reshape(-1, 2).shape[0]
    t_total = 0.0
    for _ in range(repeats):
        t0 = time.perf_counter()
        k = nf.forward(ti, tt)
        nf.adjoint(k, tt)
        t_total += time.perf_counter() - t0
    return coils * M * repeats / t_total / 1e6, threads, t_total


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def bench_c3(dev, steps, peak, N=192, spokes=20000):
    """3D NUFFT with autograd: 192^3, 16 coils, kooshball 20,000 x 384,
    os 1.25, W 4. fwd+adj Msample*coil/s with the gridding roofline (the
    path's HBM-bound case), and one loss / backward step with image and
    trajectory gradients."""
    import torch
    from mr_recon_b200.fourier import b200_nufft
    from mr_recon_b200 import synth
    C = 16
    trj = torch.from_numpy(synth.kooshball(spokes, 2 * N, N / 2.0).reshape(1, -1, 3)).to(dev)
    M = trj.shape[1]
    g = torch.Generator(device=dev).manual_seed(3)
    img = torch.randn((1, C, N, N, N), dtype=torch.complex64, device=dev, generator=g)
    nf = b200_nufft((N, N, N), oversamp=1.25, width=4)
    t0 = time.perf_counter()
    k = nf.forward(img, trj)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    nf.adjoint(k, trj)
    plan = nf._plans.entries[-1][2]
    for _ in range(3):  # warm-up: the allocator's second k-space block, caches
        k = nf.forward(img, trj)
        nf.adjoint(k, trj)
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    sev = [_events(torch) for _ in range(steps)]
    host_s = 0.0
    e0.record()
    for i in range(steps):
        sev[i][0].record()
        h0 = time.perf_counter()
        k = nf.forward(img, trj)
        nf.adjoint(k, trj)
        host_s += time.perf_counter() - h0
        sev[i][1].record()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    step_ms = [a.elapsed_time(b) for a, b in sev]
    # per-stage kernel times from a separate pass (the stage timer's events stay
    # out of the timed steps)
    plan.enable_timing(True)
    plan.timing()
    for i in range(steps):
        k = nf.forward(img, trj)
        nf.adjoint(k, trj)
    torch.cuda.synchronize()
    st = plan.timing()
    plan.enable_timing(False)
    Gos = int(math.ceil(1.25 * N)) ** 3
    alg = 8 * C * (M + Gos) + 4 * 3 * M
    g_ms = st["grid"][0] / max(1, st["grid"][1])
    i_ms = st["interp"][0] / max(1, st["interp"][1])
    # autograd: loss = ||A x - y||^2, gradients for the image and the trajectory
    x = img.clone().requires_grad_(True)
    tr = trj.clone().requires_grad_(True)
    y = (k * 0.9).detach()
    for _ in range(2):
        loss = (nf.forward(x, tr) - y).abs().square().sum()
        loss.backward()
    torch.cuda.synchronize()
    e0.record()
    loss = (nf.forward(x, tr) - y).abs().square().sum()
    loss.backward()
    e1.record()
    torch.cuda.synchronize()
    ag_ms = e0.elapsed_time(e1)
    agp = nf._plans.entries[-1][2]  # the plan bound to the differentiable trajectory
    agp.enable_timing(True)
    agp.timing()
    loss = (nf.forward(x, tr) - y).abs().square().sum()
    loss.backward()
    torch.cuda.synchronize()
    ag_stage = {k2: v[0] for k2, v in agp.timing().items() if v[1]}
    agp.enable_timing(False)
    stats = plan.stats()
    return {
        "workload": f"3D KB NUFFT fwd+adj: {N}^3 c64, 16 coils, kooshball {spokes}x{2 * N}, os 1.25, W 4",
        "value": C * M / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms, "steps": steps,
        "stage_ms": {k2: v[0] / steps for k2, v in st.items() if v[1]},
        "grid_roofline": {"bound": "hbm", "algorithmic_bytes": alg, "kernel_ms": g_ms,
                          "achieved": alg / (g_ms / 1e3) / 1e9, "peak": peak,
                          "frac": alg / (g_ms / 1e3) / 1e9 / peak, "unit": "GB/s"},
        "interp_roofline": {"achieved": alg / (i_ms / 1e3) / 1e9, "frac": alg / (i_ms / 1e3) / 1e9 / peak,
                            "kernel_ms": i_ms},
        "autograd_step_ms": ag_ms, "autograd_stage_ms": ag_stage, "plan_setup_s": setup_s, "plan": stats,
        "step_ms_each": step_ms, "host_enqueue_ms_per_step": host_s * 1e3 / steps,
    }


def bench_c4(dev, iters=30, seed=4, n_slices=64, world=1, rank=0):
    """Batched uneven CG-SENSE: 64 slices (matrix from {160..256}^2, 8-32
    coils, 10k-100k spiral samples), 30 iterations captured in one CUDA graph
    with autotuned bins/tiles, against a loop of per-slice solves on the same
    kernels. Per-slice eigenvalue normalisation (recons.py:117-123) is folded
    into the coil maps: A_s / sqrt(l_s). With several ranks the slices are
    sharded by cost (coils x samples, shard_slices): each rank solves its own
    range in one graph, the job time is the slowest rank's (no data-path
    collective), and the per-slice loop is not run."""
    import torch
    from mr_recon_b200 import synth
    from mr_recon_b200.algs import SenseCG
    from mr_recon_b200.autotune import autotune
    from mr_recon_b200.plan import Plan
    from mr_recon_b200.shard import max_over_ranks, shard_slices
    rng = np.random.RandomState(seed)
    all_sizes = rng.choice([160, 192, 224, 256], n_slices)
    all_coils = rng.randint(8, 33, n_slices)
    all_npts = rng.randint(10000, 100001, n_slices) // 16 * 16
    first, last = shard_slices([float(c) * float(m) for c, m in zip(all_coils, all_npts)], world, rank)
    sizes, coils, npts = all_sizes[first:last], all_coils[first:last], all_npts[first:last]
    xs, mps, trjs = [], [], []
    for s in range(n_slices):
        N = int(all_sizes[s])
        phantom = synth.ellipse_phantom((N, N), 20, rng)  # drawn for every slice: same data on any rank count
        if not first <= s < last:
            continue
        xs.append(phantom.astype(np.complex64).reshape(-1))
        mps.append(synth.gaussian_coil_maps((N, N), int(all_coils[s])).astype(np.complex64).reshape(-1))
        trjs.append(synth.vd_spiral(16, int(all_npts[s]) // 16, N / 2.0).reshape(-1, 2))
    mine = last - first
    if mine == 0:  # more ranks than slices: this rank only joins the timing
        b_ms = max_over_ranks(0.0, dev)
        return {"slices_this_rank": 0, "ranks": world, "ms_per_batch_graph": b_ms,
                "slice_solves_per_s_batched_graph": n_slices * 1e3 / b_ms}
    n_mine = mine
    ims = [(int(n), int(n)) for n in sizes]
    x_t = torch.from_numpy(np.concatenate(xs)).to(dev)
    m_t = torch.from_numpy(np.concatenate(mps)).to(dev)
    t_t = torch.from_numpy(np.concatenate(trjs)).to(dev)
    plan = Plan(ims, [int(m) for m in npts], [int(c) for c in coils], 1.25, (6.0, 6.0), device=dev)
    t0 = time.perf_counter()
    tune = autotune(plan, t_t)
    tune_s = time.perf_counter() - t0
    ksp = torch.empty(plan.n_ksp, dtype=torch.complex64, device=dev)
    plan.sense_forward(x_t, m_t, ksp)
    g = torch.Generator(device=dev).manual_seed(seed)
    noise = torch.randn(ksp.shape, dtype=torch.complex64, device=dev, generator=g)
    ksp += noise * (ksp.abs().square().mean().sqrt() * 10 ** (-30 / 20))
    # per-slice max eigenvalue (batched power method, setup) folded into the maps
    img_off = [int(o) for o in plan.img_off]
    nimg = [int(c) * n[0] * n[1] for c, n in zip(coils, ims)]
    xoff = np.concatenate([[0], np.cumsum([n[0] * n[1] for n in ims])])
    v = torch.randn(int(xoff[-1]), dtype=torch.complex64, device=dev, generator=g)
    z = torch.empty_like(v)
    lam = None
    for _ in range(15):
        plan.sense_normal(v, m_t, None, z)
        lam = torch.stack([z[xoff[s]:xoff[s + 1]].norm() for s in range(n_mine)])
        v = z / torch.repeat_interleave(lam, torch.tensor(np.diff(xoff), device=dev))
    lam = (lam * 1.01).double()
    m_s = m_t.clone()
    for s in range(n_mine):
        m_s[img_off[s]:img_off[s] + nimg[s]] /= float(lam[s].sqrt())
    solver = SenseCG(plan, m_s, None, iters, 1e-3, 1.0)
    solver.ksp.copy_(ksp)
    solver.solve()
    solver.capture()
    xb = solver.solve().clone()
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    reps = 5
    e0.record()
    for _ in range(reps):
        solver.graph.replay()
    e1.record()
    torch.cuda.synchronize()
    b_ms = max_over_ranks(e0.elapsed_time(e1) / reps, dev)  # the slowest rank sets the job time
    out = {
        "workload": "batched uneven CG-SENSE: 64 slices, N in {160..256}^2, 8-32 coils, 10k-100k spiral "
                    "samples, 30 iterations, lambda 1e-3",
        "slice_solves_per_s_batched_graph": n_slices * 1e3 / b_ms, "ms_per_batch_graph": b_ms,
        "ranks": world, "slices_this_rank": n_mine,
        "autotune": {k: v for k, v in tune.items()}, "autotune_s": tune_s,
        "total_coil_samples": int(sum(int(c) * int(m) for c, m in zip(all_coils, all_npts))),
    }
    if world > 1:
        return out
    # per-slice loop on the same kernels: one plan and one eager solve per slice,
    # with the batched plan's tiles, work-item sizes and gridding lane group,
    # so every slice is computed in the same order as inside the batch
    from mr_recon_b200 import _lib
    ksp_off = [int(o) for o in plan.ksp_off]
    maxc = int(max(coils))
    lanes = 8 if maxc <= 8 else (16 if maxc <= 16 else 32)
    singles = []
    for s in range(n_slices):
        p1 = Plan([ims[s]], [int(npts[s])], [int(coils[s])], 1.25, (6.0, 6.0), device=dev)
        p1.set_option(_lib.MRN_OPT_INTERP_TILE, int(tune["interp_tile"]))
        p1.set_option(_lib.MRN_OPT_INTERP_CHUNK, int(tune["interp_chunk"]))
        p1.set_option(_lib.MRN_OPT_GRID_TILE, int(tune["grid_tile"]))
        p1.set_option(_lib.MRN_OPT_GRID_CHUNK, int(tune["grid_chunk"]))
        p1.set_option(_lib.MRN_OPT_GRID_LANES, lanes)
        p1.set_traj(t_t[int(plan.trj_off[s]) // 2:int(plan.trj_off[s]) // 2 + int(npts[s])])
        s1 = SenseCG(p1, m_s[img_off[s]:img_off[s] + nimg[s]], None, iters, 1e-3, 1.0)
        s1.ksp.copy_(ksp[ksp_off[s]:ksp_off[s] + int(coils[s]) * int(npts[s])])
        singles.append(s1)
    for s1 in singles:
        s1.solve()
    torch.cuda.synchronize()
    e0.record()
    xs_loop = [s1.solve().clone() for s1 in singles]
    e1.record()
    torch.cuda.synchronize()
    l_ms = e0.elapsed_time(e1)
    xl = torch.cat(xs_loop)
    out.update({"slice_solves_per_s_per_slice_loop": n_slices * 1e3 / l_ms, "ms_per_slice_loop": l_ms,
                "speedup": l_ms / b_ms, "batched_vs_loop_rel_diff": float((xb - xl).norm() / xl.norm())})
    return out


def bench_c5(dev, iters=20, L=20):
    """Time-segmented off-resonance SENSE: 256^2, 16 coils, 4 spiral
    interleaves x 16,384 samples over a 25 ms readout, smooth B0 within
    +-200 Hz (low-order polynomial + Gaussian bump), L = 20 segments
    (b0_to_phis_alphas + alpha_segementation, zero-order interpolators as the
    reference's default); one CG-SENSE solve (20 iterations, lambda 1e-3)
    and one gradient step on the trajectory through the autograd backward of
    ||A(k) x - y||^2."""
    import torch
    from mr_recon_b200 import synth
    from mr_recon_b200.field import alpha_segementation, b0_to_phis_alphas
    from mr_recon_b200.fourier import b200_nufft
    from mr_recon_b200.linops import sense_linop
    from mr_recon_b200.recons import CG_SENSE_recon
    rng = np.random.RandomState(5)
    N, C, nint, nro = 256, 16, 4, 16384
    dt = 25e-3 / nro
    x_np = synth.ellipse_phantom((N, N), 20, rng).astype(np.complex64)
    mps_np = synth.gaussian_coil_maps((N, N), C).astype(np.complex64)
    trj_np = synth.vd_spiral(nint, nro, N / 2.0)  # (4, 16384, 2)
    yy, xx = np.meshgrid(np.linspace(-1, 1, N), np.linspace(-1, 1, N), indexing="ij")
    b0 = 0.6 * xx + 0.4 * yy - 0.5 * xx * yy + 0.3 * yy ** 2 + np.exp(-((xx - 0.25) ** 2 + (yy + 0.1) ** 2) / 0.08)
    b0 = (200.0 * b0 / np.abs(b0).max()).astype(np.float32)
    trj = torch.from_numpy(trj_np).to(dev)
    mps = torch.from_numpy(mps_np).to(dev)
    x = torch.from_numpy(x_np).to(dev)
    t0 = time.perf_counter()
    phis, alphas = b0_to_phis_alphas(torch.from_numpy(b0).to(dev), (nint, nro), 1, dt)
    sfun, tfun = alpha_segementation(phis, alphas, L, interp_type="zero", verbose=False)
    nf = b200_nufft((N, N), oversamp=1.25, width=6)
    A = sense_linop(trj, mps, nufft=nf, spatial_funcs=sfun, temporal_funcs=tfun)
    y = A.forward(x)
    g = torch.Generator(device=dev).manual_seed(5)
    y = y + torch.randn(y.shape, dtype=torch.complex64, device=dev, generator=g) * (
        y.abs().square().mean().sqrt() * 10 ** (-30 / 20))
    v = torch.randn((N, N), dtype=torch.complex64, device=dev, generator=g)
    for _ in range(15):  # power method for max_eigen (setup)
        z = A.normal(v)
        lam = float(torch.linalg.vector_norm(z))
        v = z / lam
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    rec = CG_SENSE_recon(A, y, max_iter=iters, lamda_l2=1e-3, max_eigen=lam * 1.01, verbose=False)
    e0, e1 = _events(torch)
    torch.cuda.synchronize()
    e0.record()
    rec = CG_SENSE_recon(A, y, max_iter=iters, lamda_l2=1e-3, max_eigen=lam * 1.01, verbose=False)
    e1.record()
    torch.cuda.synchronize()
    cg_ms = e0.elapsed_time(e1)
    # CG on A / sqrt(max_eigen) (recons.py:117-123) returns the image scaled by
    # sqrt(max_eigen): compare after the least-squares complex scale
    scl = (rec.conj() * x).sum() / (rec.conj() * rec).sum()
    nrmse = float((scl * rec - x).norm() / x.norm())
    # one gradient step on the trajectory: loss = ||A(k) x_hat - y||^2
    k = trj.clone().requires_grad_(True)
    A2 = sense_linop(k, mps, nufft=nf, spatial_funcs=sfun, temporal_funcs=tfun)
    xh = (scl * rec).detach()
    loss = (A2.forward(xh) - y).abs().square().sum()
    loss.backward()
    torch.cuda.synchronize()
    k.grad = None
    e0.record()
    loss = (A2.forward(xh) - y).abs().square().sum()
    loss.backward()
    with torch.no_grad():
        k_new = k - 1e-3 * k.grad / (k.grad.abs().max() + 1e-30)
    e1.record()
    torch.cuda.synchronize()
    gs_ms = e0.elapsed_time(e1)
    # least-squares interpolators (alpha_segementation interp_type='lstsq'): every
    # sample in every segment; the low-rank plan runs all 20 segments in one
    # pass, against the same kernels as one batched NUFFT of all coils x
    # segments with torch products around it
    t1 = time.perf_counter()
    s_ls, t_ls = alpha_segementation(phis, alphas, L, interp_type="lstsq", verbose=False)
    A3 = sense_linop(trj, mps, nufft=nf, spatial_funcs=s_ls, temporal_funcs=t_ls)
    torch.cuda.synchronize()
    ls_setup_s = time.perf_counter() - t1
    rec3 = CG_SENSE_recon(A3, y, max_iter=iters, lamda_l2=1e-3, max_eigen=lam * 1.01, verbose=False)
    torch.cuda.synchronize()
    e0.record()
    rec3 = CG_SENSE_recon(A3, y, max_iter=iters, lamda_l2=1e-3, max_eigen=lam * 1.01, verbose=False)
    e1.record()
    torch.cuda.synchronize()
    ls_cg_ms = e0.elapsed_time(e1)
    scl3 = (rec3.conj() * x).sum() / (rec3.conj() * rec3).sum()

    def normal_ms(op, reps=5):
        op.normal(x)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            out = op.normal(x)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, out

    lr_ms, n_lr = normal_ms(A3)
    lr_plan, A3.lr = A3.lr, None
    bt_ms, n_bt = normal_ms(A3)
    A3.lr = lr_plan
    return {
        "workload": "time-segmented B0 SENSE: 256^2, 16 coils, 4x16384 spiral over 25 ms, B0 within "
                    "+-200 Hz, L=20 segments (zero-order), CG 20 iterations lambda 1e-3",
        "cg_solve_ms": cg_ms, "solves_per_s": 1e3 / cg_ms, "recon_nrmse_vs_phantom": nrmse,
        "traj_grad_step_ms": gs_ms, "traj_grad_finite": bool(torch.isfinite(k.grad).all()),
        "traj_step_max_move": float((k_new - k).abs().max()), "setup_s": setup_s,
        "coil_segments_per_nufft": C * L,
        "lstsq": {"interp_type": "lstsq (type-3 least squares, every sample in all 20 segments)",
                  "cg_solve_ms": ls_cg_ms, "solves_per_s": 1e3 / ls_cg_ms,
                  "recon_nrmse_vs_phantom": float((scl3 * rec3 - x).norm() / x.norm()),
                  "normal_ms_lowrank_plan": lr_ms, "normal_ms_batched_nufft": bt_ms,
                  "lowrank_vs_batched_rel_diff": float((n_lr - n_bt).norm() / n_bt.norm()),
                  "setup_s": ls_setup_s},
    }


def run_reference(args, rank):
    """--impl reference: the reference's own CPU path (its triton_nufft on CPU
    tensors, from the unmodified package in baseline/_ref) on all host cores,
    rank 0 only; each step is a bounded sample (8 of the 32 coils). Without
    baseline/_ref, the oracle port stands in (kind "port")."""
    if rank != 0:
        return
    _, _, imgs, trj = make_inputs(0)
    ncores = os.cpu_count() or 1
    M = NINTL * NSAMP
    coils = 8  # a bounded sample of the 32 coils per step
    if reference_package() is not None:
        # the reference's own CPU path, all host threads on each step's coils
        for _ in range(min(args.warmup, 1)):
            cpu_reference(trj, imgs, coils, 1, ncores)
        v, thr, secs = cpu_reference(trj, imgs, coils, args.steps, ncores)
        kind, extra = "reference", {}
        sample = f"{coils} of 32 coils per step in one call on {thr} threads, full 98304-sample spiral, fwd+adj"
    else:
        # the oracle port, one coil per host thread (it is slower than the reference's CPU path)
        coils = int(max(1, min(ncores, NCOIL)))
        for _ in range(min(args.warmup, 1)):
            cpu_baseline(trj, imgs, coils, 1)
        v, thr, secs = cpu_baseline(trj, imgs, coils, args.steps)
        kind, extra = "port", {"port_vs_reference_cpu": PORT_VS_REFERENCE}
        sample = f"{coils} of 32 coils per step (one per host thread), full 98304-sample spiral, fwd+adj"
    ms = secs / args.steps * 1e3
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_coils_per_step": coils, "samples_per_coil": M},
        "cpu_baseline": dict({"value": v, "unit": UNIT, "cores": thr, "kind": kind, "sample": sample},
                             **extra, **host_info()),
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_gpu(args, rank):
    """--impl reference_gpu (not part of the default runs): the reference's own
    GPU NUFFT -- triton_nufft over its Triton interpolation and gridding
    kernels (triton_interp/ungrid.py:154-846, grid.py:158-502) -- from the
    unmodified package installed in baseline/_ref, on the headline workload
    and on this GPU, timed with CUDA events after a warm-up that includes the
    Triton compilation. Modules the KB path never calls (cupy, sigpy, ...) are
    stubbed by tests/golden/refshim.py so the package imports."""
    if rank != 0:
        return
    if reference_package() is None:
        print(json.dumps({"impl": "reference_gpu", "unavailable": "the reference is not installed in baseline/_ref"}))
        return
    import torch
    from mr_recon.fourier import triton_nufft
    dev = torch.device("cuda", 0)
    _, _, imgs_np, trj_np = make_inputs(1234)
    imgs = torch.from_numpy(imgs_np).to(dev)
    trj = torch.from_numpy(trj_np).to(dev)
    nf = triton_nufft(IM, oversamp=OS, width=W)
    for _ in range(max(3, args.warmup)):
        k = nf.forward(imgs, trj)
        nf.adjoint(k, trj)
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    e0.record()
    for _ in range(args.steps):
        k = nf.forward(imgs, trj)
        b = nf.adjoint(k, trj)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    # the B200 path on the same inputs, for the relative difference of the results
    from mr_recon_b200.fourier import b200_nufft
    ours = b200_nufft(IM, oversamp=OS, width=W)
    ko = ours.forward(imgs, trj)
    bo = ours.adjoint(k, trj)
    rel = lambda a, r: float((a - r).abs().square().sum().sqrt() / r.abs().square().sum().sqrt())  # noqa: E731
    M = NINTL * NSAMP
    # CG-SENSE with the reference's own linop and solver on its Triton NUFFT (all
    # coils in one batch; max_eigen given, as the benchmark's CG-SENSE does)
    from mr_recon.linops import batching_params, sense_linop
    from mr_recon.recons import CG_SENSE_recon
    from mr_recon_b200 import synth
    x_np, mps_np, _, _ = make_inputs(1234)
    A = sense_linop(trj[0], torch.from_numpy(mps_np).to(dev), nufft=nf,
                    bparams=batching_params(coil_batch_size=NCOIL))
    kk = A.forward(torch.from_numpy(x_np).to(dev))
    kk = torch.from_numpy(synth.add_noise(kk.cpu().numpy(), 30.0, np.random.RandomState(99))).to(dev)
    fix = np.load(CG_FIXTURE) if os.path.exists(CG_FIXTURE) else None
    me = float(fix["max_eigen"]) if fix is not None else 1.0
    xr = CG_SENSE_recon(A, kk, max_iter=20, lamda_l2=1e-3, max_eigen=me, verbose=False)
    torch.cuda.synchronize()
    e0.record()
    reps = 3
    for _ in range(reps):
        xr = CG_SENSE_recon(A, kk, max_iter=20, lamda_l2=1e-3, max_eigen=me, verbose=False)
    e1.record()
    torch.cuda.synchronize()
    cg_ms = e0.elapsed_time(e1) / reps
    cg = {"solves_per_s": 1e3 / cg_ms, "ms_per_solve": cg_ms, "iterations": 20, "lambda": 1e-3,
          "coil_batch_size": NCOIL}
    if fix is not None:
        ref = torch.from_numpy(fix["x_cg64"]).to(dev)
        cg["rel_err_vs_oracle_cg64"] = rel(xr.reshape(ref.shape), ref)
    print(json.dumps({"impl": "reference_gpu", "metric": METRIC, "value": NCOIL * M / (ms / 1e3) / 1e6,
                      "unit": UNIT, "ms_per_step": ms, "steps": args.steps, "dtype": "complex64",
                      "config": {"workload": WORKLOAD}, "cg_sense": cg,
                      "rel_diff_vs_b200": {"forward": rel(ko, k), "adjoint": rel(bo, b)}}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference_gpu"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cg", action="store_true")
    ap.add_argument("--c3-n", type=int, default=192, help="c3 image edge (192 = the configuration)")
    ap.add_argument("--c3-spokes", type=int, default=20000, help="c3 kooshball spokes (20000 = the configuration)")
    ap.add_argument("--extra", default="c3,c4,c5",
                    help="comma list of the other configurations to add to the line: c3 (3D), c4 (batched "
                         "uneven CG), c5 (B0 segments); empty for none")
    args = ap.parse_args()
    if args.impl == "ours" and args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start the ranks here when no launcher did
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.impl == "reference_gpu":
        run_reference_gpu(args, rank)
        return

    import torch
    import torch.distributed as dist
    from mr_recon_b200.fourier import b200_nufft
    from mr_recon_b200.linops import sense_linop
    from mr_recon_b200.algs import SenseCG
    from mr_recon_b200 import synth
    from mr_recon_b200.shard import max_over_ranks

    if args.warmup < 3:
        args.warmup = 3
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", device_id=dev, timeout=__import__("datetime").timedelta(seconds=120))

    x_np, mps_np, imgs_np, trj_np = make_inputs(1234 + rank)
    imgs = torch.from_numpy(imgs_np).to(dev)
    trj = torch.from_numpy(trj_np).to(dev)
    C, M = NCOIL, NINTL * NSAMP
    nf = b200_nufft(IM, oversamp=OS, width=W)
    ksp = nf.forward(imgs, trj)
    back = nf.adjoint(ksp, trj)
    torch.cuda.synchronize()
    plan = nf._plans.entries[-1][2]
    stats = plan.stats()
    stats["fft_kind"] = plan.fft_kind
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def step():
        k = nf.forward(imgs, trj)
        nf.adjoint(k, trj)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    host_s = 0.0
    hold = int(HOST_AHEAD_S * 1.965e9)  # device cycles at the top SM clock
    for i in range(args.steps):
        flush.zero_()
        # the device waits while the host enqueues this step, so the step's
        # launches are queued when its start event fires, as in a pipelined
        # loop; the host's enqueue time is reported beside, and e2e pays it
        torch.cuda._sleep(hold)
        evs[i][0].record()
        h0 = time.perf_counter()
        step()
        host_s += time.perf_counter() - h0
        evs[i][1].record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    total_ms = max_over_ranks(total_ms, dev)  # the slowest rank sets the job time
    value = world * C * M * args.steps / (total_ms / 1e3) / 1e6

    # per-stage kernel times from a separate pass of the same steps: the stage
    # timer's event pairs sit between the kernels, so they stay out of the
    # timed steps above (they cost ~11% of a config-2 step)
    plan.enable_timing(True)
    plan.timing()  # clear
    for i in range(args.steps):
        flush.zero_()
        torch.cuda._sleep(hold)
        step()
    torch.cuda.synchronize()
    stage = plan.timing()
    plan.enable_timing(False)


    # roofline of the dominant kernel (gridding or interpolation)
    peak, peak_kind = load_peaks()
    Gos = math.prod(math.ceil(OS * n) for n in IM)
    alg = 8 * C * Gos + 8 * C * M + 4 * 2 * M
    g_ms = stage["grid"][0] / max(1, stage["grid"][1])
    i_ms = stage["interp"][0] / max(1, stage["interp"][1])
    dom, dms, traffic = ("grid", g_ms, GRID_TRAFFIC_BYTES) if g_ms >= i_ms else ("interp", i_ms, INTERP_TRAFFIC_BYTES)
    achieved = alg / (dms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                "traffic_source": TRAFFIC_SOURCE,
                "algorithmic_bytes": alg, "kernel_ms": dms,
                "stage_ms_per_step": {k: v[0] / args.steps for k, v in stage.items() if v[1]},
                "host_enqueue_ms_per_step": host_s * 1e3 / args.steps}

    # end to end through the public API with pinned host buffers
    img_h = imgs.cpu().pin_memory()
    ksp_h = torch.empty(ksp.shape, dtype=ksp.dtype).pin_memory()
    ksp_in_h = ksp.cpu().pin_memory()
    out_h = torch.empty(back.shape, dtype=back.dtype).pin_memory()

    def e2e_serial_step():
        a = img_h.to(dev, non_blocking=True)
        k = nf.forward(a, trj)
        ksp_h.copy_(k, non_blocking=True)
        b = ksp_in_h.to(dev, non_blocking=True)
        o = nf.adjoint(b, trj)
        out_h.copy_(o, non_blocking=True)

    # The same calls with the host->device and device->host copies on their
    # own streams (the two copy engines), ordered by events, so the copies of
    # one step overlap each other, the kernels, and the neighbouring steps.
    main = torch.cuda.current_stream(dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def e2e_step():
        with torch.cuda.stream(s_in):
            a = img_h.to(dev, non_blocking=True)
            ev_a = s_in.record_event()
            b = ksp_in_h.to(dev, non_blocking=True)
            ev_b = s_in.record_event()
        main.wait_event(ev_a)
        a.record_stream(main)
        k = nf.forward(a, trj)
        s_out.wait_event(main.record_event())
        with torch.cuda.stream(s_out):
            ksp_h.copy_(k, non_blocking=True)
        k.record_stream(s_out)
        main.wait_event(ev_b)
        b.record_stream(main)
        o = nf.adjoint(b, trj)
        s_out.wait_event(main.record_event())
        with torch.cuda.stream(s_out):
            out_h.copy_(o, non_blocking=True)
        o.record_stream(s_out)

    ne = max(5, min(args.steps, 50))

    def time_e2e(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        s_in.wait_event(e0)
        s_out.wait_event(e0)
        for _ in range(ne):
            fn()
        main.wait_stream(s_in)
        main.wait_stream(s_out)
        e1.record(main)
        torch.cuda.synchronize()
        t = max_over_ranks(e0.elapsed_time(e1), dev)
        return world * C * M * ne / (t / 1e3) / 1e6

    e2e_val = time_e2e(e2e_step)
    # against the device-resident run (the same kernels: bit-identical)
    def _rel(a, b):
        return float((a - b).abs().square().sum().sqrt() / b.abs().square().sum().sqrt())
    match = max(_rel(out_h, back.cpu()), _rel(ksp_h, ksp.cpu()))
    e2e_serial = time_e2e(e2e_serial_step)

    # the same step replayed from one CUDA graph (static input and output
    # buffers; the plan's calls are asynchronous and capturable)
    gstream = torch.cuda.Stream(dev)
    gstream.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(gstream):
        for _ in range(3):
            step()
    torch.cuda.current_stream(dev).wait_stream(gstream)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step()
    torch.cuda.synchronize()
    gevs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        torch.cuda._sleep(hold)
        gevs[i][0].record()
        graph.replay()
        gevs[i][1].record()
    torch.cuda.synchronize()
    graph_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in gevs), dev)
    graph_value = world * C * M * args.steps / (graph_ms / 1e3) / 1e6
    del graph
    nbytes_img = img_h.numel() * 8
    nbytes_ksp = ksp_h.numel() * 8
    e2e = {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nbytes_img + nbytes_ksp,
           "d2h_bytes_per_step": nbytes_ksp + nbytes_img, "steps": ne,
           "copies": "pinned host buffers; H2D and D2H on their own streams, overlapping the kernels",
           "serial_value": e2e_serial, "rel_diff_vs_device_run": match}

    # CG-SENSE solves/s (20 iterations, lambda 1e-3), graph vs eager
    cg = None
    if not args.no_cg:
        rng = np.random.RandomState(99 + rank)
        A = sense_linop(trj[0], torch.from_numpy(mps_np).to(dev), nufft=nf)
        kk = A.forward(torch.from_numpy(x_np).to(dev))
        kk = torch.from_numpy(synth.add_noise(kk.cpu().numpy(), 30.0, rng)).to(dev)
        # the oracle's float64 CG on this problem (rank 0's inputs), computed
        # on the CPU by tests/golden/make_cg_config2.py with its max eigenvalue
        fix = np.load(CG_FIXTURE) if (rank == 0 and os.path.exists(CG_FIXTURE)) else None
        if fix is not None:
            max_eig = float(fix["max_eigen"])
        else:
            max_eig = 1.0
            for _ in range(15):  # power method (setup, not timed)
                v = torch.randn(IM, dtype=torch.complex64, device=dev) if _ == 0 else v
                z = A.normal(v)
                max_eig = float(torch.linalg.vector_norm(z))
                v = z / max_eig
            max_eig *= 1.01
        solver = SenseCG(A.plan, A.mps, A.dcf, 20, 1e-3, max_eig)
        solver.ksp.copy_(kk.reshape(-1))
        x_eager = solver.solve().clone()
        solver.capture()
        x_graph = solver.solve().clone()
        reps = 20
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record()
        for _ in range(reps):
            solver.graph.replay()
        c1.record()
        torch.cuda.synchronize()
        g_ms = c0.elapsed_time(c1) / reps
        solver.graph = None
        c0.record()
        for _ in range(5):
            solver.solve()
        c1.record()
        torch.cuda.synchronize()
        e_ms = c0.elapsed_time(c1) / 5
        # the same solve with the Toeplitz normal (FFT-only A^H A on the 2x grid)
        At = sense_linop(trj[0], torch.from_numpy(mps_np).to(dev), nufft=nf, use_toeplitz=True)
        st = SenseCG(At.plan, At.mps, At.dcf, 20, 1e-3, max_eig, toeplitz=True)
        st.ksp.copy_(kk.reshape(-1))
        st.solve()
        st.capture()
        x_toep = st.solve().clone()
        torch.cuda.synchronize()
        c0.record()
        for _ in range(reps):
            st.graph.replay()
        c1.record()
        torch.cuda.synchronize()
        t_ms = c0.elapsed_time(c1) / reps
        st.graph = None
        cg = {"solves_per_s_graph": world * 1e3 / g_ms, "solves_per_s_eager": world * 1e3 / e_ms,
              "toeplitz_solves_per_s_graph": world * 1e3 / t_ms,
              "toeplitz_vs_nufft_normal_rel_diff": float((x_toep - x_graph).norm() / x_graph.norm()),
              "ms_per_solve_graph": g_ms, "iterations": 20, "lambda": 1e-3,
              "graph_vs_eager_rel_diff": float((x_graph - x_eager).norm() / x_eager.norm()),
              "precision": "complex64 vectors and NUFFT, float64 dot products summed in a fixed order"}
        if fix is not None:
            ref = torch.from_numpy(fix["x_cg64"]).to(dev).reshape(-1)
            cg["rel_err_vs_oracle_cg64"] = float((x_graph.reshape(-1) - ref).norm() / ref.norm())
            cg["reference_f32_arith_rel_err_vs_oracle_cg64"] = float(fix["rel_f32_arith"])

    cpu = None
    rel_err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nb = int(min(NCOIL, max(1, os.cpu_count() or 1)))
        outs = {}
        v, thr, secs = cpu_baseline(trj_np, imgs_np, nb, 2, outputs=outs)
        cpu = dict({"value": v, "unit": UNIT, "cores": thr, "kind": "port",
                    "sample": f"{nb} of 32 coils (one per host thread), full 98304-sample spiral, fwd+adj, "
                              "2 repeats", "seconds": secs, "port_vs_reference_cpu": PORT_VS_REFERENCE},
                   **host_info())
        # the GPU results against the oracle's on the same coils and inputs
        k_o = torch.from_numpy(outs["ksp"]).to(dev)
        b_g = nf.adjoint(k_o, trj)

        def _r(a, b):
            return float((a - b).abs().square().sum().sqrt() / b.abs().square().sum().sqrt())
        rel_err = {"forward": _r(ksp[:, :nb], k_o),
                   "adjoint": _r(b_g, torch.from_numpy(outs["img"]).to(dev)),
                   "against": f"CPU oracle, {nb} coils, same inputs"}
        ref_cpu = cpu_reference(trj_np, imgs_np, 8, 2)
        if ref_cpu is not None:  # the reference's own CPU path: the baseline that counts
            cpu = dict({"value": ref_cpu[0], "unit": UNIT, "cores": ref_cpu[1], "kind": "reference",
                        "sample": "8 of 32 coils in one call on all host threads, full 98304-sample spiral, "
                                  "fwd+adj, 2 repeats", "seconds": ref_cpu[2],
                        "oracle_port": {"value": v, "cores": thr}}, **host_info())
        if cg is not None and "rel_err_vs_oracle_cg64" in cg:
            rel_err["cg_sense"] = cg["rel_err_vs_oracle_cg64"]

    extra = {}
    want = [e.strip() for e in args.extra.split(",") if e.strip()]
    if "c4" in want:  # every rank: the 64 slices are sharded over the ranks
        extra["c4"] = bench_c4(dev, world=world, rank=rank)
    if rank == 0:  # single-problem configurations on the first GPU
        if "c3" in want:
            extra["c3"] = bench_c3(dev, 5, peak, args.c3_n, args.c3_spokes)
        if "c5" in want:
            extra["c5"] = bench_c5(dev)

    # own kernels per fwd+adj step: interpolation and gridding, plus either the
    # four native FFT passes (pad and crop fused) or k_pre / k_post around cuFFT,
    # plus the split-tile reduction
    launches_per_step = 2 + (4 if stats["fft_kind"] == 1 else 2) + (1 if stats["split_tiles"] > 0 else 0)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "coils": C, "samples": M, "grid": [320, 320],
                       "l2": "flushed between steps (256 MB write, outside the timed events)",
                       "host_ahead": f"{HOST_AHEAD_S * 1e3:.1f} ms device-side wait before each timed step "
                                     "(outside the events) while the host enqueues it",
                       "parallelism": f"replicas x{world}", "plan": stats},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "cg_sense": cg, "rel_err": rel_err,
            "gpu_launches": launches_per_step * args.steps, "clocks": clocks,
            "graph": {"value": graph_value, "unit": UNIT, "ms_per_step": graph_ms / args.steps,
                      "note": "the same forward + adjoint step replayed from one CUDA graph"},
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
