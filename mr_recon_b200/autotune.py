"""Autotuner for the work decomposition of a plan: the tile edges and work-item
sizes of interpolation and gridding (plan options MRN_OPT_INTERP_TILE,
MRN_OPT_INTERP_CHUNK, MRN_OPT_GRID_TILE, MRN_OPT_GRID_CHUNK).

The reference has no counterpart: its Triton kernels take a fixed block of
points per program (ungrid.py:127-129, grid.py:121-123). Here the best
decomposition depends on the trajectory's density and on coils and grid
size, so ``autotune`` times a small set of candidates on the plan's own
bound trajectory (CUDA events around the interpolation and gridding stages
of a forward + adjoint on zero-filled buffers), keeps the fastest and
leaves the plan bound with it. Interpolation and gridding options are
independent, so each is tuned with the other held fixed. Results are cached
per geometry (dimension, sizes, coil and sample counts, width, oversampling)
and reused without timing.
"""

from __future__ import annotations

from typing import Dict, Optional, Sequence, Tuple

import torch

from . import _lib
from .plan import Plan

__all__ = ["autotune", "default_candidates", "clear_cache"]

_CACHE: Dict[tuple, dict] = {}


def clear_cache() -> None:
    _CACHE.clear()


def default_candidates(ndim: int) -> dict:
    """Candidate values per option. 2D gridding tiles stay at most 8 cells
    so the register-tile gridding kernel applies."""
    if ndim == 2:
        return {"interp_tile": [8, 10, 12], "interp_chunk": [128, 256],
                "grid_tile": [6, 8], "grid_chunk": [128, 192, 256, 384]}
    if ndim == 3:
        return {"interp_tile": [4, 5, 6], "interp_chunk": [256, 1024],
                "grid_tile": [6, 8], "grid_chunk": [1024, 2048, 4096]}
    return {"interp_tile": [128, 256], "interp_chunk": [512, 1024],
            "grid_tile": [128, 256], "grid_chunk": [512, 1024]}


def _key(plan: Plan) -> tuple:
    return (plan.ndim, tuple(plan.im_sizes), tuple(plan.n_pts), tuple(plan.n_coil), plan.width,
            plan.oversamp, plan.raw, str(plan.device))


def _apply(plan: Plan, opts: dict, trj: torch.Tensor) -> None:
    plan.set_option(_lib.MRN_OPT_INTERP_TILE, opts["interp_tile"])
    plan.set_option(_lib.MRN_OPT_INTERP_CHUNK, opts["interp_chunk"])
    plan.set_option(_lib.MRN_OPT_GRID_TILE, opts["grid_tile"])
    plan.set_option(_lib.MRN_OPT_GRID_CHUNK, opts["grid_chunk"])
    plan.set_traj(trj)


def _stage_ms(plan: Plan, bufs, reps: int) -> Tuple[float, float]:
    """Mean interpolation and gridding stage time (ms) over `reps` forward +
    adjoint calls, after one untimed call."""
    img, ksp = bufs
    if plan.raw:
        plan.interp(img, ksp)
        plan.grid(ksp, img)
    else:
        plan.forward(img, ksp)
        plan.adjoint(ksp, img)
    torch.cuda.synchronize(plan.device)
    plan.enable_timing(True)
    plan.timing()
    for _ in range(reps):
        if plan.raw:
            plan.interp(img, ksp)
            plan.grid(ksp, img)
        else:
            plan.forward(img, ksp)
            plan.adjoint(ksp, img)
    t = plan.timing()
    plan.enable_timing(False)
    return t["interp"][0] / reps, t["grid"][0] / reps


def autotune(plan: Plan, trj: torch.Tensor, reps: int = 3, candidates: Optional[dict] = None,
             cache: bool = True) -> dict:
    """Choose the decomposition options of ``plan`` for trajectory ``trj``
    (device float32, all slices back to back, grid units). Returns the chosen
    options with the measured stage times; the plan is left bound to ``trj``
    with them."""
    key = _key(plan)
    if cache and key in _CACHE:
        best = _CACHE[key]
        _apply(plan, best, trj)
        return dict(best, cached=True)
    cand = dict(default_candidates(plan.ndim))
    if candidates:
        cand.update(candidates)
    dev = plan.device
    n_in = plan.n_grid if plan.raw else plan.n_img
    with torch.cuda.device(dev):
        bufs = (torch.zeros(max(n_in, 1), dtype=torch.complex64, device=dev),
                torch.zeros(max(plan.n_ksp, 1), dtype=torch.complex64, device=dev))
    opts = {k: v[0] if k not in ("interp_chunk", "grid_chunk") else v[len(v) // 2] for k, v in cand.items()}
    trials = []

    def measure(o):
        _apply(plan, o, trj)
        ti, tg = _stage_ms(plan, bufs, reps)
        trials.append((dict(o), ti, tg))
        return ti, tg

    # interpolation options with gridding held fixed, then gridding
    best_i = None
    for t in cand["interp_tile"]:
        for c in cand["interp_chunk"]:
            o = dict(opts, interp_tile=t, interp_chunk=c)
            ti, _ = measure(o)
            if best_i is None or ti < best_i[0]:
                best_i = (ti, t, c)
    opts.update(interp_tile=best_i[1], interp_chunk=best_i[2])
    best_g = None
    for t in cand["grid_tile"]:
        for c in cand["grid_chunk"]:
            o = dict(opts, grid_tile=t, grid_chunk=c)
            _, tg = measure(o)
            if best_g is None or tg < best_g[0]:
                best_g = (tg, t, c)
    opts.update(grid_tile=best_g[1], grid_chunk=best_g[2])
    _apply(plan, opts, trj)
    result = dict(opts, interp_ms=best_i[0], grid_ms=best_g[0], trials=len(trials))
    if cache:
        _CACHE[key] = {k: opts[k] for k in ("interp_tile", "interp_chunk", "grid_tile", "grid_chunk")}
    return dict(result, cached=False)
