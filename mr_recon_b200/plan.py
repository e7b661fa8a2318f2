"""Python handle of an mrnufft plan (include/mrnufft.h): geometry of one or
more NUFFT slices, the bound trajectory, and typed calls into the C ABI."""

from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr


def _as_arr(vals, ctype):
    arr = (ctype * len(vals))(*vals)
    return arr


class Plan:
    """A batch of ``len(im_sizes)`` independent NUFFT problems (slices) that
    share dimension, kernel width, oversampling and beta. A raw plan also
    takes one beta per dimension (a sequence), as sigpy's gridding does."""

    def __init__(self, im_sizes: Sequence[Sequence[int]], n_pts: Sequence[int],
                 n_coil: Sequence[int], oversamp: float, width: Sequence[float],
                 beta: Optional[float] = None, raw: bool = False, apodize: bool = True,
                 tile: Optional[Sequence[int]] = None, coil_group: int = 0, max_chunk: int = 0,
                 device: Optional[torch.device] = None, fast: bool = True, warp_grid: bool = True,
                 weight_tables: bool = False, reg_grid: bool = True,
                 reg_interp: bool = True):
        lib = _lib.load()
        self.lib = lib
        self.ndim = len(im_sizes[0])
        self.nslices = len(im_sizes)
        self.im_sizes = [tuple(int(v) for v in s) for s in im_sizes]
        self.n_pts = [int(m) for m in n_pts]
        self.n_coil = [int(c) for c in n_coil]
        self.oversamp = float(oversamp)
        self.width = tuple(float(w) for w in width)
        self.raw = raw
        dev = torch.device("cuda") if device is None else torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("mr_recon_b200 plans live on a CUDA device (no CPU fallback)")
        self.device = torch.device("cuda", dev.index if dev.index is not None else torch.cuda.current_device())
        flags = (_lib.MRN_PLAN_RAW if raw else 0) | (0 if apodize else _lib.MRN_PLAN_NO_APOD)
        beta_d = None
        if beta is not None and not isinstance(beta, (int, float)):
            beta_d = [float(b) for b in beta]
            if len(beta_d) != self.ndim:
                raise ValueError(f"beta per dimension needs {self.ndim} values, got {len(beta_d)}")
            if not raw:
                raise ValueError("beta per dimension is for raw (gridding) plans")
            beta = beta_d[0]
        flat = [v for s in self.im_sizes for v in s]
        h = C.c_void_p()
        rc = lib.mrn_plan_create(
            C.byref(h), self.ndim, self.nslices, _as_arr(flat, C.c_int),
            _as_arr(self.n_pts, C.c_int64), _as_arr(self.n_coil, C.c_int), float(oversamp),
            _as_arr(list(self.width), C.c_double), float(beta) if beta is not None else -1.0,
            flags, _as_arr(list(tile), C.c_int) if tile is not None else None,
            int(coil_group), int(max_chunk), self.device.index)
        check(rc, "mrn_plan_create")
        self.handle = h
        if beta_d is not None:
            check(lib.mrn_plan_set_beta(h, _as_arr(beta_d, C.c_double)), "mrn_plan_set_beta")
        check(lib.mrn_plan_set_option(h, _lib.MRN_OPT_FAST_KERNELS, 1 if fast else 0), "mrn_plan_set_option")
        check(lib.mrn_plan_set_option(h, _lib.MRN_OPT_WARP_GRIDDING, 1 if warp_grid else 0),
              "mrn_plan_set_option")
        check(lib.mrn_plan_set_option(h, _lib.MRN_OPT_WEIGHT_TABLES, 1 if weight_tables else 0),
              "mrn_plan_set_option")
        check(lib.mrn_plan_set_option(h, _lib.MRN_OPT_REG_GRIDDING, 1 if reg_grid else 0),
              "mrn_plan_set_option")
        check(lib.mrn_plan_set_option(h, _lib.MRN_OPT_REG_INTERP, 1 if reg_interp else 0),
              "mrn_plan_set_option")
        n = self.nslices
        offs = [(C.c_int64 * n)() for _ in range(4)]
        check(lib.mrn_plan_offsets(h, *offs), "mrn_plan_offsets")
        self.img_off, self.ksp_off, self.grid_off, self.trj_off = (np.array(o[:], dtype=np.int64) for o in offs)
        sz = (C.c_int64 * 8)()
        check(lib.mrn_plan_sizes(h, sz), "mrn_plan_sizes")
        self.n_img, self.n_ksp, self.n_grid, self.n_trj, self.n_tiles = (int(v) for v in sz[:5])
        self.os_sizes = [tuple(s if raw else int(math.ceil(oversamp * s)) for s in im) for im in self.im_sizes]
        self.traj_bound = False

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.mrn_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ------------------------------------------------------------------
    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def set_traj(self, trj: torch.Tensor) -> None:
        _lib.require_cuda(trj, "trajectory")
        t = trj.detach().to(torch.float32).contiguous()
        if t.numel() != self.n_trj:
            raise ValueError(f"trajectory has {t.numel()} values, plan expects {self.n_trj}")
        with torch.cuda.device(self.device):
            check(self.lib.mrn_plan_set_traj(self.handle, ptr(t), self.stream()), "mrn_plan_set_traj")
        self.traj_bound = True

    def stats(self):
        o = (C.c_int64 * 4)()
        check(self.lib.mrn_plan_stats(self.handle, o))
        return {"interp_items": o[0], "grid_items": o[1], "grid_entries": o[2], "split_tiles": o[3]}

    @property
    def fft_kind(self) -> int:
        """mrn_plan_fft_kind: 0 cuFFT, 1 the native per-axis FFT passes for
        every grid size, 2 native for some grid sizes only."""
        r = self.lib.mrn_plan_fft_kind(self.handle)
        check(min(r, 0))
        return r

    def set_option(self, option: int, value: int) -> None:
        """mrn_plan_set_option. Chunk and tile options take effect at the next
        set_traj (the trajectory is unbound until then)."""
        check(self.lib.mrn_plan_set_option(self.handle, int(option), int(value)), "mrn_plan_set_option")
        if option in (_lib.MRN_OPT_INTERP_CHUNK, _lib.MRN_OPT_GRID_CHUNK, _lib.MRN_OPT_INTERP_TILE,
                      _lib.MRN_OPT_GRID_TILE):
            self.traj_bound = False

    STAGES = ("pre", "fft", "interp", "grid", "post", "layout_copy", "traj_grad", "cg")

    def enable_timing(self, on: bool = True) -> None:
        check(self.lib.mrn_plan_enable_timing(self.handle, 1 if on else 0))

    def timing(self):
        """Per-stage (total ms, launches) recorded since the last call."""
        ms = (C.c_double * 8)()
        cnt = (C.c_int64 * 8)()
        check(self.lib.mrn_plan_timing(self.handle, ms, cnt))
        return {s: (ms[i], cnt[i]) for i, s in enumerate(self.STAGES)}

    # ------------------------------------------------------------------
    def _call(self, name, *args):
        with torch.cuda.device(self.device):
            check(getattr(self.lib, name)(self.handle, *args, self.stream()), name)

    def forward(self, img, ksp):
        self._call("mrn_forward", ptr(img), ptr(ksp))

    def adjoint(self, ksp, img):
        self._call("mrn_adjoint", ptr(ksp), ptr(img))

    def forward_ft(self, img, grid):
        self._call("mrn_forward_ft", ptr(img), ptr(grid))

    def interp(self, grid, ksp, scale=1.0):
        self._call("mrn_interp", ptr(grid), ptr(ksp), float(scale))

    def grid(self, ksp, grid, scale=1.0):
        self._call("mrn_grid", ptr(ksp), ptr(grid), float(scale))

    def adjoint_ift(self, grid, img):
        self._call("mrn_adjoint_ift", ptr(grid), ptr(img))

    def traj_grad(self, grid, samples, out, scale=1.0):
        self._call("mrn_traj_grad", ptr(grid), ptr(samples), ptr(out), float(scale))

    def sense_forward(self, x, mps, ksp):
        self._call("mrn_sense_forward", ptr(x), ptr(mps), ptr(ksp))

    def sense_adjoint(self, ksp, dcf, mps, x, out_scale=1.0):
        self._call("mrn_sense_adjoint", ptr(ksp), ptr(dcf), ptr(mps), ptr(x), float(out_scale))

    def sense_normal(self, x, mps, dcf, out, out_scale=1.0, lam=0.0, pap=None, pap_stride=1):
        self._call("mrn_sense_normal", ptr(x), ptr(mps), ptr(dcf), ptr(out), float(out_scale),
                   float(lam), ptr(pap), int(pap_stride))

    def lr_forward(self, x, mps, w, ksp):
        """Low-rank forward: ksp = sum_j w[j] * NUFFT_j(mps[j] x[j]) (mrn_lr_forward)."""
        self._call("mrn_lr_forward", ptr(x), ptr(mps), ptr(w), ptr(ksp))

    def lr_adjoint(self, ksp, w, mps, x, out_scale=1.0):
        """Low-rank adjoint: x[j] = sum_c conj(mps[j][c]) NUFFT_j^H(conj(w[j]) ksp[c])."""
        self._call("mrn_lr_adjoint", ptr(ksp), ptr(w), ptr(mps), ptr(x), float(out_scale))

    def lr_normal(self, x, mps, w_fwd, w_adj, out, out_scale=1.0, lam=0.0):
        self._call("mrn_lr_normal", ptr(x), ptr(mps), ptr(w_fwd), ptr(w_adj), ptr(out),
                   float(out_scale), float(lam))

    def set_toeplitz(self, kern: torch.Tensor, pad_sizes) -> None:
        """Bind Toeplitz kernels (calc_teoplitz_kernels' output, per slice on
        the padded grid pad_sizes[s], slices back to back); see mrn_plan_set_toeplitz."""
        _lib.require_cuda(kern, "Toeplitz kernel")
        k = kern.detach().to(torch.complex64).contiguous()
        ps = [int(v) for s in pad_sizes for v in s]
        if k.numel() != sum(int(torch.tensor(s).prod()) for s in pad_sizes):
            raise ValueError("Toeplitz kernel size does not match the padded grids")
        arr = (C.c_int * len(ps))(*ps)
        with torch.cuda.device(self.device):
            check(self.lib.mrn_plan_set_toeplitz(self.handle, arr, ptr(k), self.stream()),
                  "mrn_plan_set_toeplitz")
        self.toeplitz_pad = [tuple(s) for s in pad_sizes]

    def toeplitz_normal(self, img, out):
        self._call("mrn_toeplitz_normal", ptr(img), ptr(out))

    def sense_normal_toeplitz(self, x, mps, out, out_scale=1.0, lam=0.0, pap=None, pap_stride=1):
        self._call("mrn_sense_normal_toeplitz", ptr(x), ptr(mps), ptr(out), float(out_scale), float(lam),
                   ptr(pap), int(pap_stride))

    def cg_init(self, b, Ab, x, r, p, state, tol):
        self._call("mrn_cg_init", ptr(b), ptr(Ab), ptr(x), ptr(r), ptr(p), ptr(state), float(tol))

    def cg_step(self, x, r, p, Ap, state):
        self._call("mrn_cg_step", ptr(x), ptr(r), ptr(p), ptr(Ap), ptr(state))

    def cg_dir(self, r, p, state):
        self._call("mrn_cg_dir", ptr(r), ptr(p), ptr(state))

    def cg_dot(self, a, b, out):
        self._call("mrn_cg_dot", ptr(a), ptr(b), ptr(out))


class PlanCache:
    """Small LRU of plans keyed by geometry and trajectory identity. Entries
    hold a reference to their trajectory tensor, so its storage cannot be
    freed and reused by another tensor while the binned plan is cached; an
    in-place change to the trajectory bumps its version and misses."""

    def __init__(self, capacity: int = 4):
        self.capacity = capacity
        self.entries = []  # (key, trj_ref, plan)

    def get(self, key, trj, make):
        for i, (k, tref, plan) in enumerate(self.entries):
            if k == key:
                self.entries.append(self.entries.pop(i))
                return plan
        plan = make()
        self.entries.append((key, trj, plan))
        while len(self.entries) > self.capacity:
            self.entries.pop(0)
        return plan

    def clear(self):
        self.entries.clear()


def traj_key(trj: Optional[torch.Tensor]):
    if trj is None:
        return None
    return (trj.data_ptr(), trj._version, tuple(trj.shape), str(trj.device), trj.dtype)
