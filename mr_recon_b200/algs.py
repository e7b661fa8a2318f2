"""Iterative algorithms with the interface of mr_recon's algs.py.

``conjugate_gradient`` (algs.py:779-872), ``power_method_operator``
(algs.py:364-400), ``FISTA`` (algs.py:655-729) and ``gradient_descent``
(algs.py:731-777) keep the reference signatures and iteration semantics. Dot
products and norms are accumulated in float64 and the CG scalars stay on the
device: the reference's per-iteration ``.item()`` host sync (algs.py:845) and
early ``break`` become a device-side "done" mask that freezes the iterate at
the same point, so results match while the loop never waits on the host.

``SenseCG`` is the fused device CG for a ``sense_linop`` on the B200 NUFFT:
every step is a kernel of libmrnufft.so and a whole solve can be captured in
one CUDA graph.
"""

from __future__ import annotations

from typing import Callable, Optional, Tuple

import torch
from tqdm import tqdm

complex_dtype = torch.complex64

__all__ = ["conjugate_gradient", "power_method_operator", "FISTA", "gradient_descent", "SenseCG",
           "density_compensation"]


def _as_f64(a: torch.Tensor) -> torch.Tensor:
    if a.is_complex():
        return torch.view_as_real(a.to(torch.complex128).contiguous())
    return a.to(torch.float64)


def _rdot(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Re <a, b> = Re sum conj(a) b, in float64 (0-dim device tensor)."""
    return (_as_f64(a) * _as_f64(b)).sum()


def conjugate_gradient(AHA: Callable, AHb: torch.Tensor, P: Optional[Callable] = None,
                       num_iters: Optional[int] = 10, lamda_l2: Optional[float] = 0.0,
                       tolerance: Optional[float] = 1e-8, return_resids: Optional[bool] = False,
                       weights: Optional[torch.Tensor] = None, verbose=True) -> torch.Tensor:
    """Complex CG for (AHA + lamda_l2 I) x = AHb starting at x0 = AHb
    (algs.py:779-872): vectors in AHb's dtype, dot products and norms in
    float64, and no host synchronisation per iteration (the stop test is a
    device-side mask, where the reference calls .item() and breaks)."""
    if P is None:
        P = lambda x: x  # noqa: E731
    if weights is not None:
        op = lambda x: AHA(x) + lamda_l2 * weights * x  # noqa: E731
    else:
        op = lambda x: AHA(x) + lamda_l2 * x  # noqa: E731
    x0 = AHb.clone()
    if num_iters == 0:
        return x0
    r = AHb - op(x0)
    z = P(r)
    p = z.clone()
    done = torch.zeros((), dtype=torch.bool, device=AHb.device)
    real = x0.real.dtype if x0.is_complex() else x0.dtype
    if return_resids:
        resids = []
        xs = [x0.clone()]
    for _ in tqdm(range(num_iters), "CG Iterations", disable=not verbose):
        Ap = op(p)
        pAp = _rdot(p, Ap)
        rz = _rdot(r, z)
        alpha = torch.where(done, torch.zeros_like(rz), rz / pAp).to(real)
        x0 = x0 + alpha * p
        r = r - alpha * Ap
        rr = _rdot(r, r)
        rnrm = rr.sqrt()
        if return_resids:
            resids.append(rnrm.item())
            xs.append(x0.clone())
        done = done | (rnrm < tolerance)
        z = P(r)
        beta = torch.where(done, torch.zeros_like(rz), _rdot(r, z) / rz).to(real)
        p = torch.where(done, p, z + beta * p)
    if return_resids:
        return resids, xs
    return x0


def power_method_operator(A: Callable, x0: torch.Tensor, num_iter: Optional[int] = 15,
                          verbose: Optional[bool] = True) -> Tuple[torch.Tensor, float]:
    """Largest eigenvalue of A by the power method (algs.py:364-400)."""
    ll = None
    for _ in tqdm(range(num_iter), "Max Eigenvalue", disable=not verbose):
        z = A(x0)
        ll = torch.linalg.vector_norm(z.to(torch.complex128))
        x0 = (z / ll).to(z.dtype)
    if verbose:
        print(f"Max Eigenvalue = {ll}")
    return x0, ll.item()


def FISTA(AHA: Callable, AHb: torch.Tensor, proxg: Callable, num_iters: Optional[int] = 20,
          ptol_exit: Optional[float] = 0.5, return_ptols: Optional[bool] = False,
          return_xs: Optional[bool] = False, x0: Optional[torch.Tensor] = None,
          verbose: Optional[bool] = True) -> torch.Tensor:
    """FISTA for ||Ax - b||^2 + g(x) (algs.py:655-729)."""
    x = AHb.clone() if x0 is None else x0
    z = x.clone()
    if num_iters <= 0:
        return x
    ptols = []
    xs = []
    for k in tqdm(range(num_iters), "FISTA Iterations", disable=not verbose):
        x_old = x.clone()
        x = z.clone()
        gr = AHA(x) - AHb
        x = proxg(x - gr)
        if k == 0:
            z = x
        else:
            step = k / (k + 3)
            z = x + step * (x - x_old)
        ptol = 100 * torch.linalg.vector_norm(x_old - x) / torch.linalg.vector_norm(x)
        ptols.append(ptol.item())
        if ptol < ptol_exit:
            if verbose:
                print(f"Tolerance reached after {k + 1} iterations, exiting FISTA")
            break
        if return_xs:
            xs.append(x.clone())
    if return_ptols:
        return ptols, x
    if return_xs:
        return xs, x
    return x


def gradient_descent(AHA: Callable, AHb: torch.Tensor, lr: float, num_iters: Optional[int] = 100,
                     lamda_l2: Optional[float] = 0.0, tolerance: Optional[float] = 1e-8,
                     return_resids: Optional[bool] = False, verbose: Optional[bool] = True):
    """Gradient descent on (AHA + lamda_l2 I) x = AHb (algs.py:731-777)."""
    x = AHb
    op = lambda v: AHA(v) + lamda_l2 * v  # noqa: E731
    resids = []
    for _ in tqdm(range(num_iters), "GD Iterations", disable=not verbose):
        grad = op(x) - AHb
        x = x - lr * grad
        nrm = torch.linalg.vector_norm(grad)
        resids.append(nrm.item())
        if nrm < tolerance:
            break
    if return_resids:
        return resids, x
    return x


class SenseCG:
    """CG-SENSE (recons.py:77-156 with max_eigen given) on a fused plan: one
    image per slice, every slice of the plan solved at once: complex64
    vectors, float64 dot products and norms summed in a fixed order. All
    scalars stay on the device (float64 state per slice), so ``capture()``
    can record the whole solve -- AHb, initial residual and ``max_iter``
    iterations -- in one CUDA graph, replayed by ``solve`` with the same bits
    as the eager solve.

    plan     : mr_recon_b200.plan.Plan with the trajectory bound
    mps      : coil maps, plan image layout (all slices back to back)
    dcf      : float32 [total samples] or None
    """

    def __init__(self, plan, mps: torch.Tensor, dcf: Optional[torch.Tensor], max_iter: int,
                 lamda_l2: float, max_eigen, tolerance: float = 1e-8, toeplitz: bool = False):
        self.plan = plan
        # normal operator: the Toeplitz one bound to the plan (FFT-only), or the NUFFT's
        self.toeplitz = bool(toeplitz)
        if self.toeplitz and getattr(plan, "toeplitz_pad", None) is None:
            raise ValueError("SenseCG(toeplitz=True) needs Toeplitz kernels bound to the plan")
        self.mps = mps
        self.dcf = dcf
        self.max_iter = int(max_iter)
        self.lam = float(lamda_l2)
        n = plan.nslices
        dev = plan.device
        me = torch.as_tensor(max_eigen, dtype=torch.float64).reshape(-1)
        if me.numel() != 1:
            raise ValueError("SenseCG takes one max_eigen for all slices")
        self.max_eigen = float(me[0])
        self.tol = float(tolerance)
        nx = sum(int(torch.tensor(s).prod()) for s in plan.im_sizes)
        mk = lambda: torch.zeros(nx, dtype=complex_dtype, device=dev)  # noqa: E731
        self.b, self.x, self.r, self.p, self.Ap = mk(), mk(), mk(), mk(), mk()
        self.state = torch.zeros(n * 8, dtype=torch.float64, device=dev)
        self.ksp = torch.zeros(plan.n_ksp, dtype=complex_dtype, device=dev)
        self.graph = None

    def _run(self):
        pl = self.plan
        s_adj = 1.0 / self.max_eigen ** 0.5
        s_nrm = 1.0 / self.max_eigen
        pl.sense_adjoint(self.ksp, self.dcf, self.mps, self.b, s_adj)
        if self.max_iter == 0:
            self.x.copy_(self.b)
            return
        if self.toeplitz:
            normal = lambda v, out, *a: pl.sense_normal_toeplitz(v, self.mps, out, *a)  # noqa: E731
        else:
            normal = lambda v, out, *a: pl.sense_normal(v, self.mps, self.dcf, out, *a)  # noqa: E731
        normal(self.b, self.Ap, s_nrm, self.lam)
        pl.cg_init(self.b, self.Ap, self.x, self.r, self.p, self.state, self.tol)
        pap = self.state[1:]
        for _ in range(self.max_iter):
            normal(self.p, self.Ap, s_nrm, self.lam, pap, 8)
            pl.cg_step(self.x, self.r, self.p, self.Ap, self.state)
            pl.cg_dir(self.r, self.p, self.state)

    def capture(self):
        """Record one full solve in a CUDA graph (after a warm-up run)."""
        s = torch.cuda.Stream(self.plan.device)
        s.wait_stream(torch.cuda.current_stream(self.plan.device))
        with torch.cuda.stream(s):
            self._run()
        torch.cuda.current_stream(self.plan.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._run()
        self.graph = g
        return self

    def solve(self, ksp: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Run one solve on ``ksp`` (plan k-space layout); returns x (a view
        of an internal buffer, overwritten by the next solve)."""
        if ksp is not None:
            self.ksp.copy_(ksp.reshape(-1))
        if self.graph is not None:
            self.graph.replay()
        else:
            self._run()
        return self.x

    def iterations(self) -> torch.Tensor:
        return self.state.view(-1, 8)[:, 5]


def density_compensation(trj: torch.Tensor, im_size: tuple, num_iters: Optional[int] = 30,
                         method: str = "sigpy", width: float = 4.0, beta: float = 8.0) -> torch.Tensor:
    """Pipe-Menon density compensation (algs.py:20-106), normalised to max 1.

    The reference delegates to sigpy.mri.pipe_menon_dcf (sigpy is not pinned in
    its environment.yml and not present here). This restates the published
    iteration (Pipe & Menon, MRM 41:179-186, 1999) on the B200 gridding and
    interpolation kernels: with G the Kaiser-Bessel gridding operator from the
    samples onto the image-size grid (width 4, beta 8, no oversampling, as the
    sigpy routine), w <- w / |G^H G w| for ``num_iters`` iterations, starting
    from w = 1; G^H G w then approaches 1 on every sample. The kernel's overall
    scale cancels in the final normalisation.

    trj : (..., d) in grid units, k_i in [-N_i/2, N_i/2) (CUDA tensor)
    returns (...) float32
    """
    from . import _lib
    from .plan import Plan
    if method.lower() != "sigpy":
        raise NotImplementedError("only the Pipe-Menon iteration ('sigpy') is provided")
    _lib.require_cuda(trj, "trajectory")
    d = trj.shape[-1]
    im_size = tuple(int(n) for n in im_size)
    if len(im_size) != d:
        raise ValueError(f"trajectory has {d} dims, im_size {len(im_size)}")
    tshape = trj.shape[:-1]
    locs = trj.detach().to(torch.float32).reshape(-1, d)
    locs = locs + torch.tensor([n // 2 for n in im_size], dtype=torch.float32, device=trj.device)
    M = locs.shape[0]
    plan = Plan([im_size], [M], [1], 1.0, (float(width),) * d, float(beta), raw=True, device=trj.device)
    plan.set_traj(locs.contiguous().reshape(-1))
    w = torch.ones(M, dtype=torch.complex64, device=trj.device)
    g = torch.empty(plan.n_grid, dtype=torch.complex64, device=trj.device)
    ghgw = torch.empty_like(w)
    for _ in range(int(num_iters)):
        plan.grid(w, g, 1.0)
        plan.interp(g, ghgw, 1.0)
        w = w / ghgw.abs()
    dcf = w.real.reshape(tshape)
    return dcf / dcf.max()

