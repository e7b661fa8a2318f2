// Low-rank SENSE operators: time-segmented off-resonance models with general
// (e.g. least-squares) temporal interpolators and subspace models.
//
// Reference: sense_linop.forward / adjoint with spatial_funcs b_l and
// temporal_funcs h_l (linops.py:1134-1228) and subspace_linop
// (linops.py:1496-1772) loop over segments and subspace coefficients in
// Python, calling the NUFFT on (C, L, ...) batches and combining the results
// with elementwise torch products and sums. Here every component j (a
// segment, or a (coefficient, segment) pair) is one slice of an uneven
// multi-slice plan whose slices share the trajectory, coil count and sample
// count; a slice's image is the component image (b_l times the coefficient
// volume). Then
//   forward: ksp[c][t] = sum_j w[j][t] NUFFT_j(mps[c] x_j)[t]
//            one pre / FFT / interpolation pass over all components into the
//            plan's sample scratch, then k_lr_combine sums the components in
//            component order with their weights (no per-component torch pass);
//   adjoint: x_j = s sum_c conj(mps[c]) NUFFT_j^H(conj(w[j]) ksp[c])
//            the gridding reads the one shared k-space block for every
//            component (the slice table with all k-space offsets 0) and
//            multiplies each staged sample by conj(w[j][t]) in its prologue,
//            so the J weighted copies of the k-space are never written.
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace mrn {
namespace {

// out[c][t] = sum_j w[j][t] tmp[j][c][t], j in order (fixed summation order).
// out may be tmp's component-0 block (each element is read for every
// component before its one write), so neither pointer is restrict.
__global__ void k_lr_combine(const float2* tmp, const float2* __restrict__ w, int nj, int ncoil,
                             int64_t m, float2* out) {
  const int64_t n = (int64_t)ncoil * m;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = i % m;
    float2 acc = make_float2(0.f, 0.f);
    for (int j = 0; j < nj; ++j) {
      const float2 a = tmp[(int64_t)j * n + i];
      const float2 b = w[(int64_t)j * m + t];
      acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
      acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
    }
    out[i] = acc;
  }
}

// Every component slice must share the coil count and sample count (the
// shared k-space block is [C][M]).
int check_lowrank(const mrn_plan* P) {
  if (!P) return MRN_ERR_ARG;
  if (!P->traj_set) return MRN_ERR_STATE;
  if (P->flags & MRN_PLAN_RAW) return MRN_ERR_UNSUPPORTED;
  const SliceGeom& g0 = P->h_slices[0];
  for (const SliceGeom& g : P->h_slices)
    if (g.ncoil != g0.ncoil || g.m != g0.m) return MRN_ERR_ARG;
  return MRN_OK;
}

float inv_width_prod(const mrn_plan* P) {
  double w = 1.0;
  for (int i = 0; i < P->ndim; ++i) w *= P->width[i];
  return (float)(1.0 / w);
}

int lr_combine(mrn_plan* P, const float2* w, float2* out, cudaStream_t st) {
  const SliceGeom& g0 = P->h_slices[0];
  const int64_t n = (int64_t)g0.ncoil * g0.m;
  if (n == 0) return MRN_OK;
  const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)P->sm_count * 16);
  k_lr_combine<<<blocks, 256, 0, st>>>(P->d_ksp_tmp, w, P->nslices, g0.ncoil, g0.m, out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

// Gridding of the shared k-space block into every component's grid, each
// sample times conj(w[j][t]).
int lr_grid(mrn_plan* P, const float2* ksp, const float2* w, cudaStream_t st) {
  SliceGeom* own = P->d_slices;
  P->d_slices = P->d_slices_kshared;
  const int rc = launch_grid_t(P, ksp, nullptr, w, kInternal, P->d_grid, inv_width_prod(P), st);
  P->d_slices = own;
  return rc;
}

}  // namespace
}  // namespace mrn

using namespace mrn;

#define RK(x)                    \
  do {                           \
    int _r = (x);                \
    if (_r != MRN_OK) return _r; \
  } while (0)
#define ST(s) ((cudaStream_t)(s))

extern "C" {

int mrn_lr_forward(mrn_plan* P, const void* x, const void* mps, const void* w, void* ksp, void* s) {
  RK(check_lowrank(P));
  if (!x || !mps || !w || !ksp) return MRN_ERR_ARG;
  RK(fwd_transform(P, kPreSense, (const float2*)x, (const float2*)mps, 1.0f, ST(s)));
  StageTimer t(P, kStageInterp, ST(s));
  RK(launch_interp(P, P->d_grid, kInternal, P->d_ksp_tmp, inv_width_prod(P), nullptr, ST(s)));
  return lr_combine(P, (const float2*)w, (float2*)ksp, ST(s));
}

int mrn_lr_adjoint(mrn_plan* P, const void* ksp, const void* w, const void* mps, void* x,
                   float out_scale, void* s) {
  RK(check_lowrank(P));
  if (!ksp || !w || !mps || !x) return MRN_ERR_ARG;
  { StageTimer t(P, kStageGrid, ST(s)); RK(lr_grid(P, (const float2*)ksp, (const float2*)w, ST(s))); }
  RK(inv_transform(P, nullptr, ST(s)));
  StageTimer t(P, kStagePost, ST(s));
  return launch_post(P, kPostSense, (const float2*)mps, (float2*)x, out_scale, nullptr, 0.f, nullptr, 0,
                     ST(s));
}

int mrn_lr_normal(mrn_plan* P, const void* x, const void* mps, const void* w_fwd, const void* w_adj,
                  void* out, float out_scale, float lam, void* s) {
  RK(check_lowrank(P));
  if (!x || !mps || !w_fwd || !w_adj || !out) return MRN_ERR_ARG;
  RK(fwd_transform(P, kPreSense, (const float2*)x, (const float2*)mps, 1.0f, ST(s)));
  {
    // the combined samples overwrite component 0's block of the scratch
    StageTimer t(P, kStageInterp, ST(s));
    RK(launch_interp(P, P->d_grid, kInternal, P->d_ksp_tmp, inv_width_prod(P), nullptr, ST(s)));
    RK(lr_combine(P, (const float2*)w_fwd, P->d_ksp_tmp, ST(s)));
  }
  { StageTimer t(P, kStageGrid, ST(s)); RK(lr_grid(P, P->d_ksp_tmp, (const float2*)w_adj, ST(s))); }
  RK(inv_transform(P, nullptr, ST(s)));
  StageTimer t(P, kStagePost, ST(s));
  return launch_post(P, kPostSense, (const float2*)mps, (float2*)out, out_scale, (const float2*)x, lam,
                     nullptr, 0, ST(s));
}

}  // extern "C"
