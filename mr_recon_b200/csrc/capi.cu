// extern "C" entry points of libmrnufft.so (declared in include/mrnufft.h).
#include <cmath>

#include "common.cuh"
#include "internal.cuh"

using namespace mrn;

namespace mrn {
int launch_cg_init(mrn_plan* P, const float2* b, const float2* Ab, float2* x, float2* r, float2* p,
                   double* state, double tol, cudaStream_t st);
int launch_cg_step(mrn_plan* P, float2* x, float2* r, const float2* p, const float2* Ap,
                   double* state, cudaStream_t st);
int launch_cg_dir(mrn_plan* P, const float2* r, float2* p, double* state, cudaStream_t st);
int launch_cg_dot(mrn_plan* P, const float2* a, const float2* b, double* out, cudaStream_t st);
}  // namespace mrn

#define RK(x)                    \
  do {                           \
    int _r = (x);                \
    if (_r != MRN_OK) return _r; \
  } while (0)

static inline float inv_wd(const mrn_plan* P) {
  double w = 1.0;
  for (int i = 0; i < P->ndim; ++i) w *= P->width[i];
  return (float)(1.0 / w);
}

static int check_ready(const mrn_plan* P, bool need_fft) {
  if (!P) return MRN_ERR_ARG;
  if (!P->traj_set) return MRN_ERR_STATE;
  if (need_fft && (P->flags & MRN_PLAN_RAW)) return MRN_ERR_UNSUPPORTED;
  return MRN_OK;
}

#define ST(s) ((cudaStream_t)(s))

extern "C" {

int mrn_forward(mrn_plan* P, const void* img, void* ksp, void* s) {
  RK(check_ready(P, true));
  if (!img || !ksp) return MRN_ERR_ARG;
  RK(fwd_transform(P, kPrePlain, (const float2*)img, nullptr, 1.0f, ST(s)));
  StageTimer t(P, kStageInterp, ST(s));
  return launch_interp(P, P->d_grid, kInternal, (float2*)ksp, inv_wd(P), nullptr, ST(s));
}

int mrn_adjoint(mrn_plan* P, const void* ksp, void* img, void* s) {
  RK(check_ready(P, true));
  if (!img || !ksp) return MRN_ERR_ARG;
  { StageTimer t(P, kStageGrid, ST(s)); RK(launch_grid(P, (const float2*)ksp, nullptr, kInternal, P->d_grid, inv_wd(P), ST(s))); }
  return inv_transform(P, (float2*)img, ST(s));
}

int mrn_forward_ft(mrn_plan* P, const void* img, void* grid, void* s) {
  if (!P || !img || !grid) return MRN_ERR_ARG;
  if (P->flags & MRN_PLAN_RAW) return MRN_ERR_UNSUPPORTED;
  RK(fwd_transform(P, kPrePlain, (const float2*)img, nullptr, 1.0f, ST(s)));
  StageTimer t(P, kStageShift, ST(s));
  return launch_shift_copy(P, P->d_grid, (float2*)grid, 1, ST(s));
}

int mrn_interp(mrn_plan* P, const void* grid, void* ksp, float scale, void* s) {
  RK(check_ready(P, false));
  if (!grid || !ksp) return MRN_ERR_ARG;
  StageTimer t(P, kStageInterp, ST(s));
  return launch_interp(P, (const float2*)grid, kUser, (float2*)ksp, scale, nullptr, ST(s));
}

int mrn_grid(mrn_plan* P, const void* ksp, void* grid, float scale, void* s) {
  RK(check_ready(P, false));
  if (!grid || !ksp) return MRN_ERR_ARG;
  StageTimer t(P, kStageGrid, ST(s));
  return launch_grid(P, (const float2*)ksp, nullptr, kUser, (float2*)grid, scale, ST(s));
}

int mrn_adjoint_ift(mrn_plan* P, const void* grid, void* img, void* s) {
  if (!P || !img || !grid) return MRN_ERR_ARG;
  if (P->flags & MRN_PLAN_RAW) return MRN_ERR_UNSUPPORTED;
  { StageTimer t(P, kStageShift, ST(s)); RK(launch_shift_copy(P, (const float2*)grid, P->d_grid, 0, ST(s))); }
  return inv_transform(P, (float2*)img, ST(s));
}

int mrn_traj_grad(mrn_plan* P, const void* grid, const void* samples, float* grad, float scale,
                  void* s) {
  RK(check_ready(P, false));
  if (!grid || !samples || !grad) return MRN_ERR_ARG;
  StageTimer t(P, kStageTrajGrad, ST(s));
  return launch_traj_grad(P, (const float2*)grid, kUser, (const float2*)samples, grad, scale, ST(s));
}

int mrn_sense_forward(mrn_plan* P, const void* x, const void* mps, void* ksp, void* s) {
  RK(check_ready(P, true));
  if (!x || !mps || !ksp) return MRN_ERR_ARG;
  RK(fwd_transform(P, kPreSense, (const float2*)x, (const float2*)mps, 1.0f, ST(s)));
  StageTimer t(P, kStageInterp, ST(s));
  return launch_interp(P, P->d_grid, kInternal, (float2*)ksp, inv_wd(P), nullptr, ST(s));
}

int mrn_sense_adjoint(mrn_plan* P, const void* ksp, const float* dcf, const void* mps, void* x,
                      float out_scale, void* s) {
  RK(check_ready(P, true));
  if (!x || !mps || !ksp) return MRN_ERR_ARG;
  { StageTimer t(P, kStageGrid, ST(s)); RK(launch_grid(P, (const float2*)ksp, dcf, kInternal, P->d_grid, inv_wd(P), ST(s))); }
  RK(inv_transform(P, nullptr, ST(s)));
  StageTimer t(P, kStagePost, ST(s));
  return launch_post(P, kPostSense, (const float2*)mps, (float2*)x, out_scale, nullptr, 0.f, nullptr,
                     0, ST(s));
}

int mrn_sense_normal(mrn_plan* P, const void* x, const void* mps, const float* dcf, void* out,
                     float out_scale, float lam, double* pap, int pap_stride, void* s) {
  RK(check_ready(P, true));
  if (!x || !mps || !out) return MRN_ERR_ARG;
  RK(fwd_transform(P, kPreSense, (const float2*)x, (const float2*)mps, 1.0f, ST(s)));
  if (ent_path_ok(P)) {
    // 2D: the samples between the two stages in gridding-entry order, with the
    // density weight applied by the interpolation (the same products, so the
    // same bits as the sample-order path)
    const EntIO eio{P->d_ent_of, dcf, P->max_coil, 0};
    { StageTimer t(P, kStageInterp, ST(s)); RK(launch_interp_reg(P, P->d_grid, kInternal, P->d_ksp_ent, inv_wd(P), nullptr, ST(s), eio)); }
    {
      StageTimer t(P, kStageGrid, ST(s));
      if (P->n_items_grid > 0) {
        RK(launch_grid_reg(P, P->d_ksp_ent, nullptr, nullptr, kInternal, P->d_grid, inv_wd(P), ST(s), P->max_coil));
        RK(launch_reduce_split(P, kInternal, P->d_grid, ST(s)));
      }
    }
  } else {
    { StageTimer t(P, kStageInterp, ST(s)); RK(launch_interp(P, P->d_grid, kInternal, P->d_ksp_tmp, inv_wd(P), nullptr, ST(s))); }
    { StageTimer t(P, kStageGrid, ST(s)); RK(launch_grid(P, P->d_ksp_tmp, dcf, kInternal, P->d_grid, inv_wd(P), ST(s))); }
  }
  RK(inv_transform(P, nullptr, ST(s)));
  StageTimer t(P, kStagePost, ST(s));
  return launch_post(P, kPostSense, (const float2*)mps, (float2*)out, out_scale, (const float2*)x,
                     lam, pap, pap_stride, ST(s));
}

int mrn_cg_init(mrn_plan* P, const void* b, const void* Ab, void* x, void* r, void* p,
                double* state, double tol, void* s) {
  if (!P || !b || !Ab || !x || !r || !p || !state) return MRN_ERR_ARG;
  StageTimer t(P, kStageCg, ST(s));
  return launch_cg_init(P, (const float2*)b, (const float2*)Ab, (float2*)x, (float2*)r, (float2*)p,
                        state, tol, ST(s));
}

int mrn_cg_step(mrn_plan* P, void* x, void* r, const void* p, const void* Ap, double* state,
                void* s) {
  if (!P || !x || !r || !p || !Ap || !state) return MRN_ERR_ARG;
  StageTimer t(P, kStageCg, ST(s));
  return launch_cg_step(P, (float2*)x, (float2*)r, (const float2*)p, (const float2*)Ap, state, ST(s));
}

int mrn_cg_dir(mrn_plan* P, const void* r, void* p, double* state, void* s) {
  if (!P || !r || !p || !state) return MRN_ERR_ARG;
  StageTimer t(P, kStageCg, ST(s));
  return launch_cg_dir(P, (const float2*)r, (float2*)p, state, ST(s));
}

int mrn_cg_dot(mrn_plan* P, const void* a, const void* b, double* out, void* s) {
  if (!P || !a || !b || !out) return MRN_ERR_ARG;
  return launch_cg_dot(P, (const float2*)a, (const float2*)b, out, ST(s));
}

}  // extern "C"
