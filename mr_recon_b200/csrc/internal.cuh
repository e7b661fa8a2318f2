// Internal launcher declarations (host side).
#pragma once

#include "common.cuh"

namespace mrn {

int cuda_fail(cudaError_t e);
extern thread_local int g_last_cuda_error;

// Opt a kernel into `dyn` bytes of dynamic shared memory when its static plus
// dynamic shared memory exceeds the 48 KB a launch gets without the opt-in.
// The largest opt-in per (kernel, device) is remembered, so the common launch
// costs one table lookup instead of two driver calls.
int set_dynamic_smem_fn(const void* kernel, size_t dyn);
template <class Kern>
inline int set_dynamic_smem(Kern kernel, size_t dyn) {
  return set_dynamic_smem_fn(reinterpret_cast<const void*>(kernel), dyn);
}

// Which grid layout a tile kernel reads or writes.
enum GridLayout { kInternal = 0, kUser = 1 };

// Cells of the largest gridding tile of the plan (the partial-tile slot size per coil).
inline int grid_tile_cells(const mrn_plan* P) {
  int c = 1;
  for (int i = 0; i < P->ndim; ++i) c *= P->tmax_gcells[i];
  return c;
}

// Partial-tile slots of split gridding tiles, as the gridding kernels take them.
inline SplitOut split_out(const mrn_plan* P) {
  SplitOut so;
  so.part = P->d_part;
  so.cell_cap = grid_tile_cells(P);
  so.slot_stride = (int64_t)P->max_coil * so.cell_cap;
  so.pad = 0;
  return so;
}

// Tile kernels (tiles.cu)
int launch_interp(mrn_plan* P, const float2* grid, GridLayout layout, float2* ksp, float scale,
                  const float2* temporal, cudaStream_t st);
int launch_grid(mrn_plan* P, const float2* ksp, const float* dcf, GridLayout layout, float2* grid,
                float scale, cudaStream_t st);
int launch_grid_t(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                  GridLayout layout, float2* grid, float scale, cudaStream_t st);
int launch_traj_grad(mrn_plan* P, const float2* grid, GridLayout layout, const float2* samples,
                     float* out, float scale, cudaStream_t st);

// Fast paths with compile-time tap counts (tiles_fast.cu)
bool fast_path_ok(const mrn_plan* P, bool gridding);
int launch_interp_fast(mrn_plan* P, const float2* grid, int layout, float2* ksp, float scale,
                       const float2* temporal, int cg, int G, int pstride, size_t smem, dim3 gdim,
                       cudaStream_t st);
int launch_grid_warp(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                     int layout, float2* grid, float scale, cudaStream_t st);
bool interp_reg_ok(const mrn_plan* P);
int launch_interp_reg(mrn_plan* P, const float2* grid, int layout, float2* ksp, float scale,
                      const float2* temporal, cudaStream_t st, EntIO eio = EntIO{nullptr, nullptr, 0, 0});
int launch_trajgrad_reg(mrn_plan* P, const float2* grid, int layout, const float2* samples, float* out,
                        float scale, cudaStream_t st);
bool grid_reg_ok(const mrn_plan* P);
bool grid_reg3_ok(const mrn_plan* P);
int launch_grid_reg3(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                     int layout, float2* grid, float scale, cudaStream_t st);
int launch_grid_reg(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                    int layout, float2* grid, float scale, cudaStream_t st, int ent_stride = 0);
// 2D normal operator with entry-major samples (EntIO): the entry map is bound
// and the register interpolation and gridding kernels apply
bool ent_path_ok(const mrn_plan* P);
int launch_reduce_split(mrn_plan* P, GridLayout layout, float2* grid, cudaStream_t st);
// 2D weight tables (wtab.cu)
bool wtab_applicable(const mrn_plan* P);
int build_wtabs(mrn_plan* P, cudaStream_t st);
int launch_interp_tab(mrn_plan* P, const float2* grid, int layout, float2* ksp, float scale,
                      const float2* temporal, int cg, int G, int pstride, size_t smem, dim3 gdim,
                      cudaStream_t st);
int launch_grid_warp_tab(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                         int layout, float2* grid, float scale, cudaStream_t st);
int launch_grid_fast(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                     int layout, float2* grid, float scale, int cg, int G, int pstride, size_t smem,
                     dim3 gdim, cudaStream_t st);

// FFT-stage kernels (fftstage.cu)
enum PreMode { kPrePlain = 0, kPreSense = 1 };
int launch_pre(mrn_plan* P, PreMode mode, const float2* src, const float2* mps, float scale,
               cudaStream_t st);
enum PostMode { kPostPlain = 0, kPostSense = 1 };
int launch_post(mrn_plan* P, PostMode mode, const float2* mps, float2* out, float scale,
                const float2* xin, float lam, double* pap, int pap_stride, cudaStream_t st);
int launch_shift_copy(mrn_plan* P, const float2* src, float2* dst, int to_user, cudaStream_t st);
// cuFFT of every FFT group, or (skip_native) of the groups the native passes
// do not cover.
int run_fft(mrn_plan* P, int direction, cudaStream_t st, bool skip_native = false);
// Apodize / pad and forward FFT of the plan grid (native passes when
// ffx_active, else k_pre + cuFFT), stage-timed; and the inverse FFT with the
// plain crop / deapodize into out, or (out == nullptr) leaving the grid for a
// SENSE post, which then reads only the lines that survive the crop.
int fwd_transform(mrn_plan* P, PreMode mode, const float2* src, const float2* mps, float scale,
                  cudaStream_t st);
int inv_transform(mrn_plan* P, float2* out, cudaStream_t st);

// Slice table upload (plan.cu): d_slices and its shared-k-space twin.
cudaError_t upload_slices(mrn_plan* P);

// Native FFT (ffx.cu). A grid buffer of FFT groups: per group its grid size,
// the offset of its [batch][nos...] block and its coils; FfxGrid is what the
// passes read (host and device slice tables, apodization, the buffer).
struct FfxGroupSpec {
  int nos[kMaxDim];
  int64_t grid_off;
  int batch;
};
struct FfxGrid {
  int ndim;
  const SliceGeom* hsl;
  const SliceGeom* dsl;
  const float* apod;
  float2* grid;
};
int ffx_build(FfxSet& S, int ndim, const std::vector<SliceGeom>& hsl, const std::vector<FfxGroupSpec>& spec);
int ffx_fwd(const FfxSet& S, const FfxGrid& G, PreMode mode, const float2* src, const float2* mps, float scale,
            cudaStream_t st);
int ffx_inv(const FfxSet& S, const FfxGrid& G, float2* out, float scale, cudaStream_t st);
int ffx_setup(mrn_plan* P);
int ffx_refresh(mrn_plan* P);  // slice flags after MRN_OPT_NATIVE_FFT changes
bool ffx_active(const mrn_plan* P);
int ffx_forward(mrn_plan* P, PreMode mode, const float2* src, const float2* mps, float scale, cudaStream_t st);
int ffx_inverse(mrn_plan* P, float2* out, float scale, cudaStream_t st);

// Toeplitz normal operator state (toeplitz.cu)
void toep_free(mrn_plan* P);

}  // namespace mrn
