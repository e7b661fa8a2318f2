// Internal declarations shared by the mrnufft CUDA sources (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <vector>

#include "../../include/mrnufft.h"

namespace mrn {

constexpr int kMaxDim = 3;
constexpr int kMaxTaps = 16;     // candidate taps per dim: floor(W) + 1 <= 16 -> W < 16
constexpr int kThreads = 256;    // threads per CTA of the tile kernels
constexpr int kMaxRedBlocks = 1024;  // CTAs per slice of the CG vector kernels
constexpr int kWarps = kThreads / 32;

// Geometry of one slice (one NUFFT problem) of a plan. Device-resident table.
struct SliceGeom {
  int n[kMaxDim];      // image size (1 for unused dims)
  int nos[kMaxDim];    // oversampled grid size (grid size for raw plans)
  int ntile[kMaxDim];  // interpolation tiles per dim
  int gntile[kMaxDim]; // gridding tiles per dim
  int hshift[kMaxDim]; // Nos//2: centred index j lives at storage (j - hshift) mod Nos
  int tile_base;       // first global interpolation tile id of this slice
  int gtile_base;      // first global gridding tile id of this slice
  int ncoil;           // image batch (coils)
  int64_t m;           // samples
  int64_t pt_off;      // first global point id (offset into concatenated points)
  int64_t img_off;     // complex offset of the slice image block [C][N...]
  int64_t ksp_off;     // complex offset of the slice samples [C][M]
  int64_t grid_off;    // complex offset in the plan's internal grid buffer
  int64_t ugrid_off;   // complex offset in a caller grid buffer (slice order)
  int64_t x_off;       // complex offset of a one-image-per-slice vector [N...]
  int64_t gos;         // prod(nos)
  int64_t nimg;        // prod(n)
  float scale[kMaxDim];  // trajectory scale ceil(os N)/N (1 for raw)
  float shift[kMaxDim];  // trajectory shift ceil(os N)//2 (0 for raw)
  int apod_off[kMaxDim]; // offset of this slice's apodization table per dim
  int64_t prow_off;      // first grid row (all dims but the last, all coils) of the slice
  int64_t irow_off;      // first image row (all coils) of the slice
  int64_t xrow_off;      // first image row of the one-image-per-slice layout
  float inv_sqrt_n;      // 1 / sqrt(prod(n)) (fourier.py:462, 522)
  int native_fft;        // the slice's FFT group runs the native passes (ffx.cu),
                         // which pad and crop it themselves
};

// Work item: one tile (or a chunk of a heavy tile) of one slice. Item lists
// are launched at a capacity fixed when the trajectory is bound; entries past
// the real items are padding with slice = -1, which the kernels skip.
struct Item {
  int slice;     // -1: padding item, nothing to do
  int tile;      // tile id local to the slice
  int start;     // first entry in the sorted arrays
  int count;     // entries in this item
  int split;     // gridding: 0 if the item owns its tile, else 1 + its partial-tile slot
  int pad[3];
};

// Where the items of a split gridding tile (one whose entries were cut into
// several items) put their partial tiles: slot s holds, for every coil, the
// tile's cells in row-major order over the tile extent. A reduction pass then
// adds the slots of each split tile in item order and stores the sum, so the
// result does not depend on which item finishes first.
struct SplitOut {
  float2* part;         // [slot][coil][cell]
  int64_t slot_stride;  // max_coil * cell_cap
  int cell_cap;         // cells of the largest gridding tile
  int pad;
};

__device__ __forceinline__ float2* split_slot(const SplitOut& so, int split, int coil, int cell) {
  return so.part + (int64_t)(split - 1) * so.slot_stride + (int64_t)coil * so.cell_cap + cell;
}

// Entry-major samples of a normal operator (2D): between interpolation and
// gridding the samples live as [gridding entry][stride] (coil c of entry e
// at e * stride + c), so the interpolation writes one contiguous row of coils
// per entry of the sample and the gridding reads each batch of entries as
// one contiguous block instead of gathering one value per coil row.
struct EntIO {
  const int* ent_of;  // interpolation: per global point, its gridding entries, [pt][4], -1 past the last
  const float* dcf;   // interpolation: density weight folded in before the write (or null)
  int stride;         // > 0: entry-major samples
  int pad;
};

constexpr int kKBTerms = 32;  // terms of the I0 power series kept in KBParams

// One axis of the native FFT (ffx.cu): length n = radix[0] * ... *
// radix[ns - 1], each radix 2, 3, 4, 5, 8 or 16; stage s reads its twiddles
// exp(-2 pi i t j / (L R)), j < L = radix[0] * ... * radix[s - 1], 1 <= t < R,
// at tw + tw_off[s] + j (R - 1) + t - 1 of the axis' table (n - 1 entries).
constexpr int kFfxMaxStages = 12;
constexpr int kFfxMaxN = 1024;
struct FfxAxis {
  int n;
  int ns;
  int radix[kFfxMaxStages];
  int tw_off[kFfxMaxStages];
  unsigned magic[kFfxMaxStages];  // floor(2^32 / L) + 1: b / L = umulhi(b, magic) for b, L <= kFfxMaxN
  int tw_base;  // first entry of this axis in the plan's twiddle table
};

// One FFT group of a grid buffer (slices of one grid size, back to back as
// [batch][nos...]). native: its slices have the same image size and every
// axis is a product of 2, 3 and 5 with at most kFfxMaxN points.
struct FfxGroup {
  bool native;
  FfxAxis ax[kMaxDim];
  int first_slice;  // geometry (image and grid size) shared by the group's slices
  int nsl;          // slices in the group
  int sl_off;       // their ids at FfxSet::d_sl + sl_off, in grid order
  int row_off;      // first grid row of each at FfxSet::d_row + row_off (nsl + 1 entries)
  int64_t nrows;    // grid rows (coils x all axes but the last) of the group
  int64_t grid_off; // complex offset of the group's block in its grid buffer
  int batch;        // coils of the group
};

// The native FFT of one grid buffer: its groups, their twiddle tables and
// slice / row lists (host side owns the device arrays; release() frees them).
struct FfxSet {
  bool ok = false;   // some group is native
  bool all = false;  // every group is native
  std::vector<FfxGroup> grp;
  float2* d_tw = nullptr;
  int* d_sl = nullptr;
  int64_t* d_row = nullptr;
  void release() {
    if (d_tw) cudaFree(d_tw);
    if (d_sl) cudaFree(d_sl);
    if (d_row) cudaFree(d_row);
    d_tw = nullptr;
    d_sl = nullptr;
    d_row = nullptr;
    grp.clear();
    ok = all = false;
  }
};

struct KBParams {
  float radius[kMaxDim];  // W_i / 2
  float beta;             // beta of dimension 0 (all dimensions when uniform_beta)
  float betad[kMaxDim];   // beta per dimension (sigpy-style per-axis kernel parameter)
  int uniform_beta;       // 1: every dimension uses beta (the fast kernels need this)
  int ntaps[kMaxDim];     // candidate taps floor(W_i) + 1
  float inv_radius[kMaxDim];  // 1 / (W_i / 2)
  int series;             // 1: coef holds the series below to float32 accuracy for this beta
  int nterms;             // terms the series needs for this beta: a multiple of 4 in [16, kKBTerms]
  float coef[kKBTerms];   // (beta^2 / 4)^k / (k!)^2, k = 0 .. kKBTerms-1
};

// Horner steps over the coefficients k = 4 blk + 3 .. 4 blk, taken only when
// the plan keeps that block (a warp-uniform branch on a kernel parameter).
// Skipped top blocks leave p = 0, so the first kept block starts the
// recurrence at its highest coefficient.
#define MRN_KB_HIGH_BLOCKS(STEP)                                   \
  _Pragma("unroll") for (int blk = kKBTerms / 4 - 1; blk >= 4; --blk) { \
    if (kb.nterms > 4 * blk) {                                     \
      _Pragma("unroll") for (int k = 4 * blk + 3; k >= 4 * blk; --k) { STEP; } \
    }                                                              \
  }

// Tap weight from |dx| with a precomputed 1/r (the validity test |dx| <= r is
// done by the caller in float32, exactly as the reference's mask), by the
// Abramowitz & Stegun polynomial approximations of I0 (the reference's
// kernel, kernels.py:180-246); differs from kb_tap only by the rounding of
// |dx|/r vs |dx|*(1/r) (<= 1 ulp).
__device__ __forceinline__ float kb_tap_as(float adx, float inv_r, float beta) {
  const float x = adx * inv_r;
  const float z = beta * sqrtf(fmaxf(1.0f - x * x, 0.0f));
  if (z < 3.75f) {
    const float y = (z * (1.0f / 3.75f)) * (z * (1.0f / 3.75f));
    return 1.0f + y * (3.5156229f + y * (3.0899424f + y * (1.2067492f +
                  y * (0.2659732f + y * (0.0360768f + y * 0.0045813f)))));
  }
  const float s = 3.75f * __frcp_rn(z);
  const float p = 0.39894228f + s * (0.01328592f + s * (0.00225319f + s * (-0.00157565f +
                  s * (0.00916281f + s * (-0.02057706f + s * (0.02635537f +
                  s * (-0.01647633f + s * 0.00392377f)))))));
  return expf(z) * rsqrtf(z) * p;
}

// The same weight from the power series I0(z) = sum_k (z^2/4)^k / (k!)^2
// (Abramowitz & Stegun 9.6.10) with z^2 = beta^2 t, t = 1 - x^2: a polynomial
// in t whose coefficients are all positive, so Horner's rule in float32 has
// no cancellation (relative error a few ulp, below the 1e-7 error of the
// A&S approximations themselves). kKBTerms fused multiply-adds with the
// coefficients in kernel parameter space: no branch, no special-function
// unit, no square root. Only the kb.nterms leading terms are evaluated: the
// series is positive with terms shrinking faster than geometrically, and the
// plan picks nterms so the dropped tail at t = 1 (where the relative tail is
// largest) is below 1e-9 of the sum.
__device__ __forceinline__ float kb_tap_series(float adx, float inv_r, const KBParams& kb) {
  const float x = adx * inv_r;
  const float t = fmaxf(1.0f - x * x, 0.0f);
  float w = 0.0f;
  MRN_KB_HIGH_BLOCKS(w = fmaf(w, t, kb.coef[k]))
#pragma unroll
  for (int k = 15; k >= 0; --k) w = fmaf(w, t, kb.coef[k]);
  return w;
}

// Weight and its derivative along the sample coordinate u for a tap at
// dx = j - u: with p(t) the series above, t = 1 - x^2, x = |dx| / r,
// dw/du = p'(t) * (dt/dx) * (dx/du) = p'(t) * (-2x) * (-sign(dx)) / r.
// p and p' come from one Horner pass (the derivative recurrence d <- d t + p).
__device__ __forceinline__ float2 kb_tap_series_du(float dx, float inv_r, const KBParams& kb) {
  const float x = fabsf(dx) * inv_r;
  const float t = fmaxf(1.0f - x * x, 0.0f);
  float p = 0.0f, d = 0.0f;
  MRN_KB_HIGH_BLOCKS(d = fmaf(d, t, p); p = fmaf(p, t, kb.coef[k]))
#pragma unroll
  for (int k = 15; k >= 0; --k) {
    d = fmaf(d, t, p);
    p = fmaf(p, t, kb.coef[k]);
  }
  const float sgn = dx > 0.0f ? 1.0f : (dx < 0.0f ? -1.0f : 0.0f);
  return make_float2(p, d * 2.0f * x * sgn * inv_r);
}

// Weight used by the fast tile kernels: the series when it converges within
// kKBTerms terms for this beta (every beta reachable with W < 8), else A&S.
__device__ __forceinline__ float kb_tap_fast(float adx, float inv_r, const KBParams& kb) {
  return kb.series ? kb_tap_series(adx, inv_r, kb) : kb_tap_as(adx, inv_r, kb.beta);
}

// --------------------------------------------------------------------------
// Kaiser-Bessel kernel value I0(beta sqrt(1 - x^2)), x = |distance| / radius,
// the unnormalised kernel of mr_recon (triton_interp/kernels.py:180-246).
// I0 is evaluated with the polynomial approximations 9.8.1 (z < 3.75) and
// 9.8.2 (z >= 3.75) of Abramowitz & Stegun, Handbook of Mathematical
// Functions, p.378 -- the same published approximation the reference uses.
// --------------------------------------------------------------------------
__device__ __forceinline__ float as_i0(float z) {
  if (z < 3.75f) {
    const float t = z * (1.0f / 3.75f);
    const float y = t * t;
    return 1.0f + y * (3.5156229f + y * (3.0899424f + y * (1.2067492f +
                  y * (0.2659732f + y * (0.0360768f + y * 0.0045813f)))));
  }
  const float s = 3.75f / z;
  const float p = 0.39894228f + s * (0.01328592f + s * (0.00225319f + s * (-0.00157565f +
                  s * (0.00916281f + s * (-0.02057706f + s * (0.02635537f +
                  s * (-0.01647633f + s * 0.00392377f)))))));
  return expf(z) * rsqrtf(z) * p;
}

// (d/dz as_i0(z)) / z, finite at z = 0 (the small-argument polynomial is even).
__device__ __forceinline__ float as_di0_over_z(float z) {
  if (z < 3.75f) {
    const float t = z * (1.0f / 3.75f);
    const float y = t * t;
    const float d = 2.0f * 3.5156229f + y * (4.0f * 3.0899424f + y * (6.0f * 1.2067492f +
                    y * (8.0f * 0.2659732f + y * (10.0f * 0.0360768f + y * (12.0f * 0.0045813f)))));
    return d * (1.0f / (3.75f * 3.75f));
  }
  const float s = 3.75f / z;
  const float p = 0.39894228f + s * (0.01328592f + s * (0.00225319f + s * (-0.00157565f +
                  s * (0.00916281f + s * (-0.02057706f + s * (0.02635537f +
                  s * (-0.01647633f + s * 0.00392377f)))))));
  const float dp = 0.01328592f + s * (2.0f * 0.00225319f + s * (3.0f * -0.00157565f +
                   s * (4.0f * 0.00916281f + s * (5.0f * -0.02057706f + s * (6.0f * 0.02635537f +
                   s * (7.0f * -0.01647633f + s * (8.0f * 0.00392377f)))))));
  const float e = expf(z) * rsqrtf(z);
  const float inv = 1.0f / z;
  // d/dz [e^z z^-1/2 p(3.75/z)] = e^z z^-1/2 (p - p/(2z) - p'(s) * 3.75/z^2)
  const float dz = e * (p - 0.5f * p * inv - dp * s * inv);
  return dz * inv;
}

// Weight of one tap: dx = (float)j - u in float32, valid iff |dx| <= r
// (the mask of weights1d..3d, kernels.py:268-393).
__device__ __forceinline__ float kb_tap(float adx, float r, float beta) {
  const float x = adx / r;
  return as_i0(beta * sqrtf(1.0f - x * x));
}

// d weight / d u for one tap (u the sample coordinate): KB'(x) * sign(u - j) / r.
__device__ __forceinline__ float kb_tap_du(float dx, float r, float beta) {
  const float adx = fabsf(dx);
  const float x = adx / r;
  const float z = beta * sqrtf(fmaxf(1.0f - x * x, 0.0f));
  const float dkb = -beta * beta * x * as_di0_over_z(z);  // d KB / d x
  const float sgn = dx > 0.0f ? -1.0f : (dx < 0.0f ? 1.0f : 0.0f);  // sign(u - j)
  return dkb * sgn / r;
}

// ---------------------------------------------------------------------------
// Run-to-run reproducible float64 reductions. Float atomics add in whatever
// order the blocks arrive; these helpers instead have every block store its
// partial sum, and the last block to finish (found with an integer counter)
// adds the partials in a fixed order.
// ---------------------------------------------------------------------------

// Call in every thread of the block after thread 0 has stored the block's
// partial sum(s) to global memory. True in every thread of the last block of
// the grid to arrive; that block then sees every other block's partials (read
// them with __ldcg) and must reset *counter to 0 before it exits.
__device__ __forceinline__ bool arrive_last_block(unsigned* counter, unsigned nblocks) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == nblocks - 1u;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Sum of src[0..n) by one warp in a fixed order: lane-strided partial sums,
// then a butterfly of shuffles. Lane 0's result is the same on every run.
__device__ __forceinline__ double warp_sum_fixed(const double* src, int64_t n, int lane) {
  double a = 0.0;
  for (int64_t i = lane; i < n; i += 32) a += __ldcg(src + i);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  return a;
}

// torch.remainder for float32 by a positive modulus (ungrid.py:873).
__device__ __forceinline__ float remainder_f32(float a, float n) {
  float m = fmodf(a, n);
  if (m < 0.0f) m = __fadd_rn(m, n);
  return m;
}

__device__ __forceinline__ int pos_mod(int a, int n) {
  int m = a % n;
  return m < 0 ? m + n : m;
}

// Balanced tile partition of [0, nos) into nt tiles: tile t = [b(t), b(t+1)),
// b(t) = floor(t * nos / nt).
__host__ __device__ __forceinline__ int tile_begin(int t, int nos, int nt) {
  return (int)(((int64_t)t * nos) / nt);
}
__host__ __device__ __forceinline__ int tile_of(int s, int nos, int nt) {
  return (int)((((int64_t)s + 1) * nt - 1) / nos);
}

// Slice of a global row index: which 0 = grid rows (prow_off), 1 = image
// rows (irow_off), 2 = one-image-per-slice rows (xrow_off).
__device__ __forceinline__ int slice_by_row(const SliceGeom* sl, int ns, int64_t row, int which) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int64_t o = which == 0 ? sl[mid].prow_off : (which == 1 ? sl[mid].irow_off : sl[mid].xrow_off);
    if (o <= row) lo = mid; else hi = mid - 1;
  }
  return lo;
}

}  // namespace mrn

// Host-side plan object (defined in plan.cu).
struct mrn_plan {
  int ndim = 0;
  int nslices = 0;
  int flags = 0;
  int device = 0;
  int sm_count = 148;  // SMs of the plan's device
  double oversamp = 1.0;
  double width[mrn::kMaxDim] = {1, 1, 1};
  double beta = 0.0;
  int tile[mrn::kMaxDim] = {1, 1, 1};   // interpolation tile edge per dim
  int gtile[mrn::kMaxDim] = {1, 1, 1};  // gridding tile edge per dim
  bool warp_grid = true;  // 2D gridding with warp-private tiles (no atomics) where it applies
  bool reg_grid = true;   // ... with the tile accumulator in registers (tiles <= 8x8)
  bool reg_interp = true;  // 2D interpolation with lane = coil over a [cell][coil] region
  int grid_lanes = 0;      // 2D register gridding: lanes per coil group (0 = from the coil group)
  int coil_group = 1;      // coils per CTA chosen at plan creation (informational)
  int coil_group_req = 0;  // caller's coil group, 0 = choose per kernel kind
  int max_coil = 1;
  int max_chunk = 1024;   // samples per interpolation work item
  int grid_chunk = 1024;  // entries per gridding work item
  int tap_max = 8;  // compile-time tap bound used (8 or 16)
  bool use_fast = true;  // use the unrolled fixed-K tile kernels where they apply
  mrn::KBParams kb{};
  std::vector<mrn::SliceGeom> h_slices;
  int64_t n_img = 0, n_ksp = 0, n_grid = 0, n_trj = 0, n_pts = 0, n_x = 0;
  int64_t n_prow = 0, n_irow = 0, n_xrow = 0;  // row counts of the grid / image layouts
  int ntiles = 0;   // interpolation tiles, all slices
  int ngtiles = 0;  // gridding tiles, all slices
  int tmax_cells[mrn::kMaxDim] = {1, 1, 1};   // largest interpolation tile extent per dim
  int tmax_gcells[mrn::kMaxDim] = {1, 1, 1};  // largest gridding tile extent per dim
  int64_t n_entries_grid = 0;  // gridding entries of the bound trajectory
  // Launch extents of the bound trajectory: upper bounds of the interpolation
  // items, gridding items and split gridding tiles (the exact counts stay on
  // the device in d_counts; mrn_plan_stats reads them).
  int64_t n_items_interp = 0, n_items_grid = 0, n_split = 0;
  int64_t cap_entries = 0, cap_items_i = 0, cap_items_g = 0;  // allocated capacities
  int64_t cap_tiles = 0;
  int64_t cap_part = 0;        // complex elements allocated in d_part
  int64_t cap_sort = 0;        // entries of the item-ordering sort buffers
  bool traj_set = false;

  // device buffers
  mrn::SliceGeom* d_slices = nullptr;
  // the slice table with every k-space offset 0: gridding through it reads
  // one shared [C][M] k-space block for all slices (low-rank adjoint, lowrank.cu)
  mrn::SliceGeom* d_slices_kshared = nullptr;
  float* d_apod = nullptr;          // apodization tables
  float4* d_coord_i = nullptr;      // interp-sorted scaled coords
  int* d_perm_i = nullptr;          // interp-sorted global point ids
  float4* d_coord_g = nullptr;      // gridding-sorted scaled coords
  int* d_perm_g = nullptr;          // gridding-sorted global point ids
  unsigned* d_key_a = nullptr;      // interp keys (unsorted)
  unsigned* d_key_is = nullptr;     // interp keys (sorted)
  unsigned* d_key_b = nullptr;      // gridding keys (unsorted)
  unsigned* d_key_g = nullptr;      // gridding keys (sorted)
  int* d_val_a = nullptr;
  int* d_val_b = nullptr;
  float4* d_coord_tmp = nullptr;    // unsorted coords
  // 2D weight tables (mrn_plan_set_traj; used when wtab_ok): per interpolation
  // sample / gridding entry in sorted order, meta = {start0, start1, taps0,
  // taps1} and the compacted valid (and, for gridding, in-tile) 1D weights,
  // 8 per dimension, zero padded.
  int4* d_wmeta_i = nullptr;
  float4* d_wtab_i = nullptr;  // [entry][4] float4 = w0[0..7], w1[0..7]
  int4* d_wmeta_g = nullptr;
  float4* d_wtab_g = nullptr;
  int64_t cap_wtab_i = 0, cap_wtab_g = 0;
  bool use_wtab = false;  // option: build and use weight tables (off: slower when L2 is cold)
  bool wtab_ok = false;   // tables of the bound trajectory are valid
  int* d_pt_slice = nullptr;        // point -> slice
  int* d_entry_cnt = nullptr;       // per point gridding entries (scan input/output)
  int* d_tile_start_i = nullptr;    // per global tile
  int* d_tile_end_i = nullptr;
  int* d_tile_start_g = nullptr;
  int* d_tile_end_g = nullptr;
  int* d_tile_nitems = nullptr;     // scan buffers
  int* d_tile_item_off = nullptr;
  mrn::Item* d_items_i = nullptr;
  mrn::Item* d_items_g = nullptr;
  int* d_counts = nullptr;          // [0] n_items_i [1] n_items_g [2] n_entries_g [3] n_split
                                    // [4] partial-tile slots in use
  int4* d_split_tiles = nullptr;    // split gridding tiles: {global tile, first slot, items, 0}
  float2* d_part = nullptr;         // partial tiles of split gridding tiles (SplitOut)
  mrn::Item* d_items_tmp = nullptr; // items before the longest-first ordering
  unsigned* d_sort_key[2] = {nullptr, nullptr};  // item ordering: keys in / out
  int* d_sort_idx[2] = {nullptr, nullptr};       // item ordering: indices in / out
  void* d_cub_tmp = nullptr;
  size_t cub_tmp_bytes = 0;
  float2* d_grid = nullptr;         // internal oversampled grid (natural order, grouped)
  float2* d_ksp_tmp = nullptr;      // sample scratch for normal operators
  // 2D normal operator in entry-major sample order (mrn_plan_set_traj): per
  // point its gridding entries ([M][4] then [M] counters), and the samples
  // as [entry][max_coil]
  int* d_ent_of = nullptr;
  float2* d_ksp_ent = nullptr;
  int64_t cap_ent_of = 0, cap_ksp_ent = 0;
  bool ent_ok = false;
  bool use_ent = true;   // option: build the entry map at mrn_plan_set_traj
  void* toep = nullptr;             // Toeplitz normal operator state (toeplitz.cu), or null
  unsigned* d_sync = nullptr;       // last-block counters: [0] k_cg_dir, [1] CG sums, [2] k_post
  double* d_red = nullptr;          // CG block partial sums, [n_slices][kMaxRedBlocks]
  double* d_rowpart = nullptr;      // k_post per-row partials of Re<x, out>, [n_xrow]
  // FFT groups: slices with identical Nos share one batched cuFFT plan
  struct FftGroup {
    int nos[mrn::kMaxDim];
    int64_t grid_off;   // complex offset in d_grid
    int batch;          // sum of coils
    cufftHandle handle;
  };
  std::vector<FftGroup> fft;
  // Native FFT (ffx.cu) of the plan grid's FFT groups; MRN_OPT_NATIVE_FFT
  // selects it (default) or cuFFT for every group.
  mrn::FfxSet ffx;
  bool use_ffx = true;

  // Optional stage timing (mrn_plan_enable_timing): CUDA event pairs recorded
  // on the launching stream around each stage, summed by mrn_plan_timing.
  struct TimingRec {
    int stage;
    cudaEvent_t a, b;
  };
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<TimingRec> timing_recs;
};

namespace mrn {
enum Stage { kStagePre = 0, kStageFft, kStageInterp, kStageGrid, kStagePost, kStageShift,
             kStageTrajGrad, kStageCg, kNumStages };

// Records a CUDA event pair around a scope when the plan's timing is on.
struct StageTimer {
  mrn_plan* P;
  int idx = -1;
  cudaStream_t st;
  StageTimer(mrn_plan* p, int stage, cudaStream_t s);
  ~StageTimer();
};
}  // namespace mrn
