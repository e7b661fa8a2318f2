// 3D gridding (type-1, samples -> oversampled grid) with the tile
// accumulator in registers: the default 3D path of launch_grid_t for kernels
// of 5..8 candidate taps per dimension (width 4 <= W < 8).
//
// Reference: triton_interp/grid.py _grid3d (:369-502) launches one Triton
// program per chunk of points and adds every tap of every batch element into
// global memory with an fp32 atomic. Here the samples are binned into 8x8x8
// tiles (plan.cu, one "entry" per sample and tile its footprint meets), and
// one CTA accumulates a whole tile for up to 16 coils without atomics. Tap
// selection and weights are the reference's: taps j = lo + q, lo = ceil(u -
// W/2), valid iff |(float)j - u| <= W/2 in float32 (kernels.py:268-393),
// weight = prod_d KB(|j_d - u_d| / (W/2)), circular cells.
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"
#include "tile_util.cuh"

namespace mrn {

// ---------------------------------------------------------------------------
// One CTA of four warps per work item (a tile, or a chunk of a heavy tile)
// and group of at most 16 coils; the tile is at most 8x8x8 cells. Thread =
// (coil = lane & 15, x-plane p = 2 warp + lane / 16); it keeps all 8 (y) x 8
// (z) complex cells of its plane in registers, so every update is a register
// FMA with a compile-time index. Per entry each thread reads the tile-aligned
// weight of its plane (zero outside the footprint) and the tile-aligned y and
// z weights; y-rows without weight are skipped by a warp-uniform branch and
// each remaining row takes 8 packed two-lane FMAs along z (fma.rn.f32x2: re
// and im of one cell). There is no data-dependent dispatch: control flow is
// uniform in the warp, and each warp takes one ballot per 32 entries of those
// with weight on its two planes.
//
// The tile-aligned weights (x carrying the scale) and the sample values
// reach shared memory in batches of 64 entries through a cp.async pipeline:
// in iteration b the values of batch b+1 and the coordinates of batch b+3
// are in flight while the weights of batch b+1 are evaluated (the K candidate
// taps of each dimension, written to their cells) and batch b is accumulated;
// one barrier per batch. No atomics; float32 accumulation in entry order, so
// results are the same on every run (split tiles write partial tiles that a
// reduction pass adds in item order).
// ---------------------------------------------------------------------------
constexpr int kG3Tile = 8;
constexpr int kG3Batch = 64;
constexpr int kG3Coils = 16;
constexpr int kG3Threads = 128;

template <int K>
__global__ void __launch_bounds__(kG3Threads, 3)
k_grid_reg3(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
            const float4* __restrict__ coord, const int* __restrict__ perm,
            const float2* __restrict__ ksp, const float* __restrict__ dcf,
            const float2* __restrict__ temporal, float2* __restrict__ grid, int layout, float scale,
            int cg, SplitOut so) {
  constexpr int T = kG3Tile, B = kG3Batch, CW = kG3Coils, NT = kG3Threads;
  static_assert(K <= T, "taps per dimension");
  static_assert(NT == 2 * B, "copy roles assume two threads per batch entry");
  __shared__ float4 s_c[3][B];        // coordinate ring
  __shared__ int s_pm[3][B];          // sample index ring
  __shared__ float s_wx[2][B][T];     // per entry: tile-aligned x weights x scale
  __shared__ float4 s_wy[2][B][2];    // per entry: tile-aligned y weights
  __shared__ float4 s_wz[2][B][4];    // per entry: tile-aligned z weights, each twice
  __shared__ float2 s_v[2][B][CW];    // per entry and coil: sample value
  __shared__ float s_d[2][B];         // per entry: density weight
  __shared__ float2 s_t[2][B];        // per entry: temporal weight

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom* gp = sl + it.slice;
  const int ncoil = gp->ncoil;
  const int c0 = blockIdx.y * cg;
  if (c0 >= ncoil) return;
  const int ncg = min(cg, ncoil - c0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int coil = lane & 15, plane = 2 * warp + (lane >> 4);
  const bool has_coil = coil < ncg;
  const Frame f = frame_of(*gp, it.tile, 3, true);
  const int64_t m = gp->m, pt_off = gp->pt_off;
  const float2* kspg = ksp + gp->ksp_off + (int64_t)c0 * m;
  const int nbatch = (it.count + B - 1) / B;
  auto batch_len = [&](int bi) { return bi < nbatch ? min(B, it.count - bi * B) : 0; };

  // coordinates and sample indices of batch bi into ring slot bi % 3
  auto copy_coords = [&](int bi) {
    const int nb = batch_len(bi), r3 = bi % 3;
    if (tid < nb) cp_async16(&s_c[r3][tid], coord + it.start + bi * B + tid);
    else if (tid >= B && tid - B < nb) cp_async4(&s_pm[r3][tid - B], perm + it.start + bi * B + tid - B);
  };
  // sample values (one 8-byte copy per entry and coil), densities, temporal weights
  auto copy_values = [&](int bi) {
    const int nb = batch_len(bi), b2 = bi & 1, r3 = bi % 3;
    for (int k = tid; k < B * CW; k += NT) {
      const int j = k >> 4, c = k & 15;
      if (j < nb && c < ncg) cp_async8(&s_v[b2][j][c], kspg + (int64_t)c * m + (s_pm[r3][j] - pt_off));
    }
    if (tid < nb) {
      if (dcf) cp_async4(&s_d[b2][tid], dcf + s_pm[r3][tid]);
    } else if (tid >= B && tid - B < nb) {
      if (temporal) cp_async8(&s_t[b2][tid - B], temporal + s_pm[r3][tid - B]);
    }
  };
  // unit (entry j, dimension i): the K candidate taps' weights, written to
  // their cells of the tile-aligned weight vector (zero elsewhere)
  auto weights = [&](int bi) {
    const int nb = batch_len(bi), b2 = bi & 1, r3 = bi % 3;
    for (int t = tid; t < 3 * B; t += NT) {
      const int j = t / 3, i = t - 3 * j;
      if (j >= nb) continue;
      const float4 c4 = s_c[r3][j];
      const float u = i == 0 ? c4.x : (i == 1 ? c4.y : c4.z);
      const float r = sel3(kb.radius, i), ir = sel3(kb.inv_radius, i);
      const int n = sel3(gp->nos, i), size = sel3(f.size, i);
      const int lo = (int)ceilf(__fsub_rn(u, r));
      int st = wrap_once(lo, n) - sel3(f.org, i);
      if (st >= size) st -= n;  // footprint wraps into this tile from the end
      float w[T];
#pragma unroll
      for (int cell = 0; cell < T; ++cell) w[cell] = 0.f;
#pragma unroll
      for (int q = 0; q < K; ++q) {
        const int cell = st + q;
        const float adx = fabsf(__fsub_rn((float)(lo + q), u));
        const float wq = (cell >= 0 && cell < size && adx <= r) ? kb_tap_fast(adx, ir, kb) : 0.f;
#pragma unroll
        for (int c = 0; c < T; ++c)
          if (c == cell) w[c] = wq;
      }
      if (i == 0) {
#pragma unroll
        for (int c = 0; c < T; ++c) s_wx[b2][j][c] = w[c] * scale;
      } else if (i == 1) {
        s_wy[b2][j][0] = make_float4(w[0], w[1], w[2], w[3]);
        s_wy[b2][j][1] = make_float4(w[4], w[5], w[6], w[7]);
      } else {
#pragma unroll
        for (int c = 0; c < T / 2; ++c) s_wz[b2][j][c] = make_float4(w[2 * c], w[2 * c], w[2 * c + 1], w[2 * c + 1]);
      }
    }
  };

  float2 acc[T][T];
#pragma unroll
  for (int a = 0; a < T; ++a)
#pragma unroll
    for (int b = 0; b < T; ++b) acc[a][b] = make_float2(0.f, 0.f);

  copy_coords(0);
  copy_coords(1);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  copy_values(0);
  cp_async_commit();
  copy_coords(2);
  cp_async_commit();
  weights(0);
  for (int bi = 0; bi < nbatch; ++bi) {
    cp_async_wait<1>();  // values of bi and coordinates of bi + 1 have landed (this thread's)
    __syncthreads();     // ... everyone's; weights of bi visible; buffers of bi - 1 free
    copy_values(bi + 1);
    cp_async_commit();
    copy_coords(bi + 3);
    cp_async_commit();
    weights(bi + 1);
    const int b2 = bi & 1, nb = batch_len(bi);
#pragma unroll 1
    for (int h32 = 0; h32 < B; h32 += 32) {
      bool meet = false;
      if (h32 + lane < nb) {
        const float2 xw = *reinterpret_cast<const float2*>(&s_wx[b2][h32 + lane][2 * warp]);
        meet = xw.x != 0.f || xw.y != 0.f;
      }
      unsigned act = __ballot_sync(0xffffffffu, meet);
      while (act) {
        const int j = h32 + __ffs(act) - 1;
        act &= act - 1u;
        const float wx = s_wx[b2][j][plane];
        float2 val = has_coil ? s_v[b2][j][coil] : make_float2(0.f, 0.f);
        if (dcf) {
          const float d = s_d[b2][j];
          val = make_float2(val.x * d, val.y * d);
        }
        if (temporal) {  // times conj(t)
          const float2 tt = s_t[b2][j];
          val = make_float2(val.x * tt.x + val.y * tt.y, val.y * tt.x - val.x * tt.y);
        }
        const float2 v = __fmul2_rn(make_float2(wx, wx), val);
        const float4 y0 = s_wy[b2][j][0], y1 = s_wy[b2][j][1];
        const float wy[T] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
        float2 wz[T];
#pragma unroll
        for (int c = 0; c < T / 2; ++c) {
          const float4 z4 = s_wz[b2][j][c];
          wz[2 * c] = make_float2(z4.x, z4.y);
          wz[2 * c + 1] = make_float2(z4.z, z4.w);
        }
#pragma unroll
        for (int y = 0; y < T; ++y) {
          if (wy[y] == 0.f) continue;  // uniform: the whole warp shares the entry
          const float2 v2 = __fmul2_rn(make_float2(wy[y], wy[y]), v);
#pragma unroll
          for (int z = 0; z < T; ++z) acc[y][z] = __ffma2_rn(wz[z], v2, acc[y][z]);
        }
      }
    }
  }
  cp_async_wait<0>();

  if (has_coil && plane < f.size[0]) {
    const int nos0 = gp->nos[0], nos1 = gp->nos[1], nos2 = gp->nos[2];
    const int hs0 = layout == kInternal ? gp->hshift[0] : 0;
    const int hs1 = layout == kInternal ? gp->hshift[1] : 0;
    const int hs2 = layout == kInternal ? gp->hshift[2] : 0;
    float2* dst = grid + (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)(c0 + coil) * gp->gos;
    const int64_t xo = (int64_t)wrap_once(f.org[0] + plane - hs0, nos0) * nos1;
    const int zs = wrap_once(f.org[2] - hs2, nos2);
#pragma unroll
    for (int y = 0; y < T; ++y) {
      if (y >= f.size[1]) break;
      float2* rowp = dst + (xo + wrap_once(f.org[1] + y - hs1, nos1)) * nos2;
#pragma unroll
      for (int z = 0; z < T; ++z) {
        if (z >= f.size[2]) break;
        int zz = zs + z;
        if (zz >= nos2) zz -= nos2;
        if (it.split)
          *split_slot(so, it.split, c0 + coil, (plane * f.size[1] + y) * f.size[2] + z) = acc[y][z];
        else
          rowp[zz] = acc[y][z];
      }
    }
  }
}

bool grid_reg3_ok(const mrn_plan* P) {
  return P->reg_grid && P->ndim == 3 && P->tmax_gcells[0] <= kG3Tile && P->tmax_gcells[1] <= kG3Tile &&
         P->tmax_gcells[2] <= kG3Tile;
}

int launch_grid_reg3(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                     int layout, float2* grid, float scale, cudaStream_t st) {
  if (P->n_items_grid == 0) return MRN_OK;
  int cg = P->coil_group_req > 0 ? std::min(P->coil_group_req, P->max_coil) : P->max_coil;
  cg = std::max(1, std::min(cg, kG3Coils));
  const int ng = (P->max_coil + cg - 1) / cg;
  cg = (P->max_coil + ng - 1) / ng;
  const dim3 gdim((unsigned)P->n_items_grid, (unsigned)ng);
  const int K = P->kb.ntaps[0];
  const SplitOut so = split_out(P);
#define MRN_G3_LAUNCH(KK)                                                                         \
  k_grid_reg3<KK><<<gdim, kG3Threads, 0, st>>>(P->d_items_g, P->d_slices, P->kb, P->d_coord_g,    \
                                               P->d_perm_g, ksp, dcf, temporal, grid, layout, scale, cg, so)
  if (K == 5) MRN_G3_LAUNCH(5);
  else if (K == 6) MRN_G3_LAUNCH(6);
  else if (K == 7) MRN_G3_LAUNCH(7);
  else MRN_G3_LAUNCH(8);
#undef MRN_G3_LAUNCH
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

}  // namespace mrn
