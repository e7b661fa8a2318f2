// Fast paths of the tile kernels for the common kernel widths: the number of
// candidate taps per dimension K = floor(W) + 1 is a compile-time constant,
// so the K^d tap loop is fully unrolled with immediate shared-memory offsets.
//
// Same algorithm and tap selection as tiles.cu (tap j = lo + q,
// lo = ceil(u - W/2), valid iff |(float)j - u| <= W/2 in float32, separable
// KB weights, circular cells); the differences are in the instruction stream:
//   * the d*K 1D weights of a sample are computed once by the G lanes that
//     share it (one weight per lane, with 1/r precomputed) and broadcast with
//     warp shuffles;
//   * an invalid tap (outside the kernel support, or, for gridding, outside
//     the tile this CTA owns) gets weight 0 in the lane that produces it and
//     is skipped by a predicate, so there is no data-dependent loop bound;
//   * the next sample's coordinates and index are loaded one iteration ahead;
//   * no integer division in the per-sample path.
// Used when every dimension has the same K in {5,6,7,8} (W in [4, 8)), d is
// 2 or 3 and every grid is at least K cells wide; gridding additionally needs
// >= 2 tiles per dimension (so a footprint meets a tile in one contiguous run).
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"
#include "tile_util.cuh"

namespace mrn {

namespace {

// a mod n for a in (-n, inf), by subtraction (region rows may wrap more than once on tiny grids)
__device__ __forceinline__ int wrap_cells(int a, int n) {
  a = a < 0 ? a + n : a;
  while (a >= n) a -= n;
  return a;
}

// 1D weights of one sample, w[i][q] for dim i, tap q (0 when invalid). The G
// lanes of a slot compute the D*K entries round-robin and exchange them by
// shuffles. With OWN, taps whose local cell st[i] + q lies outside [0,
// size[i]) are zeroed too (gridding into an owned tile).
template <int D, int K, int G, bool OWN>
__device__ __forceinline__ void sample_weights(const float* u, const int* lo, const int* st,
                                               const int* size, const KBParams& kb, int lane,
                                               float (&w)[D][K]) {
  constexpr int NW = D * K;
  constexpr int IT = (NW + G - 1) / G;
  const int lg = lane % G;
  float mine[IT];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int t = it * G + lg;
    float v = 0.f;
    if (t < NW) {
      const int i = t / K;
      const int q = t - i * K;
      const float ui = sel3(u, i), ri = sel3(kb.radius, i);
      const float adx = fabsf(__fsub_rn((float)(sel3(lo, i) + q), ui));
      bool ok = adx <= ri;
      if (OWN) {
        const int l = sel3(st, i) + q;
        ok = ok && l >= 0 && l < sel3(size, i);
      }
      if (ok) v = kb_tap_fast(adx, sel3(kb.inv_radius, i), kb);
    }
    mine[it] = v;
  }
  if (G == 1) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int q = 0; q < K; ++q) w[i][q] = mine[i * K + q];
  } else {
    const int base = lane - lg;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int q = 0; q < K; ++q) {
        const int t = i * K + q;
        w[i][q] = __shfl_sync(0xffffffffu, mine[t / G], base + (t % G));
      }
  }
}

// Region loader (tile + halo, wrapped), one warp per row.
template <int D>
__device__ __forceinline__ void load_region_f(float2* __restrict__ tile, const float2* __restrict__ grid,
                                              int64_t goff, int64_t gos, const int* nos,
                                              const int* org, const int* ext, const int* hs, int ncg,
                                              int pstride) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int inner = ext[D - 1];
  int outer = 1;
#pragma unroll
  for (int i = 0; i < D - 1; ++i) outer *= ext[i];
  const int nrows = ncg * outer;
  const int nl = nos[D - 1];
  const int s_first = wrap_once(org[D - 1] - hs[D - 1], nl);
  for (int row = warp; row < nrows; row += kWarps) {
    const int c = row / outer;
    int rr = row - c * outer;
    int l[kMaxDim] = {0, 0, 0};
#pragma unroll
    for (int i = D - 2; i >= 0; --i) {
      l[i] = rr % ext[i];
      rr /= ext[i];
    }
    int64_t base = 0;
    int lbase = 0;
#pragma unroll
    for (int i = 0; i < D - 1; ++i) {
      base = base * nos[i] + wrap_once(org[i] + l[i] - hs[i], nos[i]);
      lbase = lbase * ext[i] + l[i];
    }
    const float2* src = grid + goff + (int64_t)c * gos + base * nl;
    float2* dst = tile + c * pstride + lbase * inner;
    for (int q = lane; q < inner; q += 32) {
      int s = s_first + q;
      while (s >= nl) s -= nl;
      dst[q] = __ldg(src + s);
    }
  }
}

}  // namespace

template <int D, int K, int G>
__global__ void __launch_bounds__(kThreads)
k_interp_fast(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
              const float4* __restrict__ coord, const int* __restrict__ perm,
              const float2* __restrict__ grid, int layout, float2* __restrict__ ksp, float scale,
              const float2* __restrict__ temporal, int cg, int pstride) {
  constexpr int SLOTS = 32 / G;
  constexpr int CPL = G == 32 ? 2 : 1;
  constexpr int STRIDE = kWarps * SLOTS;
  extern __shared__ float4 smem_f4[];
  float2* tile = reinterpret_cast<float2*>(smem_f4);

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom* gp = sl + it.slice;
  const int ncoil = gp->ncoil;
  const int c0 = blockIdx.y * cg;
  if (c0 >= ncoil) return;
  const int ncg = min(cg, ncoil - c0);
  int nos[kMaxDim], hs[kMaxDim], ext[kMaxDim];
#pragma unroll
  for (int i = 0; i < kMaxDim; ++i) {
    nos[i] = gp->nos[i];
    hs[i] = (i < D && layout == kInternal) ? gp->hshift[i] : 0;
  }
  const Frame f = frame_of(*gp, it.tile, D, false);
#pragma unroll
  for (int i = 0; i < kMaxDim; ++i) ext[i] = i < D ? f.size[i] + K - 1 : 1;
  const int64_t gos = gp->gos;
  const int64_t goff = (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gos;
  const int64_t m = gp->m, pt_off = gp->pt_off, ksp_off = gp->ksp_off;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / G, lg = lane % G;
  // first sample of this warp, loaded before the region so the latencies overlap
  int el = warp * SLOTS + slot;
  const int ecl = it.count > 0 ? it.count - 1 : 0;  // interp items are never empty
  float4 c_next = coord[it.start + min(el, ecl)];
  int p_next = perm[it.start + min(el, ecl)];

  load_region_f<D>(tile, grid, goff, gos, nos, f.org, ext, hs, ncg, pstride);
  __syncthreads();

  for (int base = warp * SLOTS; base < it.count; base += STRIDE) {
    el = base + slot;
    const bool active = el < it.count;
    const float4 c4 = c_next;
    const int pm = p_next;
    {
      const int en = min(el + STRIDE, ecl);
      c_next = coord[it.start + en];
      p_next = perm[it.start + en];
    }
    const float u[3] = {c4.x, c4.y, c4.z};
    int lo[3] = {0, 0, 0}, l0[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < D; ++i) {
      lo[i] = (int)ceilf(__fsub_rn(u[i], kb.radius[i]));
      l0[i] = wrap_once(lo[i], nos[i]) - f.org[i];
    }
    float w[D][K];
    sample_weights<D, K, G, false>(u, lo, l0, f.size, kb, lane, w);
    if (!active) continue;
    const int64_t lp = pm - pt_off;
    float2 h = make_float2(scale, 0.f);
    if (temporal) {
      const float2 t = temporal[pt_off + lp];
      h = make_float2(scale * t.x, scale * t.y);
    }
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int c = lg + q * G;
      if (c >= ncg) break;
      const float2* tb = tile + c * pstride;
      float ax = 0.f, ay = 0.f;
      if (D == 2) {
#pragma unroll
        for (int a = 0; a < K; ++a) {
          const float wa = w[0][a];
          if (wa == 0.f) continue;
          const float2* rp = tb + (l0[0] + a) * ext[1] + l0[1];
#pragma unroll
          for (int b = 0; b < K; ++b) {
            const float ww = wa * w[D - 1][b];
            const float2 v = rp[b];
            ax = fmaf(ww, v.x, ax);
            ay = fmaf(ww, v.y, ay);
          }
        }
      } else {
#pragma unroll
        for (int a = 0; a < K; ++a) {
          const float wa = w[0][a];
          if (wa == 0.f) continue;
#pragma unroll
          for (int b = 0; b < K; ++b) {
            const float wab = wa * w[D > 2 ? 1 : 0][b];
            if (wab == 0.f) continue;
            const float2* rp = tb + ((l0[0] + a) * ext[1] + (l0[1] + b)) * ext[2] + l0[2];
#pragma unroll
            for (int z = 0; z < K; ++z) {
              const float ww = wab * w[D - 1][z];
              const float2 v = rp[z];
              ax = fmaf(ww, v.x, ax);
              ay = fmaf(ww, v.y, ay);
            }
          }
        }
      }
      float2* dst = ksp + ksp_off + (int64_t)(c0 + c) * m + lp;
      const float2 v = make_float2(ax * h.x - ay * h.y, ax * h.y + ay * h.x);
      if (temporal) {
        const float2 o = *dst;
        *dst = make_float2(o.x + v.x, o.y + v.y);
      } else {
        *dst = v;
      }
    }
  }
}

template <int D, int K, int G>
__global__ void __launch_bounds__(kThreads)
k_grid_fast(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
            const float4* __restrict__ coord, const int* __restrict__ perm,
            const float2* __restrict__ ksp, const float* __restrict__ dcf,
            const float2* __restrict__ temporal, float2* __restrict__ grid, int layout, float scale,
            int cg, int pstride, SplitOut so) {
  constexpr int SLOTS = 32 / G;
  constexpr int CPL = G == 32 ? 2 : 1;
  constexpr int STRIDE = kWarps * SLOTS;
  extern __shared__ float4 smem_f4[];
  float* acc_re = reinterpret_cast<float*>(smem_f4);
  float* acc_im = acc_re + (size_t)cg * pstride;

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom* gp = sl + it.slice;
  const int ncoil = gp->ncoil;
  const int c0 = blockIdx.y * cg;
  if (c0 >= ncoil) return;
  const int ncg = min(cg, ncoil - c0);
  int nos[kMaxDim], hs[kMaxDim];
#pragma unroll
  for (int i = 0; i < kMaxDim; ++i) {
    nos[i] = gp->nos[i];
    hs[i] = (i < D && layout == kInternal) ? gp->hshift[i] : 0;
  }
  const Frame f = frame_of(*gp, it.tile, D, true);
  int cells = 1;
#pragma unroll
  for (int i = 0; i < D; ++i) cells *= f.size[i];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / G, lg = lane % G;
  int el = warp * SLOTS + slot;
  const int ecl = it.count > 0 ? it.count - 1 : 0;
  float4 c_next = make_float4(0.f, 0.f, 0.f, 0.f);
  int p_next = 0;
  if (it.count > 0) {
    c_next = coord[it.start + min(el, ecl)];
    p_next = perm[it.start + min(el, ecl)];
  }
  for (int idx = threadIdx.x; idx < ncg * pstride; idx += kThreads) {
    acc_re[idx] = 0.f;
    acc_im[idx] = 0.f;
  }
  __syncthreads();

  const int64_t m = gp->m, pt_off = gp->pt_off, ksp_off = gp->ksp_off;
  for (int base = warp * SLOTS; base < it.count; base += STRIDE) {
    el = base + slot;
    const bool active = el < it.count;
    const float4 c4 = c_next;
    const int pm = p_next;
    {
      const int en = min(el + STRIDE, ecl);
      c_next = coord[it.start + en];
      p_next = perm[it.start + en];
    }
    const float u[3] = {c4.x, c4.y, c4.z};
    int lo[3] = {0, 0, 0}, st[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < D; ++i) {
      lo[i] = (int)ceilf(__fsub_rn(u[i], kb.radius[i]));
      int s = wrap_once(lo[i], nos[i]) - f.org[i];
      if (s >= f.size[i]) s -= nos[i];  // footprint wraps into this tile from the end
      st[i] = s;
    }
    float w[D][K];
    sample_weights<D, K, G, true>(u, lo, st, f.size, kb, lane, w);
    if (!active) continue;
    const int64_t lp = pm - pt_off;
    float vs = scale;
    if (dcf) vs *= dcf[pt_off + lp];
    float2 h = make_float2(vs, 0.f);
    if (temporal) {
      const float2 t = temporal[pt_off + lp];
      h = make_float2(vs * t.x, -vs * t.y);
    }
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int c = lg + q * G;
      if (c >= ncg) break;
      const float2 a0 = __ldg(ksp + ksp_off + (int64_t)(c0 + c) * m + lp);
      const float2 v = make_float2(a0.x * h.x - a0.y * h.y, a0.x * h.y + a0.y * h.x);
      float* re = acc_re + c * pstride;
      float* im = acc_im + c * pstride;
      if (D == 2) {
#pragma unroll
        for (int a = 0; a < K; ++a) {
          const float wa = w[0][a];
          if (wa == 0.f) continue;
          const int row = (st[0] + a) * f.size[1] + st[1];
          const float vx = wa * v.x, vy = wa * v.y;
#pragma unroll
          for (int b = 0; b < K; ++b) {
            const float wb = w[1][b];
            if (wb != 0.f) {
              atomicAdd(re + row + b, wb * vx);
              atomicAdd(im + row + b, wb * vy);
            }
          }
        }
      } else {
#pragma unroll
        for (int a = 0; a < K; ++a) {
          const float wa = w[0][a];
          if (wa == 0.f) continue;
#pragma unroll
          for (int b = 0; b < K; ++b) {
            const float wab = wa * w[D > 2 ? 1 : 0][b];
            if (wab == 0.f) continue;
            const int row = ((st[0] + a) * f.size[1] + (st[1] + b)) * f.size[2] + st[2];
            const float vx = wab * v.x, vy = wab * v.y;
#pragma unroll
            for (int z = 0; z < K; ++z) {
              const float wz = w[D - 1][z];
              if (wz != 0.f) {
                atomicAdd(re + row + z, wz * vx);
                atomicAdd(im + row + z, wz * vy);
              }
            }
          }
        }
      }
    }
  }
  __syncthreads();

  // write-back, one warp per row of the tile
  const int64_t gos = gp->gos;
  const int64_t goff = (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gos;
  const int inner = f.size[D - 1];
  const int outer = cells / inner;
  const int nrows = ncg * outer;
  const int nl = nos[D - 1];
  const int s_first = wrap_once(f.org[D - 1] - hs[D - 1], nl);
  for (int row = warp; row < nrows; row += kWarps) {
    const int c = row / outer;
    const int orow = row - c * outer;
    int rr = orow;
    int l[kMaxDim] = {0, 0, 0};
#pragma unroll
    for (int i = D - 2; i >= 0; --i) {
      l[i] = rr % f.size[i];
      rr /= f.size[i];
    }
    int64_t base = 0;
#pragma unroll
    for (int i = 0; i < D - 1; ++i) base = base * nos[i] + wrap_once(f.org[i] + l[i] - hs[i], nos[i]);
    float2* dst = grid + goff + (int64_t)c * gos + base * nl;
    const float* sre = acc_re + c * pstride + orow * inner;
    const float* sim = acc_im + c * pstride + orow * inner;
    for (int q = lane; q < inner; q += 32) {
      int s = s_first + q;
      if (s >= nl) s -= nl;
      const float2 v = make_float2(sre[q], sim[q]);
      if (it.split) *split_slot(so, it.split, c0 + c, orow * inner + q) = v;
      else dst[s] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// 2D gridding with warp-private tiles. One warp per work item; lanes are
// coils (CPL per lane); the warp alone owns its tile's accumulator, so each
// tap is a plain float32 shared-memory read-modify-write (LDS.64, 2 FFMA,
// STS.64) -- no atomics (shared-memory float atomics are compare-and-swap
// loops on sm_100a) and a fixed summation order, so results are bitwise
// reproducible (tiles split over several items write partial tiles that a
// reduction pass adds in item order).
// ---------------------------------------------------------------------------
template <int K, int CPL>
__global__ void __launch_bounds__(32)
k_grid_warp(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
            const float4* __restrict__ coord, const int* __restrict__ perm,
            const float2* __restrict__ ksp, const float* __restrict__ dcf,
            const float2* __restrict__ temporal, float2* __restrict__ grid, int layout, float scale,
            int cg, int pstride, SplitOut so) {
  extern __shared__ float4 smem_f4[];
  float2* acc = reinterpret_cast<float2*>(smem_f4);  // [cg][pstride]

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom* gp = sl + it.slice;
  const int ncoil = gp->ncoil;
  const int c0 = blockIdx.y * cg;
  if (c0 >= ncoil) return;
  const int ncg = min(cg, ncoil - c0);
  const int lane = threadIdx.x;
  const int nos0 = gp->nos[0], nos1 = gp->nos[1];
  const int hs0 = layout == kInternal ? gp->hshift[0] : 0;
  const int hs1 = layout == kInternal ? gp->hshift[1] : 0;
  const Frame f = frame_of(*gp, it.tile, 2, true);
  const int size1 = f.size[1];
  const int cells = f.size[0] * size1;
  const int ecl = it.count > 0 ? it.count - 1 : 0;
  float4 c_next = make_float4(0.f, 0.f, 0.f, 0.f);
  int p_next = 0;
  if (it.count > 0) {
    c_next = coord[it.start];
    p_next = perm[it.start];
  }
  for (int idx = lane; idx < ncg * pstride; idx += 32) acc[idx] = make_float2(0.f, 0.f);
  __syncwarp();

  const int64_t m = gp->m, pt_off = gp->pt_off, ksp_off = gp->ksp_off;
  for (int e = 0; e < it.count; ++e) {
    const float4 c4 = c_next;
    const int pm = p_next;
    {
      const int en = min(e + 1, ecl);
      c_next = coord[it.start + en];
      p_next = perm[it.start + en];
    }
    const float u[3] = {c4.x, c4.y, 0.f};
    int lo[3] = {0, 0, 0}, st[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      lo[i] = (int)ceilf(__fsub_rn(u[i], kb.radius[i]));
      const int n = i == 0 ? nos0 : nos1;
      int s = wrap_once(lo[i], n) - f.org[i];
      if (s >= f.size[i]) s -= n;  // footprint wraps into this tile from the end
      st[i] = s;
    }
    float w[2][K];
    sample_weights<2, K, 32, true>(u, lo, st, f.size, kb, lane, w);
    const int64_t lp = pm - pt_off;
    float vs = scale;
    if (dcf) vs *= dcf[pt_off + lp];
    float2 h = make_float2(vs, 0.f);
    if (temporal) {
      const float2 t = temporal[pt_off + lp];
      h = make_float2(vs * t.x, -vs * t.y);
    }
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int c = lane + q * 32;
      if (c >= ncg) break;
      const float2 a0 = __ldg(ksp + ksp_off + (int64_t)(c0 + c) * m + lp);
      const float2 v = make_float2(a0.x * h.x - a0.y * h.y, a0.x * h.y + a0.y * h.x);
      float2* plane = acc + c * pstride;
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const float wa = w[0][a];
        if (wa == 0.f) continue;
        float2* row = plane + (st[0] + a) * size1 + st[1];
        const float vx = wa * v.x, vy = wa * v.y;
#pragma unroll
        for (int b = 0; b < K; ++b) {
          const float wb = w[1][b];
          if (wb != 0.f) {
            float2 o = row[b];
            o.x = fmaf(wb, vx, o.x);
            o.y = fmaf(wb, vy, o.y);
            row[b] = o;
          }
        }
      }
    }
  }
  __syncwarp();

  // write-back: lanes over the cells of one coil plane at a time
  const int64_t gos = gp->gos;
  const int64_t goff = (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gos;
  for (int c = 0; c < ncg; ++c) {
    float2* dstc = grid + goff + (int64_t)c * gos;
    const float2* src = acc + c * pstride;
    for (int cell = lane; cell < cells; cell += 32) {
      const int l0 = cell / size1, l1 = cell - l0 * size1;
      const int s0 = wrap_once(f.org[0] + l0 - hs0, nos0);
      const int s1 = wrap_once(f.org[1] + l1 - hs1, nos1);
      float2* d = dstc + (int64_t)s0 * nos1 + s1;
      const float2 v = src[cell];
      if (it.split) *split_slot(so, it.split, c0 + c, cell) = v;
      else *d = v;
    }
  }
}

// ---------------------------------------------------------------------------
// 2D / 3D interpolation, lane = coil. The CTA stages its tile region (tile +
// K-1 halo, wrapped) for a group of coils in shared memory as [cell][coil]
// with an odd coil stride CS = CW + 1: the transposing load writes without
// bank conflicts and lanes reading one cell for all their coils touch
// consecutive words. Each warp then takes SUB samples at a time (one per
// group of CW = 32 / SUB lanes): the d*K 1D weights of a sample are computed
// once by its lanes and broadcast with shuffles, and each lane sums its
// coil's K^d taps along the last axis with packed two-lane FMAs
// (fma.rn.f32x2: real and imaginary part in one instruction), one shared
// load per tap, then combines the rows with the outer weights.
// ---------------------------------------------------------------------------
// Region load of the lane-per-coil kernels: the tile region (ext cells,
// wrapped) of ncg coil planes into shared memory as [cell][coil] with coil
// stride CS. Thread = one cell, looping over the coil planes with the global
// address stepped by the plane stride; kLoadBatch loads in flight per thread.
// Consecutive threads read consecutive cells of a row and write shared words
// 2 * CS apart (CS odd: no bank conflict).
template <int D, int CS>
__device__ __forceinline__ void load_region_cc(float2* __restrict__ region, const float2* __restrict__ gbase,
                                               int64_t gos, int ncg, const Frame& f, const int* ext,
                                               const int* nos, const int* hs, int tid, int nthreads) {
  constexpr int kLoadBatch = 8;
  const int inner = ext[D - 1];
  const int ncells = ext[0] * ext[1] * ext[2];
  for (int cell = tid; cell < ncells; cell += nthreads) {
    int64_t off;
    if (D == 2) {
      const int r = cell / inner, q = cell - r * inner;
      off = (int64_t)wrap_cells(f.org[0] + r - hs[0], nos[0]) * nos[1] +
            wrap_cells(f.org[1] + q - hs[1], nos[1]);
    } else {
      const int rz = cell / inner, z = cell - rz * inner;
      const int x = rz / ext[1], y = rz - x * ext[1];
      off = ((int64_t)wrap_cells(f.org[0] + x - hs[0], nos[0]) * nos[1] +
             wrap_cells(f.org[1] + y - hs[1], nos[1])) * nos[2] +
            wrap_cells(f.org[2] + z - hs[2], nos[2]);
    }
    const float2* src = gbase + off;
    float2* dst = region + cell * CS;
    for (int cb = 0; cb < ncg; cb += kLoadBatch) {
      float2 v[kLoadBatch];
#pragma unroll
      for (int u = 0; u < kLoadBatch; ++u)
        if (cb + u < ncg) v[u] = __ldg(src + (int64_t)(cb + u) * gos);
#pragma unroll
      for (int u = 0; u < kLoadBatch; ++u)
        if (cb + u < ncg) dst[cb + u] = v[u];
    }
  }
}

constexpr int kRegInterpWarps = 8;
constexpr int kInterpStage = 128;  // samples whose coordinates are staged at once

// Separable gather of one sample from the [cell][coil] region over the first
// KE taps of each axis (KE = K, or K - 1 when no axis has its last candidate
// tap inside the support, which holds unless a coordinate sits exactly W/2
// from that tap: the skipped terms have weight exactly zero).
template <int D, int K, int KE, int SUB>
__device__ __forceinline__ float2 interp_gather(const float2* rb, int inner, int ext1, int CS,
                                                const float (&w)[D][K], const float2 (&wl)[K]) {
  float2 acc = make_float2(0.f, 0.f);
  if (D == 2) {
#pragma unroll
    for (int a = 0; a < KE; ++a) {
      if (SUB == 1 && w[0][a] == 0.f) continue;
      const float2* rp = rb + a * inner * CS;
      float2 ra = make_float2(0.f, 0.f);
#pragma unroll
      for (int b = 0; b < KE; ++b) ra = __ffma2_rn(wl[b], rp[b * CS], ra);
      acc = __ffma2_rn(make_float2(w[0][a], w[0][a]), ra, acc);
    }
  } else {
#pragma unroll
    for (int a = 0; a < KE; ++a) {
      float2 pa = make_float2(0.f, 0.f);
#pragma unroll
      for (int b = 0; b < KE; ++b) {
        const float2* rp = rb + (a * ext1 + b) * inner * CS;
        float2 ra = make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < KE; ++c) ra = __ffma2_rn(wl[c], rp[c * CS], ra);
        pa = __ffma2_rn(make_float2(w[D > 2 ? 1 : 0][b], w[D > 2 ? 1 : 0][b]), ra, pa);
      }
      acc = __ffma2_rn(make_float2(w[0][a], w[0][a]), pa, acc);
    }
  }
  return acc;
}

// Register budget: three CTAs per SM (80 registers) except 3D with six or more
// taps (two); the two gather paths would otherwise raise register use and
// lower occupancy (a 2D 10^2 or 3D 4^3 tile region takes ~70 KB of shared
// memory, so three CTAs fit).
template <int D, int K, int SUB>
__global__ void __launch_bounds__(kRegInterpWarps * 32, (D == 3 && K > 5) ? 2 : 3)
k_interp_reg(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
             const float4* __restrict__ coord, const int* __restrict__ perm,
             const float2* __restrict__ grid, int layout, float2* __restrict__ ksp, float scale,
             const float2* __restrict__ temporal, int cg, EntIO eio) {
  constexpr int CW = 32 / SUB, CS = CW + 1, NW = kRegInterpWarps, NT = NW * 32;
  extern __shared__ float4 smem_f4[];
  float2* region = reinterpret_cast<float2*>(smem_f4);
  __shared__ float4 s_u[kInterpStage];  // coordinates of the staged samples
  __shared__ int s_p[kInterpStage];     // their sample indices within the slice

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom* gp = sl + it.slice;
  const int ncoil = gp->ncoil;
  const int c0 = blockIdx.y * cg;
  if (c0 >= ncoil) return;
  const int ncg = min(cg, ncoil - c0);
  int nos[3], hs[3], ext[3];
  const Frame f = frame_of(*gp, it.tile, D, false);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    nos[i] = gp->nos[i];
    hs[i] = (i < D && layout == kInternal) ? gp->hshift[i] : 0;
    ext[i] = i < D ? f.size[i] + K - 1 : 1;
  }
  const int inner = ext[D - 1];
  const int64_t gos = gp->gos;
  const float2* gbase = grid + (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gos;
  const int64_t m = gp->m, pt_off = gp->pt_off;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int coil = lane % CW, sub = lane / CW;
  const bool has_coil = coil < ncg;
  float2* kspc = ksp + gp->ksp_off + (int64_t)(c0 + (has_coil ? coil : 0)) * m;

  for (int sb = 0; sb < it.count; sb += kInterpStage) {
    const int ns = min(kInterpStage, it.count - sb);
    if (sb > 0) __syncthreads();  // every warp is done with the previous stage
    for (int j = tid; j < ns; j += NT) {
      s_u[j] = coord[it.start + sb + j];
      s_p[j] = (int)(perm[it.start + sb + j] - pt_off);
    }
    if (sb == 0) load_region_cc<D, CS>(region, gbase, gos, ncg, f, ext, nos, hs, tid, NT);
    __syncthreads();

    for (int base = warp * SUB; base < ns; base += NW * SUB) {
      const int el = base + sub;
      const bool active = el < ns;
      const float4 uu = s_u[active ? el : base];
      const float u[3] = {uu.x, uu.y, uu.z};
      int lo[3] = {0, 0, 0}, l0[3] = {0, 0, 0};
#pragma unroll
      for (int i = 0; i < D; ++i) {
        lo[i] = (int)ceilf(__fsub_rn(u[i], kb.radius[i]));
        l0[i] = wrap_once(lo[i], nos[i]) - f.org[i];
      }
      float w[D][K];
      sample_weights<D, K, CW, false>(u, lo, l0, f.size, kb, lane, w);
      if (!active || !has_coil) continue;
      float2 wl[K];  // last-axis weights, each twice
#pragma unroll
      for (int b = 0; b < K; ++b) wl[b] = make_float2(w[D - 1][b], w[D - 1][b]);
      const float2* rb = D == 2 ? region + (l0[0] * inner + l0[1]) * CS + coil
                                : region + ((l0[0] * ext[1] + l0[1]) * inner + l0[D - 1]) * CS + coil;
      bool last = false;  // some axis has its K-th candidate tap inside the support
#pragma unroll
      for (int i = 0; i < D; ++i) last |= w[i][K - 1] != 0.f;
      const float2 acc = last ? interp_gather<D, K, K, SUB>(rb, inner, ext[1], CS, w, wl)
                              : interp_gather<D, K, K - 1, SUB>(rb, inner, ext[1], CS, w, wl);
      const int lp = s_p[el];
      float2 h = make_float2(scale, 0.f);
      if (temporal) {
        const float2 t = temporal[pt_off + lp];
        h = make_float2(scale * t.x, scale * t.y);
      }
      const float2 v = make_float2(acc.x * h.x - acc.y * h.y, acc.x * h.y + acc.y * h.x);
      if (eio.stride > 0) {  // entry-major: one contiguous row of coils per entry of the sample
        const int64_t pg = pt_off + lp;
        float2 vv = v;
        if (eio.dcf) {
          const float d = eio.dcf[pg];
          vv = make_float2(v.x * d, v.y * d);
        }
        const int4 es = *reinterpret_cast<const int4*>(eio.ent_of + pg * 4);
        const int ee[4] = {es.x, es.y, es.z, es.w};
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (ee[q] >= 0) ksp[(int64_t)ee[q] * eio.stride + c0 + coil] = vv;
        continue;
      }
      float2* dst = kspc + lp;
      if (temporal) {
        const float2 o = *dst;
        *dst = make_float2(o.x + v.x, o.y + v.y);
      } else {
        *dst = v;
      }
    }
  }
}

// Separable sums of the trajectory gradient over the first KE taps of each
// axis (see interp_gather): out[i] = sum over taps of the region value times
// the weights with axis i's factor replaced by its derivative.
template <int D, int K, int KE>
__device__ __forceinline__ void trajgrad_gather(const float2* rb, int inner, int ext1, int CS,
                                                const float (&w)[D][K], const float (&dw)[D][K],
                                                float2 (&out)[3]) {
  float2 a0 = make_float2(0.f, 0.f), a1 = a0, a2 = a0;
  if (D == 2) {
#pragma unroll
    for (int a = 0; a < KE; ++a) {
      const float2* rp = rb + a * inner * CS;
      float2 r = make_float2(0.f, 0.f), rd = r;
#pragma unroll
      for (int b = 0; b < KE; ++b) {
        const float2 gv = rp[b * CS];
        r = __ffma2_rn(make_float2(w[D - 1][b], w[D - 1][b]), gv, r);
        rd = __ffma2_rn(make_float2(dw[D - 1][b], dw[D - 1][b]), gv, rd);
      }
      a0 = __ffma2_rn(make_float2(dw[0][a], dw[0][a]), r, a0);
      a1 = __ffma2_rn(make_float2(w[0][a], w[0][a]), rd, a1);
    }
  } else {
#pragma unroll
    for (int a = 0; a < KE; ++a) {
      float2 p = make_float2(0.f, 0.f), p1 = p, p2 = p;
#pragma unroll
      for (int b = 0; b < KE; ++b) {
        const float2* rp = rb + (a * ext1 + b) * inner * CS;
        float2 r = make_float2(0.f, 0.f), rd = r;
#pragma unroll
        for (int c = 0; c < KE; ++c) {
          const float2 gv = rp[c * CS];
          r = __ffma2_rn(make_float2(w[D - 1][c], w[D - 1][c]), gv, r);
          rd = __ffma2_rn(make_float2(dw[D - 1][c], dw[D - 1][c]), gv, rd);
        }
        p = __ffma2_rn(make_float2(w[D > 2 ? 1 : 0][b], w[D > 2 ? 1 : 0][b]), r, p);
        p1 = __ffma2_rn(make_float2(dw[D > 2 ? 1 : 0][b], dw[D > 2 ? 1 : 0][b]), r, p1);
        p2 = __ffma2_rn(make_float2(w[D > 2 ? 1 : 0][b], w[D > 2 ? 1 : 0][b]), rd, p2);
      }
      a0 = __ffma2_rn(make_float2(dw[0][a], dw[0][a]), p, a0);
      a1 = __ffma2_rn(make_float2(w[0][a], w[0][a]), p1, a1);
      a2 = __ffma2_rn(make_float2(w[0][a], w[0][a]), p2, a2);
    }
  }
  out[0] = a0;
  out[1] = a1;
  out[2] = a2;
}

// ---------------------------------------------------------------------------
// Trajectory gradient, lane = coil: d/du_i Re sum_c conj(S_c) (A x)_c at each
// sample, the same region staging and sample loop as k_interp_reg. Per
// sample each lane forms, for its coil, the separable sums with one factor
// replaced by the weight's derivative (2D: row sums with w1 and dw1, then
// dw0 / w0; 3D: row sums with w2 and dw2, plane sums with w1 / dw1, then
// dw0 / w0), takes Re(conj(S_c) .) and the sample's lanes sum over their
// coils with shuffles; one atomic add per sample and dimension (coil groups
// of one slice add into the same output).
// ---------------------------------------------------------------------------
template <int D, int K, int SUB>
__global__ void __launch_bounds__(kRegInterpWarps * 32)
k_trajgrad_reg(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
               const float4* __restrict__ coord, const int* __restrict__ perm,
               const float2* __restrict__ grid, int layout, const float2* __restrict__ samp,
               float* __restrict__ out, float scale, int cg) {
  constexpr int CW = 32 / SUB, CS = CW + 1, NW = kRegInterpWarps, NT = NW * 32;
  extern __shared__ float4 smem_f4[];
  float2* region = reinterpret_cast<float2*>(smem_f4);
  __shared__ float4 s_u[kInterpStage];
  __shared__ int s_p[kInterpStage];

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom* gp = sl + it.slice;
  const int ncoil = gp->ncoil;
  const int c0 = blockIdx.y * cg;
  if (c0 >= ncoil) return;
  const int ncg = min(cg, ncoil - c0);
  int nos[3], hs[3], ext[3];
  const Frame f = frame_of(*gp, it.tile, D, false);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    nos[i] = gp->nos[i];
    hs[i] = (i < D && layout == kInternal) ? gp->hshift[i] : 0;
    ext[i] = i < D ? f.size[i] + K - 1 : 1;
  }
  const int inner = ext[D - 1];
  const int64_t gos = gp->gos;
  const float2* gbase = grid + (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gos;
  const int64_t m = gp->m, pt_off = gp->pt_off;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int coil = lane % CW, sub = lane / CW;
  const bool has_coil = coil < ncg;
  const float2* sampc = samp + gp->ksp_off + (int64_t)(c0 + (has_coil ? coil : 0)) * m;
  const float osc[3] = {scale * gp->scale[0], scale * gp->scale[1], scale * gp->scale[2]};

  for (int sb = 0; sb < it.count; sb += kInterpStage) {
    const int ns = min(kInterpStage, it.count - sb);
    if (sb > 0) __syncthreads();
    for (int j = tid; j < ns; j += NT) {
      s_u[j] = coord[it.start + sb + j];
      s_p[j] = perm[it.start + sb + j];
    }
    if (sb == 0) load_region_cc<D, CS>(region, gbase, gos, ncg, f, ext, nos, hs, tid, NT);
    __syncthreads();

    for (int base = warp * SUB; base < ns; base += NW * SUB) {
      const int el = base + sub;
      const bool active = el < ns;
      const float4 uu = s_u[active ? el : base];
      const int pm = s_p[active ? el : base];
      const float2 sv = (active && has_coil) ? __ldg(sampc + (pm - pt_off)) : make_float2(0.f, 0.f);
      const float u[3] = {uu.x, uu.y, uu.z};
      int lo[3] = {0, 0, 0}, l0[3] = {0, 0, 0};
#pragma unroll
      for (int i = 0; i < D; ++i) {
        lo[i] = (int)ceilf(__fsub_rn(u[i], kb.radius[i]));
        l0[i] = wrap_once(lo[i], nos[i]) - f.org[i];
      }
      // weight and derivative of tap t = i*K + q, computed by the sample's lanes, broadcast
      constexpr int NWT = D * K, IT = (NWT + CW - 1) / CW;
      const int lg = lane % CW, lbase = lane - lg;
      float2 mine[IT];
#pragma unroll
      for (int k2 = 0; k2 < IT; ++k2) {
        const int t = k2 * CW + lg;
        float2 v = make_float2(0.f, 0.f);
        if (t < NWT) {
          const int i = t / K, q = t - (t / K) * K;
          const float ui = sel3(u, i), ri = sel3(kb.radius, i);
          const float dx = __fsub_rn((float)(sel3(lo, i) + q), ui);
          if (fabsf(dx) <= ri) {
            if (kb.series) {
              v = kb_tap_series_du(dx, sel3(kb.inv_radius, i), kb);
            } else {
              v = make_float2(kb_tap(fabsf(dx), ri, kb.beta), kb_tap_du(dx, ri, kb.beta));
            }
          }
        }
        mine[k2] = v;
      }
      float w[D][K], dw[D][K];
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int q = 0; q < K; ++q) {
          const int t = i * K + q;
          w[i][q] = __shfl_sync(0xffffffffu, mine[t / CW].x, lbase + (t % CW));
          dw[i][q] = __shfl_sync(0xffffffffu, mine[t / CW].y, lbase + (t % CW));
        }
      float g[3] = {0.f, 0.f, 0.f};
      if (active && has_coil) {
        float2 acc3[3];
        const float2* rb = D == 2 ? region + (l0[0] * inner + l0[1]) * CS + coil
                                  : region + ((l0[0] * ext[1] + l0[1]) * inner + l0[D - 1]) * CS + coil;
        bool last = false;  // some axis has its K-th candidate tap inside the support
#pragma unroll
        for (int i = 0; i < D; ++i) last |= w[i][K - 1] != 0.f;
        if (last) trajgrad_gather<D, K, K>(rb, inner, ext[1], CS, w, dw, acc3);
        else trajgrad_gather<D, K, K - 1>(rb, inner, ext[1], CS, w, dw, acc3);
        const float2 a0 = acc3[0], a1 = acc3[1], a2 = acc3[2];
        // Re(conj(S) * acc)
        g[0] = sv.x * a0.x + sv.y * a0.y;
        g[1] = sv.x * a1.x + sv.y * a1.y;
        g[2] = sv.x * a2.x + sv.y * a2.y;
      }
      // sum over the sample's coil lanes
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int o = CW / 2; o > 0; o >>= 1) g[i] += __shfl_xor_sync(0xffffffffu, g[i], o);
      if (active && coil == 0) {
#pragma unroll
        for (int i = 0; i < D; ++i) atomicAdd(out + (int64_t)pm * D + i, g[i] * osc[i]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// 2D gridding with the tile accumulator in registers. One block of two warps
// per work item; lane = coil, warp w owns rows 4w..4w+3 of the (at most) 8x8
// tile, so each lane keeps 4x8 complex cells in registers and every update
// is a register FMA with a compile-time index: no shared-memory
// read-modify-write, no atomics, float32 accumulation in a fixed order
// (reproducible results; split tiles write partial tiles that a reduction
// pass adds in item order).
//
// Entries run in batches of kRegBatch through an asynchronous pipeline
// (cp.async), one barrier per batch. In iteration b:
//   * the sample values (one 8-byte copy per entry and coil), densities and
//     temporal weights of batch b+1 are copied into shared memory;
//   * the coordinates and sample indices of batch b+3 are copied into a
//     three-slot ring;
//   * the 1D weights of batch b+1 are computed, already aligned to the
//     tile's cells (zero outside the kernel support and the tile): thread
//     (entry, dimension, half) evaluates 4 cells and stores them at once;
//   * batch b accumulates: per entry, each of the warp's tile rows with a
//     non-zero weight takes 8 packed two-lane FMAs per lane (fma.rn.f32x2:
//     real and imaginary part of a cell in one instruction); the scale is
//     folded into the row weights.
// With at most 16 coils per group a warp runs SUB = 32 / CW entry streams of
// CW lanes (CW = coil group rounded up to a power of two); their partial
// tiles are summed with shuffles before the write-back.
// ---------------------------------------------------------------------------
constexpr int kRegTile = 8;
constexpr int kRegRows = kRegTile / 2;  // tile rows per warp
constexpr int kRegBatch = 16;
constexpr int kRegStage = kRegTile * kRegTile + 1;  // cells per coil block in the write-back, padded

// Shared memory of k_grid_reg: the batch pipeline's buffers, reused after the
// last batch to stage the tile for the write-back.
template <int CW>
union G2Smem {
  struct {
    float4 c[3][kRegBatch];      // coordinate ring
    int pm[3][kRegBatch];        // sample index ring
    float4 wr[2][kRegBatch][2];  // per entry: row weights x scale (cells 0-7)
    float4 wc[2][kRegBatch][4];  // per entry: column weights, each twice (cells 0-7)
    float2 v[2][kRegBatch][CW + 1];  // per entry and coil: sample value (row padded: conflict-free copies)
    float d[2][kRegBatch];       // per entry: density weight
    float2 t[2][kRegBatch];      // per entry: temporal weight
  } b;
  float2 stage[CW][kRegStage];   // write-back: per coil, the tile's cells row-major
};

template <int K, int SUB>
__global__ void __launch_bounds__(64, 8)
k_grid_reg(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
           const float4* __restrict__ coord, const int* __restrict__ perm,
           const float2* __restrict__ ksp, const float* __restrict__ dcf,
           const float2* __restrict__ temporal, float2* __restrict__ grid, int layout, float scale,
           int cg, SplitOut so, int ent_stride) {
  constexpr int T = kRegTile, R = kRegRows, B = kRegBatch, CW = 32 / SUB;
  __shared__ G2Smem<CW> sm;
  auto& s_c = sm.b.c;
  auto& s_pm = sm.b.pm;
  auto& s_wr = sm.b.wr;
  auto& s_wc = sm.b.wc;
  auto& s_v = sm.b.v;
  auto& s_d = sm.b.d;
  auto& s_t = sm.b.t;

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom* gp = sl + it.slice;
  const int ncoil = gp->ncoil;
  const int c0 = blockIdx.y * cg;
  if (c0 >= ncoil) return;
  const int ncg = min(cg, ncoil - c0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int coil = lane % CW, sub = lane / CW;
  const int sid = warp * SUB + sub;  // copy stream of this thread
  const bool has_coil = coil < ncg;
  const int nos0 = gp->nos[0], nos1 = gp->nos[1];
  const Frame f = frame_of(*gp, it.tile, 2, true);
  const int64_t m = gp->m, pt_off = gp->pt_off;
  const int nbatch = (it.count + B - 1) / B;
  auto batch_len = [&](int bi) { return bi < nbatch ? min(B, it.count - bi * B) : 0; };

  // coordinates and sample indices of batch bi into ring slot bi % 3
  auto copy_coords = [&](int bi) {
    const int nb = batch_len(bi), r3 = bi % 3;
    if (tid < nb) cp_async16(&s_c[r3][tid], coord + it.start + bi * B + tid);
    else if (tid >= 32 && tid - 32 < nb) cp_async4(&s_pm[r3][tid - 32], perm + it.start + bi * B + tid - 32);
  };
  // values (per entry and coil), densities and temporal weights of batch bi
  auto copy_values = [&](int bi) {
    const int nb = batch_len(bi), b2 = bi & 1, r3 = bi % 3;
    if (ent_stride > 0) {  // entry-major samples: the batch's rows are contiguous
      if (has_coil) {
        const float2* eb = ksp + (int64_t)(it.start + bi * B) * ent_stride + c0 + coil;
        for (int j = sid; j < nb; j += 2 * SUB) cp_async8(&s_v[b2][j][coil], eb + (int64_t)j * ent_stride);
      }
    } else {
      // thread = (entry tid % B, coil phase tid / B): one warp copy reads 16
      // entries of each of two coil rows, i.e. consecutive samples of a row
      // (one or two 128-byte lines) rather than 32 coil rows
      const int j = tid % B;
      if (j < nb) {
        const float2* src = ksp + gp->ksp_off + (int64_t)c0 * m + (s_pm[r3][j] - pt_off);
        for (int c = tid / B; c < ncg; c += 64 / B) cp_async8(&s_v[b2][j][c], src + (int64_t)c * m);
      }
    }
    if (tid < nb) {
      if (dcf) cp_async4(&s_d[b2][tid], dcf + s_pm[r3][tid]);
    } else if (tid >= 32 && tid - 32 < nb) {
      if (temporal) cp_async8(&s_t[b2][tid - 32], temporal + s_pm[r3][tid - 32]);
    }
  };
  // tile-aligned 1D weights of batch bi: thread = (entry, dimension, half of the cells)
  auto weights = [&](int bi) {
    const int j = tid >> 2, i = (tid >> 1) & 1, h = tid & 1;
    if (j >= batch_len(bi)) return;
    const float4 c4 = s_c[bi % 3][j];
    const float u = i ? c4.y : c4.x;
    const float r = i ? kb.radius[1] : kb.radius[0];
    const float ir = i ? kb.inv_radius[1] : kb.inv_radius[0];
    const int n = i ? nos1 : nos0;
    const int size = i ? f.size[1] : f.size[0];
    const int lo = (int)ceilf(__fsub_rn(u, r));
    int st = wrap_once(lo, n) - (i ? f.org[1] : f.org[0]);
    if (st >= size) st -= n;  // footprint wraps into this tile from the end
    float w[4];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const int cell = 4 * h + l;
      const int q = cell - st;
      const float adx = fabsf(__fsub_rn((float)(lo + q), u));
      w[l] = (q >= 0 && q < K && cell < size && adx <= r) ? kb_tap_fast(adx, ir, kb) : 0.f;
    }
    if (i == 0) {
      s_wr[bi & 1][j][h] = make_float4(w[0] * scale, w[1] * scale, w[2] * scale, w[3] * scale);
    } else {
      s_wc[bi & 1][j][2 * h] = make_float4(w[0], w[0], w[1], w[1]);
      s_wc[bi & 1][j][2 * h + 1] = make_float4(w[2], w[2], w[3], w[3]);
    }
  };

  float2 acc[R][T];
#pragma unroll
  for (int a = 0; a < R; ++a)
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
    for (int j = sub; j < nb; j += SUB) {
      const float4 rw = s_wr[b2][j][warp];
      const float wr[R] = {rw.x, rw.y, rw.z, rw.w};
      float2 wc[T];
#pragma unroll
      for (int b = 0; b < T / 2; ++b) {
        const float4 c = s_wc[b2][j][b];
        wc[2 * b] = make_float2(c.x, c.y);
        wc[2 * b + 1] = make_float2(c.z, c.w);
      }
      float2 val = s_v[b2][j][coil];
      if (dcf) {
        const float d = s_d[b2][j];
        val = make_float2(val.x * d, val.y * d);
      }
      if (temporal) {  // times conj(t)
        const float2 t = s_t[b2][j];
        val = make_float2(val.x * t.x + val.y * t.y, val.y * t.x - val.x * t.y);
      }
#pragma unroll
      for (int a = 0; a < R; ++a) {
        if (SUB == 1 && wr[a] == 0.f) continue;  // uniform: one entry per warp
        const float2 v2 = make_float2(wr[a] * val.x, wr[a] * val.y);
#pragma unroll
        for (int b = 0; b < T; ++b) acc[a][b] = __ffma2_rn(wc[b], v2, acc[a][b]);  // both lanes of the cell
      }
    }
  }
  cp_async_wait<0>();

  if (SUB > 1) {
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
      for (int b = 0; b < T; ++b)
#pragma unroll
        for (int o = CW; o < 32; o <<= 1) {
          acc[a][b].x += __shfl_xor_sync(0xffffffffu, acc[a][b].x, o);
          acc[a][b].y += __shfl_xor_sync(0xffffffffu, acc[a][b].y, o);
        }
  }
  // Write-back through shared memory: each lane stores its coil's cells as a
  // row-major block (stride 65 cells: conflict-free 8-byte stores), then
  // thread t stores cell t of every coil block, so one warp store covers four
  // 64-byte rows of one coil instead of 32 coils' scattered 8-byte cells.
  __syncthreads();  // batch buffers no longer read
  if (has_coil && sub == 0) {
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
      for (int b = 0; b < T; ++b) sm.stage[coil][(warp * R + a) * T + b] = acc[a][b];
  }
  __syncthreads();
  const int row = tid >> 3, col = tid & 7;
  if (row < f.size[0] && col < f.size[1]) {
    const int hs0 = layout == kInternal ? gp->hshift[0] : 0;
    const int hs1 = layout == kInternal ? gp->hshift[1] : 0;
    const int64_t gos = gp->gos;
    float2* dst = grid + (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gos +
                  (int64_t)wrap_once(f.org[0] + row - hs0, nos0) * nos1 + wrap_once(f.org[1] + col - hs1, nos1);
    const int scell = row * f.size[1] + col;
#pragma unroll 4
    for (int c = 0; c < ncg; ++c) {
      const float2 val = sm.stage[c][tid];
      if (it.split) *split_slot(so, it.split, c0 + c, scell) = val;
      else dst[(int64_t)c * gos] = val;
    }
  }
}

// ---------------------------------------------------------------------------
// Launch helpers (called from tiles.cu when the fast path applies)
// ---------------------------------------------------------------------------
template <class Kern>
static int prep_attr(Kern kernel, size_t smem) {
  return set_dynamic_smem(kernel, smem);
}

#define MRN_FAST_G(G_, ...)                                        \
  switch (G_) {                                                    \
    case 1: { constexpr int GG = 1; __VA_ARGS__; } break;          \
    case 2: case 4: { constexpr int GG = 4; __VA_ARGS__; } break;  \
    case 8: { constexpr int GG = 8; __VA_ARGS__; } break;          \
    case 16: { constexpr int GG = 16; __VA_ARGS__; } break;        \
    default: { constexpr int GG = 32; __VA_ARGS__; } break;        \
  }

#define MRN_FAST_DK(D_, K_, ...)                                      \
  do {                                                                \
    if ((D_) == 2 && (K_) == 5) { constexpr int DD = 2, KK = 5; __VA_ARGS__; }       \
    else if ((D_) == 2 && (K_) == 6) { constexpr int DD = 2, KK = 6; __VA_ARGS__; }  \
    else if ((D_) == 2 && (K_) == 7) { constexpr int DD = 2, KK = 7; __VA_ARGS__; }  \
    else if ((D_) == 2) { constexpr int DD = 2, KK = 8; __VA_ARGS__; }               \
    else if ((K_) == 5) { constexpr int DD = 3, KK = 5; __VA_ARGS__; }               \
    else if ((K_) == 6) { constexpr int DD = 3, KK = 6; __VA_ARGS__; }               \
    else if ((K_) == 7) { constexpr int DD = 3, KK = 7; __VA_ARGS__; }               \
    else { constexpr int DD = 3, KK = 8; __VA_ARGS__; }                              \
  } while (0)

bool fast_path_ok(const mrn_plan* P, bool gridding) {
  if (!P->use_fast || P->ndim < 2 || !P->kb.uniform_beta) return false;
  const int K = P->kb.ntaps[0];
  if (K < 5 || K > 8) return false;
  for (int i = 1; i < P->ndim; ++i)
    if (P->kb.ntaps[i] != K) return false;
  // region columns wrap at most once: every grid at least K cells wide
  for (const auto& g : P->h_slices)
    for (int i = 0; i < P->ndim; ++i)
      if (g.nos[i] < K) return false;
  if (gridding) {
    for (const auto& g : P->h_slices)
      for (int i = 0; i < P->ndim; ++i)
        if (g.gntile[i] < 2) return false;
  }
  return true;
}

int launch_interp_fast(mrn_plan* P, const float2* grid, int layout, float2* ksp, float scale,
                       const float2* temporal, int cg, int G, int pstride, size_t smem, dim3 gdim,
                       cudaStream_t st) {
  int rc = MRN_OK;
  MRN_FAST_DK(P->ndim, P->kb.ntaps[0], MRN_FAST_G(G, {
    auto kern = k_interp_fast<DD, KK, GG>;
    rc = prep_attr(kern, smem);
    if (rc == MRN_OK)
      kern<<<gdim, kThreads, smem, st>>>(P->d_items_i, P->d_slices, P->kb, P->d_coord_i, P->d_perm_i,
                                         grid, layout, ksp, scale, temporal, cg, pstride);
  }));
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_grid_warp(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                     int layout, float2* grid, float scale, cudaStream_t st) {
  if (P->n_items_grid == 0) return MRN_OK;
  const int pstride = (P->tmax_gcells[0] * P->tmax_gcells[1]) | 1;
  int cg = P->coil_group_req > 0 ? std::min(P->coil_group_req, P->max_coil) : P->max_coil;
  cg = std::max(1, std::min(cg, 64));
  const int ng = (P->max_coil + cg - 1) / cg;
  cg = (P->max_coil + ng - 1) / ng;
  const size_t smem = (size_t)cg * pstride * sizeof(float2);
  if (smem > 227 * 1024) return MRN_ERR_UNSUPPORTED;
  const dim3 gdim((unsigned)P->n_items_grid, (unsigned)ng);
  int rc = MRN_OK;
  const int K = P->kb.ntaps[0];
#define MRN_WARP_LAUNCH(KK, CP)                                                                   \
  do {                                                                                            \
    auto kern = k_grid_warp<KK, CP>;                                                              \
    rc = prep_attr(kern, smem);                                                                   \
    if (rc == MRN_OK)                                                                             \
      kern<<<gdim, 32, smem, st>>>(P->d_items_g, P->d_slices, P->kb, P->d_coord_g, P->d_perm_g,   \
                                   ksp, dcf, temporal, grid, layout, scale, cg, pstride,          \
                                   split_out(P));                                                 \
  } while (0)
  const bool two = cg > 32;
  if (K == 5) { if (two) MRN_WARP_LAUNCH(5, 2); else MRN_WARP_LAUNCH(5, 1); }
  else if (K == 6) { if (two) MRN_WARP_LAUNCH(6, 2); else MRN_WARP_LAUNCH(6, 1); }
  else if (K == 7) { if (two) MRN_WARP_LAUNCH(7, 2); else MRN_WARP_LAUNCH(7, 1); }
  else { if (two) MRN_WARP_LAUNCH(8, 2); else MRN_WARP_LAUNCH(8, 1); }
#undef MRN_WARP_LAUNCH
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

// Coil group of the lane-per-coil interpolation: all coils of the widest
// slice up to 32 lanes (2D) or 16 (3D: a 4^3 tile region with its halo then
// fits three CTAs per SM), or the caller's coil_group.
static int interp_reg_sub(const mrn_plan* P, int* cg_out, int* ng_out) {
  const int cap = P->ndim == 3 ? 16 : 32;
  int cg = P->coil_group_req > 0 ? std::min(P->coil_group_req, P->max_coil) : std::min(P->max_coil, cap);
  cg = std::max(1, std::min(cg, 32));
  const int ng = (P->max_coil + cg - 1) / cg;
  cg = (P->max_coil + ng - 1) / ng;
  *cg_out = cg;
  *ng_out = ng;
  return cg <= 8 ? 4 : (cg <= 16 ? 2 : 1);
}

static size_t interp_reg_smem(const mrn_plan* P, int sub) {
  const int K = P->kb.ntaps[0];
  size_t cells = 1;
  for (int i = 0; i < P->ndim; ++i) cells *= (size_t)(P->tmax_cells[i] + K - 1);
  return cells * (32 / sub + 1) * sizeof(float2);
}

bool interp_reg_ok(const mrn_plan* P) {
  if (!P->reg_interp || (P->ndim != 2 && P->ndim != 3)) return false;
  int cg, ng;
  const int sub = interp_reg_sub(P, &cg, &ng);
  return interp_reg_smem(P, sub) + kInterpStage * (sizeof(float4) + sizeof(int)) <= 227 * 1024;
}

int launch_interp_reg(mrn_plan* P, const float2* grid, int layout, float2* ksp, float scale,
                      const float2* temporal, cudaStream_t st, EntIO eio) {
  if (P->n_items_interp == 0) return MRN_OK;
  int cg, ng;
  const int sub = interp_reg_sub(P, &cg, &ng);
  const size_t smem = interp_reg_smem(P, sub);
  const dim3 gdim((unsigned)P->n_items_interp, (unsigned)ng);
  const int K = P->kb.ntaps[0];
  int rc = MRN_OK;
#define MRN_IREG_LAUNCH(DD, KK, SS)                                                                 \
  do {                                                                                              \
    auto kern = k_interp_reg<DD, KK, SS>;                                                           \
    rc = prep_attr(kern, smem);                                                                     \
    if (rc == MRN_OK)                                                                               \
      kern<<<gdim, kRegInterpWarps * 32, smem, st>>>(P->d_items_i, P->d_slices, P->kb, P->d_coord_i, \
                                                     P->d_perm_i, grid, layout, ksp, scale, temporal, cg, \
                                                     eio);                                            \
  } while (0)
#define MRN_IREG_SUB(DD, KK)                     \
  if (sub == 4) MRN_IREG_LAUNCH(DD, KK, 4);      \
  else if (sub == 2) MRN_IREG_LAUNCH(DD, KK, 2); \
  else MRN_IREG_LAUNCH(DD, KK, 1)
#define MRN_IREG_K(DD)                      \
  if (K == 5) { MRN_IREG_SUB(DD, 5); }      \
  else if (K == 6) { MRN_IREG_SUB(DD, 6); } \
  else if (K == 7) { MRN_IREG_SUB(DD, 7); } \
  else { MRN_IREG_SUB(DD, 8); }
  if (P->ndim == 2) { MRN_IREG_K(2) }
  else { MRN_IREG_K(3) }
#undef MRN_IREG_K
#undef MRN_IREG_SUB
#undef MRN_IREG_LAUNCH
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_trajgrad_reg(mrn_plan* P, const float2* grid, int layout, const float2* samples, float* out,
                        float scale, cudaStream_t st) {
  if (P->n_items_interp == 0) return MRN_OK;
  int cg, ng;
  const int sub = interp_reg_sub(P, &cg, &ng);
  const size_t smem = interp_reg_smem(P, sub);
  const dim3 gdim((unsigned)P->n_items_interp, (unsigned)ng);
  const int K = P->kb.ntaps[0];
  int rc = MRN_OK;
#define MRN_TG_LAUNCH(DD, KK, SS)                                                                   \
  do {                                                                                              \
    auto kern = k_trajgrad_reg<DD, KK, SS>;                                                         \
    rc = prep_attr(kern, smem);                                                                     \
    if (rc == MRN_OK)                                                                               \
      kern<<<gdim, kRegInterpWarps * 32, smem, st>>>(P->d_items_i, P->d_slices, P->kb, P->d_coord_i, \
                                                     P->d_perm_i, grid, layout, samples, out, scale, cg); \
  } while (0)
#define MRN_TG_SUB(DD, KK)                     \
  if (sub == 4) MRN_TG_LAUNCH(DD, KK, 4);      \
  else if (sub == 2) MRN_TG_LAUNCH(DD, KK, 2); \
  else MRN_TG_LAUNCH(DD, KK, 1)
#define MRN_TG_K(DD)                      \
  if (K == 5) { MRN_TG_SUB(DD, 5); }      \
  else if (K == 6) { MRN_TG_SUB(DD, 6); } \
  else if (K == 7) { MRN_TG_SUB(DD, 7); } \
  else { MRN_TG_SUB(DD, 8); }
  if (P->ndim == 2) { MRN_TG_K(2) }
  else { MRN_TG_K(3) }
#undef MRN_TG_K
#undef MRN_TG_SUB
#undef MRN_TG_LAUNCH
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

bool ent_path_ok(const mrn_plan* P) {
  return P->ent_ok && P->ndim == 2 && P->use_fast && fast_path_ok(P, false) && interp_reg_ok(P) &&
         fast_path_ok(P, true) && P->warp_grid && grid_reg_ok(P) && P->cap_ksp_ent >= P->n_entries_grid * P->max_coil;
}

bool grid_reg_ok(const mrn_plan* P) {
  return P->reg_grid && P->ndim == 2 && P->tmax_gcells[0] <= kRegTile && P->tmax_gcells[1] <= kRegTile;
}

int launch_grid_reg(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                    int layout, float2* grid, float scale, cudaStream_t st, int ent_stride) {
  if (P->n_items_grid == 0) return MRN_OK;
  int cg = P->coil_group_req > 0 ? std::min(P->coil_group_req, P->max_coil) : P->max_coil;
  cg = std::max(1, std::min(cg, 32));
  const int ng = (P->max_coil + cg - 1) / cg;
  cg = (P->max_coil + ng - 1) / ng;
  // entry streams per warp: 32 lanes / (coil group rounded up to 8, 16 or 32,
  // or the lane count the plan option asks for when that is larger)
  const int lanes = std::max(cg, P->grid_lanes);
  const int sub = lanes <= 8 ? 4 : (lanes <= 16 ? 2 : 1);
  const dim3 gdim((unsigned)P->n_items_grid, (unsigned)ng);
  const int K = P->kb.ntaps[0];
#define MRN_REG_LAUNCH(KK, SS)                                                              \
  k_grid_reg<KK, SS><<<gdim, 64, 0, st>>>(P->d_items_g, P->d_slices, P->kb, P->d_coord_g, \
                                          P->d_perm_g, ksp, dcf, temporal, grid, layout, scale, cg, \
                                          split_out(P), ent_stride)
#define MRN_REG_SUB(KK)                     \
  if (sub == 4) MRN_REG_LAUNCH(KK, 4);      \
  else if (sub == 2) MRN_REG_LAUNCH(KK, 2); \
  else MRN_REG_LAUNCH(KK, 1)
  if (K == 5) { MRN_REG_SUB(5); }
  else if (K == 6) { MRN_REG_SUB(6); }
  else if (K == 7) { MRN_REG_SUB(7); }
  else { MRN_REG_SUB(8); }
#undef MRN_REG_SUB
#undef MRN_REG_LAUNCH
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_grid_fast(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                     int layout, float2* grid, float scale, int cg, int G, int pstride, size_t smem,
                     dim3 gdim, cudaStream_t st) {
  int rc = MRN_OK;
  MRN_FAST_DK(P->ndim, P->kb.ntaps[0], MRN_FAST_G(G, {
    auto kern = k_grid_fast<DD, KK, GG>;
    rc = prep_attr(kern, smem);
    if (rc == MRN_OK)
      kern<<<gdim, kThreads, smem, st>>>(P->d_items_g, P->d_slices, P->kb, P->d_coord_g, P->d_perm_g,
                                         ksp, dcf, temporal, grid, layout, scale, cg, pstride,
                                         split_out(P));
  }));
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

}  // namespace mrn
