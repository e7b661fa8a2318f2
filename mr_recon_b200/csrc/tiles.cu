// Tile kernels: type-2 interpolation (grid -> samples), type-1 gridding
// (samples -> grid) and the trajectory gradient.
//
// Reference: triton_interp/ungrid.py (_ungrid1d..3d, :154-495) and grid.py
// (_grid1d..3d, :158-502). The reference launches one Triton program per
// chunk of points, gathers each point's (next_pow2(W+1))^d neighbourhood with
// masked loads straight from global memory, recomputes the KB weights for
// every batch element, and grids with one global fp32 atomic per tap per
// batch element. Here instead:
//   * samples are pre-sorted into tiles of the oversampled grid (plan.cu);
//   * one CTA takes one work item (a tile, or a chunk of a heavy tile) for a
//     group of coils; the tile (+ halo for interpolation) lives in shared
//     memory, loaded / stored with coalesced row accesses;
//   * G lanes share one sample, each lane owning coils lane, lane+G, ...; the
//     d x (floor(W)+1) 1D KB weights of a sample are computed once,
//     cooperatively by its G lanes, and reused for all coils;
//   * gridding accumulates in shared memory (float atomics) and each tile is
//     written back once with plain coalesced stores -- no global atomics and
//     no zero fill of the output. Tiles so dense that they were split over
//     several CTAs get one partial tile per CTA, summed in item order by a
//     reduction pass, so a tile's parts add in the same order on every run.
// Tap selection and weights follow the reference exactly: taps j = lo + q,
// lo = ceil(u - W/2), valid iff |(float)j - u| <= W/2 (kernels.py:268-393),
// weight = prod_d KB(|j_d - u_d| / (W_d/2)) (norm '1'), cells wrap circularly.
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"
#include "tile_util.cuh"

namespace mrn {

using TileFrame = Frame;

__device__ __forceinline__ TileFrame tile_frame(const SliceGeom& g, int tile, int D,
                                                bool gridding = false) {
  TileFrame f;
  int rem = tile;
  int tc[kMaxDim] = {0, 0, 0};
  const int* nts = gridding ? g.gntile : g.ntile;
  for (int i = D - 1; i >= 0; --i) {
    tc[i] = rem % nts[i];
    rem /= nts[i];
  }
  for (int i = 0; i < kMaxDim; ++i) {
    if (i < D) {
      f.org[i] = tile_begin(tc[i], g.nos[i], nts[i]);
      f.size[i] = tile_begin(tc[i] + 1, g.nos[i], nts[i]) - f.org[i];
    } else {
      f.org[i] = 0;
      f.size[i] = 1;
    }
  }
  return f;
}

template <int D>
__device__ __forceinline__ float coord_of(const float4& c, int i) {
  return i == 0 ? c.x : (i == 1 ? c.y : c.z);
}

// Load the region [org, org + ext) (centred cells, wrapped) of ncg coil planes
// into shared memory [c][cells] with plane stride pstride. One warp per row.
template <int D>
__device__ __forceinline__ void load_region(float2* __restrict__ tile, const float2* __restrict__ grid,
                                            int64_t goff, int64_t gos, const SliceGeom& g,
                                            const int* org, const int* ext, const int* hs, int ncg,
                                            int pstride) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int inner = ext[D - 1];
  int outer = 1;
  for (int i = 0; i < D - 1; ++i) outer *= ext[i];
  const int nrows = ncg * outer;
  for (int row = warp; row < nrows; row += kWarps) {
    const int c = row / outer;
    int rr = row - c * outer;
    int64_t base = 0;
    int lbase = 0;
    // outer dims, last-but-one fastest
    int l[kMaxDim] = {0, 0, 0};
    for (int i = D - 2; i >= 0; --i) {
      l[i] = rr % ext[i];
      rr /= ext[i];
    }
    for (int i = 0; i < D - 1; ++i) {
      const int s = pos_mod(org[i] + l[i] - hs[i], g.nos[i]);
      base = base * g.nos[i] + s;
      lbase = lbase * ext[i] + l[i];
    }
    base *= g.nos[D - 1];
    lbase *= inner;
    const float2* src = grid + goff + (int64_t)c * gos + base;
    float2* dst = tile + c * pstride + lbase;
    const int n = g.nos[D - 1];
    for (int q = lane; q < inner; q += 32) {
      const int s = pos_mod(org[D - 1] + q - hs[D - 1], n);
      dst[q] = __ldg(src + s);
    }
  }
}

// ---------------------------------------------------------------------------
// Interpolation
// ---------------------------------------------------------------------------
template <int D, int G, int KM>
__global__ void __launch_bounds__(kThreads)
k_interp(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
         const float4* __restrict__ coord, const int* __restrict__ perm,
         const float2* __restrict__ grid, int layout, float2* __restrict__ ksp, float scale,
         const float2* __restrict__ temporal, int cg, int pstride) {
  constexpr int SLOTS = 32 / G;
  constexpr int CPL = (G >= 32) ? 2 : 1;  // coils per lane: cg <= G, or cg <= 64 for G = 32
  extern __shared__ float4 smem_f4[];
  float2* tile = reinterpret_cast<float2*>(smem_f4);
  float* wts = reinterpret_cast<float*>(tile + (size_t)cg * pstride);

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom& g = sl[it.slice];
  const int c0 = blockIdx.y * cg;
  const int ncoil = g.ncoil;
  if (c0 >= ncoil) return;
  const int ncg = min(cg, ncoil - c0);
  const TileFrame f = tile_frame(g, it.tile, D);
  int ext[kMaxDim], hs[kMaxDim];
  for (int i = 0; i < kMaxDim; ++i) {
    ext[i] = i < D ? f.size[i] + kb.ntaps[i] - 1 : 1;
    hs[i] = (i < D && layout == kInternal) ? g.hshift[i] : 0;
  }
  const int64_t goff = (layout == kInternal ? g.grid_off : g.ugrid_off) + (int64_t)c0 * g.gos;
  load_region<D>(tile, grid, goff, g.gos, g, f.org, ext, hs, ncg, pstride);
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / G, lg = lane % G;
  float* ws = wts + warp * (D * KM * SLOTS);
  const int64_t m = g.m;
  for (int base = warp * SLOTS; base < it.count; base += kWarps * SLOTS) {
    const int el = base + slot;
    const bool active = el < it.count;
    const int e = it.start + (active ? el : 0);
    const float4 c4 = coord[e];
    int lo[kMaxDim], kf[kMaxDim], kl[kMaxDim], l0[kMaxDim];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const float u = coord_of<D>(c4, i);
      const float r = kb.radius[i];
      lo[i] = (int)ceilf(__fsub_rn(u, r));
      l0[i] = pos_mod(lo[i], g.nos[i]) - f.org[i];
      kf[i] = KM;
      kl[i] = -1;
      for (int q = 0; q < kb.ntaps[i]; ++q) {
        const float dx = __fsub_rn((float)(lo[i] + q), u);
        if (fabsf(dx) <= r) { kf[i] = min(kf[i], q); kl[i] = q; }
      }
    }
    // cooperative 1D weights: lane lg of the slot computes entries lg, lg+G, ...
    for (int t = lg; t < D * KM; t += G) {
      const int i = t / KM, q = t - i * KM;
      float w = 0.f;
      if (active && q < kb.ntaps[i]) {
        const float u = coord_of<D>(c4, i);
        const float adx = fabsf(__fsub_rn((float)(lo[i] + q), u));
        if (adx <= kb.radius[i]) w = kb_tap(adx, kb.radius[i], kb.betad[i]);
      }
      ws[t * SLOTS + slot] = w;
    }
    __syncwarp();
    float2 acc[CPL];
#pragma unroll
    for (int q = 0; q < CPL; ++q) acc[q] = make_float2(0.f, 0.f);
    if (active) {
      if (D == 1) {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const float w = ws[a * SLOTS + slot];
          const int cell = l0[0] + a;
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const int c = lg + q * G;
            if (c < ncg) {
              const float2 v = tile[c * pstride + cell];
              acc[q].x = fmaf(w, v.x, acc[q].x);
              acc[q].y = fmaf(w, v.y, acc[q].y);
            }
          }
        }
      } else if (D == 2) {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const float wa = ws[a * SLOTS + slot];
          const int rowc = (l0[0] + a) * ext[1] + l0[1];
          for (int b = kf[1]; b <= kl[1]; ++b) {
            const float w = wa * ws[(KM + b) * SLOTS + slot];
            const int cell = rowc + b;
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
              const int c = lg + q * G;
              if (c < ncg) {
                const float2 v = tile[c * pstride + cell];
                acc[q].x = fmaf(w, v.x, acc[q].x);
                acc[q].y = fmaf(w, v.y, acc[q].y);
              }
            }
          }
        }
      } else {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const float wa = ws[a * SLOTS + slot];
          for (int b = kf[1]; b <= kl[1]; ++b) {
            const float wab = wa * ws[(KM + b) * SLOTS + slot];
            const int rowc = ((l0[0] + a) * ext[1] + (l0[1] + b)) * ext[2] + l0[2];
            for (int z = kf[2]; z <= kl[2]; ++z) {
              const float w = wab * ws[(2 * KM + z) * SLOTS + slot];
              const int cell = rowc + z;
#pragma unroll
              for (int q = 0; q < CPL; ++q) {
                const int c = lg + q * G;
                if (c < ncg) {
                  const float2 v = tile[c * pstride + cell];
                  acc[q].x = fmaf(w, v.x, acc[q].x);
                  acc[q].y = fmaf(w, v.y, acc[q].y);
                }
              }
            }
          }
        }
      }
      const int64_t lp = perm[e] - g.pt_off;
      float2 h = make_float2(scale, 0.f);
      if (temporal) {
        const float2 t = temporal[g.pt_off + lp];
        h = make_float2(scale * t.x, scale * t.y);
      }
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const int c = lg + q * G;
        if (c < ncg) {
          float2* dst = ksp + g.ksp_off + (int64_t)(c0 + c) * m + lp;
          const float2 v = make_float2(acc[q].x * h.x - acc[q].y * h.y, acc[q].x * h.y + acc[q].y * h.x);
          if (temporal) {
            const float2 o = *dst;
            *dst = make_float2(o.x + v.x, o.y + v.y);
          } else {
            *dst = v;
          }
        }
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Gridding
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void tile_storage(const SliceGeom& g, const TileFrame& f, const int* hs,
                                             int cell, int64_t* lin) {
  int l[kMaxDim] = {0, 0, 0};
  int rr = cell;
  for (int i = D - 1; i >= 0; --i) {
    l[i] = rr % f.size[i];
    rr /= f.size[i];
  }
  int64_t s = 0;
  for (int i = 0; i < D; ++i) s = s * g.nos[i] + pos_mod(f.org[i] + l[i] - hs[i], g.nos[i]);
  *lin = s;
}

template <int D, int G, int KM>
__global__ void __launch_bounds__(kThreads)
k_grid(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
       const float4* __restrict__ coord, const int* __restrict__ perm,
       const float2* __restrict__ ksp, const float* __restrict__ dcf,
       const float2* __restrict__ temporal, float2* __restrict__ grid, int layout, float scale,
       int cg, int pstride, SplitOut so) {
  constexpr int SLOTS = 32 / G;
  constexpr int CPL = (G >= 32) ? 2 : 1;
  extern __shared__ float4 smem_f4[];
  float* acc_re = reinterpret_cast<float*>(smem_f4);
  float* acc_im = acc_re + (size_t)cg * pstride;
  float* wts = acc_im + (size_t)cg * pstride;
  int* locs = reinterpret_cast<int*>(wts + kWarps * D * KM * SLOTS);

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom& g = sl[it.slice];
  const int c0 = blockIdx.y * cg;
  if (c0 >= g.ncoil) return;
  const int ncg = min(cg, g.ncoil - c0);
  const TileFrame f = tile_frame(g, it.tile, D, true);
  int cells = 1;
  for (int i = 0; i < D; ++i) cells *= f.size[i];
  for (int idx = threadIdx.x; idx < ncg * pstride; idx += kThreads) {
    acc_re[idx] = 0.f;
    acc_im[idx] = 0.f;
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / G, lg = lane % G;
  float* ws = wts + warp * (D * KM * SLOTS);
  int* ls = locs + warp * (D * KM * SLOTS);
  const int64_t m = g.m;
  for (int base = warp * SLOTS; base < it.count; base += kWarps * SLOTS) {
    const int el = base + slot;
    const bool active = el < it.count;
    const int e = it.start + (active ? el : 0);
    const float4 c4 = coord[e];
    int lo[kMaxDim], kf[kMaxDim], kl[kMaxDim];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const float u = coord_of<D>(c4, i);
      const float r = kb.radius[i];
      lo[i] = (int)ceilf(__fsub_rn(u, r));
      kf[i] = KM;
      kl[i] = -1;
      for (int q = 0; q < kb.ntaps[i]; ++q) {
        const float dx = __fsub_rn((float)(lo[i] + q), u);
        if (fabsf(dx) <= r) { kf[i] = min(kf[i], q); kl[i] = q; }
      }
    }
    for (int t = lg; t < D * KM; t += G) {
      const int i = t / KM, q = t - i * KM;
      float w = 0.f;
      int loc = -1;
      if (active && q < kb.ntaps[i]) {
        const float u = coord_of<D>(c4, i);
        const float adx = fabsf(__fsub_rn((float)(lo[i] + q), u));
        if (adx <= kb.radius[i]) {
          w = kb_tap(adx, kb.radius[i], kb.betad[i]);
          const int l = pos_mod(lo[i] + q, g.nos[i]) - f.org[i];
          loc = (l >= 0 && l < f.size[i]) ? l : -1;
        }
      }
      ws[t * SLOTS + slot] = w;
      ls[t * SLOTS + slot] = loc;
    }
    __syncwarp();
    if (active) {
      const int64_t lp = perm[e] - g.pt_off;
      float vs = scale;
      if (dcf) vs *= dcf[g.pt_off + lp];
      float2 h = make_float2(vs, 0.f);
      if (temporal) {  // conj(temporal) * dcf * scale
        const float2 t = temporal[g.pt_off + lp];
        h = make_float2(vs * t.x, -vs * t.y);
      }
      float2 v[CPL];
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const int c = lg + q * G;
        v[q] = make_float2(0.f, 0.f);
        if (c < ncg) {
          const float2 a = __ldg(ksp + g.ksp_off + (int64_t)(c0 + c) * m + lp);
          v[q] = make_float2(a.x * h.x - a.y * h.y, a.x * h.y + a.y * h.x);
        }
      }
      if (D == 1) {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const int la = ls[a * SLOTS + slot];
          if (la < 0) continue;
          const float w = ws[a * SLOTS + slot];
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const int c = lg + q * G;
            if (c < ncg) {
              atomicAdd(acc_re + c * pstride + la, w * v[q].x);
              atomicAdd(acc_im + c * pstride + la, w * v[q].y);
            }
          }
        }
      } else if (D == 2) {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const int la = ls[a * SLOTS + slot];
          if (la < 0) continue;
          const float wa = ws[a * SLOTS + slot];
          for (int b = kf[1]; b <= kl[1]; ++b) {
            const int lb = ls[(KM + b) * SLOTS + slot];
            if (lb < 0) continue;
            const float w = wa * ws[(KM + b) * SLOTS + slot];
            const int cell = la * f.size[1] + lb;
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
              const int c = lg + q * G;
              if (c < ncg) {
                atomicAdd(acc_re + c * pstride + cell, w * v[q].x);
                atomicAdd(acc_im + c * pstride + cell, w * v[q].y);
              }
            }
          }
        }
      } else {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const int la = ls[a * SLOTS + slot];
          if (la < 0) continue;
          const float wa = ws[a * SLOTS + slot];
          for (int b = kf[1]; b <= kl[1]; ++b) {
            const int lb = ls[(KM + b) * SLOTS + slot];
            if (lb < 0) continue;
            const float wab = wa * ws[(KM + b) * SLOTS + slot];
            const int rowc = (la * f.size[1] + lb) * f.size[2];
            for (int z = kf[2]; z <= kl[2]; ++z) {
              const int lz = ls[(2 * KM + z) * SLOTS + slot];
              if (lz < 0) continue;
              const float w = wab * ws[(2 * KM + z) * SLOTS + slot];
              const int cell = rowc + lz;
#pragma unroll
              for (int q = 0; q < CPL; ++q) {
                const int c = lg + q * G;
                if (c < ncg) {
                  atomicAdd(acc_re + c * pstride + cell, w * v[q].x);
                  atomicAdd(acc_im + c * pstride + cell, w * v[q].y);
                }
              }
            }
          }
        }
      }
    }
    __syncwarp();
  }
  __syncthreads();

  // write-back: one store per cell (into the item's partial slot for split tiles)
  int hs[kMaxDim];
  for (int i = 0; i < kMaxDim; ++i) hs[i] = (i < D && layout == kInternal) ? g.hshift[i] : 0;
  const int64_t goff = (layout == kInternal ? g.grid_off : g.ugrid_off) + (int64_t)c0 * g.gos;
  const int inner = f.size[D - 1];
  const int outer = cells / inner;
  const int nrows = ncg * outer;
  for (int row = warp; row < nrows; row += kWarps) {
    const int c = row / outer;
    const int orow = row - c * outer;
    int64_t base;
    tile_storage<D>(g, f, hs, orow * inner, &base);
    base -= pos_mod(f.org[D - 1] - hs[D - 1], g.nos[D - 1]);
    float2* dst = grid + goff + (int64_t)c * g.gos + base;
    const float* sre = acc_re + c * pstride + orow * inner;
    const float* sim = acc_im + c * pstride + orow * inner;
    for (int q = lane; q < inner; q += 32) {
      const int s = pos_mod(f.org[D - 1] + q - hs[D - 1], g.nos[D - 1]);
      const float2 v = make_float2(sre[q], sim[q]);
      if (it.split) *split_slot(so, it.split, c0 + c, orow * inner + q) = v;
      else dst[s] = v;
    }
  }
}

// Sum the partial tiles of every split gridding tile in item order and store
// the result. Work units are (split tile, group of kSplitCoils coils); a
// grid of a few CTAs per SM strides over them (the number of split tiles is
// known only on the device, counts[3]), threads over (coil, cell), each
// thread adding the tile's slots first to last with four loads in flight.
// The gridding kernel ran before on the same stream and wrote every slot
// read here (a split tile's items are slots base .. base + n - 1).
constexpr int kSplitCoils = 8;

template <int D>
__global__ void __launch_bounds__(256)
k_reduce_split(const int4* __restrict__ split_tiles, const int* __restrict__ counts,
               const SliceGeom* __restrict__ sl, int ns, int coil_groups, SplitOut so,
               float2* __restrict__ grid, int layout) {
  const int units = counts[3] * coil_groups;
  for (int unit = blockIdx.x; unit < units; unit += gridDim.x) {
    const int4 sp = split_tiles[unit / coil_groups];
    const int t = sp.x, base = sp.y, nparts = sp.z;
    int s = 0;
    {
      int lo = 0, hi = ns - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (sl[mid].gtile_base <= t) lo = mid; else hi = mid - 1;
      }
      s = lo;
    }
    const SliceGeom& g = sl[s];
    const TileFrame f = tile_frame(g, t - g.gtile_base, D, true);
    int hs[kMaxDim];
    for (int i = 0; i < kMaxDim; ++i) hs[i] = (i < D && layout == kInternal) ? g.hshift[i] : 0;
    int cells = 1;
    for (int i = 0; i < D; ++i) cells *= f.size[i];
    const int cbeg = (unit % coil_groups) * kSplitCoils;
    const int ncl = min(kSplitCoils, g.ncoil - cbeg);
    const int64_t goff = (layout == kInternal ? g.grid_off : g.ugrid_off) + (int64_t)cbeg * g.gos;
    for (int idx = threadIdx.x; idx < ncl * cells; idx += blockDim.x) {
      const int c = idx / cells, cell = idx - c * cells;
      const float2* src = split_slot(so, base + 1, cbeg + c, cell);
      float2 acc = make_float2(0.f, 0.f);
      int q = 0;
      for (; q + 4 <= nparts; q += 4) {
        float2 v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = src[(int64_t)(q + k) * so.slot_stride];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          acc.x += v[k].x;
          acc.y += v[k].y;
        }
      }
      for (; q < nparts; ++q) {
        const float2 v = src[(int64_t)q * so.slot_stride];
        acc.x += v.x;
        acc.y += v.y;
      }
      int64_t lin;
      tile_storage<D>(g, f, hs, cell, &lin);
      grid[goff + (int64_t)c * g.gos + lin] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
// Trajectory gradient: out[p, i] += scale * du_i/dk_i *
//   Re sum_c conj(S[c,p]) * sum_taps dW/du_i * G[c, tap]
// ---------------------------------------------------------------------------
template <int D, int G, int KM>
__global__ void __launch_bounds__(kThreads)
k_traj_grad(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
            const float4* __restrict__ coord, const int* __restrict__ perm,
            const float2* __restrict__ grid, int layout, const float2* __restrict__ samp,
            float* __restrict__ out, float scale, int cg, int pstride) {
  constexpr int SLOTS = 32 / G;
  constexpr int CPL = (G >= 32) ? 2 : 1;
  extern __shared__ float4 smem_f4[];
  float2* tile = reinterpret_cast<float2*>(smem_f4);
  float* wts = reinterpret_cast<float*>(tile + (size_t)cg * pstride);
  float* dws = wts + kWarps * D * KM * SLOTS;

  const Item it = items[blockIdx.x];
  if (it.slice < 0) return;  // padding past the real items
  const SliceGeom& g = sl[it.slice];
  const int c0 = blockIdx.y * cg;
  if (c0 >= g.ncoil) return;
  const int ncg = min(cg, g.ncoil - c0);
  const TileFrame f = tile_frame(g, it.tile, D);
  int ext[kMaxDim], hs[kMaxDim];
  for (int i = 0; i < kMaxDim; ++i) {
    ext[i] = i < D ? f.size[i] + kb.ntaps[i] - 1 : 1;
    hs[i] = (i < D && layout == kInternal) ? g.hshift[i] : 0;
  }
  const int64_t goff = (layout == kInternal ? g.grid_off : g.ugrid_off) + (int64_t)c0 * g.gos;
  load_region<D>(tile, grid, goff, g.gos, g, f.org, ext, hs, ncg, pstride);
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / G, lg = lane % G;
  float* ws = wts + warp * (D * KM * SLOTS);
  float* dw = dws + warp * (D * KM * SLOTS);
  const int64_t m = g.m;
  for (int base = warp * SLOTS; base < it.count; base += kWarps * SLOTS) {
    const int el = base + slot;
    const bool active = el < it.count;
    const int e = it.start + (active ? el : 0);
    const float4 c4 = coord[e];
    int lo[kMaxDim], kf[kMaxDim], kl[kMaxDim], l0[kMaxDim];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const float u = coord_of<D>(c4, i);
      const float r = kb.radius[i];
      lo[i] = (int)ceilf(__fsub_rn(u, r));
      l0[i] = pos_mod(lo[i], g.nos[i]) - f.org[i];
      kf[i] = KM;
      kl[i] = -1;
      for (int q = 0; q < kb.ntaps[i]; ++q) {
        const float dx = __fsub_rn((float)(lo[i] + q), u);
        if (fabsf(dx) <= r) { kf[i] = min(kf[i], q); kl[i] = q; }
      }
    }
    for (int t = lg; t < D * KM; t += G) {
      const int i = t / KM, q = t - i * KM;
      float w = 0.f, d = 0.f;
      if (active && q < kb.ntaps[i]) {
        const float u = coord_of<D>(c4, i);
        const float dx = __fsub_rn((float)(lo[i] + q), u);
        if (fabsf(dx) <= kb.radius[i]) {
          w = kb_tap(fabsf(dx), kb.radius[i], kb.betad[i]);
          d = kb_tap_du(dx, kb.radius[i], kb.betad[i]);
        }
      }
      ws[t * SLOTS + slot] = w;
      dw[t * SLOTS + slot] = d;
    }
    __syncwarp();
    float gsum[kMaxDim] = {0.f, 0.f, 0.f};
    if (active) {
      const int64_t lp = perm[e] - g.pt_off;
      float2 sv[CPL];
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const int c = lg + q * G;
        sv[q] = c < ncg ? __ldg(samp + g.ksp_off + (int64_t)(c0 + c) * m + lp) : make_float2(0.f, 0.f);
      }
      float2 acc[CPL][kMaxDim];
#pragma unroll
      for (int q = 0; q < CPL; ++q)
#pragma unroll
        for (int i = 0; i < kMaxDim; ++i) acc[q][i] = make_float2(0.f, 0.f);
      if (D == 1) {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const float d0 = dw[a * SLOTS + slot];
          const int cell = l0[0] + a;
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const int c = lg + q * G;
            if (c < ncg) {
              const float2 v = tile[c * pstride + cell];
              acc[q][0].x = fmaf(d0, v.x, acc[q][0].x);
              acc[q][0].y = fmaf(d0, v.y, acc[q][0].y);
            }
          }
        }
      } else if (D == 2) {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const float wa = ws[a * SLOTS + slot], da = dw[a * SLOTS + slot];
          const int rowc = (l0[0] + a) * ext[1] + l0[1];
          for (int b = kf[1]; b <= kl[1]; ++b) {
            const float wb = ws[(KM + b) * SLOTS + slot], db = dw[(KM + b) * SLOTS + slot];
            const float g0 = da * wb, g1 = wa * db;
            const int cell = rowc + b;
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
              const int c = lg + q * G;
              if (c < ncg) {
                const float2 v = tile[c * pstride + cell];
                acc[q][0].x = fmaf(g0, v.x, acc[q][0].x);
                acc[q][0].y = fmaf(g0, v.y, acc[q][0].y);
                acc[q][1].x = fmaf(g1, v.x, acc[q][1].x);
                acc[q][1].y = fmaf(g1, v.y, acc[q][1].y);
              }
            }
          }
        }
      } else {
        for (int a = kf[0]; a <= kl[0]; ++a) {
          const float wa = ws[a * SLOTS + slot], da = dw[a * SLOTS + slot];
          for (int b = kf[1]; b <= kl[1]; ++b) {
            const float wb = ws[(KM + b) * SLOTS + slot], db = dw[(KM + b) * SLOTS + slot];
            const int rowc = ((l0[0] + a) * ext[1] + (l0[1] + b)) * ext[2] + l0[2];
            for (int z = kf[2]; z <= kl[2]; ++z) {
              const float wz = ws[(2 * KM + z) * SLOTS + slot], dz = dw[(2 * KM + z) * SLOTS + slot];
              const float g0 = da * wb * wz, g1 = wa * db * wz, g2 = wa * wb * dz;
              const int cell = rowc + z;
#pragma unroll
              for (int q = 0; q < CPL; ++q) {
                const int c = lg + q * G;
                if (c < ncg) {
                  const float2 v = tile[c * pstride + cell];
                  acc[q][0].x = fmaf(g0, v.x, acc[q][0].x);
                  acc[q][0].y = fmaf(g0, v.y, acc[q][0].y);
                  acc[q][1].x = fmaf(g1, v.x, acc[q][1].x);
                  acc[q][1].y = fmaf(g1, v.y, acc[q][1].y);
                  acc[q][2].x = fmaf(g2, v.x, acc[q][2].x);
                  acc[q][2].y = fmaf(g2, v.y, acc[q][2].y);
                }
              }
            }
          }
        }
      }
      // Re(conj(S) * acc) = S.x acc.x + S.y acc.y
#pragma unroll
      for (int q = 0; q < CPL; ++q)
#pragma unroll
        for (int i = 0; i < D; ++i) gsum[i] += sv[q].x * acc[q][i].x + sv[q].y * acc[q][i].y;
    }
    // reduce over the G lanes of the slot
#pragma unroll
    for (int i = 0; i < D; ++i) {
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) gsum[i] += __shfl_xor_sync(0xffffffffu, gsum[i], o);
    }
    if (active && lg == 0) {
      const int64_t p = perm[e];
#pragma unroll
      for (int i = 0; i < D; ++i) atomicAdd(out + p * D + i, gsum[i] * scale * g.scale[i]);
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
static int pick_g(int cg) {
  if (cg <= 1) return 1;
  if (cg <= 2) return 2;
  if (cg <= 4) return 4;
  if (cg <= 8) return 8;
  if (cg <= 16) return 16;
  return 32;
}

static constexpr size_t kSmemMax = 227 * 1024;

struct Layout {
  int cg;
  int pstride;
  size_t smem;
};

// Shared-memory layout for one kernel kind: 0 interp, 1 grid, 2 traj grad.
static Layout plan_layout(const mrn_plan* P, int kind, bool fast = false) {
  const int D = P->ndim;
  int64_t cells = 1;
  for (int i = 0; i < D; ++i)
    cells *= (kind == 1) ? P->tmax_gcells[i] : (P->tmax_cells[i] + P->kb.ntaps[i] - 1);
  const int pstride = (int)(cells | 1);
  const int KM = P->tap_max;
  int cg;
  if (P->coil_group_req > 0) {
    cg = std::max(1, std::min(P->coil_group_req, P->max_coil));
  } else {
    // about 76 KB of tile data per CTA (three CTAs per SM), at most 64 coils,
    // coil groups balanced (same count, fewest coils per group)
    const size_t target = 76 * 1024;
    cg = (int)std::max<size_t>(1, target / ((size_t)pstride * 8));
    cg = std::min(std::min(cg, 64), P->max_coil);
    const int ng = (P->max_coil + cg - 1) / cg;
    cg = (P->max_coil + ng - 1) / ng;
  }
  Layout L{};
  for (;;) {
    const int G = pick_g(cg);
    const int slots = 32 / G;
    size_t per_warp = (size_t)D * KM * slots * 4;
    size_t fixed = fast ? 0 : kWarps * per_warp * (kind == 0 ? 1 : 2);
    size_t data = (size_t)cg * pstride * 8;
    size_t total = fixed + data;
    if (total <= kSmemMax || cg == 1) {
      L.cg = cg;
      L.pstride = pstride;
      L.smem = total;
      break;
    }
    cg = std::max(1, (int)((kSmemMax - fixed) / ((size_t)pstride * 8)));
    if (cg <= 0) cg = 1;
  }
  return L;
}

template <class K>
static int prepare(K kernel, size_t smem) {
  return set_dynamic_smem(kernel, smem);
}

#define MRN_DISPATCH_G(G_, ...)                     \
  switch (G_) {                                     \
    case 1: { constexpr int GG = 1; __VA_ARGS__; } break;   \
    case 2: { constexpr int GG = 2; __VA_ARGS__; } break;   \
    case 4: { constexpr int GG = 4; __VA_ARGS__; } break;   \
    case 8: { constexpr int GG = 8; __VA_ARGS__; } break;   \
    case 16: { constexpr int GG = 16; __VA_ARGS__; } break; \
    default: { constexpr int GG = 32; __VA_ARGS__; } break; \
  }

#define MRN_DISPATCH_DK(D_, KM_, ...)                                       \
  do {                                                                      \
    if ((D_) == 1 && (KM_) == 8) { constexpr int DD = 1, KK = 8; __VA_ARGS__; }        \
    else if ((D_) == 1) { constexpr int DD = 1, KK = 16; __VA_ARGS__; }                \
    else if ((D_) == 2 && (KM_) == 8) { constexpr int DD = 2, KK = 8; __VA_ARGS__; }   \
    else if ((D_) == 2) { constexpr int DD = 2, KK = 16; __VA_ARGS__; }                \
    else if ((KM_) == 8) { constexpr int DD = 3, KK = 8; __VA_ARGS__; }                \
    else { constexpr int DD = 3, KK = 16; __VA_ARGS__; }                               \
  } while (0)

int launch_interp(mrn_plan* P, const float2* grid, GridLayout layout, float2* ksp, float scale,
                  const float2* temporal, cudaStream_t st) {
  if (P->n_items_interp == 0) return MRN_OK;
  const bool fast = P->use_fast && fast_path_ok(P, false);
  const Layout L = plan_layout(P, 0, fast);
  const int G = pick_g(L.cg);
  dim3 gridDim((unsigned)P->n_items_interp, (unsigned)((P->max_coil + L.cg - 1) / L.cg));
  if (fast && interp_reg_ok(P))
    return launch_interp_reg(P, grid, (int)layout, ksp, scale, temporal, st);
  if (fast && P->wtab_ok && P->use_wtab)
    return launch_interp_tab(P, grid, (int)layout, ksp, scale, temporal, L.cg, G, L.pstride, L.smem,
                             gridDim, st);
  if (fast)
    return launch_interp_fast(P, grid, (int)layout, ksp, scale, temporal, L.cg, G, L.pstride, L.smem,
                              gridDim, st);
  int rc = MRN_OK;
  MRN_DISPATCH_DK(P->ndim, P->tap_max, MRN_DISPATCH_G(G, {
    auto kern = k_interp<DD, GG, KK>;
    rc = prepare(kern, L.smem);
    if (rc == MRN_OK)
      kern<<<gridDim, kThreads, L.smem, st>>>(P->d_items_i, P->d_slices, P->kb, P->d_coord_i,
                                              P->d_perm_i, grid, (int)layout, ksp, scale, temporal,
                                              L.cg, L.pstride);
  }));
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_grid(mrn_plan* P, const float2* ksp, const float* dcf, GridLayout layout, float2* grid,
                float scale, cudaStream_t st) {
  return launch_grid_t(P, ksp, dcf, nullptr, layout, grid, scale, st);
}

int launch_reduce_split(mrn_plan* P, GridLayout layout, float2* grid, cudaStream_t st) {
  if (P->n_split == 0) return MRN_OK;
  const int groups = (P->max_coil + kSplitCoils - 1) / kSplitCoils;
  const int64_t units = P->n_split * groups;
  const unsigned nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>(units, 4 * (int64_t)P->sm_count));
  const SplitOut so = split_out(P);
  if (P->ndim == 1)
    k_reduce_split<1><<<nb, 256, 0, st>>>(P->d_split_tiles, P->d_counts, P->d_slices, P->nslices, groups, so, grid, (int)layout);
  else if (P->ndim == 2)
    k_reduce_split<2><<<nb, 256, 0, st>>>(P->d_split_tiles, P->d_counts, P->d_slices, P->nslices, groups, so, grid, (int)layout);
  else
    k_reduce_split<3><<<nb, 256, 0, st>>>(P->d_split_tiles, P->d_counts, P->d_slices, P->nslices, groups, so, grid, (int)layout);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

// Items that own their tile store it; items of split tiles store partial
// tiles, which the reduction pass afterwards sums into the grid.
static int launch_grid_items(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                             GridLayout layout, float2* grid, float scale, cudaStream_t st) {
  const bool fast = P->use_fast && fast_path_ok(P, true);
  const Layout L = plan_layout(P, 1, fast);
  const int G = pick_g(L.cg);
  dim3 gridDim((unsigned)P->n_items_grid, (unsigned)((P->max_coil + L.cg - 1) / L.cg));
  if (fast && P->ndim == 3 && grid_reg3_ok(P))
    return launch_grid_reg3(P, ksp, dcf, temporal, (int)layout, grid, scale, st);
  if (fast && P->ndim == 2 && P->warp_grid && grid_reg_ok(P))
    return launch_grid_reg(P, ksp, dcf, temporal, (int)layout, grid, scale, st);
  if (fast && P->ndim == 2 && P->warp_grid && P->wtab_ok && P->use_wtab)
    return launch_grid_warp_tab(P, ksp, dcf, temporal, (int)layout, grid, scale, st);
  if (fast && P->ndim == 2 && P->warp_grid)
    return launch_grid_warp(P, ksp, dcf, temporal, (int)layout, grid, scale, st);
  if (fast)
    return launch_grid_fast(P, ksp, dcf, temporal, (int)layout, grid, scale, L.cg, G, L.pstride, L.smem,
                            gridDim, st);
  int rc = MRN_OK;
  const SplitOut so = split_out(P);
  MRN_DISPATCH_DK(P->ndim, P->tap_max, MRN_DISPATCH_G(G, {
    auto kern = k_grid<DD, GG, KK>;
    rc = prepare(kern, L.smem);
    if (rc == MRN_OK)
      kern<<<gridDim, kThreads, L.smem, st>>>(P->d_items_g, P->d_slices, P->kb, P->d_coord_g,
                                              P->d_perm_g, ksp, dcf, temporal, grid, (int)layout,
                                              scale, L.cg, L.pstride, so);
  }));
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_grid_t(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
                  GridLayout layout, float2* grid, float scale, cudaStream_t st) {
  if (P->n_items_grid == 0) return MRN_OK;
  const int rc = launch_grid_items(P, ksp, dcf, temporal, layout, grid, scale, st);
  if (rc != MRN_OK) return rc;
  return launch_reduce_split(P, layout, grid, st);
}

int launch_traj_grad(mrn_plan* P, const float2* grid, GridLayout layout, const float2* samples,
                     float* out, float scale, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, (size_t)P->n_trj * sizeof(float), st);
  if (e != cudaSuccess) return cuda_fail(e);
  if (P->n_items_interp == 0) return MRN_OK;
  if (P->use_fast && fast_path_ok(P, false) && interp_reg_ok(P))
    return launch_trajgrad_reg(P, grid, (int)layout, samples, out, scale, st);
  const Layout L = plan_layout(P, 2);
  const int G = pick_g(L.cg);
  dim3 gridDim((unsigned)P->n_items_interp, (unsigned)((P->max_coil + L.cg - 1) / L.cg));
  int rc = MRN_OK;
  MRN_DISPATCH_DK(P->ndim, P->tap_max, MRN_DISPATCH_G(G, {
    auto kern = k_traj_grad<DD, GG, KK>;
    rc = prepare(kern, L.smem);
    if (rc == MRN_OK)
      kern<<<gridDim, kThreads, L.smem, st>>>(P->d_items_i, P->d_slices, P->kb, P->d_coord_i,
                                              P->d_perm_i, grid, (int)layout, samples, out, scale,
                                              L.cg, L.pstride);
  }));
  if (rc != MRN_OK) return rc;
  e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

}  // namespace mrn
