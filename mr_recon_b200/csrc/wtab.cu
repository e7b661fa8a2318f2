// 2D weight tables and the kernels that use them.
//
// The Kaiser-Bessel weights of a sample depend only on the trajectory, which
// is bound once per plan and reused by every forward / adjoint / normal call
// (a CG-SENSE solve makes ~40 of them). mrn_plan_set_traj therefore evaluates
// them once (same float32 tap selection and weights as the fast kernels) and
// stores, per interpolation sample and per gridding entry in sorted order:
//   meta = {first local cell dim 0, first local cell dim 1, taps dim 0, taps dim 1}
//   w    = the valid 1D weights of each dim, compacted to the front (8 slots each)
// For gridding the valid taps are also restricted to the tile the entry
// belongs to, so the kernels run an exact tap count with no predicated-off
// shared-memory traffic. Used in 2D when K = floor(W)+1 <= 8; 3D keeps
// computing weights on the fly (its tables would not fit in L2 and would add
// HBM traffic comparable to the data).
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"
#include "tile_util.cuh"

namespace mrn {

namespace {

__device__ __forceinline__ int wrap1(int a, int n) {
  a = a < 0 ? a + n : a;
  return a >= n ? a - n : a;
}

__device__ __forceinline__ int slice_of_tile(const SliceGeom* sl, int ns, int t, bool gridding) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((gridding ? sl[mid].gtile_base : sl[mid].tile_base) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Weights of one dim for a sample at u, taps q = 0..K-1 from lo, restricted to
// local cells [0, size) when OWN (local cell of tap q is st + q); compacted.
__device__ __forceinline__ void dim_table(float u, float r, float inv_r, const KBParams& kb, int K, int st,
                                          int size, bool own, int* first, int* count, float* w8) {
  const int lo = (int)ceilf(__fsub_rn(u, r));
  int q0 = -1, n = 0;
  float tmp[kMaxTaps];
  for (int q = 0; q < K; ++q) {
    const float adx = fabsf(__fsub_rn((float)(lo + q), u));
    bool ok = adx <= r;
    if (own) ok = ok && (st + q) >= 0 && (st + q) < size;
    if (ok) {
      if (q0 < 0) q0 = q;
      tmp[n++] = kb_tap_fast(adx, inv_r, kb);
    }
  }
  for (int j = 0; j < 8; ++j) w8[j] = j < n ? tmp[j] : 0.f;
  *first = st + (q0 < 0 ? 0 : q0);
  *count = n;
}

__global__ void k_wtab(const SliceGeom* __restrict__ sl, int ns, KBParams kb,
                       const float4* __restrict__ coord, const unsigned* __restrict__ key, int64_t n,
                       int gridding, int4* __restrict__ meta, float4* __restrict__ tab) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int t = (int)key[e];
  const int s = slice_of_tile(sl, ns, t, gridding != 0);
  const SliceGeom& g = sl[s];
  int tile = t - (gridding ? g.gtile_base : g.tile_base);
  const int* nts = gridding ? g.gntile : g.ntile;
  int tc[2];
  tc[1] = tile % nts[1];
  tc[0] = tile / nts[1];
  const float4 c4 = coord[e];
  const float u[2] = {c4.x, c4.y};
  int first[2], cnt[2];
  float w[2][8];
  for (int i = 0; i < 2; ++i) {
    const int org = tile_begin(tc[i], g.nos[i], nts[i]);
    const int size = tile_begin(tc[i] + 1, g.nos[i], nts[i]) - org;
    const int lo = (int)ceilf(__fsub_rn(u[i], kb.radius[i]));
    int st = wrap1(lo, g.nos[i]) - org;
    if (gridding && st >= size) st -= g.nos[i];  // footprint wraps into the tile from the end
    dim_table(u[i], kb.radius[i], kb.inv_radius[i], kb, kb.ntaps[i], st, size, gridding != 0,
              &first[i], &cnt[i], w[i]);
  }
  meta[e] = make_int4(first[0], first[1], cnt[0], cnt[1]);
  float4* o = tab + e * 4;
  o[0] = make_float4(w[0][0], w[0][1], w[0][2], w[0][3]);
  o[1] = make_float4(w[0][4], w[0][5], w[0][6], w[0][7]);
  o[2] = make_float4(w[1][0], w[1][1], w[1][2], w[1][3]);
  o[3] = make_float4(w[1][4], w[1][5], w[1][6], w[1][7]);
}

struct Frame2 {
  int org[2];
  int size[2];
};

__device__ __forceinline__ Frame2 frame2(const SliceGeom& g, int tile, bool gridding) {
  const int* nts = gridding ? g.gntile : g.ntile;
  const int t1 = tile % nts[1], t0 = tile / nts[1];
  Frame2 f;
  f.org[0] = tile_begin(t0, g.nos[0], nts[0]);
  f.size[0] = tile_begin(t0 + 1, g.nos[0], nts[0]) - f.org[0];
  f.org[1] = tile_begin(t1, g.nos[1], nts[1]);
  f.size[1] = tile_begin(t1 + 1, g.nos[1], nts[1]) - f.org[1];
  return f;
}

__device__ __forceinline__ void load_w(const float4* __restrict__ tab, int64_t e, float (&wa)[8],
                                       float (&wb)[8]) {
  const float4* p = tab + e * 4;
  const float4 a0 = __ldg(p), a1 = __ldg(p + 1), b0 = __ldg(p + 2), b1 = __ldg(p + 3);
  wa[0] = a0.x; wa[1] = a0.y; wa[2] = a0.z; wa[3] = a0.w;
  wa[4] = a1.x; wa[5] = a1.y; wa[6] = a1.z; wa[7] = a1.w;
  wb[0] = b0.x; wb[1] = b0.y; wb[2] = b0.z; wb[3] = b0.w;
  wb[4] = b1.x; wb[5] = b1.y; wb[6] = b1.z; wb[7] = b1.w;
}

}  // namespace

// ---------------------------------------------------------------------------
// Interpolation with tables: tile + halo in shared memory as k_interp_fast;
// per sample the row sums over the valid columns are formed first and then
// weighted by the row weight.
// ---------------------------------------------------------------------------
template <int G>
__global__ void __launch_bounds__(kThreads)
k_interp_tab(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, int2 ktaps,
             const int4* __restrict__ meta, const float4* __restrict__ tab,
             const int* __restrict__ perm, const float2* __restrict__ grid, int layout,
             float2* __restrict__ ksp, float scale, const float2* __restrict__ temporal, int cg,
             int pstride) {
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
  const int nos0 = gp->nos[0], nos1 = gp->nos[1];
  const int hs0 = layout == kInternal ? gp->hshift[0] : 0;
  const int hs1 = layout == kInternal ? gp->hshift[1] : 0;
  const Frame2 f = frame2(*gp, it.tile, false);
  const int ext0 = f.size[0] + ktaps.x - 1, ext1 = f.size[1] + ktaps.y - 1;
  const int64_t gos = gp->gos;
  const int64_t goff = (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gos;
  const int64_t m = gp->m, pt_off = gp->pt_off, ksp_off = gp->ksp_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / G, lg = lane % G;

  // region load: rows (coil, x) of ext1 cells, wrapped
  {
    const int s_first = wrap1(f.org[1] - hs1, nos1);
    const int nrows = ncg * ext0;
    for (int row = warp; row < nrows; row += kWarps) {
      const int c = row / ext0, l0 = row - c * ext0;
      const int sx = wrap1(f.org[0] + l0 - hs0, nos0);
      const float2* src = grid + goff + (int64_t)c * gos + (int64_t)sx * nos1;
      float2* dst = tile + c * pstride + l0 * ext1;
      for (int q = lane; q < ext1; q += 32) {
        int s = s_first + q;
        while (s >= nos1) s -= nos1;
        dst[q] = __ldg(src + s);
      }
    }
  }
  __syncthreads();

  // one iteration of lookahead on the table row and sample index
  int4 mtN = make_int4(0, 0, 0, 0);
  float waN[8], wbN[8];
  int64_t lpN = 0;
  {
    const int el0 = warp * SLOTS + slot;
    if (el0 < it.count) {
      const int64_t e = it.start + el0;
      mtN = __ldg(meta + e);
      load_w(tab, e, waN, wbN);
      lpN = __ldg(perm + e) - pt_off;
    }
  }
  for (int base = warp * SLOTS; base < it.count; base += STRIDE) {
    const int el = base + slot;
    const int4 mt = mtN;
    float wa[8], wb[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      wa[j] = waN[j];
      wb[j] = wbN[j];
    }
    const int64_t lp = lpN;
    if (el + STRIDE < it.count) {
      const int64_t e = it.start + el + STRIDE;
      mtN = __ldg(meta + e);
      load_w(tab, e, waN, wbN);
      lpN = __ldg(perm + e) - pt_off;
    }
    if (el >= it.count) continue;  // slots diverge only here; no warp-wide ops below
    float2 h = make_float2(scale, 0.f);
    if (temporal) {
      const float2 t = temporal[pt_off + lp];
      h = make_float2(scale * t.x, scale * t.y);
    }
    const int na = mt.z, nb = mt.w;
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int c = lg + q * G;
      if (c >= ncg) break;
      const float2* rp0 = tile + c * pstride + mt.x * ext1 + mt.y;
      float ax = 0.f, ay = 0.f;
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        if (a >= na) break;
        const float2* rp = rp0 + a * ext1;
        float sx = 0.f, sy = 0.f;
#define MRN_ITAP(b)                        \
  {                                        \
    const float2 v = rp[b];                \
    sx = fmaf(wb[b], v.x, sx);             \
    sy = fmaf(wb[b], v.y, sy);             \
  }
        switch (nb) {
          case 8: MRN_ITAP(7)  // fallthrough
          case 7: MRN_ITAP(6)  // fallthrough
          case 6: MRN_ITAP(5)  // fallthrough
          case 5: MRN_ITAP(4)  // fallthrough
          case 4: MRN_ITAP(3)  // fallthrough
          case 3: MRN_ITAP(2)  // fallthrough
          case 2: MRN_ITAP(1)  // fallthrough
          case 1: MRN_ITAP(0)  // fallthrough
          default: break;
        }
#undef MRN_ITAP
        ax = fmaf(wa[a], sx, ax);
        ay = fmaf(wa[a], sy, ay);
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

// ---------------------------------------------------------------------------
// 2D warp-private gridding with tables (see k_grid_warp in tiles_fast.cu).
// ---------------------------------------------------------------------------
template <int CPL>
__global__ void __launch_bounds__(32)
k_grid_warp_tab(const Item* __restrict__ items, const SliceGeom* __restrict__ sl,
                const int4* __restrict__ meta, const float4* __restrict__ tab,
                const int* __restrict__ perm, const float2* __restrict__ ksp,
                const float* __restrict__ dcf, const float2* __restrict__ temporal,
                float2* __restrict__ grid, int layout, float scale, int cg, int pstride,
                SplitOut so) {
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
  const Frame2 f = frame2(*gp, it.tile, true);
  const int size1 = f.size[1];
  const int cells = f.size[0] * size1;
  for (int idx = lane; idx < ncg * pstride; idx += 32) acc[idx] = make_float2(0.f, 0.f);
  __syncwarp();

  const int64_t m = gp->m, pt_off = gp->pt_off, ksp_off = gp->ksp_off;
  // Software pipeline: the sample index two entries ahead, the table row, the
  // sample values and the per-sample factors one entry ahead, so the L2
  // latency of each load overlaps the previous entry's taps.
  const int n = it.count;
  const int64_t s0 = it.start;
  auto load_entry = [&](int64_t e, int64_t lpe, int4& mt, float (&wa)[8], float (&wb)[8],
                        float2 (&val)[CPL], float2& h) {
    mt = __ldg(meta + e);
    load_w(tab, e, wa, wb);
    float vs = scale;
    if (dcf) vs *= __ldg(dcf + pt_off + lpe);
    h = make_float2(vs, 0.f);
    if (temporal) {
      const float2 t = __ldg(temporal + pt_off + lpe);
      h = make_float2(vs * t.x, -vs * t.y);
    }
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int c = lane + q * 32;
      val[q] = c < ncg ? __ldg(ksp + ksp_off + (int64_t)(c0 + c) * m + lpe) : make_float2(0.f, 0.f);
    }
  };
  int4 mtN = make_int4(0, 0, 0, 0);
  float waN[8], wbN[8];
  float2 valN[CPL];
  float2 hN = make_float2(0.f, 0.f);
  int64_t lpA = 0;
  if (n > 0) {
    const int64_t lp0 = __ldg(perm + s0) - pt_off;
    load_entry(s0, lp0, mtN, waN, wbN, valN, hN);
    if (n > 1) lpA = __ldg(perm + s0 + 1) - pt_off;
  }
  for (int el = 0; el < n; ++el) {
    const int4 mt = mtN;
    float wa[8], wb[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      wa[j] = waN[j];
      wb[j] = wbN[j];
    }
    float2 val[CPL];
#pragma unroll
    for (int q = 0; q < CPL; ++q) val[q] = valN[q];
    const float2 h = hN;
    if (el + 1 < n) load_entry(s0 + el + 1, lpA, mtN, waN, wbN, valN, hN);
    if (el + 2 < n) lpA = __ldg(perm + s0 + el + 2) - pt_off;
    const int na = mt.z, nb = mt.w;
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int c = lane + q * 32;
      if (c >= ncg) break;
      const float2 a0 = val[q];
      const float2 v = make_float2(a0.x * h.x - a0.y * h.y, a0.x * h.y + a0.y * h.x);
      float2* row0 = acc + c * pstride + mt.x * size1 + mt.y;
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        if (a >= na) break;
        float2* row = row0 + a * size1;
        const float vx = wa[a] * v.x, vy = wa[a] * v.y;
#define MRN_GTAP(b)                        \
  {                                        \
    float2 o = row[b];                     \
    o.x = fmaf(wb[b], vx, o.x);            \
    o.y = fmaf(wb[b], vy, o.y);            \
    row[b] = o;                            \
  }
        switch (nb) {
          case 8: MRN_GTAP(7)  // fallthrough
          case 7: MRN_GTAP(6)  // fallthrough
          case 6: MRN_GTAP(5)  // fallthrough
          case 5: MRN_GTAP(4)  // fallthrough
          case 4: MRN_GTAP(3)  // fallthrough
          case 3: MRN_GTAP(2)  // fallthrough
          case 2: MRN_GTAP(1)  // fallthrough
          case 1: MRN_GTAP(0)  // fallthrough
          default: break;
        }
#undef MRN_GTAP
      }
    }
  }
  __syncwarp();

  const int64_t gos = gp->gos;
  const int64_t goff = (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gos;
  for (int c = 0; c < ncg; ++c) {
    float2* dstc = grid + goff + (int64_t)c * gos;
    const float2* src = acc + c * pstride;
    for (int cell = lane; cell < cells; cell += 32) {
      const int l0 = cell / size1, l1 = cell - l0 * size1;
      const int s0 = wrap1(f.org[0] + l0 - hs0, nos0);
      const int s1 = wrap1(f.org[1] + l1 - hs1, nos1);
      float2* d = dstc + (int64_t)s0 * nos1 + s1;
      const float2 v = src[cell];
      if (it.split) *split_slot(so, it.split, c0 + c, cell) = v;
      else *d = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
bool wtab_applicable(const mrn_plan* P) {
  if (!P->use_wtab || !P->use_fast || P->ndim != 2 || !P->kb.uniform_beta) return false;
  if (P->kb.ntaps[0] > 8 || P->kb.ntaps[1] > 8) return false;
  for (const auto& g : P->h_slices)
    for (int i = 0; i < 2; ++i)
      if (g.gntile[i] < 2 || g.nos[i] < P->kb.ntaps[i]) return false;
  return true;
}

// (Re)allocate a table pair for n entries when the current capacity is smaller.
static int table_capacity(int4** meta, float4** tab, int64_t* cap, int64_t n) {
  if (*cap >= n && *meta && *tab) return MRN_OK;
  if (*meta) cudaFree(*meta);
  if (*tab) cudaFree(*tab);
  *meta = nullptr;
  *tab = nullptr;
  *cap = 0;
  const size_t k = (size_t)std::max<int64_t>(n, 1);
  cudaError_t e = cudaMalloc((void**)meta, k * sizeof(int4));
  if (e == cudaSuccess) e = cudaMalloc((void**)tab, k * 4 * sizeof(float4));
  if (e != cudaSuccess) return cuda_fail(e);
  *cap = n;
  return MRN_OK;
}

int build_wtabs(mrn_plan* P, cudaStream_t st) {
  P->wtab_ok = false;
  if (!wtab_applicable(P)) return MRN_OK;
  const int64_t M = P->n_pts, E = P->n_entries_grid;
  int rc = table_capacity(&P->d_wmeta_i, &P->d_wtab_i, &P->cap_wtab_i, M);
  if (rc != MRN_OK) return rc;
  rc = table_capacity(&P->d_wmeta_g, &P->d_wtab_g, &P->cap_wtab_g, E);
  if (rc != MRN_OK) return rc;
  if (M > 0)
    k_wtab<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(P->d_slices, P->nslices, P->kb, P->d_coord_i,
                                                         P->d_key_is, M, 0, P->d_wmeta_i, P->d_wtab_i);
  if (E > 0)
    k_wtab<<<(unsigned)((E + 255) / 256), 256, 0, st>>>(P->d_slices, P->nslices, P->kb, P->d_coord_g,
                                                         P->d_key_g, E, 1, P->d_wmeta_g, P->d_wtab_g);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e);
  P->wtab_ok = true;
  return MRN_OK;
}

int launch_interp_tab(mrn_plan* P, const float2* grid, int layout, float2* ksp, float scale,
                      const float2* temporal, int cg, int G, int pstride, size_t smem, dim3 gdim,
                      cudaStream_t st) {
  int rc = MRN_OK;
  auto go = [&](auto kern) {
    rc = set_dynamic_smem(kern, smem);
    if (rc != MRN_OK) return;
    kern<<<gdim, kThreads, smem, st>>>(P->d_items_i, P->d_slices,
                                       make_int2(P->kb.ntaps[0], P->kb.ntaps[1]), P->d_wmeta_i,
                                       P->d_wtab_i, P->d_perm_i, grid, layout, ksp, scale, temporal,
                                       cg, pstride);
  };
  switch (G) {
    case 1: go(k_interp_tab<1>); break;
    case 2: case 4: go(k_interp_tab<4>); break;
    case 8: go(k_interp_tab<8>); break;
    case 16: go(k_interp_tab<16>); break;
    default: go(k_interp_tab<32>); break;
  }
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_grid_warp_tab(mrn_plan* P, const float2* ksp, const float* dcf, const float2* temporal,
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
  auto go = [&](auto kern) {
    rc = set_dynamic_smem(kern, smem);
    if (rc != MRN_OK) return;
    kern<<<gdim, 32, smem, st>>>(P->d_items_g, P->d_slices, P->d_wmeta_g, P->d_wtab_g, P->d_perm_g,
                                 ksp, dcf, temporal, grid, layout, scale, cg, pstride, split_out(P));
  };
  if (cg > 32) go(k_grid_warp_tab<2>);
  else go(k_grid_warp_tab<1>);
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

}  // namespace mrn
