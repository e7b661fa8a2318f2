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
// FMA with a compile-time index.
//
// Footprint windows. With K candidate taps per dimension a sample's footprint
// has K - 1 = KW taps per dimension unless u - W/2 is an integer (then the
// K-th candidate lies exactly on the support boundary and carries weight), so
// in every dimension the part of a footprint inside the tile fits a window of
// KW cells starting at w0 in [0, NW), NW = 8 - KW + 1 (clamped to the tile; a
// footprint cut by the tile edge has zero weights in the window's outside
// cells). Each window weight is evaluated directly from its tap (no
// tile-aligned vector is built). The window start pair (y0, z0) is the same
// for every thread of the CTA (they all accumulate the same entry), so one
// warp-uniform binary dispatch over the NW^2 pairs selects a straight-line block of KW
// rows x KW cells of packed two-lane FMAs (fma.rn.f32x2: re and im of a
// cell) on fixed registers: no FMA touches a cell outside the window and no
// row needs a test. A thread takes the x weight of its plane from the x
// window. Entries with K taps inside the tile in some dimension (exact
// boundary taps, a handful per spoke through the k-space centre) take the
// dense block instead: the warp evaluates the tile-aligned weights of all
// three dimensions itself (one lane per cell) and skips rows without weight.
//
// The weights and the sample values reach shared memory in batches of 64
// entries through a cp.async pipeline: in iteration b the values of batch
// b+1 and the coordinates of batch b+3 are in flight while the weights of
// batch b+1 are evaluated and batch b is accumulated; one barrier per batch.
// Each entry carries the mask of its x-planes with weight, so a warp takes
// one ballot per 32 entries of those touching its two planes without a
// weight load. No atomics; float32 accumulation in entry order, so results
// are the same on every run (split tiles write partial tiles that a
// reduction pass adds in item order).
// ---------------------------------------------------------------------------
constexpr int kG3Tile = 8;
constexpr int kG3Batch = 64;
constexpr int kG3Coils = 16;
constexpr int kG3Threads = 128;

namespace {

template <int B>
struct G3Smem {
  float4 c[4][B];        // coordinate ring (a batch stays until it is accumulated)
  int pm[4][B];          // sample index ring
  float wxw[2][B][8];    // per entry: x window weights x scale (first KW used)
  float wyw[2][B][8];    // per entry: y window weights
  float2 wzw[2][B][8];   // per entry: z window weights, each twice
  unsigned code[2][B];   // per entry: bytes x0, y0, z0 (bit 3: dense), x-plane mask
  float2 v[2][B][kG3Coils + 1];  // per entry and coil: sample value (row padded: conflict-free copies)
  float d[2][B];         // per entry: density weight
  float2 t[2][B];        // per entry: temporal weight
};

constexpr unsigned kG3Dense = 0x080808u;

// KW rows x KW cells of the window at (Y0, Z0): acc[Y0 + r][Z0 + c] +=
// wy[r] wz[c] v for the thread's coil and plane (v already carries the x
// weight and the scale).
template <int KW, int Y0, int Z0>
__device__ __forceinline__ void win_block(float2 (&acc)[kG3Tile][kG3Tile], const float (&wy)[KW],
                                          const float2 (&wz)[KW], float2 v) {
#pragma unroll
  for (int r = 0; r < KW; ++r) {
    const float2 v2 = __fmul2_rn(make_float2(wy[r], wy[r]), v);
#pragma unroll
    for (int c = 0; c < KW; ++c) acc[Y0 + r][Z0 + c] = __ffma2_rn(wz[c], v2, acc[Y0 + r][Z0 + c]);
  }
}

// Binary dispatch of the window code y0 * NW + z0 over [LO, HI).
template <int KW, int NW, int LO, int HI>
struct WinDispatch {
  static __device__ __forceinline__ void run(int code, float2 (&acc)[kG3Tile][kG3Tile],
                                             const float (&wy)[KW], const float2 (&wz)[KW], float2 v) {
    if constexpr (HI - LO == 1) {
      win_block<KW, LO / NW, LO % NW>(acc, wy, wz, v);
    } else {
      constexpr int MID = (LO + HI) / 2;
      if (code < MID) WinDispatch<KW, NW, LO, MID>::run(code, acc, wy, wz, v);
      else WinDispatch<KW, NW, MID, HI>::run(code, acc, wy, wz, v);
    }
  }
};

}  // namespace

template <int K, bool EXTRA>
__global__ void __launch_bounds__(kG3Threads, 3)
k_grid_reg3(const Item* __restrict__ items, const SliceGeom* __restrict__ sl, KBParams kb,
            const float4* __restrict__ coord, const int* __restrict__ perm,
            const float2* __restrict__ ksp, const float* __restrict__ dcf,
            const float2* __restrict__ temporal, float2* __restrict__ grid, int layout, float scale,
            int cg, SplitOut so) {
  constexpr int T = kG3Tile, B = kG3Batch, CW = kG3Coils, NT = kG3Threads;
  constexpr int KW = K - 1, NW = T - KW + 1;
  static_assert(K <= T, "taps per dimension");
  static_assert(NT == 2 * B, "copy roles assume two threads per batch entry");
  extern __shared__ __align__(16) unsigned char g3_smem[];
  G3Smem<B>& s = *reinterpret_cast<G3Smem<B>*>(g3_smem);

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

  // coordinates and sample indices of batch bi into ring slot bi % 4
  auto copy_coords = [&](int bi) {
    const int nb = batch_len(bi), r4 = bi & 3;
    if (tid < nb) cp_async16(&s.c[r4][tid], coord + it.start + bi * B + tid);
    else if (tid >= B && tid - B < nb) cp_async4(&s.pm[r4][tid - B], perm + it.start + bi * B + tid - B);
  };
  // sample values (one 8-byte copy per entry and coil), densities, temporal
  // weights; thread = (entry tid % B, coil phase tid / B), so one warp copy
  // reads 32 entries of one coil row (consecutive samples share lines)
  auto copy_values = [&](int bi) {
    const int nb = batch_len(bi), b2 = bi & 1, r4 = bi & 3;
    const int j = tid % B;
    if (j < nb) {
      const float2* src = kspg + (s.pm[r4][j] - pt_off);
      for (int c = tid / B; c < ncg; c += NT / B) cp_async8(&s.v[b2][j][c], src + (int64_t)c * m);
    }
    if (EXTRA) {
      if (tid < nb) {
        if (dcf) cp_async4(&s.d[b2][tid], dcf + s.pm[r4][tid]);
      } else if (tid >= B && tid - B < nb) {
        if (temporal) cp_async8(&s.t[b2][tid - B], temporal + s.pm[r4][tid - B]);
      }
    }
  };
  // Candidate taps of dimension i for coordinate u: first tap lo, its cell
  // st relative to the tile origin (wrapped), and whether the K-th candidate
  // carries weight.
  auto taps_of = [&](float u, int i, int& lo, int& st) {
    const int n = sel3(gp->nos, i), size = sel3(f.size, i);
    lo = (int)ceilf(__fsub_rn(u, sel3(kb.radius, i)));
    st = wrap_once(lo, n) - sel3(f.org, i);
    if (st >= size) st -= n;  // footprint wraps into this tile from the end
  };
  // unit (entry j, dimension i): the KW window weights, the window start, the
  // dense flag and (x) the mask of planes with weight
  auto weights = [&](int bi) {
    const int nb = batch_len(bi), b2 = bi & 1, r4 = bi & 3;
    // 3B units over NT threads; later rounds start at the other half of the
    // CTA, so the threads with a unit more are spread over the warps
    for (int rnd = 0; rnd * NT < 3 * B; ++rnd) {
      const int t = rnd * NT + (tid + rnd * (NT / 2)) % NT;
      if (t >= 3 * B) continue;
      const int j = t / 3, i = t - 3 * j;
      if (j >= nb) continue;
      const float4 c4 = s.c[r4][j];
      const float u = i == 0 ? c4.x : (i == 1 ? c4.y : c4.z);
      const float r = sel3(kb.radius, i), ir = sel3(kb.inv_radius, i);
      const int size = sel3(f.size, i);
      int lo, st;
      taps_of(u, i, lo, st);
      const bool last = fabsf(__fsub_rn((float)(lo + K - 1), u)) <= r;
      const bool dense = last && st >= 0 && st + K <= size;
      const int w0 = dense ? 0 : min(max(st, 0), size - KW);
      float ww[KW];
      unsigned mask = 0;
#pragma unroll
      for (int c = 0; c < KW; ++c) {
        const int q = w0 + c - st;
        const float adx = fabsf(__fsub_rn((float)(lo + q), u));
        const bool on = q >= 0 && q < K && adx <= r;
        ww[c] = on ? kb_tap_fast(adx, ir, kb) : 0.f;
        mask |= on ? 1u << c : 0u;
      }
      unsigned char* cb = reinterpret_cast<unsigned char*>(&s.code[b2][j]);
      cb[i] = (unsigned char)(w0 | (dense ? 8 : 0));
      if (i == 0) {
        if (dense) {  // all K candidates inside the tile
          mask = 0;
#pragma unroll
          for (int q = 0; q < K; ++q)
            if (fabsf(__fsub_rn((float)(lo + q), u)) <= r) mask |= 1u << q;
          cb[3] = (unsigned char)(mask << st);
        } else {
          cb[3] = (unsigned char)(mask << w0);
        }
#pragma unroll
        for (int c = 0; c < KW; ++c) s.wxw[b2][j][c] = ww[c] * scale;
      } else if (i == 1) {
#pragma unroll
        for (int c = 0; c < KW; ++c) s.wyw[b2][j][c] = ww[c];
      } else {
#pragma unroll
        for (int c = 0; c < KW; ++c) s.wzw[b2][j][c] = make_float2(ww[c], ww[c]);
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
      const bool meet = h32 + lane < nb && ((s.code[b2][h32 + lane] >> (24 + 2 * warp)) & 3u) != 0u;
      unsigned act = __ballot_sync(0xffffffffu, meet);
      while (act) {
        const int j = h32 + __ffs(act) - 1;
        act &= act - 1u;
        const unsigned cd = s.code[b2][j];
        float2 val = has_coil ? s.v[b2][j][coil] : make_float2(0.f, 0.f);
        if (EXTRA) {
          if (dcf) {
            const float d = s.d[b2][j];
            val = make_float2(val.x * d, val.y * d);
          }
          if (temporal) {  // times conj(t)
            const float2 tt = s.t[b2][j];
            val = make_float2(val.x * tt.x + val.y * tt.y, val.y * tt.x - val.x * tt.y);
          }
        }
        if ((cd & kG3Dense) == 0u) {  // uniform: the whole CTA shares the entry
          const int xi = plane - (int)(cd & 7u);
          const float wx = (unsigned)xi < (unsigned)KW ? s.wxw[b2][j][xi] : 0.f;
          const float2 v = __fmul2_rn(make_float2(wx, wx), val);
          float wy[KW];
          float2 wz[KW];
#pragma unroll
          for (int c = 0; c < KW; ++c) {
            wy[c] = s.wyw[b2][j][c];
            wz[c] = s.wzw[b2][j][c];
          }
          WinDispatch<KW, NW, 0, NW * NW>::run((int)((cd >> 8) & 7u) * NW + (int)((cd >> 16) & 7u), acc, wy, wz, v);
        } else {
          // dense block: lane (dimension lane / 8, cell lane % 8) evaluates one
          // tile-aligned weight; shuffles hand each thread its plane's x weight
          // and every thread the y and z vectors
          const float4 c4 = s.c[bi & 3][j];
          float w = 0.f;
          {
            const int i = min(lane >> 3, 2), cell = lane & 7;
            const float u = i == 0 ? c4.x : (i == 1 ? c4.y : c4.z);
            int lo, st;
            taps_of(u, i, lo, st);
            const int q = cell - st;
            if (cell < sel3(f.size, i) && q >= 0 && q < K) {
              const float adx = fabsf(__fsub_rn((float)(lo + q), u));
              if (adx <= sel3(kb.radius, i)) w = kb_tap_fast(adx, sel3(kb.inv_radius, i), kb);
            }
          }
          const float wx = __shfl_sync(0xffffffffu, w, plane) * scale;
          const float2 v = __fmul2_rn(make_float2(wx, wx), val);
          float wz[T];
#pragma unroll
          for (int z = 0; z < T; ++z) wz[z] = __shfl_sync(0xffffffffu, w, 16 + z);
#pragma unroll
          for (int y = 0; y < T; ++y) {
            const float wy = __shfl_sync(0xffffffffu, w, 8 + y);
            if (wy == 0.f) continue;  // uniform
            const float2 v2 = __fmul2_rn(make_float2(wy, wy), v);
#pragma unroll
            for (int z = 0; z < T; ++z) acc[y][z] = __ffma2_rn(make_float2(wz[z], wz[z]), v2, acc[y][z]);
          }
        }
      }
    }
  }
  cp_async_wait<0>();

  // Write-back through shared memory, half the tile (four x-planes) at a
  // time: the two warps holding those planes store their cells as 64 blocks
  // (plane, coil) of 8x8 cells (block stride 65 cells: conflict-free 8-byte
  // stores), then all threads store them out with consecutive lanes on
  // consecutive z-cells of a row, so one warp store covers four 64-byte rows
  // instead of 32 scattered 8-byte cells.
  constexpr int CS = T * T + 1;
  static_assert(64 * CS * sizeof(float2) <= sizeof(G3Smem<B>), "write-back staging fits");
  float2* stage = reinterpret_cast<float2*>(g3_smem);
  const int nos0 = gp->nos[0], nos1 = gp->nos[1], nos2 = gp->nos[2];
  const int hs0 = layout == kInternal ? gp->hshift[0] : 0;
  const int hs1 = layout == kInternal ? gp->hshift[1] : 0;
  const int hs2 = layout == kInternal ? gp->hshift[2] : 0;
  float2* dst = grid + (layout == kInternal ? gp->grid_off : gp->ugrid_off) + (int64_t)c0 * gp->gos;
  // this thread's cell of every block it stores: (y, z) fixed, block varies
  const int cell = tid & 63, cy = cell >> 3, cz = cell & 7;
  const bool cell_in = cy < f.size[1] && cz < f.size[2];
  int zz = wrap_once(f.org[2] - hs2, nos2) + cz;
  if (zz >= nos2) zz -= nos2;
  const int64_t yz = (int64_t)wrap_once(f.org[1] + cy - hs1, nos1) * nos2 + zz;
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    __syncthreads();  // staging buffers free (batch buffers, or the previous half)
    if ((warp >> 1) == half) {
      float2* b = stage + ((warp & 1) * 32 + lane) * CS;  // block = (plane - 4 half) * 16 + coil
#pragma unroll
      for (int y = 0; y < T; ++y)
#pragma unroll
        for (int z = 0; z < T; ++z) b[y * T + z] = acc[y][z];
    }
    __syncthreads();
#pragma unroll 4
    for (int blk = tid >> 6; blk < 64; blk += NT / 64) {
      const int bc = blk & 15, bp = 4 * half + (blk >> 4);
      if (!cell_in || bc >= ncg || bp >= f.size[0]) continue;
      const float2 val = stage[blk * CS + cell];
      if (it.split) {
        *split_slot(so, it.split, c0 + bc, (bp * f.size[1] + cy) * f.size[2] + cz) = val;
      } else {
        const int64_t xo = (int64_t)wrap_once(f.org[0] + bp - hs0, nos0) * nos1 * nos2;
        dst[(int64_t)bc * gp->gos + xo + yz] = val;
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
  const size_t smem = sizeof(G3Smem<kG3Batch>);
  const bool extra = dcf != nullptr || temporal != nullptr;
  int rc = MRN_OK;
#define MRN_G3_LAUNCH(KK, EX)                                                                     \
  do {                                                                                            \
    auto kern = k_grid_reg3<KK, EX>;                                                              \
    rc = set_dynamic_smem(kern, smem);                                                            \
    if (rc == MRN_OK)                                                                             \
      kern<<<gdim, kG3Threads, smem, st>>>(P->d_items_g, P->d_slices, P->kb, P->d_coord_g,        \
                                           P->d_perm_g, ksp, dcf, temporal, grid, layout, scale, \
                                           cg, so);                                               \
  } while (0)
  if (K == 5) { if (extra) MRN_G3_LAUNCH(5, true); else MRN_G3_LAUNCH(5, false); }
  else if (K == 6) { if (extra) MRN_G3_LAUNCH(6, true); else MRN_G3_LAUNCH(6, false); }
  else if (K == 7) { if (extra) MRN_G3_LAUNCH(7, true); else MRN_G3_LAUNCH(7, false); }
  else { if (extra) MRN_G3_LAUNCH(8, true); else MRN_G3_LAUNCH(8, false); }
#undef MRN_G3_LAUNCH
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

}  // namespace mrn
