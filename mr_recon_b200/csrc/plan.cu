// Plan creation and trajectory binning.
//
// A plan holds the geometry of n_slices NUFFT problems. mrn_plan_set_traj
// turns a trajectory into the per-tile sample lists the tile kernels consume:
//   interpolation: every sample belongs to the tile holding its first tap;
//   gridding     : every sample is listed once for each tile its footprint
//                  touches (1..2^d entries), so each tile owns its output.
// Both lists are sorted by tile with a stable radix sort (samples keep their
// trajectory order inside a tile) and cut into work items of at most
// max_chunk samples. This replaces the per-call locs preparation of the
// reference (prep_ungrid_shapes / prep_grid_shapes, ungrid.py:851-894,
// grid.py:508-553) and has no counterpart in its Triton launch (one program
// per point chunk, ungrid.py:127-129).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "common.cuh"
#include "internal.cuh"

using namespace mrn;

namespace mrn {

thread_local int g_last_cuda_error = 0;

int cuda_fail(cudaError_t e) {
  g_last_cuda_error = (int)e;
  return e == cudaErrorMemoryAllocation ? MRN_ERR_NOMEM : MRN_ERR_CUDA;
}

int set_dynamic_smem_fn(const void* kernel, size_t dyn) {
  struct Rec {
    size_t static_bytes;
    size_t opted;  // largest dynamic size opted into so far
  };
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, Rec> seen;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e);
  std::lock_guard<std::mutex> lock(mu);
  auto it = seen.find({kernel, dev});
  if (it == seen.end()) {
    cudaFuncAttributes a;
    e = cudaFuncGetAttributes(&a, kernel);
    if (e != cudaSuccess) return cuda_fail(e);
    it = seen.emplace(std::make_pair(kernel, dev), Rec{a.sharedSizeBytes, 0}).first;
  }
  Rec& r = it->second;
  if (dyn + r.static_bytes <= 48 * 1024 || dyn <= r.opted) return MRN_OK;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return cuda_fail(e);
  r.opted = dyn;
  return MRN_OK;
}

__device__ __forceinline__ int find_slice_by_point(const SliceGeom* sl, int ns, int64_t p) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (sl[mid].pt_off <= p) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int find_slice_by_tile(const SliceGeom* sl, int ns, int t, int gridding) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if ((gridding ? sl[mid].gtile_base : sl[mid].tile_base) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Distinct tiles of one dimension touched by the valid taps of a sample at
// wrapped coordinate u: taps j = lo + q, valid iff |(float)j - u| <= r (the
// float32 mask of weights1d..3d, kernels.py:268-393), cell = j mod nos.
__device__ __forceinline__ int dim_tiles(float u, float r, int ntaps, int nos, int nt,
                                         int* tiles) {
  const int lo = (int)ceilf(__fsub_rn(u, r));
  int n = 0;
  for (int q = 0; q < ntaps; ++q) {
    const float dx = __fsub_rn((float)(lo + q), u);
    if (!(fabsf(dx) <= r)) continue;
    const int t = nt == 1 ? 0 : tile_of(pos_mod(lo + q, nos), nos, nt);
    bool seen = false;
    for (int z = 0; z < n; ++z) seen |= (tiles[z] == t);
    if (!seen) tiles[n++] = t;
  }
  return n;
}

// Per sample: scaled, wrapped coordinates (fourier.py:420-430 then
// ungrid.py:873), interpolation tile key (tile of the first candidate tap),
// and the number of gridding tiles its footprint touches.
__global__ void k_prep_points(const SliceGeom* __restrict__ sl, int ns, int ndim, KBParams kb,
                              const float* __restrict__ trj, int64_t npts,
                              float4* __restrict__ coord, unsigned* __restrict__ key_i,
                              int* __restrict__ val_i, int* __restrict__ ecnt) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int s = find_slice_by_point(sl, ns, p);
  const SliceGeom& g = sl[s];
  const int64_t lp = p - g.pt_off;
  float u[kMaxDim] = {0.f, 0.f, 0.f};
  int lin = 0;
  int ntouch = 1;
  for (int i = 0; i < ndim; ++i) {
    const float k = trj[(g.pt_off + lp) * ndim + i];
    float v = __fadd_rn(__fmul_rn(k, g.scale[i]), g.shift[i]);
    v = remainder_f32(v, (float)g.nos[i]);
    u[i] = v;
    const int lo = (int)ceilf(__fsub_rn(v, kb.radius[i]));
    const int t0 = tile_of(pos_mod(lo, g.nos[i]), g.nos[i], g.ntile[i]);
    lin = lin * g.ntile[i] + t0;
    int tiles[kMaxTaps];
    ntouch *= dim_tiles(v, kb.radius[i], kb.ntaps[i], g.nos[i], g.gntile[i], tiles);
  }
  coord[p] = make_float4(u[0], u[1], u[2], 0.f);
  key_i[p] = (unsigned)(g.tile_base + lin);
  val_i[p] = (int)p;
  ecnt[p] = ntouch;
}

// Emit (tile, point) gridding entries at the scanned offsets.
__global__ void k_emit_entries(const SliceGeom* __restrict__ sl, int ns, int ndim, KBParams kb,
                               const float4* __restrict__ coord, int64_t npts,
                               const int* __restrict__ eoff, unsigned* __restrict__ key,
                               int* __restrict__ val) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int s = find_slice_by_point(sl, ns, p);
  const SliceGeom& g = sl[s];
  const float4 c4 = coord[p];
  const float uu[3] = {c4.x, c4.y, c4.z};
  int tiles[kMaxDim][kMaxTaps];
  int nt[kMaxDim] = {1, 1, 1};
  for (int i = 0; i < ndim; ++i)
    nt[i] = dim_tiles(uu[i], kb.radius[i], kb.ntaps[i], g.nos[i], g.gntile[i], tiles[i]);
  int o = eoff[p];
  for (int a = 0; a < nt[0]; ++a)
    for (int b = 0; b < (ndim > 1 ? nt[1] : 1); ++b)
      for (int c = 0; c < (ndim > 2 ? nt[2] : 1); ++c) {
        int lin = tiles[0][a];
        if (ndim > 1) lin = lin * g.gntile[1] + tiles[1][b];
        if (ndim > 2) lin = lin * g.gntile[2] + tiles[2][c];
        key[o] = (unsigned)(g.gtile_base + lin);
        val[o] = (int)p;
        ++o;
      }
}

// Per point, the gridding entries it was emitted as (positions after the
// tile sort); the slot order among a point's entries does not matter.
__global__ void k_point_entries(const int* __restrict__ perm_g, int64_t ne, int* __restrict__ ent_of,
                                int* __restrict__ cnt) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int p = perm_g[e];
  const int k = atomicAdd(cnt + p, 1);
  if (k < 4) ent_of[(int64_t)p * 4 + k] = (int)e;
}

__global__ void k_gather_coords(const float4* __restrict__ src, const int* __restrict__ perm,
                                int64_t n, float4* __restrict__ dst) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) dst[e] = src[perm[e]];
}

__global__ void k_tile_ranges(const unsigned* __restrict__ key, int64_t n, int ntiles,
                              int* __restrict__ start, int* __restrict__ end) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const unsigned k = key[e];
  if ((int)k >= ntiles) return;
  if (e == 0 || key[e - 1] != k) start[k] = (int)e;
  if (e == n - 1 || key[e + 1] != k) end[k] = (int)(e + 1);
}

__global__ void k_item_counts(const int* __restrict__ start, const int* __restrict__ end,
                              int ntiles, int chunk, int min_items, int* __restrict__ nitems) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int c = end[t] - start[t];
  nitems[t] = max(min_items, (c + chunk - 1) / chunk);
}

// Work items of every tile at the scanned offsets. Gridding tiles with more
// than one item are split tiles: each gets a run of n partial-tile slots
// (counts[4] hands them out) and a record {tile, first slot, n} in
// split_tiles (counts[3] counts them); item q of the tile writes slot
// first + q. The order in which tiles claim slots does not matter: the
// reduction adds a tile's slots in item order.
__global__ void k_emit_items(const SliceGeom* __restrict__ sl, int ns, const int* __restrict__ start,
                             const int* __restrict__ end, const int* __restrict__ nitems,
                             const int* __restrict__ ioff, int ntiles, int chunk,
                             Item* __restrict__ items, int4* __restrict__ split_tiles,
                             int* __restrict__ counts, int count_slot, int gridding) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int n = nitems[t];
  const int s = find_slice_by_tile(sl, ns, t, gridding);
  const int c = end[t] - start[t];
  int base = -1;
  if (gridding && n > 1) {
    base = atomicAdd(&counts[4], n);
    const int k = atomicAdd(&counts[3], 1);
    split_tiles[k] = make_int4(t, base, n, 0);
  }
  for (int q = 0; q < n; ++q) {
    // the tile's entries spread evenly over its items (at most chunk each)
    const int b0 = (int)(((int64_t)q * c) / n), b1 = (int)(((int64_t)(q + 1) * c) / n);
    Item it;
    it.slice = s;
    it.tile = t - (gridding ? sl[s].gtile_base : sl[s].tile_base);
    it.start = start[t] + b0;
    it.count = b1 - b0;
    it.split = base >= 0 ? base + q + 1 : 0;
    it.pad[0] = it.pad[1] = it.pad[2] = 0;
    items[ioff[t] + q] = it;
  }
  if (t == ntiles - 1) counts[count_slot] = ioff[t] + n;
}

// Sort keys of the longest-first item order: count + 1 for real items, 0 for
// the padding (slice -1) past them, so a stable descending sort keeps real
// items of equal length in tile order and leaves the padding last.
__global__ void k_item_keys(const Item* __restrict__ items, int64_t n, unsigned* __restrict__ key,
                            int* __restrict__ idx) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Item it = items[i];
  key[i] = it.slice < 0 ? 0u : (unsigned)it.count + 1u;
  idx[i] = (int)i;
}

__global__ void k_gather_items(const Item* __restrict__ src, const int* __restrict__ idx, int64_t n,
                               Item* __restrict__ dst) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

__global__ void k_total(const int* __restrict__ off, const int* __restrict__ cnt, int64_t n,
                        int* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = n > 0 ? off[n - 1] + cnt[n - 1] : 0;
}

static inline unsigned blocks_for(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Tiles per dimension for an edge length: at most ceil(nos / edge), and each
// tile at least K-1 cells wide so a kernel footprint touches at most two tiles
// per dimension (balanced partition, tile_begin / tile_of).
static int tiles_for(int nos, int edge, int K) {
  int nt = (nos + edge - 1) / edge;
  if (K > 1) nt = std::min(nt, std::max(1, nos / (K - 1)));
  return std::max(1, nt);
}


// Tile arrays are allocated for the larger of the two tilings.
// Kernel shape parameters: beta per dimension, and the I0 power series
// c_k = (beta^2/4)^k / (k!)^2 (in double) that the fast kernels evaluate,
// which exists only when every dimension has the same beta.
static void kb_set_beta(KBParams& kb, const double* betas, int ndim) {
  const double beta = betas[0];
  kb.beta = (float)beta;
  kb.uniform_beta = 1;
  for (int i = 0; i < kMaxDim; ++i) {
    kb.betad[i] = (float)(i < ndim ? betas[i] : beta);
    if (i < ndim && (float)betas[i] != kb.beta) kb.uniform_beta = 0;
  }
  const double q = beta * beta / 4.0;
  double c = 1.0, sum = 0.0;
  for (int k = 0; k < kKBTerms; ++k) {
    kb.coef[k] = (float)c;
    sum += c;
    c *= q / ((double)(k + 1) * (k + 1));
  }
  // c now holds the first omitted term; later terms shrink by q / (k+1)^2 each
  const double ratio = q / ((double)(kKBTerms + 1) * (kKBTerms + 1));
  const double tail = ratio < 1.0 ? c / (1.0 - ratio) : 1e300;
  kb.series = tail < 1e-9 * sum ? 1 : 0;
  // fewest terms (a multiple of 4, at least 16) whose dropped tail is below
  // 1e-9 of the sum; the tail after term n is bounded by the omitted terms
  // kept in coef plus the geometric bound above
  kb.nterms = kKBTerms;
  for (int n = 16; n < kKBTerms; n += 4) {
    double t = tail;
    for (int k = n; k < kKBTerms; ++k) t += (double)kb.coef[k];
    if (t < 1e-9 * sum) { kb.nterms = n; break; }
  }
}

static int64_t tile_capacity(const mrn_plan* P) { return std::max(P->ntiles, P->ngtiles); }

// Interpolation and gridding tilings of every slice, and their global tile ids.
void compute_tiling(mrn_plan* P) {
  int tiles = 0, gtiles = 0;
  for (int i = 0; i < kMaxDim; ++i) P->tmax_cells[i] = P->tmax_gcells[i] = 1;
  for (auto& g : P->h_slices) {
    int tc = 1, gc = 1;
    for (int i = 0; i < kMaxDim; ++i) {
      if (i >= P->ndim) {
        g.ntile[i] = g.gntile[i] = 1;
        continue;
      }
      const int K = P->kb.ntaps[i];
      const int nt = tiles_for(g.nos[i], P->tile[i], K);
      const int gt = tiles_for(g.nos[i], P->gtile[i], K);
      g.ntile[i] = nt;
      g.gntile[i] = gt;
      tc *= nt;
      gc *= gt;
      P->tmax_cells[i] = std::max(P->tmax_cells[i], (g.nos[i] + nt - 1) / nt);
      P->tmax_gcells[i] = std::max(P->tmax_gcells[i], (g.nos[i] + gt - 1) / gt);
    }
    g.tile_base = tiles;
    g.gtile_base = gtiles;
    tiles += tc;
    gtiles += gc;
  }
  P->ntiles = tiles;
  P->ngtiles = gtiles;
}

static cudaEvent_t pool_event(mrn_plan* P) {
  if (!P->ev_pool.empty()) {
    cudaEvent_t e = P->ev_pool.back();
    P->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

StageTimer::StageTimer(mrn_plan* p, int stage, cudaStream_t s) : P(p), st(s) {
  if (!P || !P->timing) return;
  mrn_plan::TimingRec r{stage, pool_event(P), pool_event(P)};
  if (!r.a || !r.b) return;
  cudaEventRecord(r.a, st);
  P->timing_recs.push_back(r);
  idx = (int)P->timing_recs.size() - 1;
}

StageTimer::~StageTimer() {
  if (idx >= 0) cudaEventRecord(P->timing_recs[idx].b, st);
}

// Upload the slice table and its shared-k-space twin (every ksp_off 0).
cudaError_t upload_slices(mrn_plan* P) {
  cudaError_t e = cudaMemcpy(P->d_slices, P->h_slices.data(), P->nslices * sizeof(SliceGeom),
                             cudaMemcpyHostToDevice);
  if (e != cudaSuccess || !P->d_slices_kshared) return e;
  std::vector<SliceGeom> ks(P->h_slices);
  for (auto& g : ks) g.ksp_off = 0;
  return cudaMemcpy(P->d_slices_kshared, ks.data(), P->nslices * sizeof(SliceGeom), cudaMemcpyHostToDevice);
}

template <class T>
static int dev_alloc(T** p, size_t n) {
  if (*p) { cudaFree(*p); *p = nullptr; }
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(e);
  return MRN_OK;
}

// New tile edges: recompute both tilings, grow the per-tile arrays when the
// finer tiling needs more entries, refresh the device slice table. The bound
// trajectory's binning is stale afterwards (mrn_plan_set_traj again).
static int retile(mrn_plan* P) {
  P->traj_set = false;
  P->wtab_ok = false;
  compute_tiling(P);
  const int64_t need = std::max<int64_t>(tile_capacity(P), 1);
  int rc = MRN_OK;
  if (need > P->cap_tiles) {
    int** bufs[] = {&P->d_tile_start_i, &P->d_tile_end_i, &P->d_tile_start_g, &P->d_tile_end_g,
                    &P->d_tile_nitems, &P->d_tile_item_off};
    for (int** b : bufs)
      if ((rc = dev_alloc(b, (size_t)need)) != MRN_OK) {
        P->cap_tiles = 0;
        return rc;
      }
    if ((rc = dev_alloc(&P->d_split_tiles, (size_t)need)) != MRN_OK) {
      P->cap_tiles = 0;
      return rc;
    }
    P->cap_tiles = need;
  }
  cudaError_t e = cudaSetDevice(P->device);
  if (e == cudaSuccess) e = upload_slices(P);
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

static int ensure_cub(mrn_plan* P, size_t bytes) {
  if (bytes <= P->cub_tmp_bytes && P->d_cub_tmp) return MRN_OK;
  if (P->d_cub_tmp) cudaFree(P->d_cub_tmp);
  P->d_cub_tmp = nullptr;
  cudaError_t e = cudaMalloc(&P->d_cub_tmp, bytes);
  if (e != cudaSuccess) return cuda_fail(e);
  P->cub_tmp_bytes = bytes;
  return MRN_OK;
}

}  // namespace mrn

#define CK(x)                                   \
  do {                                          \
    cudaError_t _e = (x);                       \
    if (_e != cudaSuccess) return cuda_fail(_e); \
  } while (0)
#define RK(x)                  \
  do {                         \
    int _r = (x);              \
    if (_r != MRN_OK) return _r; \
  } while (0)

extern "C" {

const char* mrn_version(void) { return "mrnufft 0.1.0 (sm_100a)"; }

const char* mrn_error_string(int code) {
  switch (code) {
    case MRN_OK: return "ok";
    case MRN_ERR_ARG: return "invalid argument";
    case MRN_ERR_WIDTH: return "kernel width out of range (1 <= width < 16)";
    case MRN_ERR_CUDA: return "CUDA error";
    case MRN_ERR_CUFFT: return "cuFFT error";
    case MRN_ERR_NOMEM: return "device allocation failed";
    case MRN_ERR_STATE: return "trajectory not set on plan";
    case MRN_ERR_UNSUPPORTED: return "unsupported configuration";
    case MRN_ERR_SCRATCH: return "problem exceeds the 32 MiB fixed scratch of mrn_interp_noalloc";
    default: return "unknown error";
  }
}

int mrn_last_cuda_error(void) { return mrn::g_last_cuda_error; }

int mrn_plan_create(mrn_plan** out, int ndim, int n_slices, const int* im_size,
                    const int64_t* n_pts, const int* n_coil, double oversamp,
                    const double* width, double beta, int flags, const int* tile,
                    int coil_group, int max_chunk, int device) {
  if (!out || !im_size || !n_pts || !n_coil || !width) return MRN_ERR_ARG;
  *out = nullptr;
  if (ndim < 1 || ndim > kMaxDim || n_slices < 1) return MRN_ERR_ARG;
  const bool raw = (flags & MRN_PLAN_RAW) != 0;
  if (!raw && !(oversamp >= 1.0)) return MRN_ERR_ARG;
  for (int i = 0; i < ndim; ++i)
    if (!(width[i] >= 1.0) || !(width[i] < (double)kMaxTaps)) return MRN_ERR_WIDTH;
  if (tile)
    for (int i = 0; i < ndim; ++i)
      if (tile[i] < 1) return MRN_ERR_ARG;
  if (coil_group < 0 || max_chunk < 0) return MRN_ERR_ARG;

  mrn_plan* P = new mrn_plan();
  P->ndim = ndim;
  P->nslices = n_slices;
  P->flags = flags;
  P->device = device;
  P->oversamp = raw ? 1.0 : oversamp;
  int maxtaps = 0;
  for (int i = 0; i < ndim; ++i) {
    P->width[i] = width[i];
    P->kb.radius[i] = (float)width[i] / 2.0f;
    P->kb.inv_radius[i] = 1.0f / P->kb.radius[i];
    P->kb.ntaps[i] = (int)std::floor(width[i]) + 1;
    maxtaps = std::max(maxtaps, P->kb.ntaps[i]);
  }
  P->tap_max = maxtaps <= 8 ? 8 : 16;
  if (beta <= 0.0) {
    if (raw) { delete P; return MRN_ERR_ARG; }
    const double w = width[0];
    beta = M_PI * std::sqrt(std::pow(w / oversamp * (oversamp - 0.5), 2) - 0.8);
  }
  P->beta = beta;
  {
    double betas[kMaxDim];
    for (int i = 0; i < kMaxDim; ++i) betas[i] = beta;
    kb_set_beta(P->kb, betas, ndim);
  }

  int maxc = 0;
  for (int s = 0; s < n_slices; ++s) {
    if (n_coil[s] < 1 || n_pts[s] < 0) { delete P; return MRN_ERR_ARG; }
    for (int i = 0; i < ndim; ++i)
      if (im_size[s * ndim + i] < 1) { delete P; return MRN_ERR_ARG; }
    maxc = std::max(maxc, n_coil[s]);
  }
  P->max_coil = maxc;

  // Built-in interpolation tile: 10 cells per edge in 2D (tile + halo as a [cell][coil]
  // region for 32 coils: three CTAs per SM), 4 in 3D (16-coil groups), 256 in 1D.
  int deftile[kMaxDim];
  for (int i = 0; i < ndim; ++i) deftile[i] = (ndim == 1) ? 256 : (ndim == 2 ? 10 : 4);
  for (int i = 0; i < ndim; ++i) P->tile[i] = tile ? tile[i] : deftile[i];
  // gridding tiles: 8x8 in 2D (one warp owns a tile), else the interpolation tile
  for (int i = 0; i < ndim; ++i) P->gtile[i] = (ndim >= 2 && !tile) ? 8 : P->tile[i];
  P->max_chunk = max_chunk > 0 ? max_chunk : (ndim == 2 ? 256 : 1024);
  // one warp grids a 2D tile item alone: shorter items keep warps balanced
  P->grid_chunk = max_chunk > 0 ? max_chunk : (ndim == 2 ? 256 : (ndim == 3 ? 4096 : 1024));

  // Slices
  int64_t img = 0, ksp = 0, ugrid = 0, trjo = 0, pts = 0, xo = 0;
  int64_t prow = 0, irow = 0, xrow = 0;
  int64_t maxe = 0;
  int64_t apodn = 0;
  P->h_slices.resize(n_slices);
  for (int s = 0; s < n_slices; ++s) {
    SliceGeom& g = P->h_slices[s];
    std::memset(&g, 0, sizeof(g));
    int64_t nimg = 1, gos = 1, spans = 1;
    for (int i = 0; i < kMaxDim; ++i) {
      g.n[i] = 1; g.nos[i] = 1; g.ntile[i] = 1; g.hshift[i] = 0; g.scale[i] = 1.f; g.shift[i] = 0.f;
    }
    for (int i = 0; i < ndim; ++i) {
      const int n = im_size[s * ndim + i];
      const int nos = raw ? n : (int)std::ceil(oversamp * n);
      g.n[i] = n;
      g.nos[i] = nos;
      g.hshift[i] = raw ? 0 : nos / 2;
      g.scale[i] = raw ? 1.0f : (float)((double)nos / (double)n);
      g.shift[i] = raw ? 0.0f : (float)(nos / 2);
      nimg *= n;
      gos *= nos;
      spans *= 2;
      g.apod_off[i] = (int)apodn;
      apodn += n;
    }
    g.ncoil = n_coil[s];
    g.m = n_pts[s];
    g.pt_off = pts;
    g.img_off = img;
    g.ksp_off = ksp;
    g.ugrid_off = ugrid;
    g.x_off = xo;
    g.gos = gos;
    g.nimg = nimg;
    g.inv_sqrt_n = (float)(1.0 / std::sqrt((double)nimg));
    g.prow_off = prow;
    g.irow_off = irow;
    g.xrow_off = xrow;
    prow += (int64_t)g.ncoil * gos / g.nos[ndim - 1];
    irow += (int64_t)g.ncoil * nimg / g.n[ndim - 1];
    xrow += nimg / g.n[ndim - 1];
    img += (int64_t)g.ncoil * nimg;
    ksp += (int64_t)g.ncoil * g.m;
    ugrid += (int64_t)g.ncoil * gos;
    trjo += g.m * ndim;
    pts += g.m;
    xo += nimg;
    maxe += spans * g.m;
  }
  P->n_img = img;
  P->n_ksp = ksp;
  P->n_grid = ugrid;
  P->n_trj = trjo;
  P->n_pts = pts;
  P->n_x = xo;
  P->n_prow = prow;
  P->n_irow = irow;
  P->n_xrow = xrow;
  compute_tiling(P);
  if (pts >= (int64_t)INT32_MAX || maxe >= (int64_t)INT32_MAX) { delete P; return MRN_ERR_UNSUPPORTED; }

  // Coil group: all coils of the widest slice, limited by shared memory.
  P->coil_group_req = coil_group > 0 ? std::min(coil_group, 64) : 0;
  if (coil_group > 0) {
    P->coil_group = std::min(coil_group, 64);
  } else {
    int64_t cells = 1;
    for (int i = 0; i < ndim; ++i) cells *= (P->tmax_cells[i] + P->kb.ntaps[i] - 1);
    const int64_t budget = 96 * 1024;  // bytes of tile data per CTA, two CTAs per SM
    int cg = (int)std::max<int64_t>(1, budget / ((cells | 1) * 8));
    cg = std::min(cg, 64);
    cg = std::min(cg, maxc);
    // balance groups: same number of groups, fewest coils per group
    const int ngroups = (maxc + cg - 1) / cg;
    cg = (maxc + ngroups - 1) / ngroups;
    P->coil_group = std::max(1, cg);
  }

  // FFT groups in first-seen order; internal grid buffer ordered by group.
  if (!raw) {
    std::vector<int> group_of(n_slices, -1);
    for (int s = 0; s < n_slices; ++s) {
      const SliceGeom& g = P->h_slices[s];
      int found = -1;
      for (size_t q = 0; q < P->fft.size(); ++q) {
        bool same = true;
        for (int i = 0; i < ndim; ++i) same &= (P->fft[q].nos[i] == g.nos[i]);
        if (same) { found = (int)q; break; }
      }
      if (found < 0) {
        mrn_plan::FftGroup fg{};
        for (int i = 0; i < kMaxDim; ++i) fg.nos[i] = g.nos[i];
        fg.batch = 0;
        fg.handle = 0;
        P->fft.push_back(fg);
        found = (int)P->fft.size() - 1;
      }
      group_of[s] = found;
      P->fft[found].batch += g.ncoil;
    }
    int64_t off = 0;
    for (size_t q = 0; q < P->fft.size(); ++q) {
      P->fft[q].grid_off = off;
      for (int s = 0; s < n_slices; ++s)
        if (group_of[s] == (int)q) {
          P->h_slices[s].grid_off = off;
          off += (int64_t)P->h_slices[s].ncoil * P->h_slices[s].gos;
        }
    }
  } else {
    for (int s = 0; s < n_slices; ++s) P->h_slices[s].grid_off = P->h_slices[s].ugrid_off;
  }

  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { delete P; return cuda_fail(e); }
  cudaDeviceGetAttribute(&P->sm_count, cudaDevAttrMultiProcessorCount, device);

  int rc = MRN_OK;
#define PK(x) do { rc = (x); if (rc != MRN_OK) { mrn_plan_destroy(P); return rc; } } while (0)
  PK(dev_alloc(&P->d_slices, n_slices));
  PK(dev_alloc(&P->d_slices_kshared, n_slices));
  e = upload_slices(P);
  if (e != cudaSuccess) { mrn_plan_destroy(P); return cuda_fail(e); }

  // Apodization tables a(x) = sqrt(beta^2 - (pi W x)^2) / sinh(.), x = (q - N//2)/Nos
  // (fourier.py:376-418), in double then rounded.
  {
    std::vector<float> ap(std::max<int64_t>(apodn, 1), 1.0f);
    if (!raw && !(flags & MRN_PLAN_NO_APOD)) {
      for (int s = 0; s < n_slices; ++s) {
        const SliceGeom& g = P->h_slices[s];
        for (int i = 0; i < ndim; ++i) {
          for (int q = 0; q < g.n[i]; ++q) {
            const double x = (double)(q - g.n[i] / 2) / (double)g.nos[i];
            const double t = M_PI * P->width[i] * x;
            const double a = std::sqrt(beta * beta - t * t);
            ap[g.apod_off[i] + q] = (float)(a / std::sinh(a));
          }
        }
      }
    }
    PK(dev_alloc(&P->d_apod, ap.size()));
    e = cudaMemcpy(P->d_apod, ap.data(), ap.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { mrn_plan_destroy(P); return cuda_fail(e); }
  }

  const int64_t np = std::max<int64_t>(pts, 1);
  PK(dev_alloc(&P->d_coord_i, np));
  PK(dev_alloc(&P->d_perm_i, np));
  PK(dev_alloc(&P->d_coord_tmp, np));
  PK(dev_alloc(&P->d_entry_cnt, 2 * np));
  PK(dev_alloc(&P->d_key_a, np));
  PK(dev_alloc(&P->d_val_a, np));
  PK(dev_alloc(&P->d_key_is, np));
  {
    // sized for the finest tiling either kind may get (plan options can change them)
    const int64_t tmax = std::max<int64_t>(tile_capacity(P), 1);
    PK(dev_alloc(&P->d_tile_start_i, tmax));
    PK(dev_alloc(&P->d_tile_end_i, tmax));
    PK(dev_alloc(&P->d_tile_start_g, tmax));
    PK(dev_alloc(&P->d_tile_end_g, tmax));
    PK(dev_alloc(&P->d_tile_nitems, tmax));
    PK(dev_alloc(&P->d_tile_item_off, tmax));
    PK(dev_alloc(&P->d_split_tiles, tmax));
    P->cap_tiles = tmax;
  }
  PK(dev_alloc(&P->d_counts, 8));
  PK(dev_alloc(&P->d_sync, 64));
  CK(cudaMemset(P->d_sync, 0, 64 * sizeof(unsigned)));
  PK(dev_alloc(&P->d_red, (size_t)n_slices * kMaxRedBlocks));
  PK(dev_alloc(&P->d_rowpart, (size_t)std::max<int64_t>(P->n_xrow, 1)));
  if (!raw) {
    PK(dev_alloc(&P->d_grid, std::max<int64_t>(P->n_grid, 1)));
    PK(dev_alloc(&P->d_ksp_tmp, std::max<int64_t>(P->n_ksp, 1)));
    for (auto& fg : P->fft) {
      int n[kMaxDim];
      for (int i = 0; i < ndim; ++i) n[i] = fg.nos[i];
      cufftResult r = cufftPlanMany(&fg.handle, ndim, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C,
                                    fg.batch);
      if (r != CUFFT_SUCCESS) { fg.handle = 0; mrn_plan_destroy(P); return MRN_ERR_CUFFT; }
    }
    PK(ffx_setup(P));
  }
#undef PK
  *out = P;
  return MRN_OK;
}

int mrn_plan_set_beta(mrn_plan* P, const double* beta) {
  if (!P || !beta || !(P->flags & MRN_PLAN_RAW)) return MRN_ERR_ARG;
  for (int i = 0; i < P->ndim; ++i)
    if (!(beta[i] > 0.0)) return MRN_ERR_ARG;
  kb_set_beta(P->kb, beta, P->ndim);
  P->beta = beta[0];
  P->traj_set = false;
  P->wtab_ok = false;
  return MRN_OK;
}

int mrn_plan_set_option(mrn_plan* P, int option, int value) {
  if (!P) return MRN_ERR_ARG;
  switch (option) {
    case MRN_OPT_FAST_KERNELS: P->use_fast = value != 0; return MRN_OK;
    case MRN_OPT_WARP_GRIDDING: P->warp_grid = value != 0; return MRN_OK;
    case MRN_OPT_WEIGHT_TABLES: P->use_wtab = value != 0; return MRN_OK;
    case MRN_OPT_REG_GRIDDING: P->reg_grid = value != 0; return MRN_OK;
    case MRN_OPT_REG_INTERP: P->reg_interp = value != 0; return MRN_OK;
    case MRN_OPT_ENTRY_MAJOR:
      P->use_ent = value != 0;
      P->traj_set = false;  // the entry map is built (or not) at mrn_plan_set_traj
      return MRN_OK;
    case MRN_OPT_NATIVE_FFT:
      P->use_ffx = value != 0;
      return ffx_refresh(P);
    case MRN_OPT_GRID_LANES:
      if (value != 0 && value != 8 && value != 16 && value != 32) return MRN_ERR_ARG;
      P->grid_lanes = value;
      return MRN_OK;
    case MRN_OPT_INTERP_CHUNK:
    case MRN_OPT_GRID_CHUNK:
      if (value < 1) return MRN_ERR_ARG;
      (option == MRN_OPT_INTERP_CHUNK ? P->max_chunk : P->grid_chunk) = value;
      P->traj_set = false;  // items are cut at mrn_plan_set_traj
      P->wtab_ok = false;
      return MRN_OK;
    case MRN_OPT_INTERP_TILE:
    case MRN_OPT_GRID_TILE:
      if (value < 1) return MRN_ERR_ARG;
      for (int i = 0; i < P->ndim; ++i) (option == MRN_OPT_INTERP_TILE ? P->tile : P->gtile)[i] = value;
      return retile(P);
    default: return MRN_ERR_ARG;
  }
}

int mrn_plan_enable_timing(mrn_plan* P, int on) {
  if (!P) return MRN_ERR_ARG;
  P->timing = on != 0;
  return MRN_OK;
}

int mrn_plan_timing(mrn_plan* P, double* ms, int64_t* count) {
  if (!P || !ms || !count) return MRN_ERR_ARG;
  for (int i = 0; i < kNumStages; ++i) { ms[i] = 0.0; count[i] = 0; }
  int rc = MRN_OK;
  for (auto& r : P->timing_recs) {
    cudaError_t e = cudaEventSynchronize(r.b);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
    if (e != cudaSuccess) rc = cuda_fail(e);
    else if (r.stage >= 0 && r.stage < kNumStages) { ms[r.stage] += t; count[r.stage] += 1; }
    P->ev_pool.push_back(r.a);
    P->ev_pool.push_back(r.b);
  }
  P->timing_recs.clear();
  return rc;
}

int mrn_plan_destroy(mrn_plan* P) {
  if (!P) return MRN_OK;
  for (auto& r : P->timing_recs) { P->ev_pool.push_back(r.a); P->ev_pool.push_back(r.b); }
  for (cudaEvent_t e : P->ev_pool)
    if (e) cudaEventDestroy(e);
  for (auto& fg : P->fft)
    if (fg.handle) cufftDestroy(fg.handle);
  toep_free(P);
  P->ffx.release();
  void* bufs[] = {P->d_slices, P->d_slices_kshared, P->d_apod, P->d_coord_i, P->d_perm_i, P->d_coord_g, P->d_perm_g,
                  P->d_key_a, P->d_key_b, P->d_key_is, P->d_key_g, P->d_val_a, P->d_val_b, P->d_coord_tmp,
                  P->d_entry_cnt, P->d_tile_start_i, P->d_tile_end_i, P->d_tile_start_g,
                  P->d_tile_end_g, P->d_tile_nitems, P->d_tile_item_off, P->d_items_i,
                  P->d_items_g, P->d_counts, P->d_split_tiles, P->d_cub_tmp, P->d_grid,
                  P->d_ksp_tmp, P->d_sync, P->d_wmeta_i, P->d_wtab_i, P->d_wmeta_g,
                  P->d_wtab_g, P->d_part, P->d_items_tmp, P->d_sort_key[0], P->d_sort_key[1],
                  P->d_sort_idx[0], P->d_sort_idx[1], P->d_red, P->d_rowpart, P->d_ent_of,
                  P->d_ksp_ent};
  for (void* b : bufs)
    if (b) cudaFree(b);
  delete P;
  return MRN_OK;
}

int mrn_plan_offsets(const mrn_plan* P, int64_t* img_off, int64_t* ksp_off, int64_t* grid_off,
                     int64_t* trj_off) {
  if (!P) return MRN_ERR_ARG;
  for (int s = 0; s < P->nslices; ++s) {
    const SliceGeom& g = P->h_slices[s];
    if (img_off) img_off[s] = g.img_off;
    if (ksp_off) ksp_off[s] = g.ksp_off;
    if (grid_off) grid_off[s] = g.ugrid_off;
    if (trj_off) trj_off[s] = g.pt_off * P->ndim;
  }
  return MRN_OK;
}

int mrn_plan_sizes(const mrn_plan* P, int64_t* o) {
  if (!P || !o) return MRN_ERR_ARG;
  o[0] = P->n_img; o[1] = P->n_ksp; o[2] = P->n_grid; o[3] = P->n_trj; o[4] = P->ntiles;
  o[5] = P->h_slices[0].nos[0]; o[6] = P->h_slices[0].nos[1]; o[7] = P->h_slices[0].nos[2];
  return MRN_OK;
}

int mrn_plan_fft_kind(const mrn_plan* P) {
  if (!P) return MRN_ERR_ARG;
  if (!ffx_active(P)) return 0;
  return P->ffx.all ? 1 : 2;
}

int mrn_plan_stats(mrn_plan* P, int64_t* o) {
  if (!P || !o) return MRN_ERR_ARG;
  int hc[4] = {0, 0, 0, 0};
  if (P->traj_set) {
    cudaError_t e = cudaSetDevice(P->device);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(hc, P->d_counts, 4 * sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e);
  }
  o[0] = hc[0]; o[1] = hc[1]; o[2] = P->n_entries_grid; o[3] = hc[3];
  return MRN_OK;
}

int mrn_plan_set_traj(mrn_plan* P, const float* trj, void* stream_) {
  if (!P || (!trj && P->n_pts > 0)) return MRN_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream_;
  const int64_t M = P->n_pts;
  const int T = P->ntiles;    // interpolation tiles
  const int TG = P->ngtiles;  // gridding tiles
  const int TT = std::max(T, TG);
  if (P->cap_tiles < TT) return MRN_ERR_STATE;  // a failed retile left the tile arrays short
  const int ndim = P->ndim;
  int bits = 1;
  while (bits < 31 && (1ll << bits) <= (long long)TT) ++bits;
  P->traj_set = false;

  // 1. coordinates, interpolation keys, gridding entry counts
  int* eoff = P->d_entry_cnt + std::max<int64_t>(M, 1);
  size_t need = 0, b = 0;
  const int Mi = (int)std::max<int64_t>(M, 1);
  cub::DeviceScan::ExclusiveSum(nullptr, b, P->d_entry_cnt, eoff, Mi, st);
  need = std::max(need, b);
  cub::DeviceScan::ExclusiveSum(nullptr, b, P->d_tile_nitems, P->d_tile_item_off, TT, st);
  need = std::max(need, b);
  cub::DeviceRadixSort::SortPairs(nullptr, b, P->d_key_a, P->d_key_is, P->d_val_a, P->d_perm_i,
                                  Mi, 0, bits, st);
  need = std::max(need, b);
  RK(ensure_cub(P, need));

  int64_t E = 0;
  if (M > 0) {
    k_prep_points<<<blocks_for(M), 256, 0, st>>>(P->d_slices, P->nslices, ndim, P->kb, trj, M,
                                                  P->d_coord_tmp, P->d_key_a, P->d_val_a,
                                                  P->d_entry_cnt);
    CK(cudaGetLastError());
    b = P->cub_tmp_bytes;
    CK(cub::DeviceScan::ExclusiveSum(P->d_cub_tmp, b, P->d_entry_cnt, eoff, (int)M, st));
    k_total<<<1, 32, 0, st>>>(eoff, P->d_entry_cnt, M, P->d_counts + 2);
    CK(cudaGetLastError());
    int hE = 0;
    CK(cudaMemcpyAsync(&hE, P->d_counts + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    E = hE;
  }
  P->n_entries_grid = E;

  // 2. gridding entry buffers grow on demand
  const int64_t capE = std::max<int64_t>(E, 1);
  if (P->cap_entries < capE) {
    RK(dev_alloc(&P->d_key_b, (size_t)capE));
    RK(dev_alloc(&P->d_val_b, (size_t)capE));
    RK(dev_alloc(&P->d_key_g, (size_t)capE));
    RK(dev_alloc(&P->d_perm_g, (size_t)capE));
    RK(dev_alloc(&P->d_coord_g, (size_t)capE));
    P->cap_entries = capE;
  }

  // 3. emit gridding entries and sort both lists by tile (stable)
  if (M > 0) {
    k_emit_entries<<<blocks_for(M), 256, 0, st>>>(P->d_slices, P->nslices, ndim, P->kb,
                                                   P->d_coord_tmp, M, eoff, P->d_key_b, P->d_val_b);
    CK(cudaGetLastError());
    b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b, P->d_key_b, P->d_key_g, P->d_val_b, P->d_perm_g,
                                    (int)std::max<int64_t>(E, 1), 0, bits, st);
    RK(ensure_cub(P, std::max(b, P->cub_tmp_bytes)));
    b = P->cub_tmp_bytes;
    CK(cub::DeviceRadixSort::SortPairs(P->d_cub_tmp, b, P->d_key_a, P->d_key_is, P->d_val_a,
                                       P->d_perm_i, (int)M, 0, bits, st));
    b = P->cub_tmp_bytes;
    CK(cub::DeviceRadixSort::SortPairs(P->d_cub_tmp, b, P->d_key_b, P->d_key_g, P->d_val_b,
                                       P->d_perm_g, (int)E, 0, bits, st));
    k_gather_coords<<<blocks_for(M), 256, 0, st>>>(P->d_coord_tmp, P->d_perm_i, M, P->d_coord_i);
    if (E > 0)
      k_gather_coords<<<blocks_for(E), 256, 0, st>>>(P->d_coord_tmp, P->d_perm_g, E, P->d_coord_g);
    CK(cudaGetLastError());
  }

  // 4. per-tile ranges
  CK(cudaMemsetAsync(P->d_tile_start_i, 0, T * sizeof(int), st));
  CK(cudaMemsetAsync(P->d_tile_end_i, 0, T * sizeof(int), st));
  CK(cudaMemsetAsync(P->d_tile_start_g, 0, TG * sizeof(int), st));
  CK(cudaMemsetAsync(P->d_tile_end_g, 0, TG * sizeof(int), st));
  CK(cudaMemsetAsync(P->d_counts, 0, 8 * sizeof(int), st));
  if (M > 0) {
    k_tile_ranges<<<blocks_for(M), 256, 0, st>>>(P->d_key_is, M, T, P->d_tile_start_i,
                                                 P->d_tile_end_i);
    if (E > 0)
      k_tile_ranges<<<blocks_for(E), 256, 0, st>>>(P->d_key_g, E, TG, P->d_tile_start_g,
                                                   P->d_tile_end_g);
  }

  // 5. work items, launched at capacities known from T, M and E alone, so the
  // host needs no further read-back: a tile with c entries makes
  // ceil(c / chunk) items (gridding: at least one), hence at most
  // T + M / chunk + 1 of them; split gridding tiles have more than gchunk
  // entries each (at most E / gchunk + 1 tiles) and ceil(c / gchunk) < 2 c / gchunk
  // items each (fewer than 2 E / gchunk slots).
  const int chunk = P->max_chunk;
  const int gchunk = P->grid_chunk;
  const int64_t max_items_i = M > 0 ? (int64_t)T + M / chunk + 1 : 0;
  const int64_t max_items_g = (int64_t)TG + E / gchunk + 1;
  const int64_t max_split = E > gchunk ? std::min<int64_t>(TG, E / gchunk + 1) : 0;
  const int64_t max_slots = max_split > 0 ? 2 * (E / gchunk) + 1 : 0;
  if (max_items_i >= (int64_t)INT32_MAX || max_items_g >= (int64_t)INT32_MAX) return MRN_ERR_UNSUPPORTED;
  if (P->cap_items_i < max_items_i) {
    RK(dev_alloc(&P->d_items_i, (size_t)max_items_i));
    P->cap_items_i = max_items_i;
  }
  if (P->cap_items_g < max_items_g) {
    RK(dev_alloc(&P->d_items_g, (size_t)max_items_g));
    P->cap_items_g = max_items_g;
  }
  const int64_t max_items = std::max(max_items_i, max_items_g);
  if (P->cap_sort < max_items) {
    RK(dev_alloc(&P->d_items_tmp, (size_t)max_items));
    for (int k = 0; k < 2; ++k) {
      RK(dev_alloc(&P->d_sort_key[k], (size_t)max_items));
      RK(dev_alloc(&P->d_sort_idx[k], (size_t)max_items));
    }
    P->cap_sort = max_items;
  }
  const int64_t part_elems = max_slots * (int64_t)P->max_coil * grid_tile_cells(P);
  if (P->cap_part < part_elems) {
    RK(dev_alloc(&P->d_part, (size_t)part_elems));
    P->cap_part = part_elems;
  }
  {
    size_t nb = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, nb, P->d_sort_key[0], P->d_sort_key[1],
                                              P->d_sort_idx[0], P->d_sort_idx[1],
                                              (int)std::max<int64_t>(max_items, 1), 0, 32, st);
    RK(ensure_cub(P, std::max(nb, P->cub_tmp_bytes)));
  }
  // Emit into the staging list (padding pre-filled with slice = -1), then
  // order longest first: CTAs start in index order, so the last wave holds
  // short items instead of a few long tiles.
  auto make_items = [&](int ntiles, int ch, int min_items, int64_t cap, int count_slot, int gridding,
                        const int* tstart, const int* tend, Item* out) -> int {
    if (cap == 0) return MRN_OK;
    CK(cudaMemsetAsync(P->d_items_tmp, 0xff, (size_t)cap * sizeof(Item), st));
    k_item_counts<<<blocks_for(ntiles), 256, 0, st>>>(tstart, tend, ntiles, ch, min_items,
                                                      P->d_tile_nitems);
    size_t nb = P->cub_tmp_bytes;
    CK(cub::DeviceScan::ExclusiveSum(P->d_cub_tmp, nb, P->d_tile_nitems, P->d_tile_item_off, ntiles, st));
    k_emit_items<<<blocks_for(ntiles), 256, 0, st>>>(P->d_slices, P->nslices, tstart, tend,
                                                     P->d_tile_nitems, P->d_tile_item_off, ntiles, ch,
                                                     P->d_items_tmp, P->d_split_tiles, P->d_counts,
                                                     count_slot, gridding);
    k_item_keys<<<blocks_for(cap), 256, 0, st>>>(P->d_items_tmp, cap, P->d_sort_key[0], P->d_sort_idx[0]);
    CK(cudaGetLastError());
    int kbits = 1;
    while (kbits < 32 && (1ll << kbits) <= (long long)ch + 1) ++kbits;
    nb = P->cub_tmp_bytes;
    CK(cub::DeviceRadixSort::SortPairsDescending(P->d_cub_tmp, nb, P->d_sort_key[0], P->d_sort_key[1],
                                                 P->d_sort_idx[0], P->d_sort_idx[1], (int)cap, 0, kbits,
                                                 st));
    k_gather_items<<<blocks_for(cap), 256, 0, st>>>(P->d_items_tmp, P->d_sort_idx[1], cap, out);
    CK(cudaGetLastError());
    return MRN_OK;
  };
  RK(make_items(T, chunk, 0, max_items_i, 0, 0, P->d_tile_start_i, P->d_tile_end_i, P->d_items_i));
  RK(make_items(TG, gchunk, 1, max_items_g, 1, 1, P->d_tile_start_g, P->d_tile_end_g, P->d_items_g));
  RK(build_wtabs(P, st));
  // 2D (at most 4 entries per point): the entry map of the entry-major normal operator
  P->ent_ok = false;
  if (P->use_ent && ndim == 2 && !(P->flags & MRN_PLAN_RAW) && M > 0 && E > 0) {
    if (P->cap_ent_of < 5 * M) {
      RK(dev_alloc(&P->d_ent_of, (size_t)(5 * M)));
      P->cap_ent_of = 5 * M;
    }
    const int64_t ke = E * (int64_t)P->max_coil;
    if (P->cap_ksp_ent < ke) {
      RK(dev_alloc(&P->d_ksp_ent, (size_t)ke));
      P->cap_ksp_ent = ke;
    }
    CK(cudaMemsetAsync(P->d_ent_of, 0xff, (size_t)(4 * M) * sizeof(int), st));
    CK(cudaMemsetAsync(P->d_ent_of + 4 * M, 0, (size_t)M * sizeof(int), st));
    k_point_entries<<<blocks_for(E), 256, 0, st>>>(P->d_perm_g, E, P->d_ent_of, P->d_ent_of + 4 * M);
    CK(cudaGetLastError());
    P->ent_ok = true;
  }
  P->n_items_interp = max_items_i;
  P->n_items_grid = max_items_g;
  P->n_split = max_split;
  P->traj_set = true;
  return MRN_OK;
}

}  // extern "C"
