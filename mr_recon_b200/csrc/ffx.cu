// Native FFT stage of the NUFFT: the d-dimensional C2C transform of the
// plan's oversampled grid as one pass per axis, with the NUFFT's zero padding
// and cropping folded into the passes.
//
// Reference: fourier.py (:470-560) apodizes and pads the image into the
// oversampled grid (centred pad + ifftshift), calls torch.fft.fftn, and on
// the adjoint calls ifftn and crops (norm=None: unnormalised transforms; the
// 1/sqrt(prod N) and the apodization are applied in the first forward / last
// adjoint pass with the same float products as k_pre / k_post).
//
// Passes. Forward: the last axis first, a half-warp per grid line, fused with the
// apodize / pad: a line whose outer storage indices fall in the zero padding
// is all zero and is neither computed nor stored. Then every other axis from
// the last-but-one to the first, a CTA per block of W adjacent columns: rows
// of the axis inside its zero padding read as zero, and the planes whose
// (untransformed) earlier-axis index lies in the padding are skipped.
// Adjoint: the first axis first (every row read, only the rows that survive
// the crop stored), the middle axis on the surviving planes likewise, and
// the last axis as a half-warp per surviving line fused with the crop /
// deapodize, or stored back in place for the SENSE coil combination, which
// reads only surviving lines.
//
// Each line is a Stockham autosort FFT in shared memory: stage s with radix R
// and L = the product of the earlier radices maps butterfly b = k L + j
// (j < L) to out[k R L + u L + j] = sum_t x[b + t n / R] w^(t j)
// e^(-+2 pi i t u / R), w = e^(-+2 pi i / (L R)) (radices 5, 3, 16, 8, 4, 2); the
// twiddles come from a table computed on the host in double precision. The
// result is in natural order after the last stage, with no bit reversal.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "internal.cuh"
#include "tile_util.cuh"

namespace mrn {

namespace {

constexpr float kSin3 = 0.866025403784438647f;   // sin(2 pi / 3)
constexpr float kCos51 = 0.309016994374947424f;  // cos(2 pi / 5)
constexpr float kCos52 = -0.809016994374947424f; // cos(4 pi / 5)
constexpr float kSin51 = 0.951056516295153572f;  // sin(2 pi / 5)
constexpr float kSin52 = 0.587785252292473129f;  // sin(4 pi / 5)
constexpr int kFfxThreads = 256;
constexpr int kFfxCols = 8;  // adjacent columns per CTA in the strided passes

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// a w (forward) or a conj(w) (inverse)
template <bool INV>
__device__ __forceinline__ float2 ctw(float2 a, float2 w) {
  return INV ? make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y)
             : make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// c (-i a) (forward) or c (+i a) (inverse)
template <bool INV>
__device__ __forceinline__ float2 rot(float2 a, float c) {
  return INV ? make_float2(-c * a.y, c * a.x) : make_float2(c * a.y, -c * a.x);
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2 (&x)[R]) {
  if constexpr (R == 2) {
    const float2 a = x[0];
    x[0] = cadd(a, x[1]);
    x[1] = csub(a, x[1]);
  } else if constexpr (R == 3) {
    const float2 s = cadd(x[1], x[2]);
    const float2 m = make_float2(x[0].x - 0.5f * s.x, x[0].y - 0.5f * s.y);
    const float2 d = rot<INV>(csub(x[1], x[2]), kSin3);
    x[0] = cadd(x[0], s);
    x[1] = cadd(m, d);
    x[2] = csub(m, d);
  } else if constexpr (R == 4) {
    const float2 a0 = cadd(x[0], x[2]), a1 = csub(x[0], x[2]);
    const float2 a2 = cadd(x[1], x[3]), a3 = rot<INV>(csub(x[1], x[3]), 1.0f);
    x[0] = cadd(a0, a2);
    x[2] = csub(a0, a2);
    x[1] = cadd(a1, a3);
    x[3] = csub(a1, a3);
  } else if constexpr (R == 8) {
    // two 4-point DFTs of the even and odd inputs, the odd ones turned by
    // w8^u = e^(-+i pi u / 4), u = 1, 2, 3
    constexpr float c = 0.707106781186547524f;  // sqrt(1/2)
    float2 e[4] = {x[0], x[2], x[4], x[6]};
    float2 o[4] = {x[1], x[3], x[5], x[7]};
    dft<4, INV>(e);
    dft<4, INV>(o);
    const float2 o1 = o[1], o3 = o[3];
    o[1] = INV ? make_float2(c * (o1.x - o1.y), c * (o1.x + o1.y)) : make_float2(c * (o1.x + o1.y), c * (o1.y - o1.x));
    o[2] = rot<INV>(o[2], 1.0f);
    o[3] = INV ? make_float2(c * (-o3.x - o3.y), c * (o3.x - o3.y)) : make_float2(c * (o3.y - o3.x), c * (-o3.x - o3.y));
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x[u] = cadd(e[u], o[u]);
      x[u + 4] = csub(e[u], o[u]);
    }
  } else if constexpr (R == 16) {
    // 4 x 4: 4-point DFTs of the inputs r, r + 4, r + 8, r + 12, each
    // output u1 turned by w16^(r u1), then 4-point DFTs across r; output
    // u1 + 4 u2
    constexpr float c16[10] = {1.0f, 0.923879532511286756f, 0.707106781186547524f, 0.382683432365089772f, 0.0f,
                               -0.382683432365089772f, -0.707106781186547524f, -0.923879532511286756f, -1.0f,
                               -0.923879532511286756f};
    constexpr float s16[10] = {0.0f, 0.382683432365089772f, 0.707106781186547524f, 0.923879532511286756f, 1.0f,
                               0.923879532511286756f, 0.707106781186547524f, 0.382683432365089772f, 0.0f,
                               -0.382683432365089772f};
    float2 a[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll
      for (int m = 0; m < 4; ++m) a[r][m] = x[4 * m + r];
      dft<4, INV>(a[r]);
    }
#pragma unroll
    for (int u1 = 0; u1 < 4; ++u1) {
      float2 col[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int k = r * u1;
        const float2 v = a[r][u1];
        if (k == 0) col[r] = v;
        else if (k == 4) col[r] = rot<INV>(v, 1.0f);
        else col[r] = INV ? make_float2(v.x * c16[k] - v.y * s16[k], v.x * s16[k] + v.y * c16[k])
                          : make_float2(v.x * c16[k] + v.y * s16[k], v.y * c16[k] - v.x * s16[k]);
      }
      dft<4, INV>(col);
#pragma unroll
      for (int u2 = 0; u2 < 4; ++u2) x[u1 + 4 * u2] = col[u2];
    }
  } else {  // R == 5
    const float2 a1 = cadd(x[1], x[4]), b1 = csub(x[1], x[4]);
    const float2 a2 = cadd(x[2], x[3]), b2 = csub(x[2], x[3]);
    const float2 r1 = make_float2(x[0].x + kCos51 * a1.x + kCos52 * a2.x, x[0].y + kCos51 * a1.y + kCos52 * a2.y);
    const float2 r2 = make_float2(x[0].x + kCos52 * a1.x + kCos51 * a2.x, x[0].y + kCos52 * a1.y + kCos51 * a2.y);
    const float2 p1 = rot<INV>(make_float2(kSin51 * b1.x + kSin52 * b2.x, kSin51 * b1.y + kSin52 * b2.y), 1.0f);
    const float2 p2 = rot<INV>(make_float2(kSin52 * b1.x - kSin51 * b2.x, kSin52 * b1.y - kSin51 * b2.y), 1.0f);
    x[0] = cadd(x[0], cadd(a1, a2));
    x[1] = cadd(r1, p1);
    x[4] = csub(r1, p1);
    x[2] = cadd(r2, p2);
    x[3] = csub(r2, p2);
  }
}

// Butterfly bi of a stage (radix R, L, nr = n / R) over elements ES apart;
// k = bi / L by a multiply-high with the stage's magic (the first stage has
// L = 1 and no twiddles).
template <int R, bool INV, int ES, bool FIRST>
__device__ __forceinline__ void bfly(const float2* __restrict__ a, float2* __restrict__ b, int L, unsigned magic,
                                     int nr, const float2* __restrict__ tw, int bi) {
  const int k = FIRST ? bi : (int)__umulhi((unsigned)bi, magic);
  const int j = FIRST ? 0 : bi - k * L;
  float2 x[R];
#pragma unroll
  for (int t = 0; t < R; ++t) x[t] = a[(bi + t * nr) * ES];
  if (!FIRST) {
    const float2* tj = tw + j * (R - 1);
#pragma unroll
    for (int t = 1; t < R; ++t) x[t] = ctw<INV>(x[t], tj[t - 1]);
  }
  dft<R, INV>(x);
  const int ob = k * R * L + j;
#pragma unroll
  for (int u = 0; u < R; ++u) b[(ob + u * L) * ES] = x[u];
}

// Axis plan in shared memory (kernel parameters indexed at run time would go
// through local memory).
struct FfxShared {
  int radix[kFfxMaxStages];
  int tw_off[kFfxMaxStages];
  unsigned magic[kFfxMaxStages];
};

__device__ __forceinline__ void stage_axis(FfxShared& sa, float2* tw, const FfxAxis& ax,
                                           const float2* __restrict__ twg) {
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < kFfxMaxStages; ++i) {
      sa.radix[i] = ax.radix[i];
      sa.tw_off[i] = ax.tw_off[i];
      sa.magic[i] = ax.magic[i];
    }
  }
  for (int i = threadIdx.x; i < ax.n - 1; i += blockDim.x) tw[i] = twg[ax.tw_base + i];
}

// All butterflies of one stage of a line (ES = 1) by the 16 lanes of a
// half-warp (hl: lane within the half).
template <int R, bool INV, bool FIRST>
__device__ __forceinline__ void line_stage(const float2* a, float2* b, int L, unsigned magic, int nr,
                                           const float2* tw, int hl) {
  for (int bi = hl; bi < nr; bi += 16) bfly<R, INV, 1, FIRST>(a, b, L, magic, nr, tw, bi);
}

// One stage over W adjacent columns (elements W apart) by a CTA.
template <int R, bool INV, bool FIRST, int W>
__device__ __forceinline__ void cols_stage(const float2* a, float2* b, int L, unsigned magic, int nr,
                                           const float2* tw, int tid, int nt) {
  for (int idx = tid; idx < nr * W; idx += nt) {
    const int bi = idx / W, w = idx - bi * W;
    bfly<R, INV, W, FIRST>(a + w, b + w, L, magic, nr, tw, bi);
  }
}

#define MRN_FFX_STAGE(CALL)                                  \
  do {                                                       \
    if (s == 0) {                                            \
      switch (R) {                                           \
        case 16: CALL(16, true); break;                     \
        case 8: CALL(8, true); break;                        \
        case 4: CALL(4, true); break;                        \
        case 5: CALL(5, true); break;                        \
        case 3: CALL(3, true); break;                        \
        default: CALL(2, true); break;                       \
      }                                                      \
    } else {                                                 \
      switch (R) {                                           \
        case 16: CALL(16, false); break;                     \
        case 8: CALL(8, false); break;                       \
        case 4: CALL(4, false); break;                       \
        case 5: CALL(5, false); break;                       \
        case 3: CALL(3, false); break;                       \
        default: CALL(2, false); break;                      \
      }                                                      \
    }                                                        \
  } while (0)

// One line of n points by a half-warp: a holds the input, b is scratch;
// returns the buffer that holds the transform. Both halves of the warp run
// every stage's __syncwarp; an inactive half (no line) skips the butterflies.
template <bool INV>
__device__ __forceinline__ float2* line_fft(float2* a, float2* b, int n, int ns, const FfxShared& sa,
                                            const float2* tw, int hl, bool active) {
  int L = 1;
  for (int s = 0; s < ns; ++s) {
    const int R = sa.radix[s], nr = n / R;
    const unsigned magic = sa.magic[s];
    const float2* t = tw + sa.tw_off[s];
    if (active) {
#define MRN_LINE_CALL(RR, FF) line_stage<RR, INV, FF>(a, b, L, magic, nr, t, hl)
      MRN_FFX_STAGE(MRN_LINE_CALL);
#undef MRN_LINE_CALL
    }
    __syncwarp();
    float2* tmp = a;
    a = b;
    b = tmp;
    L *= R;
  }
  return a;
}

// Slice k of the group holding group row `row` (grow: first row of each of
// the gns slices, then the total).
__device__ __forceinline__ void row_slice(const int64_t* __restrict__ grow, int gns, int64_t row, int& k) {
  int lo = 0, hi = gns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (grow[mid] <= row) lo = mid; else hi = mid - 1;
  }
  k = lo;
}

// index i of an axis of n image points in nos grid points survives the crop
// (is not zero padding): the image index (i + n / 2) mod nos is below n
__device__ __forceinline__ bool kept(int i, int n, int nos) {
  int q = i + n / 2;
  if (q >= nos) q -= nos;
  return q < n;
}

// Geometry of group row `row` (a grid line along the last axis): slice,
// coil, the line's storage index within the coil, the image row it carries
// (qlin, in image rows) and the outer apodization factor; false if an outer
// storage index lies in the zero padding (the line is zero / cropped away).
template <int D>
__device__ __forceinline__ bool row_geom(const SliceGeom* __restrict__ sl, const int* __restrict__ gsl,
                                         const int64_t* __restrict__ grow, int gns, const float* __restrict__ apod,
                                         int64_t row, int n, float scale, const SliceGeom*& gp, int& c,
                                         int64_t& lrow, int64_t& qlin, float& aout) {
  int k = 0;
  row_slice(grow, gns, row, k);
  gp = sl + gsl[k];
  const SliceGeom& g = *gp;
  const int64_t r = row - grow[k];
  const int64_t outer = g.gos / n;
  c = (int)(r / outer);
  int64_t o = r - (int64_t)c * outer;
  lrow = o;
  int st[kMaxDim] = {0, 0, 0};
  for (int i = D - 2; i >= 0; --i) {
    st[i] = (int)(o % g.nos[i]);
    o /= g.nos[i];
  }
  aout = scale * g.inv_sqrt_n;
  qlin = 0;
  for (int i = 0; i < D - 1; ++i) {
    int q = st[i] + g.n[i] / 2;
    if (q >= g.nos[i]) q -= g.nos[i];
    if (q >= g.n[i]) return false;
    aout *= apod[g.apod_off[i] + q];
    qlin = qlin * g.n[i] + q;
  }
  return true;
}

// Forward pass over the last axis fused with the apodize / pad (k_pre's
// products): each half-warp takes one grid row (slice, coil, outer storage
// index); a row whose outer index is zero padding is neither computed nor
// stored (the next pass reads it as zero).
template <int D, bool SENSE>
__global__ void __launch_bounds__(kFfxThreads)
k_ffx_rows_fwd(const SliceGeom* __restrict__ sl, const int* __restrict__ gsl, const int64_t* __restrict__ grow,
               int gns, const float* __restrict__ apod, const float2* __restrict__ src,
               const float2* __restrict__ mps, float scale, float2* __restrict__ grid, int64_t nrows, FfxAxis ax,
               const float2* __restrict__ twg) {
  extern __shared__ float2 fsm[];
  __shared__ FfxShared sa;
  const int n = ax.n, nw = blockDim.x >> 5;
  float2* tw = fsm;
  stage_axis(sa, tw, ax, twg);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
  const int64_t row = ((int64_t)blockIdx.x * nw + warp) * 2 + half;
  const SliceGeom* gp = sl;
  int c = 0;
  int64_t lrow = 0, qlin = 0;
  float aout = 0.f;
  const bool active = row < nrows && row_geom<D>(sl, gsl, grow, gns, apod, row, n, scale, gp, c, lrow, qlin, aout);
  float2* A = fsm + n + (warp * 2 + half) * 2 * n;
  float2* B = A + n;
  const int nl = gp->n[D - 1], h = nl / 2;
  const int64_t q0 = qlin * nl;
  const float* al = apod + gp->apod_off[D - 1];
  const float2* mrow = SENSE ? mps + gp->img_off + (int64_t)c * gp->nimg + q0 : nullptr;
  // the image row lands in B (the FFT's scratch) with every copy in flight
  // at once, then is apodized and placed into A
  if (active) {
    const float2* srow = SENSE ? src + gp->x_off + q0 : src + gp->img_off + (int64_t)c * gp->nimg + q0;
    for (int q = hl; q < nl; q += 16) cp_async8(&B[q], srow + q);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncwarp();
  if (active)
    for (int j = hl; j < n; j += 16) {
      int q = j + h;
      if (q >= n) q -= n;
      float2 v = make_float2(0.f, 0.f);
      if (q < nl) {
        float2 x = B[q];
        if (SENSE) {
          const float2 m = __ldg(mrow + q);
          x = make_float2(x.x * m.x - x.y * m.y, x.x * m.y + x.y * m.x);
        }
        const float a = aout * al[q];
        v = make_float2(x.x * a, x.y * a);
      }
      A[j] = v;
    }
  __syncwarp();
  const float2* res = line_fft<false>(A, B, n, ax.ns, sa, tw, hl, active);
  if (!active) return;
  float2* dst = grid + gp->grid_off + (int64_t)c * gp->gos + lrow * n;
#pragma unroll 4
  for (int j = hl; j < n; j += 16) dst[j] = res[j];
}

// Inverse pass over the last axis of the rows that survive the crop (a
// half-warp per row): POST crops and deapodizes into the image (k_post's
// products), else the row is stored back for the SENSE coil combination.
template <int D, bool POST>
__global__ void __launch_bounds__(kFfxThreads)
k_ffx_rows_inv(const SliceGeom* __restrict__ sl, const int* __restrict__ gsl, const int64_t* __restrict__ grow,
               int gns, const float* __restrict__ apod, float2* __restrict__ grid, float scale,
               float2* __restrict__ out, int64_t nrows, FfxAxis ax, const float2* __restrict__ twg) {
  extern __shared__ float2 fsm[];
  __shared__ FfxShared sa;
  const int n = ax.n, nw = blockDim.x >> 5;
  float2* tw = fsm;
  stage_axis(sa, tw, ax, twg);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
  const int64_t row = ((int64_t)blockIdx.x * nw + warp) * 2 + half;
  const SliceGeom* gp = sl;
  int c = 0;
  int64_t lrow = 0, qlin = 0;
  float aout = 0.f;
  const bool active = row < nrows && row_geom<D>(sl, gsl, grow, gns, apod, row, n, scale, gp, c, lrow, qlin, aout);
  float2* gline = grid + gp->grid_off + (int64_t)c * gp->gos + lrow * n;
  float2* A = fsm + n + (warp * 2 + half) * 2 * n;
  float2* B = A + n;
  if (active)
    for (int j = hl; j < n; j += 16) cp_async8(&A[j], gline + j);
  cp_async_commit();
  cp_async_wait<0>();
  __syncwarp();
  const float2* res = line_fft<true>(A, B, n, ax.ns, sa, tw, hl, active);
  if (!active) return;
  if (!POST) {
#pragma unroll 4
    for (int j = hl; j < n; j += 16) gline[j] = res[j];
    return;
  }
  const int nl = gp->n[D - 1], h = nl / 2;
  const float* al = apod + gp->apod_off[D - 1];
  float2* orow = out + gp->img_off + (int64_t)c * gp->nimg + qlin * nl;
#pragma unroll 4
  for (int j = hl; j < nl; j += 16) {
    int sj = j - h;
    if (sj < 0) sj += n;
    const float2 y = res[sj];
    const float a = aout * al[j];
    orow[j] = make_float2(y.x * a, y.y * a);
  }
}

// All stages of a column block's FFT (W columns, elements W apart) by a CTA;
// on return A holds the transform (B is scratch).
template <bool INV, int W>
__device__ __forceinline__ void cols_fft(float2*& A, float2*& B, int n, int ns, const FfxShared& sa,
                                         const float2* tw, int tid) {
  int L = 1;
  for (int s = 0; s < ns; ++s) {
    const int R = sa.radix[s], nr = n / R;
    const unsigned magic = sa.magic[s];
    const float2* t = tw + sa.tw_off[s];
#define MRN_COLS_CALL(RR, FF) cols_stage<RR, INV, FF, W>(A, B, L, magic, nr, t, tid, kFfxThreads)
    MRN_FFX_STAGE(MRN_COLS_CALL);
#undef MRN_COLS_CALL
    __syncthreads();
    float2* tmp = A;
    A = B;
    B = tmp;
    L *= R;
  }
}

// Copy a column block [n][W] into shared memory (cp.async); rows outside
// `keep` (zero padding of the axis, when masked) and columns past the end
// read as zero.
template <int W>
__device__ __forceinline__ void cols_load(float2* A, const float2* base, int64_t stride, int wn, int n, int n_img,
                                          bool mask, int tid) {
  for (int idx = tid; idx < n * W; idx += kFfxThreads) {
    const int rr = idx / W, w = idx - rr * W;
    if (w < wn && (!mask || kept(rr, n_img, n))) cp_async8(&A[idx], base + rr * stride + w);
    else A[idx] = make_float2(0.f, 0.f);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
}

// One strided axis: the grid as [outer][n][stride] (stride = product of the
// later axes' sizes), a CTA per (outer index, block of W adjacent columns).
// Forward: rows in the axis' zero padding read as zero; inverse: only rows
// that survive the crop are stored. skip_nos > 0: the outer index's
// earlier-axis coordinate (outer mod skip_nos) must survive the crop (its
// plane is zero padding in the forward direction, unused in the inverse).
template <bool INV, int W>
__global__ void __launch_bounds__(kFfxThreads)
k_ffx_cols(float2* __restrict__ grid, FfxAxis ax, const float2* __restrict__ twg, int64_t stride,
           int64_t nib, int n_img, int skip_n, int skip_nos) {
  const int64_t blk = blockIdx.x;
  const int64_t o = blk / nib, ib = blk - o * nib;
  if (skip_nos > 0 && !kept((int)(o % skip_nos), skip_n, skip_nos)) return;  // whole CTA
  extern __shared__ float2 fsm[];
  __shared__ FfxShared sa;
  const int n = ax.n, tid = threadIdx.x;
  float2* tw = fsm;
  float2* A = fsm + n;
  float2* B = A + n * W;
  stage_axis(sa, tw, ax, twg);
  const int64_t w0 = ib * W;
  const int wn = (int)min((int64_t)W, stride - w0);
  float2* base = grid + o * n * stride + w0;
  cols_load<W>(A, base, stride, wn, n, n_img, !INV, tid);
  cols_fft<INV, W>(A, B, n, ax.ns, sa, tw, tid);
  for (int idx = tid; idx < n * W; idx += kFfxThreads) {
    const int rr = idx / W, w = idx - rr * W;
    if (w < wn && (!INV || kept(rr, n_img, n))) base[rr * stride + w] = A[idx];
  }
}

int rows_warps(int n) {
  // twiddles + two lines (a half-warp each) of two buffers of n points per
  // warp within 48 KB
  const int w = (int)((48 * 1024 / sizeof(float2) - n) / (4 * n));
  return std::max(1, std::min(8, w));
}

// One strided pass of group q along axis a.
template <int W>
int launch_cols_w(const FfxSet& S, const FfxGrid& G, int q, int a, bool inv, cudaStream_t st) {
  const int D = G.ndim;
  const FfxGroup& fg = S.grp[q];
  const SliceGeom& g = G.hsl[fg.first_slice];
  const FfxAxis& ax = fg.ax[a];
  int64_t stride = 1, outer = fg.batch;
  for (int i = a + 1; i < D; ++i) stride *= g.nos[i];
  for (int i = 0; i < a; ++i) outer *= g.nos[i];
  const int64_t nib = (stride + W - 1) / W;
  const int64_t nblocks = outer * nib;
  if (nblocks <= 0) return MRN_OK;
  if (nblocks > 0x7fffffffLL) return MRN_ERR_UNSUPPORTED;
  const size_t smem = ((size_t)ax.n + 2 * (size_t)ax.n * W) * sizeof(float2);
  const int skip_n = a == 1 ? g.n[0] : 0, skip_nos = a == 1 ? g.nos[0] : 0;
  float2* grid = G.grid + fg.grid_off;
  const unsigned nb = (unsigned)nblocks;
  int rc;
  if (inv) {
    auto kernf = k_ffx_cols<true, W>;
    rc = set_dynamic_smem(kernf, smem);
    if (rc == MRN_OK)
      kernf<<<nb, kFfxThreads, smem, st>>>(grid, ax, S.d_tw, stride, nib, g.n[a], skip_n, skip_nos);
  } else {
    auto kernf = k_ffx_cols<false, W>;
    rc = set_dynamic_smem(kernf, smem);
    if (rc == MRN_OK)
      kernf<<<nb, kFfxThreads, smem, st>>>(grid, ax, S.d_tw, stride, nib, g.n[a], skip_n, skip_nos);
  }
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

// 3D grids (the passes stream from HBM) take blocks of 16 columns (128-byte
// row segments) while those fit in 100 KB of shared memory; 2D grids, which
// stay in L2, take 8 (more CTAs per SM).
int launch_cols(const FfxSet& S, const FfxGrid& G, int q, int a, bool inv, cudaStream_t st) {
  const int n = S.grp[q].ax[a].n;
  if (G.ndim == 3 && ((size_t)n + 32 * (size_t)n) * sizeof(float2) <= 100 * 1024)
    return launch_cols_w<16>(S, G, q, a, inv, st);
  return launch_cols_w<kFfxCols>(S, G, q, a, inv, st);
}

// Last-axis pass of group q: forward fused with the pad (mode), or inverse
// with the crop into out (out != nullptr) or stored back in place.
int launch_rows(const FfxSet& S, const FfxGrid& G, int q, bool inv, PreMode mode, const float2* src,
                const float2* mps, float2* out, float scale, cudaStream_t st) {
  const int D = G.ndim;
  const FfxGroup& fg = S.grp[q];
  const FfxAxis& ax = fg.ax[D - 1];
  const int nw = rows_warps(ax.n);
  const unsigned blocks = (unsigned)((fg.nrows + 2 * nw - 1) / (2 * nw));
  if (blocks == 0) return MRN_OK;
  const size_t smem = ((size_t)ax.n + 4 * (size_t)nw * ax.n) * sizeof(float2);
  const int* gsl = S.d_sl + fg.sl_off;
  const int64_t* grow = S.d_row + fg.row_off;
  const bool sense = mode == kPreSense;
  int rc = MRN_OK;
#define MRN_FFX_ROWS(DD, SS)                                                                       \
  do {                                                                                             \
    auto kern = k_ffx_rows_fwd<DD, SS>;                                                            \
    rc = set_dynamic_smem(kern, smem);                                                             \
    if (rc == MRN_OK)                                                                              \
      kern<<<blocks, nw * 32, smem, st>>>(G.dsl, gsl, grow, fg.nsl, G.apod, src, mps, scale, G.grid, \
                                          fg.nrows, ax, S.d_tw);                                   \
  } while (0)
#define MRN_FFX_IROWS(DD, PP)                                                                      \
  do {                                                                                             \
    auto kern = k_ffx_rows_inv<DD, PP>;                                                            \
    rc = set_dynamic_smem(kern, smem);                                                             \
    if (rc == MRN_OK)                                                                              \
      kern<<<blocks, nw * 32, smem, st>>>(G.dsl, gsl, grow, fg.nsl, G.apod, G.grid, scale, out,   \
                                          fg.nrows, ax, S.d_tw);                                   \
  } while (0)
  if (!inv) {
    if (D == 2) { if (sense) MRN_FFX_ROWS(2, true); else MRN_FFX_ROWS(2, false); }
    else { if (sense) MRN_FFX_ROWS(3, true); else MRN_FFX_ROWS(3, false); }
  } else {
    if (D == 2) { if (out) MRN_FFX_IROWS(2, true); else MRN_FFX_IROWS(2, false); }
    else { if (out) MRN_FFX_IROWS(3, true); else MRN_FFX_IROWS(3, false); }
  }
#undef MRN_FFX_ROWS
#undef MRN_FFX_IROWS
  if (rc != MRN_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

// Radices for n: the 5s and 3s first (the first stage, which has no
// twiddles, stores R apart, and an odd R keeps those stores free of bank
// conflicts), then the power of two 2^e as 8s and one 4 or 2, or as 16s and
// one 8, 4 or 2 where that takes fewer stages; false if n has another prime
// factor.
bool ffx_factor(int n, FfxAxis& ax) {
  ax = FfxAxis{};
  ax.n = n;
  if (n < 2 || n > kFfxMaxN) return false;
  int m = n, s = 0, e = 0;
  auto push = [&](int r) {
    if (s == kFfxMaxStages) return false;
    ax.radix[s++] = r;
    return true;
  };
  for (int r : {5, 3})
    while (m % r == 0) {
      if (!push(r)) return false;
      m /= r;
    }
  while (m % 2 == 0) {
    ++e;
    m /= 2;
  }
  if (m != 1) return false;
  const int stages8 = (e + 2) / 3, stages16 = (e + 3) / 4;
  const int big = stages16 < stages8 ? 4 : 3;  // log2 of the main radix
  for (; e >= big; e -= big)
    if (!push(1 << big)) return false;
  if (e > 0 && !push(1 << e)) return false;
  ax.ns = s;
  return true;
}

template <class T>
int upload(T** dst, const std::vector<T>& v) {
  if (*dst) cudaFree(*dst);
  *dst = nullptr;
  if (cudaMalloc(dst, std::max<size_t>(1, v.size()) * sizeof(T)) != cudaSuccess) return MRN_ERR_CUDA;
  if (!v.empty() && cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return MRN_ERR_CUDA;
  return MRN_OK;
}

FfxGrid plan_grid(mrn_plan* P) {
  return FfxGrid{P->ndim, P->h_slices.data(), P->d_slices, P->d_apod, P->d_grid};
}

}  // namespace

// Build the native FFT of a grid buffer: per group spec (grid size, block
// offset, coils), the group's slices (those of that grid size, in slice
// order), its axes' twiddle tables and slice / row lists. A group whose
// slices differ in image size, or with an axis that has a prime factor above
// 5 or more than kFfxMaxN points, is not native.
int ffx_build(FfxSet& S, int ndim, const std::vector<SliceGeom>& hsl, const std::vector<FfxGroupSpec>& spec) {
  S.release();
  if ((ndim != 2 && ndim != 3) || hsl.empty()) return MRN_OK;
  const int D = ndim;
  std::vector<float2> tab;
  std::vector<int> sl_ids;
  std::vector<int64_t> rows;
  int nnative = 0;
  for (const FfxGroupSpec& gs : spec) {
    FfxGroup fg{};
    fg.native = true;
    fg.first_slice = -1;
    fg.sl_off = (int)sl_ids.size();
    fg.row_off = (int)rows.size();
    fg.grid_off = gs.grid_off;
    fg.batch = gs.batch;
    int64_t r = 0;
    for (int s = 0; s < (int)hsl.size(); ++s) {
      const SliceGeom& g = hsl[s];
      bool same = true;
      for (int i = 0; i < D; ++i) same &= g.nos[i] == gs.nos[i];
      if (!same) continue;
      if (fg.first_slice < 0) fg.first_slice = s;
      const SliceGeom& g0 = hsl[fg.first_slice];
      for (int i = 0; i < D; ++i) fg.native &= g.n[i] == g0.n[i];
      sl_ids.push_back(s);
      rows.push_back(r);
      r += (int64_t)g.ncoil * (g.gos / g.nos[D - 1]);
      ++fg.nsl;
    }
    rows.push_back(r);
    fg.nrows = r;
    if (fg.first_slice < 0) fg.native = false;
    for (int i = 0; i < D; ++i) {
      FfxAxis& ax = fg.ax[i];
      if (!ffx_factor(gs.nos[i], ax)) {
        fg.native = false;
        continue;
      }
      ax.tw_base = (int)tab.size();
      int L = 1, off = 0;
      for (int st = 0; st < ax.ns; ++st) {
        const int R = ax.radix[st];
        ax.tw_off[st] = off;
        ax.magic[st] = L > 1 ? (unsigned)((1ull << 32) / (unsigned long long)L + 1ull) : 0u;
        for (int j = 0; j < L; ++j)
          for (int t = 1; t < R; ++t) {
            const double ang = -2.0 * M_PI * (double)t * (double)j / (double)(L * R);
            tab.push_back(make_float2((float)std::cos(ang), (float)std::sin(ang)));
          }
        off += L * (R - 1);
        L *= R;
      }
    }
    nnative += fg.native ? 1 : 0;
    S.grp.push_back(fg);
  }
  if (nnative == 0) {
    S.grp.clear();
    return MRN_OK;
  }
  int rc = upload(&S.d_tw, tab);
  if (rc == MRN_OK) rc = upload(&S.d_sl, sl_ids);
  if (rc == MRN_OK) rc = upload(&S.d_row, rows);
  if (rc != MRN_OK) {
    S.release();
    return rc;
  }
  S.ok = true;
  S.all = nnative == (int)spec.size();
  return MRN_OK;
}

int ffx_fwd(const FfxSet& S, const FfxGrid& G, PreMode mode, const float2* src, const float2* mps, float scale,
            cudaStream_t st) {
  for (size_t q = 0; q < S.grp.size(); ++q) {
    if (!S.grp[q].native) continue;
    int rc = launch_rows(S, G, (int)q, false, mode, src, mps, nullptr, scale, st);
    for (int a = G.ndim - 2; a >= 0 && rc == MRN_OK; --a) rc = launch_cols(S, G, (int)q, a, false, st);
    if (rc != MRN_OK) return rc;
  }
  return MRN_OK;
}

int ffx_inv(const FfxSet& S, const FfxGrid& G, float2* out, float scale, cudaStream_t st) {
  for (size_t q = 0; q < S.grp.size(); ++q) {
    if (!S.grp[q].native) continue;
    int rc = MRN_OK;
    for (int a = 0; a <= G.ndim - 2 && rc == MRN_OK; ++a) rc = launch_cols(S, G, (int)q, a, true, st);
    if (rc == MRN_OK) rc = launch_rows(S, G, (int)q, true, kPrePlain, nullptr, nullptr, out, scale, st);
    if (rc != MRN_OK) return rc;
  }
  return MRN_OK;
}

bool ffx_active(const mrn_plan* P) { return P->ffx.ok && P->use_ffx; }

// Per-slice flags: the slice's group runs the native passes (and k_pre /
// k_post leave it alone).
int ffx_refresh(mrn_plan* P) {
  if (P->h_slices.empty() || !P->d_slices) return MRN_OK;
  const int D = P->ndim;
  for (auto& g : P->h_slices) {
    g.native_fft = 0;
    if (!P->use_ffx) continue;
    for (const auto& fg : P->ffx.grp) {
      bool same = fg.native;
      for (int i = 0; i < D && same; ++i) same = g.nos[i] == fg.ax[i].n;
      if (same) g.native_fft = 1;
    }
  }
  return upload_slices(P) == cudaSuccess ? MRN_OK : MRN_ERR_CUDA;
}

// The plan grid's native FFT (plan creation, after the FFT groups exist).
int ffx_setup(mrn_plan* P) {
  P->ffx.release();
  if (P->flags & MRN_PLAN_RAW) return MRN_OK;
  std::vector<FfxGroupSpec> spec;
  for (const auto& f : P->fft) {
    FfxGroupSpec gs{};
    for (int i = 0; i < kMaxDim; ++i) gs.nos[i] = f.nos[i];
    gs.grid_off = f.grid_off;
    gs.batch = f.batch;
    spec.push_back(gs);
  }
  const int rc = ffx_build(P->ffx, P->ndim, P->h_slices, spec);
  if (rc != MRN_OK) return rc;
  return ffx_refresh(P);
}

// Apodize / pad (plain image or SENSE x * maps) and forward FFT of the grid.
int ffx_forward(mrn_plan* P, PreMode mode, const float2* src, const float2* mps, float scale, cudaStream_t st) {
  return ffx_fwd(P->ffx, plan_grid(P), mode, src, mps, scale, st);
}

// Inverse FFT of the grid; out != nullptr: crop / deapodize into the image
// batch (plain adjoint), else the surviving lines stay in the grid.
int ffx_inverse(mrn_plan* P, float2* out, float scale, cudaStream_t st) {
  return ffx_inv(P->ffx, plan_grid(P), out, scale, st);
}

}  // namespace mrn
