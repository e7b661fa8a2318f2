// FFT stage of the NUFFT: fused pre-FFT (apodize, scale, centred zero-pad,
// ifftshift, optional coil-map product) and post-iFFT (fftshift, centred crop,
// scale, apodize, optional conj(coil-map) sum) kernels around batched cuFFT.
//
// Reference: triton_nufft.forward_FT_only / adjoint_iFT_only
// (fourier.py:432-468, 505-525) do clone, d in-place apodization passes, a
// division, utils.resize (utils.py:41-84) and fft()/ifft() (fourier.py:37-61)
// with two shift copies each. Here the shifts and the pad/crop are index maps:
//   image cell q (per dim)  <->  FFT storage cell (q - N//2) mod Nos,
// which is exactly ifftshift(resize(x)) on the way in and resize(fftshift(y))
// on the way out, for even and odd sizes alike. The oversampled grid is kept
// in natural FFT order; the interpolation/gridding kernels address centred
// cell k at storage (k - Nos//2) mod Nos, which is the reference's fftshift.
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace mrn {

// One warp per grid row (all dims but the last) of one coil of one slice.
template <int D>
__global__ void __launch_bounds__(256)
k_pre(const SliceGeom* __restrict__ sl, int ns, const float* __restrict__ apod,
      const float2* __restrict__ src, const float2* __restrict__ mps, int mode, float scale,
      float2* __restrict__ grid, int64_t nrows) {
  const int64_t row = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const int s = slice_by_row(sl, ns, row, 0);
  const SliceGeom& g = sl[s];
  if (g.native_fft) return;  // padded by the native forward pass
  const int64_t r = row - g.prow_off;
  const int64_t outer = g.gos / g.nos[D - 1];
  const int c = (int)(r / outer);
  int64_t o = r - (int64_t)c * outer;
  // storage coords of the outer dims -> image coords
  float aout = scale * g.inv_sqrt_n;
  bool valid = true;
  int64_t qlin = 0;
  int st[kMaxDim] = {0, 0, 0};
  for (int i = D - 2; i >= 0; --i) {
    st[i] = (int)(o % g.nos[i]);
    o /= g.nos[i];
  }
  for (int i = 0; i < D - 1; ++i) {
    const int q = (st[i] + g.n[i] / 2) % g.nos[i];
    valid &= q < g.n[i];
    if (q < g.n[i]) aout *= apod[g.apod_off[i] + q];
    qlin = qlin * g.n[i] + q;
  }
  const int nl = g.n[D - 1], nosl = g.nos[D - 1];
  float2* dst = grid + g.grid_off + (int64_t)c * g.gos + (r - (int64_t)c * outer) * nosl;
  if (!valid) {
    for (int j = lane; j < nosl; j += 32) dst[j] = make_float2(0.f, 0.f);
    return;
  }
  qlin *= nl;
  const float* al = apod + g.apod_off[D - 1];
  const float2* srow;
  const float2* mrow = nullptr;
  if (mode == kPreSense) {
    srow = src + g.x_off + qlin;
    mrow = mps + g.img_off + (int64_t)c * g.nimg + qlin;
  } else {
    srow = src + g.img_off + (int64_t)c * g.nimg + qlin;
  }
  const int h = nl / 2;
#pragma unroll 4
  for (int j = lane; j < nosl; j += 32) {
    int q = j + h;
    if (q >= nosl) q -= nosl;
    float2 v = make_float2(0.f, 0.f);
    if (q < nl) {
      float2 x = __ldg(srow + q);
      if (mrow) {
        const float2 m = __ldg(mrow + q);
        x = make_float2(x.x * m.x - x.y * m.y, x.x * m.y + x.y * m.x);
      }
      const float a = aout * al[q];
      v = make_float2(x.x * a, x.y * a);
    }
    dst[j] = v;
  }
}

// One warp per image row. Plain: rows over (slice, coil, outer image index),
// out[c][q] = Y_c[(q - N//2) mod Nos] * apod(q) * scale.
// Sense: rows over (slice, outer image index), out[q] = scale * apod(q) *
// sum_c conj(mps_c[q]) Y_c[...] (+ lam * xin[q]); pap[slice] += Re<xin, out>,
// summed reproducibly: each row's warp stores its partial in rowpart[row] and
// the last block adds every slice's rows in row order.
template <int D>
__device__ __forceinline__ void post_row(const SliceGeom* __restrict__ sl, int ns, const float* __restrict__ apod,
                                         const float2* __restrict__ grid, const float2* __restrict__ mps,
                                         int mode, float scale, float2* __restrict__ out,
                                         const float2* __restrict__ xin, float lam,
                                         double* __restrict__ rowpart, int64_t row, int lane);

template <int D>
__global__ void __launch_bounds__(256)
k_post(const SliceGeom* __restrict__ sl, int ns, const float* __restrict__ apod,
       const float2* __restrict__ grid, const float2* __restrict__ mps, int mode, float scale,
       float2* __restrict__ out, const float2* __restrict__ xin, float lam, double* __restrict__ pap,
       int pap_stride, int64_t nrows, double* __restrict__ rowpart, unsigned* __restrict__ counter) {
  const int64_t row = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row < nrows)
    post_row<D>(sl, ns, apod, grid, mps, mode, scale, out, xin, lam, pap ? rowpart : nullptr, row, lane);
  if (!pap) return;
  __syncthreads();  // this block's row partials are stored before thread 0 arrives
  if (!arrive_last_block(counter, gridDim.x)) return;
  const int warp = threadIdx.x >> 5;
  for (int q = warp; q < ns; q += 8) {
    const SliceGeom& g = sl[q];
    const double v = warp_sum_fixed(rowpart + g.xrow_off, g.nimg / g.n[D - 1], lane);
    if (lane == 0) pap[(int64_t)q * pap_stride] += v;
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0u;
}

template <int D>
__device__ __forceinline__ void post_row(const SliceGeom* __restrict__ sl, int ns, const float* __restrict__ apod,
                                         const float2* __restrict__ grid, const float2* __restrict__ mps,
                                         int mode, float scale, float2* __restrict__ out,
                                         const float2* __restrict__ xin, float lam,
                                         double* __restrict__ rowpart, int64_t row, int lane) {
  const int s = slice_by_row(sl, ns, row, mode == kPostSense ? 2 : 1);
  const SliceGeom& g = sl[s];
  if (mode == kPostPlain && g.native_fft) return;  // cropped by the native inverse pass
  const int64_t r = row - (mode == kPostSense ? g.xrow_off : g.irow_off);
  const int64_t outer = g.nimg / g.n[D - 1];
  const int c_plain = mode == kPostSense ? 0 : (int)(r / outer);
  int64_t o = r - (int64_t)c_plain * outer;
  const int64_t orow = o;
  float aout = scale * g.inv_sqrt_n;
  int64_t slin = 0;
  int q[kMaxDim] = {0, 0, 0};
  for (int i = D - 2; i >= 0; --i) {
    q[i] = (int)(o % g.n[i]);
    o /= g.n[i];
  }
  for (int i = 0; i < D - 1; ++i) {
    aout *= apod[g.apod_off[i] + q[i]];
    int sidx = q[i] - g.n[i] / 2;
    if (sidx < 0) sidx += g.nos[i];
    slin = slin * g.nos[i] + sidx;
  }
  const int nl = g.n[D - 1], nosl = g.nos[D - 1];
  slin *= nosl;
  const float* al = apod + g.apod_off[D - 1];
  const int h = nl / 2;
  double part = 0.0;
  if (mode == kPostPlain) {
    const float2* yrow = grid + g.grid_off + (int64_t)c_plain * g.gos + slin;
    float2* orow_p = out + g.img_off + (int64_t)c_plain * g.nimg + orow * nl;
#pragma unroll 4
    for (int j = lane; j < nl; j += 32) {
      int sj = j - h;
      if (sj < 0) sj += nosl;
      const float2 y = yrow[sj];
      const float a = aout * al[j];
      orow_p[j] = make_float2(y.x * a, y.y * a);
    }
  } else {
    float2* orow_p = out + g.x_off + orow * nl;
    const float2* xrow = xin ? xin + g.x_off + orow * nl : nullptr;
    for (int j = lane; j < nl; j += 32) {
      int sj = j - h;
      if (sj < 0) sj += nosl;
      float ax = 0.f, ay = 0.f;
#pragma unroll 4
      for (int c = 0; c < g.ncoil; ++c) {
        const float2 y = grid[g.grid_off + (int64_t)c * g.gos + slin + sj];
        const float2 m = __ldg(mps + g.img_off + (int64_t)c * g.nimg + orow * nl + j);
        // conj(m) * y
        ax += m.x * y.x + m.y * y.y;
        ay += m.x * y.y - m.y * y.x;
      }
      const float a = aout * al[j];
      float2 v = make_float2(ax * a, ay * a);
      if (xrow) {
        const float2 xv = xrow[j];
        v.x += lam * xv.x;
        v.y += lam * xv.y;
        part += (double)xv.x * v.x + (double)xv.y * v.y;
      }
      orow_p[j] = v;
    }
    if (rowpart) {
      for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
      if (lane == 0) rowpart[row] = part;
    }
  }
}

// Copy between the caller's centred grid layout (slice order) and the
// internal natural-order layout (FFT groups): centred k <-> storage (k - Nos//2) mod Nos.
template <int D>
__global__ void k_shift_copy(const SliceGeom* __restrict__ sl, int ns, const float2* __restrict__ src,
                             float2* __restrict__ dst, int to_user, int64_t total) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sl[mid].ugrid_off <= idx) lo = mid; else hi = mid - 1;
  }
  const SliceGeom& g = sl[lo];
  const int64_t r = idx - g.ugrid_off;
  const int64_t c = r / g.gos;
  int64_t cell = r - c * g.gos;
  int k[kMaxDim] = {0, 0, 0};
  for (int i = D - 1; i >= 0; --i) {
    k[i] = (int)(cell % g.nos[i]);
    cell /= g.nos[i];
  }
  int64_t slin = 0;
  for (int i = 0; i < D; ++i) {
    int s = k[i] - g.hshift[i];
    if (s < 0) s += g.nos[i];
    slin = slin * g.nos[i] + s;
  }
  const int64_t ii = g.grid_off + c * g.gos + slin;
  if (to_user) dst[idx] = src[ii];
  else dst[ii] = src[idx];
}

int launch_pre(mrn_plan* P, PreMode mode, const float2* src, const float2* mps, float scale,
               cudaStream_t st) {
  const int64_t nrows = P->n_prow;
  const unsigned blocks = (unsigned)((nrows + 7) / 8);
  if (blocks == 0) return MRN_OK;
  if (P->ndim == 1)
    k_pre<1><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, P->d_apod, src, mps, mode, scale, P->d_grid, nrows);
  else if (P->ndim == 2)
    k_pre<2><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, P->d_apod, src, mps, mode, scale, P->d_grid, nrows);
  else
    k_pre<3><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, P->d_apod, src, mps, mode, scale, P->d_grid, nrows);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

// SENSE post with one block per image row and one thread per pixel (the
// per-warp row kernel above leaves a single 2D image on a few hundred warps):
// out[q] = scale * apod(q) * sum_c conj(mps_c[q]) Y_c[(q - N//2) mod Nos]
// (+ lam * xin[q]), coils summed in order as there. With pap the row's
// Re<xin, out> is a fixed-order block sum into rowpart[row], and the last
// block adds every slice's rows in row order into pap[slice * pap_stride].
template <int D>
__global__ void __launch_bounds__(256)
k_post_sense(const SliceGeom* __restrict__ sl, int ns, const float* __restrict__ apod,
             const float2* __restrict__ grid, const float2* __restrict__ mps, float scale,
             float2* __restrict__ out, const float2* __restrict__ xin, float lam,
             double* __restrict__ pap, int pap_stride, double* __restrict__ rowpart,
             unsigned* __restrict__ counter) {
  __shared__ double red[8];
  const int64_t row = blockIdx.x;
  const int s = slice_by_row(sl, ns, row, 2);
  const SliceGeom& g = sl[s];
  int64_t o = row - g.xrow_off;
  const int64_t orow = o;
  float aout = scale * g.inv_sqrt_n;
  int64_t slin = 0;
  int q[kMaxDim] = {0, 0, 0};
  for (int i = D - 2; i >= 0; --i) {
    q[i] = (int)(o % g.n[i]);
    o /= g.n[i];
  }
  for (int i = 0; i < D - 1; ++i) {
    aout *= apod[g.apod_off[i] + q[i]];
    int sidx = q[i] - g.n[i] / 2;
    if (sidx < 0) sidx += g.nos[i];
    slin = slin * g.nos[i] + sidx;
  }
  const int nl = g.n[D - 1], nosl = g.nos[D - 1], h = nl / 2;
  slin *= nosl;
  const float* al = apod + g.apod_off[D - 1];
  const float2* gbase = grid + g.grid_off + slin;
  const float2* mbase = mps + g.img_off + orow * nl;
  float2* orow_p = out + g.x_off + orow * nl;
  const float2* xrow = xin ? xin + g.x_off + orow * nl : nullptr;
  double part = 0.0;
  for (int j = threadIdx.x; j < nl; j += blockDim.x) {
    int sj = j - h;
    if (sj < 0) sj += nosl;
    float ax = 0.f, ay = 0.f;
#pragma unroll 8
    for (int c = 0; c < g.ncoil; ++c) {
      const float2 y = gbase[(int64_t)c * g.gos + sj];
      const float2 m = __ldg(mbase + (int64_t)c * g.nimg + j);
      // conj(m) * y
      ax += m.x * y.x + m.y * y.y;
      ay += m.x * y.y - m.y * y.x;
    }
    const float a = aout * al[j];
    float2 v = make_float2(ax * a, ay * a);
    if (xrow) {
      const float2 xv = xrow[j];
      v.x += lam * xv.x;
      v.y += lam * xv.y;
      part += (double)xv.x * v.x + (double)xv.y * v.y;
    }
    orow_p[j] = v;
  }
  if (!pap) return;
  for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[warp] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    rowpart[row] = t;
  }
  __syncthreads();  // the row partial is stored before thread 0 arrives
  if (!arrive_last_block(counter, gridDim.x)) return;
  for (int qs = warp; qs < ns; qs += (int)(blockDim.x >> 5)) {
    const SliceGeom& gq = sl[qs];
    const double v = warp_sum_fixed(rowpart + gq.xrow_off, gq.nimg / gq.n[D - 1], lane);
    if (lane == 0) pap[(int64_t)qs * pap_stride] += v;
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0u;
}

int launch_post(mrn_plan* P, PostMode mode, const float2* mps, float2* out, float scale,
                const float2* xin, float lam, double* pap, int pap_stride, cudaStream_t st) {
  const int64_t nrows = mode == kPostSense ? P->n_xrow : P->n_irow;
  if (mode != kPostSense) pap = nullptr;  // Re<x, out> exists only for the SENSE form
  const unsigned blocks = (unsigned)((nrows + 7) / 8);
  if (blocks == 0) return MRN_OK;
  if (mode == kPostSense) {
    int nl = 1;
    for (const auto& g : P->h_slices) nl = std::max(nl, g.n[P->ndim - 1]);
    const unsigned threads = nl <= 64 ? 64 : (nl <= 128 ? 128 : 256);
    const unsigned rows = (unsigned)nrows;
    if (P->ndim == 1)
      k_post_sense<1><<<rows, threads, 0, st>>>(P->d_slices, P->nslices, P->d_apod, P->d_grid, mps, scale, out, xin, lam, pap, pap_stride, P->d_rowpart, P->d_sync + 2);
    else if (P->ndim == 2)
      k_post_sense<2><<<rows, threads, 0, st>>>(P->d_slices, P->nslices, P->d_apod, P->d_grid, mps, scale, out, xin, lam, pap, pap_stride, P->d_rowpart, P->d_sync + 2);
    else
      k_post_sense<3><<<rows, threads, 0, st>>>(P->d_slices, P->nslices, P->d_apod, P->d_grid, mps, scale, out, xin, lam, pap, pap_stride, P->d_rowpart, P->d_sync + 2);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MRN_OK : cuda_fail(e);
  }
  if (P->ndim == 1)
    k_post<1><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, P->d_apod, P->d_grid, mps, mode, scale, out, xin, lam, pap, pap_stride, nrows, P->d_rowpart, P->d_sync + 2);
  else if (P->ndim == 2)
    k_post<2><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, P->d_apod, P->d_grid, mps, mode, scale, out, xin, lam, pap, pap_stride, nrows, P->d_rowpart, P->d_sync + 2);
  else
    k_post<3><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, P->d_apod, P->d_grid, mps, mode, scale, out, xin, lam, pap, pap_stride, nrows, P->d_rowpart, P->d_sync + 2);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_shift_copy(mrn_plan* P, const float2* src, float2* dst, int to_user, cudaStream_t st) {
  const int64_t total = P->n_grid;
  const unsigned blocks = (unsigned)((total + 255) / 256);
  if (blocks == 0) return MRN_OK;
  if (P->ndim == 1)
    k_shift_copy<1><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, src, dst, to_user, total);
  else if (P->ndim == 2)
    k_shift_copy<2><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, src, dst, to_user, total);
  else
    k_shift_copy<3><<<blocks, 256, 0, st>>>(P->d_slices, P->nslices, src, dst, to_user, total);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int fwd_transform(mrn_plan* P, PreMode mode, const float2* src, const float2* mps, float scale,
                  cudaStream_t st) {
  if (ffx_active(P)) {
    StageTimer t(P, kStageFft, st);
    if (!P->ffx.all) {  // groups left to cuFFT: pad them (k_pre skips native slices) and transform
      int rc = launch_pre(P, mode, src, mps, scale, st);
      if (rc == MRN_OK) rc = run_fft(P, CUFFT_FORWARD, st, true);
      if (rc != MRN_OK) return rc;
    }
    return ffx_forward(P, mode, src, mps, scale, st);
  }
  {
    StageTimer t(P, kStagePre, st);
    const int rc = launch_pre(P, mode, src, mps, scale, st);
    if (rc != MRN_OK) return rc;
  }
  StageTimer t(P, kStageFft, st);
  return run_fft(P, CUFFT_FORWARD, st);
}

int inv_transform(mrn_plan* P, float2* out, cudaStream_t st) {
  if (ffx_active(P)) {
    StageTimer t(P, kStageFft, st);
    int rc = ffx_inverse(P, out, 1.0f, st);
    if (rc != MRN_OK || P->ffx.all) return rc;
    rc = run_fft(P, CUFFT_INVERSE, st, true);  // k_post then skips native slices
    if (rc != MRN_OK || !out) return rc;
    return launch_post(P, kPostPlain, nullptr, out, 1.0f, nullptr, 0.f, nullptr, 0, st);
  }
  {
    StageTimer t(P, kStageFft, st);
    const int rc = run_fft(P, CUFFT_INVERSE, st);
    if (rc != MRN_OK) return rc;
  }
  if (!out) return MRN_OK;
  StageTimer t(P, kStagePost, st);
  return launch_post(P, kPostPlain, nullptr, out, 1.0f, nullptr, 0.f, nullptr, 0, st);
}

int run_fft(mrn_plan* P, int direction, cudaStream_t st, bool skip_native) {
  for (size_t q = 0; q < P->fft.size(); ++q) {
    auto& fg = P->fft[q];
    if (skip_native && q < P->ffx.grp.size() && P->ffx.grp[q].native) continue;
    if (cufftSetStream(fg.handle, st) != CUFFT_SUCCESS) return MRN_ERR_CUFFT;
    cufftComplex* p = reinterpret_cast<cufftComplex*>(P->d_grid + fg.grid_off);
    if (cufftExecC2C(fg.handle, p, p, direction) != CUFFT_SUCCESS) return MRN_ERR_CUFFT;
  }
  return MRN_OK;
}

}  // namespace mrn
