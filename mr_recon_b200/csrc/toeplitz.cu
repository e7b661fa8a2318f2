// Toeplitz (FFT-only) normal operator A^H A of the NUFFT: the kernel K is the
// centred FFT of the point-spread function on a padded grid (normally twice
// the image size), and
//   normal(x)_c = crop(IFFT(K * FFT(pad(x_c))))           (plain, per image)
//   normal(x)   = sum_c conj(S_c) crop(IFFT(K * FFT(pad(S_c x))))   (SENSE)
// with centred orthonormal FFTs (ifftshift -> fftn -> fftshift) and the
// centred pad / crop of PadLast.
//
// Reference: NUFFT.normal_toeplitz (fourier.py:302-352), the Toeplitz branch
// of sense_linop.normal (linops.py:1249-1308) and calc_teoplitz_kernels
// (fourier.py:552-582), which pad, FFT, multiply, inverse-FFT and crop with
// separate torch passes (and for SENSE an einsum over coils). Here the pad,
// the coil-map product and both shifts are index maps of one pre kernel:
// padded FFT storage cell s (per dimension) holds centred cell
// p = (s + np//2) mod np, i.e. image cell q = p - (np - n)/2; the kernel is
// reordered to storage order once, with the orthonormal scaling 1/prod(np) of
// the two FFTs folded in; the crop, conj(coil-map) sum, lambda x and
// Re<x, out> are one post kernel. cuFFT does the two batched transforms.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "internal.cuh"

namespace mrn {

// per slice: padded grid geometry of the Toeplitz operator
struct ToepGeom {
  int n[kMaxDim];    // image size (1 for unused dims)
  int np[kMaxDim];   // padded (FFT) size
  int off[kMaxDim];  // (np - n) / 2, the centred pad offset
  int ncoil;
  int64_t gp;        // prod(np)
  int64_t grid_off;  // complex offset of the slice's [C][np...] block in the Toeplitz grid
  int64_t kern_off;  // complex offset of the slice's kernel (storage order, scaled)
  int64_t img_off;   // image layout [C][N...] offset (plain mode input/output, SENSE maps)
  int64_t x_off;     // one-image-per-slice offset (SENSE x / out)
  int64_t nimg;      // prod(n)
  int64_t prow_off;  // first padded row (all dims but the last, all coils)
  int64_t irow_off;  // first image row, all coils (plain output rows)
  int64_t xrow_off;  // first image row, one image (SENSE output rows)
};

struct ToepState {
  std::vector<ToepGeom> h;
  ToepGeom* d = nullptr;
  float2* grid = nullptr;  // padded grids, per slice [C][np...] in FFT storage order
  float2* kern = nullptr;  // kernels in storage order, scaled by 1 / prod(np)
  int64_t n_grid = 0, n_kern = 0, n_prow = 0;
  struct Group {
    int np[kMaxDim];
    int64_t grid_off;
    int batch;
    cufftHandle handle;
  };
  std::vector<Group> fft;
};

__device__ __forceinline__ int toep_slice(const ToepGeom* g, int ns, int64_t row, int which) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int64_t o = which == 0 ? g[mid].prow_off : (which == 1 ? g[mid].irow_off : g[mid].xrow_off);
    if (o <= row) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// One warp per padded row (all dims but the last) of one coil of one slice:
// grid[c][s] = pad(x_c)[p(s)] (plain) or pad(S_c x)[p(s)] (SENSE).
template <int D>
__global__ void __launch_bounds__(256)
k_toep_pre(const ToepGeom* __restrict__ tg, int ns, const float2* __restrict__ src,
           const float2* __restrict__ mps, float2* __restrict__ grid, int64_t nrows) {
  const int64_t row = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const ToepGeom& g = tg[toep_slice(tg, ns, row, 0)];
  const int64_t r = row - g.prow_off;
  const int64_t outer = g.gp / g.np[D - 1];
  const int c = (int)(r / outer);
  int64_t o = r - (int64_t)c * outer;
  const int64_t orow = o;
  bool valid = true;
  int64_t qlin = 0;
  int st[kMaxDim] = {0, 0, 0};
  for (int i = D - 2; i >= 0; --i) {
    st[i] = (int)(o % g.np[i]);
    o /= g.np[i];
  }
  for (int i = 0; i < D - 1; ++i) {
    int p = st[i] + g.np[i] / 2;
    if (p >= g.np[i]) p -= g.np[i];
    const int q = p - g.off[i];
    valid &= q >= 0 && q < g.n[i];
    qlin = qlin * g.n[i] + q;
  }
  const int nl = g.n[D - 1], npl = g.np[D - 1], offl = g.off[D - 1], hl = npl / 2;
  float2* dst = grid + g.grid_off + (int64_t)c * g.gp + orow * npl;
  if (!valid) {
    for (int j = lane; j < npl; j += 32) dst[j] = make_float2(0.f, 0.f);
    return;
  }
  qlin *= nl;
  const float2* srow = mps ? src + g.x_off + qlin : src + g.img_off + (int64_t)c * g.nimg + qlin;
  const float2* mrow = mps ? mps + g.img_off + (int64_t)c * g.nimg + qlin : nullptr;
#pragma unroll 4
  for (int j = lane; j < npl; j += 32) {
    int p = j + hl;
    if (p >= npl) p -= npl;
    const int q = p - offl;
    float2 v = make_float2(0.f, 0.f);
    if (q >= 0 && q < nl) {
      v = __ldg(srow + q);
      if (mrow) {
        const float2 m = __ldg(mrow + q);
        v = make_float2(v.x * m.x - v.y * m.y, v.x * m.y + v.y * m.x);
      }
    }
    dst[j] = v;
  }
}

// grid[c][s] *= kern[s] for every coil of slice blockIdx.y (storage order).
__global__ void __launch_bounds__(256)
k_toep_mul(const ToepGeom* __restrict__ tg, const float2* __restrict__ kern, float2* __restrict__ grid) {
  const ToepGeom& g = tg[blockIdx.y];
  const int64_t total = (int64_t)g.ncoil * g.gp;
  float2* gs = grid + g.grid_off;
  const float2* ks = kern + g.kern_off;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e % g.gp;
    const float2 k = __ldg(ks + j);
    const float2 v = gs[e];
    gs[e] = make_float2(v.x * k.x - v.y * k.y, v.x * k.y + v.y * k.x);
  }
}

// Reorder a centred kernel (caller layout, per slice [np...]) into FFT storage
// order and scale it: kern[s] = src[p(s)] * scale.
template <int D>
__global__ void k_toep_kernel(const ToepGeom* __restrict__ tg, int ns, const float2* __restrict__ src,
                              float2* __restrict__ kern, int64_t total) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tg[mid].kern_off <= e) lo = mid; else hi = mid - 1;
  }
  const ToepGeom& g = tg[lo];
  int64_t rem = e - g.kern_off;
  int64_t plin = 0;
  int s[kMaxDim] = {0, 0, 0};
  for (int i = D - 1; i >= 0; --i) {
    s[i] = (int)(rem % g.np[i]);
    rem /= g.np[i];
  }
  for (int i = 0; i < D; ++i) {
    int p = s[i] + g.np[i] / 2;
    if (p >= g.np[i]) p -= g.np[i];
    plin = plin * g.np[i] + p;
  }
  const float2 v = src[g.kern_off + plin];
  const float sc = 1.0f / (float)g.gp;
  kern[e] = make_float2(v.x * sc, v.y * sc);
}

// One warp per image row. Plain: out[c][q] = grid[c][s(q)]. SENSE: out[q] =
// scale * sum_c conj(mps_c[q]) grid[c][s(q)] (+ lam * xin[q]); with pap, the
// row's Re<xin, out> goes to rowpart[row] and the last block adds each
// slice's rows in row order into pap[slice * pap_stride] (same bits on every
// run, as the NUFFT's k_post).
template <int D>
__global__ void __launch_bounds__(256)
k_toep_post(const ToepGeom* __restrict__ tg, int ns, const float2* __restrict__ grid,
            const float2* __restrict__ mps, float scale, float2* __restrict__ out,
            const float2* __restrict__ xin, float lam, double* __restrict__ pap, int pap_stride,
            int64_t nrows, double* __restrict__ rowpart, unsigned* __restrict__ counter) {
  const int64_t row = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row < nrows) {
    const bool sense = mps != nullptr;
    const ToepGeom& g = tg[toep_slice(tg, ns, row, sense ? 2 : 1)];
    const int64_t r = row - (sense ? g.xrow_off : g.irow_off);
    const int64_t outer = g.nimg / g.n[D - 1];
    const int c_plain = sense ? 0 : (int)(r / outer);
    int64_t o = r - (int64_t)c_plain * outer;
    const int64_t orow = o;
    int q[kMaxDim] = {0, 0, 0};
    for (int i = D - 2; i >= 0; --i) {
      q[i] = (int)(o % g.n[i]);
      o /= g.n[i];
    }
    int64_t slin = 0;
    for (int i = 0; i < D - 1; ++i) {
      int s = q[i] + g.off[i] - g.np[i] / 2;
      if (s < 0) s += g.np[i];
      slin = slin * g.np[i] + s;
    }
    const int nl = g.n[D - 1], npl = g.np[D - 1], sh = g.off[D - 1] - npl / 2;
    slin *= npl;
    double part = 0.0;
    if (!sense) {
      const float2* yrow = grid + g.grid_off + (int64_t)c_plain * g.gp + slin;
      float2* orow_p = out + g.img_off + (int64_t)c_plain * g.nimg + orow * nl;
      for (int j = lane; j < nl; j += 32) {
        int s = j + sh;
        if (s < 0) s += npl;
        orow_p[j] = yrow[s];
      }
    } else {
      float2* orow_p = out + g.x_off + orow * nl;
      const float2* xrow = xin ? xin + g.x_off + orow * nl : nullptr;
      for (int j = lane; j < nl; j += 32) {
        int s = j + sh;
        if (s < 0) s += npl;
        float ax = 0.f, ay = 0.f;
#pragma unroll 4
        for (int c = 0; c < g.ncoil; ++c) {
          const float2 y = grid[g.grid_off + (int64_t)c * g.gp + slin + s];
          const float2 m = __ldg(mps + g.img_off + (int64_t)c * g.nimg + orow * nl + j);
          ax += m.x * y.x + m.y * y.y;  // conj(m) * y
          ay += m.x * y.y - m.y * y.x;
        }
        float2 v = make_float2(ax * scale, ay * scale);
        if (xrow) {
          const float2 xv = xrow[j];
          v.x += lam * xv.x;
          v.y += lam * xv.y;
          part += (double)xv.x * v.x + (double)xv.y * v.y;
        }
        orow_p[j] = v;
      }
      if (pap) {
        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
        if (lane == 0) rowpart[row] = part;
      }
    }
  }
  if (!pap) return;
  __syncthreads();
  if (!arrive_last_block(counter, gridDim.x)) return;
  const int warp = threadIdx.x >> 5;
  for (int qs = warp; qs < ns; qs += 8) {
    const ToepGeom& g = tg[qs];
    const double v = warp_sum_fixed(rowpart + g.xrow_off, g.nimg / g.n[D - 1], lane);
    if (lane == 0) pap[(int64_t)qs * pap_stride] += v;
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0u;
}

// SENSE form of the post step with one block per image row and one thread
// per pixel (same per-pixel arithmetic and coil order as k_toep_post; the
// row's Re<xin, out> is a fixed-order block sum).
template <int D>
__global__ void __launch_bounds__(256)
k_toep_post_sense(const ToepGeom* __restrict__ tg, int ns, const float2* __restrict__ grid,
                  const float2* __restrict__ mps, float scale, float2* __restrict__ out,
                  const float2* __restrict__ xin, float lam, double* __restrict__ pap, int pap_stride,
                  double* __restrict__ rowpart, unsigned* __restrict__ counter) {
  __shared__ double red[8];
  const int64_t row = blockIdx.x;
  const ToepGeom& g = tg[toep_slice(tg, ns, row, 2)];
  int64_t o = row - g.xrow_off;
  const int64_t orow = o;
  int q[kMaxDim] = {0, 0, 0};
  for (int i = D - 2; i >= 0; --i) {
    q[i] = (int)(o % g.n[i]);
    o /= g.n[i];
  }
  int64_t slin = 0;
  for (int i = 0; i < D - 1; ++i) {
    int sidx = q[i] + g.off[i] - g.np[i] / 2;
    if (sidx < 0) sidx += g.np[i];
    slin = slin * g.np[i] + sidx;
  }
  const int nl = g.n[D - 1], npl = g.np[D - 1], sh = g.off[D - 1] - npl / 2;
  slin *= npl;
  float2* orow_p = out + g.x_off + orow * nl;
  const float2* xrow = xin ? xin + g.x_off + orow * nl : nullptr;
  double part = 0.0;
  for (int j = threadIdx.x; j < nl; j += blockDim.x) {
    int sj = j + sh;
    if (sj < 0) sj += npl;
    float ax = 0.f, ay = 0.f;
#pragma unroll 8
    for (int c = 0; c < g.ncoil; ++c) {
      const float2 y = grid[g.grid_off + (int64_t)c * g.gp + slin + sj];
      const float2 m = __ldg(mps + g.img_off + (int64_t)c * g.nimg + orow * nl + j);
      ax += m.x * y.x + m.y * y.y;  // conj(m) * y
      ay += m.x * y.y - m.y * y.x;
    }
    float2 v = make_float2(ax * scale, ay * scale);
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
  __syncthreads();
  if (!arrive_last_block(counter, gridDim.x)) return;
  for (int qs = warp; qs < ns; qs += (int)(blockDim.x >> 5)) {
    const ToepGeom& gq = tg[qs];
    const double v = warp_sum_fixed(rowpart + gq.xrow_off, gq.nimg / gq.n[D - 1], lane);
    if (lane == 0) pap[(int64_t)qs * pap_stride] += v;
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0u;
}

static ToepState* toep(mrn_plan* P) { return static_cast<ToepState*>(P->toep); }

void toep_free(mrn_plan* P) {
  ToepState* T = toep(P);
  if (!T) return;
  for (auto& fg : T->fft)
    if (fg.handle) cufftDestroy(fg.handle);
  if (T->d) cudaFree(T->d);
  if (T->grid) cudaFree(T->grid);
  if (T->kern) cudaFree(T->kern);
  delete T;
  P->toep = nullptr;
}

}  // namespace mrn

using namespace mrn;

#define CKT(x)                                   \
  do {                                           \
    cudaError_t _e = (x);                        \
    if (_e != cudaSuccess) return cuda_fail(_e); \
  } while (0)

extern "C" {

int mrn_plan_set_toeplitz(mrn_plan* P, const int* pad_size, const void* kern, void* stream) {
  if (!P || !pad_size || !kern || (P->flags & MRN_PLAN_RAW)) return MRN_ERR_ARG;
  const int D = P->ndim;
  cudaStream_t st = (cudaStream_t)stream;
  for (int s = 0; s < P->nslices; ++s)
    for (int i = 0; i < D; ++i) {
      const int np = pad_size[s * D + i], n = P->h_slices[s].n[i];
      // PadLast pads (np - n) / 2 on both sides: np - n must be even
      if (np < n || ((np - n) & 1)) return MRN_ERR_ARG;
    }
  // same padded sizes as before: keep buffers and FFT plans, refresh the kernel
  ToepState* T = toep(P);
  bool same = T != nullptr;
  if (same)
    for (int s = 0; s < P->nslices && same; ++s)
      for (int i = 0; i < D; ++i) same &= T->h[s].np[i] == pad_size[s * D + i];
  if (!same) {
    toep_free(P);
    T = new ToepState();
    P->toep = T;
    T->h.resize(P->nslices);
    int64_t goff = 0, koff = 0, prow = 0;
    for (int s = 0; s < P->nslices; ++s) {
      const SliceGeom& g = P->h_slices[s];
      ToepGeom& t = T->h[s];
      int64_t gp = 1;
      for (int i = 0; i < kMaxDim; ++i) {
        t.n[i] = i < D ? g.n[i] : 1;
        t.np[i] = i < D ? pad_size[s * D + i] : 1;
        t.off[i] = (t.np[i] - t.n[i]) / 2;
        gp *= t.np[i];
      }
      t.ncoil = g.ncoil;
      t.gp = gp;
      t.kern_off = koff;
      t.img_off = g.img_off;
      t.x_off = g.x_off;
      t.nimg = g.nimg;
      t.irow_off = g.irow_off;
      t.xrow_off = g.xrow_off;
      t.prow_off = prow;
      prow += (int64_t)g.ncoil * gp / t.np[D - 1];
      koff += gp;
    }
    // grid blocks grouped by padded size (one batched cuFFT plan per group)
    for (int s = 0; s < P->nslices; ++s) {
      ToepGeom& t = T->h[s];
      int found = -1;
      for (size_t q = 0; q < T->fft.size(); ++q) {
        bool eq = true;
        for (int i = 0; i < D; ++i) eq &= T->fft[q].np[i] == t.np[i];
        if (eq) { found = (int)q; break; }
      }
      if (found < 0) {
        ToepState::Group fg{};
        for (int i = 0; i < kMaxDim; ++i) fg.np[i] = t.np[i];
        T->fft.push_back(fg);
        found = (int)T->fft.size() - 1;
      }
      T->fft[found].batch += t.ncoil;
    }
    for (size_t q = 0; q < T->fft.size(); ++q) {
      T->fft[q].grid_off = goff;
      for (int s = 0; s < P->nslices; ++s) {
        ToepGeom& t = T->h[s];
        bool eq = true;
        for (int i = 0; i < D; ++i) eq &= T->fft[q].np[i] == t.np[i];
        if (!eq) continue;
        t.grid_off = goff;
        goff += (int64_t)t.ncoil * t.gp;
      }
    }
    T->n_grid = goff;
    T->n_kern = koff;
    T->n_prow = prow;
    CKT(cudaSetDevice(P->device));
    CKT(cudaMalloc(&T->d, P->nslices * sizeof(ToepGeom)));
    CKT(cudaMemcpy(T->d, T->h.data(), P->nslices * sizeof(ToepGeom), cudaMemcpyHostToDevice));
    CKT(cudaMalloc(&T->grid, std::max<int64_t>(goff, 1) * sizeof(float2)));
    CKT(cudaMalloc(&T->kern, std::max<int64_t>(koff, 1) * sizeof(float2)));
    for (auto& fg : T->fft) {
      int n[kMaxDim];
      for (int i = 0; i < D; ++i) n[i] = fg.np[i];
      if (cufftPlanMany(&fg.handle, D, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, fg.batch) != CUFFT_SUCCESS) {
        fg.handle = 0;
        toep_free(P);
        return MRN_ERR_CUFFT;
      }
    }
  }
  const unsigned nb = (unsigned)((T->n_kern + 255) / 256);
  if (D == 1) k_toep_kernel<1><<<nb, 256, 0, st>>>(T->d, P->nslices, (const float2*)kern, T->kern, T->n_kern);
  else if (D == 2) k_toep_kernel<2><<<nb, 256, 0, st>>>(T->d, P->nslices, (const float2*)kern, T->kern, T->n_kern);
  else k_toep_kernel<3><<<nb, 256, 0, st>>>(T->d, P->nslices, (const float2*)kern, T->kern, T->n_kern);
  CKT(cudaGetLastError());
  return MRN_OK;
}

}  // extern "C"

namespace mrn {

// pre (pad, optional coil-map product) -> FFT -> x K -> inverse FFT -> post
static int toep_apply(mrn_plan* P, const float2* src, const float2* mps, float2* out, float scale,
                      const float2* xin, float lam, double* pap, int pap_stride, cudaStream_t st) {
  ToepState* T = toep(P);
  if (!T) return MRN_ERR_STATE;
  const int D = P->ndim, ns = P->nslices;
  {
    StageTimer t(P, kStagePre, st);
    const unsigned nb = (unsigned)((T->n_prow + 7) / 8);
    if (D == 1) k_toep_pre<1><<<nb, 256, 0, st>>>(T->d, ns, src, mps, T->grid, T->n_prow);
    else if (D == 2) k_toep_pre<2><<<nb, 256, 0, st>>>(T->d, ns, src, mps, T->grid, T->n_prow);
    else k_toep_pre<3><<<nb, 256, 0, st>>>(T->d, ns, src, mps, T->grid, T->n_prow);
    CKT(cudaGetLastError());
  }
  {
    StageTimer t(P, kStageFft, st);
    for (auto& fg : T->fft) {
      if (cufftSetStream(fg.handle, st) != CUFFT_SUCCESS) return MRN_ERR_CUFFT;
      cufftComplex* p = reinterpret_cast<cufftComplex*>(T->grid + fg.grid_off);
      if (cufftExecC2C(fg.handle, p, p, CUFFT_FORWARD) != CUFFT_SUCCESS) return MRN_ERR_CUFFT;
    }
    int64_t most = 1;
    for (const auto& t : T->h) most = std::max<int64_t>(most, (int64_t)t.ncoil * t.gp);
    const unsigned nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((most + 255) / 256,
                                                                        (8 * (int64_t)P->sm_count + ns - 1) / ns));
    k_toep_mul<<<dim3(nb, (unsigned)ns), 256, 0, st>>>(T->d, T->kern, T->grid);
    CKT(cudaGetLastError());
    for (auto& fg : T->fft) {
      cufftComplex* p = reinterpret_cast<cufftComplex*>(T->grid + fg.grid_off);
      if (cufftExecC2C(fg.handle, p, p, CUFFT_INVERSE) != CUFFT_SUCCESS) return MRN_ERR_CUFFT;
    }
  }
  StageTimer t(P, kStagePost, st);
  const int64_t nrows = mps ? P->n_xrow : P->n_irow;
  const unsigned nb = (unsigned)((nrows + 7) / 8);
  if (nb == 0) return MRN_OK;
  if (mps) {
    int nl = 1;
    for (const auto& tgh : T->h) nl = std::max(nl, tgh.n[D - 1]);
    const unsigned threads = nl <= 64 ? 64 : (nl <= 128 ? 128 : 256);
    const unsigned rows = (unsigned)nrows;
    if (D == 1)
      k_toep_post_sense<1><<<rows, threads, 0, st>>>(T->d, ns, T->grid, mps, scale, out, xin, lam, pap, pap_stride, P->d_rowpart, P->d_sync + 3);
    else if (D == 2)
      k_toep_post_sense<2><<<rows, threads, 0, st>>>(T->d, ns, T->grid, mps, scale, out, xin, lam, pap, pap_stride, P->d_rowpart, P->d_sync + 3);
    else
      k_toep_post_sense<3><<<rows, threads, 0, st>>>(T->d, ns, T->grid, mps, scale, out, xin, lam, pap, pap_stride, P->d_rowpart, P->d_sync + 3);
    CKT(cudaGetLastError());
    return MRN_OK;
  }
  if (!mps) pap = nullptr;
  if (D == 1)
    k_toep_post<1><<<nb, 256, 0, st>>>(T->d, ns, T->grid, mps, scale, out, xin, lam, pap, pap_stride, nrows, P->d_rowpart, P->d_sync + 3);
  else if (D == 2)
    k_toep_post<2><<<nb, 256, 0, st>>>(T->d, ns, T->grid, mps, scale, out, xin, lam, pap, pap_stride, nrows, P->d_rowpart, P->d_sync + 3);
  else
    k_toep_post<3><<<nb, 256, 0, st>>>(T->d, ns, T->grid, mps, scale, out, xin, lam, pap, pap_stride, nrows, P->d_rowpart, P->d_sync + 3);
  CKT(cudaGetLastError());
  return MRN_OK;
}

}  // namespace mrn

extern "C" {

int mrn_toeplitz_normal(mrn_plan* P, const void* img, void* out, void* stream) {
  if (!P || !img || !out) return MRN_ERR_ARG;
  return toep_apply(P, (const float2*)img, nullptr, (float2*)out, 1.0f, nullptr, 0.f, nullptr, 0,
                    (cudaStream_t)stream);
}

int mrn_sense_normal_toeplitz(mrn_plan* P, const void* x, const void* mps, void* out, float out_scale,
                              float lam, double* pap, int pap_stride, void* stream) {
  if (!P || !x || !mps || !out) return MRN_ERR_ARG;
  return toep_apply(P, (const float2*)x, (const float2*)mps, (float2*)out, out_scale, (const float2*)x,
                    lam, pap, pap_stride, (cudaStream_t)stream);
}

}  // extern "C"
