// Conjugate-gradient vector steps for a batch of independent systems, one
// image per slice (the loop body of conjugate_gradient, algs.py:779-872).
// Vectors are complex64; every dot product and norm is a float64 sum in a
// fixed order that depends on the slice's own length alone (chunk partials
// added in chunk order by the last block, whatever the launch's grid and
// whatever other slices share the plan), and
// the per-slice scalars never leave the device, so a solve can be captured in
// a CUDA graph (the reference calls .item() every iteration, algs.py:845) and
// replays to the same bits as the eager solve. State per slice, float64[8]:
//   [0] rz   [1] pAp (accumulated)   [2] rr (accumulated)   [3] done
//   [4] tol^2   [5] iterations done   [6] alpha   [7] beta
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace mrn {

constexpr int kCgThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < kCgThreads / 32) t = red[threadIdx.x];
  if (w == 0)
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  return t;  // valid in thread 0
}

// A slice of n elements is summed in chunks of chunk_len(n) elements (a
// multiple of kCgChunk, at most kMaxRedBlocks chunks): chunk c is reduced by
// one block (thread t takes elements c * len + t + k * kCgThreads, then a
// fixed tree), its partial goes to part[slice][c], and the last block adds
// the partials in chunk order. Which block takes a chunk does not matter, so
// the sums are the same for any grid and any other slices in the plan.
constexpr int kCgChunk = kCgThreads * 4;

__device__ __forceinline__ int64_t chunk_len(int64_t n) {
  const int64_t span = (int64_t)kCgChunk * kMaxRedBlocks;
  return (int64_t)kCgChunk * max((n + span - 1) / span, (int64_t)1);
}

__device__ __forceinline__ int64_t chunk_count(int64_t n) {
  const int64_t len = chunk_len(n);
  return (n + len - 1) / len;
}

// The last block adds each slice's chunk partials in chunk order (one warp
// per slice) and adds the total to out[slice * stride], skipping slices whose
// state says done when `state` is given. The result is the same on every
// run, eager or replayed from a graph.
__device__ __forceinline__ void slice_sums(const SliceGeom* __restrict__ sl, double* __restrict__ part,
                                           unsigned* __restrict__ counter, double* __restrict__ out,
                                           int stride, const double* __restrict__ state) {
  const int ns = gridDim.y;
  if (!arrive_last_block(counter, (unsigned)(gridDim.x * ns))) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = warp; q < ns; q += kCgThreads / 32) {
    if (state && state[q * 8 + 3] != 0.0) continue;
    const double v = warp_sum_fixed(part + (int64_t)q * kMaxRedBlocks, chunk_count(sl[q].nimg), lane);
    if (lane == 0) out[(int64_t)q * stride] += v;
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0u;
}

// Chunk loop of one block over its slice: body(k) for every element k of the
// chunk (global index), then the chunk's float64 partial into part.
template <class Body>
__device__ __forceinline__ void chunk_loop(const SliceGeom& g, int s, double* __restrict__ part,
                                           double* red, Body body) {
  const int64_t len = chunk_len(g.nimg), nch = chunk_count(g.nimg);
  for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t e1 = min((c + 1) * len, g.nimg);
    double acc = 0.0;
    for (int64_t i = c * len + threadIdx.x; i < e1; i += kCgThreads) acc += body(g.x_off + i);
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[(int64_t)s * kMaxRedBlocks + c] = acc;
  }
}

// r = b - Ab; p = r; x = b; state[0] += |r|^2; state[4] = tol^2
__global__ void __launch_bounds__(kCgThreads)
k_cg_init(const SliceGeom* __restrict__ sl, const float2* __restrict__ b, const float2* __restrict__ Ab,
          float2* __restrict__ x, float2* __restrict__ r, float2* __restrict__ p,
          double* __restrict__ state, double tol2, double* __restrict__ part, unsigned* __restrict__ counter) {
  __shared__ double red[kCgThreads / 32];
  const int s = blockIdx.y;
  const SliceGeom& g = sl[s];
  chunk_loop(g, s, part, red, [&](int64_t k) {
    const float2 bb = b[k], ab = Ab[k];
    const float2 rr = make_float2(bb.x - ab.x, bb.y - ab.y);
    r[k] = rr;
    p[k] = rr;
    x[k] = bb;
    return (double)rr.x * rr.x + (double)rr.y * rr.y;
  });
  if (threadIdx.x == 0 && blockIdx.x == 0) state[s * 8 + 4] = tol2;
  slice_sums(sl, part, counter, state + 0, 8, nullptr);
}

// alpha = rz / pAp; x += alpha p; r -= alpha Ap; state[2] += |r|^2 (skipped when done)
__global__ void __launch_bounds__(kCgThreads)
k_cg_step(const SliceGeom* __restrict__ sl, float2* __restrict__ x, float2* __restrict__ r,
          const float2* __restrict__ p, const float2* __restrict__ Ap, double* __restrict__ state,
          double* __restrict__ part, unsigned* __restrict__ counter) {
  __shared__ double red[kCgThreads / 32];
  const int s = blockIdx.y;
  const SliceGeom& g = sl[s];
  const double* S = state + s * 8;
  if (S[3] == 0.0) {  // uniform over the block: the whole slice is done or not
    const float alpha = (float)(S[0] / S[1]);
    chunk_loop(g, s, part, red, [&](int64_t k) {
      const float2 pp = p[k], ap = Ap[k];
      float2 xx = x[k], rr = r[k];
      xx.x = fmaf(alpha, pp.x, xx.x);
      xx.y = fmaf(alpha, pp.y, xx.y);
      rr.x = fmaf(-alpha, ap.x, rr.x);
      rr.y = fmaf(-alpha, ap.y, rr.y);
      x[k] = xx;
      r[k] = rr;
      return (double)rr.x * rr.x + (double)rr.y * rr.y;
    });
  }
  slice_sums(sl, part, counter, state + 2, 8, state);
}

// done |= rr < tol^2; beta = rr / rz; p = r + beta p; then (last block) rz = rr,
// pAp = rr = 0, iterations += 1.
__global__ void __launch_bounds__(kCgThreads)
k_cg_dir(const SliceGeom* __restrict__ sl, int ns, const float2* __restrict__ r,
         float2* __restrict__ p, double* __restrict__ state, unsigned* __restrict__ counter) {
  const int s = blockIdx.y;
  const SliceGeom& g = sl[s];
  double* S = state + s * 8;
  const bool done = S[3] != 0.0 || S[2] < S[4];
  if (!done) {
    const float beta = (float)(S[2] / S[0]);
    for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < g.nimg;
         i += (int64_t)gridDim.x * kCgThreads) {
      const int64_t k = g.x_off + i;
      const float2 rr = r[k];
      float2 pp = p[k];
      pp.x = fmaf(beta, pp.x, rr.x);
      pp.y = fmaf(beta, pp.y, rr.y);
      p[k] = pp;
    }
  }
  __syncthreads();
  if (!arrive_last_block(counter, gridDim.x * gridDim.y)) return;
  for (int q = threadIdx.x; q < ns; q += kCgThreads) {
    double* T = state + q * 8;
    if (T[3] == 0.0) {
      T[6] = T[0] / T[1];
      if (T[2] < T[4]) {
        T[3] = 1.0;
      } else {
        T[7] = T[2] / T[0];
        T[0] = T[2];
      }
      T[5] += 1.0;
    }
    T[1] = 0.0;
    T[2] = 0.0;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// out[slice] += Re<a, b> = sum Re(conj(a) b)
__global__ void __launch_bounds__(kCgThreads)
k_cg_dot(const SliceGeom* __restrict__ sl, const float2* __restrict__ a, const float2* __restrict__ b,
         double* __restrict__ out, double* __restrict__ part, unsigned* __restrict__ counter) {
  __shared__ double red[kCgThreads / 32];
  const int s = blockIdx.y;
  const SliceGeom& g = sl[s];
  chunk_loop(g, s, part, red, [&](int64_t k) {
    const float2 aa = a[k], bb = b[k];
    return (double)aa.x * bb.x + (double)aa.y * bb.y;
  });
  slice_sums(sl, part, counter, out, 1, nullptr);
}

// One block per chunk of the longest slice (the reductions' order does not
// depend on this choice).
static dim3 cg_grid(const mrn_plan* P) {
  int64_t mx = 1;
  for (const auto& g : P->h_slices) mx = std::max<int64_t>(mx, g.nimg);
  const int64_t span = (int64_t)kCgChunk * kMaxRedBlocks;
  const int64_t len = (int64_t)kCgChunk * std::max<int64_t>((mx + span - 1) / span, 1);
  const int64_t bx = std::min<int64_t>(std::max<int64_t>((mx + len - 1) / len, 1), kMaxRedBlocks);
  return dim3((unsigned)bx, (unsigned)P->nslices);
}

int launch_cg_init(mrn_plan* P, const float2* b, const float2* Ab, float2* x, float2* r, float2* p,
                   double* state, double tol, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(state, 0, (size_t)P->nslices * 8 * sizeof(double), st);
  if (e != cudaSuccess) return cuda_fail(e);
  k_cg_init<<<cg_grid(P), kCgThreads, 0, st>>>(P->d_slices, b, Ab, x, r, p, state, tol * tol,
                                                P->d_red, P->d_sync + 1);
  e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_cg_step(mrn_plan* P, float2* x, float2* r, const float2* p, const float2* Ap, double* state,
                   cudaStream_t st) {
  k_cg_step<<<cg_grid(P), kCgThreads, 0, st>>>(P->d_slices, x, r, p, Ap, state, P->d_red, P->d_sync + 1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_cg_dir(mrn_plan* P, const float2* r, float2* p, double* state, cudaStream_t st) {
  k_cg_dir<<<cg_grid(P), kCgThreads, 0, st>>>(P->d_slices, P->nslices, r, p, state, P->d_sync);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

int launch_cg_dot(mrn_plan* P, const float2* a, const float2* b, double* out, cudaStream_t st) {
  k_cg_dot<<<cg_grid(P), kCgThreads, 0, st>>>(P->d_slices, a, b, out, P->d_red, P->d_sync + 1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}

}  // namespace mrn
