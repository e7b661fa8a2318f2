// Allocation-free type-2 interpolation (mrn_interp_noalloc).
//
// Who needs it: code that must not allocate device memory at call time --
// e.g. work issued while a CUDA graph is being captured (cudaMalloc is not
// allowed inside a capture), real-time reconstruction loops whose memory is
// reserved up front by the host application, or frameworks whose caching
// allocator owns the whole device and forbids driver allocations. The regular
// path needs a plan (mrn_plan_create allocates the binned trajectory, the
// oversampled grid and the cuFFT plans); this entry point needs none.
//
// How: the same taps and Kaiser-Bessel weights as mrn_interp on a raw plan
// (tap j = lo + q, lo = ceil(u - W/2), valid iff |(float)j - u| <= W/2,
// separable weights, circular wrap), computed in two steps that talk through
// one fixed scratch array in device memory:
//   1. one thread per sample writes its tap origins and d x K weights;
//   2. one thread per (sample, coil) gathers the grid with them.
// The scratch is a file-scope __device__ array of kNoAllocScratchBytes, so
// every GPU that loads the library holds it for the life of the process.
// All calls share it: calls that overlap on the GPU (different streams, or
// different host threads) race on it and must be serialised by the caller.
// Every scratch entry a call reads is written earlier in the same call, so
// nothing has to be cleared between calls.
#include <mutex>

#include "common.cuh"
#include "internal.cuh"

namespace mrn {

constexpr size_t kNoAllocScratchBytes = 32ull << 20;  // 32 MiB per device

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_na_mutex;
void* g_na_ptr[64] = {nullptr};  // device address of the scratch, per device

// Per-device set-up: the host-side name of the array is only a stand-in, so
// the device address is looked up once per device, with that device current.
int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e);
  if (dev < 0 || dev >= 64) return MRN_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e);
    g_na_ptr[dev] = p;
  }
  *out = g_na_ptr[dev];
  return MRN_OK;
}

struct NaGeom {
  int ndim;
  int nos[kMaxDim];
  int K;  // candidate taps per dim (max over dims)
  int ntaps[kMaxDim];
  float radius[kMaxDim];
  float beta;
};

// Step 1: tap origins (int32 [p][d]) and weights (float [p][d][K], 0 for
// invalid taps) of every sample.
__global__ void k_na_weights(NaGeom g, const float* __restrict__ locs, int64_t npts,
                             int* __restrict__ lo_out, float* __restrict__ w_out) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  for (int i = 0; i < g.ndim; ++i) {
    const float u = remainder_f32(locs[p * g.ndim + i], (float)g.nos[i]);
    const float r = g.radius[i];
    const int lo = (int)ceilf(__fsub_rn(u, r));
    lo_out[p * g.ndim + i] = lo;
    float* w = w_out + (p * g.ndim + i) * g.K;
    for (int q = 0; q < g.K; ++q) {
      float v = 0.f;
      if (q < g.ntaps[i]) {
        const float adx = fabsf(__fsub_rn((float)(lo + q), u));
        if (adx <= r) v = kb_tap(adx, r, g.beta);
      }
      w[q] = v;
    }
  }
}

// Step 2: out[c][p] = sum over taps of prod_d w * grid[c][cell], one thread
// per (sample, coil), samples fastest.
__global__ void k_na_gather(NaGeom g, int ncoil, int64_t npts, const int* __restrict__ lo_in,
                            const float* __restrict__ w_in, const float2* __restrict__ grid,
                            float2* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * ncoil) return;
  const int64_t p = t % npts;
  const int c = (int)(t / npts);
  int64_t gsize = 1;
  for (int i = 0; i < g.ndim; ++i) gsize *= g.nos[i];
  const float2* gc = grid + (int64_t)c * gsize;
  int lo[kMaxDim] = {0, 0, 0};
  int n[kMaxDim] = {1, 1, 1};
  for (int i = 0; i < g.ndim; ++i) {
    lo[i] = lo_in[p * g.ndim + i];
    n[i] = g.ntaps[i];
  }
  const float* w0 = w_in + (p * g.ndim + 0) * g.K;
  const float* w1 = w_in + (p * g.ndim + (g.ndim > 1 ? 1 : 0)) * g.K;
  const float* w2 = w_in + (p * g.ndim + (g.ndim > 2 ? 2 : 0)) * g.K;
  float ax = 0.f, ay = 0.f;
  for (int a = 0; a < n[0]; ++a) {
    const float wa = w0[a];
    if (wa == 0.f) continue;
    const int s0 = pos_mod(lo[0] + a, g.nos[0]);
    for (int b = 0; b < n[1]; ++b) {
      const float wab = g.ndim > 1 ? wa * w1[b] : wa;
      if (wab == 0.f) continue;
      const int s1 = g.ndim > 1 ? pos_mod(lo[1] + b, g.nos[1]) : 0;
      for (int z = 0; z < n[2]; ++z) {
        const float w = g.ndim > 2 ? wab * w2[z] : wab;
        if (w == 0.f) continue;
        const int s2 = g.ndim > 2 ? pos_mod(lo[2] + z, g.nos[2]) : 0;
        int64_t lin = s0;
        if (g.ndim > 1) lin = lin * g.nos[1] + s1;
        if (g.ndim > 2) lin = lin * g.nos[2] + s2;
        const float2 v = __ldg(gc + lin);
        ax = fmaf(w, v.x, ax);
        ay = fmaf(w, v.y, ay);
      }
    }
  }
  out[(int64_t)c * npts + p] = make_float2(ax, ay);
}

}  // namespace
}  // namespace mrn

using namespace mrn;

extern "C" int mrn_interp_noalloc(int ndim, const int* grid_size, int n_coil, int64_t n_pts,
                                  const double* width, double beta, const void* grid,
                                  const float* locs, void* out, void* stream) {
  if (ndim < 1 || ndim > kMaxDim || !grid_size || !width || n_coil < 1 || n_pts < 0)
    return MRN_ERR_ARG;
  if (!(beta > 0.0)) return MRN_ERR_ARG;
  NaGeom g{};
  g.ndim = ndim;
  g.beta = (float)beta;
  g.K = 1;
  for (int i = 0; i < kMaxDim; ++i) {
    g.nos[i] = 1;
    g.ntaps[i] = 1;
    g.radius[i] = 0.5f;
  }
  for (int i = 0; i < ndim; ++i) {
    if (grid_size[i] < 1) return MRN_ERR_ARG;
    if (!(width[i] >= 1.0) || !(width[i] < (double)kMaxTaps)) return MRN_ERR_WIDTH;
    g.nos[i] = grid_size[i];
    g.radius[i] = (float)width[i] / 2.0f;
    g.ntaps[i] = (int)floor(width[i]) + 1;
    g.K = g.ntaps[i] > g.K ? g.ntaps[i] : g.K;
  }
  // scratch layout: [lo: n_pts*d int32][weights: n_pts*d*K float32], 256-B aligned.
  // The sample count is bounded first, so the byte counts below cannot wrap.
  if ((uint64_t)n_pts > (uint64_t)(kNoAllocScratchBytes / ((size_t)ndim * (1 + g.K) * sizeof(float))))
    return MRN_ERR_SCRATCH;
  const size_t lo_bytes = (((size_t)n_pts * ndim * sizeof(int)) + 255) & ~(size_t)255;
  const size_t need = lo_bytes + (size_t)n_pts * ndim * g.K * sizeof(float);
  if (need > kNoAllocScratchBytes) return MRN_ERR_SCRATCH;
  if (n_pts == 0) return MRN_OK;
  if (!grid || !locs || !out) return MRN_ERR_ARG;
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc != MRN_OK) return rc;
  int* lo = reinterpret_cast<int*>(base);
  float* w = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(base) + lo_bytes);
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned b1 = (unsigned)((n_pts + 255) / 256);
  k_na_weights<<<b1, 256, 0, st>>>(g, locs, n_pts, lo, w);
  const int64_t work = n_pts * n_coil;  // n_pts < 2^23 here, so no overflow
  if ((work + 255) / 256 > (int64_t)INT32_MAX) return MRN_ERR_ARG;
  const unsigned b2 = (unsigned)((work + 255) / 256);
  k_na_gather<<<b2, 256, 0, st>>>(g, n_coil, n_pts, lo, w, (const float2*)grid, (float2*)out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MRN_OK : cuda_fail(e);
}
