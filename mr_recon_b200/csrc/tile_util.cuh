// Small device helpers shared by the tile kernels (sm_100a): tile frames,
// single-step circular wraps, and cp.async copies into shared memory.
#pragma once

#include "common.cuh"

namespace mrn {

struct Frame {
  int org[kMaxDim];
  int size[kMaxDim];
};

__device__ __forceinline__ Frame frame_of(const SliceGeom& g, int tile, int D, bool gridding) {
  Frame f;
  int rem = tile;
  int tc[kMaxDim] = {0, 0, 0};
  const int* nts = gridding ? g.gntile : g.ntile;
  for (int i = D - 1; i >= 0; --i) {
    tc[i] = rem % nts[i];
    rem /= nts[i];
  }
#pragma unroll
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

__device__ __forceinline__ int wrap_once(int a, int n) {
  // a in (-n, 2n): a mod n
  a = a < 0 ? a + n : a;
  return a >= n ? a - n : a;
}

template <class T>
__device__ __forceinline__ T sel3(const T* v, int i) { return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace mrn
