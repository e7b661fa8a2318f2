// Micro-benchmark: throughput of shared-memory atomic adds on sm_100a (float via
// atomicAdd, float via PTX red.shared.add.f32, int32 via atomicAdd). Standalone:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o smem_atomics smem_atomics.cu
#include <cstdio>
#include <cuda_runtime.h>
__global__ void k_generic(float* out, int iters) {
  extern __shared__ float s[];
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) s[i] = 0.f;
  __syncthreads();
  float* p = s + (threadIdx.x & 31) * 33;
  for (int it = 0; it < iters; ++it) atomicAdd(p + (it & 7), 1.0f);
  __syncthreads();
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}
__global__ void k_ptx(float* out, int iters) {
  extern __shared__ float s[];
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) s[i] = 0.f;
  __syncthreads();
  unsigned base = (unsigned)__cvta_generic_to_shared(s + (threadIdx.x & 31) * 33);
  for (int it = 0; it < iters; ++it) {
    unsigned a = base + (it & 7) * 4;
    asm volatile("red.shared.add.f32 [%0], %1;" :: "r"(a), "f"(1.0f) : "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}
__global__ void k_int(float* out, int iters) {
  extern __shared__ int si[];
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) si[i] = 0;
  __syncthreads();
  int* p = si + (threadIdx.x & 31) * 33;
  for (int it = 0; it < iters; ++it) atomicAdd(p + (it & 7), 1);
  __syncthreads();
  if (threadIdx.x == 0) out[blockIdx.x] = (float)si[0];
}
int main() {
  float* d; cudaMalloc(&d, 4096 * 4);
  cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
  const int iters = 4096, blocks = 148 * 8, threads = 256;
  for (int k = 0; k < 3; ++k) {
    for (int rep = 0; rep < 2; ++rep) {
      cudaEventRecord(a);
      if (k == 0) k_generic<<<blocks, threads, 16384>>>(d, iters);
      if (k == 1) k_ptx<<<blocks, threads, 16384>>>(d, iters);
      if (k == 2) k_int<<<blocks, threads, 16384>>>(d, iters);
      cudaEventRecord(b); cudaEventSynchronize(b);
      float ms; cudaEventElapsedTime(&ms, a, b);
      double ops = (double)blocks * threads * iters;
      if (rep) printf("%s: %.3f ms, %.1f G lane-atomics/s, err=%s\n", k == 0 ? "atomicAdd(float) generic" : (k == 1 ? "red.shared.add.f32 ptx" : "atomicAdd(int) shared"), ms, ops / ms / 1e6, cudaGetErrorString(cudaGetLastError()));
    }
  }
  float h; cudaMemcpy(&h, d, 4, cudaMemcpyDeviceToHost); printf("check %f (expect %d)\n", h, 8 * iters / 8 * 1);
  return 0;
}
