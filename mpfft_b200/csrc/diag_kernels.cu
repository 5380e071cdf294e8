// Diagnostics used by the benchmark to state the roofline it measures against:
// the integer multiply-add rate of this GPU, measured live.
//
// The multiprecision kernels are bound by 32x32->64-bit limb products, each
// one low-half and one high-half multiply-add (or one wide multiply-add).
// These kernels run long independent chains of each form so the rate seen is
// the issue limit of the integer pipe, not latency.
#include <cstdint>

#include <cuda_runtime.h>

namespace mpfft {

__global__ void diag_imad_lo(uint32_t *out, int reps) {
  uint32_t a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = threadIdx.x + i;
  const uint32_t m = 0x9e3779b1u + blockIdx.x;
#pragma unroll 1
  for (int r = 0; r < reps; ++r) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = a[i] * m + a[(i + 1) & 7];
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) x ^= a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

__global__ void diag_imad_wide(uint64_t *out, int reps) {
  uint64_t a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = threadIdx.x + i;
  const uint32_t m = 0x9e3779b1u + blockIdx.x;
#pragma unroll 1
  for (int r = 0; r < reps; ++r) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = (uint64_t)(uint32_t)a[i] * m + a[(i + 1) & 7];
    }
  }
  uint64_t x = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) x ^= a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

// ops/s of 32-bit multiply-add (wide = 0) or 32x32+64 -> 64 multiply-add (wide = 1)
cudaError_t diag_imad_rate(int wide, double *ops_per_s) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256, reps = 4000;
  void *buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, (size_t)blocks * threads * 8);
  if (e != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float ms = 0;
  for (int pass = 0; pass < 2; ++pass) {  // pass 0 warms up
    const int r = pass ? reps : 10;
    cudaEventRecord(e0);
    if (wide) diag_imad_wide<<<blocks, threads>>>((uint64_t *)buf, r);
    else diag_imad_lo<<<blocks, threads>>>((uint32_t *)buf, r);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
  }
  e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  *ops_per_s = (double)blocks * threads * reps * 16 * 8 / (ms * 1e-3);
  return e;
}

}  // namespace mpfft
