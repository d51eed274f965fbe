// sph_peak.cu — FFMA / DFMA chain probe of the non-tensor FP pipes
// (include/sph_peak.h).  Eight independent accumulators per thread keep the
// pipe busy; the result is stored only if it is impossible, which keeps the
// arithmetic alive without memory traffic.
#include <cuda_runtime.h>

#include "sph_peak.h"

namespace {

constexpr int CHAINS = 8;
constexpr int ITERS = 4096;

template <class T>
__global__ void __launch_bounds__(256) k_fma(T* out, T b, T c) {
  T a[CHAINS];
#pragma unroll
  for (int k = 0; k < CHAINS; ++k) a[k] = T(threadIdx.x + k) * T(1e-7);
  for (int i = 0; i < ITERS; ++i) {
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) a[k] = fma(a[k], b, c);
  }
  T s = T(0);
#pragma unroll
  for (int k = 0; k < CHAINS; ++k) s += a[k];
  if (s == T(-12345.678)) out[blockIdx.x] = s;
}

template <class T>
double run(int reps) {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1.0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = nsm * 8, threads = 256;
  T* out = nullptr;
  if (cudaMalloc(&out, sizeof(T) * blocks) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const T b = T(0.999999), c = T(1e-6);
  k_fma<T><<<blocks, threads>>>(out, b, c);  // warm-up
  cudaEventRecord(e0);
  for (int r = 0; r < reps; ++r) k_fma<T><<<blocks, threads>>>(out, b, c);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess || ms <= 0.f) return -1.0;
  double flops = 2.0 * double(CHAINS) * ITERS * double(blocks) * threads * reps;
  return flops / (double(ms) * 1e-3);
}

}  // namespace

extern "C" double sph_peak_flops(int precision, int reps) {
  if (reps < 1) reps = 1;
  return precision == 1 ? run<double>(reps) : run<float>(reps);
}
