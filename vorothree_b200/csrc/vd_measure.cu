// vd_measure.cu -- FMA-chain microbenchmark for the FP64 / FP32 pipe peaks
// (the denominators of the clip kernel's roofline; no vendor number is used).
#include <cuda_runtime.h>

#include "../../include/voronoid_b200.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chain(T* out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (T)-1.2345) out[blockIdx.x] = s;  // keeps the chains live
}

template <typename T>
int run(double* tflops) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return VD_ECUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  T* out = nullptr;
  if (cudaMalloc(&out, 4096 * sizeof(T)) != cudaSuccess) return VD_ENOMEM;
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma_chain<T><<<blocks, threads>>>(out, 256, (T)0.999, (T)0.001);  // warm-up
  cudaEventRecord(e0);
  k_fma_chain<T><<<blocks, threads>>>(out, iters, (T)0.999, (T)0.001);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return VD_ECUDA;
  const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return VD_OK;
}

}  // namespace

extern "C" int vd_measure_fma_peak(int fp64, double* tflops) {
  if (!tflops) return VD_EINVAL;
  return fp64 ? run<double>(tflops) : run<float>(tflops);
}
