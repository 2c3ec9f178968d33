// FP64 / FP32 non-tensor peak microbenchmark: the roofline denominator of the J/K kernels
// (which run on the FP64 pipe).  Every thread advances 8 independent FMA chains for `iters`
// iterations; grid = 8 CTAs of 256 threads per SM.  Timed with CUDA events on a private stream.
#include <cuda_runtime.h>

#include "../../include/sqb200.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chain(T* out, int iters, T a, T b) {
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == (T)-12345.0) out[blockIdx.x] = s;   // keeps the chains live
}

template <typename T>
int run(int device, int iters, double* tflops) {
  if (cudaSetDevice(device) != cudaSuccess) return SQB200_ENODEV;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int grid = sms * 8, block = 256;
  T* out = nullptr;
  cudaStream_t st;
  cudaEvent_t e0, e1;
  if (cudaMalloc(&out, grid * sizeof(T)) != cudaSuccess) return SQB200_ENOMEM;
  cudaStreamCreate(&st);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const T a = (T)0.999999, b = (T)1e-7;
  k_fma_chain<T><<<grid, block, 0, st>>>(out, iters / 4, a, b);   // warm-up
  cudaEventRecord(e0, st);
  k_fma_chain<T><<<grid, block, 0, st>>>(out, iters, a, b);
  cudaEventRecord(e1, st);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(out);
  if (err != cudaSuccess) return SQB200_ECUDA;
  const double flops = 2.0 * 8 * 16 * (double)iters * grid * block;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return SQB200_OK;
}

}  // namespace

extern "C" int sqb200_peak_fma(int device, int fp64_iters, double* fp64_tflops, double* fp32_tflops) {
  if (!fp64_tflops || !fp32_tflops || fp64_iters <= 0) return SQB200_EINVAL;
  int rc = run<double>(device, fp64_iters, fp64_tflops);
  if (rc) return rc;
  return run<float>(device, fp64_iters * 2, fp32_tflops);
}
