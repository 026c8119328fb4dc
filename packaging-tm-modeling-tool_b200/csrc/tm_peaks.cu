// CUDA-core FMA throughput of the current device, FP32 and FP64 (no counterpart in the reference):
// the denominators of the compute roofline of the matrix-free level-0 kernels, which are bound by
// CUDA-core arithmetic rather than by HBM. Every thread runs independent chains of fused
// multiply-adds on register values; the grid fills every SM several times over.
#include <cuda_runtime.h>

#include "tm_internal.h"

namespace tmg {
namespace {

constexpr int PK_CHAINS = 8;
constexpr int PK_ITERS = 4096;

template <class T>
__global__ void __launch_bounds__(256) k_fma_peak(T seed, T* out) {
  T a[PK_CHAINS];
#pragma unroll
  for (int q = 0; q < PK_CHAINS; q++) a[q] = seed + (T)(threadIdx.x + q);
  const T m = (T)0.999999, c = (T)1e-7;
  for (int it = 0; it < PK_ITERS; it++) {
#pragma unroll
    for (int u = 0; u < 8; u++)
#pragma unroll
      for (int q = 0; q < PK_CHAINS; q++) a[q] = fma(a[q], m, c);
  }
  T s = 0;
#pragma unroll
  for (int q = 0; q < PK_CHAINS; q++) s += a[q];
  if (s == (T)-1) out[0] = s;   // never true: keeps the chains live
}

template <class T>
double fma_peak(int dev) {
  int sms = 0;
  TM_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DBuf<T> out;
  out.alloc(1);
  cudaStream_t st;
  TM_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaEvent_t a, b;
  TM_CUDA_CHECK(cudaEventCreate(&a));
  TM_CUDA_CHECK(cudaEventCreate(&b));
  const int blocks = sms * 8, threads = 256;
  k_fma_peak<T><<<blocks, threads, 0, st>>>((T)1, out.p);   // warm-up
  TM_CUDA_CHECK(cudaEventRecord(a, st));
  const int reps = 5;
  for (int r = 0; r < reps; r++) k_fma_peak<T><<<blocks, threads, 0, st>>>((T)1, out.p);
  TM_CUDA_CHECK(cudaEventRecord(b, st));
  TM_CUDA_CHECK(cudaEventSynchronize(b));
  TM_CUDA_CHECK(cudaGetLastError());
  float ms = 0;
  TM_CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamDestroy(st);
  const double flops = 2.0 * PK_CHAINS * 8 * (double)PK_ITERS * blocks * threads * reps;
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace
}  // namespace tmg

extern "C" tm_status tm_device_peaks(double* fp32_tflops, double* fp64_tflops) {
  using namespace tmg;
  try {
    require_device();
    int dev = 0;
    TM_CUDA_CHECK(cudaGetDevice(&dev));
    if (fp32_tflops) *fp32_tflops = fma_peak<float>(dev);
    if (fp64_tflops) *fp64_tflops = fma_peak<double>(dev);
    return TM_OK;
  } catch (const Error& e) {
    set_last_error(e.msg);
    return e.status;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return TM_CUDA;
  }
}
