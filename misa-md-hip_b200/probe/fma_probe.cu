// CUDA-core FMA throughput probe: the FP64 / FP32 denominators of the benchmark's
// roofline (the pool's measured peaks cover HBM copies and bf16 tensor work only).  A
// measurement tool of bench.py, built into its own library (libmb_probe.so) and not part
// of the plugin's interface.
//
//   int mb_probe_fma_peaks(double *fp64_tflops, double *fp32_tflops);
//     0 on success, else the cudaError_t of the first failing call.
#include <cuda_runtime.h>

#define PROBE_CUDA(call)                                                                                       \
  do {                                                                                                         \
    cudaError_t e_ = (call);                                                                                   \
    if (e_ != cudaSuccess) return (int)e_;                                                                     \
  } while (0)

namespace {

template <class T>
__global__ void __launch_bounds__(256) k_fma_chain(T *out, int iters, T a, T b) {
  T x0 = threadIdx.x * (T)1e-3, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3, x4 = x0 + (T)4, x5 = x0 + (T)5,
    x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int k = 0; k < iters; k++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
      x0 = x0 * a + b;
      x1 = x1 * a + b;
      x2 = x2 * a + b;
      x3 = x3 * a + b;
      x4 = x4 * a + b;
      x5 = x5 * a + b;
      x6 = x6 * a + b;
      x7 = x7 * a + b;
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == (T)-12345.678) out[0] = s; // never true; keeps the chains alive
}

template <class T>
int time_fma(double *tflops) {
  int dev = 0, sms = 148;
  PROBE_CUDA(cudaGetDevice(&dev));
  PROBE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  T *out = nullptr;
  PROBE_CUDA(cudaMalloc(&out, sizeof(T)));
  cudaEvent_t e0, e1;
  PROBE_CUDA(cudaEventCreate(&e0));
  PROBE_CUDA(cudaEventCreate(&e1));
  const int blocks = sms * 8, threads = 256, iters = 4096;
  k_fma_chain<T><<<blocks, threads>>>(out, 64, (T)0.999, (T)1e-4); // warm-up
  PROBE_CUDA(cudaEventRecord(e0));
  k_fma_chain<T><<<blocks, threads>>>(out, iters, (T)0.999, (T)1e-4);
  PROBE_CUDA(cudaEventRecord(e1));
  PROBE_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  PROBE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return 0;
}

} // namespace

extern "C" int mb_probe_fma_peaks(double *fp64_tflops, double *fp32_tflops) {
  if (!fp64_tflops || !fp32_tflops) return (int)cudaErrorInvalidValue;
  int rc = time_fma<double>(fp64_tflops);
  if (rc == 0) rc = time_fma<float>(fp32_tflops);
  return rc;
}
