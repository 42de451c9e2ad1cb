// fp64_peak.cu — measures the FP64 FMA throughput of the device (the roofline
// denominator for the SNAP kernels, which run on the FP64 CUDA-core pipe).
//
// Each thread runs 8 independent FMA chains for `iters` iterations; the result is
// stored so that nothing is optimised away.  flops = 2 * 8 * iters * threads.
#include <cuda_runtime.h>

#include <cstdint>

namespace {
__global__ void __launch_bounds__(256) k_dfma(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
  double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
  for (int k = 0; k < iters; k++) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      x0 = fma(x0, a, b);
      x1 = fma(x1, a, b);
      x2 = fma(x2, a, b);
      x3 = fma(x3, a, b);
      x4 = fma(x4, a, b);
      x5 = fma(x5, a, b);
      x6 = fma(x6, a, b);
      x7 = fma(x7, a, b);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}
}  // namespace

extern "C" __attribute__((visibility("default"))) int ipg_probe_fp64_peak(int device, int repeats, double* tflops,
                                                                          double* best_ms) {
  if (cudaSetDevice(device) != cudaSuccess) return -2;
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 4096;
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * threads * blocks) != cudaSuccess) return -3;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_dfma<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < repeats; r++) {
    cudaEventRecord(e0);
    k_dfma<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  int st = cudaGetLastError() == cudaSuccess ? 0 : -2;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  double flops = 2.0 * 8.0 * 4.0 * (double)iters * threads * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  if (best_ms) *best_ms = best;
  return st;
}
