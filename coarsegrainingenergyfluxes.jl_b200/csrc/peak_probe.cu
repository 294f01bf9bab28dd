// Throughput probe for the roofline denominator of the FP64 direct sum: a long chain of
// independent double-precision FMAs over every SM, timed with CUDA events.  Built as a separate
// library (libcgef_peak.so) used only by the benchmark.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

__global__ void dfma_loop(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" double cgef_peak_fp64_tflops(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return -1.0;
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 4096;
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  dfma_loop<<<blocks, threads>>>(out, 64, 0.999, 0.001);
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0);
    dfma_loop<<<blocks, threads>>>(out, iters, 0.999, 0.001);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  const double flops = 2.0 * 32.0 * iters * static_cast<double>(blocks) * threads;
  return flops / (best * 1e-3) / 1e12;
}
