// FP64 FMA throughput probe of the benchmark, the denominator of the solver's
// FP64 roofline (the measured-peaks file holds HBM and bf16 only).  Built as its
// own library (libgem_bench_probe.so); the product library does not contain it.
#include <cuda_runtime.h>

namespace {
__global__ void fma_chain(double* out, int iters, double a, double b) {
  double x[8];
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-9 + k;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = __fma_rn(x[k], a, b);
  double s = 0;
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 12345.678) out[0] = s;   // keeps the chain alive
}
}  // namespace

extern "C" double gem_probe_fp64_tflops(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return -1.0;
  const int threads = 512, blocks = nsm * 4, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_chain<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);   // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0);
    fma_chain<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
  return flops / (best * 1e-3) / 1e12;
}
