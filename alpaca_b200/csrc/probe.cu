// Measurement helpers for bench.py (not part of the C ABI of the engine):
// the FP64 FMA-pipe peak of the device, measured with independent DFMA chains.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) dfma_chains(double a, double b, int iters, double *out) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-9 + c;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

}  // namespace

extern "C" int alp_probe_fp64_peak(int iters, int ctas_per_sm, double *tflops) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double *out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return 2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int const grid = sms * ctas_per_sm, threads = 256;
  dfma_chains<<<grid, threads>>>(0.999999, 1e-7, iters / 10, out);  // warm-up
  cudaEventRecord(e0);
  dfma_chains<<<grid, threads>>>(0.999999, 1e-7, iters, out);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  double const flops = 2.0 * kChains * (double)iters * grid * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
