// FP64 FMA throughput of the device, measured by the library's own kernel: the ceiling for
// the B-spline advection kernels' arithmetic (their FP64 fraction is reported against it).
// Every thread runs eight independent dependency chains acc = fma(acc, m, c); a grid of
// eight 256-thread blocks per SM keeps every FP64 pipe busy.  No host-side state.
#include <cuda_runtime.h>

#include <algorithm>

#define CFD2LCS_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_fma_probe(double *out, int iters) {
  double acc[kChains];
#pragma unroll
  for (int u = 0; u < kChains; u++) acc[u] = 1e-3 * (threadIdx.x + u);
  const double m = 0.9999999, c = 1e-9;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < kChains; u++) acc[u] = fma(acc[u], m, c);
  }
  double s = 0;
#pragma unroll
  for (int u = 0; u < kChains; u++) s += acc[u];
  if (s == -1.0) out[0] = s;  // never true; keeps the chains live
}

}  // namespace

// Measures the device's FP64 FMA rate: best of `reps` launches of `iters` iterations.
// tflops receives 2 flops per FMA / kernel time, in TFLOP/s.  Returns 0, or a CUDA error code.
CFD2LCS_EXPORT int cfd2lcs_b200_fp64_fma_rate(int iters, int reps, double *tflops) {
  if (!tflops || iters <= 0 || reps <= 0) return (int)cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return (int)e;
  cudaStream_t st = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  double *out = nullptr;
  const int blocks = 8 * sms, threads = 256;
  float best = 0.f;
  if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) == cudaSuccess && (e = cudaEventCreate(&a)) == cudaSuccess &&
      (e = cudaEventCreate(&b)) == cudaSuccess && (e = cudaMalloc(&out, sizeof(double))) == cudaSuccess) {
    k_fma_probe<<<blocks, threads, 0, st>>>(out, iters);  // warm-up
    for (int r = 0; r < reps && e == cudaSuccess; r++) {
      cudaEventRecord(a, st);
      k_fma_probe<<<blocks, threads, 0, st>>>(out, iters);
      cudaEventRecord(b, st);
      if ((e = cudaEventSynchronize(b)) == cudaSuccess) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        best = r == 0 ? ms : std::min(best, ms);
      }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  if (out) cudaFree(out);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) return (int)e;
  const double flops = 2.0 * kChains * (double)iters * blocks * threads;
  *tflops = best > 0.f ? flops / (best * 1e-3) / 1e12 : 0.0;
  return 0;
}
