// Throughput of the two pipes the pair kernels are bound by, measured on
// the device in use: FP32 fused multiply-adds (the FMA pipe) and
// special-function operations (ex2, the MUFU / XU pipe).  The roofline of
// the evaluation kernel divides by these instead of the nominal per-SM
// rates.  Every thread runs eight independent chains of the operation, with
// the whole device full of warps, so the pipe and not the chains' latency
// is the limit; the chains' values stay bounded (a contraction toward a
// fixed point, and 2^-y for y in (0, 1]).
#include <cuda_runtime.h>

#include "internal.cuh"

namespace pdgpu {

constexpr int kPeakChains = 8;
constexpr int kPeakThreads = 256;

__global__ void __launch_bounds__(kPeakThreads) k_peak_fma(float *sink, int iters, float a, float b) {
  float x[kPeakChains];
#pragma unroll
  for (int k = 0; k < kPeakChains; k++) x[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 16; r++)
#pragma unroll
      for (int k = 0; k < kPeakChains; k++) x[k] = __fmaf_rn(x[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kPeakChains; k++) s += x[k];
  sink[(blockIdx.x * blockDim.x + threadIdx.x) & 1023] = s;  // keeps the chains alive
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__global__ void __launch_bounds__(kPeakThreads) k_peak_mufu(float *sink, int iters) {
  float y[kPeakChains];
#pragma unroll
  for (int k = 0; k < kPeakChains; k++) y[k] = 0.5f + 0.01f * (float)k;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 16; r++)
#pragma unroll
      for (int k = 0; k < kPeakChains; k++) y[k] = ex2_approx(-y[k]);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kPeakChains; k++) s += y[k];
  sink[(blockIdx.x * blockDim.x + threadIdx.x) & 1023] = s;
}

// out[0]: FP32 flop/s (an FMA is 2 flop), out[1]: ex2 operations/s, out[2]:
// the SMs the launches covered.  The best of three timed launches each,
// after one untimed.
cudaError_t measure_pipe_peaks(cudaStream_t st, double *out) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_peak_fma, kPeakThreads, 0);
  if (e != cudaSuccess) return e;
  int per_sm_mufu = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_mufu, k_peak_mufu, kPeakThreads, 0);
  if (e != cudaSuccess) return e;
  float *sink = nullptr;
  if ((e = cudaMallocAsync((void **)&sink, 1024 * sizeof(float), st)) != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int it_fma = 2048, it_mufu = 256;
  double best[2] = {0.0, 0.0};
  for (int pipe = 0; pipe < 2 && e == cudaSuccess; pipe++) {
    const int blocks = sms * (pipe == 0 ? per_sm : per_sm_mufu);
    const int iters = pipe == 0 ? it_fma : it_mufu;
    for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
      cudaEventRecord(a, st);
      if (pipe == 0)
        k_peak_fma<<<blocks, kPeakThreads, 0, st>>>(sink, iters, 0.999f, 1e-4f);
      else
        k_peak_mufu<<<blocks, kPeakThreads, 0, st>>>(sink, iters);
      cudaEventRecord(b, st);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaEventSynchronize(b);
      float ms = 0.f;
      if (e == cudaSuccess) cudaEventElapsedTime(&ms, a, b);
      if (rep == 0 || ms <= 0.f) continue;  // the first launch is a warm-up
      const double ops = (double)blocks * kPeakThreads * kPeakChains * 16.0 * iters * (pipe == 0 ? 2.0 : 1.0);
      const double rate = ops / (ms * 1e-3);
      if (rate > best[pipe]) best[pipe] = rate;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFreeAsync(sink, st);
  out[0] = best[0];
  out[1] = best[1];
  out[2] = sms;
  return e;
}

}  // namespace pdgpu
