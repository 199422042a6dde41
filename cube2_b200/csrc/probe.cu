// FP32 FMA throughput probe: the measured denominator for the PP kernel's
// roofline (the PP pair force runs on the FP32 CUDA cores, not the tensor cores).
#include "common.cuh"

namespace cube {

constexpr int kProbeIters = 8192;
constexpr int kProbeChains = 8;

__global__ void __launch_bounds__(256) k_fma_probe(float seed, float *sink) {
  float a[kProbeChains];
#pragma unroll
  for (int c = 0; c < kProbeChains; c++) a[c] = seed + threadIdx.x * 1e-7f + c;
  const float m = 0.9999999f, k = 1e-7f;
  for (int i = 0; i < kProbeIters; i++) {
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) a[c] = fmaf(a[c], m, k);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kProbeChains; c++) s += a[c];
  if (s == 12345.678f) *sink = s;  // keeps the chains live
}

cudaError_t fma_probe(cudaStream_t s, int num_sms, float *ms, double *flops) {
  float *sink = nullptr;
  cudaError_t e = cudaMallocAsync(&sink, sizeof(float), s);
  if (e != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int blocks = num_sms * 16;
  k_fma_probe<<<blocks, 256, 0, s>>>(1.0f, sink);  // warm-up
  cudaEventRecord(a, s);
  for (int r = 0; r < 5; r++) k_fma_probe<<<blocks, 256, 0, s>>>(1.0f + r, sink);
  cudaEventRecord(b, s);
  e = cudaEventSynchronize(b);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, a, b);
  *flops = 5.0 * blocks * 256.0 * kProbeIters * kProbeChains * 2.0;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFreeAsync(sink, s);
  cudaStreamSynchronize(s);
  return e == cudaSuccess ? cudaGetLastError() : e;
}

}  // namespace cube
