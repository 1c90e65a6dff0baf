// fp32_peak.cu -- measured FP32 FMA throughput of the current device, for the
// benchmark's roofline.  Built on its own into libmdbas_peak.so (bench-side
// measurement code, not part of libmdbas_nb.so).
//
// The pair kernel is bound by the FP32 pipes, whose peak is not among the
// driver-measured peaks (a copy bandwidth and a bf16 GEMM).  Two probes run
// 8 independent FMA chains per thread on every SM (16 warps per SM): one in
// scalar FFMA, one in packed f32x2 FMA (two FMAs per instruction).  Each
// reports 2 flops per FMA over the CUDA-event time of its best launch.
#include <cuda_runtime.h>

namespace {

constexpr int kProbeIters = 4096;

__global__ void __launch_bounds__(512) k_ffma_probe(float *out, float a, float b) {
  float v0 = threadIdx.x * 1e-7f, v1 = v0 + 1e-7f, v2 = v0 + 2e-7f, v3 = v0 + 3e-7f;
  float v4 = v0 + 4e-7f, v5 = v0 + 5e-7f, v6 = v0 + 6e-7f, v7 = v0 + 7e-7f;
#pragma unroll 16
  for (int i = 0; i < kProbeIters; ++i) {
    v0 = fmaf(v0, a, b);
    v1 = fmaf(v1, a, b);
    v2 = fmaf(v2, a, b);
    v3 = fmaf(v3, a, b);
    v4 = fmaf(v4, a, b);
    v5 = fmaf(v5, a, b);
    v6 = fmaf(v6, a, b);
    v7 = fmaf(v7, a, b);
  }
  const float s = ((v0 + v1) + (v2 + v3)) + ((v4 + v5) + (v6 + v7));
  if (s == 123.456f) out[blockIdx.x] = s;  // keeps the chains live
}

// The same work in packed f32x2 FMAs: 4 chains of pairs = 8 FMAs per step.
__global__ void __launch_bounds__(512) k_ffma2_probe(float *out, float a, float b) {
  const float t = threadIdx.x * 1e-7f;
  float2 v0 = make_float2(t, t + 1e-7f), v1 = make_float2(t + 2e-7f, t + 3e-7f);
  float2 v2 = make_float2(t + 4e-7f, t + 5e-7f), v3 = make_float2(t + 6e-7f, t + 7e-7f);
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll 16
  for (int i = 0; i < kProbeIters; ++i) {
    v0 = __ffma2_rn(v0, a2, b2);
    v1 = __ffma2_rn(v1, a2, b2);
    v2 = __ffma2_rn(v2, a2, b2);
    v3 = __ffma2_rn(v3, a2, b2);
  }
  const float s = ((v0.x + v0.y) + (v1.x + v1.y)) + ((v2.x + v2.y) + (v3.x + v3.y));
  if (s == 123.456f) out[blockIdx.x] = s;
}

}  // namespace

// tflops[0]: scalar FFMA, tflops[1]: packed f32x2 FMA; ms[0..1] their best
// launch times.  Returns 0, or the CUDA error code.
extern "C" int mdbas_peak_fp32(int device, double tflops[2], double ms[2]) {
  cudaError_t err = cudaSetDevice(device);
  if (err != cudaSuccess) return (int)err;
  int sms = 0;
  if ((err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
    return (int)err;
  float *out = nullptr;
  if ((err = cudaMalloc(&out, sizeof(float) * sms * 4)) != cudaSuccess) return (int)err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 2, threads = 512;
  const double flops = 2.0 * 8.0 * (double)kProbeIters * (double)blocks * (double)threads;
  for (int kind = 0; kind < 2; ++kind) {
    float best = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {
      cudaEventRecord(e0, 0);
      if (kind == 0)
        k_ffma_probe<<<blocks, threads>>>(out, 0.9999999f, 1e-7f);
      else
        k_ffma2_probe<<<blocks, threads>>>(out, 0.9999999f, 1e-7f);
      cudaEventRecord(e1, 0);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0 && t < best) best = t;  // first launch is a warm-up
    }
    tflops[kind] = flops / ((double)best * 1e-3) / 1e12;
    ms[kind] = best;
  }
  err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return (int)err;
}
