// probe.cu -- the device's fp64 fused-multiply-add rate, measured: the
// denominator of the FFT encode's fp64 fraction (the FFT passes run on the
// same fp64 pipe, as adds, multiplies and FMAs).
//
// Each thread runs kProbeChains independent chains x <- x * m + c (m, c
// kernel arguments near 1 and 0, so nothing folds and x stays near the fixed
// point c / (1 - m) = 1: no overflow, no subnormals) at full occupancy; the
// chains' sum is stored only if it equals a value it cannot reach, which
// keeps every thread's chains live without a store per thread.
#include "ctx.cuh"

namespace cuot {
namespace {

constexpr int kProbeChains = 8;
constexpr int kProbeThreads = 256;
constexpr int kProbeCtasPerSm = 8;  // 2048 threads per SM
constexpr int kProbeIters = 1 << 16;

__global__ void __launch_bounds__(kProbeThreads) fp64_fma_probe(int iters, double m, double c, double *out) {
  double x[kProbeChains];
#pragma unroll
  for (int k = 0; k < kProbeChains; k++) x[k] = 1.0 + 1e-3 * double(threadIdx.x + k);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < kProbeChains; k++) x[k] = fma(x[k], m, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kProbeChains; k++) s += x[k];
  if (s == -1.0) out[0] = s;
}

}  // namespace
}  // namespace cuot

using namespace cuot;

extern "C" int cuot_measure_fp64_tflops(cuot_ctx *ctx, int reps, double *tflops) {
  if (!ctx || !tflops || reps < 1 || reps > 1000) return fail(CUOT_EINVAL, "bad argument");
  DeviceGuard g(ctx);
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess || sms < 1) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "multiprocessor count query failed");
  }
  double *out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int s = CUOT_OK;
  if (cudaMalloc(&out, 16) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    s = fail(CUOT_ECUDA, "fp64 probe set-up failed");
  }
  const unsigned grid = unsigned(sms) * kProbeCtasPerSm;
  float best = 0.0f;
  for (int r = 0; s == CUOT_OK && r <= reps; r++) {  // launch 0 warms up
    cudaEventRecord(e0, st);
    fp64_fma_probe<<<grid, kProbeThreads, 0, st>>>(kProbeIters, 0.9999999, 1e-7, out);
    cudaEventRecord(e1, st);
    if ((s = launch_status(1)) != CUOT_OK) break;
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      cudaGetLastError();
      s = fail(CUOT_ECUDA, "fp64 probe failed");
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && (best == 0.0f || ms < best)) best = ms;
  }
  if (s == CUOT_OK) {
    const double flops = 2.0 * kProbeChains * double(kProbeIters) * double(grid) * kProbeThreads;
    *tflops = best > 0.0f ? flops / (double(best) * 1e-3) / 1e12 : 0.0;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (out) cudaFree(out);
  return s;
}
