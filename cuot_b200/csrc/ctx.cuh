// ctx.cuh -- the context object behind the opaque cuot_ctx handle.
#pragma once
#include "common.cuh"

struct cuot_ctx {
  int device;
  uint32_t *t0_d;          // T0 table (256 words) for staging into shared memory
  void *scratch;           // grow-only scratch arena
  uint64_t scratch_bytes;
  void *qc_tables[32];     // NTT twiddle tables per log2(n) (qc.cu)
  int pprf_threads;        // threads per tree CTA (128 or 256)
  int qc_planes_per_pass;  // 0: automatic
};

namespace cuot {
// Records a failure message for cuot_last_error() and returns `status`.
int fail(int status, const char *fmt, ...);
// Makes ctx's device current for the lifetime of the guard.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(const cuot_ctx *c) {
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};
// Returns a scratch pointer of at least `bytes` (grows the arena with
// cudaMalloc when needed; growing synchronises the device).
int scratch(cuot_ctx *ctx, uint64_t bytes, void **out);
// One-time per-device initialisation of module constants (pprf.cu).
int pprf_init_device();
// Frees the context's cached QC tables (qc.cu).
void qc_free_ctx_tables(cuot_ctx *ctx);
// QC helpers used by the batched engine (qc.cu).
int qc_prepare(cuot_ctx *ctx, int e);
int qc_build_ahat(cuot_ctx *ctx, int e, const uint64_t *a_d, uint32_t *Y, uint2 *ahat, cudaStream_t st);
int qc_encode_jobs(cuot_ctx *ctx, int e, uint64_t *planes, int njobs, const uint2 *const *ahats,
                   uint32_t *Y, int batch, cudaStream_t st);
int qc_default_batch(uint64_t n, int nplanes);
int transpose_launch(const void *in, uint64_t rows, uint64_t row_bytes, uint64_t col_lo,
                     uint64_t col_hi, void *out, cudaStream_t st);
}  // namespace cuot
