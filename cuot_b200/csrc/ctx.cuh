// ctx.cuh -- the context object behind the opaque cuot_ctx handle.
#pragma once
#include "common.cuh"

struct cuot_ctx {
  int device;
  uint32_t *t0_d;          // T0 table (256 words) for staging into shared memory
  void *scratch;           // grow-only scratch arena
  uint64_t scratch_bytes;
  void *qc_tables[32];     // NTT twiddle tables per log2(n) (qc.cu)
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
}  // namespace cuot
