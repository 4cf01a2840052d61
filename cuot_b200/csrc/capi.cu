// capi.cu -- context lifetime, status strings, error reporting, scratch.
#include <cstdarg>
#include <cstdio>
#include <atomic>
#include <mutex>
#include <string>
#include "ctx.cuh"

namespace cuot {
static thread_local std::string g_err;

int fail(int status, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return status;
}

static std::atomic<unsigned long long> g_launches{0};

int launch_status(int nlaunch) {
  g_launches.fetch_add((unsigned long long)nlaunch, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CUOT_ECUDA, "CUDA launch failed: %s", cudaGetErrorString(e));
  return CUOT_OK;
}

int scratch(cuot_ctx *ctx, uint64_t bytes, void **out) {
  if (bytes > ctx->scratch_bytes) {
    // Growing frees the old arena; cudaFree waits for work that may use it.
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(CUOT_ENOMEM, "scratch allocation of %llu bytes failed: %s",
                  (unsigned long long)bytes, cudaGetErrorString(e));
    }
    ctx->scratch = p;
    ctx->scratch_bytes = bytes;
  }
  *out = ctx->scratch;
  return CUOT_OK;
}
}  // namespace cuot

using namespace cuot;

extern "C" {

const char *cuot_version(void) { return "cuot-b200 0.1 (sm_100a)"; }

const char *cuot_status_string(int s) {
  switch (s) {
    case CUOT_OK: return "ok";
    case CUOT_EINVAL: return "invalid argument";
    case CUOT_ENOMEM: return "out of device memory";
    case CUOT_ECUDA: return "CUDA error";
    case CUOT_ETIMEOUT: return "timed out";
    case CUOT_ENOTSUP: return "not supported";
    default: return "unknown status";
  }
}

const char *cuot_last_error(void) { return g_err.c_str(); }

unsigned long long cuot_launch_count(void) { return g_launches.load(); }

int cuot_ctx_create(int device, cuot_ctx **out) {
  if (!out) return fail(CUOT_EINVAL, "out is null");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return fail(CUOT_EINVAL, "device %d not available (%d devices)", device, n);
  }
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "cudaSetDevice(%d) failed", device);
  }
  cuot_ctx *c = new cuot_ctx{};
  c->device = device;
  int st = CUOT_OK;
  if (cudaMalloc(&c->t0_d, 256 * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    st = fail(CUOT_ENOMEM, "table allocation failed");
  } else if (cudaMemcpy(c->t0_d, host_t0_table(), 256 * sizeof(uint32_t),
                        cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    st = fail(CUOT_ECUDA, "table upload failed");
  } else {
    st = pprf_init_device();
  }
  cudaSetDevice(prev);
  if (st != CUOT_OK) {
    if (c->t0_d) cudaFree(c->t0_d);
    delete c;
    return st;
  }
  *out = c;
  return CUOT_OK;
}

int cuot_ctx_destroy(cuot_ctx *c) {
  if (!c) return CUOT_OK;
  {
    DeviceGuard g(c);
    qc_free_ctx_tables(c);
    if (c->scratch) cudaFree(c->scratch);
    if (c->t0_d) cudaFree(c->t0_d);
  }
  delete c;
  return CUOT_OK;
}

int cuot_ctx_reserve(cuot_ctx *c, uint64_t bytes) {
  if (!c) return fail(CUOT_EINVAL, "ctx is null");
  DeviceGuard g(c);
  void *p;
  return scratch(c, bytes, &p);
}

uint64_t cuot_ctx_scratch_bytes(const cuot_ctx *c) { return c ? c->scratch_bytes : 0; }

}  // extern "C"
