// capi.cu -- context lifetime, status strings, error reporting, scratch.
#include <cstring>
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
  c->pprf_threads = 256;
  c->qc_planes_per_pass = 0;
  c->qc_streams = 2;
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
    if (c->qcf_margin) cudaFree(c->qcf_margin);
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

int cuot_qc_fft_margin(cuot_ctx *c, double *out, int reset) {
  if (!c || !out) return fail(CUOT_EINVAL, "null argument");
  if (!c->qcf_margin) return fail(CUOT_EINVAL, "margin recording is off (CUOT_TUNE_QC_RECORD_MARGIN)");
  DeviceGuard g(c);
  uint32_t bits = 0;
  if (cudaMemcpy(&bits, c->qcf_margin, sizeof(bits), cudaMemcpyDeviceToHost) != cudaSuccess ||
      (reset && cudaMemset(c->qcf_margin, 0, sizeof(bits)) != cudaSuccess)) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "margin read failed");
  }
  float f;
  std::memcpy(&f, &bits, sizeof(f));
  *out = double(f);
  return CUOT_OK;
}

int cuot_ctx_set_tuning(cuot_ctx *c, int key, int64_t value) {
  if (!c) return fail(CUOT_EINVAL, "ctx is null");
  switch (key) {
    case CUOT_TUNE_PPRF_THREADS:
      if (value != 128 && value != 256) return fail(CUOT_EINVAL, "threads per tree must be 128 or 256");
      c->pprf_threads = int(value);
      return CUOT_OK;
    case CUOT_TUNE_QC_PLANES:
      if (value < 0 || value > 4096) return fail(CUOT_EINVAL, "planes per pass out of range");
      c->qc_planes_per_pass = int(value);
      return CUOT_OK;
    case CUOT_TUNE_QC_BACKEND:
      if (value < 0 || value > 2) return fail(CUOT_EINVAL, "QC backend must be 0 (automatic), 1 (NTT) or 2 (FFT)");
      c->qc_backend = int(value);
      return CUOT_OK;
    case CUOT_TUNE_QC_STREAMS:
      if (value != 1 && value != 2) return fail(CUOT_EINVAL, "QC streams must be 1 or 2");
      c->qc_streams = int(value);
      return CUOT_OK;
    case CUOT_TUNE_QC_RECORD_MARGIN: {
      if (value != 0 && value != 1) return fail(CUOT_EINVAL, "QC margin recording must be 0 or 1");
      DeviceGuard g(c);
      if (value == 0) {
        if (c->qcf_margin) cudaFree(c->qcf_margin);
        c->qcf_margin = nullptr;
        return CUOT_OK;
      }
      if (!c->qcf_margin) {
        if (cudaMalloc(&c->qcf_margin, sizeof(uint32_t)) != cudaSuccess) {
          cudaGetLastError();
          c->qcf_margin = nullptr;
          return fail(CUOT_ENOMEM, "margin word allocation failed");
        }
      }
      if (cudaMemset(c->qcf_margin, 0, sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        return fail(CUOT_ECUDA, "margin word reset failed");
      }
      return CUOT_OK;
    }
    default:
      return fail(CUOT_EINVAL, "unknown tuning key %d", key);
  }
}

}  // extern "C"
