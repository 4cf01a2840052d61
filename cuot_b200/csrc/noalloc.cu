// noalloc.cu -- a Ferret PPRF sender entry point that allocates nothing.
//
// The ordinary entry point (cuot_ferret_pprf_sender) takes its level
// ping-pong buffer from the context's scratch arena, which may call
// cudaMalloc, and needs a context, whose creation calls cudaMalloc.  Some
// callers cannot allocate device memory at call time: a serving process whose
// whole HBM budget is owned by its own pool allocator, or a latency-critical
// path where cudaMalloc/cudaFree would implicitly synchronise the device and
// stall every other stream.  This file gives them the same kernel with its
// scratch in a fixed file-scope device array and the AES table in another,
// so a call does no allocation at all.
//
// The arrays are part of the loaded module: every GPU that loads libcuot
// holds them (16 MiB + 1 KiB) until the process exits.
#include <mutex>

#include "pprf_kernel.cuh"

namespace cuot {
namespace {

// Largest t * 2^h (leaves) a call may ask for: 2^20 blocks = 16 MiB.
constexpr uint64_t kNoAllocMaxLeaves = 1ull << 20;

// Scratch for the intermediate tree levels.  Every call on a device uses the
// same array.  Nothing in it has to start at zero: the kernel writes every
// level entry before reading it.
__device__ __align__(256) Blk g_noalloc_scratch[kNoAllocMaxLeaves];
// T0 table staged into shared memory by the kernel.
__device__ __align__(256) uint32_t g_noalloc_t0[256];

struct DeviceState {
  bool ready = false;
  Blk *scratch = nullptr;   // device address of g_noalloc_scratch
  uint32_t *t0 = nullptr;   // device address of g_noalloc_t0
};

std::mutex g_mu;
DeviceState g_state[64];

int setup_error(const char *what, cudaError_t e) {
  cudaGetLastError();
  return fail(CUOT_ECUDA, "no-alloc set-up: %s failed: %s", what, cudaGetErrorString(e));
}

// One-time set-up for the current device: upload the key schedules and the
// T0 table into this file's arrays and look up their device addresses (in
// host code the array names are only host-side stand-ins).
int setup_current_device(DeviceState **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return setup_error("cudaGetDevice", e);
  if (dev < 0 || dev >= 64) return fail(CUOT_EINVAL, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState &s = g_state[dev];
  if (!s.ready) {
    if ((e = pprf_upload_keys()) != cudaSuccess) return setup_error("key upload", e);
    if ((e = cudaMemcpyToSymbol(g_noalloc_t0, host_t0_table(), sizeof(uint32_t) * 256)) != cudaSuccess)
      return setup_error("table upload", e);
    if ((e = cudaGetSymbolAddress(reinterpret_cast<void **>(&s.scratch), g_noalloc_scratch)) != cudaSuccess)
      return setup_error("cudaGetSymbolAddress(scratch)", e);
    if ((e = cudaGetSymbolAddress(reinterpret_cast<void **>(&s.t0), g_noalloc_t0)) != cudaSuccess)
      return setup_error("cudaGetSymbolAddress(table)", e);
    if ((e = cudaFuncSetAttribute(pprf_tree_kernel<FERRET_SEND>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, kTableBytes)) != cudaSuccess)
      return setup_error("cudaFuncSetAttribute", e);
    s.ready = true;
  }
  *out = &s;
  return CUOT_OK;
}

}  // namespace
}  // namespace cuot

using namespace cuot;

extern "C" int cuot_ferret_pprf_sender_noalloc(const cuot_block *roots_d, uint64_t t, int h,
                                               const cuot_block *delta, cuot_block *leaves_d,
                                               cuot_block *lsum_d, cuot_block *rsum_d,
                                               cuot_block *secret_sum_d, void *stream) {
  if (!roots_d || !delta || !leaves_d || !lsum_d || !rsum_d || !secret_sum_d)
    return fail(CUOT_EINVAL, "null argument");
  if (t < 1 || t > 0x7fffffffull) return fail(CUOT_EINVAL, "t=%llu out of range", (unsigned long long)t);
  if (h < 1 || h > 20) return fail(CUOT_EINVAL, "h=%d out of range [1,20]", h);
  if ((t << h) > kNoAllocMaxLeaves)
    return fail(CUOT_EINVAL,
                "t * 2^h = %llu leaves exceeds the no-alloc limit of %llu (16 MiB of scratch); "
                "use cuot_ferret_pprf_sender",
                (unsigned long long)(t << h), (unsigned long long)kNoAllocMaxLeaves);
  DeviceState *s = nullptr;
  CUOT_TRY(setup_current_device(&s));
  PprfArgs a{};
  a.t = t;
  a.h = h;
  a.t0 = s->t0;
  a.roots = reinterpret_cast<const Blk *>(roots_d);
  a.leaves = reinterpret_cast<Blk *>(leaves_d);
  a.scratch = s->scratch;
  a.delta = host_load_blk(delta);
  a.lsum = reinterpret_cast<Blk *>(lsum_d);
  a.rsum = reinterpret_cast<Blk *>(rsum_d);
  a.ss_out = reinterpret_cast<Blk *>(secret_sum_d);
  pprf_tree_kernel<FERRET_SEND><<<dim3(unsigned(t)), kPprfThreads, kTableBytes,
                                  static_cast<cudaStream_t>(stream)>>>(a);
  return launch_status();
}
