// pprf.cu -- GGM PPRF expansion (Ferret MPCOT and SOT seed expansion).
//
// One CTA expands one whole tree, level by level: level l+1 = children of
// level l with the emp-ot TwoKeyPRP node function (left = AES_k0(p) ^ p,
// right = AES_k1(p) ^ p, ferret/twokeyprp.h:7-63).  The per-level left/right
// XOR sums are reduced in-CTA with warp shuffles, so no level ever goes to
// the host and no per-level launch or device synchronisation is needed
// (cuOT launches aesExpand128 + xor_reduce passes + two cudaMemcpy2D per
// level, dev_layer.cu:36-42).  The receiver's punctured-path correction is
// applied in the same kernel right after the level's sums are known.
//
// Levels ping-pong between the caller's leaf buffer and a scratch buffer of
// the same size (the tree's slice of each), chosen so that the last level
// lands in the leaf buffer.  Intermediate levels stay in L2 (at most
// 3 CTAs x 2 x 2^(h-1) blocks per SM are live).
#include "pprf_kernel.cuh"

namespace cuot {

int pprf_init_device() {
  cudaError_t e = pprf_upload_keys();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "GGM key upload failed: %s", cudaGetErrorString(e));
  }
  return CUOT_OK;
}

template <int MODE>
static int launch_pprf(cuot_ctx *ctx, PprfArgs &a, cudaStream_t st) {
  static bool attr_set[64] = {false};
  const int dev = ctx->device;
  if (dev < 64 && !attr_set[dev]) {
    cudaError_t e = cudaFuncSetAttribute(pprf_tree_kernel<MODE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kTableBytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(CUOT_ECUDA, "cudaFuncSetAttribute failed: %s", cudaGetErrorString(e));
    }
    attr_set[dev] = true;
  }
  a.t0 = ctx->t0_d;
  void *scr = nullptr;
  CUOT_TRY(scratch(ctx, (a.t << a.h) * sizeof(Blk), &scr));
  a.scratch = static_cast<Blk *>(scr);
  pprf_tree_kernel<MODE><<<dim3((unsigned)a.t), ctx->pprf_threads, kTableBytes, st>>>(a);
  return launch_status();
}

static int check_tree_shape(uint64_t t, int h) {
  if (t < 1 || t > 0x7fffffffull) return fail(CUOT_EINVAL, "t=%llu out of range", (unsigned long long)t);
  if (h < 1 || h > 30) return fail(CUOT_EINVAL, "h=%d out of range [1,30]", h);
  if ((t << h) >> h != t) return fail(CUOT_EINVAL, "t * 2^h overflows");
  return CUOT_OK;
}

}  // namespace cuot

using namespace cuot;

extern "C" {

int cuot_ferret_pprf_sender(cuot_ctx *ctx, const cuot_block *roots_d, uint64_t t, int h,
                            const cuot_block *delta, cuot_block *leaves_d,
                            cuot_block *lsum_d, cuot_block *rsum_d,
                            cuot_block *secret_sum_d, void *stream) {
  if (!ctx || !roots_d || !delta || !leaves_d || !lsum_d || !rsum_d || !secret_sum_d)
    return fail(CUOT_EINVAL, "null argument");
  CUOT_TRY(check_tree_shape(t, h));
  DeviceGuard g(ctx);
  PprfArgs a{};
  a.t = t; a.h = h;
  a.roots = reinterpret_cast<const Blk *>(roots_d);
  a.leaves = reinterpret_cast<Blk *>(leaves_d);
  a.delta = host_load_blk(delta);
  a.lsum = reinterpret_cast<Blk *>(lsum_d);
  a.rsum = reinterpret_cast<Blk *>(rsum_d);
  a.ss_out = reinterpret_cast<Blk *>(secret_sum_d);
  return launch_pprf<FERRET_SEND>(ctx, a, static_cast<cudaStream_t>(stream));
}

int cuot_ferret_pprf_recver(cuot_ctx *ctx, const cuot_block *mc_d, const uint8_t *choice_d,
                            const cuot_block *secret_sum_d, uint64_t t, int h,
                            cuot_block *leaves_d, void *stream) {
  if (!ctx || !mc_d || !choice_d || !secret_sum_d || !leaves_d)
    return fail(CUOT_EINVAL, "null argument");
  CUOT_TRY(check_tree_shape(t, h));
  DeviceGuard g(ctx);
  PprfArgs a{};
  a.t = t; a.h = h;
  a.mc = reinterpret_cast<const Blk *>(mc_d);
  a.choice = choice_d;
  a.ss_in = reinterpret_cast<const Blk *>(secret_sum_d);
  a.leaves = reinterpret_cast<Blk *>(leaves_d);
  return launch_pprf<FERRET_RECV>(ctx, a, static_cast<cudaStream_t>(stream));
}

int cuot_sot_pprf_sender(cuot_ctx *ctx, const cuot_block *roots_d, uint64_t t, int h,
                         const cuot_block *delta, const cuot_block *base0_d,
                         const cuot_block *base1_d, cuot_block *leaves_d,
                         cuot_block *m0_d, cuot_block *m1_d, void *stream) {
  if (!ctx || !roots_d || !delta || !base0_d || !base1_d || !leaves_d || !m0_d || !m1_d)
    return fail(CUOT_EINVAL, "null argument");
  CUOT_TRY(check_tree_shape(t, h));
  DeviceGuard g(ctx);
  PprfArgs a{};
  a.t = t; a.h = h;
  a.roots = reinterpret_cast<const Blk *>(roots_d);
  a.leaves = reinterpret_cast<Blk *>(leaves_d);
  a.delta = host_load_blk(delta);
  a.base0 = reinterpret_cast<const Blk *>(base0_d);
  a.base1 = reinterpret_cast<const Blk *>(base1_d);
  a.m0 = reinterpret_cast<Blk *>(m0_d);
  a.m1 = reinterpret_cast<Blk *>(m1_d);
  return launch_pprf<SOT_SEND>(ctx, a, static_cast<cudaStream_t>(stream));
}

int cuot_sot_pprf_recver(cuot_ctx *ctx, const cuot_block *m0_d, const cuot_block *m1_d,
                         const cuot_block *mc_d, const uint8_t *choice_d, uint64_t t,
                         int h, cuot_block *leaves_d, void *stream) {
  if (!ctx || !m0_d || !m1_d || !mc_d || !choice_d || !leaves_d)
    return fail(CUOT_EINVAL, "null argument");
  CUOT_TRY(check_tree_shape(t, h));
  DeviceGuard g(ctx);
  PprfArgs a{};
  a.t = t; a.h = h;
  a.m0_in = reinterpret_cast<const Blk *>(m0_d);
  a.m1_in = reinterpret_cast<const Blk *>(m1_d);
  a.mc = reinterpret_cast<const Blk *>(mc_d);
  a.choice = choice_d;
  a.leaves = reinterpret_cast<Blk *>(leaves_d);
  return launch_pprf<SOT_RECV>(ctx, a, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
