// aes_bitslice.cu -- bitsliced AES-128 ECB (cuot_aes128_ecb_bitsliced): the
// register-only alternative to the T-table AES (cuot_aes128_ecb, lpn.cu), for
// measuring which of the two is faster on this GPU.  Each thread encrypts 32
// blocks as one bitsliced state (aes_bitslice.cuh).
#include "aes_bitslice.cuh"
#include "ctx.cuh"

namespace cuot {
namespace {

constexpr int kBsThreads = 128;

// Warps take tiles of 1024 consecutive blocks; lane l of a warp takes blocks
// l + 32 b (b < 32) of its tile, so each of the 32 load and store
// instructions of a tile covers 512 contiguous bytes.
__global__ void __launch_bounds__(kBsThreads) ecb_bitsliced_kernel(BitslicedKey key, Blk *io, uint64_t n) {
  __shared__ BitslicedKey sk;
  for (int i = threadIdx.x; i < 11 * 128; i += blockDim.x) (&sk.m[0][0])[i] = (&key.m[0][0])[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t tile = warp; tile * 1024 < n; tile += nwarps) {
    const uint64_t base = tile * 1024 + uint64_t(lane);
    uint32_t words[4][32];
#pragma unroll
    for (int b = 0; b < 32; b++) {
      const uint64_t i = base + 32u * uint64_t(b);
      const Blk v = i < n ? ld_blk(io + i) : Blk{{0, 0, 0, 0}};
#pragma unroll
      for (int w = 0; w < 4; w++) words[w][b] = v.w[w];
    }
    uint32_t s[128];
    bs_from_words(words, s);
    bs_encrypt(s, sk);
    bs_to_words(s, words);
#pragma unroll
    for (int b = 0; b < 32; b++) {
      const uint64_t i = base + 32u * uint64_t(b);
      if (i < n) st_blk(io + i, Blk{{words[0][b], words[1][b], words[2][b], words[3][b]}});
    }
  }
}

}  // namespace
}  // namespace cuot

using namespace cuot;

extern "C" int cuot_aes128_ecb_bitsliced(cuot_ctx *ctx, const uint8_t key[16], cuot_block *io_d,
                                         uint64_t nblocks, void *stream) {
  if (!ctx || !key || (!io_d && nblocks)) return fail(CUOT_EINVAL, "null argument");
  if (nblocks == 0) return CUOT_OK;
  DeviceGuard g(ctx);
  AesKey k;
  host_aes_key_expand(key, &k);
  BitslicedKey bk;
  bitsliced_key(k.rk, &bk);
  int sms = 148, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ecb_bitsliced_kernel, kBsThreads, 0);
  if (per_sm < 1) per_sm = 1;
  const uint64_t tiles = (nblocks + 1023) / 1024, warps_per_cta = kBsThreads / 32;
  const uint64_t need = (tiles + warps_per_cta - 1) / warps_per_cta;
  const uint64_t cap = uint64_t(sms) * uint64_t(per_sm);
  const unsigned grid = unsigned(need < cap ? need : cap);
  ecb_bitsliced_kernel<<<grid, kBsThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      bk, reinterpret_cast<Blk *>(io_d), nblocks);
  return launch_status();
}
