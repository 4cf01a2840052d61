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
#include "ctx.cuh"

namespace cuot {

// Fixed GGM keys: k0 = zero_block, k1 = makeBlock(0, 1) (spcot_sender.h:63).
__constant__ AesKey c_ggm_rk[2];

int pprf_init_device() {
  AesKey k[2];
  uint8_t key[16] = {0};
  host_aes_key_expand(key, &k[0]);
  key[0] = 1;
  host_aes_key_expand(key, &k[1]);
  cudaError_t e = cudaMemcpyToSymbol(c_ggm_rk, k, sizeof k);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "GGM key upload failed: %s", cudaGetErrorString(e));
  }
  return CUOT_OK;
}

enum PprfMode { FERRET_SEND = 0, FERRET_RECV = 1, SOT_SEND = 2, SOT_RECV = 3 };

struct PprfArgs {
  uint64_t t;
  int h;
  const uint32_t *t0;
  const Blk *roots;  // senders
  Blk *leaves, *scratch;
  Blk delta;
  // Ferret sender outputs [t][h], [t]
  Blk *lsum, *rsum, *ss_out;
  // receivers
  const Blk *mc;          // Ferret [t][h]; SOT [h][t]
  const uint8_t *choice;  // Ferret [t][h]; SOT [h][t]
  const Blk *ss_in;       // Ferret [t]
  // SOT sender inputs [h][t], outputs [h+1][t]; SOT receiver inputs [h+1][t]
  const Blk *base0, *base1;
  Blk *m0, *m1;
  const Blk *m0_in, *m1_in;
};

constexpr int kPprfThreads = 256;

__device__ __forceinline__ Blk mask_lsb(Blk b) {
  b.w[0] &= ~1u;  // emp-ot `& one`, one = makeBlock(~0, ~1)
  return b;
}

template <int MODE>
__global__ void __launch_bounds__(kPprfThreads, 3) pprf_tree_kernel(PprfArgs a) {
  extern __shared__ __align__(16) uint32_t smem_tab[];
  __shared__ Blk red[2][kPprfThreads / 32];
  __shared__ unsigned long long s_ap;

  stage_table(smem_tab, a.t0);
  const uint64_t tree = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const TabRef T{reinterpret_cast<const char *>(smem_tab), uint32_t(lane) * 4u};
  const int h = a.h;
  const uint64_t W = 1ull << h;
  Blk *const bufs[2] = {a.leaves + tree * W, a.scratch + tree * W};
  Blk root{{0, 0, 0, 0}};
  if (MODE == FERRET_SEND || MODE == SOT_SEND) root = ldg_blk(a.roots + tree);
  if (tid == 0) s_ap = 0;
  __syncthreads();

  for (int l = 0; l < h; l++) {
    const Blk *in = bufs[(h - l) & 1];
    Blk *out = bufs[(h - l - 1) & 1];
    const bool last = (l == h - 1);
    const uint64_t np = 1ull << l;
    Blk accL{{0, 0, 0, 0}}, accR{{0, 0, 0, 0}};
    for (uint64_t i = tid; i < np; i += kPprfThreads) {
      const Blk p = (l == 0) ? root : ld_blk(in + i);
      uint32_t L[4] = {p.w[0], p.w[1], p.w[2], p.w[3]};
      uint32_t R[4] = {p.w[0], p.w[1], p.w[2], p.w[3]};
      aes_enc2(T, L, c_ggm_rk[0], R, c_ggm_rk[1]);
      Blk cl{{L[0] ^ p.w[0], L[1] ^ p.w[1], L[2] ^ p.w[2], L[3] ^ p.w[3]}};
      Blk cr{{R[0] ^ p.w[0], R[1] ^ p.w[1], R[2] ^ p.w[2], R[3] ^ p.w[3]}};
      accL = blk_xor(accL, cl);
      accR = blk_xor(accR, cr);
      if ((MODE == FERRET_SEND || MODE == FERRET_RECV) && last) {
        cl = mask_lsb(cl);
        cr = mask_lsb(cr);
      }
      if (last) {
        st_blk_cs(out + 2 * i, cl);
        st_blk_cs(out + 2 * i + 1, cr);
      } else {
        st_blk(out + 2 * i, cl);
        st_blk(out + 2 * i + 1, cr);
      }
    }
    accL = warp_xor(accL);
    accR = warp_xor(accR);
    if (lane == 0) {
      red[0][warp] = accL;
      red[1][warp] = accR;
    }
    __syncthreads();
    if (tid == 0) {
      Blk S[2] = {{{0, 0, 0, 0}}, {{0, 0, 0, 0}}};
#pragma unroll
      for (int w = 0; w < kPprfThreads / 32; w++) {
        S[0] = blk_xor(S[0], red[0][w]);
        S[1] = blk_xor(S[1], red[1][w]);
      }
      if (MODE == FERRET_SEND) {
        // ot_msg_0/1 of level l (spcot_sender.h:66-84), host layout [t][h]
        st_blk(a.lsum + tree * h + l, S[0]);
        st_blk(a.rsum + tree * h + l, S[1]);
        if (last)  // secret_sum = XOR(masked leaves) ^ delta (spcot_sender.h:49-58)
          st_blk(a.ss_out + tree, blk_xor(mask_lsb(blk_xor(S[0], S[1])), a.delta));
      } else if (MODE == SOT_SEND) {
        const uint64_t o = uint64_t(l) * a.t + tree;
        const Blk b0 = ldg_blk(a.base0 + o), b1 = ldg_blk(a.base1 + o);
        st_blk(a.m0 + o, blk_xor(b0, S[0]));
        st_blk(a.m1 + o, blk_xor(b1, S[1]));
        if (last) {  // extra row that carries delta (silent/sender.cu:97-102)
          const uint64_t o2 = uint64_t(l + 1) * a.t + tree;
          st_blk(a.m0 + o2, blk_xor(blk_xor(b0, S[1]), a.delta));
          st_blk(a.m1 + o2, blk_xor(blk_xor(b1, S[0]), a.delta));
        }
      } else if (MODE == FERRET_RECV) {
        // spcot_recver.h:71-95: b = 0 -> fill the even child, puncture the odd.
        const int b = a.choice[tree * h + l] ? 1 : 0;
        const Blk m = ldg_blk(a.mc + tree * h + l);
        const uint64_t ap = s_ap;
        const uint64_t f = 2 * ap + b, pun = 2 * ap + 1 - b;
        // The node at f currently holds X (garbage, derived from the unknown
        // punctured parent).  S_b includes X, so X ^ S_b ^ m is the XOR of
        // the other same-side nodes with m: the sender's node.
        const Blk fix = blk_xor(S[b], m);
        if (!last) {
          st_blk(out + f, blk_xor(ld_blk(out + f), fix));
          s_ap = pun;
        } else {
          // Leaves are stored masked.  Filled leaf (masked) = X' ^ mask(fix).
          st_blk(out + f, blk_xor(ld_blk(out + f), mask_lsb(fix)));
          // Punctured leaf = XOR of all other masked leaves ^ secret_sum
          // (spcot_recver.h:53-64) = mask(S0 ^ S1 ^ fix) ^ G' ^ ss, with G'
          // the masked garbage leaf at `pun` (its term cancels).
          const Blk g = ld_blk(out + pun);
          Blk r = blk_xor(mask_lsb(blk_xor(blk_xor(S[0], S[1]), fix)), g);
          r = blk_xor(r, ldg_blk(a.ss_in + tree));
          st_blk(out + pun, r);
        }
      } else {  // SOT_RECV (silent/recver.cu:98-115, 143-155)
        const uint64_t o = uint64_t(l) * a.t + tree;
        const int c = a.choice[o] ? 1 : 0;
        const Blk *mcur = c ? a.m1_in : a.m0_in;
        const Blk mcv = ldg_blk(a.mc + o);
        const Blk dec = blk_xor(ldg_blk(mcur + o), mcv);
        const uint64_t ap = s_ap;
        const uint64_t f = 2 * ap + c, pun = 2 * ap + 1 - c;
        st_blk(out + f, blk_xor(ld_blk(out + f), blk_xor(dec, S[c])));
        s_ap = pun;
        if (last) {
          const Blk dec2 = blk_xor(ldg_blk(mcur + uint64_t(l + 1) * a.t + tree), mcv);
          st_blk(out + pun, blk_xor(ld_blk(out + pun), blk_xor(dec2, S[1 - c])));
        }
      }
    }
    __syncthreads();
  }
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
  pprf_tree_kernel<MODE><<<dim3((unsigned)a.t), kPprfThreads, kTableBytes, st>>>(a);
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
  a.delta = *reinterpret_cast<const Blk *>(delta);
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
  a.delta = *reinterpret_cast<const Blk *>(delta);
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
