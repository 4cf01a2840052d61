// pprf_kernel.cuh -- the GGM PPRF tree kernel (one CTA per tree), shared by
// the translation units that launch it.  Each including file gets its own
// copy of the fixed-key schedule in constant memory and must upload it once
// per device before the first launch (pprf_upload_keys).
#pragma once
#include "ctx.cuh"

namespace cuot {
// Internal linkage: every including translation unit gets its own kernel
// instances bound to its own constant-memory key copy.
namespace {

// Fixed GGM keys: k0 = zero_block, k1 = makeBlock(0, 1) (spcot_sender.h:63).
__constant__ AesKey c_ggm_rk[2];

// Uploads this translation unit's copy of the GGM key schedules to the
// current device.
inline cudaError_t pprf_upload_keys() {
  AesKey k[2];
  uint8_t key[16] = {0};
  host_aes_key_expand(key, &k[0]);
  key[0] = 1;
  host_aes_key_expand(key, &k[1]);
  return cudaMemcpyToSymbol(c_ggm_rk, k, sizeof k);
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

// Threads per tree (CTA size): 256 by default, 128 selectable (tuning);
// the kernels are compiled for at most kPprfThreads.
constexpr int kPprfThreads = 256;

__device__ __forceinline__ Blk mask_lsb(Blk b) {
  b.w[0] &= ~1u;  // emp-ot `& one`, one = makeBlock(~0, ~1)
  return b;
}

// Shared-memory state of one tree expansion: per-warp level sums (left,
// right), double-buffered by level parity, and the receiver's path.
struct PprfSmem {
  Blk red[2][2][kPprfThreads / 32];
  unsigned long long ap;
};

// Expands tree `tree` of the instance described by `a` with the whole CTA
// (blockDim.x <= kPprfThreads threads, a multiple of 32).  scratch_tree: 2^h blocks for the level ping-pong.
// The T-table must already be staged (and synced) in shared memory.
template <int MODE>
__device__ __forceinline__ void pprf_tree(const PprfArgs &a, uint64_t tree, Blk *scratch_tree,
                                          const TabRef &T, PprfSmem &sm) {
  unsigned long long &s_ap = sm.ap;
  // Senders: the sums of level l leave the CTA (global stores by thread 0)
  // and nothing of them is read back, so one barrier per level suffices,
  // with the warp partials double-buffered by level parity: thread 0 reads
  // red[l & 1] before it enters level l + 1, and red[l & 1] is written again
  // only after the barrier that ends level l + 1.  Receivers patch a node of
  // the level just written, which the next level reads, so they keep a
  // second barrier.
  constexpr bool kSend = MODE == FERRET_SEND || MODE == SOT_SEND;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int h = a.h;
  const uint64_t W = 1ull << h;
  Blk *const bufs[2] = {a.leaves + tree * W, scratch_tree};
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
    for (uint64_t i = tid; i < np; i += blockDim.x) {
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
    Blk(&red)[2][kPprfThreads / 32] = sm.red[l & 1];
    if (lane == 0) {
      red[0][warp] = accL;
      red[1][warp] = accR;
    }
    __syncthreads();
    if (tid == 0) {
      Blk S[2] = {{{0, 0, 0, 0}}, {{0, 0, 0, 0}}};
#pragma unroll
      for (int w = 0; w < int(blockDim.x >> 5); w++) {
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
    if (!kSend) __syncthreads();
  }
}

// One CTA per tree of a single instance.
template <int MODE>
__global__ void __launch_bounds__(kPprfThreads, 3) pprf_tree_kernel(PprfArgs a) {
  extern __shared__ __align__(16) uint32_t smem_tab[];
  __shared__ PprfSmem sm;
  stage_table(smem_tab, a.t0);
  const TabRef T{reinterpret_cast<const char *>(smem_tab), uint32_t(threadIdx.x & 31) * 4u};
  const uint64_t tree = blockIdx.x;
  pprf_tree<MODE>(a, tree, a.scratch + (tree << a.h), T, sm);
}

}  // namespace
}  // namespace cuot
