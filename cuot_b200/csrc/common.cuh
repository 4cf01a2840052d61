// common.cuh -- shared device/host definitions for libcuot (sm_100a).
//
// Blocks are 16 bytes with the memory image of emp-tool's `block` and cuOT's
// `blk` (gpu/gpu_define.h:12-16): four little-endian uint32 words, word 0 =
// bytes 0..3.  AES state words here are the FIPS-197 columns read as
// little-endian uint32 (row r of column c = byte r of word c), so blocks are
// encrypted without any byte swapping (cuOT's kernel swaps every word,
// gpu/aes_op.cu:117-171).
#pragma once
#include <cstring>
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/cuot.h"

namespace cuot {

struct __align__(16) Blk { uint32_t w[4]; };
// A block from a host pointer with no alignment guarantee (a cuot_block is
// 4-byte aligned; dereferencing it as the 16-byte-aligned Blk would let the
// compiler use an aligned vector load).
__host__ inline Blk host_load_blk(const void *p) {
  Blk b;
  std::memcpy(b.w, p, 16);
  return b;
}

__host__ __device__ __forceinline__ Blk blk_xor(Blk a, Blk b) {
  Blk r;
#pragma unroll
  for (int i = 0; i < 4; i++) r.w[i] = a.w[i] ^ b.w[i];
  return r;
}

__device__ __forceinline__ Blk ld_blk(const Blk *p) {
  uint4 v = *reinterpret_cast<const uint4 *>(p);
  return Blk{{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ Blk ldg_blk(const Blk *p) {
  uint4 v = __ldg(reinterpret_cast<const uint4 *>(p));
  return Blk{{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ void st_blk(Blk *p, Blk b) {
  *reinterpret_cast<uint4 *>(p) = make_uint4(b.w[0], b.w[1], b.w[2], b.w[3]);
}
// Streaming store for outputs nobody re-reads soon (leaves, LPN rows).
__device__ __forceinline__ void st_blk_cs(Blk *p, Blk b) {
  __stcs(reinterpret_cast<uint4 *>(p), make_uint4(b.w[0], b.w[1], b.w[2], b.w[3]));
}

// ---------------------------------------------------------------------------
// AES-128 round keys: 44 little-endian words (FIPS-197 key schedule), and
// rkr[i] = rotr8(rk[i]) so a round folds its key into the rotated half:
// rotl8(x ^ rotr8(k)) = rotl8(x) ^ k saves one instruction per column.
struct AesKey { uint32_t rk[44]; uint32_t rkr[44]; };

// Host side (aes_host.cu): the S-box is computed from GF(2^8) inversion and
// the affine map; T0[x] = 2S | S<<8 | S<<16 | 3S<<24 (MixColumns column of
// S[x], little-endian).
void host_aes_key_expand(const uint8_t key[16], AesKey *out);
const uint32_t *host_t0_table();
void host_aes_encrypt(const AesKey &k, const uint8_t in[16], uint8_t out[16]);

// ---------------------------------------------------------------------------
// Shared-memory T-table.  Row x (256 bytes) holds T0[x] replicated in words
// 0..31 and T2[x] = rotl16(T0[x]) replicated in words 32..63, so lane l
// always reads bank l (conflict-free) and the byte offset of entry x for lane
// l is (x << 8) | (l << 2): one PRMT builds it from the state word and the
// lane offset.  T1 = rotl8(T0) and T3 = rotl8(T2) come from one funnel shift.
constexpr int kTableWords = 256 * 64;
constexpr int kTableBytes = kTableWords * 4;  // 64 KiB

__device__ __forceinline__ void stage_table(uint32_t *tab, const uint32_t *t0_g) {
  for (int i = threadIdx.x; i < kTableWords; i += blockDim.x) {
    int x = i >> 6, col = i & 63;
    uint32_t v = __ldg(&t0_g[x]);
    if (col >= 32) v = __funnelshift_l(v, v, 16);
    tab[i] = v;
  }
}

struct TabRef {
  const char *tab;   // shared-memory table (generic pointer into smem)
  uint32_t lane4;    // (lane id) * 4
};

// (byte b of s) << 8 | lane4: PRMT with byte0 <- lane4.b0 (index 4),
// byte1 <- s.b_b (index b), bytes 2,3 <- lane4.b1 (index 5, always zero).
template <int b>
__device__ __forceinline__ uint32_t tab_off(uint32_t s, uint32_t lane4) {
  return __byte_perm(s, lane4, 0x5504u | (uint32_t(b) << 4));
}
template <int b>
__device__ __forceinline__ uint32_t t0(const TabRef &t, uint32_t s) {
  return *reinterpret_cast<const uint32_t *>(t.tab + tab_off<b>(s, t.lane4));
}
template <int b>
__device__ __forceinline__ uint32_t t2(const TabRef &t, uint32_t s) {
  return *reinterpret_cast<const uint32_t *>(t.tab + tab_off<b>(s, t.lane4) + 128);
}
__device__ __forceinline__ uint32_t rotl8(uint32_t x) { return __funnelshift_l(x, x, 8); }

// out_c = T0[b0(s_c)] ^ T1[b1(s_c+1)] ^ T2[b2(s_c+2)] ^ T3[b3(s_c+3)] ^ k_c
//       = T0[..] ^ T2[..] ^ rotl8(T0[b1(s_c+1)] ^ T2[b3(s_c+3)] ^ rotr8(k_c))
__device__ __forceinline__ uint32_t round_col(const TabRef &t, uint32_t a, uint32_t b,
                                              uint32_t c, uint32_t d, uint32_t kr) {
  return t0<0>(t, a) ^ t2<2>(t, c) ^ rotl8(t0<1>(t, b) ^ t2<3>(t, d) ^ kr);
}

// Final round column: S[b0(a)] | S[b1(b)]<<8 | S[b2(c)]<<16 | S[b3(d)]<<24.
// T2[x] byte 0 = S[x], T0[x] byte 1 = S[x], T0[x] byte 2 = S[x],
// T2[x] byte 3 = S[x].
__device__ __forceinline__ uint32_t final_col(const TabRef &t, uint32_t a, uint32_t b,
                                              uint32_t c, uint32_t d, uint32_t k) {
  uint32_t ta = t2<0>(t, a), tb = t0<1>(t, b), tc = t0<2>(t, c), td = t2<3>(t, d);
  uint32_t lo = __byte_perm(ta, tb, 0x3350u);  // byte0 = ta.b0, byte1 = tb.b1
  uint32_t hi = __byte_perm(tc, td, 0x7200u);  // byte2 = tc.b2, byte3 = td.b3
  return __byte_perm(lo, hi, 0x7610u) ^ k;
}

// AES-128 encryption of one block.  The key schedule is indexed with
// compile-time indices after unrolling, so kernel-parameter or __constant__
// schedules become constant-bank operands.
__device__ __forceinline__ void aes_enc(const TabRef &t, uint32_t (&x)[4], const AesKey &key) {
  const uint32_t *rk = key.rk, *kr = key.rkr;
  uint32_t s0 = x[0] ^ rk[0], s1 = x[1] ^ rk[1], s2 = x[2] ^ rk[2], s3 = x[3] ^ rk[3];
#pragma unroll
  for (int r = 1; r < 10; r++) {
    uint32_t o0 = round_col(t, s0, s1, s2, s3, kr[4 * r + 0]);
    uint32_t o1 = round_col(t, s1, s2, s3, s0, kr[4 * r + 1]);
    uint32_t o2 = round_col(t, s2, s3, s0, s1, kr[4 * r + 2]);
    uint32_t o3 = round_col(t, s3, s0, s1, s2, kr[4 * r + 3]);
    s0 = o0; s1 = o1; s2 = o2; s3 = o3;
  }
  x[0] = final_col(t, s0, s1, s2, s3, rk[40]);
  x[1] = final_col(t, s1, s2, s3, s0, rk[41]);
  x[2] = final_col(t, s2, s3, s0, s1, rk[42]);
  x[3] = final_col(t, s3, s0, s1, s2, rk[43]);
}

// Two independent blocks interleaved for instruction-level parallelism.
__device__ __forceinline__ void aes_enc2(const TabRef &t, uint32_t (&a)[4], const AesKey &KA,
                                         uint32_t (&b)[4], const AesKey &KB) {
  const uint32_t *ka = KA.rk, *kb = KB.rk, *kar = KA.rkr, *kbr = KB.rkr;
  uint32_t s0 = a[0] ^ ka[0], s1 = a[1] ^ ka[1], s2 = a[2] ^ ka[2], s3 = a[3] ^ ka[3];
  uint32_t u0 = b[0] ^ kb[0], u1 = b[1] ^ kb[1], u2 = b[2] ^ kb[2], u3 = b[3] ^ kb[3];
#pragma unroll
  for (int r = 1; r < 10; r++) {
    uint32_t o0 = round_col(t, s0, s1, s2, s3, kar[4 * r + 0]);
    uint32_t p0 = round_col(t, u0, u1, u2, u3, kbr[4 * r + 0]);
    uint32_t o1 = round_col(t, s1, s2, s3, s0, kar[4 * r + 1]);
    uint32_t p1 = round_col(t, u1, u2, u3, u0, kbr[4 * r + 1]);
    uint32_t o2 = round_col(t, s2, s3, s0, s1, kar[4 * r + 2]);
    uint32_t p2 = round_col(t, u2, u3, u0, u1, kbr[4 * r + 2]);
    uint32_t o3 = round_col(t, s3, s0, s1, s2, kar[4 * r + 3]);
    uint32_t p3 = round_col(t, u3, u0, u1, u2, kbr[4 * r + 3]);
    s0 = o0; s1 = o1; s2 = o2; s3 = o3;
    u0 = p0; u1 = p1; u2 = p2; u3 = p3;
  }
  a[0] = final_col(t, s0, s1, s2, s3, ka[40]);
  b[0] = final_col(t, u0, u1, u2, u3, kb[40]);
  a[1] = final_col(t, s1, s2, s3, s0, ka[41]);
  b[1] = final_col(t, u1, u2, u3, u0, kb[41]);
  a[2] = final_col(t, s2, s3, s0, s1, ka[42]);
  b[2] = final_col(t, u2, u3, u0, u1, kb[42]);
  a[3] = final_col(t, s3, s0, s1, s2, ka[43]);
  b[3] = final_col(t, u3, u0, u1, u2, kb[43]);
}

// Rounds 2..10 of two blocks given their states after round 1 (round key 1
// included).
__device__ __forceinline__ void aes_enc2_from_round2(const TabRef &t, uint32_t (&a)[4],
                                                     uint32_t (&b)[4], const AesKey &K) {
  const uint32_t *kr = K.rkr, *rk = K.rk;
  uint32_t s0 = a[0], s1 = a[1], s2 = a[2], s3 = a[3];
  uint32_t u0 = b[0], u1 = b[1], u2 = b[2], u3 = b[3];
#pragma unroll
  for (int r = 2; r < 10; r++) {
    uint32_t o0 = round_col(t, s0, s1, s2, s3, kr[4 * r + 0]);
    uint32_t p0 = round_col(t, u0, u1, u2, u3, kr[4 * r + 0]);
    uint32_t o1 = round_col(t, s1, s2, s3, s0, kr[4 * r + 1]);
    uint32_t p1 = round_col(t, u1, u2, u3, u0, kr[4 * r + 1]);
    uint32_t o2 = round_col(t, s2, s3, s0, s1, kr[4 * r + 2]);
    uint32_t p2 = round_col(t, u2, u3, u0, u1, kr[4 * r + 2]);
    uint32_t o3 = round_col(t, s3, s0, s1, s2, kr[4 * r + 3]);
    uint32_t p3 = round_col(t, u3, u0, u1, u2, kr[4 * r + 3]);
    s0 = o0; s1 = o1; s2 = o2; s3 = o3;
    u0 = p0; u1 = p1; u2 = p2; u3 = p3;
  }
  a[0] = final_col(t, s0, s1, s2, s3, rk[40]);
  b[0] = final_col(t, u0, u1, u2, u3, rk[40]);
  a[1] = final_col(t, s1, s2, s3, s0, rk[41]);
  b[1] = final_col(t, u1, u2, u3, u0, rk[41]);
  a[2] = final_col(t, s2, s3, s0, s1, rk[42]);
  b[2] = final_col(t, u2, u3, u0, u1, rk[42]);
  a[3] = final_col(t, s3, s0, s1, s2, rk[43]);
  b[3] = final_col(t, u3, u0, u1, u2, rk[43]);
}

// ---------------------------------------------------------------------------
// Warp / block XOR reductions of a block value.
__device__ __forceinline__ Blk warp_xor(Blk v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int i = 0; i < 4; i++) v.w[i] ^= __shfl_xor_sync(0xffffffffu, v.w[i], o);
  return v;
}

// ---------------------------------------------------------------------------
// Host-side helpers.
#define CUOT_TRY(expr)                                                         \
  do {                                                                         \
    int _s = (expr);                                                           \
    if (_s != CUOT_OK) return _s;                                              \
  } while (0)

// Counts `nlaunch` kernel launches and maps cudaGetLastError() to
// CUOT_OK / CUOT_ECUDA.
int launch_status(int nlaunch = 1);

}  // namespace cuot
