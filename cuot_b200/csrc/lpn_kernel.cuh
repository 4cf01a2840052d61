// lpn_kernel.cuh -- device code of the Ferret primal LPN rows (emp-ot
// LpnF2::__compute4 / __compute1, lpn_f2.h:46-79), shared by the single-
// instance kernel (lpn.cu) and the batched engine (batch.cu).
#pragma once
#include "ctx.cuh"

namespace cuot {
namespace {

struct LpnArgs {
  AesKey key;
  const uint32_t *t0;
  const Blk *kk;
  Blk *e;                 // row `row_lo` of the n-row matrix
  // Dual-role launches (both roles of one extension on this GPU): the second
  // role's kk and rows, XORed with the same public index matrix; else null.
  const Blk *kk2;
  Blk *e2;
  int64_t n, k, tail;     // tail: first row handled by the one-row path
  int64_t row_lo;         // first row held in e (a multiple of 4)
  int64_t g0, ngroups;    // 4-row groups [g0, g0 + ngroups)
  int64_t j0, ntail;      // one-row rows [j0, j0 + ntail)
  uint32_t mask;
  int d;
};

constexpr int kLpnThreads = 256;

__device__ __forceinline__ uint32_t lpn_idx(uint32_t w, uint32_t mask, uint32_t k) {
  uint32_t x = w & mask;
  return x >= k ? x - k : x;
}

// Rows 4g..4g+3 for d = D known at compile time.
// The D plaintexts makeBlock(i, m) = {m, 0, i_lo, i_hi} (m < D < 256) differ
// only in byte 0, so after AddRoundKey they differ only in byte 0 of column
// 0.  Round 1 reads that byte only for output column 0 (ShiftRows keeps row
// 0 in place); output columns 1..3 and three of column 0's four lookups are
// the same for all D blocks and are computed once per group.
// DUAL: both roles (kk/e and kk2/e2) from one index computation.
template <int D, bool DUAL = false>
__device__ __forceinline__ void lpn_group4(const LpnArgs &a, const TabRef &T, int64_t g) {
  static_assert(D <= 256, "the round-1 sharing needs m < 256");
  const int64_t i = 4 * g;
  const uint32_t k = uint32_t(a.k), mask = a.mask;
  const AesKey &K = a.key;
  Blk acc[4], acc2[4];
#pragma unroll
  for (int m = 0; m < 4; m++) acc[m] = acc2[m] = Blk{{0, 0, 0, 0}};
  // makeBlock(i, m): low qword m, high qword i.
  const uint32_t ilo = uint32_t(uint64_t(i)), ihi = uint32_t(uint64_t(i) >> 32);
  const uint32_t s1 = K.rk[1], s2 = ilo ^ K.rk[2], s3 = ihi ^ K.rk[3];
  const uint32_t s0hi = K.rk[0];  // bytes 1..3 of column 0 for every m
  const uint32_t c1 = round_col(T, s1, s2, s3, s0hi, K.rkr[5]);
  const uint32_t c2 = round_col(T, s2, s3, s0hi, s1, K.rkr[6]);
  const uint32_t c3 = round_col(T, s3, s0hi, s1, s2, K.rkr[7]);
  const uint32_t c0x = t2<2>(T, s2) ^ rotl8(t0<1>(T, s1) ^ t2<3>(T, s3) ^ K.rkr[4]);
#pragma unroll
  for (int m = 0; m < D; m += 2) {
    uint32_t x[4] = {t0<0>(T, uint32_t(m) ^ K.rk[0]) ^ c0x, c1, c2, c3};
    uint32_t y[4] = {t0<0>(T, uint32_t(m + 1) ^ K.rk[0]) ^ c0x, c1, c2, c3};
    aes_enc2_from_round2(T, x, y, K);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int word = 4 * m + q;  // compile-time after unrolling
      const uint32_t idx = lpn_idx(x[q], mask, k);
      acc[word / D] = blk_xor(acc[word / D], ldg_blk(a.kk + idx));
      if constexpr (DUAL) acc2[word / D] = blk_xor(acc2[word / D], ldg_blk(a.kk2 + idx));
    }
    if (m + 1 < D) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int word = 4 * (m + 1) + q;
        const uint32_t idx = lpn_idx(y[q], mask, k);
        acc[word / D] = blk_xor(acc[word / D], ldg_blk(a.kk + idx));
        if constexpr (DUAL) acc2[word / D] = blk_xor(acc2[word / D], ldg_blk(a.kk2 + idx));
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 4; m++) {
    Blk *p = a.e + (i - a.row_lo) + m;
    st_blk_cs(p, blk_xor(ld_blk(p), acc[m]));
    if constexpr (DUAL) {
      Blk *p2 = a.e2 + (i - a.row_lo) + m;
      st_blk_cs(p2, blk_xor(ld_blk(p2), acc2[m]));
    }
  }
}

// Rows 4g..4g+3 for any d (1..32); the second role too when a.kk2 is set.
__device__ void lpn_group4_dyn(const LpnArgs &a, const TabRef &T, int64_t g) {
  const int64_t i = 4 * g;
  const uint32_t k = uint32_t(a.k), mask = a.mask;
  const bool dual = a.kk2 != nullptr;
  Blk acc[4] = {{{0, 0, 0, 0}}, {{0, 0, 0, 0}}, {{0, 0, 0, 0}}, {{0, 0, 0, 0}}};
  Blk acc2[4] = {{{0, 0, 0, 0}}, {{0, 0, 0, 0}}, {{0, 0, 0, 0}}, {{0, 0, 0, 0}}};
  const uint32_t ilo = uint32_t(uint64_t(i)), ihi = uint32_t(uint64_t(i) >> 32);
  for (int m = 0; m < a.d; m++) {
    uint32_t x[4] = {uint32_t(m), 0u, ilo, ihi};
    aes_enc(T, x, a.key);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int word = 4 * m + q;
      const uint32_t idx = lpn_idx(x[q], mask, k);
      const Blk v = ldg_blk(a.kk + idx);
      const Blk v2 = dual ? ldg_blk(a.kk2 + idx) : Blk{{0, 0, 0, 0}};
      const int row = word / a.d;
#pragma unroll
      for (int r = 0; r < 4; r++)
        if (r == row) {
          acc[r] = blk_xor(acc[r], v);
          acc2[r] = blk_xor(acc2[r], v2);
        }
    }
  }
#pragma unroll
  for (int m = 0; m < 4; m++) {
    Blk *p = a.e + (i - a.row_lo) + m;
    st_blk_cs(p, blk_xor(ld_blk(p), acc[m]));
    if (dual) {
      Blk *p2 = a.e2 + (i - a.row_lo) + m;
      st_blk_cs(p2, blk_xor(ld_blk(p2), acc2[m]));
    }
  }
}

// One tail row (emp-ot __compute1, lpn_f2.h:61-70); both roles when a.kk2
// is set.
__device__ void lpn_row1(const LpnArgs &a, const TabRef &T, int64_t j) {
  const int nb = (a.d + 3) / 4;
  const uint32_t k = uint32_t(a.k);
  const bool dual = a.kk2 != nullptr;
  const uint32_t jlo = uint32_t(uint64_t(j)), jhi = uint32_t(uint64_t(j) >> 32);
  Blk acc{{0, 0, 0, 0}}, acc2{{0, 0, 0, 0}};
  int done = 0;
  for (int m = 0; m < nb; m++) {
    uint32_t x[4] = {uint32_t(m), 0u, jlo, jhi};
    aes_enc(T, x, a.key);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (done < a.d) {
        acc = blk_xor(acc, ldg_blk(a.kk + (x[q] % k)));
        if (dual) acc2 = blk_xor(acc2, ldg_blk(a.kk2 + (x[q] % k)));
      }
      done++;
    }
  }
  Blk *p = a.e + (j - a.row_lo);
  st_blk(p, blk_xor(ld_blk(p), acc));
  if (dual) {
    Blk *p2 = a.e2 + (j - a.row_lo);
    st_blk(p2, blk_xor(ld_blk(p2), acc2));
  }
}

}  // namespace
}  // namespace cuot
