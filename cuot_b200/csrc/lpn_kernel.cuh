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
template <int D>
__device__ __forceinline__ void lpn_group4(const LpnArgs &a, const TabRef &T, int64_t g) {
  const int64_t i = 4 * g;
  const uint32_t k = uint32_t(a.k), mask = a.mask;
  Blk acc[4];
#pragma unroll
  for (int m = 0; m < 4; m++) acc[m] = Blk{{0, 0, 0, 0}};
  // makeBlock(i, m): low qword m, high qword i.
  const uint32_t ilo = uint32_t(uint64_t(i)), ihi = uint32_t(uint64_t(i) >> 32);
#pragma unroll
  for (int m = 0; m < D; m += 2) {
    uint32_t x[4] = {uint32_t(m), 0u, ilo, ihi};
    uint32_t y[4] = {uint32_t(m + 1), 0u, ilo, ihi};
    if (m + 1 < D) {
      aes_enc2(T, x, a.key, y, a.key);
    } else {
      aes_enc(T, x, a.key);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int word = 4 * m + q;  // compile-time after unrolling
      const Blk v = ldg_blk(a.kk + lpn_idx(x[q], mask, k));
      acc[word / D] = blk_xor(acc[word / D], v);
    }
    if (m + 1 < D) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int word = 4 * (m + 1) + q;
        const Blk v = ldg_blk(a.kk + lpn_idx(y[q], mask, k));
        acc[word / D] = blk_xor(acc[word / D], v);
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 4; m++) {
    Blk *p = a.e + (i - a.row_lo) + m;
    st_blk_cs(p, blk_xor(ld_blk(p), acc[m]));
  }
}

// Rows 4g..4g+3 for any d (1..32).
__device__ void lpn_group4_dyn(const LpnArgs &a, const TabRef &T, int64_t g) {
  const int64_t i = 4 * g;
  const uint32_t k = uint32_t(a.k), mask = a.mask;
  Blk acc[4] = {{{0, 0, 0, 0}}, {{0, 0, 0, 0}}, {{0, 0, 0, 0}}, {{0, 0, 0, 0}}};
  const uint32_t ilo = uint32_t(uint64_t(i)), ihi = uint32_t(uint64_t(i) >> 32);
  for (int m = 0; m < a.d; m++) {
    uint32_t x[4] = {uint32_t(m), 0u, ilo, ihi};
    aes_enc(T, x, a.key);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int word = 4 * m + q;
      const Blk v = ldg_blk(a.kk + lpn_idx(x[q], mask, k));
      const int row = word / a.d;
#pragma unroll
      for (int r = 0; r < 4; r++)
        if (r == row) acc[r] = blk_xor(acc[r], v);
    }
  }
#pragma unroll
  for (int m = 0; m < 4; m++) {
    Blk *p = a.e + (i - a.row_lo) + m;
    st_blk_cs(p, blk_xor(ld_blk(p), acc[m]));
  }
}

// One tail row (emp-ot __compute1, lpn_f2.h:61-70).
__device__ void lpn_row1(const LpnArgs &a, const TabRef &T, int64_t j) {
  const int nb = (a.d + 3) / 4;
  const uint32_t k = uint32_t(a.k);
  const uint32_t jlo = uint32_t(uint64_t(j)), jhi = uint32_t(uint64_t(j) >> 32);
  Blk acc{{0, 0, 0, 0}};
  int done = 0;
  for (int m = 0; m < nb; m++) {
    uint32_t x[4] = {uint32_t(m), 0u, jlo, jhi};
    aes_enc(T, x, a.key);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (done < a.d) acc = blk_xor(acc, ldg_blk(a.kk + (x[q] % k)));
      done++;
    }
  }
  Blk *p = a.e + (j - a.row_lo);
  st_blk(p, blk_xor(ld_blk(p), acc));
}

}  // namespace
}  // namespace cuot
