// aes_bitslice.cuh -- bitsliced AES-128 encryption of 32 blocks at once, in
// registers (no table lookups): the alternative to the shared-memory T-table
// AES of common.cuh, kept so the two can be measured against each other on
// the same GPU (cuot_aes128_ecb vs cuot_aes128_ecb_bitsliced).
//
// State: s[8p + j] holds bit j of state byte p (p = r + 4c in FIPS-197
// order, i.e. byte p of the block in memory) of 32 blocks, block b in bit b.
// SubBytes is the generated GF(2) circuit of bitslice_sbox.cuh, ShiftRows a
// renaming of byte positions, MixColumns XORs and bitsliced xtime, and
// AddRoundKey an XOR with masks that are all-ones where the round key's bit
// is set.  The functions are __host__ __device__ so the host can check them.
#pragma once
#include <stdint.h>

#include "bitslice_sbox.cuh"

namespace cuot {

// 32x32 bit-matrix transpose in place (H. S. Warren, Hacker's Delight,
// 2nd ed., 7-3): afterwards bit j of a[i] is the old bit i of a[j].
__host__ __device__ __forceinline__ void transpose32(uint32_t (&a)[32]) {
  uint32_t m = 0x0000FFFFu;
#pragma unroll
  for (int j = 16; j != 0; j >>= 1, m ^= (m << j)) {
#pragma unroll
    for (int k = 0; k < 32; k = (k + j + 1) & ~j) {
      const uint32_t t = ((a[k] >> j) ^ a[k + j]) & m;
      a[k + j] ^= t;
      a[k] ^= t << j;
    }
  }
}

// Round-key masks of an expanded AES-128 key: m[r][8p + j] = ~0 if bit j of
// byte p of round key r is set, else 0.
struct BitslicedKey {
  uint32_t m[11][128];
};

// rk: the 44 little-endian words of the FIPS-197 key schedule.
__host__ inline void bitsliced_key(const uint32_t rk[44], BitslicedKey *out) {
  for (int r = 0; r < 11; r++)
    for (int p = 0; p < 16; p++) {
      const uint32_t byte = (rk[4 * r + p / 4] >> (8 * (p % 4))) & 0xffu;
      for (int j = 0; j < 8; j++) out->m[r][8 * p + j] = ((byte >> j) & 1u) ? 0xffffffffu : 0u;
    }
}

__host__ __device__ __forceinline__ void bs_add_key(uint32_t (&s)[128], const uint32_t *m) {
#pragma unroll
  for (int i = 0; i < 128; i++) s[i] ^= m[i];
}

__host__ __device__ __forceinline__ void bs_sub_bytes(uint32_t (&s)[128]) {
#pragma unroll
  for (int p = 0; p < 16; p++) {
    uint32_t x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = s[8 * p + j];
    sbox_bitsliced(x);
#pragma unroll
    for (int j = 0; j < 8; j++) s[8 * p + j] = x[j];
  }
}

// ShiftRows: new byte (r, c) = old byte (r, c + r mod 4).
__host__ __device__ __forceinline__ void bs_shift_rows(uint32_t (&s)[128]) {
  uint32_t t[128];
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int j = 0; j < 8; j++) t[8 * (r + 4 * c) + j] = s[8 * (r + 4 * ((c + r) & 3)) + j];
#pragma unroll
  for (int i = 0; i < 128; i++) s[i] = t[i];
}

// MixColumns: out_r = 2 (a_r ^ a_{r+1}) ^ a_{r+1} ^ a_{r+2} ^ a_{r+3}
//                   = xtime(a_r ^ a_{r+1}) ^ (a_0 ^ a_1 ^ a_2 ^ a_3) ^ a_r.
__host__ __device__ __forceinline__ void bs_mix_columns(uint32_t (&s)[128]) {
#pragma unroll
  for (int c = 0; c < 4; c++) {
    uint32_t a[4][8], tot[8];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int j = 0; j < 8; j++) a[r][j] = s[8 * (r + 4 * c) + j];
#pragma unroll
    for (int j = 0; j < 8; j++) tot[j] = a[0][j] ^ a[1][j] ^ a[2][j] ^ a[3][j];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      uint32_t t[8];
#pragma unroll
      for (int j = 0; j < 8; j++) t[j] = a[r][j] ^ a[(r + 1) & 3][j];
      // xtime: multiply by X modulo X^8 + X^4 + X^3 + X + 1
      const uint32_t x[8] = {t[7], t[0] ^ t[7], t[1], t[2] ^ t[7], t[3] ^ t[7], t[4], t[5], t[6]};
#pragma unroll
      for (int j = 0; j < 8; j++) s[8 * (r + 4 * c) + j] = x[j] ^ tot[j] ^ a[r][j];
    }
  }
}

// Encrypts the 32 blocks of the bitsliced state in place under `k`.
__host__ __device__ __forceinline__ void bs_encrypt(uint32_t (&s)[128], const BitslicedKey &k) {
  bs_add_key(s, k.m[0]);
#pragma unroll 1
  for (int r = 1; r < 10; r++) {
    bs_sub_bytes(s);
    bs_shift_rows(s);
    bs_mix_columns(s);
    bs_add_key(s, k.m[r]);
  }
  bs_sub_bytes(s);
  bs_shift_rows(s);
  bs_add_key(s, k.m[10]);
}

// words[w][b] = word w of block b  <->  s[32 w + k] (bit b = block b).
__host__ __device__ __forceinline__ void bs_from_words(uint32_t (&words)[4][32], uint32_t (&s)[128]) {
#pragma unroll
  for (int w = 0; w < 4; w++) {
    transpose32(words[w]);
#pragma unroll
    for (int k = 0; k < 32; k++) s[32 * w + k] = words[w][k];
  }
}
__host__ __device__ __forceinline__ void bs_to_words(uint32_t (&s)[128], uint32_t (&words)[4][32]) {
#pragma unroll
  for (int w = 0; w < 4; w++) {
#pragma unroll
    for (int k = 0; k < 32; k++) words[w][k] = s[32 * w + k];
    transpose32(words[w]);
  }
}

}  // namespace cuot
