// test_bitslice_host.cu -- host-side check of the bitsliced AES core
// (cuot_b200/csrc/aes_bitslice.cuh, whose functions are __host__
// __device__): 32 random blocks under random keys, encrypted bitsliced on the
// CPU, against the oracle's AES-128 (FIPS-197).  Needs no GPU; built with nvcc
// and run by tests/test_bitslice.py.
#include <cstdio>
#include <cstring>
#include <random>

#include "aes_bitslice.cuh"
#include "cuot_oracle.h"

int main() {
  std::mt19937_64 rng(7);
  int fails = 0;
  for (int trial = 0; trial < 20; trial++) {
    uint8_t key[16], rk[176], in[32][16], ref[32][16];
    for (auto &b : key) b = uint8_t(rng());
    for (auto &blk : in)
      for (auto &b : blk) b = uint8_t(rng());
    or_aes128_key_expand(key, rk);
    or_aes128_encrypt(rk, &in[0][0], &ref[0][0], 32);
    uint32_t w44[44];
    std::memcpy(w44, rk, 176);  // little-endian words of the FIPS schedule
    cuot::BitslicedKey bk;
    cuot::bitsliced_key(w44, &bk);
    uint32_t words[4][32], s[128];
    for (int b = 0; b < 32; b++)
      for (int w = 0; w < 4; w++) std::memcpy(&words[w][b], &in[b][4 * w], 4);
    cuot::bs_from_words(words, s);
    cuot::bs_encrypt(s, bk);
    cuot::bs_to_words(s, words);
    for (int b = 0; b < 32; b++) {
      uint8_t out[16];
      for (int w = 0; w < 4; w++) std::memcpy(&out[4 * w], &words[w][b], 4);
      if (std::memcmp(out, ref[b], 16)) fails++;
    }
  }
  std::printf(fails ? "FAIL %d blocks\n" : "PASS\n", fails);
  return fails ? 1 : 0;
}
