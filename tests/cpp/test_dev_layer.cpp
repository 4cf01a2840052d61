// test_dev_layer.cpp -- drives the reference-signature adapter
// (include/cuot_dev_layer.h) the way emp-ot's callers do (MpcotReg::
// exec_parallel_sender/recver, mpcot_reg.h:130-157; LpnF2::compute,
// lpn_f2.h:81-87) and checks every output bit-exact against the CPU oracle.
// Built and run by tests/test_gpu_dev_layer.py.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "cuot_dev_layer.h"
#include "cuot_oracle.h"

static int fails = 0;
#define CHECK(c, msg)                                   \
  do {                                                  \
    if (!(c)) { std::printf("FAIL: %s\n", msg); fails++; } \
  } while (0)

int main() {
  const int t = 37, depth = 9, k = 3001;
  const uint64_t n = uint64_t(t) << depth;
  std::mt19937_64 rng(42);
  auto rnd_blocks = [&](size_t m) {
    std::vector<blk> v(m);
    for (auto &b : v)
      for (auto &w : b.data) w = uint32_t(rng());
    return v;
  };
  // FerretCOT owns expSeed, MpcotReg owns buffer/separated (ferret_cot.hpp:21,
  // mpcot_reg.h:55-61); the roots sit in the first t blocks of expSeed.
  Mat expanded({n}), buffer({n}), sep({n});
  std::vector<blk> roots = rnd_blocks(t);
  cudaMemcpy(expanded.data(), roots.data(), t * 16, cudaMemcpyHostToDevice);
  blk delta = rnd_blocks(1)[0];
  delta.data[0] |= 1;
  std::vector<blk> m0(t * depth), m1(t * depth), ss(t);
  int tt[1] = {t};
  cuda_mpcot_sender(&expanded, &buffer, &sep, m0.data(), m1.data(), ss.data(), tt, depth, &delta, 1);
  std::vector<blk> leaves(n);
  cudaMemcpy(leaves.data(), expanded.data(), n * 16, cudaMemcpyDeviceToHost);

  std::vector<or_block> oleaves(n), olsum(t * depth), orsum(t * depth), oss(t);
  or_block od;
  std::memcpy(&od, &delta, 16);
  or_ferret_pprf_sender(reinterpret_cast<or_block *>(roots.data()), t, depth, od, oleaves.data(),
                        olsum.data(), orsum.data(), oss.data(), 4);
  CHECK(!std::memcmp(leaves.data(), oleaves.data(), n * 16), "sender leaves");
  CHECK(!std::memcmp(m0.data(), olsum.data(), t * depth * 16), "lSum");
  CHECK(!std::memcmp(m1.data(), orsum.data(), t * depth * 16), "rSum");
  CHECK(!std::memcmp(ss.data(), oss.data(), t * 16), "secret_sum");

  // Receiver: choices [tree][depth], chosen messages from the OT.
  std::vector<uint8_t> ch(t * depth);
  std::vector<blk> mc(t * depth);
  for (int i = 0; i < t * depth; i++) {
    ch[i] = rng() & 1;
    mc[i] = ch[i] ? m1[i] : m0[i];
  }
  std::vector<bool> unused;
  bool *choices = new bool[t * depth];
  for (int i = 0; i < t * depth; i++) choices[i] = ch[i] != 0;
  Mat rexp({n}), rbuf({n}), rsep({n});
  cuda_mpcot_recver(&rexp, &rbuf, &rsep, mc.data(), ss.data(), tt, depth, choices, 1);
  std::vector<blk> rl(n);
  cudaMemcpy(rl.data(), rexp.data(), n * 16, cudaMemcpyDeviceToHost);
  std::vector<or_block> orl(n);
  or_ferret_pprf_recver(reinterpret_cast<or_block *>(mc.data()), ch.data(), oss.data(), t, depth, orl.data(), 4);
  CHECK(!std::memcmp(rl.data(), orl.data(), n * 16), "receiver leaves");
  delete[] choices;

  // LPN on the sender's leaves: key = emp AES_KEY round keys (first 16 bytes = seed).
  std::vector<blk> kk = rnd_blocks(k);
  uint32_t key[44] = {0};
  for (int i = 0; i < 4; i++) key[i] = uint32_t(rng());
  Mat pub, kk_d[1];
  int64_t nn_rows[1] = {int64_t(n)};
  std::vector<blk> nn(n);
  cuda_primal_lpn(Sender, &pub, 10, nn_rows, k, key, &expanded, nn.data(), kk_d, kk.data(), 1);
  or_lpn_primal(reinterpret_cast<const uint8_t *>(key), reinterpret_cast<or_block *>(kk.data()), k, 10,
                oleaves.data(), int64_t(n), 4);
  CHECK(!std::memcmp(nn.data(), oleaves.data(), n * 16), "lpn output");

  std::printf(fails ? "FAILED (%d)\n" : "PASS\n", fails);
  return fails ? 1 : 0;
}
