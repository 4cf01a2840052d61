// test_sot.cpp -- drives the SOT role adapter (include/cuot_sot.h) the way a
// caller of cuOT's silent/ classes does (construct sender and receiver, fill
// the base-OT arrays, seed_expand, dual_lpn) and checks the outputs against
// the CPU oracle and against the COT correlation w = v ^ c * delta.
// Built and run by tests/test_gpu_sot_adapter.py.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "cuot_oracle.h"
#include "cuot_sot.h"

static int fails = 0;
#define CHECK(c, msg)                                      \
  do {                                                     \
    if (!(c)) { std::printf("FAIL: %s\n", msg); fails++; } \
  } while (0)

template <typename T>
static std::vector<T> d2h(const void *p, size_t n) {
  std::vector<T> v(n);
  cudaMemcpy(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost);
  return v;
}

static void run(int logOT, uint64_t nTree, bool bytes, bool with_oracle, uint64_t seed) {
  std::mt19937_64 rng(seed);
  SilentConfig cfg{};
  cfg.id = 0;
  cfg.logOT = logOT;
  cfg.nTree = nTree;
  cfg.baseOT = SimplestOT_t;
  cfg.pprf = Aes_t;
  cfg.dualLPN = QuasiCyclic_t;
  cfg.gpuPerParty = 1;
  for (int i = 0; i < 4; i++) {
    cfg.qcKey[i] = uint32_t(rng());
    cfg.seed[i] = uint32_t(rng());
  }
  uint64_t depth = uint64_t(logOT);
  for (uint64_t x = nTree; x > 1; x >>= 1) depth--;
  std::vector<uint64_t> masks(depth);
  std::vector<uint8_t> chb(depth * nTree);
  for (uint64_t d = 0; d < depth; d++) {
    masks[d] = rng();
    for (uint64_t j = 0; j < nTree; j++) chb[d * nTree + j] = bytes ? uint8_t(rng() & 1) : uint8_t((masks[d] >> j) & 1);
  }
  if (bytes) cfg.choiceBytes = chb.data();
  else cfg.choices = masks.data();

  SOTSender s(cfg);
  SOTRecver r(cfg);
  r.other = &s;
  const uint64_t n = s.numOT, t = nTree;
  // base OT (host protocol; here an ideal one): sender messages, chosen ones
  for (uint64_t i = 0; i < depth * t; i++) {
    for (int w = 0; w < 4; w++) {
      SOTSender::m0_h[i].data[w] = uint32_t(rng());
      SOTSender::m1_h[i].data[w] = uint32_t(rng());
    }
    SOTRecver::mc_h[i] = chb[i] ? SOTSender::m1_h[i] : SOTSender::m0_h[i];
  }
  std::vector<blk> roots = d2h<blk>(s.fullVector->data(), t);
  s.seed_expand();
  r.get_punc_key();
  r.seed_expand();
  std::vector<blk> v_exp = d2h<blk>(s.fullVector->data(), n);
  std::vector<blk> w_exp = d2h<blk>(r.puncVector->data(), n);
  if (with_oracle) {
    std::vector<or_block> lv(n), om0((depth + 1) * t), om1((depth + 1) * t), rl(n), mc(depth * t);
    or_block dl;
    std::memcpy(&dl, &s.delta_h, 16);
    or_sot_pprf_sender(reinterpret_cast<const or_block *>(roots.data()), int64_t(t), int(depth), dl,
                       reinterpret_cast<const or_block *>(SOTSender::m0_h),
                       reinterpret_cast<const or_block *>(SOTSender::m1_h), lv.data(), om0.data(), om1.data(), 8);
    CHECK(std::memcmp(lv.data(), v_exp.data(), n * 16) == 0, "sender leaves vs oracle");
    CHECK(std::memcmp(om0.data(), d2h<blk>(s.m0.data(), (depth + 1) * t).data(), (depth + 1) * t * 16) == 0,
          "sender m0 vs oracle");
    std::memcpy(mc.data(), SOTRecver::mc_h, depth * t * 16);
    or_sot_pprf_recver(om0.data(), om1.data(), mc.data(), chb.data(), int64_t(t), int(depth), rl.data(), 8);
    CHECK(std::memcmp(rl.data(), w_exp.data(), n * 16) == 0, "receiver leaves vs oracle");
  }
  s.dual_lpn();
  r.dual_lpn();
  std::vector<blk> v = d2h<blk>(s.fullVector->data(), n);
  std::vector<blk> w = d2h<blk>(r.puncVector->data(), n);
  std::vector<uint64_t> c = d2h<uint64_t>(r.choiceVector.data(), n / 64);
  if (with_oracle) {
    std::vector<uint64_t> a(n / 64);
    or_qc_gen_a(reinterpret_cast<const uint8_t *>(cfg.qcKey), n, a.data());
    std::vector<or_block> io(n);
    std::memcpy(io.data(), v_exp.data(), n * 16);
    or_sot_dual_lpn(a.data(), io.data(), n, 8);
    CHECK(std::memcmp(io.data(), v.data(), n * 16) == 0, "sender dual LPN vs oracle");
  }
  uint64_t bad = 0, ones = 0;
  for (uint64_t i = 0; i < n; i++) {
    const bool ci = (c[i / 64] >> (i % 64)) & 1;
    ones += ci;
    for (int k = 0; k < 4; k++)
      if ((v[i].data[k] ^ w[i].data[k]) != (ci ? s.delta_h.data[k] : 0u)) bad++;
  }
  CHECK(bad == 0, "COT correlation w = v ^ c * delta");
  CHECK(ones > n / 3 && ones < 2 * n / 3, "choice vector balance");
  std::printf("logOT=%d nTree=%llu %s: %llu correlation mismatches\n", logOT, (unsigned long long)nTree,
              bytes ? "byte choices" : "64-bit masks", (unsigned long long)bad);
}

int main() {
  try {
    run(16, 16, false, true, 1);     // the reference's choice masks
    run(14, 64, false, true, 2);
    run(17, 256, true, false, 3);    // beyond the reference's 64-tree limit
  } catch (const std::exception &e) {
    std::printf("FAIL: exception %s\n", e.what());
    fails++;
  }
  std::printf(fails ? "FAILED %d\n" : "PASS\n", fails);
  return fails ? 1 : 0;
}
