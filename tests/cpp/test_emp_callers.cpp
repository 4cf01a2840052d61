// test_emp_callers.cpp -- the drop-in check for the Ferret boundary.
//
// Compiles the reference's OWN emp-ot callers, unchanged from the reference
// tree, against include/cuot_dev_layer.h and links libcuot.so in place of
// cuOT's gpu/ library:
//   ferret/emp-ot/emp-ot/ferret/mpcot_reg.h  MpcotReg::mpcot ->
//       mpcot_init_sender/recver, exec_parallel_sender/recver ->
//       cuda_mpcot_sender / cuda_mpcot_recver   (mpcot_reg.h:80-157)
//   ferret/emp-ot/emp-ot/ferret/preot.h      OTPre (the OT of the level sums)
//   ferret/emp-ot/emp-ot/ferret/lpn_f2.h     LpnF2::compute -> seed_gen ->
//       cuda_primal_lpn with the PRP's expanded AES schedule (lpn_f2.h:81-87)
// over the emp-tool shim (oracle/emp_shim).  Both parties run in this process
// and talk through an in-memory channel, with dealer-made pre-COTs, as
// FerretCOT::extend drives them (ferret_cot.hpp:80-103).  The GPU outputs are
// then checked against the same reference headers' CPU code: SPCOT_Sender /
// SPCOT_Recver::compute per tree and LpnF2::task over [0, n).
//
// Built by oracle/build_ref.sh (it needs the reference tree) into
// oracle/_ref/test_emp_callers, run by tests/test_gpu_emp_callers.py.
#include "emp-tool/emp-tool.h"
#include "emp-ot/ferret/mpcot_reg.h"
#include "emp-ot/ferret/lpn_f2.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <deque>

namespace {

int fails = 0;
#define CHECK(c, ...)                         \
  do {                                        \
    if (!(c)) {                               \
      std::printf("FAIL: " __VA_ARGS__);      \
      std::printf("\n");                      \
      fails++;                                \
    }                                         \
  } while (0)

// A byte channel: one party writes everything before the other reads.
class MemIO {
 public:
  void send_data(const void *p, int n) {
    const uint8_t *b = static_cast<const uint8_t *>(p);
    q_.insert(q_.end(), b, b + n);
  }
  void recv_data(void *p, int n) {
    if (int(q_.size()) < n) {
      std::printf("FAIL: channel underflow\n");
      std::exit(1);
    }
    uint8_t *b = static_cast<uint8_t *>(p);
    for (int i = 0; i < n; i++) {
      b[i] = q_.front();
      q_.pop_front();
    }
  }
  void send_block(const block *p, int n) { send_data(p, n * int(sizeof(block))); }
  void recv_block(block *p, int n) { recv_data(p, n * int(sizeof(block))); }
  void flush() {}
  size_t pending() const { return q_.size(); }

 private:
  std::deque<uint8_t> q_;
};

std::vector<block> download(const Mat &m, uint64_t n) {
  std::vector<block> v(n);
  cudaMemcpy(v.data(), m.data(), n * sizeof(block), cudaMemcpyDeviceToHost);
  return v;
}

bool same(const block &a, const block &b) { return std::memcmp(&a, &b, sizeof(block)) == 0; }

int run(int t, int h, int k) {
  const int64_t n = int64_t(t) << h;
  PRG prg;
  MemIO io;
  block delta;
  prg.random_block(&delta, 1);
  delta = (delta & makeBlock(~0ULL, ~1ULL)) ^ makeBlock(0, 1);  // ferret_cot.hpp:27-31

  // Dealer pre-COTs for the t*h level OTs: sender s_i (LSB 0), receiver
  // r_i = s_i ^ b_i * delta, so LSB(r_i) = b_i is the receiver's choice.
  const int npre = t * h;
  std::vector<block> pre_s(npre), pre_r(npre);
  prg.random_block(pre_s.data(), npre);
  for (int i = 0; i < npre; i++) {
    pre_s[i] = pre_s[i] & makeBlock(~0ULL, ~1ULL);
    bool b = false;
    prg.random_bool(&b, 1);
    pre_r[i] = b ? (pre_s[i] ^ delta) : pre_s[i];
  }
  OTPre<MemIO> ot_s(&io, h, t), ot_r(&io, h, t);
  ot_s.send_pre(pre_s.data(), delta);
  ot_r.recv_pre(pre_r.data());

  int tt[1] = {t};
  int64_t rows[1] = {n};
  MpcotReg<MemIO> mp_s(ALICE, 1, int(n), tt, h, &io), mp_r(BOB, 1, int(n), tt, h, &io);
  // FerretCOT owns the MPCOT outputs (expSeed, ferret_cot.hpp:19-22); the
  // adapter takes the tree roots from their first t blocks.
  Mat exp_s({uint64_t(n)}), exp_r({uint64_t(n)});
  std::vector<block> roots(t);
  prg.random_block(roots.data(), t);
  cudaMemcpy(exp_s.data(), roots.data(), t * sizeof(block), cudaMemcpyHostToDevice);

  // MpcotReg::mpcot's own steps (mpcot_reg.h:80-106).  The receiver's choice
  // array is filled here, tree after tree, from its pre-COT bits:
  // mpcot_init_recver (mpcot_reg.h:116-128) passes the same `choice` pointer
  // to OTPre::choices_recver for every tree, so only choice[0..h) is ever
  // written and the rest of the array stays uninitialised.
  mp_s.sender_init(delta);
  mp_s.mpcot_init_sender(&ot_s);
  mp_s.exec_parallel_sender(&ot_s, &exp_s);
  mp_r.recver_init();
  std::vector<uint8_t> choice_bytes(size_t(t) * h);
  bool *choice = reinterpret_cast<bool *>(choice_bytes.data());
  for (int i = 0; i < t; i++) ot_r.choices_recver(choice + size_t(i) * h);
  ot_r.reset();
  mp_r.exec_parallel_recver(&ot_r, &exp_r, choice);
  CHECK(io.pending() == 0, "MPCOT left %zu bytes in the channel", io.pending());

  std::vector<block> ls = download(exp_s, n), lr = download(exp_r, n);
  // The reference's CPU SPCOT per tree: the GPU sender's leaves, and the
  // receiver's reconstruction from the messages its OT choices select.
  int bad_s = 0, bad_r = 0, bad_cot = 0;
  for (int i = 0; i < t; i++) {
    SPCOT_Sender<MemIO> s(&io, h + 1);
    s.seed = roots[i];
    std::vector<block> tree(size_t(1) << h);
    s.compute(tree.data(), delta);
    for (int j = 0; j < (1 << h); j++) bad_s += !same(tree[j], ls[(size_t(i) << h) + j]);

    SPCOT_Recver<MemIO> r(&io, h + 1);
    for (int l = 0; l < h; l++) {
      r.b[l] = ot_r.bits[i * h + l];
      r.m[l] = r.b[l] ? s.m[h + l] : s.m[l];
    }
    r.secret_sum_f2 = s.secret_sum_f2;
    const int pos = r.get_index();
    std::vector<block> rtree((size_t(1) << h) + 4);
    r.compute(rtree.data());
    for (int j = 0; j < (1 << h); j++) {
      bad_r += !same(rtree[j], lr[(size_t(i) << h) + j]);
      block d = ls[(size_t(i) << h) + j] ^ lr[(size_t(i) << h) + j];
      bad_cot += !same(d, j == pos ? delta : zero_block);
    }
  }
  CHECK(bad_s == 0, "%d sender leaves differ from SPCOT_Sender::compute", bad_s);
  CHECK(bad_r == 0, "%d receiver leaves differ from SPCOT_Recver::compute", bad_r);
  CHECK(bad_cot == 0, "%d leaves break the COT correlation", bad_cot);

  // Primal LPN through LpnF2::compute (seed sent ALICE -> BOB, key = the
  // PRP's round keys), both roles, against LpnF2::task on the CPU.
  std::vector<block> kk_s(k), kk_r(k), nn_s(n), nn_r(n);
  prg.random_block(kk_s.data(), k);
  for (int i = 0; i < k; i++) {
    bool b = false;
    prg.random_bool(&b, 1);
    kk_r[i] = b ? (kk_s[i] ^ delta) : kk_s[i];
  }
  LpnF2<MemIO, 10> lpn_s(ALICE, rows, k, &io, 1), lpn_r(BOB, rows, k, &io, 1);
  lpn_s.compute(nn_s.data(), &exp_s, kk_s.data());
  lpn_r.compute(nn_r.data(), &exp_r, kk_r.data());
  CHECK(same(lpn_s.seed, lpn_r.seed), "the receiver did not get the sender's LPN seed");
  std::vector<block> cpu_s = ls, cpu_r = lr;
  lpn_s.task(cpu_s.data(), kk_s.data(), 0, n);
  lpn_r.task(cpu_r.data(), kk_r.data(), 0, n);
  int bad_ls = 0, bad_lr = 0;
  for (int64_t i = 0; i < n; i++) {
    bad_ls += !same(cpu_s[i], nn_s[i]);
    bad_lr += !same(cpu_r[i], nn_r[i]);
  }
  CHECK(bad_ls == 0, "%d sender LPN rows differ from LpnF2::task", bad_ls);
  CHECK(bad_lr == 0, "%d receiver LPN rows differ from LpnF2::task", bad_lr);
  std::printf("t=%d h=%d k=%d n=%lld: sender/receiver MPCOT and LPN checked\n", t, h, k, (long long)n);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  int dev = 0;
  if (cudaGetDeviceCount(&dev) != cudaSuccess || dev < 1) {
    std::printf("SKIP: no CUDA device\n");
    return 0;
  }
  run(64, 10, 8192);    // the reference's CPU-runnable configuration
  run(37, 9, 3001);     // ragged t and k
  run(20, 13, 452000);  // 20 trees of ferret_b13's depth and k
  if (fails) {
    std::printf("%d checks failed\n", fails);
    return 1;
  }
  std::printf("PASS\n");
  return 0;
}
