// sot_compat.cu -- the reference's SOT role classes (include/cuot_sot.h)
// over the C ABI: SOTSender / SOTRecver with seed_expand() and dual_lpn()
// as in silent/sender.cu and silent/recver.cu.
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cuot_sot.h"
#include "ctx.cuh"

namespace {

void sot_cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
  }
}
void sot_check(int st, const char *what) {
  if (st != CUOT_OK)
    throw std::runtime_error(std::string(what) + ": " + cuot_status_string(st) + " " + cuot_last_error());
}
uint64_t ilog2(uint64_t x) {
  uint64_t r = 0;
  while ((1ull << (r + 1)) <= x) r++;
  return r;
}

}  // namespace

blk *SOTSender::m0_h = nullptr;
blk *SOTSender::m1_h = nullptr;
blk *SOTRecver::mc_h = nullptr;

// silent/roles.h:33-38: depth = logOT - log2(nTree)
SOT::SOT(SilentConfig config) : mConfig(config) {
  if (config.nTree < 1 || (config.nTree & (config.nTree - 1)))
    throw std::runtime_error("SOT: nTree must be a power of two");
  if (config.gpuPerParty != 1 && config.gpuPerParty != 0)
    throw std::runtime_error("SOT: one GPU per party here (cuot_b200.shard splits an instance)");
  mDepth = uint64_t(config.logOT) - ilog2(config.nTree);
  numOT = 1ull << config.logOT;
  numLeaves = 1ull << mDepth;
  if (mDepth < 1) throw std::runtime_error("SOT: logOT must exceed log2(nTree)");
  if (!config.choiceBytes && config.nTree > 64)
    throw std::runtime_error("SOT: more than 64 trees need choiceBytes");
  sot_cuda_check(cudaSetDevice(config.id), "cudaSetDevice");
  sot_check(cuot_ctx_create(config.id, &ctx_), "cuot_ctx_create");
  m0.resize({mDepth + 1, mConfig.nTree});
  m1.resize({mDepth + 1, mConfig.nTree});
  sot_cuda_check(cudaMalloc(&a_d_, numOT / 8), "cudaMalloc a");
  sot_check(cuot_qc_gen_a(ctx_, reinterpret_cast<const uint8_t *>(mConfig.qcKey), numOT, a_d_, stream_),
            "cuot_qc_gen_a");
  sot_check(cuot_qc_plan_create(ctx_, a_d_, numOT, stream_, &plan_), "cuot_qc_plan_create");
  sync();
}

SOT::~SOT() {
  if (plan_) cuot_qc_plan_destroy(plan_);
  if (a_d_) cudaFree(a_d_);
  if (ctx_) cuot_ctx_destroy(ctx_);
}

void SOT::sync() { sot_cuda_check(cudaStreamSynchronize(static_cast<cudaStream_t>(stream_)), "sync"); }

// ---------------------------------------------------------------- sender
// sender.cu:12-47: delta and the tree roots (rows [0, nTree) of fullVector).
SOTSender::SOTSender(SilentConfig config) : SOT(config) {
  mRole = Sender;
  fullVector = new Mat({numOT, 1});
  std::vector<blk> init(mConfig.nTree + 1);
  cuot_block *tmp = nullptr;
  sot_cuda_check(cudaMalloc(&tmp, init.size() * sizeof(blk)), "cudaMalloc");
  sot_check(cuot_prg_fill(ctx_, reinterpret_cast<const uint8_t *>(mConfig.seed), 0, tmp, init.size(), stream_),
            "cuot_prg_fill");
  sot_cuda_check(cudaMemcpy(init.data(), tmp, init.size() * sizeof(blk), cudaMemcpyDeviceToHost), "D2H");
  cudaFree(tmp);
  delta_h = init[mConfig.nTree];
  sot_cuda_check(cudaMemcpy(fullVector->data(), init.data(), mConfig.nTree * sizeof(blk), cudaMemcpyHostToDevice),
                 "H2D roots");
  if (mConfig.id == 0 && !SOTSender::m0_h) {
    SOTSender::m0_h = new blk[(mDepth + 1) * mConfig.nTree]();
    SOTSender::m1_h = new blk[(mDepth + 1) * mConfig.nTree]();
  }
}

SOTSender::~SOTSender() {
  delete fullVector;
  if (mConfig.id == 0) {
    delete[] SOTSender::m0_h;
    delete[] SOTSender::m1_h;
    SOTSender::m0_h = SOTSender::m1_h = nullptr;
  }
}

// sender.cu:76-108: all levels in one launch; m0/m1 = masked level sums.
void SOTSender::seed_expand() {
  sot_cuda_check(cudaSetDevice(mConfig.id), "cudaSetDevice");
  const uint64_t t = mConfig.nTree, h = mDepth;
  Mat base0({h, t}), base1({h, t}), roots({t});
  sot_cuda_check(cudaMemcpy(base0.data(), SOTSender::m0_h, h * t * sizeof(blk), cudaMemcpyHostToDevice), "H2D m0");
  sot_cuda_check(cudaMemcpy(base1.data(), SOTSender::m1_h, h * t * sizeof(blk), cudaMemcpyHostToDevice), "H2D m1");
  sot_cuda_check(cudaMemcpy(roots.data(), fullVector->data(), t * sizeof(blk), cudaMemcpyDeviceToDevice), "roots");
  cuot_block d;
  std::memcpy(&d, &delta_h, sizeof(d));
  auto cb = [](const Mat &m) { return reinterpret_cast<cuot_block *>(m.data()); };
  sot_check(cuot_sot_pprf_sender(ctx_, cb(roots), t, int(h), &d, cb(base0), cb(base1), cb(*fullVector), cb(m0),
                                 cb(m1), stream_),
            "cuot_sot_pprf_sender");
  sync();
}

// sender.cu:110-119: transpose, exact QC encode of the 128 planes, transpose.
void SOTSender::dual_lpn() {
  sot_cuda_check(cudaSetDevice(mConfig.id), "cudaSetDevice");
  sot_check(cuot_qc_plan_dual_lpn(plan_, reinterpret_cast<cuot_block *>(fullVector->data()), stream_),
            "cuot_qc_plan_dual_lpn");
  sync();
}

// ---------------------------------------------------------------- receiver
// recver.cu:12-50: punctured positions from the choice bits and the choice
// vector c = a * e.
SOTRecver::SOTRecver(SilentConfig config) : SOT(config) {
  mRole = Recver;
  const uint64_t t = mConfig.nTree, h = mDepth;
  puncVector = new Mat({numOT, 1});
  std::vector<uint8_t> ch(h * t);
  for (uint64_t d = 0; d < h; d++)
    for (uint64_t j = 0; j < t; j++)
      ch[d * t + j] = mConfig.choiceBytes ? (mConfig.choiceBytes[d * t + j] & 1)
                                          : uint8_t((mConfig.choices[d] >> j) & 1);
  // recver.cu:77-86: id = sum over levels of (1 - choice) bits, from the top
  std::vector<uint64_t> pos(t);
  for (uint64_t j = 0; j < t; j++) {
    uint64_t id = 0;
    for (uint64_t d = 0; d < h; d++) id = 2 * id + (1 - ch[d * t + j]);
    pos[j] = id + j * numLeaves;
  }
  sot_cuda_check(cudaMalloc(&choice_d_, ch.size()), "cudaMalloc choices");
  sot_cuda_check(cudaMemcpy(choice_d_, ch.data(), ch.size(), cudaMemcpyHostToDevice), "H2D choices");
  sot_cuda_check(cudaMalloc(&puncPos, t * sizeof(uint64_t)), "cudaMalloc puncPos");
  sot_cuda_check(cudaMemcpy(puncPos, pos.data(), t * sizeof(uint64_t), cudaMemcpyHostToDevice), "H2D puncPos");
  choiceVector.resize({numOT / 128});
  sot_check(cuot_qc_encode_sparse(ctx_, a_d_, puncPos, int(t), numOT,
                                  reinterpret_cast<uint64_t *>(choiceVector.data()), stream_),
            "cuot_qc_encode_sparse");
  sync();
  if (mConfig.id == 0 && !SOTRecver::mc_h) SOTRecver::mc_h = new blk[h * t]();
}

SOTRecver::~SOTRecver() {
  delete puncVector;
  if (puncPos) cudaFree(puncPos);
  if (choice_d_) cudaFree(choice_d_);
  if (mConfig.id == 0) {
    delete[] SOTRecver::mc_h;
    SOTRecver::mc_h = nullptr;
  }
}

void SOTRecver::get_punc_key() {
  if (!other) throw std::runtime_error("SOTRecver::get_punc_key: no sender");
  m0 = other->m0;
  m1 = other->m1;
}

// recver.cu:124-163
void SOTRecver::seed_expand() {
  sot_cuda_check(cudaSetDevice(mConfig.id), "cudaSetDevice");
  const uint64_t t = mConfig.nTree, h = mDepth;
  Mat mc({h, t});
  sot_cuda_check(cudaMemcpy(mc.data(), SOTRecver::mc_h, h * t * sizeof(blk), cudaMemcpyHostToDevice), "H2D mc");
  auto cb = [](const Mat &m) { return reinterpret_cast<cuot_block *>(m.data()); };
  sot_check(cuot_sot_pprf_recver(ctx_, cb(m0), cb(m1), cb(mc), choice_d_, t, int(h), cb(*puncVector), stream_),
            "cuot_sot_pprf_recver");
  sync();
}

// recver.cu:168-174
void SOTRecver::dual_lpn() {
  sot_cuda_check(cudaSetDevice(mConfig.id), "cudaSetDevice");
  sot_check(cuot_qc_plan_dual_lpn(plan_, reinterpret_cast<cuot_block *>(puncVector->data()), stream_),
            "cuot_qc_plan_dual_lpn");
  sync();
}
