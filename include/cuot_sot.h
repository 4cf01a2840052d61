// cuot_sot.h -- C++ adapter with the reference's SOT role interface
// (silent/roles.h:15-85: SilentConfig, SOT, SOTSender, SOTRecver), implemented
// on top of the C ABI in cuot.h.  A caller written against cuOT's silent/
// classes constructs the same objects, fills the same static base-OT arrays
// and calls seed_expand() / dual_lpn(); the outputs stay in the same Mat
// members (fullVector, puncVector, choiceVector).
//
// Differences from the reference, all by design:
//  * semantics are emp-ot's (the GGM node is TwoKeyPRP with fixed keys, so
//    leftKey/rightKey are accepted and unused; the QC encode is the exact
//    GF(2) product instead of the float cuFFT path);
//  * base_ot() is host protocol and stays with the caller: it fills
//    SOTSender::m0_h / m1_h and SOTRecver::mc_h ([depth][nTree] blocks), as
//    the reference's base_ot() does (sender.cu:60-72, recver.cu:63-75);
//  * delta, the tree roots and the QC polynomial come from `seed` and
//    `qcKey` (the reference draws them with rand(); both parties must agree
//    on qcKey);
//  * nTree is not limited to 64: `choiceBytes` ([depth][nTree] bytes) may be
//    given instead of the 64-bit masks `choices`;
//  * one GPU per instance (gpuPerParty = 1); cuot_b200.shard splits one
//    instance over several GPUs.
// Calls block until their device work is done, like the reference.  Errors
// throw std::runtime_error.
#pragma once
#include <cstdint>

#include "cuot.h"
#include "cuot_dev_layer.h"

enum BaseOTType { SimplestOT_t };
enum PprfType { Aes_t };
enum LPNType { QuasiCyclic_t, PrimalLpn_t };

struct SilentConfig {
  int id, logOT;
  uint64_t nTree;
  BaseOTType baseOT;
  PprfType pprf;
  uint32_t leftKey[4];
  uint32_t rightKey[4];
  LPNType dualLPN;
  uint64_t *choices;           // [depth]: bit t = tree t's choice bit at that level
  int gpuPerParty;
  // extensions (zero-initialised by the reference's aggregate initialisers)
  uint32_t qcKey[4];           // key of the QC polynomial a (both parties)
  uint32_t seed[4];            // sender: delta and roots
  const uint8_t *choiceBytes;  // [depth][nTree]; used instead of `choices` when set
};

class SOT {
 public:
  Role mRole;
  SilentConfig mConfig;
  uint64_t mDepth, numOT, numLeaves;
  Mat m0, m1;  // [depth + 1][nTree] masked level sums (sender output, receiver input)

  explicit SOT(SilentConfig config);
  virtual ~SOT();
  virtual void seed_expand() = 0;
  virtual void dual_lpn() = 0;

 protected:
  cuot_ctx *ctx_ = nullptr;
  uint64_t *a_d_ = nullptr;        // QC polynomial, numOT bits
  cuot_qc_plan *plan_ = nullptr;   // its transform
  void *stream_ = nullptr;
  void sync();
};

class SOTSender : public SOT {
 public:
  Mat *fullVector;   // numOT blocks: roots in rows [0, nTree) before seed_expand, then v
  blk delta_h;
  static blk *m0_h, *m1_h;  // [depth][nTree] base-OT sender messages (caller-filled)

  explicit SOTSender(SilentConfig config);
  ~SOTSender() override;
  void seed_expand() override;
  void dual_lpn() override;
};

class SOTRecver : public SOT {
 public:
  Mat *puncVector;      // numOT blocks: w after seed_expand / dual_lpn
  Mat choiceVector;     // numOT bits: c = a * e (encode_sparse of the punctured positions)
  uint64_t *puncPos;    // device, [nTree] punctured leaf index of each tree
  SOTSender *other = nullptr;
  static blk *mc_h;     // [depth][nTree] chosen base-OT messages (caller-filled)

  explicit SOTRecver(SilentConfig config);
  ~SOTRecver() override;
  void get_punc_key();  // m0, m1 = the sender's (recver.cu:118-122)
  void seed_expand() override;
  void dual_lpn() override;

 private:
  uint8_t *choice_d_ = nullptr;  // [depth][nTree] bytes
};
