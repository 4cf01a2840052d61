// cuot_dev_layer.h -- C++ adapter with the reference's own GPU operator
// signatures (ferret/emp-ot/emp-ot/ferret/dev_layer.h:9-18), implemented on
// top of the C ABI in cuot.h.  emp-ot's callers (MpcotReg::exec_parallel_*,
// mpcot_reg.h:130-157; LpnF2::compute, lpn_f2.h:81-87; FerretCOT,
// ferret_cot.hpp:13-22) compile against this header and link libcuot.so in
// place of cuOT's gpu/ library.
//
// Semantics are emp-ot's CPU semantics (SPCOT_Sender/SPCOT_Recver,
// LpnF2::task over [0, n)), which is what cuOT's GPU path is meant to compute.
// Like the reference these calls are blocking: they return once the host
// outputs are written.  Failures throw std::runtime_error (the reference's Mat
// throws on allocation failure, gpu/gpu_data.cu:11-14).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "cuot.h"

// Types of gpu/gpu_define.h:10-16.
enum Role { Sender, Recver };
struct OTblock { uint32_t data[4]; };
using blk = OTblock;

// Device matrix of blocks: the subset of cuOT's Mat (gpu/gpu_matrix.h:9-40,
// gpu/gpu_data.h) that the Ferret callers use.  Memory is on the device that
// was current when the storage was (re)allocated.
class Mat {
 public:
  Mat() = default;
  explicit Mat(std::vector<uint64_t> dim);
  Mat(const Mat &other);
  ~Mat();
  Mat &operator=(const Mat &other);
  blk *data() const { return ptr_; }
  blk *data(std::vector<uint64_t> pos) const;
  uint64_t size() const;
  uint64_t size_bytes() const { return size() * sizeof(blk); }
  uint64_t dim(uint32_t i) const { return dim_.at(i); }
  std::vector<uint64_t> dims() const { return dim_; }
  // Keeps the first min(old, new) blocks.
  void resize(std::vector<uint64_t> dim);
  void clear();

 private:
  blk *ptr_ = nullptr;
  uint64_t cap_ = 0;  // blocks allocated
  int device_ = 0;
  std::vector<uint64_t> dim_;
};

void cuda_setdev(int gpu);

// dev_layer.h:11-12.  roots: the first t[g] blocks of expanded[g]; out:
// expanded[g] = leaves (LSB cleared), lSum_h/rSum_h [tree][depth] and
// secret_sum[tree] on the host (trees of GPU g follow those of GPU g-1).
// buffer[g] and sep[g] are used as device scratch.
void cuda_mpcot_sender(Mat *expanded, Mat *buffer, Mat *sep, blk *lSum_h, blk *rSum_h,
                       blk *secret_sum, int *t, int depth, blk *delta, int ngpu);

// dev_layer.h:14-15.  cSum_h [tree][depth] chosen OT messages, choices
// [tree][depth] (false punctures the right child), secret_sum[tree] (host);
// out: expanded[g] = receiver leaves.
void cuda_mpcot_recver(Mat *expanded, Mat *buffer, Mat *sep, blk *cSum_h, blk *secret_sum,
                       int *t, int depth, bool *choices, int ngpu);

// dev_layer.h:17-18.  key: emp AES_KEY round keys; its first 16 bytes (the
// LPN seed) are the key.  expanded[g] holds rows [sum_{g'<g} n[g'], +n[g]) of
// the noise vector; kk (host, k blocks) is copied to kk_d[g]; out: nn (host,
// all rows).  pubMats is accepted for signature compatibility and unused:
// the index matrix is generated inside the kernel.
void cuda_primal_lpn(Role role, Mat *pubMats, int64_t d, int64_t *n, int k, uint32_t *key,
                     Mat *expanded, blk *nn, Mat *kk_d, blk *kk, int ngpu);
