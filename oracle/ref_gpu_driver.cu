// ref_gpu_driver.cu -- TEST INFRASTRUCTURE ONLY: speed context and pins.
//
// Drives the reference's own GPU path, compiled from the reference tree for
// sm_100a by oracle/build_ref.sh into oracle/_ref/librefgpu.so (only the
// ref_gpu_* entry points below are exported, so the reference's Mat and
// dev_layer names cannot collide with libcuot's adapter of the same names):
//   cuda_mpcot_sender   ferret/emp-ot/emp-ot/ferret/dev_layer.cu:20-59
//   cuda_primal_lpn     ferret/emp-ot/emp-ot/ferret/dev_layer.cu:161-186
//   QuasiCyclic::encode_dense + two Mat::bit_transpose, the content of
//                       SOTSender::dual_lpn (silent/sender.cu:110-119,
//                       silent/quasi_cyclic.cu:118-128, gpu/gpu_matrix.cu:95-121)
// These outputs are not the oracle's semantics: the reference GPU path uses a
// non-FIPS key schedule, other GGM keys and no parent XOR, races on its level
// sums and rounds a float FFT.  The tests compare Mat::bit_transpose with
// this library's transpose, and the MPCOT leaves and the LPN outputs with the
// oracle's restatement of those GPU semantics (or_compat_*).  Every entry
// point accepts only shapes for which the reference kernels' index
// arithmetic (none of them checks bounds) stays inside the buffers the
// reference's own callers allocate:
//   MPCOT: t * 2^h a multiple of 1024 leaves (aesExpand128 launches whole
//     blocks of 512 threads per level, so the last level of t * 2^h / 2 parents
//     must fill them exactly; the earlier, narrower levels then read and write
//     inside the t * 2^h-block matrices);
//   LPN: n a multiple of 2048 (make_block and lpn_single_row launch exactly
//     n*d/4 / 1024 and n / 1024 full blocks of 1024 threads);
//   transpose: n a multiple of 256 rows, at most 2^23 (beyond that the
//     kernel's row-block count no longer covers the grid);
//   QC encode: n a power of two in [2^17, 2^23] (a's make_block launch needs
//     n / 128 to be a multiple of 1024).
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cufft.h>

#include "dev_layer.h"
#include "gpu_define.h"
#include "gpu_matrix.h"
#include "gpu_ops.h"
#include "lpn.h"
#include "pprf.h"
// QuasiCyclic keeps its `a` (a64) private; this harness reads it back to pin
// the restatement of how the constructor makes it.  Every header that
// quasi_cyclic.h includes is already in, so the access change reaches only
// that one class definition.
#define private public
#include "quasi_cyclic.h"
#undef private

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool pow2(uint64_t n) { return n && !(n & (n - 1)); }

}  // namespace

extern "C" {

// Mean wall-clock ms of the reference's blocking cuda_mpcot_sender for t
// trees of depth h (one GPU), over `reps` calls after one warm-up call.
__attribute__((visibility("default"))) double ref_gpu_mpcot_sender_ms(int t, int h, int reps) {
  const uint64_t n = uint64_t(t) << h;
  if (t < 1 || h < 1 || h > 20 || n < 1024 || n % 1024 || reps < 1) return -1.0;
  // FerretCOT::expSeed and MpcotReg::buffer / separated (ferret_cot.hpp:19-22,
  // mpcot_reg.h:55-61): t * 2^h blocks each
  Mat expanded({n}), buffer({n}), sep({n});
  expanded.clear();
  std::vector<blk> ls(size_t(t) * h), rs(size_t(t) * h), ss(t);
  blk delta{{1, 2, 3, 4}};
  int tt[1] = {t};
  cuda_mpcot_sender(&expanded, &buffer, &sep, ls.data(), rs.data(), ss.data(), tt, h, &delta, 1);
  const double t0 = now_ms();
  for (int i = 0; i < reps; i++)
    cuda_mpcot_sender(&expanded, &buffer, &sep, ls.data(), rs.data(), ss.data(), tt, h, &delta, 1);
  return (now_ms() - t0) / reps;
}

// Mean wall-clock ms of the reference's blocking cuda_primal_lpn (index
// matrix generation, kk upload, lpn_single_row, nn download) for n rows,
// k inputs, d = 10.
__attribute__((visibility("default"))) double ref_gpu_primal_lpn_ms(int64_t n, int k, int reps) {
  const int64_t d = 10;
  if (n < 2048 || n % 2048 || k < 1 || reps < 1) return -1.0;
  // LpnF2's pubMats / kk_d (lpn_f2.h:32-38) and the MPCOT output rows
  Mat pub({uint64_t((n * d + 3) / 4)}), kk_d({uint64_t(k)}), expanded({uint64_t(n)});
  expanded.clear();
  std::vector<blk> kk(k), nn(n);
  for (int i = 0; i < k; i++)
    for (int w = 0; w < 4; w++) kk[i].data[w] = uint32_t(i * 2654435761u + w);
  uint32_t key[44] = {0x01020304, 0x05060708, 0x090a0b0c, 0x0d0e0f10};
  int64_t rows[1] = {n};
  cuda_primal_lpn(Sender, &pub, d, rows, k, key, &expanded, nn.data(), &kk_d, kk.data(), 1);
  const double t0 = now_ms();
  for (int i = 0; i < reps; i++)
    cuda_primal_lpn(Sender, &pub, d, rows, k, key, &expanded, nn.data(), &kk_d, kk.data(), 1);
  return (now_ms() - t0) / reps;
}

// Mean ms of one role's SOT dual LPN on the reference's GPU path: the
// leaves (n blocks) to 128 bit planes, QuasiCyclic(Sender, 2n, n,
// 128).encode_dense, and back (silent/sender.cu:110-119), device time with
// a synchronisation on both sides.  The QuasiCyclic set-up (a and its
// transform) is outside the timed region, as in the reference's constructor.
__attribute__((visibility("default"))) double ref_gpu_sot_dual_lpn_ms(uint64_t n, int reps) {
  if (!pow2(n) || n < (1ull << 17) || n > (1ull << 23) || reps < 1) return -1.0;
  Mat b({n, 1});
  b.clear();
  QuasiCyclic qc(Sender, 2 * n, n, 128);
  auto one = [&] {
    b.bit_transpose(0, 0);  // (n, 1) -> (128, n / 128)
    qc.encode_dense(b);
    b.bit_transpose(0, 0);  // back to (n, 1)
  };
  one();
  cudaDeviceSynchronize();
  const double t0 = now_ms();
  for (int i = 0; i < reps; i++) one();
  cudaDeviceSynchronize();
  return (now_ms() - t0) / reps;
}

// Leaves of the reference's cuda_mpcot_sender (one GPU) for t roots and
// delta (host, 16 bytes each): out = t * 2^h blocks, tree-major (the
// function leaves them in `expanded`, dev_layer.cu:46-49).  0 on success.
__attribute__((visibility("default"))) int ref_gpu_mpcot_sender_leaves(int t, int h, const uint8_t *roots,
                                                                       const uint8_t *delta, uint8_t *out) {
  const uint64_t n = uint64_t(t) << h;
  if (t < 1 || h < 1 || h > 20 || n < 1024 || n % 1024) return -1;
  Mat expanded({n}), buffer({n}), sep({n});
  expanded.clear();
  if (cudaMemcpy(expanded.data(), roots, size_t(t) * 16, cudaMemcpyHostToDevice) != cudaSuccess) return -2;
  std::vector<blk> ls(size_t(t) * h), rs(size_t(t) * h), ss(t);
  blk dl;
  memcpy(&dl, delta, 16);
  int tt[1] = {t};
  cuda_mpcot_sender(&expanded, &buffer, &sep, ls.data(), rs.data(), ss.data(), tt, h, &dl, 1);
  if (cudaMemcpy(out, expanded.data(), n * 16, cudaMemcpyDeviceToHost) != cudaSuccess) return -3;
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

// The reference's cuda_primal_lpn (d = 10, one GPU) on n rows `in` (host)
// with k blocks kk (host) and the 16-byte AES key it takes from the front of
// LpnF2's expanded schedule (lpn_f2.h:85, dev_layer.cu:168): out (host) = the
// rows after the LPN.  n a multiple of 2048.  0 on success.
__attribute__((visibility("default"))) int ref_gpu_primal_lpn_run(int64_t n, int k, const uint8_t *key16,
                                                                  const uint8_t *kk, const uint8_t *in,
                                                                  uint8_t *out) {
  const int64_t d = 10;
  if (n < 2048 || n % 2048 || k < 1) return -1;
  Mat pub({uint64_t((n * d + 3) / 4)}), kk_d({uint64_t(k)}), expanded({uint64_t(n)});
  if (cudaMemcpy(expanded.data(), in, size_t(n) * 16, cudaMemcpyHostToDevice) != cudaSuccess) return -2;
  uint32_t key[44] = {0};
  memcpy(key, key16, 16);
  std::vector<blk> kkh(k);
  memcpy(kkh.data(), kk, size_t(k) * 16);
  int64_t rows[1] = {n};
  cuda_primal_lpn(Sender, &pub, d, rows, k, key, &expanded, reinterpret_cast<blk *>(out), &kk_d, kkh.data(), 1);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

// The reference's QuasiCyclic(Sender, 2n, n, 128).encode_dense on 128 bit
// planes of n bits (host, plane r at r * n / 8 bytes): out (host) = its float
// (cuFFT) encode of them.  Its `a` is AES'(make_block(i)), i < n / 128, under
// a key of four rand() values drawn in its constructor
// (silent/quasi_cyclic.cu:59-66): srand(seed) first, the same four values go
// to key_out (16 bytes), so a caller can rebuild `a`.  n a power of two in
// [2^17, 2^23].  a_out (optional, n / 8 bytes): the constructor's `a`.  0 on
// success.
__attribute__((visibility("default"))) int ref_gpu_qc_encode(uint64_t n, unsigned seed, const uint8_t *in,
                                                             uint8_t *out, uint8_t *key_out, uint8_t *a_out) {
  if (!pow2(n) || n < (1ull << 17) || n > (1ull << 23)) return -1;
  srand(seed);
  uint32_t key[4];
  for (int i = 0; i < 4; i++) key[i] = uint32_t(rand());
  memcpy(key_out, key, 16);
  srand(seed);
  QuasiCyclic qc(Sender, 2 * n, n, 128);
  if (a_out && cudaMemcpy(a_out, qc.a64.data(), n / 8, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
  Mat b({128, n / 128});
  if (cudaMemcpy(b.data(), in, n * 16, cudaMemcpyHostToDevice) != cudaSuccess) return -2;
  qc.encode_dense(b);
  if (cudaMemcpy(out, b.data(), n * 16, cudaMemcpyDeviceToHost) != cudaSuccess) return -3;
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

// The reference's Mat::bit_transpose of n rows of one block each: in (host,
// n * 16 bytes) -> out (host, 128 planes of n / 8 bytes).  0 on success.
__attribute__((visibility("default"))) int ref_gpu_bit_transpose(const uint8_t *in, uint64_t n, uint8_t *out) {
  if (n < 256 || n % 256 || n > (1ull << 23)) return -1;
  Mat m({n, 1});
  if (cudaMemcpy(m.data(), in, n * 16, cudaMemcpyHostToDevice) != cudaSuccess) return -2;
  m.bit_transpose(0, 0);
  if (cudaMemcpy(out, m.data(), n * 16, cudaMemcpyDeviceToHost) != cudaSuccess) return -3;
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

}  // extern "C"
