// emp_ref.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points over the reference's OWN emp-ot Ferret code, compiled from
// the reference tree by oracle/build_ref.sh into oracle/_ref/libempref.so:
//   ferret/emp-ot/emp-ot/ferret/twokeyprp.h      TwoKeyPRP (GGM node)
//   ferret/emp-ot/emp-ot/ferret/spcot_sender.h   SPCOT_Sender::compute
//   ferret/emp-ot/emp-ot/ferret/spcot_recver.h   SPCOT_Recver::compute
//   ferret/emp-ot/emp-ot/ferret/lpn_f2.h         LpnF2::task
// over the emp-tool shim in oracle/emp_shim (emp-tool is not vendored).
// The tests use it to pin the C oracle (oracle/cuot_oracle.c) and the CUDA
// path to the reference's GGM tree, OT messages, leaf mask, secret sum,
// receiver reconstruction and LPN index matrix.  Nothing in the product
// loads it.
#include "emp-tool/emp-tool.h"

// lpn_f2.h names cuOT's device layer (Mat, cuda_setdev, cuda_primal_lpn,
// Role; gpu/gpu_matrix.h, dev_layer.h) without including it.  LpnF2::task,
// the only member used here, touches none of them, so host stand-ins with
// no storage are enough for its constructor.
enum Role { Sender, Recver };
struct blk { uint32_t data[4]; };
class Mat {
 public:
  void resize(std::vector<uint64_t> dim) { dim_ = dim; }
 private:
  std::vector<uint64_t> dim_;
};
inline void cuda_setdev(int) {}
void cuda_primal_lpn(Role role, Mat *pubMats, int64_t d, int64_t *n, int k, uint32_t *key,
                     Mat *expanded, blk *nn, Mat *kk_d, blk *kk, int ngpu);

#include "emp-ot/ferret/spcot_sender.h"
#include "emp-ot/ferret/spcot_recver.h"
#include "emp-ot/ferret/lpn_f2.h"

#include <utility>

namespace {

// SPCOT_* keep an IO pointer but compute() never uses it.
struct NullIO {
  void send_data(const void *, int) {}
  void recv_data(void *, int) {}
  void flush() {}
};

inline block load(const uint8_t *p) {
  block b;
  std::memcpy(&b, p, sizeof(block));
  return b;
}
inline void store(uint8_t *p, block b) { std::memcpy(p, &b, sizeof(block)); }

template <int D>
void lpn_task(const uint8_t *seed, const uint8_t *kk, int k, uint8_t *nn, int64_t n, int64_t start,
              int64_t end) {
  int64_t rows[1] = {n};
  NullIO io;
  LpnF2<NullIO, D> lpn(ALICE, rows, k, &io, 1);
  lpn.seed = load(seed);
  lpn.task(reinterpret_cast<block *>(nn), reinterpret_cast<const block *>(kk), start, end);
}

template <int... Ds>
bool lpn_dispatch(int d, std::integer_sequence<int, Ds...>, const uint8_t *seed, const uint8_t *kk,
                  int k, uint8_t *nn, int64_t n, int64_t start, int64_t end) {
  bool hit = false;
  ((d == Ds + 1 ? (lpn_task<Ds + 1>(seed, kk, k, nn, n, start, end), hit = true) : false), ...);
  return hit;
}

}  // namespace

extern "C" {

// AES-128 ECB through the shim (AES_set_encrypt_key + AES_ecb_encrypt_blks),
// so the tests can pin the shim itself to FIPS-197 and cryptoTools.
void ref_emp_aes_ecb(const uint8_t *key, const uint8_t *in, uint8_t *out, uint64_t nblocks) {
  AES_KEY k;
  AES_set_encrypt_key(load(key), &k);
  for (uint64_t i = 0; i < nblocks; ++i) {
    block b = load(in + 16 * i);
    AES_ecb_encrypt_blks(&b, 1, &k);
    store(out + 16 * i, b);
  }
}

// One tree of SPCOT_Sender (depth_in = h + 1, seed = root): leaves (2^h
// blocks, LSB cleared), ot_msg_0 / ot_msg_1 per level (h blocks each) and
// secret_sum_f2 = XOR(leaves) ^ delta.  Needs h >= 2: ggm_tree_gen always
// expands level 1 with node_expand_2to4 (spcot_sender.h:71-73).
int ref_spcot_sender(const uint8_t *root, int h, const uint8_t *delta, uint8_t *leaves,
                     uint8_t *m0, uint8_t *m1, uint8_t *secret_sum) {
  if (h < 2 || h > 24) return -1;
  NullIO io;
  SPCOT_Sender<NullIO> s(&io, h + 1);
  s.seed = load(root);
  std::vector<block> tree(size_t(1) << h);
  s.compute(tree.data(), load(delta));
  std::memcpy(leaves, tree.data(), tree.size() * sizeof(block));
  std::memcpy(m0, s.m, size_t(h) * sizeof(block));
  std::memcpy(m1, s.m + h, size_t(h) * sizeof(block));
  store(secret_sum, s.secret_sum_f2);
  return 0;
}

// One tree of SPCOT_Recver: b[l] is the choice of level l (false = the
// punctured node is the right child), m[l] the received message m_b[l].
// Writes the 2^h reconstructed leaves and the punctured leaf's index.
int ref_spcot_recver(int h, const uint8_t *b, const uint8_t *m, const uint8_t *secret_sum,
                     uint8_t *leaves, int *choice_pos) {
  if (h < 1 || h > 24) return -1;
  NullIO io;
  SPCOT_Recver<NullIO> r(&io, h + 1);
  for (int l = 0; l < h; ++l) {
    r.b[l] = b[l] != 0;
    r.m[l] = load(m + 16 * l);
  }
  r.secret_sum_f2 = load(secret_sum);
  *choice_pos = r.get_index();
  // layer_recover expands the whole level in place, so the last level writes
  // exactly 2^h blocks (node_expand_4to8 at i = 2^(h-1) - 4 reaches 2^h - 1).
  std::vector<block> tree((size_t(1) << h) + 4);
  r.compute(tree.data());
  std::memcpy(leaves, tree.data(), (size_t(1) << h) * sizeof(block));
  return 0;
}

// Both roles of `T` trees of one MPCOT, one thread: SPCOT_Sender::compute per
// tree (seed = roots[i]), the level OT by selection (choice[i*h + l] picks
// ot_msg_1), then SPCOT_Recver::compute.  leaves_s / leaves_r: T * 2^h blocks
// each, tree-major.  h >= 2.
int ref_mpcot_trees(const uint8_t *roots, int T, int h, const uint8_t *delta, const uint8_t *choice,
                    uint8_t *leaves_s, uint8_t *leaves_r) {
  if (h < 2 || h > 24 || T < 0) return -1;
  NullIO io;
  const size_t W = size_t(1) << h;
  std::vector<block> rtree(W + 4);
  for (int i = 0; i < T; ++i) {
    SPCOT_Sender<NullIO> s(&io, h + 1);
    s.seed = load(roots + 16 * size_t(i));
    block *tree = reinterpret_cast<block *>(leaves_s) + size_t(i) * W;
    s.compute(tree, load(delta));
    SPCOT_Recver<NullIO> r(&io, h + 1);
    for (int l = 0; l < h; ++l) {
      r.b[l] = choice[size_t(i) * h + l] != 0;
      r.m[l] = r.b[l] ? s.m[h + l] : s.m[l];
    }
    r.secret_sum_f2 = s.secret_sum_f2;
    r.get_index();
    r.compute(rtree.data());
    std::memcpy(leaves_r + size_t(i) * W * 16, rtree.data(), W * sizeof(block));
  }
  return 0;
}

// LpnF2<IO, d>::task(nn, kk, start, end) with seed = `seed`: nn[i] ^= the d
// indexed kk blocks for rows [start, end), the last <= 4 rows through
// __compute1.  d in [1, 32].
int ref_lpn_task(const uint8_t *seed, const uint8_t *kk, int k, int d, uint8_t *nn, int64_t n,
                 int64_t start, int64_t end) {
  if (k < 1 || start < 0 || end > n || start > end) return -1;
  return lpn_dispatch(d, std::make_integer_sequence<int, 32>{}, seed, kk, k, nn, n, start, end) ? 0
                                                                                               : -1;
}

}  // extern "C"
