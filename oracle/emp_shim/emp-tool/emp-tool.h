// emp-tool/emp-tool.h -- TEST INFRASTRUCTURE ONLY.
//
// A stand-in for the emp-tool headers (emp-toolkit/emp-tool @ 44b1dde, the
// commit ferret/build.sh clones; not vendored in the reference) with just the
// primitives that the reference's own emp-ot Ferret headers use:
// twokeyprp.h, spcot_sender.h, spcot_recver.h, lpn_f2.h, preot.h and
// mpcot_reg.h.  With this directory first on the include path those headers
// compile unchanged from the reference tree, so the oracle and the CUDA path
// can be checked against the reference's own GGM, LPN and OT-message code.
//
// What is restated here, from emp-tool's published behaviour:
//  * block = __m128i; makeBlock(hi, lo) puts `lo` in bytes 0..7.
//  * AES_KEY = 11 FIPS-197 round keys + a round count; AES_set_encrypt_key
//    expands the key with AESKEYGENASSIST (Intel's AES-NI white paper,
//    Gueron 2010); AES_ecb_encrypt_blks / ParaEnc<K, N> encrypt in place with
//    AESENC/AESENCLAST, ParaEnc's block i*N + j under key i.
//  * PRP(key).permute_block = AES-ECB in place under `key`.
//  * PRG = AES-CTR under a seed (a fixed per-process sequence of seeds when
//    none is given, so runs are repeatable).
//  * CCRH::H(x) = AES_0(s(x)) ^ s(x), s(x) = (hi ^ lo, hi), the circular
//    correlation-robust hash.  Only determinism matters where preot.h uses it
//    (both parties run in one process through this same header).
// Hash, GaloisFieldPacking, uni_hash_coeff_gen and vector_inn_prdt_sum_red
// are declared so that the headers' malicious-mode code compiles; nothing
// here calls them, and they abort if called.
#ifndef CUOT_EMP_TOOL_SHIM_H
#define CUOT_EMP_TOOL_SHIM_H

#include <immintrin.h>
#include <wmmintrin.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <iostream>
#include <string>
#include <vector>

namespace emp {

using std::vector;
typedef __m128i block;

const static int ALICE = 1;
const static int BOB = 2;
const static int PUBLIC = 0;

inline block makeBlock(uint64_t high, uint64_t low) { return _mm_set_epi64x((long long)high, (long long)low); }
const static block zero_block = _mm_setzero_si128();
const static block all_one_block = _mm_set_epi64x(-1LL, -1LL);

inline bool getLSB(const block &x) { return (_mm_cvtsi128_si64(x) & 1) == 1; }

inline bool cmpBlock(const block *x, const block *y, int nblocks) {
  return std::memcmp(x, y, size_t(nblocks) * sizeof(block)) == 0;
}

inline void xorBlocks_arr(block *res, const block *x, block y, int nblocks) {
  for (int i = 0; i < nblocks; ++i) res[i] = x[i] ^ y;
}

inline void xorBlocks_arr(block *res, const block *x, const block *y, int nblocks) {
  for (int i = 0; i < nblocks; ++i) res[i] = x[i] ^ y[i];
}

inline void vector_self_xor(block *sum, const block *data, int n) {
  block s = zero_block;
  for (int i = 0; i < n; ++i) s = s ^ data[i];
  *sum = s;
}

[[noreturn]] inline void error(const char *s, int line = 0, const char *file = nullptr) {
  std::fprintf(stderr, "emp error: %s\n", s);
  std::abort();
}

[[noreturn]] inline void shim_missing(const char *what) {
  std::fprintf(stderr, "emp-tool shim: %s is not provided\n", what);
  std::abort();
}

// ---- AES-128 -----------------------------------------------------------

struct AES_KEY {
  block rd_key[11];
  unsigned int rounds;
};

namespace shim_detail {
// One step of the AES-128 key schedule: `assist` = AESKEYGENASSIST(prev, rcon).
inline block expand_step(block prev, block assist) {
  assist = _mm_shuffle_epi32(assist, 0xff);
  prev = _mm_xor_si128(prev, _mm_slli_si128(prev, 4));
  prev = _mm_xor_si128(prev, _mm_slli_si128(prev, 4));
  prev = _mm_xor_si128(prev, _mm_slli_si128(prev, 4));
  return _mm_xor_si128(prev, assist);
}
}  // namespace shim_detail

inline void AES_set_encrypt_key(const block userkey, AES_KEY *key) {
  using shim_detail::expand_step;
  block *k = key->rd_key;
  k[0] = userkey;
  k[1] = expand_step(k[0], _mm_aeskeygenassist_si128(k[0], 0x01));
  k[2] = expand_step(k[1], _mm_aeskeygenassist_si128(k[1], 0x02));
  k[3] = expand_step(k[2], _mm_aeskeygenassist_si128(k[2], 0x04));
  k[4] = expand_step(k[3], _mm_aeskeygenassist_si128(k[3], 0x08));
  k[5] = expand_step(k[4], _mm_aeskeygenassist_si128(k[4], 0x10));
  k[6] = expand_step(k[5], _mm_aeskeygenassist_si128(k[5], 0x20));
  k[7] = expand_step(k[6], _mm_aeskeygenassist_si128(k[6], 0x40));
  k[8] = expand_step(k[7], _mm_aeskeygenassist_si128(k[7], 0x80));
  k[9] = expand_step(k[8], _mm_aeskeygenassist_si128(k[8], 0x1b));
  k[10] = expand_step(k[9], _mm_aeskeygenassist_si128(k[9], 0x36));
  key->rounds = 10;
}

inline block aes_encrypt_one(const AES_KEY *key, block x) {
  x = _mm_xor_si128(x, key->rd_key[0]);
  for (unsigned r = 1; r < key->rounds; ++r) x = _mm_aesenc_si128(x, key->rd_key[r]);
  return _mm_aesenclast_si128(x, key->rd_key[key->rounds]);
}

inline void AES_ecb_encrypt_blks(block *blks, unsigned int nblks, const AES_KEY *key) {
  for (unsigned i = 0; i < nblks; ++i) blks[i] = aes_encrypt_one(key, blks[i]);
}

// Block i*NumEncs + j is encrypted under keys[i].
template <int NumKeys, int NumEncs>
inline void ParaEnc(block *blks, AES_KEY *keys) {
  for (int i = 0; i < NumKeys; ++i)
    for (int j = 0; j < NumEncs; ++j) blks[i * NumEncs + j] = aes_encrypt_one(&keys[i], blks[i * NumEncs + j]);
}

class PRP {
 public:
  AES_KEY aes;
  PRP(const char *key = nullptr) {
    block k = zero_block;
    if (key != nullptr) std::memcpy(&k, key, sizeof(block));
    aes_set_key(k);
  }
  PRP(const block &key) { aes_set_key(key); }
  void aes_set_key(const block &v) { AES_set_encrypt_key(v, &aes); }
  void permute_block(block *data, int nblocks) { AES_ecb_encrypt_blks(data, unsigned(nblocks), &aes); }
};

// ---- PRG: AES-CTR ---------------------------------------------------------

class PRG {
 public:
  AES_KEY aes;
  uint64_t counter = 0;
  PRG(const void *seed = nullptr, int id = 0) {
    block s;
    if (seed != nullptr) {
      std::memcpy(&s, seed, sizeof(block));
    } else {
      static uint64_t next = 0x5eed0000ULL;  // repeatable default seeds
      s = makeBlock(0x9e3779b97f4a7c15ULL, next++);
    }
    reseed(&s, uint64_t(id));
  }
  void reseed(const block *seed, uint64_t id = 0) {
    AES_set_encrypt_key(*seed ^ makeBlock(id, 0), &aes);
    counter = 0;
  }
  void random_block(block *data, int nblocks = 1) {
    for (int i = 0; i < nblocks; ++i) data[i] = aes_encrypt_one(&aes, makeBlock(0, counter++));
  }
  void random_data(void *data, int nbytes) {
    unsigned char *p = static_cast<unsigned char *>(data);
    while (nbytes > 0) {
      block b;
      random_block(&b, 1);
      int c = nbytes < 16 ? nbytes : 16;
      std::memcpy(p, &b, size_t(c));
      p += c;
      nbytes -= c;
    }
  }
  void random_bool(bool *data, int length) {
    for (int i = 0; i < length; ++i) {
      unsigned char c;
      random_data(&c, 1);
      data[i] = (c & 1) != 0;
    }
  }
};

// ---- CCRH: circular correlation-robust hash --------------------------------

class CCRH {
 public:
  AES_KEY aes;
  CCRH() { AES_set_encrypt_key(zero_block, &aes); }
  static block sigma(block x) {
    uint64_t lo = uint64_t(_mm_cvtsi128_si64(x));
    uint64_t hi = uint64_t(_mm_extract_epi64(x, 1));
    return makeBlock(hi ^ lo, hi);
  }
  block H(block in) const {
    block s = sigma(in);
    return aes_encrypt_one(&aes, s) ^ s;
  }
  void Hn(block *out, const block *in, int length, block *scratch = nullptr) const {
    for (int i = 0; i < length; ++i) out[i] = H(in[i]);
  }
};

// ---- declared for the malicious-mode code paths; never called here --------

class Hash {
 public:
  void hash_once(void *dgst, const void *data, int nbyte) { shim_missing("Hash::hash_once"); }
};

class GaloisFieldPacking {
 public:
  void packing(block *res, block *data) { shim_missing("GaloisFieldPacking::packing"); }
};

inline void uni_hash_coeff_gen(block *coeff, block seed, int sz) { shim_missing("uni_hash_coeff_gen"); }

inline void vector_inn_prdt_sum_red(block *res, const block *a, const block *b, int sz) {
  shim_missing("vector_inn_prdt_sum_red");
}

}  // namespace emp

#endif
