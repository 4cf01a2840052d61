// ref_driver.cpp -- C entry points over the reference's own vendored
// cryptoTools AES and PRNG (silent/lib/cryptoTools/Crypto/{AES,PRNG}.cpp),
// compiled from the reference tree into oracle/_ref/libctref.so by
// oracle/build_ref.sh.  TEST INFRASTRUCTURE ONLY: used to pin the oracle's
// AES and seeded PRG against the reference's implementation.
#include "cryptoTools/Crypto/AES.h"
#include "cryptoTools/Crypto/PRNG.h"
#include <cstring>
using namespace osuCrypto;

extern "C" {
// AES-128 ECB under `key` (16-byte image), cryptoTools AES<NI>::setKey +
// ecbEncBlocks.
void ref_aes_ecb(const unsigned char *key, const unsigned char *in,
                 unsigned char *out, unsigned long long nblocks) {
  block k;
  std::memcpy(&k, key, 16);
  AES aes(k);
  for (unsigned long long i = 0; i < nblocks; i++) {
    block p, c;
    std::memcpy(&p, in + 16 * i, 16);
    aes.ecbEncBlock(p, c);
    std::memcpy(out + 16 * i, &c, 16);
  }
}
// First `nblocks` blocks of PRNG(seed).
void ref_prng(const unsigned char *seed, unsigned char *out,
              unsigned long long nblocks) {
  block s;
  std::memcpy(&s, seed, 16);
  PRNG prng(s);
  prng.get(out, nblocks * 16);
}
}
