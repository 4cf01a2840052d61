// aes_host.cu -- host-side AES-128 key schedule and T-table (FIPS-197).
// The S-box is derived from GF(2^8) inversion followed by the affine map,
// not copied from a table.
#include <cstring>
#include <mutex>
#include "common.cuh"

namespace cuot {
namespace {
uint8_t gmul(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  while (b) {
    if (b & 1) r ^= a;
    a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
    b >>= 1;
  }
  return r;
}
uint8_t rotl(uint8_t x, int s) { return (uint8_t)((x << s) | (x >> (8 - s))); }

struct Tables {
  uint8_t sbox[256];
  uint32_t t0[256];
  Tables() {
    for (int x = 0; x < 256; x++) {
      uint8_t inv = 0;
      for (int y = 1; x && y < 256; y++)
        if (gmul((uint8_t)x, (uint8_t)y) == 1) { inv = (uint8_t)y; break; }
      sbox[x] = (uint8_t)(inv ^ rotl(inv, 1) ^ rotl(inv, 2) ^ rotl(inv, 3) ^
                          rotl(inv, 4) ^ 0x63);
    }
    for (int x = 0; x < 256; x++) {
      uint32_t s = sbox[x];
      t0[x] = gmul((uint8_t)s, 2) | (s << 8) | (s << 16) |
              ((uint32_t)gmul((uint8_t)s, 3) << 24);
    }
  }
};
const Tables &tables() {
  static Tables t;
  return t;
}
}  // namespace

const uint32_t *host_t0_table() { return tables().t0; }

void host_aes_key_expand(const uint8_t key[16], AesKey *out) {
  const uint8_t *sb = tables().sbox;
  uint8_t rk[176];
  std::memcpy(rk, key, 16);
  uint8_t rcon = 1;
  for (int i = 4; i < 44; i++) {
    uint8_t t[4];
    std::memcpy(t, rk + 4 * (i - 1), 4);
    if (i % 4 == 0) {
      uint8_t u = t[0];
      t[0] = (uint8_t)(sb[t[1]] ^ rcon);
      t[1] = sb[t[2]];
      t[2] = sb[t[3]];
      t[3] = sb[u];
      rcon = gmul(rcon, 2);
    }
    for (int j = 0; j < 4; j++) rk[4 * i + j] = (uint8_t)(rk[4 * (i - 4) + j] ^ t[j]);
  }
  std::memcpy(out->rk, rk, 176);  // little-endian words
  for (int i = 0; i < 44; i++) out->rkr[i] = (out->rk[i] >> 8) | (out->rk[i] << 24);
}

// One block, FIPS-197 rounds over the T-table (column j of a round =
// T0[row-0 byte of column j] ^ rotl8/16/24 of T0 of the row-1/2/3 bytes of
// columns j+1, j+2, j+3 (ShiftRows) ^ round key); little-endian columns.
void host_aes_encrypt(const AesKey &k, const uint8_t in[16], uint8_t out[16]) {
  const uint32_t *t0 = tables().t0;
  const uint8_t *sb = tables().sbox;
  auto rotl = [](uint32_t x, int s) { return (x << s) | (x >> (32 - s)); };
  uint32_t s[4], n[4];
  std::memcpy(s, in, 16);
  for (int j = 0; j < 4; j++) s[j] ^= k.rk[j];
  for (int r = 1; r < 10; r++) {
    for (int j = 0; j < 4; j++)
      n[j] = t0[s[j] & 255] ^ rotl(t0[(s[(j + 1) & 3] >> 8) & 255], 8) ^
             rotl(t0[(s[(j + 2) & 3] >> 16) & 255], 16) ^ rotl(t0[s[(j + 3) & 3] >> 24], 24) ^ k.rk[4 * r + j];
    std::memcpy(s, n, 16);
  }
  for (int j = 0; j < 4; j++)
    n[j] = (uint32_t(sb[s[j] & 255]) | (uint32_t(sb[(s[(j + 1) & 3] >> 8) & 255]) << 8) |
            (uint32_t(sb[(s[(j + 2) & 3] >> 16) & 255]) << 16) | (uint32_t(sb[s[(j + 3) & 3] >> 24]) << 24)) ^
           k.rk[40 + j];
  std::memcpy(out, n, 16);
}
}  // namespace cuot
