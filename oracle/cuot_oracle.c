/*
 * cuot_oracle.c -- CPU oracle for the silent-OT hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see cuot_oracle.h).  The product never links or
 * calls this file; tests, smoke() and bench.py's CPU legs load it as the
 * checker and as the timed CPU baseline.
 *
 * Pinning: the AES here is checked against FIPS-197 Appendix C.1, against
 * OpenSSL (python `cryptography`) and against the reference's own vendored
 * cryptoTools AES/PRNG built from source into oracle/_ref (see
 * oracle/build_ref.sh and tests/test_oracle.py).  The GGM, LPN and QC
 * restatements follow the reference's CPU code line by line as cited; the
 * reference ships no golden vectors for them (its only end-to-end check,
 * test/test.h:152-170, is commented out), so those are pinned by the
 * properties the protocol guarantees (COT correlation, sender/receiver
 * agreement, linearity) and by a pure-Python restatement in the tests.
 */
#define _GNU_SOURCE
#include "cuot_oracle.h"
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#if defined(__x86_64__)
#include <immintrin.h>
#include <wmmintrin.h>
#define OR_X86 1
#endif

/* ======================================================================== */
/* AES-128, restated from FIPS-197 (the S-box is derived from GF(2^8)       */
/* inversion plus the affine map, not copied from a table).                 */
/* ======================================================================== */

static uint8_t g_sbox[256];
static pthread_once_t g_sbox_once = PTHREAD_ONCE_INIT;

static uint8_t gf_mul(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  while (b) {
    if (b & 1) r ^= a;
    a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
    b >>= 1;
  }
  return r;
}

static uint8_t rotl8(uint8_t x, int s) {
  return (uint8_t)((x << s) | (x >> (8 - s)));
}

static void build_sbox(void) {
  for (int x = 0; x < 256; x++) {
    uint8_t inv = 0;
    if (x) {
      for (int y = 1; y < 256; y++)
        if (gf_mul((uint8_t)x, (uint8_t)y) == 1) { inv = (uint8_t)y; break; }
    }
    g_sbox[x] = (uint8_t)(inv ^ rotl8(inv, 1) ^ rotl8(inv, 2) ^ rotl8(inv, 3) ^
                          rotl8(inv, 4) ^ 0x63);
  }
}

static const uint8_t *sbox(void) {
  pthread_once(&g_sbox_once, build_sbox);
  return g_sbox;
}

/* FIPS-197 sec. 5.2 key expansion.  (cuOT's GPU schedule XORs Rcon[i-1]
 * instead, gpu/aes_expand.cu:59 with gpu/utilsBox.h:61; emp-tool and
 * cryptoTools use the standard one, which is what the CPU path computes.) */
void or_aes128_key_expand(const uint8_t key[16], uint8_t rk[176]) {
  const uint8_t *sb = sbox();
  memcpy(rk, key, 16);
  uint8_t rcon = 1;
  for (int i = 4; i < 44; i++) {
    uint8_t t[4];
    memcpy(t, rk + 4 * (i - 1), 4);
    if (i % 4 == 0) {
      uint8_t u = t[0];
      t[0] = (uint8_t)(sb[t[1]] ^ rcon);
      t[1] = sb[t[2]];
      t[2] = sb[t[3]];
      t[3] = sb[u];
      rcon = gf_mul(rcon, 2);
    }
    for (int j = 0; j < 4; j++) rk[4 * i + j] = (uint8_t)(rk[4 * (i - 4) + j] ^ t[j]);
  }
}

void or_aes128_encrypt_portable(const uint8_t rk[176], const uint8_t *in,
                                uint8_t *out, size_t nblocks) {
  const uint8_t *sb = sbox();
  for (size_t b = 0; b < nblocks; b++) {
    uint8_t s[16], t[16];
    for (int i = 0; i < 16; i++) s[i] = (uint8_t)(in[16 * b + i] ^ rk[i]);
    for (int round = 1; round <= 10; round++) {
      /* SubBytes + ShiftRows: state byte (row r, column c) lives at r + 4c. */
      for (int c = 0; c < 4; c++)
        for (int r = 0; r < 4; r++) t[r + 4 * c] = sb[s[r + 4 * ((c + r) & 3)]];
      if (round < 10) {
        for (int c = 0; c < 4; c++) {
          uint8_t a0 = t[4 * c], a1 = t[4 * c + 1], a2 = t[4 * c + 2], a3 = t[4 * c + 3];
          s[4 * c + 0] = (uint8_t)(gf_mul(a0, 2) ^ gf_mul(a1, 3) ^ a2 ^ a3);
          s[4 * c + 1] = (uint8_t)(a0 ^ gf_mul(a1, 2) ^ gf_mul(a2, 3) ^ a3);
          s[4 * c + 2] = (uint8_t)(a0 ^ a1 ^ gf_mul(a2, 2) ^ gf_mul(a3, 3));
          s[4 * c + 3] = (uint8_t)(gf_mul(a0, 3) ^ a1 ^ a2 ^ gf_mul(a3, 2));
        }
      } else {
        memcpy(s, t, 16);
      }
      for (int i = 0; i < 16; i++) s[i] ^= rk[16 * round + i];
    }
    memcpy(out + 16 * b, s, 16);
  }
}

#ifdef OR_X86
__attribute__((target("aes,sse4.1")))
static void aesni_encrypt(const uint8_t rk[176], const uint8_t *in,
                          uint8_t *out, size_t nblocks) {
  __m128i k[11];
  for (int i = 0; i < 11; i++) k[i] = _mm_loadu_si128((const __m128i *)(rk + 16 * i));
  size_t b = 0;
  for (; b + 8 <= nblocks; b += 8) {
    __m128i x[8];
    for (int j = 0; j < 8; j++)
      x[j] = _mm_xor_si128(_mm_loadu_si128((const __m128i *)(in + 16 * (b + j))), k[0]);
    for (int r = 1; r < 10; r++)
      for (int j = 0; j < 8; j++) x[j] = _mm_aesenc_si128(x[j], k[r]);
    for (int j = 0; j < 8; j++)
      _mm_storeu_si128((__m128i *)(out + 16 * (b + j)), _mm_aesenclast_si128(x[j], k[10]));
  }
  for (; b < nblocks; b++) {
    __m128i x = _mm_xor_si128(_mm_loadu_si128((const __m128i *)(in + 16 * b)), k[0]);
    for (int r = 1; r < 10; r++) x = _mm_aesenc_si128(x, k[r]);
    _mm_storeu_si128((__m128i *)(out + 16 * b), _mm_aesenclast_si128(x, k[10]));
  }
}
#endif

int or_have_aesni(void) {
#ifdef OR_X86
  __builtin_cpu_init();
  return __builtin_cpu_supports("aes") && __builtin_cpu_supports("sse4.1");
#else
  return 0;
#endif
}

void or_aes128_encrypt(const uint8_t rk[176], const uint8_t *in, uint8_t *out,
                       size_t nblocks) {
#ifdef OR_X86
  static int have = -1;
  if (have < 0) have = or_have_aesni();
  if (have) { aesni_encrypt(rk, in, out, nblocks); return; }
#endif
  or_aes128_encrypt_portable(rk, in, out, nblocks);
}

/* ======================================================================== */
/* Seeded host PRG: cryptoTools PRNG (silent/lib/cryptoTools/Crypto/        */
/* PRNG.cpp:44-56,100-106; AES.cpp:302-320): key = seed, stream block i =   */
/* AES_seed(toBlock(i)), i.e. the counter i little-endian in bytes 0..7.    */
/* ======================================================================== */
void or_prg_fill(const uint8_t seed[16], uint64_t block_offset, uint8_t *out,
                 size_t nblocks) {
  uint8_t rk[176];
  or_aes128_key_expand(seed, rk);
  uint8_t ctr[16 * 64];
  size_t done = 0;
  while (done < nblocks) {
    size_t m = nblocks - done < 64 ? nblocks - done : 64;
    memset(ctr, 0, 16 * m);
    for (size_t j = 0; j < m; j++) {
      uint64_t c = block_offset + done + j;
      memcpy(ctr + 16 * j, &c, 8);
    }
    or_aes128_encrypt(rk, ctr, out + 16 * done, m);
    done += m;
  }
}

/* ======================================================================== */
/* Small thread pool helper for the CPU baseline (parallel-for over a range). */
/* ======================================================================== */
typedef void (*range_fn)(void *ctx, int64_t lo, int64_t hi);
typedef struct { range_fn fn; void *ctx; int64_t lo, hi; } range_job;

static void *range_thread(void *p) {
  range_job *j = (range_job *)p;
  j->fn(j->ctx, j->lo, j->hi);
  return NULL;
}

/* Splits [0, n) into `threads` contiguous pieces whose boundaries are
 * multiples of `align`. */
static void parallel_for(int64_t n, int threads, int64_t align, range_fn fn,
                         void *ctx) {
  if (threads <= 1 || n <= align) { fn(ctx, 0, n); return; }
  if (threads > 256) threads = 256;
  pthread_t th[256];
  range_job jobs[256];
  int64_t units = (n + align - 1) / align;
  if (threads > units) threads = (int)units;
  int started = 0;
  for (int i = 0; i < threads; i++) {
    int64_t lo = (units * i / threads) * align;
    int64_t hi = (units * (i + 1) / threads) * align;
    if (hi > n) hi = n;
    jobs[i].fn = fn; jobs[i].ctx = ctx; jobs[i].lo = lo; jobs[i].hi = hi;
    if (i == threads - 1) { fn(ctx, lo, hi); continue; }
    if (pthread_create(&th[i], NULL, range_thread, &jobs[i]) == 0) started = i + 1;
    else fn(ctx, lo, hi);
  }
  for (int i = 0; i < started; i++) pthread_join(th[i], NULL);
}

/* ======================================================================== */
/* GGM node function: emp-ot TwoKeyPRP (ferret/emp-ot/emp-ot/ferret/        */
/* twokeyprp.h:7-63) with the keys spcot_sender.h:63 / spcot_recver.h:68    */
/* use: k0 = zero_block, k1 = makeBlock(0, 1).                              */
/*   left  = AES_k0(p) ^ p,   right = AES_k1(p) ^ p.                        */
/* ======================================================================== */
static uint8_t g_rk0[176], g_rk1[176];
static pthread_once_t g_rk_once = PTHREAD_ONCE_INIT;
static void build_rk(void) {
  uint8_t k[16] = {0};
  or_aes128_key_expand(k, g_rk0);
  k[0] = 1; /* makeBlock(0, 1): low qword = 1 */
  or_aes128_key_expand(k, g_rk1);
}

void or_ggm_node(const or_block *parent, or_block *left, or_block *right) {
  pthread_once(&g_rk_once, build_rk);
  or_block p = *parent, l, r;
  or_aes128_encrypt(g_rk0, (const uint8_t *)&p, (uint8_t *)&l, 1);
  or_aes128_encrypt(g_rk1, (const uint8_t *)&p, (uint8_t *)&r, 1);
  l.lo ^= p.lo; l.hi ^= p.hi;
  r.lo ^= p.lo; r.hi ^= p.hi;
  *left = l;
  *right = r;
}

/* Expands `np` parents stored at buf[0..np) into 2*np children at
 * buf[0..2np) in heap order (children of i at 2i, 2i+1), in place, walking
 * from the last parent down exactly as twokeyprp.h's callers do
 * (spcot_sender.h:73-84).  Accumulates XOR of even/odd children. */
static void expand_level_inplace(or_block *buf, int64_t np, or_block *even_sum,
                                 or_block *odd_sum) {
  pthread_once(&g_rk_once, build_rk);
  or_block es = {0, 0}, os = {0, 0};
  int64_t i = np;
  while (i > 0) {
    int64_t c = i >= 4 ? 4 : i;
    int64_t i0 = i - c;
    or_block p[4], a[4], b[4];
    for (int64_t j = 0; j < c; j++) p[j] = buf[i0 + j];
    or_aes128_encrypt(g_rk0, (const uint8_t *)p, (uint8_t *)a, (size_t)c);
    or_aes128_encrypt(g_rk1, (const uint8_t *)p, (uint8_t *)b, (size_t)c);
    for (int64_t j = 0; j < c; j++) {
      or_block L = {a[j].lo ^ p[j].lo, a[j].hi ^ p[j].hi};
      or_block R = {b[j].lo ^ p[j].lo, b[j].hi ^ p[j].hi};
      buf[2 * (i0 + j)] = L;
      buf[2 * (i0 + j) + 1] = R;
      es.lo ^= L.lo; es.hi ^= L.hi;
      os.lo ^= R.lo; os.hi ^= R.hi;
    }
    i = i0;
  }
  if (even_sum) *even_sum = es;
  if (odd_sum) *odd_sum = os;
}

/* ---- Ferret MPCOT sender ------------------------------------------------
 * Per tree (one SPCOT_Sender per tree, tree-major output, mpcot_reg.h:130-
 * 143): expand the root h levels (spcot_sender.h:61-86), recording for level
 * d (children at depth d+1) lsum[t][d] = XOR of even children (ot_msg_0) and
 * rsum[t][d] = XOR of odd children (ot_msg_1).  Then clear each leaf's LSB
 * (`& one`, one = makeBlock(~0, ~1)) and secret_sum = XOR(leaves) ^ delta
 * (spcot_sender.h:47-58).  Host layout [tree][depth] as dev_layer.cu:27-28. */
typedef struct {
  const or_block *roots; int h; or_block delta;
  or_block *leaves, *lsum, *rsum, *ss;
} fsend_ctx;

static void fsend_range(void *vc, int64_t lo, int64_t hi) {
  fsend_ctx *c = (fsend_ctx *)vc;
  int64_t w = (int64_t)1 << c->h;
  for (int64_t t = lo; t < hi; t++) {
    or_block *tree = c->leaves + t * w;
    tree[0] = c->roots[t];
    for (int d = 0; d < c->h; d++)
      expand_level_inplace(tree, (int64_t)1 << d, &c->lsum[t * c->h + d],
                           &c->rsum[t * c->h + d]);
    or_block s = c->delta;
    for (int64_t i = 0; i < w; i++) {
      tree[i].lo &= ~(uint64_t)1;
      s.lo ^= tree[i].lo; s.hi ^= tree[i].hi;
    }
    c->ss[t] = s;
  }
}

void or_ferret_pprf_sender(const or_block *roots, int64_t t, int h,
                           or_block delta, or_block *leaves, or_block *lsum,
                           or_block *rsum, or_block *secret_sum, int threads) {
  fsend_ctx c = {roots, h, delta, leaves, lsum, rsum, secret_sum};
  parallel_for(t, threads, 1, fsend_range, &c);
}

/* ---- Ferret MPCOT receiver ----------------------------------------------
 * spcot_recver.h:33-95: choice bit b[d] = choice[t][d]; at level d the
 * receiver holds mc[t][d] = ot_msg_{b}[d].  b == 0 fills the even child of
 * the punctured parent with (XOR of even nodes) ^ mc and punctures the odd
 * child; b == 1 the mirror image.  The two children of the punctured parent
 * are zeroed first (spcot_recver.h:75).  Finally the punctured leaf is
 * zeroed, every leaf gets its LSB cleared, and the punctured leaf becomes
 * XOR(other leaves) ^ secret_sum (spcot_recver.h:53-64).  The tree root is
 * unknown to the receiver; it starts from zero, which does not change the
 * result. */
typedef struct {
  const or_block *mc; const uint8_t *choice; const or_block *ss;
  int h; or_block *leaves;
} frecv_ctx;

static void frecv_range(void *vc, int64_t lo, int64_t hi) {
  frecv_ctx *c = (frecv_ctx *)vc;
  int64_t w = (int64_t)1 << c->h;
  for (int64_t t = lo; t < hi; t++) {
    or_block *tree = c->leaves + t * w;
    tree[0].lo = tree[0].hi = 0;
    int64_t pos = 0;
    for (int d = 0; d < c->h; d++) {
      expand_level_inplace(tree, (int64_t)1 << d, NULL, NULL);
      int64_t f = 2 * pos;
      tree[f].lo = tree[f].hi = 0;
      tree[f + 1].lo = tree[f + 1].hi = 0;
      int b = c->choice[t * c->h + d] ? 1 : 0;
      int64_t fill = f + b;
      or_block s = c->mc[t * c->h + d];
      int64_t nn = (int64_t)2 << d;
      for (int64_t i = b; i < nn; i += 2) { s.lo ^= tree[i].lo; s.hi ^= tree[i].hi; }
      tree[fill] = s;
      pos = f + (1 - b);
    }
    tree[pos].lo = tree[pos].hi = 0;
    or_block s = {0, 0};
    for (int64_t i = 0; i < w; i++) {
      tree[i].lo &= ~(uint64_t)1;
      s.lo ^= tree[i].lo; s.hi ^= tree[i].hi;
    }
    s.lo ^= c->ss[t].lo; s.hi ^= c->ss[t].hi;
    tree[pos] = s;
  }
}

void or_ferret_pprf_recver(const or_block *mc, const uint8_t *choice,
                           const or_block *secret_sum, int64_t t, int h,
                           or_block *leaves, int threads) {
  frecv_ctx c = {mc, choice, secret_sum, h, leaves};
  parallel_for(t, threads, 1, frecv_range, &c);
}

/* ======================================================================== */
/* Ferret primal LPN: emp-ot LpnF2 (ferret/emp-ot/emp-ot/ferret/lpn_f2.h).  */
/*   mask = smallest 2^b - 1 >= k                     (lpn_f2.h:27-31)      */
/*   rows i..i+3 (i a multiple of 4, i < n-4): d blocks makeBlock(i, m),    */
/*     m < d, AES-encrypted under key = seed; u32 word 10m'+j of the output */
/*     gives row i+m' term j: idx = w & mask, idx -= k if idx >= k          */
/*                                                     (lpn_f2.h:46-59)     */
/*   remaining rows (j >= n-4 after the stride-4 loop): ceil(d/4) blocks    */
/*     makeBlock(j, m), idx = r[jj] % k                (lpn_f2.h:61-79)     */
/* The whole range [0, n) is one task (the GPU replaces emp's thread split, */
/* lpn_f2.h:100-115); threads here split at multiples of 4 and reproduce    */
/* exactly the single-range result.                                         */
/* ======================================================================== */
typedef struct {
  uint8_t rk[176]; const or_block *kk; int64_t k, n, tail; int d, mask;
  or_block *nn;
} lpn_ctx;

static void lpn_range(void *vc, int64_t lo, int64_t hi) {
  lpn_ctx *c = (lpn_ctx *)vc;
  int d = c->d;
  or_block tmp[64];
  for (int64_t i = lo; i < hi && i < c->tail; i += 4) {
    for (int m = 0; m < d; m++) { tmp[m].lo = (uint64_t)m; tmp[m].hi = (uint64_t)i; }
    or_aes128_encrypt(c->rk, (const uint8_t *)tmp, (uint8_t *)tmp, (size_t)d);
    const uint32_t *r = (const uint32_t *)tmp;
    for (int m = 0; m < 4; m++) {
      or_block acc = c->nn[i + m];
      for (int j = 0; j < d; j++) {
        int64_t idx = (int64_t)(*r++ & (uint32_t)c->mask);
        if (idx >= c->k) idx -= c->k;
        acc.lo ^= c->kk[idx].lo; acc.hi ^= c->kk[idx].hi;
      }
      c->nn[i + m] = acc;
    }
  }
  int nb = d / 4 + (d % 4 != 0);
  int64_t j0 = lo > c->tail ? lo : c->tail;
  for (int64_t j = j0; j < hi; j++) {
    for (int m = 0; m < nb; m++) { tmp[m].lo = (uint64_t)m; tmp[m].hi = (uint64_t)j; }
    or_aes128_encrypt(c->rk, (const uint8_t *)tmp, (uint8_t *)tmp, (size_t)nb);
    const uint32_t *r = (const uint32_t *)tmp;
    or_block acc = c->nn[j];
    for (int jj = 0; jj < d; jj++) {
      int64_t idx = (int64_t)(r[jj] % (uint32_t)c->k);
      acc.lo ^= c->kk[idx].lo; acc.hi ^= c->kk[idx].hi;
    }
    c->nn[j] = acc;
  }
}

void or_lpn_primal(const uint8_t seed[16], const or_block *kk, int64_t k,
                   int d, or_block *nn, int64_t n, int threads) {
  lpn_ctx c;
  or_aes128_key_expand(seed, c.rk);
  c.kk = kk; c.k = k; c.n = n; c.d = d; c.nn = nn;
  int mask = 1;
  while (mask < k) { mask <<= 1; mask |= 1; }
  c.mask = mask;
  /* first row handled by __compute1: the stride-4 loop runs while j < n-4 */
  int64_t tail = 0;
  while (tail < n - 4) tail += 4;
  c.tail = tail;
  parallel_for(n, threads, 4, lpn_range, &c);
}

/* ======================================================================== */
/* cuOT's GPU path restated (compat semantics; see cuot_oracle.h).  Used    */
/* only to pin how the reference's own GPU kernels differ from emp-ot.      */
/* ======================================================================== */

/* FIPS-197 key expansion with the round constants one entry early: round i
 * uses Rcon[i - 1] of the table 0x8d, 0x01, 0x02, ... (gpu/aes_expand.cu:59,
 * gpu/utilsBox.h:61), i.e. 0x8d, then the standard 0x01 .. 0x1b. */
void or_compat_key_expand(const uint8_t key[16], uint8_t rk[176]) {
  const uint8_t *sb = sbox();
  memcpy(rk, key, 16);
  uint8_t rcon = 0x8d;
  for (int i = 4; i < 44; i++) {
    uint8_t t[4];
    memcpy(t, rk + 4 * (i - 1), 4);
    if (i % 4 == 0) {
      uint8_t u = t[0];
      t[0] = (uint8_t)(sb[t[1]] ^ rcon);
      t[1] = sb[t[2]];
      t[2] = sb[t[3]];
      t[3] = sb[u];
      /* the table continues 0x01, 0x02, ... after 0x8d (0x8d * 2 in GF(2^8)
       * would be 0x01 too: 0x8d is the inverse of 2) */
      rcon = gf_mul(rcon, 2);
    }
    for (int j = 0; j < 4; j++) rk[4 * i + j] = (uint8_t)(rk[4 * (i - 4) + j] ^ t[j]);
  }
}

/* 16-byte key whose first little-endian 32-bit word is w (the rest zero),
 * as cuda_mpcot_sender's k0_blk / k1_blk (dev_layer.cu:22-23). */
static void compat_word_key(uint32_t w, uint8_t key[16]) {
  memset(key, 0, 16);
  for (int i = 0; i < 4; i++) key[i] = (uint8_t)(w >> (8 * i));
}

typedef struct {
  const or_block *roots; int h; or_block delta; or_block *leaves; or_block *ss;
  uint8_t rk0[176], rk1[176];
} csend_ctx;

/* Trees [lo, hi): level d's node j (tree-major) has children 2j (key 0) and
 * 2j + 1 (key 1), each AES'(node) with no XOR of the parent (aes_op.cu:
 * 176-266 writes the cipher text itself). */
static void csend_range(void *vc, int64_t lo, int64_t hi) {
  csend_ctx *c = (csend_ctx *)vc;
  const int64_t w = (int64_t)1 << c->h;
  for (int64_t t = lo; t < hi; t++) {
    or_block *tree = c->leaves + t * w;
    tree[0] = c->roots[t];
    for (int d = 0; d < c->h; d++) {
      const int64_t width = (int64_t)1 << d;
      /* in place, from the last node down, so no parent is overwritten early */
      for (int64_t j = width - 1; j >= 0; j--) {
        or_block p = tree[j], l, r;
        or_aes128_encrypt(c->rk0, (const uint8_t *)&p, (uint8_t *)&l, 1);
        or_aes128_encrypt(c->rk1, (const uint8_t *)&p, (uint8_t *)&r, 1);
        tree[2 * j] = l;
        tree[2 * j + 1] = r;
      }
    }
    or_block s = c->delta;
    for (int64_t i = 0; i < w; i++) { s.lo ^= tree[i].lo; s.hi ^= tree[i].hi; }
    if (c->ss) c->ss[t] = s;
  }
}

void or_compat_ferret_sender(const or_block *roots, int64_t t, int h,
                             or_block delta, or_block *leaves,
                             or_block *secret_sum, int threads) {
  csend_ctx c;
  c.roots = roots; c.h = h; c.delta = delta; c.leaves = leaves; c.ss = secret_sum;
  uint8_t k[16];
  compat_word_key(3242342u, k);
  or_compat_key_expand(k, c.rk0);
  compat_word_key(8993849u, k);
  or_compat_key_expand(k, c.rk1);
  parallel_for(t, threads, 1, csend_range, &c);
}

typedef struct {
  uint8_t rk[176]; const or_block *kk; int64_t k; int d; or_block *nn; int64_t start;
} clpn_ctx;

static void clpn_range(void *vc, int64_t lo, int64_t hi) {
  clpn_ctx *c = (clpn_ctx *)vc;
  for (int64_t i = lo; i < hi; i++) {
    or_block acc = c->nn[i];
    /* words [i d, i d + d) of the encrypted index blocks */
    const int64_t w0 = i * c->d, b0 = w0 / 4, b1 = (w0 + c->d - 1) / 4;
    uint32_t words[4 * 12];
    for (int64_t b = b0; b <= b1; b++) {
      or_block pt = {4 * (uint64_t)((b + c->start) / 10), (uint64_t)(b % 10)}, ct;
      or_aes128_encrypt(c->rk, (const uint8_t *)&pt, (uint8_t *)&ct, 1);
      memcpy(words + 4 * (b - b0), &ct, 16);
    }
    for (int j = 0; j < c->d; j++) {
      const uint32_t w = words[w0 + j - 4 * b0];
      const or_block *x = &c->kk[w % (uint64_t)c->k];
      acc.lo ^= x->lo; acc.hi ^= x->hi;
    }
    c->nn[i] = acc;
  }
}

void or_compat_lpn(const uint8_t key[16], const or_block *kk, int64_t k,
                   int d, or_block *nn, int64_t n, int64_t start, int threads) {
  clpn_ctx c;
  or_compat_key_expand(key, c.rk);
  c.kk = kk; c.k = k; c.d = d; c.nn = nn; c.start = start;
  parallel_for(n, threads, 1, clpn_range, &c);
}

/* ======================================================================== */
/* Bit transpose: cuOT bit_transposer (gpu/gpu_ops.cu:31-70) as driven by   */
/* Mat::bit_transpose (gpu/gpu_matrix.cu:95-121): input row r bit c (LSB-   */
/* first inside each byte, bytes in order) becomes output row (c - col_lo)  */
/* bit r.  rows must be a multiple of 8; output rows are rows/8 bytes.      */
/* ======================================================================== */
void or_bit_transpose(const uint8_t *in, uint64_t rows, uint64_t row_bytes,
                      uint64_t col_lo, uint64_t col_hi, uint8_t *out) {
  uint64_t orow_bytes = rows / 8;
  memset(out, 0, (col_hi - col_lo) * orow_bytes);
  for (uint64_t r = 0; r < rows; r++) {
    const uint8_t *row = in + r * row_bytes;
    for (uint64_t c = col_lo; c < col_hi; c++) {
      if ((row[c >> 3] >> (c & 7)) & 1)
        out[(c - col_lo) * orow_bytes + (r >> 3)] |= (uint8_t)(1u << (r & 7));
    }
  }
}

/* ======================================================================== */
/* Quasi-cyclic dual LPN (SOT), silent/quasi_cyclic.cu.                     */
/* ======================================================================== */

/* a = n bits of AES output of counter blocks: block i has low qword
 * 4*floor(i/10) and high qword i mod 10 (make_block, gpu/gpu_ops.cu:102-109),
 * encrypted under `key` (quasi_cyclic.cu:57-66), FIPS AES. */
void or_qc_gen_a(const uint8_t key[16], uint64_t n, uint64_t *a) {
  uint8_t rk[176];
  or_aes128_key_expand(key, rk);
  uint64_t nb = (n + 127) / 128;
  or_block *blk = (or_block *)malloc(nb * sizeof(or_block));
  for (uint64_t i = 0; i < nb; i++) { blk[i].lo = 4 * (i / 10); blk[i].hi = i % 10; }
  or_aes128_encrypt(rk, (const uint8_t *)blk, (uint8_t *)blk, nb);
  memcpy(a, blk, (n + 7) / 8);
  free(blk);
}

/* carry-less 64x64 -> 128 */
#ifdef OR_X86
__attribute__((target("pclmul,sse4.1")))
static void clmul_x86(uint64_t a, uint64_t b, uint64_t *lo, uint64_t *hi) {
  __m128i r = _mm_clmulepi64_si128(_mm_cvtsi64_si128((long long)a),
                                   _mm_cvtsi64_si128((long long)b), 0);
  *lo = (uint64_t)_mm_cvtsi128_si64(r);
  *hi = (uint64_t)_mm_extract_epi64(r, 1);
}
#endif
static void clmul_portable(uint64_t a, uint64_t b, uint64_t *lo, uint64_t *hi) {
  uint64_t l = 0, h = 0;
  for (int i = 0; i < 64; i++)
    if ((b >> i) & 1) { l ^= a << i; if (i) h ^= a >> (64 - i); }
  *lo = l; *hi = h;
}
static int g_have_pclmul = -1;
static void clmul64(uint64_t a, uint64_t b, uint64_t *lo, uint64_t *hi) {
#ifdef OR_X86
  if (g_have_pclmul < 0) {
    __builtin_cpu_init();
    g_have_pclmul = __builtin_cpu_supports("pclmul") && __builtin_cpu_supports("sse4.1");
  }
  if (g_have_pclmul) { clmul_x86(a, b, lo, hi); return; }
#endif
  clmul_portable(a, b, lo, hi);
}

/* r[0..2n) = a[0..n) * b[0..n) over GF(2) (schoolbook) */
static void gf2_mul_school(const uint64_t *a, const uint64_t *b, size_t n,
                           uint64_t *r) {
  memset(r, 0, 2 * n * sizeof(uint64_t));
  for (size_t i = 0; i < n; i++) {
    if (!a[i]) continue;
    for (size_t j = 0; j < n; j++) {
      uint64_t lo, hi;
      clmul64(a[i], b[j], &lo, &hi);
      r[i + j] ^= lo;
      r[i + j + 1] ^= hi;
    }
  }
}

/* Karatsuba over GF(2)[x] on 64-bit words, n a power of two; tmp >= 4n. */
static void gf2_mul_kara(const uint64_t *a, const uint64_t *b, size_t n,
                         uint64_t *r, uint64_t *tmp) {
  if (n <= 16) { gf2_mul_school(a, b, n, r); return; }
  size_t m = n / 2;
  uint64_t *as = tmp, *bs = tmp + m, *mid = tmp + 2 * m, *rest = tmp + 4 * m;
  gf2_mul_kara(a, b, m, r, rest);               /* r[0..2m)  = a0 b0 */
  gf2_mul_kara(a + m, b + m, m, r + 2 * m, rest); /* r[2m..4m) = a1 b1 */
  for (size_t i = 0; i < m; i++) { as[i] = a[i] ^ a[m + i]; bs[i] = b[i] ^ b[m + i]; }
  gf2_mul_kara(as, bs, m, mid, rest);           /* (a0+a1)(b0+b1) */
  for (size_t i = 0; i < 2 * m; i++) mid[i] ^= r[i] ^ r[2 * m + i];
  for (size_t i = 0; i < 2 * m; i++) r[m + i] ^= mid[i];
}

/* out = a * b mod (x^n - 1) over GF(2); n a multiple of 64.  This is the
 * exact value silent/quasi_cyclic.cu:118-128 approximates with float cuFFT:
 * with mIn = 2n, mOut = n (silent/sender.cu:39) the product of the n-bit a
 * and the zero-padded plane b is folded by float_to_bit_and_modp
 * (quasi_cyclic.cu:34-49): out_j = c_j ^ c_{n+j}. */
void or_gf2_cyclic_mul(const uint64_t *a, const uint64_t *b, uint64_t n,
                       uint64_t *out) {
  size_t nw = (size_t)(n / 64), p = 1;
  while (p < nw) p <<= 1;
  uint64_t *A = (uint64_t *)calloc(p, 8), *B = (uint64_t *)calloc(p, 8);
  uint64_t *R = (uint64_t *)malloc(2 * p * 8), *T = (uint64_t *)malloc(4 * p * 8 + 64);
  memcpy(A, a, nw * 8);
  memcpy(B, b, nw * 8);
  gf2_mul_kara(A, B, p, R, T);
  /* fold: bit j of the product for j >= n goes to j - n */
  memcpy(out, R, nw * 8);
  for (size_t i = nw; i < 2 * p; i++) {
    if (R[i]) out[i - nw] ^= R[i]; /* 2p <= 4nw, and the product has < 2n bits */
  }
  free(A); free(B); free(R); free(T);
}

typedef struct { const uint64_t *a; uint64_t *planes; uint64_t n; } qc_ctx;
static void qc_range(void *vc, int64_t lo, int64_t hi) {
  qc_ctx *c = (qc_ctx *)vc;
  uint64_t nw = c->n / 64;
  uint64_t *o = (uint64_t *)malloc(nw * 8);
  for (int64_t r = lo; r < hi; r++) {
    or_gf2_cyclic_mul(c->a, c->planes + r * nw, c->n, o);
    memcpy(c->planes + r * nw, o, nw * 8);
  }
  free(o);
}

/* QuasiCyclic::encode_dense (quasi_cyclic.cu:118-128): every plane r of
 * n bits is replaced by a * plane_r mod (x^n - 1). */
void or_qc_encode(const uint64_t *a, uint64_t *planes, uint64_t n, int nplanes,
                  int threads) {
  qc_ctx c = {a, planes, n};
  parallel_for(nplanes, threads, 1, qc_range, &c);
}

/* QuasiCyclic::encode_sparse (quasi_cyclic.cu:130-161): out = a * e mod
 * (x^n - 1) with e the indicator of the `weight` positions pos[] (each
 * < n; the reference skips positions > mOut, quasi_cyclic.cu:139).  The
 * reference's shift by 64 at alignment 0 is undefined behaviour; the exact
 * value is computed here. */
void or_qc_encode_sparse(const uint64_t *a, const uint64_t *pos, int weight,
                         uint64_t n, uint64_t *out) {
  uint64_t nw = n / 64;
  memset(out, 0, nw * 8);
  for (int i = 0; i < weight; i++) {
    uint64_t p = pos[i];
    if (p >= n) continue;
    /* out ^= a * x^p mod (x^n - 1): cyclic rotation of a by p bits */
    uint64_t ws = p / 64, bs = p % 64;
    for (uint64_t w = 0; w < nw; w++) {
      uint64_t v = a[w];
      uint64_t dst = (w + ws) % nw;
      out[dst] ^= v << bs;
      if (bs) out[(dst + 1) % nw] ^= v >> (64 - bs);
    }
  }
}

/* SOT dual_lpn (silent/sender.cu:110-119, silent/recver.cu:168-174) with one
 * GPU per party: transpose the n x 128 leaf blocks into 128 planes, encode
 * each plane, transpose back. */
void or_sot_dual_lpn(const uint64_t *a, or_block *io, uint64_t n, int threads) {
  uint8_t *planes = (uint8_t *)malloc(n * 16);
  or_bit_transpose((const uint8_t *)io, n, 16, 0, 128, planes);
  or_qc_encode(a, (uint64_t *)planes, n, 128, threads);
  or_bit_transpose(planes, 128, n / 8, 0, n, (uint8_t *)io);
  free(planes);
}

/* ======================================================================== */
/* SOT PPRF (silent/sender.cu:76-108, silent/recver.cu:124-163), with the    */
/* emp-ot node function above.  Layouts follow the reference's Mats:        */
/* base0/base1/mc are [h][t], m0/m1 are [h+1][t] (sender.cu:20-21,          */
/* recver.cu:22-24), leaves tree-major.                                      */
/*   sender: m0[d] = base0[d] ^ L_d, m1[d] = base1[d] ^ R_d (d < h);         */
/*           m0[h] = base0[h-1] ^ R_{h-1} ^ delta,                            */
/*           m1[h] = base1[h-1] ^ L_{h-1} ^ delta (sender.cu:81-102).         */
/*   receiver: per level d, choice c = choice[d][t]; the node 2*ap + c is     */
/*           corrected with (m_c[d] ^ mc[d]) ^ own side-c sum; ap moves to    */
/*           2*ap + 1 - c (recver.cu:98-115,143-155); after the last level    */
/*           the punctured leaf is corrected with (m_c[h] ^ mc[h-1]) ^ own    */
/*           side-(1-c) sum, giving sender_leaf ^ delta.                      */
/* ======================================================================== */
typedef struct {
  const or_block *roots; int64_t t; int h; or_block delta;
  const or_block *b0, *b1; or_block *leaves, *m0, *m1;
} ssend_ctx;

static void ssend_range(void *vc, int64_t lo, int64_t hi) {
  ssend_ctx *c = (ssend_ctx *)vc;
  int64_t w = (int64_t)1 << c->h, T = c->t;
  for (int64_t t = lo; t < hi; t++) {
    or_block *tree = c->leaves + t * w;
    tree[0] = c->roots[t];
    for (int d = 0; d < c->h; d++) {
      or_block L, R;
      expand_level_inplace(tree, (int64_t)1 << d, &L, &R);
      or_block a = c->b0[d * T + t], b = c->b1[d * T + t];
      c->m0[d * T + t] = (or_block){a.lo ^ L.lo, a.hi ^ L.hi};
      c->m1[d * T + t] = (or_block){b.lo ^ R.lo, b.hi ^ R.hi};
      if (d == c->h - 1) {
        c->m0[(d + 1) * T + t] = (or_block){a.lo ^ R.lo ^ c->delta.lo, a.hi ^ R.hi ^ c->delta.hi};
        c->m1[(d + 1) * T + t] = (or_block){b.lo ^ L.lo ^ c->delta.lo, b.hi ^ L.hi ^ c->delta.hi};
      }
    }
  }
}

void or_sot_pprf_sender(const or_block *roots, int64_t t, int h,
                        or_block delta, const or_block *base0,
                        const or_block *base1, or_block *leaves, or_block *m0,
                        or_block *m1, int threads) {
  ssend_ctx c = {roots, t, h, delta, base0, base1, leaves, m0, m1};
  parallel_for(t, threads, 1, ssend_range, &c);
}

typedef struct {
  const or_block *m0, *m1, *mc; const uint8_t *choice; int64_t t; int h;
  or_block *leaves;
} srecv_ctx;

static void srecv_range(void *vc, int64_t lo, int64_t hi) {
  srecv_ctx *c = (srecv_ctx *)vc;
  int64_t w = (int64_t)1 << c->h, T = c->t;
  for (int64_t t = lo; t < hi; t++) {
    or_block *tree = c->leaves + t * w;
    tree[0].lo = tree[0].hi = 0;
    int64_t ap = 0;
    for (int d = 0; d < c->h; d++) {
      or_block S[2];
      expand_level_inplace(tree, (int64_t)1 << d, &S[0], &S[1]);
      int cb = c->choice[d * T + t] ? 1 : 0;
      const or_block *mcur = cb ? c->m1 : c->m0;
      or_block dec = {mcur[d * T + t].lo ^ c->mc[d * T + t].lo,
                      mcur[d * T + t].hi ^ c->mc[d * T + t].hi};
      int64_t f = 2 * ap + cb;
      tree[f].lo ^= dec.lo ^ S[cb].lo;
      tree[f].hi ^= dec.hi ^ S[cb].hi;
      ap = 2 * ap + (1 - cb);
      if (d == c->h - 1) {
        or_block dec2 = {mcur[(d + 1) * T + t].lo ^ c->mc[d * T + t].lo,
                         mcur[(d + 1) * T + t].hi ^ c->mc[d * T + t].hi};
        tree[ap].lo ^= dec2.lo ^ S[1 - cb].lo;
        tree[ap].hi ^= dec2.hi ^ S[1 - cb].hi;
      }
    }
  }
}

void or_sot_pprf_recver(const or_block *m0, const or_block *m1,
                        const or_block *mc, const uint8_t *choice, int64_t t,
                        int h, or_block *leaves, int threads) {
  srecv_ctx c = {m0, m1, mc, choice, t, h, leaves};
  parallel_for(t, threads, 1, srecv_range, &c);
}

/* ======================================================================== */
/* GF(2^128) (emp-tool gfmul semantics: natural bit order, reduction        */
/* polynomial x^128 + x^7 + x^2 + x + 1) and the per-tree chi sums of the   */
/* malicious consistency check (spcot_sender.h:88-98, spcot_recver.h:97-107).*/
/* ======================================================================== */
void or_gf128_mul(const or_block *a, const or_block *b, or_block *out) {
  uint64_t r[4] = {0, 0, 0, 0}, lo, hi;
  clmul64(a->lo, b->lo, &lo, &hi); r[0] ^= lo; r[1] ^= hi;
  clmul64(a->lo, b->hi, &lo, &hi); r[1] ^= lo; r[2] ^= hi;
  clmul64(a->hi, b->lo, &lo, &hi); r[1] ^= lo; r[2] ^= hi;
  clmul64(a->hi, b->hi, &lo, &hi); r[2] ^= lo; r[3] ^= hi;
  /* fold x^128 * (r2 + r3 x^64) with x^128 = x^7 + x^2 + x + 1, twice */
  for (int pass = 0; pass < 2; pass++) {
    uint64_t h0 = r[2], h1 = r[3];
    r[2] = r[3] = 0;
    /* (h0 + h1 x^64) * (1 + x + x^2 + x^7) */
    const int sh[4] = {0, 1, 2, 7};
    for (int k = 0; k < 4; k++) {
      int s = sh[k];
      r[0] ^= h0 << s;
      r[1] ^= (h1 << s) | (s ? h0 >> (64 - s) : 0);
      r[2] ^= s ? h1 >> (64 - s) : 0;
    }
  }
  out->lo = r[0];
  out->hi = r[1];
}

typedef struct {
  const or_block *leaves;
  const or_block *seeds;
  or_block *out;
  int h;
} chi_ctx;

static void chi_range(void *p, int64_t lo, int64_t hi) {
  chi_ctx *c = (chi_ctx *)p;
  const int64_t L = (int64_t)1 << c->h;
  for (int64_t j = lo; j < hi; j++) {
    or_block chi = c->seeds[j], acc = {0, 0}, prod;
    for (int64_t i = 0; i < L; i++) {
      or_gf128_mul(&chi, &c->leaves[j * L + i], &prod);
      acc.lo ^= prod.lo;
      acc.hi ^= prod.hi;
      or_gf128_mul(&chi, &c->seeds[j], &chi);
    }
    c->out[j] = acc;
  }
}

void or_ferret_chi_sum(const or_block *leaves, int64_t t, int h,
                       const or_block *seeds, or_block *out, int threads) {
  chi_ctx c = {leaves, seeds, out, h};
  parallel_for(t, threads, 1, chi_range, &c);
}
