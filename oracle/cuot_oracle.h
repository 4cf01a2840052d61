/*
 * cuot_oracle.h -- CPU oracle for the silent-OT hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the cuot_b200 package,
 * libcuot.so, the C ABI in include/) links, loads or calls this code.  It is
 * loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
 * and reference legs, where it is the checker (or the timed CPU baseline),
 * never the thing measured on the GPU.
 *
 * Every routine restates the reference's CPU semantics for one step of the
 * path (emp-ot / cryptoTools, FIPS-197 AES), citing the reference file:line it
 * follows.  Blocks are 16 bytes with the same memory image as emp-tool's
 * `block` (__m128i; makeBlock(hi, lo) puts `lo` in bytes 0..7) and cuOT's
 * `blk` (4 x uint32, gpu/gpu_define.h:12-16).
 */
#ifndef CUOT_ORACLE_H
#define CUOT_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { uint64_t lo, hi; } or_block;

/* ---- AES-128 (FIPS-197) ------------------------------------------------ */
void or_aes128_key_expand(const uint8_t key[16], uint8_t rk[176]);
void or_aes128_encrypt(const uint8_t rk[176], const uint8_t *in, uint8_t *out,
                       size_t nblocks);
/* Portable (table-free, byte-wise) encryption, used to cross-check the
 * AES-NI path. */
void or_aes128_encrypt_portable(const uint8_t rk[176], const uint8_t *in,
                                uint8_t *out, size_t nblocks);
int or_have_aesni(void);

/* ---- seeded host PRG (cryptoTools PRNG restated) ------------------------ */
void or_prg_fill(const uint8_t seed[16], uint64_t block_offset, uint8_t *out,
                 size_t nblocks);

/* ---- Ferret GGM (emp-ot SPCOT sender/receiver) --------------------------- */
void or_ggm_node(const or_block *parent, or_block *left, or_block *right);
void or_ferret_pprf_sender(const or_block *roots, int64_t t, int h,
                           or_block delta, or_block *leaves, or_block *lsum,
                           or_block *rsum, or_block *secret_sum, int threads);
void or_ferret_pprf_recver(const or_block *mc, const uint8_t *choice,
                           const or_block *secret_sum, int64_t t, int h,
                           or_block *leaves, int threads);

/* ---- Ferret primal LPN (emp-ot LpnF2::task over [0, n)) ----------------- */
void or_lpn_primal(const uint8_t seed[16], const or_block *kk, int64_t k,
                   int d, or_block *nn, int64_t n, int threads);

/* ---- cuOT's own GPU path, restated (compat semantics) --------------------
 * Not the path's semantics: the reference's GPU kernels differ from emp-ot in
 * documented ways, restated here so tests can pin exactly those differences
 * against the reference kernels run on a B200.
 *   key schedule: FIPS-197 with round i's Rcon taken one entry early, i.e.
 *     0x8d, 0x01, 0x02, ..., 0x1b (gpu/aes_expand.cu:52-65, utilsBox.h:61);
 *   GGM node: child_y = AES'_{k_y}(parent) without the parent XOR, keys with
 *     first word 3242342 (left) and 8993849 (right) (aesExpand128,
 *     gpu/aes_op.cu:176-266; keys dev_layer.cu:22-23); no leaf LSB mask;
 *   secret sum: XOR of a tree's leaves ^ delta (dev_layer.cu:50-53);
 *   LPN: index block b (b in [0, n d / 4)) = (low 64 bits 4 floor((b + start)
 *     / 10), high 64 bits b mod 10) encrypted under AES'_key (make_block,
 *     gpu/gpu_ops.cu:102-109; dev_layer.cu:167-169), row i XORs kk[w % k]
 *     for the d consecutive 32-bit words w from word i d on
 *     (lpn_single_row, dev_layer.cu:146-159). */
void or_compat_key_expand(const uint8_t key[16], uint8_t rk[176]);
void or_compat_ferret_sender(const or_block *roots, int64_t t, int h,
                             or_block delta, or_block *leaves,
                             or_block *secret_sum, int threads);
void or_compat_lpn(const uint8_t key[16], const or_block *kk, int64_t k,
                   int d, or_block *nn, int64_t n, int64_t start, int threads);

/* ---- bit transpose (cuOT bit_transposer semantics) ---------------------- */
void or_bit_transpose(const uint8_t *in, uint64_t rows, uint64_t row_bytes,
                      uint64_t col_lo, uint64_t col_hi, uint8_t *out);

/* ---- SOT quasi-cyclic dual LPN ------------------------------------------ */
void or_qc_gen_a(const uint8_t key[16], uint64_t n, uint64_t *a);
void or_gf2_cyclic_mul(const uint64_t *a, const uint64_t *b, uint64_t n,
                       uint64_t *out);
void or_qc_encode(const uint64_t *a, uint64_t *planes, uint64_t n, int nplanes,
                  int threads);
void or_qc_encode_sparse(const uint64_t *a, const uint64_t *pos, int weight,
                         uint64_t n, uint64_t *out);
void or_sot_dual_lpn(const uint64_t *a, or_block *io, uint64_t n,
                     int threads);

/* ---- SOT PPRF (silent/sender.cu, silent/recver.cu structure) ------------ */
void or_sot_pprf_sender(const or_block *roots, int64_t t, int h,
                        or_block delta, const or_block *base0,
                        const or_block *base1, or_block *leaves, or_block *m0,
                        or_block *m1, int threads);
void or_sot_pprf_recver(const or_block *m0, const or_block *m1,
                        const or_block *mc, const uint8_t *choice, int64_t t,
                        int h, or_block *leaves, int threads);

/* ---- Ferret malicious consistency check: per-tree chi sums -------------- */
/* GF(2^128) with the natural bit order (bit i of the little-endian block is
 * the coefficient of x^i), reduced mod x^128 + x^7 + x^2 + x + 1: emp-tool's
 * gfmul (emp-tool/utils/f2k.h @ 44b1dde, not vendored). */
void or_gf128_mul(const or_block *a, const or_block *b, or_block *out);
/* out[j] = sum_{i < 2^h} seed_j^(i+1) * leaves[j*2^h + i]: emp-tool's
 * uni_hash_coeff_gen (chi_i = seed^(i+1)) followed by
 * vector_inn_prdt_sum_red, as spcot_sender.h:88-98 / spcot_recver.h:97-107
 * use them on one tree (seed = the first half of Hash(secret_sum)). */
void or_ferret_chi_sum(const or_block *leaves, int64_t t, int h,
                       const or_block *seeds, or_block *out, int threads);

#ifdef __cplusplus
}
#endif
#endif
