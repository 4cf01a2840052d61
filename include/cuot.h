/*
 * cuot.h -- C ABI of libcuot, a B200 (sm_100a) silent-OT correlation engine.
 *
 * Drop-in boundary for cuOT's hot path (GGM PPRF expansion -> Ferret primal
 * LPN or SOT quasi-cyclic encode -> 128-plane bit transpose).  Plain C types
 * only: device pointers, sizes, an opaque context and a cudaStream_t passed
 * as void*.  Every call is stream-ordered, returns a status code, and never
 * synchronises the device unless its comment says so.
 *
 * Calls with nothing to do (zero LPN rows, zero AES blocks, zero transpose
 * rows) return CUOT_OK without launching and accept null data pointers; a
 * zero tree count, plane count or instance count is CUOT_EINVAL.
 *
 * Blocks are 16 bytes with the memory image of emp-tool's `block` and cuOT's
 * `blk` (gpu/gpu_define.h:12-16).  Bit vectors are little-endian: bit j of a
 * vector is bit (j % 8) of byte j / 8.
 *
 * The C++ adapter with the reference's own dev_layer.h signatures is in
 * include/cuot_dev_layer.h.
 */
#ifndef CUOT_H
#define CUOT_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define CUOT_OK 0
#define CUOT_EINVAL 1   /* bad argument (shape, alignment, null pointer) */
#define CUOT_ENOMEM 2   /* device allocation failed */
#define CUOT_ECUDA 3    /* a CUDA launch or runtime call failed */
#define CUOT_ETIMEOUT 4 /* a bounded device or host wait ran out */
#define CUOT_ENOTSUP 5  /* shape or mode this build does not support */

typedef struct { uint32_t w[4]; } cuot_block;
typedef struct cuot_ctx cuot_ctx;

const char *cuot_version(void);
const char *cuot_status_string(int status);
/* Detail of the last failure on the calling thread ("" if none). */
const char *cuot_last_error(void);
/* Number of kernels this library has launched in the process (diagnostic). */
unsigned long long cuot_launch_count(void);
/* Diagnostic: the fp64 fused-multiply-add rate of ctx's device in TFLOP/s
 * (2 flops per FMA), from a kernel of independent FMA chains at full
 * occupancy timed with CUDA events: the best of `reps` (1..1000) launches
 * after one warm-up, about 9 ms each on B200.  Synchronises.  The measured
 * denominator of the fp64 FFT encode's fraction. */
int cuot_measure_fp64_tflops(cuot_ctx *ctx, int reps, double *tflops);

/* ---- context -------------------------------------------------------------
 * A context binds one CUDA device, its AES tables and a grow-only scratch
 * arena.  Replaces the per-call Aes / Mat set-up of the reference
 * (gpu/aes_expand.cu:18-30, gpu/gpu_data.cu:7-15). */
int cuot_ctx_create(int device, cuot_ctx **out);
int cuot_ctx_destroy(cuot_ctx *ctx);
/* Pre-size the scratch arena (call before capturing a CUDA graph). */
int cuot_ctx_reserve(cuot_ctx *ctx, uint64_t bytes);
uint64_t cuot_ctx_scratch_bytes(const cuot_ctx *ctx);
/* Tuning knobs of the single-instance calls made on this context (the
 * autotuner in cuot_b200/autotune.py sets them from its measurements):
 *   CUOT_TUNE_PPRF_THREADS  threads per tree CTA, 128 or 256 (default 256)
 *   CUOT_TUNE_QC_PLANES     planes per QC pass, 0 = automatic (512 MiB of
 *                           intermediate)
 *   CUOT_TUNE_QC_BACKEND    transform of the exact QC encode: 0 automatic
 *                           (fp64 FFT for n <= 2^22; dual LPNs at 2^23 and
 *                           2^24 as GF(2) Karatsuba over 2^22 FFTs; the NTT
 *                           mod 469762049 above), 1 the NTT everywhere, 2 as
 *                           0.  Plans and batches keep the backend they were
 *                           created with; set it before creating them.
 *   CUOT_TUNE_QC_STREAMS    streams of one FFT encode, 1 or 2 (default 2:
 *                           groups of about 32 MiB of intermediate alternate
 *                           between the caller's stream and a second stream
 *                           of the context, joined back before the call
 *                           returns).  1 keeps all work on the caller's
 *                           stream, for callers that already overlap several
 *                           encodes (the server's slots).  Applies to later
 *                           calls and plans; a graph batch keeps the value
 *                           of its first run (the graph is captured then).
 *   CUOT_TUNE_QC_RECORD_MARGIN  diagnostic, 0 (default) or 1: the fp64 FFT
 *                           encodes of this context record the largest
 *                           distance |v - round(v)| between a computed
 *                           product coefficient and the integer it rounds to
 *                           (exactness needs < 1/2), read by
 *                           cuot_qc_fft_margin.  Setting 1 allocates and
 *                           zeroes one device word (synchronous: not during
 *                           stream capture); plans and batches made later
 *                           record too. */
#define CUOT_TUNE_PPRF_THREADS 1
#define CUOT_TUNE_QC_PLANES 2
#define CUOT_TUNE_QC_BACKEND 3
#define CUOT_TUNE_QC_STREAMS 4
#define CUOT_TUNE_QC_RECORD_MARGIN 5
int cuot_ctx_set_tuning(cuot_ctx *ctx, int key, int64_t value);
/* The largest |v - round(v)| the context's fp64 FFT encodes have rounded
 * since recording was switched on or last reset (reset != 0 zeroes it after
 * the read).  Synchronous.  CUOT_EINVAL when recording is off.  No
 * counterpart in the reference (its float cuFFT encode truncates without a
 * bound, silent/quasi_cyclic.cu:34-49). */
int cuot_qc_fft_margin(cuot_ctx *ctx, double *out, int reset);

/* ---- AES-128 ECB ---------------------------------------------------------
 * In-place FIPS-197 AES-128 of `nblocks` blocks under `key` (host, 16 bytes).
 * Replaces Aes::encrypt / aesEncrypt128 (gpu/aes_expand.cu:32-36,
 * gpu/aes_op.cu:90-174); unlike the reference it uses the standard key
 * schedule (the reference XORs Rcon[i-1], gpu/aes_expand.cu:59). */
int cuot_aes128_ecb(cuot_ctx *ctx, const uint8_t key[16], cuot_block *io_d,
                    uint64_t nblocks, void *stream);
/* The same encryption, bitsliced: 32 blocks per thread as 128 bit-planes in
 * registers, the S-box as a GF(2) circuit (tower-field inversion), no table
 * lookups.  Same results as cuot_aes128_ecb; kept to measure the two AES
 * designs against each other on the same GPU (the library's PPRF and LPN
 * use the faster one, the T-table).  No counterpart in the reference. */
int cuot_aes128_ecb_bitsliced(cuot_ctx *ctx, const uint8_t key[16], cuot_block *io_d,
                              uint64_t nblocks, void *stream);

/* Seeded PRG on the device: blocks [block_offset, +nblocks) of the
 * cryptoTools PRNG stream for `seed` (block i = AES_seed(i as a little-endian
 * 128-bit counter), silent/lib/cryptoTools/Crypto/PRNG.cpp:44-56,100-106).
 * Used to derive request inputs without a host round-trip. */
int cuot_prg_fill(cuot_ctx *ctx, const uint8_t seed[16], uint64_t block_offset,
                  cuot_block *out_d, uint64_t nblocks, void *stream);

/* ---- Ferret MPCOT: t GGM trees of depth h --------------------------------
 * Node function: emp-ot TwoKeyPRP (ferret/twokeyprp.h:7-63): left =
 * AES_0(p) ^ p, right = AES_{makeBlock(0,1)}(p) ^ p.
 *
 * Sender (replaces cuda_mpcot_sender, dev_layer.cu:20-59; semantics of
 * SPCOT_Sender::ggm_tree_gen, spcot_sender.h:47-86):
 *   roots_d        [t]            tree roots
 *   delta          host pointer to the correlation delta
 *   leaves_d       [t][2^h]       out: leaves with the LSB cleared
 *   lsum_d, rsum_d [t][h]         out: XOR of even / odd children per level
 *   secret_sum_d   [t]            out: XOR(leaves) ^ delta
 * Receiver (replaces cuda_mpcot_recver, dev_layer.cu:87-144; semantics of
 * SPCOT_Recver, spcot_recver.h:33-95):
 *   mc_d           [t][h]         chosen OT messages (ot_msg_{b})
 *   choice_d       [t][h] bytes   b = 0 punctures the right child
 *   secret_sum_d   [t]            the sender's secret sums
 *   leaves_d       [t][2^h]       out: sender leaves, except the punctured
 *                                 leaf = sender leaf ^ delta
 * h in [1, 30]; t >= 1. */
int cuot_ferret_pprf_sender(cuot_ctx *ctx, const cuot_block *roots_d,
                            uint64_t t, int h, const cuot_block *delta,
                            cuot_block *leaves_d, cuot_block *lsum_d,
                            cuot_block *rsum_d, cuot_block *secret_sum_d,
                            void *stream);
int cuot_ferret_pprf_recver(cuot_ctx *ctx, const cuot_block *mc_d,
                            const uint8_t *choice_d,
                            const cuot_block *secret_sum_d, uint64_t t, int h,
                            cuot_block *leaves_d, void *stream);

/* Allocation-free Ferret sender.  No counterpart in the reference.
 * Same arguments and results as cuot_ferret_pprf_sender, without a context,
 * on the calling thread's current device, and it never allocates device
 * memory (no cudaMalloc/cudaFree, no allocating library call).  It is for
 * callers that cannot allocate at call time: a serving process whose HBM is
 * owned by its own pool allocator, or a latency-critical path that cannot
 * afford the implicit device synchronisation of cudaMalloc/cudaFree.
 * Scratch lives in a fixed 16 MiB device array inside libcuot (held by every
 * GPU that loads the library until the process exits), so t * 2^h may not
 * exceed 2^20 leaves; larger requests return CUOT_EINVAL.
 * The first call on a device does a one-time set-up (uploads the AES keys
 * and table, looks up the array's device address), which synchronises; make
 * that first call before any stream capture.  All calls on a device share
 * the one scratch array: calls that overlap on the GPU (other streams, other
 * host threads) race, so order them (e.g. one stream). */
int cuot_ferret_pprf_sender_noalloc(const cuot_block *roots_d, uint64_t t,
                                    int h, const cuot_block *delta,
                                    cuot_block *leaves_d, cuot_block *lsum_d,
                                    cuot_block *rsum_d,
                                    cuot_block *secret_sum_d, void *stream);

/* ---- Ferret primal LPN -----------------------------------------------------
 * e_io_d[i] ^= XOR_{j<d} kk_d[idx(i, j)] for i < n, with the index matrix of
 * emp-ot LpnF2::task over [0, n) (lpn_f2.h:46-79) under AES key `seed`.
 * Replaces cuda_primal_lpn (dev_layer.cu:161-186).  1 <= d <= 32,
 * 1 <= k < 2^31. */
int cuot_lpn_primal(cuot_ctx *ctx, const uint8_t seed[16],
                    const cuot_block *kk_d, int64_t k, int d,
                    cuot_block *e_io_d, int64_t n, void *stream);
/* Rows [row_lo, row_hi) of the same n-row LPN (e_rows_d holds those rows),
 * for splitting the rows over GPUs with kk replicated (the reference splits
 * rows per GPU and offsets the counters, dev_layer.cu:166-176).  row_lo is a
 * multiple of 4; row_hi is a multiple of 4 or n.  Shards computed this way
 * are bit-identical to the unsplit result. */
int cuot_lpn_primal_range(cuot_ctx *ctx, const uint8_t seed[16],
                          const cuot_block *kk_d, int64_t k, int d,
                          cuot_block *e_rows_d, int64_t row_lo,
                          int64_t row_hi, int64_t n, void *stream);
/* Both roles of one extension when they run on the same GPU (a dealer, a
 * test harness, the batched engine and server, which hold both parties):
 * the two calls LpnF2::compute makes, one per party with the seed ALICE sends
 * BOB (lpn_f2.h:81-101), share the public index matrix, so it is generated
 * once and each index gathers from both kk_send_d and kk_recv_d.  Equal to
 * cuot_lpn_primal on (kk_send_d, e_send_io_d) and on (kk_recv_d,
 * e_recv_io_d); the two row arrays must not alias. */
int cuot_lpn_primal_dual(cuot_ctx *ctx, const uint8_t seed[16],
                         const cuot_block *kk_send_d, const cuot_block *kk_recv_d,
                         int64_t k, int d, cuot_block *e_send_io_d,
                         cuot_block *e_recv_io_d, int64_t n, void *stream);

/* ---- SOT PPRF ----------------------------------------------------------------
 * Structure of SOTSender/SOTRecver::seed_expand (silent/sender.cu:76-108,
 * silent/recver.cu:124-163) with the emp-ot node function above.
 * Sender: base0_d/base1_d [h][t] base-OT messages; out m0_d/m1_d [h+1][t]:
 *   m0[d] = base0[d] ^ L_d, m1[d] = base1[d] ^ R_d (d < h),
 *   m0[h] = base0[h-1] ^ R_{h-1} ^ delta, m1[h] = base1[h-1] ^ L_{h-1} ^ delta.
 * Receiver: mc_d [h][t] chosen base-OT messages, choice_d [h][t] bytes;
 *   out leaves = sender leaves except the punctured one = sender leaf ^ delta.
 */
int cuot_sot_pprf_sender(cuot_ctx *ctx, const cuot_block *roots_d, uint64_t t,
                         int h, const cuot_block *delta,
                         const cuot_block *base0_d, const cuot_block *base1_d,
                         cuot_block *leaves_d, cuot_block *m0_d,
                         cuot_block *m1_d, void *stream);
int cuot_sot_pprf_recver(cuot_ctx *ctx, const cuot_block *m0_d,
                         const cuot_block *m1_d, const cuot_block *mc_d,
                         const uint8_t *choice_d, uint64_t t, int h,
                         cuot_block *leaves_d, void *stream);

/* ---- bit transpose -----------------------------------------------------------
 * Mat::bit_transpose (gpu/gpu_matrix.cu:95-121): input `rows` rows of
 * `row_bytes` bytes; output row (c - col_lo) bit r = input row r bit c for
 * c in [col_lo, col_hi).  Output rows are rows/8 bytes.  rows % 8 == 0,
 * col_lo % 8 == 0, col_hi % 8 == 0, col_hi <= 8 * row_bytes.  Any alignment
 * of in_d / out_d works; 16-byte-aligned pointers with 16-byte rows -> 128
 * planes (rows % 128 == 0), or 128 planes -> 16-byte rows (col_lo == 0,
 * col_hi % 128 == 0, row_bytes % 16 == 0), take the fastest kernels. */
int cuot_bit_transpose(cuot_ctx *ctx, const void *in_d, uint64_t rows,
                       uint64_t row_bytes, uint64_t col_lo, uint64_t col_hi,
                       void *out_d, void *stream);

/* ---- host transfer -----------------------------------------------------------
 * Copies `bytes` of device memory to mapped pinned host memory with the SMs'
 * own stores instead of a copy engine.  For the small results a caller needs
 * on the host in the middle of a step (the level and secret sums that
 * cuda_mpcot_sender returns, dev_layer.cu:40-41): on B200 a DMA copy waits
 * behind every copy already queued on the engines, in either direction, so
 * with the previous step's outputs still streaming to the host (hundreds of
 * MB) it would hold the step up; this copy does not queue there.  dst_h must
 * be pinned and mapped (cudaHostAlloc / cudaMallocHost, or cudaHostRegister
 * with cudaHostRegisterMapped); otherwise CUOT_EINVAL.  Stream-ordered on the
 * current device; the bytes are in host memory once the stream passes an
 * event recorded after the call.  No counterpart call in the reference. */
int cuot_copy_to_host(const void *src_d, void *dst_h, uint64_t bytes, void *stream);

/* ---- Ferret session: set-up + rcot buffer loop -------------------------------
 * FerretCOT's data flow (ferret_cot.hpp:99-210) with both parties on one GPU
 * and an ideal transport between them (the receiver's MPCOT OT messages are
 * selected by the LSB of its pre-COTs, as OTPre over the pre-COTs would
 * deliver them; secret sums and the LPN seed are handed over directly).
 * Parameters as PrimalLPNParameter (constants.h:9-25).  create() runs the
 * set-up extension on dealer base COTs; every extension consumes M = k + t*h
 * + 128 pre-COTs of each role, writes n COTs of each role into ot_s_d /
 * ot_r_d (caller-owned, n blocks each; w = v ^ x * delta, x = LSB(w)) and
 * keeps the last M as the next pre-COTs on the device.  rcot() returns num
 * COTs of each role (device), extending whenever the buffer runs dry.  All
 * randomness comes from `seed` (AES-CTR blocks, as cuot_prg_fill).  Calls are
 * stream-ordered on `stream`; create() synchronises once. */
typedef struct {
  int64_t n, t, k, log_bin_sz, n_pre, t_pre, k_pre, log_bin_sz_pre;
} cuot_ferret_param;
typedef struct {
  int64_t M, ot_limit, ot_used, extensions;
  cuot_block delta;
} cuot_ferret_session_state;
typedef struct cuot_ferret_session cuot_ferret_session;
int cuot_ferret_session_create(cuot_ctx *ctx, const cuot_ferret_param *param,
                               const uint8_t seed[16], int d, cuot_block *ot_s_d,
                               cuot_block *ot_r_d, void *stream,
                               cuot_ferret_session **out);
int cuot_ferret_session_extend(cuot_ferret_session *s);
int cuot_ferret_session_rcot(cuot_ferret_session *s, int64_t num,
                             cuot_block *v_d, cuot_block *w_d);
int cuot_ferret_session_info(const cuot_ferret_session *s,
                             cuot_ferret_session_state *out);
int cuot_ferret_session_destroy(cuot_ferret_session *s);

/* ---- Ferret malicious consistency check ------------------------------------
 * out_d[j] = sum_{i < 2^h} seed_j^(i+1) * leaves[j*2^h + i] over GF(2^128)
 * (natural bit order, mod x^128 + x^7 + x^2 + x + 1), for every tree j < t:
 * the per-tree check values of SPCOT_Sender/SPCOT_Recver::
 * consistency_check_msg_gen (spcot_sender.h:88-98, spcot_recver.h:97-107),
 * all trees in one launch.  seeds_d[j] = the first 16 bytes of
 * Hash(secret_sum_j) (host side, as the reference derives it).  The sender
 * passes its leaves (V_j), the receiver its leaves (W_j); then
 * V_j ^ W_j = seed_j^(alpha_j + 1) * Delta for the punctured leaf alpha_j. */
int cuot_ferret_chi_sum(cuot_ctx *ctx, const cuot_block *leaves_d, uint64_t t,
                        int h, const cuot_block *seeds_d, cuot_block *out_d,
                        void *stream);

/* ---- SOT quasi-cyclic dual LPN ------------------------------------------------
 * a = n bits of AES_key(make_block counters) (silent/quasi_cyclic.cu:57-66,
 * gpu/gpu_ops.cu:102-109).  encode: every plane r (n bits, planes
 * consecutive) becomes a * plane_r mod (x^n - 1) over GF(2), exactly
 * (replaces the float cuFFT path of QuasiCyclic::encode_dense,
 * quasi_cyclic.cu:118-128).  n a power of two in [2^10, 2^25].  The
 * product is an fp64 FFT carrying four planes per transform for n <= 2^22
 * (exact: the rounding error of the convolution stays below 1/2), GF(2)
 * Karatsuba over that FFT for dual LPNs at 2^23 and 2^24, and a number-
 * theoretic transform mod 469762049 otherwise (CUOT_TUNE_QC_BACKEND).
 * encode_sparse: out = a * e mod (x^n - 1), e = indicator of pos_d[0..w)
 * (QuasiCyclic::encode_sparse, quasi_cyclic.cu:130-161).
 * dual_lpn: io_d holds n blocks; block j becomes XOR_{i: a_i = 1}
 * io[(j - i) mod n], i.e. transpose -> encode 128 planes -> transpose back
 * (SOTSender::dual_lpn, silent/sender.cu:110-119). */
int cuot_qc_gen_a(cuot_ctx *ctx, const uint8_t key[16], uint64_t n,
                  uint64_t *a_d, void *stream);
int cuot_qc_encode(cuot_ctx *ctx, const uint64_t *a_d, uint64_t *planes_io_d,
                   uint64_t n, int nplanes, void *stream);
int cuot_qc_encode_sparse(cuot_ctx *ctx, const uint64_t *a_d,
                          const uint64_t *pos_d, int weight, uint64_t n,
                          uint64_t *out_d, void *stream);
int cuot_sot_dual_lpn(cuot_ctx *ctx, const uint64_t *a_d, cuot_block *io_d,
                      uint64_t n, void *stream);
/* Rate-1/2 dual LPN over 2n noise blocks e = (e0, e1):
 *   out[i] = e0[i] ^ (a * e1 mod x^n - 1)[i]   per bit plane, i < n.
 * in_d: 2n blocks (the expansion of 2t trees); out_d: n blocks (may equal
 * in_d).  The reference SOT encodes only the rate-1 form
 * (quasi_cyclic.cu:118-128); this is the 2n-leaf variant of the same code,
 * built from the same exact product. */
int cuot_sot_dual_lpn_r2(cuot_ctx *ctx, const uint64_t *a_d, const cuot_block *in_d,
                         uint64_t n, cuot_block *out_d, void *stream);
/* Receiver choice bits of the rate-1/2 form: out = e0 ^ a * e1 for the
 * sparse 2n-bit noise e given by its nonzero positions pos_d[0..weight) in
 * [0, 2n) (positions < n are e0, the rest e1; others are ignored). */
int cuot_qc_encode_sparse_r2(cuot_ctx *ctx, const uint64_t *a_d,
                             const uint64_t *pos_d, int weight, uint64_t n,
                             uint64_t *out_d, void *stream);

/* QC plan: the counterpart of the QuasiCyclic object (quasi_cyclic.h:8-26,
 * ctor quasi_cyclic.cu:51-106), which transforms `a` once and reuses it for
 * every encode.  plan_create transforms a_d (n bits) on `stream` and keeps
 * the transform in its own device buffer; the twiddle tables are cached in
 * the context (the first use of a size synchronises the device).
 * plan_encode / plan_dual_lpn do what cuot_qc_encode / cuot_sot_dual_lpn do
 * without re-transforming `a`.  set_batch bounds how many planes share one
 * intermediate pass (4 bytes per coefficient per plane of scratch). */
typedef struct cuot_qc_plan cuot_qc_plan;
int cuot_qc_plan_create(cuot_ctx *ctx, const uint64_t *a_d, uint64_t n,
                        void *stream, cuot_qc_plan **out);
int cuot_qc_plan_destroy(cuot_qc_plan *plan);
int cuot_qc_plan_set_batch(cuot_qc_plan *plan, int planes_per_batch);
int cuot_qc_plan_encode(cuot_qc_plan *plan, uint64_t *planes_io_d,
                        int nplanes, void *stream);
int cuot_qc_plan_dual_lpn(cuot_qc_plan *plan, cuot_block *io_d, void *stream);
int cuot_qc_plan_dual_lpn_r2(cuot_qc_plan *plan, const cuot_block *in_d,
                             cuot_block *out_d, void *stream);

/* ---- batched engine ------------------------------------------------------
 * Many OT-extension instances of uneven n and depth, both roles each, run as
 * one device program of two branches: Ferret (one
 * persistent PPRF launch over all Ferret sender trees -- per-tree work queue,
 * deepest trees first --, one over the receivers, one persistent LPN launch
 * over all Ferret rows, both roles of a row from one index computation) and
 * SOT (the same PPRF launches over the SOT trees, then for each transform
 * size one set of QC transform passes spanning the planes of every instance
 * of that size; cfg.schedule chooses whether the parts overlap).  On first run
 * the whole program is captured into a CUDA graph (cfg.use_graph) and
 * replayed afterwards.
 * No counterpart call in the reference, which runs one instance per call
 * (FerretCOT::extend, ferret_cot.hpp:80-91; SOT roles, silent/roles.h).
 * Each item produces v (sender) and w (receiver) with w = v except on the
 * COT positions (Ferret: w_i = v_i ^ delta at the punctured leaves' images
 * after LPN; SOT: w_j = v_j ^ c_j * delta with c = a * e). */
#define CUOT_KIND_FERRET 0
#define CUOT_KIND_SOT 1

typedef struct {
  int kind;                       /* CUOT_KIND_* */
  int h;                          /* tree depth, 1..20 */
  uint64_t t;                     /* trees; n = t << h */
  cuot_block delta;               /* correlation delta */
  const cuot_block *roots_d;      /* [t] sender tree roots */
  const uint8_t *choice_d;        /* Ferret [t][h], SOT [h][t] */
  cuot_block *v_d;                /* [n] out: sender output */
  cuot_block *w_d;                /* [n] out: receiver output */
  /* Ferret */
  int64_t k;                      /* LPN inputs */
  int d;                          /* LPN terms per row */
  uint8_t lpn_seed[16];
  const cuot_block *kk_send_d;    /* [k] */
  const cuot_block *kk_recv_d;    /* [k] */
  /* SOT (n a power of two in [2^10, 2^25]) */
  const cuot_block *base0_d;      /* [h][t] sender base-OT messages */
  const cuot_block *base1_d;      /* [h][t] */
  const cuot_block *mc_d;         /* [h][t] receiver's chosen messages */
  const uint64_t *a_d;            /* [n/64] QC polynomial */
  const uint64_t *punct_d;        /* [t] receiver's punctured leaf indices */
  uint64_t *cbits_d;              /* [n/64] out: receiver choice bits a*e */
} cuot_batch_item;

typedef struct {
  int pprf_threads;        /* threads per tree CTA: 128 or 256 (0: 256) */
  int ctas_per_sm;         /* persistent PPRF/LPN grid: CTAs per SM (0: 3) */
  int lpn_rows_per_task;   /* LPN work-queue granularity, multiple of 4 (0: 65536) */
  int qc_planes_per_pass;  /* planes per QC pass (0: 512 MiB of intermediate) */
  int use_graph;           /* capture into a CUDA graph on first run */
  int schedule;            /* CUOT_BATCH_SERIAL (0, default): every launch
                              in one chain on the caller's stream;
                              CUOT_BATCH_FORK_FERRET: the Ferret branch on a
                              stream of its own beside the SOT chain;
                              CUOT_BATCH_FORK_SIZES: the Ferret branch and each
                              SOT transform size side by side.  On B200 the
                              chain was fastest (64-instance mix: 86.1 ms
                              against 88.7 and 97.3 ms). */
} cuot_batch_config;
#define CUOT_BATCH_SERIAL 0
#define CUOT_BATCH_FORK_FERRET 1
#define CUOT_BATCH_FORK_SIZES 2

typedef struct cuot_batch cuot_batch;
/* Validates the items, allocates the batch's device state and transforms
 * every SOT item's `a` (synchronises the device). */
int cuot_batch_create(cuot_ctx *ctx, const cuot_batch_item *items, int count,
                      const cuot_batch_config *cfg, cuot_batch **out);
/* One step: every item, both roles, on `stream` (the same stream for every
 * run when graphs are used). */
int cuot_batch_run(cuot_batch *b, void *stream);
/* The same items through the single-instance entry points, one instance at
 * a time (the plain path the batched form is compared with). */
int cuot_batch_run_plain(cuot_batch *b, void *stream);
int cuot_batch_destroy(cuot_batch *b);
/* Kernels launched by one batched run (known after the first run). */
int cuot_batch_kernels_per_run(const cuot_batch *b);
/* Makes `stream` wait until item `item`'s outputs (v, w and, for SOT, cbits)
 * are final in the batched run last enqueued (cuot_batch_run or
 * cuot_batch_run_phases), which for all but the last items is before the run
 * ends: the Ferret items are final after the LPN, each SOT size class after
 * its own encodes.  A host copy of an item can start there.  Waits on nothing
 * before the first run.  Does not block the host. */
int cuot_batch_wait_item(cuot_batch *b, int item, void *stream);
/* The item's completion point, in the order a CUOT_BATCH_SERIAL run reaches
 * them: 0 for Ferret items, then 1, 2, ... for the SOT sizes, largest first.
 * Items of one rank complete together; -1 for a bad argument. */
int cuot_batch_item_rank(const cuot_batch *b, int item);
/* Diagnostic: the batched program without a graph, timed per phase with
 * events (synchronises): phase_ms[0..3] = sender PPRF (+ OT selection),
 * receiver PPRF, LPN, SOT encodes. */
int cuot_batch_run_phases(cuot_batch *b, void *stream, float *phase_ms);

/* ---- Serving: continuous batching of OT-extension requests ------------------
 * No counterpart in the reference, which runs one instance per call.  Each
 * request is one extension with both roles (Ferret: MPCOT + primal LPN with
 * d = 10 and k inputs; SOT: PPRF + exact QC dual LPN + the receiver's choice
 * bits a*e), its inputs derived on the device from `seed`: AES-CTR blocks
 * [0, t) are the roots, the next ceil(t*h/16) blocks' byte LSBs the choice
 * bits (Ferret [t][h], SOT [h][t]), then kk_send, kk_recv (k blocks each) or
 * base0, base1 ([h][t] each).  Its scalars are blocks 2^40 + {0, 1, 2}
 * (cuot_request_scalars).  The server keeps `slots` contexts busy, admitting
 * queued requests in arrival order while a slot is free and the request's
 * footprint fits budget_bytes minus the slots' reserved scratch; at most
 * max_big (>= 1) requests with n >= big_n (0: no limit) run at once, and
 * smaller ones may pass a big one waiting for that reason.  Requests with
 * n < high_priority_below_n run on a high-priority stream.  A request waiting
 * longer than max_queue_wait seconds (0: forever) times out; one that can
 * never run (bad shape, n > 2^max_log_n, footprint above the budget) is
 * rejected.  Results: v_h / w_h (n blocks) and c_h (SOT, n bits) when non-null
 * (pinned host memory keeps the copies asynchronous); t_admit and t_done are
 * seconds from the start of run().  With dry_run_service_s > 0 no device work
 * is done: every request takes that long (host-only scheduling tests). */
#define CUOT_REQ_PENDING 0
#define CUOT_REQ_QUEUED 1
#define CUOT_REQ_RUNNING 2
#define CUOT_REQ_DONE 3
#define CUOT_REQ_TIMEOUT 4
#define CUOT_REQ_CANCELLED 5
#define CUOT_REQ_REJECTED 6
#define CUOT_REQ_FAILED 7
typedef struct {
  int kind;           /* CUOT_KIND_* */
  int h;              /* tree depth */
  uint64_t t;         /* trees; n = t << h */
  int64_t k;          /* Ferret LPN inputs */
  uint8_t seed[16];
  double arrival;     /* seconds from the start of run() */
  cuot_block *v_h;    /* [n] out (optional) */
  cuot_block *w_h;    /* [n] out (optional) */
  uint64_t *c_h;      /* [n/64] out (optional, SOT) */
  int status;         /* out: CUOT_REQ_* */
  double t_admit;     /* out: -1 if never admitted */
  double t_done;      /* out: -1 if not done */
} cuot_request;
typedef struct {
  int slots;                       /* concurrent requests (contexts), 1..256 */
  int max_log_n;                   /* largest request, 10..25 (0: 24) */
  double budget_bytes;             /* device bytes for slots' scratch + requests */
  double max_queue_wait;           /* seconds; 0: no timeout */
  uint64_t big_n;                  /* 0: no big-request limit */
  int max_big;
  uint64_t high_priority_below_n;  /* 0: one stream priority */
  double dry_run_service_s;        /* > 0: host-only mode */
} cuot_server_config;
typedef struct {
  double wall_s;          /* run() duration */
  double max_used_bytes;  /* peak footprint of admitted requests */
} cuot_server_stats;
typedef struct cuot_server cuot_server;
/* Creates the slots' contexts and streams, reserves their scratch and builds
 * the QC tables of every size up to 2^max_log_n (synchronises). */
int cuot_server_create(int device, const cuot_server_config *cfg,
                       cuot_server **out);
/* Device bytes reserved by the slots (taken from the budget). */
int cuot_server_reserved_bytes(const cuot_server *s, uint64_t *out);
/* Replaces the scheduling policy (budget_bytes, max_queue_wait, big_n,
 * max_big, high_priority_below_n) for later run() calls; the other fields
 * are fixed at creation. */
int cuot_server_configure(cuot_server *s, const cuot_server_config *cfg);
/* Cancels reqs[index] of the current (or next) run() if it is still queued;
 * callable from another thread while run() is in progress. */
int cuot_server_cancel(cuot_server *s, int index);
/* Serves `count` requests until each is done, timed out, cancelled or
 * rejected (blocks).  Returns CUOT_ECUDA if a request's device work failed
 * (that and the running requests end as CUOT_REQ_FAILED). */
int cuot_server_run(cuot_server *s, cuot_request *reqs, int count,
                    cuot_server_stats *stats);
int cuot_server_destroy(cuot_server *s);
/* Delta (LSB set), LPN seed and QC key of a request with this seed. */
int cuot_request_scalars(const uint8_t seed[16], cuot_block out[3]);
/* Device bytes a request holds while admitted. */
int cuot_request_footprint(const cuot_request *r, uint64_t *out);

#ifdef __cplusplus
}
#endif
#endif /* CUOT_H */
