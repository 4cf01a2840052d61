// ctx.cuh -- the context object behind the opaque cuot_ctx handle.
#pragma once
#include "common.cuh"

struct cuot_ctx {
  int device;
  uint32_t *t0_d;          // T0 table (256 words) for staging into shared memory
  void *scratch;           // grow-only scratch arena
  uint64_t scratch_bytes;
  void *qc_tables[32];     // NTT twiddle tables per log2(n) (qc.cu)
  void *qcf_tables[32];    // FFT twiddle tables per log2(n) (qc_fft.cu)
  int pprf_threads;        // threads per tree CTA (128 or 256)
  int qc_planes_per_pass;  // 0: automatic
  int qc_backend;          // CUOT_TUNE_QC_BACKEND value: 0 automatic, 1 NTT, 2 FFT
  int qc_streams;          // CUOT_TUNE_QC_STREAMS value: 1 or 2 (FFT group schedule)
  uint32_t *qcf_margin;    // CUOT_TUNE_QC_RECORD_MARGIN: device word, max |v - round(v)| as float bits
};

namespace cuot {
// Records a failure message for cuot_last_error() and returns `status`.
int fail(int status, const char *fmt, ...);
// Makes ctx's device current for the lifetime of the guard.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(const cuot_ctx *c) {
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};
// Returns a scratch pointer of at least `bytes` (grows the arena with
// cudaMalloc when needed; growing synchronises the device).
int scratch(cuot_ctx *ctx, uint64_t bytes, void **out);
// One-time per-device initialisation of module constants (pprf.cu).
int pprf_init_device();
// Frees the context's cached QC tables (qc.cu).
void qc_free_ctx_tables(cuot_ctx *ctx);
// Scratch bytes of the one-shot dual LPN (cuot_sot_dual_lpn, or with r2
// cuot_sot_dual_lpn_r2) of n = 2^e on ctx (qc.cu).
uint64_t qc_one_shot_dual_bytes(const cuot_ctx *ctx, int e, bool r2);
// QC helpers used by the batched engine (qc.cu).  The backend (NTT or FFT)
// of an n = 2^e encode follows the context's CUOT_TUNE_QC_BACKEND; A_hat
// and intermediate sizes depend on it.
int qc_prepare(cuot_ctx *ctx, int e);
uint64_t qc_ahat_bytes(const cuot_ctx *ctx, int e);
// Encodes of two sizes with the same lane share per-size FFT state (the
// tables' second stream, events and plane-parity words) and must not run at
// the same time; different lanes may.
int qc_lane(const cuot_ctx *ctx, int e);
uint64_t qc_y_bytes(const cuot_ctx *ctx, int e, int batch);
int qc_build_ahat(cuot_ctx *ctx, int e, const uint64_t *a_d, void *Y, void *ahat, cudaStream_t st);
int qc_encode_jobs(cuot_ctx *ctx, int e, uint64_t *planes, int njobs, const void *const *ahats,
                   void *Y, int batch, cudaStream_t st);
// n = 2^e blocks into a job's encode layout (16n bytes) and back.
int qc_job_to_layout(const cuot_ctx *ctx, int e, const cuot_block *in, void *job, cudaStream_t st);
int qc_job_from_layout(const cuot_ctx *ctx, int e, const void *job, cuot_block *out, cudaStream_t st);
int qc_default_batch(uint64_t n, int nplanes);
// FP64 FFT backend of the QC encode (qc_fft.cu): n = 2^e, 10 <= e <= kQcfMaxE.
constexpr int kQcfMaxE = 22;
// n = 2^22 packs centred planes against `a` or its complement (whichever is
// lighter); A_hat then carries a 256-byte trailer (the weight of `a`).
constexpr bool qcf_center(int e) { return e >= 22; }
constexpr uint64_t qcf_ahat_bytes(int e) { return (16ull << e) + (qcf_center(e) ? 256 : 0); }
// A_hat of each transform y of a launch: p[(first + y) / per] (4 planes per transform).
struct QcfAhatTab {
  const void *p[16];
  int first;
  int per;
  // When non-null (the context records rounding margins), the last inverse
  // pass atomically raises *margin to the largest |v - round(v)| it rounds,
  // as the bit pattern of a non-negative float.
  uint32_t *margin;
};
struct QcfTables;
bool qcf_supported(int e);
int qcf_get_tables(cuot_ctx *ctx, int e, QcfTables **out);
void qcf_free_ctx_tables(cuot_ctx *ctx);
// A_hat (n complex doubles) of `a`; Y holds 16n bytes.
int qcf_build_ahat(const QcfTables *t, const uint64_t *a_d, void *Y, void *ahat, cudaStream_t st);
// Planes p < nplanes: in + p * stride -> out + p * stride (64-bit words),
// written or XORed (accumulate); Y holds round4(batch) * 4n bytes.
int qcf_encode(const QcfTables *t, const QcfAhatTab &ahat, const uint64_t *in, uint64_t *out, uint64_t stride,
               int accumulate, int nplanes, void *Y, int batch, cudaStream_t st);
// The same encode on the tile layout (qcf_gather's output, 16n bytes per 32
// transforms), in place; batch: planes per launch group.
int qcf_encode_tiles(const QcfTables *t, const QcfAhatTab &ahat, uint32_t *tiles, int ntransforms, void *Y,
                     int batch, cudaStream_t st);
// n = 2^e blocks -> tile layout of their 128 planes, and back (optionally
// XORed with xor_in).
int qcf_gather(int e, const cuot_block *in, uint32_t *tiles, cudaStream_t st);
int qcf_scatter(int e, const uint32_t *tiles, const cuot_block *xor_in, cuot_block *out, cudaStream_t st);
// GF(2) Karatsuba over the FFT (qc_kara.cu): the dual LPN of n = 2^e,
// kQcfMaxE < e <= kQcfMaxE + kQckMaxLevels, as 3^(e - kQcfMaxE) exact
// 2^kQcfMaxE FFT dual LPNs.
constexpr int kQckMaxLevels = 2;
bool qck_supported(int e);
uint64_t qck_ahat_bytes(int e);          // the leaves' transforms
uint64_t qck_scratch_bytes(int e);       // block scratch of a dual LPN
uint64_t qck_bits_scratch_bytes(int e);  // bit scratch of the A_hat build
// bits: qck_bits_scratch_bytes(e); Y: 16 * 2^kQcfMaxE bytes.
int qck_build_ahat(const QcfTables *leaf, int e, const uint64_t *a_d, void *bits, void *Y, void *ahat,
                   cudaStream_t st);
// out = (xor_in ^) a * in blockwise (n blocks; in == out allowed); Y holds the
// leaf FFT passes' intermediate for `batch` planes.
int qck_dual_lpn(const QcfTables *leaf, int e, const void *ahat, const cuot_block *in, const cuot_block *xor_in,
                 cuot_block *out, void *scratch, void *Y, int batch, cudaStream_t st);
int transpose_launch(const void *in, uint64_t rows, uint64_t row_bytes, uint64_t col_lo,
                     uint64_t col_hi, void *out, cudaStream_t st);
}  // namespace cuot
