// qc.cu -- exact quasi-cyclic encode over GF(2)[x]/(x^n - 1) (SOT dual LPN):
// the entry points, the choice of transform per size (the fp64 FFT of
// qc_fft.cu up to 2^22, GF(2) Karatsuba over it in qc_kara.cu for dual LPNs
// at 2^23 and 2^24, the number-theoretic transform below otherwise), the
// sparse encode and the AES-CTR helpers.
//
// The reference multiplies with float32 cuFFT and recovers bits by truncating
// the unnormalised result (silent/quasi_cyclic.cu:34-49, 118-128), which is
// not exact.  Here out_r = a * b_r mod (x^n - 1) is the parity of the
// integer cyclic convolution, whose coefficients lie in [0, n]; it is
// computed exactly with a number-theoretic transform over
//   p = 7 * 2^26 + 1 = 469762049 (prime, 3 a primitive root),
// so every coefficient < n <= 2^26 < p is recovered exactly and its parity
// is the GF(2) coefficient.  n = 2^e, 10 <= e <= 26.
//
// Four-step NTT, n = N1 * N2, input index j = N2*j1 + j2, output k = k1 + N1*k2:
//   A  (columns): per plane and 8 columns j2: load bits, N1-point DIF NTT
//      over j1 (natural -> bit-reversed row label r), multiply by
//      w_n^(j2 * rev(r)), store Y[r][j2].
//   B  (rows):   per row r: N2-point DIF NTT, multiply by A_hat / n (Shoup),
//      N2-point DIT inverse NTT (bit-reversed -> natural), store.
//   C  (columns): per plane and 8 columns: multiply by w_n^-(j2 * rev(r)),
//      N1-point DIT inverse over r (-> natural j1), reduce mod p, take the
//      parity, pack 8 bits per byte.
// Butterflies use Harvey's lazy reduction (values kept in [0, 2p)) and
// Shoup multiplication by precomputed twiddles (w, floor(w * 2^32 / p)).
// A_hat is the NTT of `a` in the same (r, q) label order, computed on the
// device with passes A and B-forward; planes are processed in batches so
// the 4-byte-per-coefficient intermediate stays within a bounded footprint.
#include <cstdlib>
#include <vector>
#include "ctx.cuh"

namespace cuot {

constexpr uint32_t kP = 469762049u;
constexpr uint32_t kG = 3u;
// Launch shape of the NTT passes (compile-time knobs, swept on B200):
// threads per CTA, CTAs per SM the register budget is sized for, the unroll
// depth of the column passes' strided global loads, and the elements per
// CTA of the row pass.
#ifndef CUOT_QC_THREADS
#define CUOT_QC_THREADS 256
#endif
#ifndef CUOT_QC_MIN_BLOCKS
#define CUOT_QC_MIN_BLOCKS 4
#endif
#ifndef CUOT_QC_COL_UNROLL
#define CUOT_QC_COL_UNROLL 8
#endif
#ifndef CUOT_QC_ROW_ELEMS
#define CUOT_QC_ROW_ELEMS 8192
#endif
#ifndef CUOT_QC_ROWS_K3
#define CUOT_QC_ROWS_K3 4
#endif
#ifndef CUOT_QC_PAIR_ROWS
#define CUOT_QC_PAIR_ROWS 1
#endif
#ifndef CUOT_QC_THREADS_L11
#define CUOT_QC_THREADS_L11 256
#endif
#ifndef CUOT_QC_THREADS_L12
#define CUOT_QC_THREADS_L12 512
#endif
constexpr int kQcThreads = CUOT_QC_THREADS;
// Threads per CTA of a pass over 2^LG-point transforms: the 2048- and
// 4096-point passes hold 2-4x the shared memory per CTA, so fewer CTAs fit
// an SM; bigger CTAs keep the same threads per SM.  Registers stay at
// 64 per thread (threads x CTAs per SM = 1024).
template <int LG>
constexpr int qc_threads() {
  return LG >= 12 ? CUOT_QC_THREADS_L12 : LG >= 11 ? CUOT_QC_THREADS_L11 : kQcThreads;
}
template <int LG>
constexpr int qc_min_blocks() {
  return (kQcThreads * CUOT_QC_MIN_BLOCKS) / qc_threads<LG>() > 0 ? (kQcThreads * CUOT_QC_MIN_BLOCKS) / qc_threads<LG>() : 1;
}
constexpr int kQcColUnroll = CUOT_QC_COL_UNROLL;
constexpr int kCW = 8;  // columns per CTA in the column passes

__host__ __device__ __forceinline__ uint32_t mulmod(uint32_t a, uint32_t b) {
  return uint32_t((uint64_t)a * b % kP);
}
__host__ __device__ inline uint32_t powmod(uint32_t b, uint64_t e) {
  uint64_t r = 1, x = b;
  while (e) {
    if (e & 1) r = r * x % kP;
    x = x * x % kP;
    e >>= 1;
  }
  return uint32_t(r);
}
__host__ __device__ __forceinline__ uint2 shoup_pair(uint32_t w) {
  return make_uint2(w, uint32_t((uint64_t(w) << 32) / kP));
}
// x * w mod p, result in [0, 2p), for any x < 2^32.
__device__ __forceinline__ uint32_t shoup_mul(uint32_t x, uint2 w) {
  const uint32_t q = __umulhi(x, w.y);
  return x * w.x - q * kP;
}
__device__ __forceinline__ uint32_t red2p(uint32_t x) { return x >= 2 * kP ? x - 2 * kP : x; }
__device__ __forceinline__ unsigned brev(unsigned x, int bits) { return __brev(x) >> (32 - bits); }

// ---------------------------------------------------------------------------
// In-shared-memory transforms over `rows` rows of length N = 2^lg at row
// stride `ld` = N + 4 words (so the column kernels' row-interleaved
// accesses hit distinct banks); element i of a row lives at word swz(i), an
// XOR swizzle of its low five bits by the bits above, which keeps every radix
// pass's strided accesses conflict-free (2-way at most for some 16-point
// passes).
// The lg radix-2 stages are grouped into passes of K <= 4 stages: a thread
// loads the 2^K elements of one group into registers, runs K stages there,
// and stores them back, so shared memory is touched once per pass instead of
// once per stage.  Stage twiddles are Shoup pairs in shared memory, stored
// per stage: stage s (pairs 2^s apart) reads tw[2^s - 1 + off] =
// w_N^(off * N / 2^(s+1)) for off < 2^s, so a warp's twiddle reads are
// consecutive.  DIF forward: natural in, bit-reversed out.  DIT inverse:
// bit-reversed in, natural out (unscaled).  Values stay in [0, 2p).
__host__ __device__ constexpr int swz(int i) { return i + 3 * (i >> 5); }
// Additive padding: 3 words after every 32.  Within a radix group the
// element offsets (m << s_lo) occupy bits disjoint from the group base and
// the sum never carries across a 32-word boundary, so
// swz(base + (m << s_lo)) = swz(base) + swz(m << s_lo): the element address
// is the group's base address plus a compile-time immediate (no per-element
// arithmetic).  Conflict-free or 2-way for every pass shape used here.
// Row stride: padded length rounded to 4 (mod 32) words, so the column
// kernels' row-interleaved accesses hit distinct banks.
__host__ __device__ constexpr int padded_len(int n) {
  return (swz(n - 1) + 1) + ((4 - (swz(n - 1) + 1)) % 32 + 32) % 32;
}

// Per-plane `a` transforms for one row pass (passed by value).
constexpr int kAhatTab = 16;
struct AhatTab {
  const uint2 *p[kAhatTab];
  int per;    // planes per entry
  int first;  // plane offset of launch plane 0 inside entry 0
};
__host__ inline AhatTab single_ahat(const uint2 *a) {
  AhatTab t{};
  t.p[0] = a;
  t.per = 1 << 30;
  t.first = 0;
  return t;
}

__device__ __forceinline__ uint32_t umin2p(uint32_t a) {
  return min(a, a - 2 * kP);  // a in [0, 4p) -> [0, 2p)
}
__device__ __forceinline__ void bf_dif(uint32_t &u, uint32_t &v, uint2 w) {
  const uint32_t a = umin2p(u + v);
  v = shoup_mul(u - v + 2 * kP, w);
  u = a;
}
__device__ __forceinline__ uint32_t umin4p(uint32_t a) {
  return min(a, a - 4 * kP);  // a in [0, 8p) -> [0, 4p)
}
// DIT butterfly without reductions: u + t and u - t + 2p, t = v * w in [0, 2p).
__device__ __forceinline__ void bf_dit_lazy(uint32_t &u, uint32_t &v, uint2 w) {
  const uint32_t t = shoup_mul(v, w);
  v = u - t + 2 * kP;
  u = u + t;
}

// Group order within a row for a pass with S_LO < 5: a warp then spans
// 2^(5 - S_LO) values t of the group bits above S_LO, whose bases differ by
// multiples of 2^(S_LO + K) and (through the padding) by 3 * 2^(S_LO+K-5)
// words per step of t.  Consecutive t would put two lanes on one bank; taking
// t in steps of 2^(5 - K) (a rotation of its low bits, a bijection) spreads
// the lanes over all 32 banks.  Conflict-free for every pass of LG >= 10.
template <int LG, int K, int S_LO>
__device__ __forceinline__ int group_hi(int t) {
  constexpr int H = LG - K - S_LO, A = 5 - S_LO, SB = 5 - K;
  if constexpr (S_LO < 5 && S_LO + K >= 5 && SB > 0 && A > 0 && A + SB <= H) {
    constexpr int LB = A + SB, M = (1 << LB) - 1;
    const int low = t & M;
    return (t & ~M) | (((low << SB) | (low >> A)) & M);
  } else {
    return t;
  }
}

// The K stages of one group on NV rows at once: every twiddle is loaded once
// and applied to all NV rows (the rows of a pass share their twiddles).
template <int K, int S_LO, bool DIF, int NV>
__device__ __forceinline__ void group_stages(uint32_t (&v)[NV][1 << K], const uint2 *twg) {
  constexpr int R = 1 << K;
  if (DIF) {
#pragma unroll
    for (int j = K - 1; j >= 0; j--) {
#pragma unroll
      for (int m = 0; m < R; m++) {
        if (m & (1 << j)) continue;
        // stage s = S_LO + j reads tw[2^s - 1 + off], off = glo | low j bits of m << S_LO
        const uint2 w = twg[(1 << (S_LO + j)) - 1 + ((m & ((1 << j) - 1)) << S_LO)];
#pragma unroll
        for (int q = 0; q < NV; q++) bf_dif(v[q][m], v[q][m | (1 << j)], w);
      }
    }
  } else {
    // Lazy DIT: skip the per-butterfly reductions; with inputs in [0, 2p)
    // values grow by at most 2p per stage (u + t, u - t + 2p with t < 2p),
    // and 8p < 2^32, so three stages run unreduced; 4- and 5-stage passes
    // bring values back under 4p after their second (and fourth) stage.
    // Outputs in [0, 2p).
#pragma unroll
    for (int j = 0; j < K; j++) {
#pragma unroll
      for (int m = 0; m < R; m++) {
        if (m & (1 << j)) continue;
        const uint2 w = twg[(1 << (S_LO + j)) - 1 + ((m & ((1 << j) - 1)) << S_LO)];
#pragma unroll
        for (int q = 0; q < NV; q++) bf_dit_lazy(v[q][m], v[q][m | (1 << j)], w);
      }
      if ((K == 4 && j == 1) || (K == 5 && (j == 1 || j == 3))) {
#pragma unroll
        for (int q = 0; q < NV; q++)
#pragma unroll
          for (int m = 0; m < R; m++) v[q][m] = umin4p(v[q][m]);
      }
    }
#pragma unroll
    for (int q = 0; q < NV; q++)
#pragma unroll
      for (int m = 0; m < R; m++) v[q][m] = umin2p(umin4p(v[q][m]));
  }
}

// Groups of a pass as NV rows x (groups per row): thread w takes group g of
// rows row0 + q * rows / NV, q < NV.
template <int LG, int K, int S_LO, bool DIF, int NV>
__device__ __forceinline__ void ntt_pass_rows(uint32_t *x, int rows, int ld, const uint2 *tw,
                                              const uint2 *__restrict__ ah) {
  constexpr int R = 1 << K;
  constexpr int NGR_LG = LG - K;
  constexpr int LOWMASK = (1 << S_LO) - 1;
  const int rstep = rows / NV;
  for (int w = threadIdx.x; w < (rstep << NGR_LG); w += blockDim.x) {
    const int row = w >> NGR_LG, g = w & ((1 << NGR_LG) - 1);
    const int glo = g & LOWMASK;
    const int base = glo | (group_hi<LG, K, S_LO>(g >> S_LO) << (S_LO + K));
    const uint2 *twg = tw + glo;
    uint32_t v[NV][R];
#pragma unroll
    for (int q = 0; q < NV; q++) {
      const uint32_t *xr = x + (row + q * rstep) * ld + swz(base);
#pragma unroll
      for (int m = 0; m < R; m++) v[q][m] = xr[swz(m << S_LO)];
    }
    group_stages<K, S_LO, DIF, NV>(v, twg);
    if (DIF && S_LO == 0 && ah != nullptr) {
#pragma unroll
      for (int q = 0; q < NV; q++) {
        const uint4 *a4 = reinterpret_cast<const uint4 *>(ah + ((row + q * rstep) << LG) + base);
#pragma unroll
        for (int m = 0; m < R; m += 2) {
          const uint4 a = __ldg(a4 + m / 2);
          v[q][m] = shoup_mul(v[q][m], make_uint2(a.x, a.y));
          v[q][m + 1] = shoup_mul(v[q][m + 1], make_uint2(a.z, a.w));
        }
      }
    }
#pragma unroll
    for (int q = 0; q < NV; q++) {
      uint32_t *xr = x + (row + q * rstep) * ld + swz(base);
#pragma unroll
      for (int m = 0; m < R; m++) xr[swz(m << S_LO)] = v[q][m];
    }
  }
}

// One pass of K radix-2 stages [S_LO, S_LO + K) of a 2^LG-point transform on
// `rows` rows, everything but the row count known at compile time.  For
// LG >= 10 an even row count runs two rows per thread, so each twiddle load
// serves both (measured: n = 2^20 1.75 -> 1.69 ms per 128 planes; smaller
// transforms lose more parallelism than they save).
// ah (optional, the last DIF pass only): after its stages, element `pos` of
// row `row` is multiplied by ah[row * 2^LG + pos] (the pointwise product).
template <int LG, int K, int S_LO, bool DIF>
__device__ __forceinline__ void ntt_pass(uint32_t *x, int rows, int ld, const uint2 *tw,
                                         const uint2 *__restrict__ ah = nullptr) {
  if (CUOT_QC_PAIR_ROWS && LG >= 10 && K <= 3 && (rows & 3) == 0)
    ntt_pass_rows<LG, K, S_LO, DIF, CUOT_QC_ROWS_K3>(x, rows, ld, tw, ah);
  else if (CUOT_QC_PAIR_ROWS && LG >= 10 && (rows & 1) == 0)
    ntt_pass_rows<LG, K, S_LO, DIF, 2>(x, rows, ld, tw, ah);
  else
    ntt_pass_rows<LG, K, S_LO, DIF, 1>(x, rows, ld, tw, ah);
  __syncthreads();
}

// Full 2^LG-point transform as ceil(LG/4) passes of near-equal size (DIF
// from the top stage down, DIT from stage 0 up).  Caller has synced.
template <int LG, bool DIF, int PIDX = 0, int DONE = 0>
__device__ __forceinline__ void ntt_smem(uint32_t *x, int rows, int ld, const uint2 *tw,
                                         const uint2 *ah = nullptr) {
  constexpr int P = (LG + 3) / 4;
  if constexpr (PIDX < P) {
    constexpr int K = LG / P + (PIDX < LG % P ? 1 : 0);
    constexpr int S_LO = DIF ? (LG - DONE - K) : DONE;
    ntt_pass<LG, K, S_LO, DIF>(x, rows, ld, tw, DIF && S_LO == 0 ? ah : nullptr);
    ntt_smem<LG, DIF, PIDX + 1, DONE + K>(x, rows, ld, tw, ah);
  }
}

__device__ __forceinline__ void stage_tw(uint2 *dst, const uint2 *src, int cnt) {
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) dst[i] = __ldg(&src[i]);
}

// Pass A.  bits: plane-major, plane_words 32-bit words per plane.
// grid (N2 / kCW, nplanes_batch).  Y: [plane][N1][N2].
template <int E1>
__global__ void __launch_bounds__(qc_threads<E1>(), qc_min_blocks<E1>()) qc_col_fwd(
    const uint32_t *__restrict__ bits, uint64_t plane_words, int e2,
    const uint2 *__restrict__ tw1f, const uint2 *__restrict__ fsf, uint32_t *__restrict__ Y) {
  extern __shared__ uint32_t xs[];
  constexpr int N1 = 1 << E1, ld = padded_len(N1);
  const int N2 = 1 << e2;
  uint2 *tws = reinterpret_cast<uint2 *>(xs + kCW * ld + (kCW * ld & 1));
  stage_tw(tws, tw1f, N1 - 1);
  const int c0 = blockIdx.x * kCW;
  const uint64_t plane = blockIdx.y;
  const uint32_t *pb = bits + plane * plane_words;
#pragma unroll kQcColUnroll
  for (int j1 = threadIdx.x; j1 < N1; j1 += blockDim.x) {
    const uint64_t bit = uint64_t(j1) * N2 + c0;
    const uint32_t w = __ldg(&pb[bit >> 5]) >> (bit & 31);
#pragma unroll
    for (int c = 0; c < kCW; c++) xs[c * ld + swz(j1)] = (w >> c) & 1u;
  }
  __syncthreads();
  ntt_smem<E1, true>(xs, kCW, ld, tws);
  // x w_n^(j2 * rev(r)) on the way out; fsf is [r][j2], read coalesced
  uint32_t *Yp = Y + plane * (uint64_t(N1) << e2);
#pragma unroll kQcColUnroll
  for (int idx = threadIdx.x; idx < kCW * N1; idx += blockDim.x) {
    const int r = idx / kCW, c = idx % kCW;
    const uint64_t o = uint64_t(r) * N2 + c0 + c;
    Yp[o] = shoup_mul(xs[c * ld + swz(r)], __ldg(&fsf[o]));
  }
}

// Pass B.  grid (N1 / rows_per_cta, nplanes_batch).  mode 0: forward,
// pointwise by the plane's ahat, inverse.  mode 1: forward only (used to
// build ahat).  Plane y of the launch uses ahat.p[(ahat.first + y) / ahat.per]
// (planes of several encodes, each with its own `a`, can share a launch).
template <int E2>
__global__ void __launch_bounds__(qc_threads<E2>(), qc_min_blocks<E2>()) qc_row(
    uint32_t *__restrict__ Y, int e1, int rows_per_cta,
    const uint2 *__restrict__ tw2f, const uint2 *__restrict__ tw2i,
    AhatTab ahat_tab, int mode) {
  extern __shared__ uint32_t xs[];
  constexpr int N2 = 1 << E2, ld = padded_len(N2);
  const int N1 = 1 << e1;
  uint2 *twf = reinterpret_cast<uint2 *>(xs + rows_per_cta * ld + (rows_per_cta * ld & 1));
  uint2 *twi = twf + N2;
  stage_tw(twf, tw2f, N2 - 1);
  if (mode == 0) stage_tw(twi, tw2i, N2 - 1);
  const uint64_t plane = blockIdx.y;
  const int r0 = blockIdx.x * rows_per_cta;
  uint32_t *Yp = Y + (plane * N1 + r0) * uint64_t(N2);
  const int cnt4 = rows_per_cta * N2 / 4;
  // 4 consecutive elements per thread: they share a 32-word chunk, so one
  // padded base address serves all four
#pragma unroll 2
  for (int i4 = threadIdx.x; i4 < cnt4; i4 += blockDim.x) {
    const int i = 4 * i4;
    const uint4 q = reinterpret_cast<const uint4 *>(Yp)[i4];
    uint32_t *d = xs + (i >> E2) * ld + swz(i & (N2 - 1));
    d[0] = q.x; d[1] = q.y; d[2] = q.z; d[3] = q.w;
  }
  __syncthreads();
  if (mode == 0) {
    const uint2 *ah = ahat_tab.p[(ahat_tab.first + blockIdx.y) / ahat_tab.per] + uint64_t(r0) * N2;
    ntt_smem<E2, true>(xs, rows_per_cta, ld, twf, ah);  // forward, then x ahat / n in registers
    ntt_smem<E2, false>(xs, rows_per_cta, ld, twi);
  } else {
    ntt_smem<E2, true>(xs, rows_per_cta, ld, twf);
  }
#pragma unroll 2
  for (int i4 = threadIdx.x; i4 < cnt4; i4 += blockDim.x) {
    const int i = 4 * i4;
    const uint32_t *d = xs + (i >> E2) * ld + swz(i & (N2 - 1));
    reinterpret_cast<uint4 *>(Yp)[i4] = make_uint4(d[0], d[1], d[2], d[3]);
  }
}

// Pass C.  grid (N2 / kCW, nplanes_batch).  out: plane-major bits, written
// (accumulate == 0) or XORed into (accumulate == 1; the rate-1/2 form).
template <int E1>
__global__ void __launch_bounds__(qc_threads<E1>(), qc_min_blocks<E1>()) qc_col_inv(
    const uint32_t *__restrict__ Y, int e2, const uint2 *__restrict__ fsi,
    const uint2 *__restrict__ tw1i, uint8_t *__restrict__ out, uint64_t plane_bytes, int accumulate) {
  extern __shared__ uint32_t xs[];
  constexpr int N1 = 1 << E1, ld = padded_len(N1);
  const int N2 = 1 << e2;
  uint2 *tws = reinterpret_cast<uint2 *>(xs + kCW * ld + (kCW * ld & 1));
  stage_tw(tws, tw1i, N1 - 1);
  const int c0 = blockIdx.x * kCW;
  const uint64_t plane = blockIdx.y;
  const uint32_t *Yp = Y + plane * (uint64_t(N1) << e2);
#pragma unroll kQcColUnroll
  for (int idx = threadIdx.x; idx < kCW * N1; idx += blockDim.x) {
    const int r = idx / kCW, c = idx % kCW;
    const uint64_t o = uint64_t(r) * N2 + c0 + c;
    xs[c * ld + swz(r)] = shoup_mul(Yp[o], __ldg(&fsi[o]));  // x w_n^-(j2 * rev(r))
  }
  __syncthreads();
  ntt_smem<E1, false>(xs, kCW, ld, tws);
  uint8_t *ob = out + plane * plane_bytes;
  for (int j1 = threadIdx.x; j1 < N1; j1 += blockDim.x) {
    uint32_t byte = 0;
#pragma unroll
    for (int c = 0; c < kCW; c++) {
      uint32_t v = xs[c * ld + swz(j1)];
      v = v >= kP ? v - kP : v;  // exact coefficient in [0, n]
      byte |= (v & 1u) << c;
    }
    uint8_t *o = ob + ((uint64_t(j1) * N2 + c0) >> 3);
    *o = uint8_t(accumulate ? (*o ^ byte) : byte);
  }
}

// Table generation (one-time per n).
// Per-stage layout: entry 2^s - 1 + off (off < 2^s) = root^(off * N / 2^(s+1)).
__global__ void qc_gen_twiddles(int lg, uint32_t root, uint2 *tw) {
  const int N = 1 << lg;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N - 1; i += gridDim.x * blockDim.x) {
    const int s = 31 - __clz(i + 1), off = i + 1 - (1 << s);
    tw[i] = shoup_pair(powmod(root, uint64_t(off) * uint64_t(N >> (s + 1))));
  }
}
// Four-step twiddles, [r][j2]: entry r * N2 + j2 = wn^(j2 * rev(r)).
__global__ void qc_gen_fourstep(int e1, int e2, uint32_t wn, uint2 *fs) {
  const uint64_t n = 1ull << (e1 + e2);
  const uint64_t N2 = 1ull << e2;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t r = i >> e2, j2 = i & (N2 - 1);
    const uint64_t k1 = brev(unsigned(r), e1);
    fs[i] = shoup_pair(powmod(wn, (j2 * k1) & (n - 1)));
  }
}
// ahat[i] = pair(v * n^-1), from the forward transform of a.
__global__ void qc_make_ahat(const uint32_t *v, uint64_t n, uint32_t ninv, uint2 *ahat) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t x = v[i] % kP;
    ahat[i] = shoup_pair(mulmod(x, ninv));
  }
}

// a = n bits of AES_key(make_block(i)): block i = (lo 4*floor(i/10), hi i%10).
__global__ void qc_make_counters(Blk *b, uint64_t nb) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nb;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t lo = 4 * (i / 10), hi = i % 10;
    b[i] = Blk{{uint32_t(lo), uint32_t(lo >> 32), uint32_t(hi), uint32_t(hi >> 32)}};
  }
}

// Counter blocks of the cryptoTools PRNG stream: block i = (lo = off + i, hi = 0).
__global__ void prg_make_counters(Blk *b, uint64_t nb, uint64_t off) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nb;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t c = off + i;
    b[i] = Blk{{uint32_t(c), uint32_t(c >> 32), 0u, 0u}};
  }
}

// Sparse encode: out = XOR_i rot(a, pos_i).  Grid: x over output words (256
// consecutive words per CTA, so the reads of `a` coalesce), y over chunks of
// kSparseChunk positions staged in shared memory; each thread XORs its
// chunk's partial into out (zeroed by the caller) with one 64-bit atomic.
// r2 (rate-1/2 noise of 2n positions): positions p < n contribute x^p
// itself, positions p in [n, 2n) contribute rot(a, p - n).
constexpr int kSparseChunk = 256;
__global__ void __launch_bounds__(256) qc_sparse(const uint64_t *__restrict__ a, const uint64_t *__restrict__ pos,
                                                 int weight, uint64_t n, uint64_t *__restrict__ out, int r2) {
  __shared__ uint64_t sp[kSparseChunk];
  const uint64_t nw = n / 64;
  const int i0 = blockIdx.y * kSparseChunk;
  const int cnt = min(kSparseChunk, weight - i0);
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) sp[i] = __ldg(&pos[i0 + i]);
  __syncthreads();
  const uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  uint64_t acc = 0;
#pragma unroll 4
  for (int i = 0; i < cnt; i++) {
    uint64_t p = sp[i];
    if (r2) {
      if (p < n) {
        if ((p >> 6) == w) acc ^= 1ull << (p & 63);
        continue;
      }
      p -= n;
    }
    if (p >= n) continue;
    const uint64_t ws = p >> 6, bs = p & 63;
    // bit (64w + b) of rot(a, p) = bit (64w + b - p) mod n of a
    const uint64_t src = w >= ws ? w - ws : w + nw - ws;
    uint64_t v = __ldg(&a[src]) << bs;
    if (bs) v |= __ldg(&a[src ? src - 1 : nw - 1]) >> (64 - bs);
    acc ^= v;
  }
  if (acc) atomicXor(reinterpret_cast<unsigned long long *>(out + w), (unsigned long long)acc);
}

// Window form of the sparse encode (r2 = 0, fewer than 2^31 output words).
// Positions listed in tree order (one punctured leaf per GGM tree of 2^h
// leaves) lie close together, so the 257-word windows of `a` that a chunk's
// positions rotate into the CTA's 256 output words overlap almost entirely:
// the CTA stages their union (span + 257 words, span = the chunk's largest
// minus smallest word shift) in shared memory once, and every (word,
// position) pair then reads shared memory instead of L2.  A chunk whose
// positions spread wider than kSparseWin (any order is accepted) takes the
// global-memory loop of qc_sparse.  Positions >= n contribute nothing, as
// there.
constexpr int kSparseWin = 4608;  // words of `a` (36 KiB)
__global__ void __launch_bounds__(256) qc_sparse_win(const uint64_t *__restrict__ a, const uint64_t *__restrict__ pos,
                                                     int weight, int chunk, uint64_t n, uint64_t *__restrict__ out) {
  __shared__ uint64_t win[kSparseWin];
  __shared__ uint32_t sws[kSparseChunk];  // word shift, or ~0u for a position >= n
  __shared__ uint8_t sbs[kSparseChunk];   // bit shift
  __shared__ unsigned long long wmin, wmax;
  const uint64_t nw = n / 64;
  const int i0 = blockIdx.y * chunk;
  const int cnt = min(chunk, weight - i0);
  if (threadIdx.x == 0) {
    wmin = ~0ull;
    wmax = 0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const uint64_t p = __ldg(&pos[i0 + i]);
    if (p < n) {
      sws[i] = uint32_t(p >> 6);
      sbs[i] = uint8_t(p & 63);
      atomicMin(&wmin, (unsigned long long)(p >> 6));
      atomicMax(&wmax, (unsigned long long)(p >> 6));
    } else {
      sws[i] = ~0u;
    }
  }
  __syncthreads();
  if (wmin > wmax) return;  // no position below n in this chunk (the same for every thread)
  const uint64_t span = wmax - wmin;
  const uint64_t w = uint64_t(blockIdx.x) * 256 + threadIdx.x;
  uint64_t acc = 0;
  if (span + 257 <= uint64_t(kSparseWin)) {
    // win[j] = a[(W0 - wmax - 1 + j) mod nw], W0 = the CTA's first output word;
    // word w = W0 + t under word shift ws needs a[w - ws] = win[t + wmax - ws + 1]
    // and its lower neighbour win[t + wmax - ws], both inside [0, span + 257)
    const uint64_t start = (uint64_t(blockIdx.x) * 256 + nw - wmax - 1) % nw;
    const int len = int(span) + 257;
    for (int j = threadIdx.x; j < len; j += blockDim.x) win[j] = __ldg(&a[(start + uint64_t(j)) % nw]);
    __syncthreads();
    if (w < nw) {
      const int t1 = int(threadIdx.x) + int(wmax) + 1;
#pragma unroll 4
      for (int i = 0; i < cnt; i++) {
        const uint32_t ws = sws[i];
        if (ws == ~0u) continue;
        const int bs = sbs[i];
        const int idx = t1 - int(ws);
        uint64_t v = win[idx] << bs;
        if (bs) v |= win[idx - 1] >> (64 - bs);
        acc ^= v;
      }
    }
  } else if (w < nw) {
    for (int i = 0; i < cnt; i++) {
      const uint32_t ws32 = sws[i];
      if (ws32 == ~0u) continue;
      const uint64_t ws = ws32;
      const int bs = sbs[i];
      const uint64_t src = w >= ws ? w - ws : w + nw - ws;
      uint64_t v = __ldg(&a[src]) << bs;
      if (bs) v |= __ldg(&a[src ? src - 1 : nw - 1]) >> (64 - bs);
      acc ^= v;
    }
  }
  if (w < nw && acc) atomicXor(reinterpret_cast<unsigned long long *>(out + w), (unsigned long long)acc);
}

static int launch_sparse(const uint64_t *a_d, const uint64_t *pos_d, int weight, uint64_t n, uint64_t *out_d,
                         int r2, cudaStream_t st) {
  if (cudaMemsetAsync(out_d, 0, n / 8, st) != cudaSuccess) return launch_status(0);
  if (weight == 0) return launch_status(0);
  const uint64_t nw = n / 64;
  const unsigned gx = unsigned((nw + 255) / 256);
  const bool win = !r2 && nw < (1ull << 31);
  // Window chunk: in tree order (one position in each run of n / weight
  // bits) `chunk` consecutive positions span less than chunk * n / weight
  // bits, i.e. chunk * nw / weight words; the chunk is chosen so that this
  // fits kSparseWin - 257 (a multiple of 32 in [32, kSparseChunk]).
  int chunk = kSparseChunk;
  if (win) {
    const uint64_t sp = nw / uint64_t(weight) > 1 ? nw / uint64_t(weight) : 1;
    const uint64_t c = uint64_t(kSparseWin - 257) / sp;
    chunk = c >= uint64_t(kSparseChunk) ? kSparseChunk : c < 32 ? 32 : int(c / 32 * 32);
  }
  // at most 65,535 chunks per launch (grid y)
  const int per_launch = 65535 * chunk;
  int launches = 0;
  for (int off = 0; off < weight; off += per_launch) {
    const int wpart = weight - off < per_launch ? weight - off : per_launch;
    const dim3 grid(gx, unsigned((wpart + chunk - 1) / chunk));
    if (win)
      qc_sparse_win<<<grid, 256, 0, st>>>(a_d, pos_d + off, wpart, chunk, n, out_d);
    else
      qc_sparse<<<grid, 256, 0, st>>>(a_d, pos_d + off, wpart, n, out_d, r2);
    launches++;
  }
  return launch_status(launches);
}

// ---------------------------------------------------------------------------
struct QcTables {
  int e, e1, e2;
  uint2 *tw1f, *tw1i, *tw2f, *tw2i, *fsf, *fsi;
};

static int split_e(int e, int *e1, int *e2) {
  int a = e / 2;
  if (a > 12) a = 12;
  *e1 = a;
  *e2 = e - a;
  return CUOT_OK;
}

static int dev_alloc(void **p, size_t bytes) {
  *p = nullptr;
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ENOMEM, "QC table allocation of %zu bytes failed", bytes);
  }
  return CUOT_OK;
}

static void free_tables(QcTables *t) {
  if (!t) return;
  cudaFree(t->tw1f); cudaFree(t->tw1i); cudaFree(t->tw2f); cudaFree(t->tw2i);
  cudaFree(t->fsf); cudaFree(t->fsi);
  delete t;
}

// Builds (once per context and n) the twiddle tables.  Synchronises the
// device the first time a size is used.
static int get_tables(cuot_ctx *ctx, int e, QcTables **out) {
  if (ctx->qc_tables[e]) {
    *out = static_cast<QcTables *>(ctx->qc_tables[e]);
    return CUOT_OK;
  }
  QcTables *t = new QcTables{};
  t->e = e;
  split_e(e, &t->e1, &t->e2);
  const uint64_t n = 1ull << e, N1 = 1ull << t->e1, N2 = 1ull << t->e2;
  int st = CUOT_OK;
  if ((st = dev_alloc((void **)&t->tw1f, N1 * 8)) || (st = dev_alloc((void **)&t->tw1i, N1 * 8)) ||
      (st = dev_alloc((void **)&t->tw2f, N2 * 8)) || (st = dev_alloc((void **)&t->tw2i, N2 * 8)) ||
      (st = dev_alloc((void **)&t->fsf, n * 8)) || (st = dev_alloc((void **)&t->fsi, n * 8))) {
    free_tables(t);
    return st;
  }
  const uint32_t wn = powmod(kG, (kP - 1) >> e);
  const uint32_t wni = powmod(wn, kP - 2);
  const uint32_t w1 = powmod(wn, N2), w1i = powmod(w1, kP - 2);   // N1-th root
  const uint32_t w2 = powmod(wn, N1), w2i = powmod(w2, kP - 2);   // N2-th root
  qc_gen_twiddles<<<64, 256>>>(t->e1, w1, t->tw1f);
  qc_gen_twiddles<<<64, 256>>>(t->e1, w1i, t->tw1i);
  qc_gen_twiddles<<<64, 256>>>(t->e2, w2, t->tw2f);
  qc_gen_twiddles<<<64, 256>>>(t->e2, w2i, t->tw2i);
  qc_gen_fourstep<<<1024, 256>>>(t->e1, t->e2, wn, t->fsf);
  qc_gen_fourstep<<<1024, 256>>>(t->e1, t->e2, wni, t->fsi);
  if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    free_tables(t);
    return fail(CUOT_ECUDA, "QC table generation failed");
  }
  ctx->qc_tables[e] = t;
  *out = t;
  return CUOT_OK;
}

void qc_free_ctx_tables(cuot_ctx *ctx) {
  for (int e = 0; e < 32; e++) {
    free_tables(static_cast<QcTables *>(ctx->qc_tables[e]));
    ctx->qc_tables[e] = nullptr;
  }
  qcf_free_ctx_tables(ctx);
}

static int col_smem(const QcTables *t) {
  const int ld = padded_len(1 << t->e1);
  return (kCW * ld + 1) * 4 + (1 << t->e1) * 8;
}
static int qc_threads_rt(int lg) {
  return lg >= 12 ? CUOT_QC_THREADS_L12 : lg >= 11 ? CUOT_QC_THREADS_L11 : kQcThreads;
}
static int row_rows(const QcTables *t) {
  const int N2 = 1 << t->e2;
  int r = int(int64_t(CUOT_QC_ROW_ELEMS) * qc_threads_rt(t->e2) / kQcThreads / N2);
  if (r < 1) r = 1;
  if (r > (1 << t->e1)) r = 1 << t->e1;
  return r;
}
static int row_smem(const QcTables *t) {
  const int ld = padded_len(1 << t->e2);
  return (row_rows(t) * ld + 1) * 4 + (1 << t->e2) * 16;
}

// Compile-time transform sizes: e1 in [5, 12], e2 in [5, 14].
#define CUOT_E1_CASES(X) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)
#define CUOT_E2_CASES(X) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14)

static int set_attrs(const QcTables *t) {
  (void)t;
  static bool done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && done[dev]) return CUOT_OK;
  const int big = 200 * 1024;
  bool ok = true;
#define SET1(E)                                                                              \
  ok &= cudaFuncSetAttribute(qc_col_fwd<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, big) == cudaSuccess; \
  ok &= cudaFuncSetAttribute(qc_col_inv<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, big) == cudaSuccess;
#define SET2(E) ok &= cudaFuncSetAttribute(qc_row<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, big) == cudaSuccess;
  CUOT_E1_CASES(SET1)
  CUOT_E2_CASES(SET2)
#undef SET1
#undef SET2
  if (!ok) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "QC smem attribute failed");
  }
  if (dev < 64) done[dev] = true;
  return CUOT_OK;
}

static void launch_col_fwd(const QcTables *t, dim3 grid, cudaStream_t st, const uint32_t *bits,
                           uint64_t plane_words, uint32_t *Y) {
  switch (t->e1) {
#define L1(E) case E: qc_col_fwd<E><<<grid, qc_threads<E>(), col_smem(t), st>>>(bits, plane_words, t->e2, t->tw1f, t->fsf, Y); break;
    CUOT_E1_CASES(L1)
#undef L1
  }
}
static void launch_row(const QcTables *t, dim3 grid, cudaStream_t st, uint32_t *Y, const AhatTab &ahat, int mode) {
  switch (t->e2) {
#define L2(E) case E: qc_row<E><<<grid, qc_threads<E>(), row_smem(t), st>>>(Y, t->e1, row_rows(t), t->tw2f, t->tw2i, ahat, mode); break;
    CUOT_E2_CASES(L2)
#undef L2
  }
}
static void launch_col_inv(const QcTables *t, dim3 grid, cudaStream_t st, const uint32_t *Y, uint8_t *out,
                           uint64_t plane_bytes, int accumulate = 0) {
  switch (t->e1) {
#define L3(E) case E: qc_col_inv<E><<<grid, qc_threads<E>(), col_smem(t), st>>>(Y, t->e2, t->fsi, t->tw1i, out, plane_bytes, accumulate); break;
    CUOT_E1_CASES(L3)
#undef L3
  }
}

// Computes ahat (n Shoup pairs) from a (n bits) using Y (n words) as scratch.
static int build_ahat(const QcTables *t, const uint64_t *a_d, uint32_t *Y, uint2 *ahat,
                      cudaStream_t st) {
  const int N1 = 1 << t->e1, N2 = 1 << t->e2;
  const uint64_t n = 1ull << t->e;
  launch_col_fwd(t, dim3(N2 / kCW, 1), st, reinterpret_cast<const uint32_t *>(a_d), n / 32, Y);
  launch_row(t, dim3(N1 / row_rows(t), 1), st, Y, single_ahat(nullptr), 1);
  const uint32_t ninv = powmod(uint32_t(n % kP), kP - 2);
  qc_make_ahat<<<1024, 256, 0, st>>>(Y, n, ninv, ahat);
  return launch_status(3);
}

int transpose_launch(const void *in, uint64_t rows, uint64_t row_bytes, uint64_t col_lo,
                     uint64_t col_hi, void *out, cudaStream_t st);

// Encodes `nplanes` planes of n bits in batches: plane p is read from
// in + p * stride (64-bit words) and its product written to (accumulate:
// XORed into) out + p * stride.  in == out encodes in place.
static int encode_planes_strided(const QcTables *t, const uint2 *ahat, const uint64_t *in,
                                 uint64_t *out, uint64_t stride, int accumulate, int nplanes,
                                 uint32_t *Y, int batch, cudaStream_t st) {
  const int N1 = 1 << t->e1, N2 = 1 << t->e2;
  for (int p0 = 0; p0 < nplanes; p0 += batch) {
    const int nb = nplanes - p0 < batch ? nplanes - p0 : batch;
    launch_col_fwd(t, dim3(N2 / kCW, nb), st, reinterpret_cast<const uint32_t *>(in + uint64_t(p0) * stride),
                   stride * 2, Y);
    launch_row(t, dim3(N1 / row_rows(t), nb), st, Y, single_ahat(ahat), 0);
    launch_col_inv(t, dim3(N2 / kCW, nb), st, Y, reinterpret_cast<uint8_t *>(out + uint64_t(p0) * stride),
                   stride * 8, accumulate);
  }
  return launch_status(3 * ((nplanes + batch - 1) / batch));
}

static int check_n(uint64_t n, int *e) {
  if (n < 1024 || n > (1ull << 25) || (n & (n - 1)))
    return fail(CUOT_EINVAL, "QC n=%llu must be a power of two in [2^10, 2^25]",
                (unsigned long long)n);
  *e = __builtin_ctzll(n);
  return CUOT_OK;
}

// Planes per batch: up to 512 MiB of 4-byte-per-plane intermediate.
// Measured on B200 with the NTT (n = 2^20 / 2^22, one role): 64 MiB batches
// 2.02 / 9.19 ms, 512 MiB batches 1.83 / 7.96 ms -- more CTAs per launch
// outweigh the intermediate spilling out of L2.
static int default_batch(uint64_t n, int nplanes) {
  uint64_t b = (512ull << 20) / (4 * n);
  if (b < 1) b = 1;
  if (b > uint64_t(nplanes)) b = nplanes;
  return int(b);
}

// ---- backend selection -------------------------------------------------------
// Transform of the dual LPN of n = 2^e: the fp64 FFT (qc_fft.cu) up to 2^22,
// GF(2) Karatsuba over it (qc_kara.cu) for 2^23 and 2^24, the NTT above and
// whenever the context asks for it.  Plane encodes (cuot_qc_encode and
// cuot_qc_plan_encode) take the FFT or the NTT.
enum QcKind { kQcNtt = 0, kQcFft = 1, kQcKara = 2 };

static QcKind dual_kind(const cuot_ctx *ctx, int e) {
  if (ctx->qc_backend == 1) return kQcNtt;
  if (qcf_supported(e)) return kQcFft;
  if (qck_supported(e)) return kQcKara;
  return kQcNtt;
}

static QcKind plane_kind(const cuot_ctx *ctx, int e) { return dual_kind(ctx, e) == kQcFft ? kQcFft : kQcNtt; }

// Intermediate bytes of a pass over `batch` planes: 4 bytes per plane and
// coefficient for both transforms (the FFT packs 4 planes in 16 bytes, in
// whole transforms, and builds A_hat in one 16n-byte transform).
static uint64_t y_bytes(bool fft, int e, int batch) {
  if (!fft) return uint64_t(batch) << (e + 2);
  uint64_t b = (uint64_t(batch) + 3) & ~3ull;
  return (b < 4 ? 4 : b) << (e + 2);
}

// Planes per pass of the Karatsuba leaves (2^22-point FFTs).
static int leaf_batch(const cuot_ctx *ctx) {
  return ctx->qc_planes_per_pass > 0 ? ctx->qc_planes_per_pass : default_batch(1ull << kQcfMaxE, 128);
}

// Bytes of A_hat: NTT n Shoup pairs; FFT n complex doubles; Karatsuba the
// 3^L leaf transforms, followed (with_planes) by the NTT's for plane encodes.
static uint64_t ahat_bytes(QcKind k, int e, bool with_planes) {
  if (k == kQcFft) return qcf_ahat_bytes(e);
  if (k == kQcKara) return qck_ahat_bytes(e) + (with_planes ? 8ull << e : 0);
  return 8ull << e;
}

// Scratch of the A_hat build.
static uint64_t ahat_scratch_bytes(QcKind k, int e) {
  if (k == kQcFft) return 16ull << e;
  if (k == kQcKara) {
    const uint64_t kb = qck_bits_scratch_bytes(e) + (16ull << kQcfMaxE);
    return kb > (4ull << e) ? kb : (4ull << e);
  }
  return 4ull << e;
}

// Scratch of a dual LPN (rate 1, or rate 1/2 with r2): the planes / tile
// words (and the 2n-bit planes of the rate-1/2 form) or the Karatsuba
// split blocks, then the pass intermediate.
static uint64_t dual_scratch_bytes(const cuot_ctx *ctx, QcKind k, int e, int batch, bool r2) {
  if (k == kQcKara) return qck_scratch_bytes(e) + y_bytes(true, kQcfMaxE, leaf_batch(ctx));
  return ((r2 ? 32ull : 16ull) << e) + y_bytes(k == kQcFft, e, batch);
}
static uint64_t dual_y_offset(QcKind k, int e, bool r2) {
  if (k == kQcKara) return qck_scratch_bytes(e);
  return (r2 ? 32ull : 16ull) << e;
}

struct QcEngine {
  QcKind kind;
  QcTables *t;   // NTT tables (NTT, and Karatsuba plans' plane encodes)
  QcfTables *f;  // FFT tables (FFT: of n; Karatsuba: of the 2^22 leaves)
};

static int engine(cuot_ctx *ctx, int e, QcKind kind, QcEngine *g) {
  g->kind = kind;
  g->t = nullptr;
  g->f = nullptr;
  if (kind == kQcFft) return qcf_get_tables(ctx, e, &g->f);
  if (kind == kQcKara) CUOT_TRY(qcf_get_tables(ctx, kQcfMaxE, &g->f));
  CUOT_TRY(get_tables(ctx, e, &g->t));
  return set_attrs(g->t);
}

static QcfAhatTab single_tab(const void *ahat) {
  QcfAhatTab tab{};
  tab.p[0] = ahat;
  tab.per = 1 << 30;
  return tab;
}

// A_hat of `a` into ahat (ahat_bytes(kind, e, with_planes)); scr holds
// ahat_scratch_bytes(kind, e).
static int eng_ahat(const QcEngine &g, int e, const uint64_t *a_d, void *scr, void *ahat, bool with_planes,
                    cudaStream_t st) {
  if (g.kind == kQcFft) return qcf_build_ahat(g.f, a_d, scr, ahat, st);
  if (g.kind == kQcKara) {
    const uint64_t bb = qck_bits_scratch_bytes(e);
    CUOT_TRY(qck_build_ahat(g.f, e, a_d, scr, static_cast<uint8_t *>(scr) + bb, ahat, st));
    if (!with_planes) return CUOT_OK;
    ahat = static_cast<uint8_t *>(ahat) + qck_ahat_bytes(e);
  }
  return build_ahat(g.t, a_d, static_cast<uint32_t *>(scr), static_cast<uint2 *>(ahat), st);
}

// Planes p < nplanes: in + p * stride -> out + p * stride (64-bit words),
// written or XORed into (accumulate).  A Karatsuba plan encodes planes with
// the NTT A_hat stored after its leaves.
static int eng_encode(const QcEngine &g, int e, const void *ahat, const uint64_t *in, uint64_t *out, uint64_t stride,
                      int accumulate, int nplanes, void *Y, int batch, cudaStream_t st) {
  if (g.kind == kQcFft) return qcf_encode(g.f, single_tab(ahat), in, out, stride, accumulate, nplanes, Y, batch, st);
  if (g.kind == kQcKara) ahat = static_cast<const uint8_t *>(ahat) + qck_ahat_bytes(e);
  return encode_planes_strided(g.t, static_cast<const uint2 *>(ahat), in, out, stride, accumulate, nplanes,
                               static_cast<uint32_t *>(Y), batch, st);
}

// Dual LPN of n blocks: out = (xor_in ^) a * in blockwise; r2 = the rate-1/2
// form (in holds 2n blocks: out = in[0, n) ^ a * in[n, 2n)).  scr holds
// dual_scratch_bytes.
static int eng_dual(cuot_ctx *ctx, const QcEngine &g, int e, const void *ahat, const cuot_block *in, cuot_block *out,
                    bool r2, uint8_t *scr, int batch, cudaStream_t st) {
  const uint64_t n = 1ull << e;
  void *Y = scr + dual_y_offset(g.kind, e, r2);
  const cuot_block *src = r2 ? in + n : in;
  const cuot_block *xor_in = r2 ? in : nullptr;
  if (g.kind == kQcKara) return qck_dual_lpn(g.f, e, ahat, src, xor_in, out, scr, Y, leaf_batch(ctx), st);
  if (g.kind == kQcFft) {
    uint32_t *tiles = reinterpret_cast<uint32_t *>(scr);
    CUOT_TRY(qcf_gather(e, src, tiles, st));
    CUOT_TRY(qcf_encode_tiles(g.f, single_tab(ahat), tiles, 32, Y, batch, st));
    return qcf_scatter(e, tiles, xor_in, out, st);
  }
  uint64_t *pl = reinterpret_cast<uint64_t *>(scr);
  if (!r2) {
    CUOT_TRY(transpose_launch(in, n, 16, 0, 128, scr, st));
    CUOT_TRY(eng_encode(g, e, ahat, pl, pl, n / 64, 0, 128, Y, batch, st));
    return transpose_launch(scr, 128, n / 8, 0, n, out, st);
  }
  // 128 planes of 2n bits (stride n/32 words); e1's product XORed into e0's
  CUOT_TRY(transpose_launch(in, 2 * n, 16, 0, 128, scr, st));
  CUOT_TRY(eng_encode(g, e, ahat, pl + n / 64, pl, n / 32, 1, 128, Y, batch, st));
  return transpose_launch(scr, 128, n / 4, 0, n, out, st);
}

// ---- helpers for the batched engine (batch.cu) ----------------------------
int qc_prepare(cuot_ctx *ctx, int e) {
  QcEngine g;
  return engine(ctx, e, dual_kind(ctx, e), &g);
}

uint64_t qc_ahat_bytes(const cuot_ctx *ctx, int e) { return ahat_bytes(dual_kind(ctx, e), e, false); }

int qc_lane(const cuot_ctx *ctx, int e) {
  const QcKind k = dual_kind(ctx, e);
  if (k == kQcFft) return e;
  if (k == kQcKara) return kQcfMaxE;  // its leaves run on the 2^22 FFT tables
  return 64 + e;                      // NTT tables hold no per-call state
}

uint64_t qc_y_bytes(const cuot_ctx *ctx, int e, int batch) {
  const QcKind k = dual_kind(ctx, e);
  const uint64_t y = k == kQcKara ? dual_scratch_bytes(ctx, k, e, batch, false) : y_bytes(k == kQcFft, e, batch);
  const uint64_t a = ahat_scratch_bytes(k, e);
  return y > a ? y : a;
}

int qc_build_ahat(cuot_ctx *ctx, int e, const uint64_t *a_d, void *Y, void *ahat, cudaStream_t st) {
  QcEngine g;
  CUOT_TRY(engine(ctx, e, dual_kind(ctx, e), &g));
  return eng_ahat(g, e, a_d, Y, ahat, false, st);
}

int qc_job_to_layout(const cuot_ctx *ctx, int e, const cuot_block *in, void *job, cudaStream_t st) {
  const QcKind k = dual_kind(ctx, e);
  if (k == kQcFft) return qcf_gather(e, in, static_cast<uint32_t *>(job), st);
  if (k == kQcKara) {
    if (cudaMemcpyAsync(job, in, 16ull << e, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return launch_status(0);
    return CUOT_OK;
  }
  return transpose_launch(in, 1ull << e, 16, 0, 128, job, st);
}

int qc_job_from_layout(const cuot_ctx *ctx, int e, const void *job, cuot_block *out, cudaStream_t st) {
  const QcKind k = dual_kind(ctx, e);
  if (k == kQcFft) return qcf_scatter(e, static_cast<const uint32_t *>(job), nullptr, out, st);
  if (k == kQcKara) {
    if (cudaMemcpyAsync(out, job, 16ull << e, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return launch_status(0);
    return CUOT_OK;
  }
  return transpose_launch(job, 128, (1ull << e) / 8, 0, 1ull << e, out, st);
}

// Encodes `njobs` consecutive jobs (16n bytes each: 128 planes, the FFT's
// tile layout, or the blocks themselves for Karatsuba) in place; job j uses
// ahats[j] (host array of device pointers).  Y holds qc_y_bytes(batch).
int qc_encode_jobs(cuot_ctx *ctx, int e, uint64_t *planes, int njobs, const void *const *ahats, void *Y,
                   int batch, cudaStream_t st) {
  QcEngine g;
  CUOT_TRY(engine(ctx, e, dual_kind(ctx, e), &g));
  const uint64_t n = 1ull << e;
  if (g.kind == kQcKara) {
    for (int j = 0; j < njobs; j++) {
      cuot_block *blk = reinterpret_cast<cuot_block *>(planes) + uint64_t(j) * n;
      CUOT_TRY(eng_dual(ctx, g, e, ahats[j], blk, blk, false, static_cast<uint8_t *>(Y), batch, st));
    }
    return CUOT_OK;
  }
  if (g.kind == kQcFft) {
    int bt = batch < 4 ? 1 : batch / 4;
    if (bt > 32 * 15) bt = 32 * 15;  // a launch may span at most 16 jobs
    uint32_t *tiles = reinterpret_cast<uint32_t *>(planes);
    for (int t0 = 0; t0 < 32 * njobs; t0 += bt) {
      const int ntr = 32 * njobs - t0 < bt ? 32 * njobs - t0 : bt;
      QcfAhatTab tab{};
      tab.per = 32;
      tab.first = t0 % 32;
      for (int j = 0; j < 16 && t0 / 32 + j < njobs; j++) tab.p[j] = ahats[t0 / 32 + j];
      CUOT_TRY(qcf_encode_tiles(g.f, tab, tiles + uint64_t(t0) * (n / 8), ntr, Y, 4 * ntr, st));
    }
    return CUOT_OK;
  }
  const int nplanes = 128 * njobs;
  // a launch may span at most kAhatTab jobs
  if (batch > 128 * (kAhatTab - 1)) batch = 128 * (kAhatTab - 1);
  int launches = 0;
  for (int p0 = 0; p0 < nplanes; p0 += batch) {
    const int nb = nplanes - p0 < batch ? nplanes - p0 : batch;
    uint64_t *pl = planes + uint64_t(p0) * (n / 64);
    const int N1 = 1 << g.t->e1, N2 = 1 << g.t->e2;
    AhatTab tab{};
    tab.per = 128;
    tab.first = p0 % 128;
    for (int j = 0; j < kAhatTab && p0 / 128 + j < njobs; j++) tab.p[j] = static_cast<const uint2 *>(ahats[p0 / 128 + j]);
    launch_col_fwd(g.t, dim3(N2 / kCW, nb), st, reinterpret_cast<const uint32_t *>(pl), n / 32,
                   static_cast<uint32_t *>(Y));
    launch_row(g.t, dim3(N1 / row_rows(g.t), nb), st, static_cast<uint32_t *>(Y), tab, 0);
    launch_col_inv(g.t, dim3(N2 / kCW, nb), st, static_cast<const uint32_t *>(Y), reinterpret_cast<uint8_t *>(pl),
                   n / 8);
    launches += 3;
  }
  return launch_status(launches);
}

int qc_default_batch(uint64_t n, int nplanes) { return default_batch(n, nplanes); }

static int one_shot_batch(const cuot_ctx *ctx, uint64_t n) {
  const int batch = ctx->qc_planes_per_pass > 0 ? ctx->qc_planes_per_pass : default_batch(n, 128);
  return batch > 128 ? 128 : batch;
}

// Scratch of cuot_sot_dual_lpn (r2: cuot_sot_dual_lpn_r2) at n = 2^e on ctx.
uint64_t qc_one_shot_dual_bytes(const cuot_ctx *ctx, int e, bool r2) {
  const QcKind kind = dual_kind(ctx, e);
  const uint64_t ds = dual_scratch_bytes(ctx, kind, e, one_shot_batch(ctx, 1ull << e), r2);
  const uint64_t as = ahat_scratch_bytes(kind, e);
  return ahat_bytes(kind, e, false) + (ds > as ? ds : as);
}

}  // namespace cuot

using namespace cuot;

struct cuot_qc_plan {
  cuot_ctx *ctx;
  int e;
  uint64_t n;
  QcKind kind;
  void *ahat;
  int batch;
};

extern "C" {

int cuot_qc_gen_a(cuot_ctx *ctx, const uint8_t key[16], uint64_t n, uint64_t *a_d, void *stream) {
  if (!ctx || !key || !a_d) return fail(CUOT_EINVAL, "null argument");
  if (n == 0 || n % 128) return fail(CUOT_EINVAL, "n=%llu must be a multiple of 128", (unsigned long long)n);
  DeviceGuard g(ctx);
  const uint64_t nb = n / 128;
  qc_make_counters<<<256, 256, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<Blk *>(a_d), nb);
  CUOT_TRY(launch_status());
  return cuot_aes128_ecb(ctx, key, reinterpret_cast<cuot_block *>(a_d), nb, stream);
}

int cuot_prg_fill(cuot_ctx *ctx, const uint8_t seed[16], uint64_t block_offset, cuot_block *out_d,
                  uint64_t nblocks, void *stream) {
  if (!ctx || !seed || (!out_d && nblocks)) return fail(CUOT_EINVAL, "null argument");
  if (nblocks == 0) return CUOT_OK;
  DeviceGuard g(ctx);
  prg_make_counters<<<512, 256, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<Blk *>(out_d), nblocks,
                                                                        block_offset);
  CUOT_TRY(launch_status());
  return cuot_aes128_ecb(ctx, seed, out_d, nblocks, stream);
}

int cuot_qc_plan_create(cuot_ctx *ctx, const uint64_t *a_d, uint64_t n, void *stream,
                        cuot_qc_plan **out) {
  if (!ctx || !a_d || !out) return fail(CUOT_EINVAL, "null argument");
  *out = nullptr;
  int e;
  CUOT_TRY(check_n(n, &e));
  DeviceGuard dg(ctx);
  cuot_qc_plan *pl = new cuot_qc_plan{ctx, e, n, dual_kind(ctx, e), nullptr, 0};
  QcEngine g;
  int st = engine(ctx, e, pl->kind, &g);
  if (st == CUOT_OK) st = dev_alloc(&pl->ahat, ahat_bytes(pl->kind, e, true));
  void *scr = nullptr;
  if (st == CUOT_OK) st = scratch(ctx, ahat_scratch_bytes(pl->kind, e), &scr);
  if (st == CUOT_OK) st = eng_ahat(g, e, a_d, scr, pl->ahat, true, static_cast<cudaStream_t>(stream));
  if (st != CUOT_OK) {
    if (pl->ahat) cudaFree(pl->ahat);
    delete pl;
    return st;
  }
  pl->batch = ctx->qc_planes_per_pass > 0 ? ctx->qc_planes_per_pass : default_batch(n, 128);
  *out = pl;
  return CUOT_OK;
}

int cuot_qc_plan_destroy(cuot_qc_plan *pl) {
  if (!pl) return CUOT_OK;
  DeviceGuard g(pl->ctx);
  cudaFree(pl->ahat);
  delete pl;
  return CUOT_OK;
}

int cuot_qc_plan_set_batch(cuot_qc_plan *pl, int planes_per_batch) {
  if (!pl || planes_per_batch < 1) return fail(CUOT_EINVAL, "bad batch");
  pl->batch = planes_per_batch;
  return CUOT_OK;
}

int cuot_qc_plan_encode(cuot_qc_plan *pl, uint64_t *planes_io_d, int nplanes, void *stream) {
  if (!pl || !planes_io_d || nplanes < 1) return fail(CUOT_EINVAL, "bad argument");
  cuot_ctx *ctx = pl->ctx;
  DeviceGuard dg(ctx);
  QcEngine g;
  CUOT_TRY(engine(ctx, pl->e, pl->kind, &g));
  const int batch = pl->batch < nplanes ? pl->batch : nplanes;
  void *scr;
  CUOT_TRY(scratch(ctx, y_bytes(pl->kind == kQcFft, pl->e, batch), &scr));
  return eng_encode(g, pl->e, pl->ahat, planes_io_d, planes_io_d, pl->n / 64, 0, nplanes, scr, batch,
                    static_cast<cudaStream_t>(stream));
}

int cuot_qc_plan_dual_lpn(cuot_qc_plan *pl, cuot_block *io_d, void *stream) {
  if (!pl || !io_d) return fail(CUOT_EINVAL, "bad argument");
  cuot_ctx *ctx = pl->ctx;
  DeviceGuard dg(ctx);
  QcEngine g;
  CUOT_TRY(engine(ctx, pl->e, pl->kind, &g));
  const int batch = pl->batch < 128 ? pl->batch : 128;
  void *scr;
  CUOT_TRY(scratch(ctx, dual_scratch_bytes(ctx, pl->kind, pl->e, batch, false), &scr));
  return eng_dual(ctx, g, pl->e, pl->ahat, io_d, io_d, false, static_cast<uint8_t *>(scr), batch,
                  static_cast<cudaStream_t>(stream));
}

int cuot_qc_plan_dual_lpn_r2(cuot_qc_plan *pl, const cuot_block *in_d, cuot_block *out_d, void *stream) {
  if (!pl || !in_d || !out_d) return fail(CUOT_EINVAL, "bad argument");
  cuot_ctx *ctx = pl->ctx;
  DeviceGuard dg(ctx);
  QcEngine g;
  CUOT_TRY(engine(ctx, pl->e, pl->kind, &g));
  const int batch = pl->batch < 128 ? pl->batch : 128;
  void *scr;
  CUOT_TRY(scratch(ctx, dual_scratch_bytes(ctx, pl->kind, pl->e, batch, true), &scr));
  return eng_dual(ctx, g, pl->e, pl->ahat, in_d, out_d, true, static_cast<uint8_t *>(scr), batch,
                  static_cast<cudaStream_t>(stream));
}

int cuot_qc_encode(cuot_ctx *ctx, const uint64_t *a_d, uint64_t *planes_io_d, uint64_t n,
                   int nplanes, void *stream) {
  if (!ctx || !a_d || !planes_io_d || nplanes < 1) return fail(CUOT_EINVAL, "bad argument");
  int e;
  CUOT_TRY(check_n(n, &e));
  DeviceGuard dg(ctx);
  QcEngine g;
  const QcKind kind = plane_kind(ctx, e);
  CUOT_TRY(engine(ctx, e, kind, &g));
  int batch = ctx->qc_planes_per_pass > 0 ? ctx->qc_planes_per_pass : default_batch(n, nplanes);
  if (batch > nplanes) batch = nplanes;
  const uint64_t ab = ahat_bytes(kind, e, false);
  void *scr;
  CUOT_TRY(scratch(ctx, ab + y_bytes(kind == kQcFft, e, batch), &scr));
  void *Y = static_cast<uint8_t *>(scr) + ab;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUOT_TRY(eng_ahat(g, e, a_d, Y, scr, false, st));
  return eng_encode(g, e, scr, planes_io_d, planes_io_d, n / 64, 0, nplanes, Y, batch, st);
}

// One-shot dual LPN (both forms): A_hat and the dual LPN's scratch in the
// context's arena.
static int one_shot_dual(cuot_ctx *ctx, const uint64_t *a_d, const cuot_block *in_d, cuot_block *out_d, uint64_t n,
                         bool r2, void *stream) {
  int e;
  CUOT_TRY(check_n(n, &e));
  DeviceGuard dg(ctx);
  QcEngine g;
  const QcKind kind = dual_kind(ctx, e);
  CUOT_TRY(engine(ctx, e, kind, &g));
  const int batch = one_shot_batch(ctx, n);
  const uint64_t ab = ahat_bytes(kind, e, false);
  void *scr;
  CUOT_TRY(scratch(ctx, qc_one_shot_dual_bytes(ctx, e, r2), &scr));
  uint8_t *work = static_cast<uint8_t *>(scr) + ab;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUOT_TRY(eng_ahat(g, e, a_d, work, scr, false, st));
  return eng_dual(ctx, g, e, scr, in_d, out_d, r2, work, batch, st);
}

int cuot_sot_dual_lpn(cuot_ctx *ctx, const uint64_t *a_d, cuot_block *io_d, uint64_t n,
                      void *stream) {
  if (!ctx || !a_d || !io_d) return fail(CUOT_EINVAL, "bad argument");
  return one_shot_dual(ctx, a_d, io_d, io_d, n, false, stream);
}

int cuot_sot_dual_lpn_r2(cuot_ctx *ctx, const uint64_t *a_d, const cuot_block *in_d, uint64_t n,
                         cuot_block *out_d, void *stream) {
  if (!ctx || !a_d || !in_d || !out_d) return fail(CUOT_EINVAL, "bad argument");
  return one_shot_dual(ctx, a_d, in_d, out_d, n, true, stream);
}

int cuot_qc_encode_sparse(cuot_ctx *ctx, const uint64_t *a_d, const uint64_t *pos_d, int weight,
                          uint64_t n, uint64_t *out_d, void *stream) {
  if (!ctx || !a_d || !out_d || (weight > 0 && !pos_d) || weight < 0)
    return fail(CUOT_EINVAL, "bad argument");
  if (n == 0 || n % 64) return fail(CUOT_EINVAL, "n must be a positive multiple of 64");
  if (weight > (1 << 24)) return fail(CUOT_EINVAL, "weight %d above 2^24", weight);
  DeviceGuard g(ctx);
  return launch_sparse(a_d, pos_d, weight, n, out_d, 0, static_cast<cudaStream_t>(stream));
}

int cuot_qc_encode_sparse_r2(cuot_ctx *ctx, const uint64_t *a_d, const uint64_t *pos_d, int weight,
                             uint64_t n, uint64_t *out_d, void *stream) {
  if (!ctx || !a_d || !out_d || (weight > 0 && !pos_d) || weight < 0)
    return fail(CUOT_EINVAL, "bad argument");
  if (n == 0 || n % 64) return fail(CUOT_EINVAL, "n must be a positive multiple of 64");
  if (weight > (1 << 24)) return fail(CUOT_EINVAL, "weight %d above 2^24", weight);
  DeviceGuard g(ctx);
  return launch_sparse(a_d, pos_d, weight, n, out_d, 1, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
