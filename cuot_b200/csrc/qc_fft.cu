// qc_fft.cu -- exact quasi-cyclic encode through a double-precision complex
// FFT (the default backend for n = 2^e, 10 <= e <= 22).
//
// out_r = a * e_r mod (x^n - 1) over GF(2) is the parity of the integer
// cyclic convolution, whose coefficients lie in [0, w(a)] (w: weight).  Four
// planes share one complex transform, with base B = 2^21 for n <= 2^20 and
// B = 2^21 + 1 for n >= 2^21:
//   x_j = (e0_j + B e1_j) + i (e2_j + B e3_j),
// and since `a` is real, IFFT(FFT(x) . FFT(a)) = (a*e0 + B a*e1) + i (a*e2
// + B a*e3): every product coefficient is an integer V = c0 + B c1 below
// 2^43 with c0, c1 in [0, W] (W < B), so c1 = floor(V / B) and c0 = V - B c1.
// For B = 2^21 the two planes' bits are bits 0 and 21 of V; for B = 2^21 + 1,
// with hi = V >> 21, lo = V mod 2^21 and d = hi - lo, c1 = hi - [d > 0] -
// [d > B] and c0 has the parity of lo ^ c1 (B odd).
// At n = 2^22 two exact changes keep the rounding error small:
//  * `a` is replaced by its complement when w(a) > n/2 (the weight is
//    counted on the device when A_hat is built and kept in A_hat's trailer);
//    a * e = w(e) - ~a * e coefficientwise, so each plane's result is XORed
//    with the parity of the plane's weight (XOR-reduced by the forward pass).
//    The coefficients then lie in [0, W] with W = min(w(a), n - w(a)) <= 2^21.
//  * the planes are centred, x_j = (e0_j - 1/2) + B (e1_j - 1/2) + i (...),
//    which moves every product coefficient by -(1 + B) W / 2 = -(2^20 + 1) W,
//    an integer added back after rounding.
// The computed values differ from the integers by less than 1/2, so rounding
// recovers them exactly: by the error bound for FFT-based convolution
// (Percival, "Rapid multiplication modulo the sum and difference of highly
// composite numbers", Math. Comp. 72 (2003), Thm. 5.1) the error is at most
// ||x||_2 ||a||_2 ((1+eps)^{3m} (1+eps sqrt5)^{3m+1} (1+beta)^{3m} - 1) with
// m = log2 n, eps = 2^-53 and twiddle error beta <= 4 eps, where ||x||_2
// ||a||_2 <= sqrt(2n) (1 + B) sqrt(n) (centred: sqrt(2n) (1 + B) / 2
// sqrt(W)): below 2^41.5 * 436.4 * 2^-53 < 0.16 for n = 2^20, 2^42.5 *
// 458.2 * 2^-53 < 0.32 for n = 2^21 and 2^42 * 479.9 * 2^-53 < 0.24 for
// n = 2^22 (smaller n: smaller bound).
//
// Work per plane and radix-2 stage is one fp64 operation (a complex
// butterfly shared by four planes), against several integer instructions
// per plane in the number-theoretic transform of qc.cu.
//
// Four-step transform, n = N1 * N2 (N1 = 2^e1 <= 1024, N1 <= N2 <= 4096), input
// index j = N2*j1 + j2, frequency k = k1 + N1*k2:
//   A (columns): 8 columns j2 of one transform per CTA (4 for the 1024-point
//     columns of the tile layout): load the plane bits, N1-point DIF FFT over
//     j1 (frequencies land in bit-reversed row order r), multiply by
//     w_n^(j2 * rev(r)), store Y[r][j2].
//   B (rows): 4 rows (2 at N2 = 2048, 1 at 4096) per CTA: N2-point DIF FFT, multiply by A_hat (the
//     transform of `a` in the same layout, scaled by 1/n), N2-point DIT
//     inverse, store.
//   C (columns): multiply by w_n^-(j2 * rev(r)), N1-point DIT inverse over r,
//     round, extract the four planes' bits, store (or XOR) 8 columns per byte
//     (4-column CTAs: one 16-bit half of the tile word).
// An N-point transform runs in shared memory as 2-3 passes of 2^K-point
// butterflies in registers (K <= 4, constant internal twiddles), each pass
// followed by one multiplication with w_S^(base * q) from a table.  The 8
// transforms (columns) of a CTA sit in rows of N + 1 complex values and the 8
// lanes of each quarter-warp work on the same item of the 8 transforms; with
// 4 (2, 1) per CTA, rows of N + 2 (N + 4, N) and an XOR swizzle (spos), so
// the passes' shared-memory exchanges are conflict-free.
#include "ctx.cuh"

namespace cuot {

constexpr double kRoundMagic = 6755399441055744.0;  // 1.5 * 2^52

// Radix-8 plans for the 4096-point rows (8^4) and the 1024-point transforms
// (8 8 4 4): one more shared-memory pass than radix 16, but few enough live
// registers (78-80) for three CTAs per SM.  Measured on B200 (n = 2^22 dual
// LPN of both roles): radix 16 7.04 ms, both radix-8 plans 7.89 ms, rows only
// 8.45 ms, 1024-point only 8.36 ms; off.
constexpr bool kQcfRow12Radix8 = false;
constexpr bool kQcfL10Radix8 = false;
// Radix plan of an N = 2^L point transform, 5 <= L <= 12: K bits per pass.
__host__ __device__ constexpr int qcf_npass(int L) {
  return L <= 8 ? 2 : (L == 12 && kQcfRow12Radix8) || (L == 10 && kQcfL10Radix8) ? 4 : 3;
}
__host__ __device__ constexpr int qcf_k(int L, int p) {
  return L == 12 && kQcfRow12Radix8 ? 3
       : L == 10 && kQcfL10Radix8 ? (p < 2 ? 3 : 2)
       : L == 5 ? (p == 0 ? 3 : 2)
       : L == 6 ? 3
       : L == 7 ? (p == 0 ? 4 : 3)
       : L == 8 ? 4
       : L == 9 ? 3
       : L == 10 ? (p == 0 ? 4 : 3)
       : L == 11 ? (p == 2 ? 3 : 4)
       : 4;
}
// log2 of the sub-transform size at the start of pass p
__host__ __device__ constexpr int qcf_ls(int L, int p) { return p == 0 ? L : qcf_ls(L, p - 1) - qcf_k(L, p - 1); }
// Twiddle table of an N-point transform in pass order: pass p's factors
// w_S^(base q) (q in [1, 2^K), base < M = S / 2^K) at tw_off(p) + (q-1) M + base,
// so lanes at consecutive bases read consecutive entries and lanes at the
// same base read the same entry (no bank conflicts).  At most N entries.
__host__ __device__ constexpr int qcf_tw_off(int L, int p) {
  return p == 0 ? 0 : qcf_tw_off(L, p - 1) + ((1 << qcf_k(L, p - 1)) - 1) * ((1 << qcf_ls(L, p - 1)) >> qcf_k(L, p - 1));
}
__host__ __device__ constexpr int qcf_threads(int L) { return L >= 10 ? 512 : L == 9 ? 256 : L == 8 ? 128 : 64; }
// Column CTAs per SM: three up to 512 points and for 4-column CTAs, one for
// 8 columns of 1024 points (143 KB of shared memory).
__host__ __device__ constexpr int qcf_col_ctas(int L, int KC) {
  return L >= 10 ? (KC == 8 ? 1 : kQcfL10Radix8 ? 3 : 2) : 3;
}
// four-step factor tables per column: 2^lo + 2^(e1 - lo) entries (global
// row stride), staged with an odd row stride so the 8 columns of a
// quarter-warp hit distinct banks
__host__ __device__ constexpr int qcf_fs_lo(int e1) { return (e1 + 1) / 2; }
__host__ __device__ constexpr int qcf_fs_width(int e1) { return (1 << qcf_fs_lo(e1)) + (1 << (e1 - qcf_fs_lo(e1))); }
__host__ __device__ constexpr int qcf_fs_ld(int e1) { return qcf_fs_width(e1) + 1; }
// Start of column c's factor row in shared memory.  In a 4-column CTA a
// quarter-warp reads 4 columns x 2 items whose high-table entries lie 2
// apart, so with rows of W = 1 (mod 8) columns c and c + 2 would share a
// bank group; columns 2 and 3 start 2 values further on, which gives the 8
// lanes 8 distinct groups (a model of the reads: 1,088 wavefronts per
// 1024-point CTA before, the ideal 576 after).
__host__ __device__ constexpr int qcf_fs_col(int e1, int kc, int c) {
  return c * qcf_fs_ld(e1) + (kc == 4 ? 2 * (c >> 1) : 0);
}
__host__ __device__ constexpr int qcf_fs_span(int e1, int kc) { return qcf_fs_col(e1, kc, kc - 1) + qcf_fs_ld(e1); }
// Columns per CTA of the column passes: 8 (one tile byte per plane and row),
// or 4 for the 1024-point columns of the tile layout, whose 8-column CTAs
// (143 KB) would run one per SM; two CTAs then share each tile byte and
// write one 16-bit half of its word each (see qcf_col_inv).
__host__ __device__ constexpr int qcf_col_threads(int L, int KC) { return KC == 8 ? qcf_threads(L) : qcf_threads(L) / 2; }
// Rows per CTA of the row pass, so that two CTAs fit an SM: 4 up to 1024
// points, 2 for 2048, 1 for 4096 (its first pass's twiddles are read
// through L1, only the middle pass's are staged).
__host__ __device__ constexpr int qcf_rows(int L) { return L >= 12 ? 1 : L == 11 ? 2 : 4; }
// Row pass reads pass 0's twiddles from global memory through L1.
__host__ __device__ constexpr bool qcf_row_tg0(int L) { return L >= 12; }
// Row CTAs per SM (launch bound).
__host__ __device__ constexpr int qcf_row_ctas(int L) {
  return (L == 12 && kQcfRow12Radix8) || (L == 10 && kQcfL10Radix8) ? 3 : 2;
}
__host__ __device__ constexpr int qcf_row_threads(int L) {
  return L >= 11 ? 256 : qcf_threads(L) / 2 < 32 ? 32 : qcf_threads(L) / 2;
}
// Packing base 2^21 + qcf_wide(e) (2^21 + 1 from n = 2^21, where a product
// coefficient can equal 2^21).
__host__ __device__ constexpr int qcf_wide(int e) { return e >= 21 ? 1 : 0; }
// Split of n = 2^e into N1 = 2^e1 column points (at most 512 up to 2^21, so
// three column CTAs fit an SM; 1024 at 2^22) and N2 = 2^(e - e1) row points
// (at most 4096).
__host__ __device__ constexpr int qcf_e1(int e) { return e >= 22 ? e - 12 : e / 2 < 9 ? e / 2 : 9; }
// The centred mode is n = 2^22, the only size with 1024-point columns.
__host__ __device__ constexpr bool qcf_col_center(int e1) { return e1 >= 10; }
static_assert(qcf_col_center(qcf_e1(22)) && !qcf_col_center(qcf_e1(21)) && qcf_center(22) && !qcf_center(21),
              "centred mode <=> 1024-point columns");
// Columns per CTA of the tile-layout column passes of n = 2^e.
__host__ __device__ constexpr int qcf_tile_kc(int e) { return qcf_e1(e) >= 10 ? 4 : 8; }
// Centring offset (1 + B) / 2 of the n = 2^22 packing (B = 2^21 + 1).
constexpr int64_t kCenter = (1 << 20) + 1;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// a * w
__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
  return make_double2(fma(a.x, w.x, -(a.y * w.y)), fma(a.x, w.y, a.y * w.x));
}
// a * conj(w)
__device__ __forceinline__ double2 cmulc(double2 a, double2 w) {
  return make_double2(fma(a.x, w.x, a.y * w.y), fma(a.y, w.x, -(a.x * w.y)));
}

// Stores of the intermediate that the next pass reads back carry an L2
// evict-last hint, and its last reader (the inverse column pass) loads it
// evict-first, so the other stream's passes and A_hat push it out of L2
// later (measured: sot_n22 7.07 -> 6.97 ms, the 64-instance mix 82.0 -> 81.4 ms).
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void st_keep(double2 *a, double2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(v.x), "d"(v.y), "l"(pol)
               : "memory");
}

// cos(2 pi J / 16) and sin(2 pi J / 16) for J in [0, 8)
__device__ __forceinline__ constexpr double c16(int J) {
  return J == 0 ? 1.0
       : J == 1 ? 0.92387953251128675613
       : J == 2 ? 0.70710678118654752440
       : J == 3 ? 0.38268343236508977173
       : J == 4 ? 0.0
       : J == 5 ? -0.38268343236508977173
       : J == 6 ? -0.70710678118654752440
                : -0.92387953251128675613;
}
__device__ __forceinline__ constexpr double s16(int J) { return c16(J >= 4 ? J - 4 : 4 - J); }

// v * w16^J (forward, w16 = exp(-2 pi i / 16)) or v * conj(w16^J) (INV),
// J in [0, 8); J is a compile-time constant after unrolling.
template <bool INV>
__device__ __forceinline__ double2 wmul16(double2 v, int J) {
  constexpr double r = 0.70710678118654752440;
  if (J == 0) return v;
  if (J == 4) return INV ? make_double2(-v.y, v.x) : make_double2(v.y, -v.x);
  if (J == 2) return INV ? make_double2((v.x - v.y) * r, (v.x + v.y) * r) : make_double2((v.x + v.y) * r, (v.y - v.x) * r);
  if (J == 6) return INV ? make_double2(-(v.x + v.y) * r, (v.x - v.y) * r) : make_double2((v.y - v.x) * r, -(v.x + v.y) * r);
  const double c = c16(J), s = s16(J);
  return INV ? make_double2(fma(v.x, c, -(v.y * s)), fma(v.y, c, v.x * s))
             : make_double2(fma(v.x, c, v.y * s), fma(v.y, c, -(v.x * s)));
}

// 2^K-point DFT in registers, natural order in, bit-reversed order out.
template <int K>
__device__ __forceinline__ void dif_regs(double2 (&x)[1 << K]) {
  constexpr int R = 1 << K;
#pragma unroll
  for (int t = 0; t < K; t++) {
    const int h = R >> (t + 1);
#pragma unroll
    for (int m = 0; m < R; m++) {
      if (m & h) continue;
      const double2 u = x[m], v = x[m + h];
      x[m] = cadd(u, v);
      x[m + h] = wmul16<false>(csub(u, v), (m & (h - 1)) * (8 / h));
    }
  }
}
// Its inverse (times 2^K): bit-reversed order in, natural order out.
template <int K>
__device__ __forceinline__ void dit_regs(double2 (&x)[1 << K]) {
  constexpr int R = 1 << K;
#pragma unroll
  for (int t = K - 1; t >= 0; t--) {
    const int h = R >> (t + 1);
#pragma unroll
    for (int m = 0; m < R; m++) {
      if (m & h) continue;
      const double2 u = x[m], v = wmul16<true>(x[m + h], (m & (h - 1)) * (8 / h));
      x[m] = cadd(u, v);
      x[m + h] = csub(u, v);
    }
  }
}

// Item w of pass P over an N = 2^L point transform: 2^K elements
// blk*S + base + M*m (S = 2^LS, M = S / 2^K).
template <int L, int P>
struct Pass {
  static constexpr int K = qcf_k(L, P), R = 1 << K, LS = qcf_ls(L, P), M = (1 << LS) >> K;
  static constexpr int items = (1 << L) >> K;
  __device__ static int first(int w) { return ((w / M) << LS) + (w % M); }
  __device__ static int base(int w) { return w % M; }
};

// Twiddles of a DIF pass after its butterflies: x[m] holds frequency
// q = rev_K(m) of its sub-transform; multiply by w_S^(base q) (table in pass
// order, qcf_tw_off).
// TG: T is in global memory (read through L1) instead of shared memory.
// REL: T points at pass P's part of the table instead of its start.
template <int L, int P, bool INV, bool TG = false, bool REL = false>
__device__ __forceinline__ void pass_twiddle(double2 (&x)[Pass<L, P>::R], int base, const double2 *T) {
  using Q = Pass<L, P>;
  if (Q::M == 1) return;
  const double2 *Tp = T + (REL ? 0 : qcf_tw_off(L, P)) + base;
#pragma unroll
  for (int m = 1; m < Q::R; m++) {
    const int q = __brev(m) >> (32 - Q::K);
    const double2 w = TG ? __ldg(&Tp[(q - 1) * Q::M]) : Tp[(q - 1) * Q::M];
    x[m] = INV ? cmulc(x[m], w) : cmul(x[m], w);
  }
}

// Shared-memory position of element i of a transform.  NT = 8 transforms per
// CTA: rows of N + 1 values, the 8 lanes of a quarter-warp are the 8
// transforms at one item, no swizzle.  NT = 4 (2, 1): rows of N + 2 (N + 4,
// N) values, a quarter-warp is 4 transforms x 2 consecutive items (2 x 4,
// 1 x 8), and XORing bits [0, 1) ([0, 2), [0, 3)) of i with the bits above
// K_last keeps both the early passes (items differ in the low bits) and the
// last pass (items differ from bit K_last up) conflict-free.
template <int L, int NT>
__device__ __forceinline__ int spos(int i) {
  if constexpr (NT == 8) return i;
  return i ^ ((i >> qcf_k(L, qcf_npass(L) - 1)) & (NT == 4 ? 1 : NT == 2 ? 3 : 7));
}
template <int NT>
__host__ __device__ constexpr int sld(int N) { return NT == 8 ? N + 1 : NT == 4 ? N + 2 : NT == 2 ? N + 4 : N; }

// One pass entirely in shared memory (xs rows of sld<NT>(N) complex values).
template <int L, int P, bool INV, int NT, bool TG = false, bool REL = false>
__device__ __forceinline__ void smem_pass(double2 *xs, const double2 *T) {
  using Q = Pass<L, P>;
  constexpr int ld = sld<NT>(1 << L);
  for (int it = threadIdx.x; it < NT * Q::items; it += blockDim.x) {
    const int c = it & (NT - 1), w = it / NT;
    double2 *row = xs + c * ld;
    const int i0 = Q::first(w);
    double2 x[Q::R];
#pragma unroll
    for (int m = 0; m < Q::R; m++) x[m] = row[spos<L, NT>(i0 + Q::M * m)];
    if (!INV) {
      dif_regs<Q::K>(x);
      pass_twiddle<L, P, false, TG, REL>(x, Q::base(w), T);
    } else {
      pass_twiddle<L, P, true, TG, REL>(x, Q::base(w), T);
      dit_regs<Q::K>(x);
    }
#pragma unroll
    for (int m = 0; m < Q::R; m++) row[spos<L, NT>(i0 + Q::M * m)] = x[m];
  }
}

// Middle pass P (REL: T is pass 1's part of the table, so pass P's part
// starts tw_off(P) - tw_off(1) further on).
template <int L, int P, bool INV, int NT, bool TG, bool REL>
__device__ __forceinline__ void middle_pass(double2 *xs, const double2 *T) {
  __syncthreads();
  smem_pass<L, P, INV, NT, TG, REL>(xs, REL ? T + (qcf_tw_off(L, P) - qcf_tw_off(L, 1)) : T);
}
// Middle passes [1, npass - 1) forward, or in reverse order inverse.
template <int L, bool INV, int NT, bool TG = false, bool REL = false>
__device__ __forceinline__ void middle_passes(double2 *xs, const double2 *T) {
  constexpr int NP = qcf_npass(L);
  static_assert(NP <= 4, "at most two middle passes");
  if constexpr (!INV) {
    if constexpr (NP >= 3) middle_pass<L, 1, INV, NT, TG, REL>(xs, T);
    if constexpr (NP >= 4) middle_pass<L, 2, INV, NT, TG, REL>(xs, T);
  } else {
    if constexpr (NP >= 4) middle_pass<L, 2, INV, NT, TG, REL>(xs, T);
    if constexpr (NP >= 3) middle_pass<L, 1, INV, NT, TG, REL>(xs, T);
  }
  __syncthreads();
}

// w_n^(j2 * k1) for the CTA's column c and k1 = rev_e1(r), from the column's
// two factor tables in shared memory (low lo bits of k1, high bits), for the
// 2^K rows r = i0 + m (m < 2^K) of one item of the last column pass (i0 a
// multiple of 2^K): k1 = rev(i0) | rev_K(m) << (E1 - K), and since E1 - K >= lo
// every row shares the low table entry, read once.
template <int E1, int K, int KC>
__device__ __forceinline__ void fourstep_ws(const double2 *fs, int c, int i0, double2 (&w)[1 << K]) {
  constexpr int lo = qcf_fs_lo(E1);
  static_assert(E1 - K >= lo, "the rows of an item share the low factor");
  const int k10 = __brev(i0) >> (32 - E1);
  const double2 *fc = fs + qcf_fs_col(E1, KC, c);
  const double2 wl = fc[k10 & ((1 << lo) - 1)];
  const double2 *hi = fc + (1 << lo) + (k10 >> lo);
#pragma unroll
  for (int m = 0; m < (1 << K); m++) w[m] = cmul(wl, hi[(__brev(m) >> (32 - K)) << (E1 - K - lo)]);
}

__device__ __forceinline__ void stage(double2 *dst, const double2 *src, int cnt) {
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) dst[i] = __ldg(&src[i]);
}
// The KC columns' four-step factor rows (global stride W) into their rows
// in shared memory (qcf_fs_col).
template <int E1, int KC>
__device__ __forceinline__ void stage_fs(double2 *dst, const double2 *fs, int c0) {
  constexpr int W = qcf_fs_width(E1);
  const double2 *src = fs + uint64_t(c0) * W;
  for (int i = threadIdx.x; i < KC * W; i += blockDim.x) dst[qcf_fs_col(E1, KC, i / W) + i % W] = __ldg(&src[i]);
}

// Pass A.  grid (N2 / KC, transforms).  in: plane p at in + p * stride_bytes;
// transform y holds planes 4y .. 4y+3 (< nplanes) with base 2^21 + wide;
// one_plane: `a` (real part only; centred mode: its complement if wa[0] >
// n / 2).  With tiles != nullptr the input is in the tile layout
// instead: word tiles[y][tile][j1] holds the four planes' bytes of the 8
// columns of the CTA's tile in row j1 (qcf_gather), so the CTA reads N1
// consecutive words.  centred mode (par !=
// nullptr): planes centred, and par[y] ^= the XOR of the CTA's words (byte q:
// column parities of plane 4y + q; only the CTA's KC columns).  CEN: the
// kernel has the centred mode (compiled in for the 1024-point columns of
// n = 2^22 only).
template <int E1, int KC, bool CEN>
__global__ void __launch_bounds__(qcf_col_threads(E1, KC), qcf_col_ctas(E1, KC)) qcf_col_fwd(
    const uint8_t *__restrict__ in, uint64_t stride_bytes, int nplanes, int one_plane, int e2, int wide,
    const uint32_t *__restrict__ tiles, const double2 *__restrict__ T1, const double2 *__restrict__ fs,
    double2 *__restrict__ Y, const unsigned long long *__restrict__ wa, uint32_t *__restrict__ par) {
  constexpr int N1 = 1 << E1, ld = sld<KC>(N1);
  const uint32_t base = (1u << 21) + uint32_t(wide);
  const double center = CEN && par ? double(kCenter) : 0.0;
  const uint32_t comp = CEN && wa && *wa > (1ull << (E1 + e2 - 1)) ? 1u : 0u;
  constexpr int NP = qcf_npass(E1);
  extern __shared__ double2 sm[];
  double2 *xs = sm, *fss = xs + KC * ld;
  uint32_t *bits = reinterpret_cast<uint32_t *>(fss + qcf_fs_span(E1, KC));
  const double2 *Ts = T1;  // pass twiddles read through L1
  const int c0 = blockIdx.x * KC, sub = c0 & 7;  // sub: the CTA's first bit in each tile byte
  const int p0 = 4 * blockIdx.y;
  stage_fs<E1, KC>(fss, fs, c0);
  if (tiles) {
    const uint32_t *tp = tiles + (uint64_t(blockIdx.y) << (E1 + e2 - 3)) + (uint64_t(c0 >> 3) << E1);
    for (int j1 = threadIdx.x; j1 < N1; j1 += blockDim.x) bits[j1] = __ldg(tp + j1);
  } else {
    for (int j1 = threadIdx.x; j1 < N1; j1 += blockDim.x) {
      const uint64_t byte = ((uint64_t(j1) << e2) | uint64_t(c0)) >> 3;
      uint32_t word = 0;
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (p0 + q < nplanes) word |= uint32_t(__ldg(in + uint64_t(p0 + q) * stride_bytes + byte)) << (8 * q);
      bits[j1] = word;
    }
  }
  __syncthreads();
  if (CEN && par) {  // plane weight parities (XOR of the CTA's words)
    constexpr uint32_t mask = KC == 8 ? 0xffffffffu : 0x0f0f0f0fu;
    uint32_t x = 0;
    for (int j1 = threadIdx.x; j1 < N1; j1 += blockDim.x) x ^= bits[j1] & (mask << sub);
    x = __reduce_xor_sync(0xffffffffu, x);
    if ((threadIdx.x & 31) == 0 && x) atomicXor(par + blockIdx.y, x);
  }
  {  // pass 0 from the bits
    using Q = Pass<E1, 0>;
    for (int it = threadIdx.x; it < KC * Q::items; it += blockDim.x) {
      const int c = it & (KC - 1), w = it / KC;
      const int i0 = Q::first(w);
      double2 x[Q::R];
#pragma unroll
      for (int m = 0; m < Q::R; m++) {
        const uint32_t b = bits[i0 + Q::M * m] >> (sub + c);
        if (one_plane) {
          x[m] = make_double2(double((b ^ comp) & 1u), 0.0);
        } else {
          x[m] = make_double2(double((b & 1u) + ((b >> 8) & 1u) * base) - center,
                              double(((b >> 16) & 1u) + ((b >> 24) & 1u) * base) - center);
        }
      }
      dif_regs<Q::K>(x);
      pass_twiddle<E1, 0, false, true>(x, Q::base(w), Ts);
      double2 *row = xs + c * ld;
#pragma unroll
      for (int m = 0; m < Q::R; m++) row[spos<E1, KC>(i0 + Q::M * m)] = x[m];
    }
  }
  middle_passes<E1, false, KC, true>(xs, Ts);
  {  // last pass (M = 1), then the four-step twiddle, to global
    using Q = Pass<E1, NP - 1>;
    static_assert(Q::M == 1, "last pass");
    double2 *Yp = Y + (uint64_t(blockIdx.y) << (E1 + e2));
    for (int it = threadIdx.x; it < KC * Q::items; it += blockDim.x) {
      const int c = it & (KC - 1), w = it / KC;
      const int i0 = Q::first(w);
      double2 x[Q::R];
#pragma unroll
      for (int m = 0; m < Q::R; m++) x[m] = xs[c * ld + spos<E1, KC>(i0 + m)];
      dif_regs<Q::K>(x);
      double2 fw[Q::R];
      fourstep_ws<E1, Q::K, KC>(fss, c, i0, fw);
      const uint64_t pol = l2_evict_last_policy();
#pragma unroll
      for (int m = 0; m < Q::R; m++) st_keep(&Yp[(uint64_t(i0 + m) << e2) + c0 + c], cmul(x[m], fw[m]), pol);
    }
  }
}

// Pass B.  grid (N1 / qcf_rows(e2), transforms).  mode 0: forward, pointwise by the
// transform's A_hat (ahat.p[(ahat.first + y) / ahat.per]), inverse, in place.
// mode 1: forward only, times `scale`, written to `out` (builds A_hat).
// A_hat is stored in the order the last pass consumes it: for the NT rows
// from r0, element m of item w of row c at r0 * N2 + (m * items + w) * NT + c,
// so each warp reads 512 contiguous bytes per load.
template <int E2>
__global__ void __launch_bounds__(qcf_row_threads(E2), qcf_row_ctas(E2)) qcf_row(
    double2 *__restrict__ Y, int e1, const double2 *__restrict__ T2, QcfAhatTab ahat, int mode,
    double2 *__restrict__ out, double scale) {
  constexpr int NT = qcf_rows(E2);
  constexpr int N2 = 1 << E2, ld = sld<NT>(N2);
  constexpr int NP = qcf_npass(E2);
  // G0: pass 0's twiddles through L1 from T2, shared memory holds pass 1's
  constexpr bool G0 = qcf_row_tg0(E2);
  extern __shared__ double2 sm[];
  double2 *xs = sm, *Ts = xs + NT * ld;
  const double2 *T0 = G0 ? T2 : Ts;
  const int r0 = blockIdx.x * NT;
  if (mode == 0 && threadIdx.x == 0) {
    // The pointwise product reads this CTA's A_hat rows (NT * N2 contiguous
    // values, 64 KiB) in the middle of the kernel; start moving them into L2
    // now, so those reads do not wait for DRAM.
    const double2 *ahp = static_cast<const double2 *>(ahat.p[(ahat.first + blockIdx.y) / ahat.per]) +
                         (uint64_t(r0) << E2);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(ahp), "r"(uint32_t(NT * N2 * 16)) : "memory");
  }
  if constexpr (G0)
    stage(Ts, T2 + qcf_tw_off(E2, 1), qcf_tw_off(E2, NP - 1) - qcf_tw_off(E2, 1));
  else
    stage(Ts, T2, N2);
  double2 *Yp = Y + (uint64_t(blockIdx.y) << (e1 + E2)) + (uint64_t(r0) << E2);
  __syncthreads();
  {  // pass 0 from global
    using Q = Pass<E2, 0>;
    for (int it = threadIdx.x; it < NT * Q::items; it += blockDim.x) {
      const int c = it & (NT - 1), w = it / NT;
      const int i0 = Q::first(w);
      const double2 *src = Yp + (uint64_t(c) << E2) + i0;
      double2 x[Q::R];
#pragma unroll
      for (int m = 0; m < Q::R; m++) x[m] = src[Q::M * m];
      dif_regs<Q::K>(x);
      pass_twiddle<E2, 0, false, G0>(x, Q::base(w), T0);
      double2 *row = xs + c * ld;
#pragma unroll
      for (int m = 0; m < Q::R; m++) row[spos<E2, NT>(i0 + Q::M * m)] = x[m];
    }
  }
  middle_passes<E2, false, NT, false, G0>(xs, Ts);
  {  // last forward pass; pointwise product; first inverse pass
    using Q = Pass<E2, NP - 1>;
    const double2 *ah = mode == 0 ? static_cast<const double2 *>(ahat.p[(ahat.first + blockIdx.y) / ahat.per]) +
                                        (uint64_t(r0) << E2)
                                  : nullptr;
    for (int it = threadIdx.x; it < NT * Q::items; it += blockDim.x) {
      const int c = it & (NT - 1), w = it / NT;
      const int i0 = Q::first(w);
      double2 *row = xs + c * ld;
      double2 x[Q::R];
#pragma unroll
      for (int m = 0; m < Q::R; m++) x[m] = row[spos<E2, NT>(i0 + m)];
      dif_regs<Q::K>(x);
      if (mode == 1) {
        double2 *o = out + (uint64_t(r0) << E2) + it;
#pragma unroll
        for (int m = 0; m < Q::R; m++) o[m * NT * Q::items] = make_double2(x[m].x * scale, x[m].y * scale);
        continue;
      }
      // A_hat is read once per transform: evict-first, so it does not push the
      // intermediate that the inverse column pass reads next out of L2
      // (measured: the 64-instance mix 0.6 % faster, n = 2^20 1.1 %, 2^22 0.4 % slower)
      const double2 *a = ah + it;
#pragma unroll
      for (int m = 0; m < Q::R; m++) x[m] = cmul(x[m], __ldcs(&a[m * NT * Q::items]));
      dit_regs<Q::K>(x);
#pragma unroll
      for (int m = 0; m < Q::R; m++) row[spos<E2, NT>(i0 + m)] = x[m];
    }
  }
  if (mode == 1) return;
  middle_passes<E2, true, NT, false, G0>(xs, Ts);
  {  // inverse of pass 0, to global
    using Q = Pass<E2, 0>;
    for (int it = threadIdx.x; it < NT * Q::items; it += blockDim.x) {
      const int c = it & (NT - 1), w = it / NT;
      const int i0 = Q::first(w);
      const double2 *row = xs + c * ld;
      double2 x[Q::R];
#pragma unroll
      for (int m = 0; m < Q::R; m++) x[m] = row[spos<E2, NT>(i0 + Q::M * m)];
      pass_twiddle<E2, 0, true, G0>(x, Q::base(w), T0);
      dit_regs<Q::K>(x);
      double2 *dst = Yp + (uint64_t(c) << E2) + i0;
      const uint64_t pol = l2_evict_last_policy();
#pragma unroll
      for (int m = 0; m < Q::R; m++) st_keep(&dst[Q::M * m], x[m], pol);
    }
  }
}

// The two planes' bits (c0 & 1, c1 & 1) of a product coefficient v ~ V -
// shift, V = c0 + B c1, B = 2^21 + wide, c0 and c1 in [0, 2^21] (see the top
// of the file).  For |v| < 2^51, v + 1.5 * 2^52 lies in [2^52, 2^53), where
// doubles are the integers: its bit pattern minus that of 1.5 * 2^52 is
// round(v).
__device__ __forceinline__ void plane_bits(double v, int wide, int64_t shift, uint32_t &p0, uint32_t &p1) {
  const double r = v + kRoundMagic;
  if (!wide) {
    const uint32_t lw = uint32_t(__double2loint(r));
    p0 = lw & 1u;
    p1 = (lw >> 21) & 1u;
    return;
  }
  const uint64_t V = uint64_t(__double_as_longlong(r) - __double_as_longlong(kRoundMagic) + shift);
  const uint32_t lo = uint32_t(V) & 0x1FFFFFu, hi = uint32_t(V >> 21);
  const int d = int(hi) - int(lo);
  const uint32_t c1 = hi - uint32_t(d > 0) - uint32_t(d > (1 << 21) + 1);
  p0 = (lo ^ c1) & 1u;
  p1 = c1 & 1u;
}

// Pass C.  grid (N2 / KC, transforms).  out: plane p at out + p * stride_bytes,
// written (accumulate == 0) or XORed into (accumulate == 1); with tiles !=
// nullptr the result goes to the tile layout instead (one word per row; for
// KC = 4, the CTA writes 16-bit half sub / 4 of the word, nibble q = plane
// 4y + q's bits of its 4 columns, which qcf_scatter puts back in byte
// order).  KC = 4 writes tiles only.
// centred mode (par != nullptr): the transform's A_hat trailer (ahat) gives
// w(a); the centring shift is added back and, for a complemented `a`, each
// plane's weight parity (par[y]) is XORed in (CEN: as for qcf_col_fwd).
template <int E1, int KC, bool CEN>
__global__ void __launch_bounds__(qcf_col_threads(E1, KC), qcf_col_ctas(E1, KC)) qcf_col_inv(
    const double2 *__restrict__ Y, int e2, int wide, const double2 *__restrict__ T1, const double2 *__restrict__ fs,
    uint8_t *__restrict__ out, uint64_t stride_bytes, int nplanes, int accumulate, uint32_t *__restrict__ tiles,
    QcfAhatTab ahat, const uint32_t *__restrict__ par) {
  constexpr int N1 = 1 << E1, ld = sld<KC>(N1);
  constexpr int NP = qcf_npass(E1);
  extern __shared__ double2 sm[];
  double2 *xs = sm, *fss = xs + KC * ld;
  const double2 *Ts = T1;  // pass twiddles read through L1
  const int c0 = blockIdx.x * KC;
  const int p0 = 4 * blockIdx.y;
  int64_t shift = 0;
  uint32_t flip = 0;  // bit q: XOR into plane 4y + q
  if (CEN && par) {
    const uint64_t n = 1ull << (E1 + e2);
    const uint64_t w = *reinterpret_cast<const unsigned long long *>(
        static_cast<const uint8_t *>(ahat.p[(ahat.first + blockIdx.y) / ahat.per]) + 16 * n);
    const bool comp = w > n / 2;
    shift = kCenter * int64_t(comp ? n - w : w);
    if (comp) {
      const uint32_t pw = par[blockIdx.y];
#pragma unroll
      for (int q = 0; q < 4; q++) flip |= (uint32_t(__popc((pw >> (8 * q)) & 0xffu)) & 1u) << q;
    }
  }
  stage_fs<E1, KC>(fss, fs, c0);
  __syncthreads();
  {  // inverse of the last pass, from global
    using Q = Pass<E1, NP - 1>;
    const double2 *Yp = Y + (uint64_t(blockIdx.y) << (E1 + e2));
    for (int it = threadIdx.x; it < KC * Q::items; it += blockDim.x) {
      const int c = it & (KC - 1), w = it / KC;
      const int i0 = Q::first(w);
      double2 x[Q::R], fw[Q::R];
#pragma unroll
      for (int m = 0; m < Q::R; m++) x[m] = __ldcs(&Yp[(uint64_t(i0 + m) << e2) + c0 + c]);
      fourstep_ws<E1, Q::K, KC>(fss, c, i0, fw);
#pragma unroll
      for (int m = 0; m < Q::R; m++) x[m] = cmulc(x[m], fw[m]);
      dit_regs<Q::K>(x);
#pragma unroll
      for (int m = 0; m < Q::R; m++) xs[c * ld + spos<E1, KC>(i0 + m)] = x[m];
    }
  }
  middle_passes<E1, true, KC, true>(xs, Ts);
  {  // inverse of pass 0; round; the KC columns' bits of each plane form a byte (nibble)
    using Q = Pass<E1, 0>;
    static_assert((KC * Q::items) % 32 == 0, "whole warps at the ballots");
    const int lane = threadIdx.x & 31;
    for (int it = threadIdx.x; it < KC * Q::items; it += blockDim.x) {
      const int c = it & (KC - 1), w = it / KC;
      const int i0 = Q::first(w);
      const double2 *row = xs + c * ld;
      double2 x[Q::R];
#pragma unroll
      for (int m = 0; m < Q::R; m++) x[m] = row[spos<E1, KC>(i0 + Q::M * m)];
      pass_twiddle<E1, 0, true, true>(x, Q::base(w), Ts);
      dit_regs<Q::K>(x);
      if (ahat.margin) {  // rounding-margin record (diagnostic mode only)
        double mx = 0.0;
#pragma unroll
        for (int m = 0; m < Q::R; m++)
          mx = fmax(mx, fmax(fabs(x[m].x - rint(x[m].x)), fabs(x[m].y - rint(x[m].y))));
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) atomicMax(ahat.margin, __float_as_uint(float(mx)));
      }
#pragma unroll
      for (int m = 0; m < Q::R; m++) {
        uint32_t pl[4];
        plane_bits(x[m].x, wide, shift, pl[0], pl[1]);
        plane_bits(x[m].y, wide, shift, pl[2], pl[3]);
        if constexpr (CEN) {
#pragma unroll
          for (int q = 0; q < 4; q++) pl[q] ^= (flip >> q) & 1u;
        }
        const int j1 = i0 + Q::M * m;
        constexpr uint32_t cm = (1u << KC) - 1;
        uint32_t word = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) word |= ((__ballot_sync(0xffffffffu, pl[q]) >> (lane & ~(KC - 1))) & cm) << (KC * q);
        if (c != 0) continue;
        const uint64_t wi = (uint64_t(blockIdx.y) << (E1 + e2 - 3)) + (uint64_t(c0 >> 3) << E1) + j1;
        if constexpr (KC == 4) {
          reinterpret_cast<uint16_t *>(tiles)[2 * wi + ((c0 & 7) >> 2)] = uint16_t(word);
          continue;
        }
        if (tiles) {
          tiles[wi] = word;
          continue;
        }
        const uint64_t byte = ((uint64_t(j1) << e2) | uint64_t(c0)) >> 3;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (p0 + q < nplanes) {
            const uint8_t v = uint8_t(word >> (8 * q));
            uint8_t *o = out + uint64_t(p0 + q) * stride_bytes + byte;
            *o = accumulate ? uint8_t(*o ^ v) : v;
          }
        }
      }
    }
  }
}

// 8x8 bit-matrix transpose of x (row i = byte i, column j = bit j) by three
// delta swaps (H. S. Warren, Hacker's Delight, 2nd ed., section 7-3).
__device__ __forceinline__ uint64_t transpose8(uint64_t x) {
  uint64_t t;
  t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
  x ^= t ^ (t << 7);
  t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
  x ^= t ^ (t << 14);
  t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
  x ^= t ^ (t << 28);
  return x;
}

// Tile layout of 128 planes of n = N1 * N2 bits (the dual LPN's input and
// output): word tiles[t][g][j1] (t < 32 transforms, g < N2 / 8 column tiles,
// j1 < N1 rows) holds, in byte q, bits (N2 j1 + 8 g + c), c < 8, of plane
// 4t + q, so a column CTA's words are contiguous.  The 8 blocks
// j = 8 (N2/8 j1 + g) + c of the block vector give all 32 words of one
// (g, j1): per 32-bit word wd and byte k of the blocks, the 8x8 bit transpose
// of those 8 bytes yields planes 32 wd + 8 k + b in byte b, i.e. words
// t = 8 wd + 2 k (low half) and t + 1 (high half).  Thread u = g N1 + j1
// (j1 fastest): its tile words are written coalesced and its 8 blocks are
// one 128-byte line.
__global__ void __launch_bounds__(256) qcf_gather(const uint4 *__restrict__ in, uint64_t ngroups, int e1, int e2,
                                                  uint32_t *__restrict__ tiles) {
  for (uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < ngroups;
       u += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t g = ((u & ((1ull << e1) - 1)) << (e2 - 3)) | (u >> e1);  // block group N2/8 j1 + g
    uint32_t w[8][4];
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const uint4 v = __ldg(&in[8 * g + c]);
      w[c][0] = v.x; w[c][1] = v.y; w[c][2] = v.z; w[c][3] = v.w;
    }
#pragma unroll
    for (int wd = 0; wd < 4; wd++) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        uint64_t x = 0;
#pragma unroll
        for (int c = 0; c < 8; c++) x |= uint64_t((w[c][wd] >> (8 * k)) & 0xffu) << (8 * c);
        x = transpose8(x);
        const int t = 8 * wd + 2 * k;
        tiles[uint64_t(t) * ngroups + u] = uint32_t(x);
        tiles[uint64_t(t + 1) * ngroups + u] = uint32_t(x >> 32);
      }
    }
  }
}

// Nibbles 0..3 of x at bits 0, 8, 16, 24.
__device__ __forceinline__ uint32_t spread_nibbles(uint32_t x) {
  x = (x | (x << 8)) & 0x00FF00FFu;
  return (x | (x << 4)) & 0x0F0F0F0Fu;
}

// The inverse of qcf_gather; out[j] = (xor_in ? xor_in[j] : 0) ^ block j.
// HALVES: the words hold two 16-bit halves from 4-column CTAs (low: columns
// 0-3, high: 4-7; nibble q of each: plane q), put back in byte order first
// (a template parameter: a runtime branch in the unrolled loop cost the
// loads' overlap, 2-7 % of the small dual LPNs).
template <bool HALVES>
__global__ void __launch_bounds__(256) qcf_scatter(const uint32_t *__restrict__ tiles, uint64_t ngroups, int e1,
                                                   int e2, const uint4 *__restrict__ xor_in, uint4 *__restrict__ out) {
  for (uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < ngroups;
       u += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t g = ((u & ((1ull << e1) - 1)) << (e2 - 3)) | (u >> e1);
    uint32_t w[8][4];
#pragma unroll
    for (int c = 0; c < 8; c++)
#pragma unroll
      for (int wd = 0; wd < 4; wd++) w[c][wd] = 0;
#pragma unroll
    for (int wd = 0; wd < 4; wd++) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int t = 8 * wd + 2 * k;
        uint32_t lo = __ldg(&tiles[uint64_t(t) * ngroups + u]), hi = __ldg(&tiles[uint64_t(t + 1) * ngroups + u]);
        if constexpr (HALVES) {
          lo = spread_nibbles(lo & 0xffffu) | (spread_nibbles(lo >> 16) << 4);
          hi = spread_nibbles(hi & 0xffffu) | (spread_nibbles(hi >> 16) << 4);
        }
        uint64_t x = uint64_t(lo) | uint64_t(hi) << 32;
        x = transpose8(x);
#pragma unroll
        for (int c = 0; c < 8; c++) w[c][wd] |= uint32_t((x >> (8 * c)) & 0xffu) << (8 * k);
      }
    }
#pragma unroll
    for (int c = 0; c < 8; c++) {
      uint4 v = make_uint4(w[c][0], w[c][1], w[c][2], w[c][3]);
      if (xor_in) {
        const uint4 a = __ldg(&xor_in[8 * g + c]);
        v.x ^= a.x; v.y ^= a.y; v.z ^= a.z; v.w ^= a.w;
      }
      out[8 * g + c] = v;
    }
  }
}

// Adds the weight of a (`words` 64-bit words) to *w.
__global__ void __launch_bounds__(256) qcf_weight(const uint64_t *__restrict__ a, uint64_t words,
                                                  unsigned long long *w) {
  unsigned long long c = 0;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < words; i += uint64_t(gridDim.x) * blockDim.x)
    c += __popcll(__ldg(&a[i]));
#pragma unroll
  for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(w, c);
}

// Table generation (one-time per n).  T: the pass-ordered twiddles of an
// N = 2^L point transform (entries past the last pass's offset unused).
__global__ void qcf_gen_roots(int L, double2 *T) {
  const int N = 1 << L;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    int p = 0;
    while (p + 1 < qcf_npass(L) && k >= qcf_tw_off(L, p + 1)) p++;
    const int K = qcf_k(L, p), LS = qcf_ls(L, p), M = (1 << LS) >> K;
    const int q = (k - qcf_tw_off(L, p)) / M + 1, base = (k - qcf_tw_off(L, p)) % M;
    const int e = (base * q) & ((1 << LS) - 1);
    double s, c;
    sincospi(2.0 * double(e) / double(1 << LS), &s, &c);
    T[k] = make_double2(c, -s);
  }
}
// fs[j2][u] = w_n^(j2 u) (u < 2^lo), fs[j2][2^lo + v] = w_n^(j2 v 2^lo).
__global__ void qcf_gen_fourstep(int e1, int e2, double2 *fs) {
  const int lo = qcf_fs_lo(e1), W = qcf_fs_width(e1);
  const uint64_t n = 1ull << (e1 + e2), N2 = 1ull << e2;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N2 * W;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t j2 = i / W, u = i % W;
    const uint64_t k = u < (1u << lo) ? u : (u - (1u << lo)) << lo;
    const uint64_t m = (j2 * k) & (n - 1);
    double s, c;
    sincospi(2.0 * double(m) / double(n), &s, &c);
    fs[i] = make_double2(c, -s);
  }
}

// Plane parity words per encode call in centred mode (one per transform).
constexpr int kQcfParCap = 4096;

struct QcfTables {
  int e, e1, e2;
  double2 *T1, *T2, *fs;
  uint32_t *par;          // centred mode: kQcfParCap plane-parity words
  const cuot_ctx *owner;  // context that caches the tables (its qc_streams)
  cudaStream_t aux;    // second stream of the two-stream group schedule
  cudaEvent_t ev[2];   // fork / join
};

namespace {

int qcf_alloc(void **p, size_t bytes) {
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(CUOT_ENOMEM, "QC FFT table allocation of %zu bytes failed", bytes);
  }
  return CUOT_OK;
}

void qcf_free(QcfTables *t) {
  if (!t) return;
  cudaFree(t->T1);
  cudaFree(t->T2);
  cudaFree(t->fs);
  cudaFree(t->par);
  if (t->aux) cudaStreamDestroy(t->aux);
  for (cudaEvent_t e : t->ev)
    if (e) cudaEventDestroy(e);
  delete t;
}

int col_smem(int e1, int kc) {
  const int N1 = 1 << e1;
  return (kc * (kc == 8 ? sld<8>(N1) : sld<4>(N1)) + qcf_fs_span(e1, kc)) * 16 + N1 * 4;
}
int row_smem(int e2) {
  const int N2 = 1 << e2;
  const int rows = qcf_rows(e2);
  const int ld = rows == 4 ? sld<4>(N2) : rows == 2 ? sld<2>(N2) : sld<1>(N2);
  const int tw = qcf_row_tg0(e2) ? qcf_tw_off(e2, qcf_npass(e2) - 1) - qcf_tw_off(e2, 1) : N2;
  return (rows * ld + tw) * 16;
}

#define QCF_CASES(X) X(5) X(6) X(7) X(8) X(9) X(10)
#define QCF_ROW_CASES(X) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)

int set_attrs() {
  static bool done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && done[dev]) return CUOT_OK;
  bool ok = true;
#define QCF_SETK(E, K)                                                                                  \
  ok &= cudaFuncSetAttribute(qcf_col_fwd<E, K, qcf_col_center(E)>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             col_smem(E, K)) == cudaSuccess;                                                \
  ok &= cudaFuncSetAttribute(qcf_col_inv<E, K, qcf_col_center(E)>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             col_smem(E, K)) == cudaSuccess;
#define QCF_SET(E) QCF_SETK(E, 8)
#define QCF_SETR(E) \
  ok &= cudaFuncSetAttribute(qcf_row<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_smem(E)) == cudaSuccess;
  QCF_CASES(QCF_SET)
  QCF_SETK(10, 4)
  QCF_ROW_CASES(QCF_SETR)
#undef QCF_SETK
#undef QCF_SET
#undef QCF_SETR
  if (!ok) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "QC FFT shared-memory attribute failed");
  }
  if (dev < 64) done[dev] = true;
  return CUOT_OK;
}

// par: plane-parity words of the launch's transforms (centred encodes), wa:
// the weight of `a` (centred A_hat builds), else null.
void launch_col_fwd(const QcfTables *t, int ntr, cudaStream_t st, const uint8_t *in, uint64_t stride_bytes,
                    int nplanes, int one_plane, const uint32_t *tiles, double2 *Y,
                    const unsigned long long *wa = nullptr, uint32_t *par = nullptr) {
  const int kc = tiles ? qcf_tile_kc(t->e) : 8;
  const dim3 grid((1u << t->e2) / kc, ntr);
#define QCF_LK(E, K)                                                                                           \
  qcf_col_fwd<E, K, qcf_col_center(E)><<<grid, qcf_col_threads(E, K), col_smem(E, K), st>>>(                  \
      in, stride_bytes, nplanes, one_plane, t->e2, qcf_wide(t->e), tiles, t->T1, t->fs, Y, wa, par);
  if (kc == 4) {
    QCF_LK(10, 4)
    return;
  }
  switch (t->e1) {
#define QCF_L(E) \
  case E:        \
    QCF_LK(E, 8) \
    break;
    QCF_CASES(QCF_L)
#undef QCF_L
#undef QCF_LK
  }
}
void launch_row(const QcfTables *t, int ntr, cudaStream_t st, double2 *Y, const QcfAhatTab &ahat, int mode,
                double2 *out, double scale) {
  const dim3 grid((1u << t->e1) / qcf_rows(t->e2), ntr);
  switch (t->e2) {
#define QCF_L(E)                                                                                         \
  case E:                                                                                                \
    qcf_row<E><<<grid, qcf_row_threads(E), row_smem(E), st>>>(Y, t->e1, t->T2, ahat, mode, out, scale);  \
    break;
    QCF_ROW_CASES(QCF_L)
#undef QCF_L
  }
}
void launch_col_inv(const QcfTables *t, int ntr, cudaStream_t st, const double2 *Y, uint8_t *out,
                    uint64_t stride_bytes, int nplanes, int accumulate, uint32_t *tiles, const QcfAhatTab &ahat,
                    const uint32_t *par) {
  const int kc = tiles ? qcf_tile_kc(t->e) : 8;
  const dim3 grid((1u << t->e2) / kc, ntr);
#define QCF_LK(E, K)                                                                                         \
  qcf_col_inv<E, K, qcf_col_center(E)><<<grid, qcf_col_threads(E, K), col_smem(E, K), st>>>(                \
      Y, t->e2, qcf_wide(t->e), t->T1, t->fs, out, stride_bytes, nplanes, accumulate, tiles, ahat, par);
  if (kc == 4) {
    QCF_LK(10, 4)
    return;
  }
  switch (t->e1) {
#define QCF_L(E) \
  case E:        \
    QCF_LK(E, 8) \
    break;
    QCF_CASES(QCF_L)
#undef QCF_L
#undef QCF_LK
  }
}

}  // namespace

bool qcf_supported(int e) { return e >= 10 && e <= kQcfMaxE; }

int qcf_get_tables(cuot_ctx *ctx, int e, QcfTables **out) {
  if (!qcf_supported(e)) return fail(CUOT_ENOTSUP, "QC FFT backend: n = 2^%d outside [2^10, 2^%d]", e, kQcfMaxE);
  if (ctx->qcf_tables[e]) {
    *out = static_cast<QcfTables *>(ctx->qcf_tables[e]);
    return CUOT_OK;
  }
  CUOT_TRY(set_attrs());
  QcfTables *t = new QcfTables{};
  t->e = e;
  t->owner = ctx;
  t->e1 = qcf_e1(e);
  t->e2 = e - t->e1;
  const uint64_t N1 = 1ull << t->e1, N2 = 1ull << t->e2;
  int st = CUOT_OK;
  if ((st = qcf_alloc((void **)&t->T1, N1 * 16)) || (st = qcf_alloc((void **)&t->T2, N2 * 16)) ||
      (st = qcf_alloc((void **)&t->fs, N2 * qcf_fs_width(t->e1) * 16)) ||
      (qcf_center(e) && (st = qcf_alloc((void **)&t->par, kQcfParCap * 4)))) {
    qcf_free(t);
    return st;
  }
  if (cudaStreamCreateWithFlags(&t->aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&t->ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&t->ev[1], cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    qcf_free(t);
    return fail(CUOT_ECUDA, "QC FFT stream / event creation failed");
  }
  qcf_gen_roots<<<8, 256>>>(t->e1, t->T1);
  qcf_gen_roots<<<8, 256>>>(t->e2, t->T2);
  qcf_gen_fourstep<<<256, 256>>>(t->e1, t->e2, t->fs);
  if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    qcf_free(t);
    return fail(CUOT_ECUDA, "QC FFT table generation failed");
  }
  ctx->qcf_tables[e] = t;
  *out = t;
  return CUOT_OK;
}

void qcf_free_ctx_tables(cuot_ctx *ctx) {
  for (int e = 0; e < 32; e++) {
    qcf_free(static_cast<QcfTables *>(ctx->qcf_tables[e]));
    ctx->qcf_tables[e] = nullptr;
  }
}

int qcf_build_ahat(const QcfTables *t, const uint64_t *a_d, void *Y, void *ahat, cudaStream_t st) {
  const uint64_t n = 1ull << t->e;
  unsigned long long *wa = nullptr;
  int launches = 2;
  if (qcf_center(t->e)) {  // w(a) into the trailer; the transform is of the lighter of a, ~a
    wa = reinterpret_cast<unsigned long long *>(static_cast<uint8_t *>(ahat) + 16 * n);
    if (cudaMemsetAsync(wa, 0, 8, st) != cudaSuccess) return launch_status(0);
    qcf_weight<<<148, 256, 0, st>>>(a_d, n / 64, wa);
    launches++;
  }
  launch_col_fwd(t, 1, st, reinterpret_cast<const uint8_t *>(a_d), n / 8, 1, 1, nullptr, static_cast<double2 *>(Y),
                 wa);
  launch_row(t, 1, st, static_cast<double2 *>(Y), QcfAhatTab{}, 1, static_cast<double2 *>(ahat), 1.0 / double(n));
  return launch_status(launches);
}

// Zeroes the plane-parity words of `ntr` transforms (centred mode).
static int clear_par(const QcfTables *t, int ntr, cudaStream_t st) {
  if (!t->par) return CUOT_OK;
  if (ntr > kQcfParCap) return fail(CUOT_EINVAL, "QC FFT: %d transforms in one call (at most %d)", ntr, kQcfParCap);
  return cudaMemsetAsync(t->par, 0, size_t(ntr) * 4, st) == cudaSuccess ? CUOT_OK : launch_status(0);
}

int qcf_encode(const QcfTables *t, const QcfAhatTab &ahat, const uint64_t *in, uint64_t *out, uint64_t stride,
               int accumulate, int nplanes, void *Y, int batch, cudaStream_t st) {
  batch = (batch + 3) & ~3;
  int launches = 0;
  for (int p0 = 0; p0 < nplanes; p0 += batch) {
    const int nb = nplanes - p0 < batch ? nplanes - p0 : batch;
    const int ntr = (nb + 3) / 4;
    QcfAhatTab tab = ahat;
    tab.first += p0 / 4;
    tab.margin = t->owner->qcf_margin;
    CUOT_TRY(clear_par(t, ntr, st));
    launch_col_fwd(t, ntr, st, reinterpret_cast<const uint8_t *>(in + uint64_t(p0) * stride), stride * 8, nb, 0,
                   nullptr, static_cast<double2 *>(Y), nullptr, t->par);
    launch_row(t, ntr, st, static_cast<double2 *>(Y), tab, 0, nullptr, 0.0);
    launch_col_inv(t, ntr, st, static_cast<const double2 *>(Y), reinterpret_cast<uint8_t *>(out + uint64_t(p0) * stride),
                   stride * 8, nb, accumulate, nullptr, tab, t->par);
    launches += 3;
  }
  return launch_status(launches);
}

int qcf_encode_tiles(const QcfTables *t, const QcfAhatTab &ahat, uint32_t *tiles, int ntransforms, void *Y,
                     int batch, cudaStream_t st) {
  const int bt = batch < 4 ? 1 : batch / 4;  // transforms per launch group
  const uint64_t words = 1ull << (t->e - 3);  // per transform
  const uint64_t ybytes = 16ull << t->e;      // intermediate of one transform
  int launches = 0;
  // Two-stream schedule: groups of G transforms (about 32 MiB of
  // intermediate each) alternate between the caller's stream and t->aux,
  // each stream with its own part of Y, so the intermediate of the two groups
  // in flight stays in L2 and one group's passes fill the other's wave tails.
  // Measured on B200 (one role's 128 planes): n = 2^20, G = 2: 0.78 ms
  // against 0.80 ms for one launch group of all 32 transforms; n = 2^18,
  // G = 8: 0.20 against 0.23 ms; n = 2^22, G = 1: 3.86 against 4.04 ms (at
  // 2^21, G = 1, 1.74 against 1.71 ms); with the current passes, n = 2^22
  // 3.48 against 3.65 ms on one stream, 2^21 1.59 against 1.61 ms, and a
  // third stream loses everywhere (2^20 0.83, 2^21 1.71, 2^22 3.50 ms:
  // intermediate evicted from L2).  It needs Y for 2G transforms.  A context
  // with CUOT_TUNE_QC_STREAMS = 1 keeps every group on the caller's stream
  // (callers that already run several encodes at once, such as the server).
  uint64_t g64 = (32ull << 20) / ybytes;
  const int G = g64 < 1 ? 1 : int(g64);
  CUOT_TRY(clear_par(t, ntransforms, st));
  uint32_t *par = t->par;
  if (t->owner->qc_streams == 2 && 2 * G <= bt && ntransforms > G) {
    cudaEventRecord(t->ev[0], st);
    cudaStreamWaitEvent(t->aux, t->ev[0], 0);
    int g = 0;
    for (int t0 = 0; t0 < ntransforms; t0 += G, g++) {
      const int ntr = ntransforms - t0 < G ? ntransforms - t0 : G;
      cudaStream_t s = (g & 1) ? t->aux : st;
      double2 *Yg = reinterpret_cast<double2 *>(static_cast<uint8_t *>(Y) + uint64_t(g & 1) * G * ybytes);
      QcfAhatTab tab = ahat;
      tab.first += t0;
      tab.margin = t->owner->qcf_margin;
      uint32_t *tp = tiles + uint64_t(t0) * words;
      uint32_t *pp = par ? par + t0 : nullptr;
      launch_col_fwd(t, ntr, s, nullptr, 0, 4 * ntr, 0, tp, Yg, nullptr, pp);
      launch_row(t, ntr, s, Yg, tab, 0, nullptr, 0.0);
      launch_col_inv(t, ntr, s, Yg, nullptr, 0, 4 * ntr, 0, tp, tab, pp);
      launches += 3;
    }
    cudaEventRecord(t->ev[1], t->aux);
    cudaStreamWaitEvent(st, t->ev[1], 0);
    return launch_status(launches);
  }
  for (int t0 = 0; t0 < ntransforms; t0 += bt) {
    const int ntr = ntransforms - t0 < bt ? ntransforms - t0 : bt;
    QcfAhatTab tab = ahat;
    tab.first += t0;
    tab.margin = t->owner->qcf_margin;
    uint32_t *tp = tiles + uint64_t(t0) * words;
    uint32_t *pp = par ? par + t0 : nullptr;
    launch_col_fwd(t, ntr, st, nullptr, 0, 4 * ntr, 0, tp, static_cast<double2 *>(Y), nullptr, pp);
    launch_row(t, ntr, st, static_cast<double2 *>(Y), tab, 0, nullptr, 0.0);
    launch_col_inv(t, ntr, st, static_cast<const double2 *>(Y), nullptr, 0, 4 * ntr, 0, tp, tab, pp);
    launches += 3;
  }
  return launch_status(launches);
}

int qcf_gather(int e, const cuot_block *in, uint32_t *tiles, cudaStream_t st) {
  const uint64_t ng = 1ull << (e - 3);
  const int e1 = qcf_e1(e);
  qcf_gather<<<unsigned((ng + 255) / 256), 256, 0, st>>>(reinterpret_cast<const uint4 *>(in), ng, e1, e - e1, tiles);
  return launch_status();
}

int qcf_scatter(int e, const uint32_t *tiles, const cuot_block *xor_in, cuot_block *out, cudaStream_t st) {
  const uint64_t ng = 1ull << (e - 3);
  const int e1 = qcf_e1(e);
  const dim3 grid(unsigned((ng + 255) / 256));
  if (qcf_tile_kc(e) == 4)
    qcf_scatter<true><<<grid, 256, 0, st>>>(tiles, ng, e1, e - e1, reinterpret_cast<const uint4 *>(xor_in),
                                            reinterpret_cast<uint4 *>(out));
  else
    qcf_scatter<false><<<grid, 256, 0, st>>>(tiles, ng, e1, e - e1, reinterpret_cast<const uint4 *>(xor_in),
                                             reinterpret_cast<uint4 *>(out));
  return launch_status();
}

}  // namespace cuot
