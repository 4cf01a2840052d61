// qc_kara.cu -- exact QC dual LPN for n = 2^23 and 2^24 as GF(2) Karatsuba
// over the fp64 FFT of qc_fft.cu (which is exact up to 2^22).
//
// Block j of the dual LPN holds coefficient j of all 128 bit planes, so with
// y = x^2, a(x) = a0(y) + x a1(y) (a0 / a1: even / odd bits of a) and
// e(x) = e0(y) + x e1(y) (e0 / e1: even / odd blocks),
//   a e mod (x^n - 1) = [a0 e0 + y a1 e1](y) + x [a0 e1 + a1 e0](y)
// mod y^(n/2) - 1, and over GF(2) a0 e1 + a1 e0 = (a0+a1)(e0+e1) + a0 e0 +
// a1 e1.  Three products of half size per level:
//   P1 = a0 e0, P2 = a1 e1, P3 = (a0 ^ a1)(e0 ^ e1),
//   out[2k] = P1[k] ^ P2[k-1 mod n/2],  out[2k+1] = P3[k] ^ P1[k] ^ P2[k].
// One level turns 2^23 into three 2^22 FFT dual LPNs, two levels turn 2^24
// into nine; each leaf is the exact FFT path, so the result is exact.  The
// transforms of the 3^L leaf polynomials are computed once (the plan's
// A_hat, leaves in the order P1, P2, P3 per level, depth first).
#include "ctx.cuh"

namespace cuot {
namespace {

// 32 bits from the even bits of x.
__device__ __forceinline__ uint64_t even_bits(uint64_t x) {
  x &= 0x5555555555555555ull;
  x = (x | (x >> 1)) & 0x3333333333333333ull;
  x = (x | (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
  x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
  x = (x | (x >> 16)) & 0x00000000FFFFFFFFull;
  return x;
}

// a (2 * hw words) -> a0 (even bits), a1 (odd bits), a01 = a0 ^ a1 (hw words each).
__global__ void qck_split_bits(const uint64_t *__restrict__ a, uint64_t hw, uint64_t *__restrict__ a0,
                               uint64_t *__restrict__ a1, uint64_t *__restrict__ a01) {
  for (uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < hw; w += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t x = a[2 * w], y = a[2 * w + 1];
    const uint64_t e = even_bits(x) | (even_bits(y) << 32);
    const uint64_t o = even_bits(x >> 1) | (even_bits(y >> 1) << 32);
    a0[w] = e;
    a1[w] = o;
    a01[w] = e ^ o;
  }
}

// in (2 * half blocks) -> p1 (even blocks), p2 (odd blocks), p3 = p1 ^ p2.
__global__ void qck_split(const uint4 *__restrict__ in, uint64_t half, uint4 *__restrict__ p1, uint4 *__restrict__ p2,
                          uint4 *__restrict__ p3) {
  for (uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < half; k += uint64_t(gridDim.x) * blockDim.x) {
    const uint4 u = __ldg(&in[2 * k]), v = __ldg(&in[2 * k + 1]);
    p1[k] = u;
    p2[k] = v;
    p3[k] = make_uint4(u.x ^ v.x, u.y ^ v.y, u.z ^ v.z, u.w ^ v.w);
  }
}

__device__ __forceinline__ uint4 x4(uint4 a, uint4 b) { return make_uint4(a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w); }

// out[2k] = (xor_in) ^ P1[k] ^ P2[k-1], out[2k+1] = (xor_in) ^ P3[k] ^ P1[k] ^ P2[k].
__global__ void qck_combine(const uint4 *__restrict__ p1, const uint4 *__restrict__ p2, const uint4 *__restrict__ p3,
                            uint64_t half, const uint4 *xor_in, uint4 *out) {
  for (uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < half; k += uint64_t(gridDim.x) * blockDim.x) {
    const uint4 a = __ldg(&p1[k]), b = __ldg(&p2[k]), bp = __ldg(&p2[k ? k - 1 : half - 1]), c = __ldg(&p3[k]);
    uint4 ev = x4(a, bp), od = x4(x4(c, a), b);
    if (xor_in) {
      ev = x4(ev, xor_in[2 * k]);
      od = x4(od, xor_in[2 * k + 1]);
    }
    out[2 * k] = ev;
    out[2 * k + 1] = od;
  }
}

unsigned grid_for(uint64_t items) {
  uint64_t g = (items + 255) / 256;
  return unsigned(g > 148 * 16 ? 148 * 16 : (g ? g : 1));
}

uint64_t pow3(int l) {
  uint64_t r = 1;
  while (l-- > 0) r *= 3;
  return r;
}

constexpr uint64_t kLeafN = 1ull << kQcfMaxE;
constexpr uint64_t kLeafAhat = qcf_ahat_bytes(kQcfMaxE);  // bytes of one leaf's transform

int ahat_tree(const QcfTables *leaf, int e, const uint64_t *a, uint8_t *bits, void *Y, uint8_t *ahat, cudaStream_t st) {
  if (e == kQcfMaxE) return qcf_build_ahat(leaf, a, Y, ahat, st);
  const uint64_t hw = (1ull << e) / 128;  // words of each half
  uint64_t *a0 = reinterpret_cast<uint64_t *>(bits), *a1 = a0 + hw, *a01 = a1 + hw;
  qck_split_bits<<<grid_for(hw), 256, 0, st>>>(a, hw, a0, a1, a01);
  CUOT_TRY(launch_status());
  const uint64_t sub = pow3(e - 1 - kQcfMaxE) * kLeafAhat;
  uint8_t *rest = reinterpret_cast<uint8_t *>(a01 + hw);
  CUOT_TRY(ahat_tree(leaf, e - 1, a0, rest, Y, ahat, st));
  CUOT_TRY(ahat_tree(leaf, e - 1, a1, rest, Y, ahat + sub, st));
  return ahat_tree(leaf, e - 1, a01, rest, Y, ahat + 2 * sub, st);
}

int kara(const QcfTables *leaf, int e, const uint8_t *ahat, const cuot_block *in, const cuot_block *xor_in,
         cuot_block *out, uint8_t *scr, void *Y, int batch, cudaStream_t st) {
  if (e == kQcfMaxE) {
    uint32_t *tiles = reinterpret_cast<uint32_t *>(scr);
    QcfAhatTab tab{};
    tab.p[0] = ahat;
    tab.per = 1 << 30;
    CUOT_TRY(qcf_gather(e, in, tiles, st));
    CUOT_TRY(qcf_encode_tiles(leaf, tab, tiles, 32, Y, batch, st));
    return qcf_scatter(e, tiles, xor_in, out, st);
  }
  const uint64_t half = 1ull << (e - 1);
  cuot_block *p1 = reinterpret_cast<cuot_block *>(scr), *p2 = p1 + half, *p3 = p2 + half;
  qck_split<<<grid_for(half), 256, 0, st>>>(reinterpret_cast<const uint4 *>(in), half, reinterpret_cast<uint4 *>(p1),
                                            reinterpret_cast<uint4 *>(p2), reinterpret_cast<uint4 *>(p3));
  CUOT_TRY(launch_status());
  const uint64_t sub = pow3(e - 1 - kQcfMaxE) * kLeafAhat;
  uint8_t *rest = reinterpret_cast<uint8_t *>(p3 + half);
  CUOT_TRY(kara(leaf, e - 1, ahat, p1, nullptr, p1, rest, Y, batch, st));
  CUOT_TRY(kara(leaf, e - 1, ahat + sub, p2, nullptr, p2, rest, Y, batch, st));
  CUOT_TRY(kara(leaf, e - 1, ahat + 2 * sub, p3, nullptr, p3, rest, Y, batch, st));
  qck_combine<<<grid_for(half), 256, 0, st>>>(reinterpret_cast<const uint4 *>(p1), reinterpret_cast<const uint4 *>(p2),
                                              reinterpret_cast<const uint4 *>(p3), half,
                                              reinterpret_cast<const uint4 *>(xor_in), reinterpret_cast<uint4 *>(out));
  return launch_status();
}

}  // namespace

bool qck_supported(int e) { return e > kQcfMaxE && e <= kQcfMaxE + kQckMaxLevels; }

uint64_t qck_ahat_bytes(int e) { return pow3(e - kQcfMaxE) * kLeafAhat; }

uint64_t qck_scratch_bytes(int e) {
  // split blocks of every level (3 halves each) + the leaf's tile words
  uint64_t b = 16 * kLeafN;
  for (int l = e; l > kQcfMaxE; l--) b += 3 * 16 * (1ull << (l - 1));
  return b;
}

uint64_t qck_bits_scratch_bytes(int e) {
  uint64_t b = 0;
  for (int l = e; l > kQcfMaxE; l--) b += 3 * (1ull << (l - 1)) / 8;
  return b;
}

int qck_build_ahat(const QcfTables *leaf, int e, const uint64_t *a_d, void *bits, void *Y, void *ahat,
                   cudaStream_t st) {
  return ahat_tree(leaf, e, a_d, static_cast<uint8_t *>(bits), Y, static_cast<uint8_t *>(ahat), st);
}

int qck_dual_lpn(const QcfTables *leaf, int e, const void *ahat, const cuot_block *in, const cuot_block *xor_in,
                 cuot_block *out, void *scratch, void *Y, int batch, cudaStream_t st) {
  return kara(leaf, e, static_cast<const uint8_t *>(ahat), in, xor_in, out, static_cast<uint8_t *>(scratch), Y, batch,
              st);
}

}  // namespace cuot
