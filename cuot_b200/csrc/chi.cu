// chi.cu -- per-tree chi sums of Ferret's malicious consistency check.
//
// For tree j with seed s_j (the first 16 bytes of Hash(secret_sum_j)), the
// sender's check value is V_j = sum_{i < 2^h} s_j^(i+1) * v_{j,i} over
// GF(2^128), and the receiver computes the same sum W_j over its leaves
// (spcot_sender.h:88-98, spcot_recver.h:97-107: uni_hash_coeff_gen followed
// by vector_inn_prdt_sum_red).  Field: natural bit order (bit i of the
// little-endian block is the coefficient of x^i), reduction polynomial
// x^128 + x^7 + x^2 + x + 1 (emp-tool's gfmul).
//
// B200 has no carry-less multiply, so one CTA per tree turns the sum into a
// polynomial evaluation with a single repeated multiplier:
//   thread j (of 256) runs Horner over its leaves i = j + 256 q with the
//   multiplier u = s^256:  P_j = sum_q v_{j+256q} u^q;
//   then sum_j s^j P_j is folded in 8 levels of a binary tree (level l
//   multiplies by s^(2^l)), and V = s * (that sum).
// Multiplication by the fixed u uses byte tables in shared memory: T[k][b] =
// u * (b x^(8k)), so u * x = XOR_k T[k][byte k of x] -- 16 conflict-light
// 128-bit lookups per leaf instead of a 128 x 128 carry-less product.  The
// squarings s^(2^l) spread bits (squaring is linear in characteristic 2);
// the few general products (tree levels) are bit-serial.
#include "ctx.cuh"

namespace cuot {
namespace {

constexpr int kChiThreads = 256;
constexpr int kChiTableBytes = 16 * 256 * 16;

struct U128 {
  uint64_t lo, hi;
};

__device__ __forceinline__ U128 u128(const uint4 v) {
  return U128{uint64_t(v.x) | (uint64_t(v.y) << 32), uint64_t(v.z) | (uint64_t(v.w) << 32)};
}
__device__ __forceinline__ uint4 to_u4(U128 a) {
  return make_uint4(uint32_t(a.lo), uint32_t(a.lo >> 32), uint32_t(a.hi), uint32_t(a.hi >> 32));
}
__device__ __forceinline__ U128 xor128(U128 a, U128 b) { return U128{a.lo ^ b.lo, a.hi ^ b.hi}; }
// a * x, reduced (x^128 = x^7 + x^2 + x + 1)
__device__ __forceinline__ U128 mulx(U128 a) {
  const uint64_t c = a.hi >> 63;
  return U128{(a.lo << 1) ^ (c * 0x87ull), (a.hi << 1) | (a.lo >> 63)};
}
// general product: r = XOR_i a_i (b x^i), with b x^i advanced by one mulx per
// bit, so the dependency chain is the short mulx and the accumulation
// pipelines behind it
__device__ U128 gmul(U128 a, U128 b) {
  U128 r{0, 0}, bx = b;
#pragma unroll 8
  for (int i = 0; i < 128; i++) {
    const uint64_t m = 0 - ((i < 64 ? a.lo >> i : a.hi >> (i - 64)) & 1);
    r.lo ^= bx.lo & m;
    r.hi ^= bx.hi & m;
    bx = mulx(bx);
  }
  return r;
}
// bits i -> 2i of a 32-bit word
__device__ __forceinline__ uint64_t spread32(uint32_t x) {
  uint64_t v = x;
  v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
  v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
  v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
  v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull;
  return v;
}
// a^2: squaring is GF(2)-linear (bit i -> bit 2i), then the high 128 bits
// are folded with x^128 = x^7 + x^2 + x + 1 (twice: the first fold spills
// at most 7 bits)
__device__ U128 gsqr(U128 a) {
  uint64_t r0 = spread32(uint32_t(a.lo)), r1 = spread32(uint32_t(a.lo >> 32));
  uint64_t r2 = spread32(uint32_t(a.hi)), r3 = spread32(uint32_t(a.hi >> 32));
#pragma unroll
  for (int pass = 0; pass < 2; pass++) {
    const uint64_t h0 = r2, h1 = r3;
    r2 = r3 = 0;
    r0 ^= h0 ^ (h0 << 1) ^ (h0 << 2) ^ (h0 << 7);
    r1 ^= h1 ^ (h1 << 1) ^ (h1 << 2) ^ (h1 << 7) ^ (h0 >> 63) ^ (h0 >> 62) ^ (h0 >> 57);
    r2 ^= (h1 >> 63) ^ (h1 >> 62) ^ (h1 >> 57);
  }
  return U128{r0, r1};
}

// u * x with the byte tables T (16 x 256 entries)
__device__ __forceinline__ U128 tmul(const uint4 *__restrict__ T, const uint4 x) {
  uint4 r = make_uint4(0, 0, 0, 0);
  const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
  for (int k = 0; k < 16; k++) {
    const uint4 e = T[k * 256 + ((w[k >> 2] >> (8 * (k & 3))) & 255)];
    r.x ^= e.x; r.y ^= e.y; r.z ^= e.z; r.w ^= e.w;
  }
  return u128(r);
}

__global__ void __launch_bounds__(kChiThreads) chi_sum_kernel(const uint4 *__restrict__ leaves, int h,
                                                              const uint4 *__restrict__ seeds,
                                                              uint4 *__restrict__ out) {
  extern __shared__ uint4 T[];         // [16][256]: u * (b x^(8k))
  __shared__ uint4 basis[128];         // u * x^m
  __shared__ uint4 P[kChiThreads];     // per-thread partial sums, then the tree
  __shared__ uint4 spow[9];            // s^(2^l), l = 0..8 (spow[8] = u)
  const int tree = blockIdx.x;
  const U128 s = u128(__ldg(&seeds[tree]));
  if (threadIdx.x == 0) {
    U128 c = s;
    spow[0] = to_u4(c);
    for (int l = 1; l <= 8; l++) {
      c = gsqr(c);
      spow[l] = to_u4(c);
    }
    U128 b = c;  // u * x^0
    for (int m = 0; m < 128; m++) {
      basis[m] = to_u4(b);
      b = mulx(b);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 16 * 256; e += blockDim.x) {
    const int k = e >> 8, byte = e & 255;
    uint4 r = make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if ((byte >> j) & 1) {
        const uint4 v = basis[8 * k + j];
        r.x ^= v.x; r.y ^= v.y; r.z ^= v.z; r.w ^= v.w;
      }
    }
    T[e] = r;
  }
  __syncthreads();
  // Horner over this thread's leaves j + 256 q, highest q first
  const int64_t L = int64_t(1) << h;
  const uint4 *lv = leaves + tree * L;
  const int j = threadIdx.x;
  U128 acc{0, 0};
  if (j < L) {
    const int64_t Q = L > kChiThreads ? L / kChiThreads : 1;
    for (int64_t q = Q - 1; q >= 0; q--) {
      acc = xor128(tmul(T, to_u4(acc)), u128(__ldg(&lv[j + kChiThreads * q])));
    }
  }
  P[j] = to_u4(acc);
  __syncthreads();
  // sum_j s^j P_j: level l folds P[i + 2^l] * s^(2^l) into P[i], i = 0 mod 2^(l+1)
  for (int l = 0; l < 8; l++) {
    const int stride = 1 << l;
    if ((j & (2 * stride - 1)) == 0) {
      const U128 c = u128(spow[l]);
      P[j] = to_u4(xor128(u128(P[j]), gmul(c, u128(P[j + stride]))));
    }
    __syncthreads();
  }
  if (j == 0) out[tree] = to_u4(gmul(s, u128(P[0])));
}

}  // namespace
}  // namespace cuot

using namespace cuot;

extern "C" {

int cuot_ferret_chi_sum(cuot_ctx *ctx, const cuot_block *leaves_d, uint64_t t, int h,
                        const cuot_block *seeds_d, cuot_block *out_d, void *stream) {
  if (!ctx || !leaves_d || !seeds_d || !out_d) return fail(CUOT_EINVAL, "null argument");
  if (t < 1 || t > 0x7fffffffull) return fail(CUOT_EINVAL, "t=%llu out of range", (unsigned long long)t);
  if (h < 1 || h > 30) return fail(CUOT_EINVAL, "h=%d out of range [1,30]", h);
  DeviceGuard g(ctx);
  static bool attr_set[64] = {false};
  if (ctx->device < 64 && !attr_set[ctx->device]) {
    if (cudaFuncSetAttribute(chi_sum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kChiTableBytes) !=
        cudaSuccess) {
      cudaGetLastError();
      return fail(CUOT_ECUDA, "chi kernel attribute failed");
    }
    attr_set[ctx->device] = true;
  }
  chi_sum_kernel<<<dim3((unsigned)t), kChiThreads, kChiTableBytes, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const uint4 *>(leaves_d), h, reinterpret_cast<const uint4 *>(seeds_d),
      reinterpret_cast<uint4 *>(out_d));
  return launch_status();
}

}  // extern "C"
