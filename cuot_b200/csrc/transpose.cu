// transpose.cu -- bit-matrix transpose (Mat::bit_transpose semantics,
// gpu/gpu_matrix.cu:95-121 with bit_transposer, gpu/gpu_ops.cu:31-70):
// output row (c - col_lo) bit r = input row r bit c, bits LSB-first.
//
// Fast paths (the two SOT shapes):
//   blocks -> planes: rows of 16 bytes, plane range multiple of 32.
//   planes -> blocks: up to 128 rows (planes) of n bits -> n rows.
// Both move 32x32 bit tiles with a five-step warp-shuffle transpose (one
// word per lane), stage through padded shared memory (stride 33 words, no
// bank conflicts) and read/write HBM with coalesced 16-byte or 128-byte
// accesses.  Any other shape uses a byte-granular 8x8 kernel.
#include "ctx.cuh"

namespace cuot {

// Lane i holds row i of a 32x32 bit tile (bit j = column j).  Returns the
// word of column `lane` (bit i = row i).
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane) {
  const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const int s = 16 >> k;
    const uint32_t m = masks[k];
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, s);
    if (lane & s) x = (x & ~m) | ((y >> s) & m);
    else x = (x & m) | ((y << s) & ~m);
  }
  return x;
}

constexpr int kTrThreads = 256;     // 8 warps
constexpr int kTrGroups = 32;       // row groups of 32 rows per CTA (128 B of each plane row)
constexpr int kTrStride = kTrGroups + 1;

// blocks -> planes.  in: rows x 16 bytes.  out: nplanes rows of rows/8 bytes.
__global__ void __launch_bounds__(kTrThreads) tr_blocks_to_planes(
    const uint4 *__restrict__ in, uint64_t rows, int col_lo, int nplanes,
    uint32_t *__restrict__ out) {
  __shared__ uint32_t st[128 * kTrStride];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t ngroups = rows / 32;
  const uint64_t g0 = uint64_t(blockIdx.x) * kTrGroups;
  const int wlo = col_lo / 32, nw = nplanes / 32;
  // all of a warp's row groups are loaded before any is transposed, so each
  // warp keeps kPer loads in flight
  constexpr int kPer = kTrGroups / (kTrThreads / 32);
  uint4 v[kPer];
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    const uint64_t g = g0 + warp + j * (kTrThreads / 32);
    v[j] = g < ngroups ? __ldcs(in + g * 32 + lane) : make_uint4(0, 0, 0, 0);
  }
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    const int gg = warp + j * (kTrThreads / 32);
    const uint32_t w[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (q < wlo || q >= wlo + nw) continue;
      const uint32_t col = warp_transpose32(w[q], lane);
      st[((q - wlo) * 32 + lane) * kTrStride + gg] = col;
    }
  }
  __syncthreads();
  const uint64_t words_per_plane = rows / 32;
  const int gvalid = int(ngroups - g0 < uint64_t(kTrGroups) ? ngroups - g0 : uint64_t(kTrGroups));
  for (int p = warp; p < nplanes; p += kTrThreads / 32) {
#pragma unroll
    for (int x = lane; x < kTrGroups; x += 32)
      if (x < gvalid) out[uint64_t(p) * words_per_plane + g0 + x] = st[p * kTrStride + x];
  }
}

// planes -> blocks.  in: nrows (<= 128, multiple of 32) rows of ncols bits.
// out: ncols rows of nrows/8 bytes.
__global__ void __launch_bounds__(kTrThreads) tr_planes_to_blocks(
    const uint32_t *__restrict__ in, int nrows, uint64_t ncols, uint64_t in_row_words,
    uint32_t *__restrict__ out) {
  __shared__ uint32_t st[128 * kTrStride];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t ngroups = ncols / 32;
  const uint64_t g0 = uint64_t(blockIdx.x) * kTrGroups;
  const int gvalid = int(ngroups - g0 < uint64_t(kTrGroups) ? ngroups - g0 : uint64_t(kTrGroups));
  // each warp's plane rows are loaded together (up to 16 loads in flight per
  // 32-word chunk of the rows)
  constexpr int kPer = 128 / (kTrThreads / 32);
#pragma unroll
  for (int x0 = 0; x0 < kTrGroups; x0 += 32) {
    const int x = x0 + lane;
    uint32_t v[kPer];
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      const int p = warp + j * (kTrThreads / 32);
      v[j] = (p < nrows && x < gvalid) ? __ldcs(in + uint64_t(p) * in_row_words + g0 + x) : 0u;
    }
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      const int p = warp + j * (kTrThreads / 32);
      if (p < nrows && x < gvalid) st[p * kTrStride + x] = v[j];
    }
  }
  __syncthreads();
  const int nq = nrows / 32;
  for (int gg = warp; gg < gvalid; gg += kTrThreads / 32) {
    uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < nq) w[q] = warp_transpose32(st[(q * 32 + lane) * kTrStride + gg], lane);
    const uint64_t row = (g0 + gg) * 32 + lane;
    if (nq == 4) {
      reinterpret_cast<uint4 *>(out)[row] = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
      for (int q = 0; q < nq; q++) out[row * nq + q] = w[q];
    }
  }
}

// Generic: thread (i, jb) transposes the 8x8 bit tile formed by input rows
// 8i..8i+7 at byte column col_lo/8 + jb.
__global__ void tr_generic(const uint8_t *__restrict__ in, uint64_t rows, uint64_t row_bytes,
                           uint64_t byte_lo, uint64_t nbytes_cols, uint8_t *__restrict__ out) {
  const uint64_t nrb = rows / 8;
  const uint64_t total = nrb * nbytes_cols;
  for (uint64_t id = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; id < total;
       id += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t i = id % nrb, jb = id / nrb;
    uint64_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; k++)
      x |= uint64_t(in[(8 * i + k) * row_bytes + byte_lo + jb]) << (8 * k);
    // bit (8r + c) -> bit (8c + r): three delta swaps (Hacker's Delight 7-3)
    uint64_t t;
    t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;  x ^= t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull; x ^= t ^ (t << 14);
    t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull; x ^= t ^ (t << 28);
#pragma unroll
    for (int k = 0; k < 8; k++) out[(8 * jb + k) * nrb + i] = uint8_t(x >> (8 * k));
  }
}

int transpose_launch(const void *in, uint64_t rows, uint64_t row_bytes, uint64_t col_lo,
                     uint64_t col_hi, void *out, cudaStream_t st) {
  const uint64_t ncols = col_hi - col_lo;
  if (row_bytes == 16 && rows % 32 == 0 && col_lo % 32 == 0 && ncols % 32 == 0 && ncols > 0) {
    const uint64_t ngroups = rows / 32;
    const uint64_t grid = (ngroups + kTrGroups - 1) / kTrGroups;
    if (grid > 0x7fffffffull) return fail(CUOT_EINVAL, "too many rows");
    tr_blocks_to_planes<<<unsigned(grid), kTrThreads, 0, st>>>(
        static_cast<const uint4 *>(in), rows, int(col_lo), int(ncols),
        static_cast<uint32_t *>(out));
    return launch_status();
  }
  if (rows % 32 == 0 && rows <= 128 && col_lo == 0 && ncols == row_bytes * 8 &&
      ncols % 32 == 0 && (row_bytes % 4) == 0) {
    const uint64_t ngroups = ncols / 32;
    const uint64_t grid = (ngroups + kTrGroups - 1) / kTrGroups;
    if (grid > 0x7fffffffull) return fail(CUOT_EINVAL, "too many columns");
    tr_planes_to_blocks<<<unsigned(grid), kTrThreads, 0, st>>>(
        static_cast<const uint32_t *>(in), int(rows), ncols, row_bytes / 4,
        static_cast<uint32_t *>(out));
    return launch_status();
  }
  const uint64_t total = (rows / 8) * (ncols / 8);
  uint64_t grid = (total + 255) / 256;
  if (grid > 65535ull * 16) grid = 65535ull * 16;
  if (grid == 0) return CUOT_OK;
  tr_generic<<<unsigned(grid), 256, 0, st>>>(static_cast<const uint8_t *>(in), rows,
                                              row_bytes, col_lo / 8, ncols / 8,
                                              static_cast<uint8_t *>(out));
  return launch_status();
}

// Device -> mapped host memory through SM stores (16-byte words when both
// ends and the size allow it, bytes otherwise).
__global__ void host_store16(const uint4 *__restrict__ src, uint4 *__restrict__ dst, uint64_t n) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    dst[i] = __ldg(&src[i]);
}
__global__ void host_store1(const uint8_t *__restrict__ src, uint8_t *__restrict__ dst, uint64_t n) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    dst[i] = src[i];
}

}  // namespace cuot

using namespace cuot;

extern "C" int cuot_bit_transpose(cuot_ctx *ctx, const void *in_d, uint64_t rows,
                                  uint64_t row_bytes, uint64_t col_lo, uint64_t col_hi,
                                  void *out_d, void *stream) {
  if (!ctx || !in_d || !out_d) return fail(CUOT_EINVAL, "null argument");
  if (rows % 8 || col_lo % 8 || col_hi % 8 || col_hi <= col_lo || col_hi > row_bytes * 8)
    return fail(CUOT_EINVAL, "bad transpose shape rows=%llu row_bytes=%llu cols=[%llu,%llu)",
                (unsigned long long)rows, (unsigned long long)row_bytes,
                (unsigned long long)col_lo, (unsigned long long)col_hi);
  if (rows == 0) return CUOT_OK;
  DeviceGuard g(ctx);
  return transpose_launch(in_d, rows, row_bytes, col_lo, col_hi, out_d,
                          static_cast<cudaStream_t>(stream));
}

extern "C" int cuot_copy_to_host(const void *src_d, void *dst_h, uint64_t bytes, void *stream) {
  if (bytes == 0) return CUOT_OK;
  if (!src_d || !dst_h) return fail(CUOT_EINVAL, "null argument");
  void *dst = nullptr;
  if (cudaHostGetDevicePointer(&dst, dst_h, 0) != cudaSuccess || !dst) {
    cudaGetLastError();
    return fail(CUOT_EINVAL, "destination is not mapped pinned host memory");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool v16 = (reinterpret_cast<uintptr_t>(src_d) % 16 == 0) && (reinterpret_cast<uintptr_t>(dst) % 16 == 0) &&
                   bytes % 16 == 0;
  const uint64_t n = v16 ? bytes / 16 : bytes;
  uint64_t grid = (n + 255) / 256;
  if (grid > 148 * 8) grid = 148 * 8;
  if (v16)
    host_store16<<<unsigned(grid), 256, 0, st>>>(static_cast<const uint4 *>(src_d), static_cast<uint4 *>(dst), n);
  else
    host_store1<<<unsigned(grid), 256, 0, st>>>(static_cast<const uint8_t *>(src_d), static_cast<uint8_t *>(dst), n);
  return launch_status();
}
