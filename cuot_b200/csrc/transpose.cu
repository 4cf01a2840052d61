// transpose.cu -- bit-matrix transpose (Mat::bit_transpose semantics,
// gpu/gpu_matrix.cu:95-121 with bit_transposer, gpu/gpu_ops.cu:31-70):
// output row (c - col_lo) bit r = input row r bit c, bits LSB-first.
//
// Fast paths (the SOT shapes):
//   blocks -> all 128 planes, and 128 planes -> blocks: 16-byte global
//     accesses on both sides, plane rows staged in an XOR-swizzled shared
//     tile (tr_blocks_to_planes128, tr_planes128_to_blocks);
//   blocks -> any multiple of 32 planes, and up to 128 planes -> blocks:
//     padded shared tile (stride 33 words), 4-byte plane-row accesses.
// All move 32x32 bit tiles with a five-stage warp-shuffle transpose (one word
// per lane).  Any other shape, or a pointer not aligned for the fast path's
// accesses, uses a byte-granular 8x8 kernel.
#include "ctx.cuh"

namespace cuot {

// Per-lane constants of warp_transpose32: byte-permute selectors of the
// 16- and 8-bit stages, rotate amounts and keep-masks of the 4-, 2- and
// 1-bit stages.
struct TrLane {
  uint32_t sel16, sel8, amt[3], keep[3];
};
__device__ __forceinline__ TrLane tr_lane(int lane) {
  TrLane t;
  t.sel16 = (lane & 16) ? 0x3276u : 0x5410u;  // (y.hi16, x.hi16) : (x.lo16, y.lo16) as (hi, lo)
  t.sel8 = (lane & 8) ? 0x3715u : 0x6240u;
  const uint32_t m[3] = {0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int s = 4 >> k;
    const bool up = lane & s;
    t.amt[k] = up ? 32 - s : s;
    t.keep[k] = up ? ~m[k] : m[k];
  }
  return t;
}

// Lane i holds row i of a 32x32 bit tile (bit j = column j).  Returns the
// word of column `lane` (bit i = row i).  Five exchange stages with the lane
// 16, 8, 4, 2, 1 apart: a lane keeps the half of its word whose column bit
// equals its own lane bit and takes the other half from its partner.  The
// 16- and 8-bit stages are one byte permute each; the others rotate the
// partner's word by s (lower lane) or 32 - s (upper lane), which lands the
// wanted half in place either way, and merge by a bit-select.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, const TrLane &t) {
  uint32_t y = __shfl_xor_sync(0xffffffffu, x, 16);
  x = __byte_perm(x, y, t.sel16);
  y = __shfl_xor_sync(0xffffffffu, x, 8);
  x = __byte_perm(x, y, t.sel8);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    y = __shfl_xor_sync(0xffffffffu, x, 4 >> k);
    const uint32_t r = __funnelshift_l(y, y, t.amt[k]);
    x = (x & t.keep[k]) | (r & ~t.keep[k]);
  }
  return x;
}

constexpr int kTrThreads = 256;     // 8 warps

// 128-plane fast paths.  A CTA moves kTrG groups of 32 rows: 16 * 32 * kTrG
// bytes of blocks <-> 128 plane rows of 4 * kTrG bytes.  The plane rows are
// staged in shared memory as [plane][kTrG / 4 chunks of 16 bytes] with chunk
// c of plane p at c ^ (p & 7): a warp storing one chunk of 32 planes and a
// warp reading 8 consecutive chunks of a plane both hit 8 distinct 16-byte
// bank groups per quarter-warp (conflict-free).  Global memory is read and
// written in 16-byte words only.
constexpr int kTrG = 32;
constexpr int kTrCh = kTrG / 4;                   // 16-byte chunks per plane row
constexpr int kTrCpw = kTrCh / (kTrThreads / 32);  // chunks per warp
static_assert(kTrCpw >= 1 && kTrCh >= 8, "tile shape");

// blocks -> planes, all 128 planes.  in: rows x 16 bytes (rows % 128 == 0).
// out: 128 rows of rows / 8 bytes.
__global__ void __launch_bounds__(kTrThreads) tr_blocks_to_planes128(const uint4 *__restrict__ in, uint64_t rows,
                                                                     uint4 *__restrict__ out) {
  __shared__ uint4 st[128 * kTrCh];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const TrLane tl = tr_lane(lane);
  const uint64_t ngroups = rows / 32;
  const uint64_t g0 = uint64_t(blockIdx.x) * kTrG;
  const int gvalid = int(ngroups - g0 < uint64_t(kTrG) ? ngroups - g0 : uint64_t(kTrG));  // multiple of 4
  // the warp's 4 * kTrCpw row groups are all loaded before any is transposed
  uint4 v[4 * kTrCpw];
#pragma unroll
  for (int c = 0; c < kTrCpw; c++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int gg = (warp * kTrCpw + c) * 4 + j;
      v[c * 4 + j] = gg < gvalid ? __ldcs(in + (g0 + gg) * 32 + lane) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
  for (int c = 0; c < kTrCpw; c++) {
    const int ch = warp * kTrCpw + c;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uint32_t o[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint4 &x = v[c * 4 + j];
        o[j] = warp_transpose32(q == 0 ? x.x : q == 1 ? x.y : q == 2 ? x.z : x.w, tl);
      }
      const int p = q * 32 + lane;
      st[p * kTrCh + (ch ^ (p & 7))] = make_uint4(o[0], o[1], o[2], o[3]);
    }
  }
  __syncthreads();
  const uint64_t row4 = rows / 128;  // 16-byte words per plane row
  for (int i = threadIdx.x; i < 128 * kTrCh; i += kTrThreads) {
    const int p = i / kTrCh, ch = i % kTrCh;
    if (4 * ch < gvalid) out[uint64_t(p) * row4 + g0 / 4 + ch] = st[p * kTrCh + (ch ^ (p & 7))];
  }
}

// planes -> blocks, 128 planes.  in: 128 rows of in_row4 16-byte words, of
// which the first ncols / 128 are read (ncols % 128 == 0).  out: ncols rows of
// 16 bytes.
__global__ void __launch_bounds__(kTrThreads) tr_planes128_to_blocks(const uint4 *__restrict__ in, uint64_t ncols,
                                                                     uint64_t in_row4, uint4 *__restrict__ out) {
  __shared__ uint4 st[128 * kTrCh];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const TrLane tl = tr_lane(lane);
  const uint64_t ngroups = ncols / 32;
  const uint64_t g0 = uint64_t(blockIdx.x) * kTrG;
  const int gvalid = int(ngroups - g0 < uint64_t(kTrG) ? ngroups - g0 : uint64_t(kTrG));  // multiple of 4
  constexpr int kLd = 128 * kTrCh / kTrThreads;
  uint4 v[kLd];
#pragma unroll
  for (int j = 0; j < kLd; j++) {
    const int i = threadIdx.x + j * kTrThreads, p = i / kTrCh, ch = i % kTrCh;
    v[j] = 4 * ch < gvalid ? __ldcs(in + uint64_t(p) * in_row4 + g0 / 4 + ch) : make_uint4(0, 0, 0, 0);
  }
#pragma unroll
  for (int j = 0; j < kLd; j++) {
    const int i = threadIdx.x + j * kTrThreads, p = i / kTrCh, ch = i % kTrCh;
    st[p * kTrCh + (ch ^ (p & 7))] = v[j];
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < kTrCpw; c++) {
    const int ch = warp * kTrCpw + c;
    if (4 * ch >= gvalid) break;
    uint32_t o[4][4];  // [row group j][plane word q]
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int p = q * 32 + lane;
      const uint4 x = st[p * kTrCh + (ch ^ (p & 7))];
      o[0][q] = warp_transpose32(x.x, tl);
      o[1][q] = warp_transpose32(x.y, tl);
      o[2][q] = warp_transpose32(x.z, tl);
      o[3][q] = warp_transpose32(x.w, tl);
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
      out[(g0 + ch * 4 + j) * 32 + lane] = make_uint4(o[j][0], o[j][1], o[j][2], o[j][3]);
  }
}

constexpr int kTrGroups = 32;       // row groups of 32 rows per CTA (128 B of each plane row)
constexpr int kTrStride = kTrGroups + 1;

// blocks -> planes, any multiple of 32 planes from col_lo.  in: rows x 16
// bytes.  out: nplanes rows of rows/8 bytes.
__global__ void __launch_bounds__(kTrThreads) tr_blocks_to_planes(
    const uint4 *__restrict__ in, uint64_t rows, int col_lo, int nplanes,
    uint32_t *__restrict__ out) {
  __shared__ uint32_t st[128 * kTrStride];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const TrLane tl = tr_lane(lane);
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
      const uint32_t col = warp_transpose32(w[q], tl);
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

// planes -> blocks.  in: nrows (<= 128, multiple of 32) rows of in_row_words
// 32-bit words, of which the first ncols bits are read.  out: ncols rows of
// nrows/8 bytes.
__global__ void __launch_bounds__(kTrThreads) tr_planes_to_blocks(
    const uint32_t *__restrict__ in, int nrows, uint64_t ncols, uint64_t in_row_words,
    uint32_t *__restrict__ out) {
  __shared__ uint32_t st[128 * kTrStride];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const TrLane tl = tr_lane(lane);
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
      if (q < nq) w[q] = warp_transpose32(st[(q * 32 + lane) * kTrStride + gg], tl);
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

static bool aligned(const void *p, uintptr_t a) { return reinterpret_cast<uintptr_t>(p) % a == 0; }

int transpose_launch(const void *in, uint64_t rows, uint64_t row_bytes, uint64_t col_lo,
                     uint64_t col_hi, void *out, cudaStream_t st) {
  const uint64_t ncols = col_hi - col_lo;
  if (row_bytes == 16 && rows % 128 == 0 && col_lo == 0 && ncols == 128 && aligned(in, 16) && aligned(out, 16)) {
    const uint64_t grid = (rows / 32 + kTrG - 1) / kTrG;
    if (grid > 0x7fffffffull) return fail(CUOT_EINVAL, "too many rows");
    tr_blocks_to_planes128<<<unsigned(grid), kTrThreads, 0, st>>>(static_cast<const uint4 *>(in), rows,
                                                                   static_cast<uint4 *>(out));
    return launch_status();
  }
  if (rows == 128 && col_lo == 0 && ncols % 128 == 0 && ncols <= row_bytes * 8 && row_bytes % 16 == 0 &&
      aligned(in, 16) && aligned(out, 16)) {
    const uint64_t grid = (ncols / 32 + kTrG - 1) / kTrG;
    if (grid > 0x7fffffffull) return fail(CUOT_EINVAL, "too many columns");
    tr_planes128_to_blocks<<<unsigned(grid), kTrThreads, 0, st>>>(static_cast<const uint4 *>(in), ncols,
                                                                   row_bytes / 16, static_cast<uint4 *>(out));
    return launch_status();
  }
  if (row_bytes == 16 && rows % 32 == 0 && col_lo % 32 == 0 && ncols % 32 == 0 && ncols > 0 &&
      aligned(in, 16) && aligned(out, 4)) {
    const uint64_t ngroups = rows / 32;
    const uint64_t grid = (ngroups + kTrGroups - 1) / kTrGroups;
    if (grid > 0x7fffffffull) return fail(CUOT_EINVAL, "too many rows");
    tr_blocks_to_planes<<<unsigned(grid), kTrThreads, 0, st>>>(
        static_cast<const uint4 *>(in), rows, int(col_lo), int(ncols),
        static_cast<uint32_t *>(out));
    return launch_status();
  }
  if (rows % 32 == 0 && rows <= 128 && col_lo == 0 && ncols <= row_bytes * 8 && ncols % 32 == 0 &&
      (row_bytes % 4) == 0 && aligned(in, 4) && aligned(out, rows == 128 ? 16 : 4)) {
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
  if (!ctx || ((!in_d || !out_d) && rows > 0)) return fail(CUOT_EINVAL, "null argument");
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
