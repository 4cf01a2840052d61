// lpn.cu -- Ferret primal LPN and plain AES-128 ECB.
//
// LPN: e[i] ^= XOR_{j<d} kk[idx(i, j)] with emp-ot's index matrix
// (lpn_f2.h:46-79, one task over [0, n)):
//   rows i..i+3 (i % 4 == 0, i < tail): the d blocks makeBlock(i, m), m < d,
//     are AES-encrypted under the seed key; their 4d little-endian u32 words
//     give row i + q/d, term q%d: idx = w & mask, minus k if >= k.
//   rows j >= tail (tail = first multiple of 4 >= n-4): ceil(d/4) blocks
//     makeBlock(j, m), idx = w % k.
// The index AES runs in the same kernel as the gather, so the n*d index
// matrix never touches HBM (cuOT materialises it, dev_layer.cu:171-173).
// kk (k blocks) is read through the read-only path and stays L2-resident.
#include "lpn_kernel.cuh"

namespace cuot {

// D = 0: any d (a.d); D > 0: d = D.  DUAL: both roles (a.kk2 / a.e2 set).
template <int D, bool DUAL>
__global__ void __launch_bounds__(kLpnThreads) lpn_kernel(LpnArgs a) {
  extern __shared__ __align__(16) uint32_t smem_tab[];
  stage_table(smem_tab, a.t0);
  __syncthreads();
  const TabRef T{reinterpret_cast<const char *>(smem_tab), uint32_t(threadIdx.x & 31) * 4u};
  const int64_t total = a.ngroups + a.ntail;
  for (int64_t w = int64_t(blockIdx.x) * kLpnThreads + threadIdx.x; w < total;
       w += int64_t(gridDim.x) * kLpnThreads) {
    if (w < a.ngroups) {
      if (D > 0) lpn_group4<(D > 0 ? D : 1), DUAL>(a, T, a.g0 + w);
      else lpn_group4_dyn(a, T, a.g0 + w);
    } else {
      lpn_row1(a, T, a.j0 + (w - a.ngroups));
    }
  }
}

// Plain in-place AES-128 ECB, two blocks per thread.
__global__ void __launch_bounds__(kLpnThreads) ecb_kernel(AesKey key, const uint32_t *t0,
                                                          Blk *io, uint64_t n) {
  extern __shared__ __align__(16) uint32_t smem_tab[];
  stage_table(smem_tab, t0);
  __syncthreads();
  const TabRef T{reinterpret_cast<const char *>(smem_tab), uint32_t(threadIdx.x & 31) * 4u};
  const uint64_t half = (n + 1) / 2;
  for (uint64_t i = uint64_t(blockIdx.x) * kLpnThreads + threadIdx.x; i < half;
       i += uint64_t(gridDim.x) * kLpnThreads) {
    const uint64_t j = i + half;  // second block, keeps both accesses coalesced
    Blk p = ld_blk(io + i);
    uint32_t x[4] = {p.w[0], p.w[1], p.w[2], p.w[3]};
    if (j < n) {
      Blk q = ld_blk(io + j);
      uint32_t y[4] = {q.w[0], q.w[1], q.w[2], q.w[3]};
      aes_enc2(T, x, key, y, key);
      st_blk(io + j, Blk{{y[0], y[1], y[2], y[3]}});
    } else {
      aes_enc(T, x, key);
    }
    st_blk(io + i, Blk{{x[0], x[1], x[2], x[3]}});
  }
}

static int grid_for(cuot_ctx *ctx, const void *fn, int64_t work, int *grid) {
  int per_sm = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kLpnThreads, kTableBytes);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  if (per_sm < 1) per_sm = 1;
  int64_t need = (work + kLpnThreads - 1) / kLpnThreads;
  int64_t cap = int64_t(per_sm) * sms * 8;
  *grid = int(need < cap ? (need > 0 ? need : 1) : cap);
  return CUOT_OK;
}

template <typename F>
static int set_smem(F fn) {
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kTableBytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "cudaFuncSetAttribute failed: %s", cudaGetErrorString(e));
  }
  return CUOT_OK;
}

template <int D, bool DUAL>
int launch_lpn(cuot_ctx *ctx, const LpnArgs &a, cudaStream_t st) {
  CUOT_TRY(set_smem(lpn_kernel<D, DUAL>));
  int grid = 1;
  grid_for(ctx, (const void *)lpn_kernel<D, DUAL>, a.ngroups + a.ntail, &grid);
  lpn_kernel<D, DUAL><<<grid, kLpnThreads, kTableBytes, st>>>(a);
  return launch_status();
}

// Rows [row_lo, row_hi) of one task over [0, n) (lpn_f2.h:72-79), for one
// role (kk2 == e2 == nullptr) or for both roles of one extension.
int lpn_rows(cuot_ctx *ctx, const uint8_t seed[16], const cuot_block *kk_d, const cuot_block *kk2_d,
             int64_t k, int d, cuot_block *e_rows_d, cuot_block *e2_rows_d, int64_t row_lo, int64_t row_hi,
             int64_t n, void *stream) {
  if (k < 1 || k > 0x7fffffffll) return fail(CUOT_EINVAL, "k=%lld out of range", (long long)k);
  if (d < 1 || d > 32) return fail(CUOT_EINVAL, "d=%d out of range [1,32]", d);
  if (n < 0 || row_lo < 0 || row_hi < row_lo || row_hi > n)
    return fail(CUOT_EINVAL, "bad row range [%lld,%lld) of n=%lld", (long long)row_lo,
                (long long)row_hi, (long long)n);
  if (row_lo % 4 || (row_hi % 4 && row_hi != n))
    return fail(CUOT_EINVAL, "row range must start at a multiple of 4 and end at one or at n");
  if (row_hi == row_lo) return CUOT_OK;
  DeviceGuard g(ctx);
  LpnArgs a{};
  host_aes_key_expand(seed, &a.key);
  a.t0 = ctx->t0_d;
  a.kk = reinterpret_cast<const Blk *>(kk_d);
  a.e = reinterpret_cast<Blk *>(e_rows_d);
  a.kk2 = reinterpret_cast<const Blk *>(kk2_d);
  a.e2 = reinterpret_cast<Blk *>(e2_rows_d);
  a.n = n; a.k = k; a.d = d; a.row_lo = row_lo;
  uint32_t mask = 1;
  while (int64_t(mask) < k) mask = (mask << 1) | 1u;  // lpn_f2.h:27-31
  a.mask = mask;
  int64_t tail = 0;
  if (n > 4) tail = ((n - 4) + 3) / 4 * 4;  // lpn_f2.h:75: groups while j < n - 4
  a.tail = tail;
  const int64_t gend = (row_hi < tail ? row_hi : tail);
  a.g0 = row_lo / 4;
  a.ngroups = gend > row_lo ? (gend - row_lo) / 4 : 0;
  a.j0 = row_lo > tail ? row_lo : tail;
  a.ntail = row_hi > a.j0 ? row_hi - a.j0 : 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool dual = kk2_d != nullptr;
  if (d == 10) return dual ? launch_lpn<10, true>(ctx, a, st) : launch_lpn<10, false>(ctx, a, st);
  return launch_lpn<0, false>(ctx, a, st);  // lpn_group4_dyn / lpn_row1 read a.kk2 themselves
}

}  // namespace cuot

using namespace cuot;

extern "C" {

int cuot_lpn_primal_dual(cuot_ctx *ctx, const uint8_t seed[16], const cuot_block *kk_send_d,
                         const cuot_block *kk_recv_d, int64_t k, int d, cuot_block *e_send_io_d,
                         cuot_block *e_recv_io_d, int64_t n, void *stream) {
  if (!ctx || !seed || ((!kk_send_d || !kk_recv_d || !e_send_io_d || !e_recv_io_d) && n > 0))
    return fail(CUOT_EINVAL, "null argument");
  if (n > 0 && e_send_io_d == e_recv_io_d) return fail(CUOT_EINVAL, "the two roles' rows must not alias");
  return lpn_rows(ctx, seed, kk_send_d, kk_recv_d, k, d, e_send_io_d, e_recv_io_d, 0, n, n, stream);
}

int cuot_lpn_primal_range(cuot_ctx *ctx, const uint8_t seed[16], const cuot_block *kk_d,
                          int64_t k, int d, cuot_block *e_rows_d, int64_t row_lo, int64_t row_hi,
                          int64_t n, void *stream) {
  if (!ctx || !seed || ((!kk_d || !e_rows_d) && row_hi > row_lo)) return fail(CUOT_EINVAL, "null argument");
  return lpn_rows(ctx, seed, kk_d, nullptr, k, d, e_rows_d, nullptr, row_lo, row_hi, n, stream);
}

int cuot_lpn_primal(cuot_ctx *ctx, const uint8_t seed[16], const cuot_block *kk_d,
                    int64_t k, int d, cuot_block *e_io_d, int64_t n, void *stream) {
  return cuot_lpn_primal_range(ctx, seed, kk_d, k, d, e_io_d, 0, n, n, stream);
}

int cuot_aes128_ecb(cuot_ctx *ctx, const uint8_t key[16], cuot_block *io_d,
                    uint64_t nblocks, void *stream) {
  if (!ctx || !key || (!io_d && nblocks)) return fail(CUOT_EINVAL, "null argument");
  if (nblocks == 0) return CUOT_OK;
  DeviceGuard g(ctx);
  AesKey k;
  host_aes_key_expand(key, &k);
  CUOT_TRY(set_smem(ecb_kernel));
  int grid = 1;
  grid_for(ctx, (const void *)ecb_kernel, int64_t((nblocks + 1) / 2), &grid);
  ecb_kernel<<<grid, kLpnThreads, kTableBytes, static_cast<cudaStream_t>(stream)>>>(
      k, ctx->t0_d, reinterpret_cast<Blk *>(io_d), nblocks);
  return launch_status();
}

}  // extern "C"
