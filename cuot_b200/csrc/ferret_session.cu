// ferret_session.cu -- FerretCOT's set-up instance and rcot buffer loop
// (ferret_cot.hpp:99-210) with device-resident state, both parties on one
// GPU and an ideal transport between them.
//
// One extension (ferret_cot.hpp:83-97) consumes M = k + t*h + 128 pre-COTs
// P of each role: P[0, t*h) feed the MPCOT's OTs -- the receiver's choice bit
// of OT i is LSB(P_recv[i]) and it receives the level sum that bit selects
// (OTPre over the pre-COTs, preot.h:26-82) -- and the LPN input is
// P[128, 128 + k) (lpn->compute(..., ot_input + consist_check_cot_num)).
// Its n outputs are ot_limit = n - M usable COTs followed by the M pre-COTs
// of the next extension (ferret_cot.hpp:102).  Set-up runs one extension of
// the pre-parameters on dealer base COTs (ferret_cot.hpp:150-170).
//
// Randomness: scalar i of the session is block i of the AES-CTR stream of the
// session seed (the cryptoTools PRNG, as cuot_prg_fill): block 0 = delta
// (LSB set), blocks 1, 2 = seeds of the dealer's base-COT v and choice
// streams, blocks 16 + 2e and 17 + 2e = the LPN seed and the roots seed of
// extension e (e = 0 is the set-up).
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "ctx.cuh"

namespace cuot {
namespace {

constexpr int64_t kConsistCheckCots = 128;  // mpcot_reg.h:44

// choice[i] = LSB(pre_r[i]); mc[i] = choice[i] ? rsum[i] : lsum[i]
__global__ void session_ot_kernel(const uint4 *__restrict__ pre_r, const uint4 *__restrict__ lsum,
                                  const uint4 *__restrict__ rsum, uint8_t *__restrict__ choice,
                                  uint4 *__restrict__ mc, int64_t m) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    const uint8_t c = uint8_t(pre_r[i].x & 1);
    choice[i] = c;
    mc[i] = c ? rsum[i] : lsum[i];
  }
}

// Dealer base COTs: v with its LSB cleared, w = v ^ x * delta (x = LSB of x_i)
__global__ void session_dealer_kernel(uint4 *__restrict__ v, const uint4 *__restrict__ x, uint4 *__restrict__ w,
                                      uint4 delta, int64_t m) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    uint4 a = v[i];
    a.x &= ~1u;
    v[i] = a;
    if (x[i].x & 1) {
      a.x ^= delta.x; a.y ^= delta.y; a.z ^= delta.z; a.w ^= delta.w;
    }
    w[i] = a;
  }
}

}  // namespace
}  // namespace cuot

using namespace cuot;

struct cuot_ferret_session {
  cuot_ctx *ctx;
  cuot_ferret_param p;
  int d;
  cudaStream_t st;
  AesKey key;                    // session seed's AES key (scalar derivation)
  cuot_block delta;
  cuot_block *ot_s, *ot_r;       // caller's n-block output buffers
  cuot_block *pre_s, *pre_r;     // M pre-COTs of each role
  cuot_block *roots, *lsum, *rsum, *mc, *ss, *tmp_n_s, *tmp_n_r;
  uint8_t *choice;
  int64_t extensions, ot_used, M, ot_limit;
};

namespace {

cuot_block scalar(const cuot_ferret_session *s, uint64_t i) {
  uint8_t ctr[16] = {0}, out[16];
  std::memcpy(ctr, &i, 8);
  host_aes_encrypt(s->key, ctr, out);
  cuot_block b;
  std::memcpy(&b, out, 16);
  return b;
}

int dalloc(void **p, size_t bytes) {
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ENOMEM, "ferret session: cudaMalloc of %zu bytes failed", bytes);
  }
  return CUOT_OK;
}

// One extension (ferret_cot.hpp:83-97): MPCOT of both roles over the OTs on
// mp_s / mp_r (t*h pre-COTs), LPN with kk_s / kk_r (k pre-COTs), into out_s / out_r.
int extend_once(cuot_ferret_session *s, int64_t t, int h, int64_t k, const cuot_block *mp_r, const cuot_block *kk_s,
                const cuot_block *kk_r, cuot_block *out_s, cuot_block *out_r) {
  const uint64_t e = uint64_t(s->extensions);
  const cuot_block lpn_seed = scalar(s, 16 + 2 * e), root_seed = scalar(s, 17 + 2 * e);
  CUOT_TRY(cuot_prg_fill(s->ctx, reinterpret_cast<const uint8_t *>(&root_seed), 0, s->roots, uint64_t(t), s->st));
  CUOT_TRY(cuot_ferret_pprf_sender(s->ctx, s->roots, uint64_t(t), h, &s->delta, out_s, s->lsum, s->rsum, s->ss,
                                   s->st));
  const int64_t m = t * h;
  session_ot_kernel<<<256, 256, 0, s->st>>>(reinterpret_cast<const uint4 *>(mp_r),
                                            reinterpret_cast<const uint4 *>(s->lsum),
                                            reinterpret_cast<const uint4 *>(s->rsum), s->choice,
                                            reinterpret_cast<uint4 *>(s->mc), m);
  CUOT_TRY(launch_status());
  CUOT_TRY(cuot_ferret_pprf_recver(s->ctx, s->mc, s->choice, s->ss, uint64_t(t), h, out_r, s->st));
  const uint8_t *ls = reinterpret_cast<const uint8_t *>(&lpn_seed);
  // both parties' LpnF2::compute with the seed ALICE sent BOB, in one launch
  CUOT_TRY(cuot_lpn_primal_dual(s->ctx, ls, kk_s, kk_r, k, s->d, out_s, out_r, t << h, s->st));
  s->extensions++;
  return CUOT_OK;
}

int copy_d2d(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "ferret session: copy failed");
  }
  return CUOT_OK;
}

}  // namespace

extern "C" {

int cuot_ferret_session_destroy(cuot_ferret_session *s) {
  if (!s) return CUOT_OK;
  DeviceGuard g(s->ctx);
  for (void *p : {(void *)s->pre_s, (void *)s->pre_r, (void *)s->roots, (void *)s->lsum, (void *)s->rsum,
                  (void *)s->mc, (void *)s->ss, (void *)s->choice, (void *)s->tmp_n_s, (void *)s->tmp_n_r})
    if (p) cudaFree(p);
  delete s;
  return CUOT_OK;
}

int cuot_ferret_session_create(cuot_ctx *ctx, const cuot_ferret_param *p, const uint8_t seed[16], int d,
                               cuot_block *ot_s_d, cuot_block *ot_r_d, void *stream, cuot_ferret_session **out) {
  if (!ctx || !p || !seed || !ot_s_d || !ot_r_d || !out) return fail(CUOT_EINVAL, "bad argument");
  if (p->t < 1 || p->log_bin_sz < 1 || p->log_bin_sz > 30 || p->n != (p->t << p->log_bin_sz) || p->t_pre < 1 ||
      p->log_bin_sz_pre < 1 || p->log_bin_sz_pre > 30 || p->n_pre != (p->t_pre << p->log_bin_sz_pre) || p->k < 1 ||
      p->k_pre < 1 || p->n_pre < p->k + p->t * p->log_bin_sz + kConsistCheckCots)
    return fail(CUOT_EINVAL, "LPN parameter not matched");  // constants.h:14-18
  if (d < 1 || d > 32) return fail(CUOT_EINVAL, "d=%d out of range", d);
  DeviceGuard g(ctx);
  cuot_ferret_session *s = new cuot_ferret_session();
  std::memset(s, 0, sizeof(*s));
  s->ctx = ctx;
  s->p = *p;
  s->d = d;
  s->st = static_cast<cudaStream_t>(stream);
  s->ot_s = ot_s_d;
  s->ot_r = ot_r_d;
  s->M = p->k + p->t * p->log_bin_sz + kConsistCheckCots;
  s->ot_limit = p->n - s->M;
  host_aes_key_expand(seed, &s->key);
  s->delta = scalar(s, 0);
  s->delta.w[0] |= 1;  // ferret_cot.hpp:27-31
  const int64_t tmax = p->t > p->t_pre ? p->t : p->t_pre;
  const int64_t thmax = std::max(p->t * p->log_bin_sz, p->t_pre * p->log_bin_sz_pre);
  int st = CUOT_OK;
  if ((st = dalloc((void **)&s->pre_s, s->M * 16)) || (st = dalloc((void **)&s->pre_r, s->M * 16)) ||
      (st = dalloc((void **)&s->roots, tmax * 16)) || (st = dalloc((void **)&s->lsum, thmax * 16)) ||
      (st = dalloc((void **)&s->rsum, thmax * 16)) || (st = dalloc((void **)&s->mc, thmax * 16)) ||
      (st = dalloc((void **)&s->ss, tmax * 16)) || (st = dalloc((void **)&s->choice, thmax)) ||
      (st = dalloc((void **)&s->tmp_n_s, p->n_pre * 16)) || (st = dalloc((void **)&s->tmp_n_r, p->n_pre * 16))) {
    cuot_ferret_session_destroy(s);
    return st;
  }
  // set-up: dealer base COTs -- t_pre*h_pre for the MPCOT, k_pre + 128 for the LPN
  const int64_t nb_mp = p->t_pre * p->log_bin_sz_pre, nb = nb_mp + p->k_pre + kConsistCheckCots;
  cuot_block *bv = nullptr, *bx = nullptr, *bw = nullptr;
  if ((st = dalloc((void **)&bv, nb * 16)) || (st = dalloc((void **)&bx, nb * 16)) ||
      (st = dalloc((void **)&bw, nb * 16))) {
    if (bv) cudaFree(bv);
    if (bx) cudaFree(bx);
    cuot_ferret_session_destroy(s);
    return st;
  }
  const cuot_block sv = scalar(s, 1), sx = scalar(s, 2);
  uint4 dl;
  std::memcpy(&dl, &s->delta, 16);
  if (!(st = cuot_prg_fill(ctx, reinterpret_cast<const uint8_t *>(&sv), 0, bv, nb, s->st)) &&
      !(st = cuot_prg_fill(ctx, reinterpret_cast<const uint8_t *>(&sx), 0, bx, nb, s->st))) {
    session_dealer_kernel<<<256, 256, 0, s->st>>>(reinterpret_cast<uint4 *>(bv), reinterpret_cast<const uint4 *>(bx),
                                                   reinterpret_cast<uint4 *>(bw), dl, nb);
    st = launch_status();
  }
  const int64_t c = kConsistCheckCots;
  if (!st)
    st = extend_once(s, p->t_pre, int(p->log_bin_sz_pre), p->k_pre, bw, bv + nb_mp + c, bw + nb_mp + c, s->tmp_n_s,
                     s->tmp_n_r);
  if (!st) st = copy_d2d(s->pre_s, s->tmp_n_s, s->M * 16, s->st);
  if (!st) st = copy_d2d(s->pre_r, s->tmp_n_r, s->M * 16, s->st);
  if (!st && cudaStreamSynchronize(s->st) != cudaSuccess) {
    cudaGetLastError();
    st = fail(CUOT_ECUDA, "ferret session set-up failed");
  }
  cudaFree(bv);
  cudaFree(bx);
  cudaFree(bw);
  if (st) {
    cuot_ferret_session_destroy(s);
    return st;
  }
  s->ot_used = s->ot_limit;
  *out = s;
  return CUOT_OK;
}

// extend_f2k (ferret_cot.hpp:99-106): one extension into the caller's output
// buffers; the last M outputs become the next pre-COTs.
int cuot_ferret_session_extend(cuot_ferret_session *s) {
  if (!s) return fail(CUOT_EINVAL, "null session");
  DeviceGuard g(s->ctx);
  const cuot_ferret_param &p = s->p;
  const int64_t c = kConsistCheckCots;
  CUOT_TRY(extend_once(s, p.t, int(p.log_bin_sz), p.k, s->pre_r, s->pre_s + c, s->pre_r + c, s->ot_s, s->ot_r));
  CUOT_TRY(copy_d2d(s->pre_s, s->ot_s + s->ot_limit, s->M * 16, s->st));
  CUOT_TRY(copy_d2d(s->pre_r, s->ot_r + s->ot_limit, s->M * 16, s->st));
  s->ot_used = 0;
  return CUOT_OK;
}

// rcot (ferret_cot.hpp:178-210): num COTs of each role into v_d / w_d.
int cuot_ferret_session_rcot(cuot_ferret_session *s, int64_t num, cuot_block *v_d, cuot_block *w_d) {
  if (!s || num < 0 || (num && (!v_d || !w_d))) return fail(CUOT_EINVAL, "bad argument");
  DeviceGuard g(s->ctx);
  int64_t done = 0;
  while (done < num) {
    if (s->ot_used == s->ot_limit) CUOT_TRY(cuot_ferret_session_extend(s));
    const int64_t take = std::min(num - done, s->ot_limit - s->ot_used);
    CUOT_TRY(copy_d2d(v_d + done, s->ot_s + s->ot_used, take * 16, s->st));
    CUOT_TRY(copy_d2d(w_d + done, s->ot_r + s->ot_used, take * 16, s->st));
    s->ot_used += take;
    done += take;
  }
  return CUOT_OK;
}

int cuot_ferret_session_info(const cuot_ferret_session *s, cuot_ferret_session_state *out) {
  if (!s || !out) return fail(CUOT_EINVAL, "bad argument");
  out->M = s->M;
  out->ot_limit = s->ot_limit;
  out->ot_used = s->ot_used;
  out->extensions = s->extensions;
  out->delta = s->delta;
  return CUOT_OK;
}

}  // extern "C"
