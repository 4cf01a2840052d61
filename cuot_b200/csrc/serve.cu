// serve.cu -- continuous batching of OT-extension requests on one GPU.
//
// A request is one OT extension (Ferret-style: MPCOT + primal LPN, or SOT:
// PPRF + exact QC encode + choice-bit encode) with both roles.  The server
// keeps `slots` executors busy -- each a libcuot context and two CUDA streams
// (normal and high priority) -- admitting queued requests in arrival order as
// soon as a slot is free and the request's device footprint fits the HBM
// budget, so requests overlap on the GPU.  Optional scheduling knobs: at most
// `max_big` requests with n >= big_n in flight (one already fills the GPU;
// smaller requests may pass a big one waiting for that reason; memory stays
// head-of-line) and small requests (n < high_priority_below_n) on the slot's
// high-priority stream.  Host-side failure handling: queue timeouts,
// cancellation (before or during run), rejection of requests that can never
// fit.  Completion is polled with event queries; nothing waits on the device.
//
// A request's inputs are derived on the device from its seed (the cryptoTools
// PRNG stream): roots [0, t), ceil(t*h/16) blocks whose bytes' LSBs are the
// choice bits, then kk_s, kk_r (Ferret) or base0, base1 (SOT).  Its scalars
// are blocks 2^40 + {0, 1, 2} of the same stream: delta (LSB set), the LPN
// seed, the QC key.  Device buffers are stream-ordered allocations, freed in
// stream order after the request's last kernel and host copies.
//
// With dry_run_service_s > 0 there is no GPU work: each request "runs" for
// that long (host-only tests of the scheduling logic).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "common.cuh"
#include "ctx.cuh"

namespace cuot {
namespace {

__global__ void serve_choice_kernel(const uint8_t *__restrict__ raw, uint8_t *__restrict__ choice, int64_t m) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x)
    choice[i] = raw[i] & 1;
}
// out[i] = choice[i] ? b1[i] : b0[i]
__global__ void serve_select_kernel(const uint8_t *__restrict__ choice, const uint4 *__restrict__ b0,
                                    const uint4 *__restrict__ b1, uint4 *__restrict__ out, int64_t m) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = choice[i] ? b1[i] : b0[i];
}
// punctured leaf of each SOT tree from its [h][t] choice bits (silent/recver.cu:77-86)
__global__ void serve_pos_kernel(const uint8_t *__restrict__ choice, uint64_t t, int h, uint64_t *__restrict__ pos) {
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < t; j += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t id = 0;
    for (int d = 0; d < h; d++) id = 2 * id + (1 - choice[uint64_t(d) * t + j]);
    pos[j] = id + (j << h);
  }
}

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

uint64_t req_n(const cuot_request &r) { return r.t << r.h; }

// Device bytes one request holds while admitted (inputs, both roles' outputs
// and per-request intermediates); the slots' scratch is reserved apart.
uint64_t footprint(const cuot_request &r) {
  const uint64_t n = req_n(r), t = r.t, h = uint64_t(r.h);
  uint64_t b = 2 * 16 * n + 16 * t + t * h;
  if (r.kind == CUOT_KIND_FERRET)
    b += 2 * 16 * uint64_t(r.k) + 4 * 16 * t * h + 16 * t;
  else
    b += 3 * 16 * h * t + 2 * 16 * (h + 1) * t + n / 8 + n / 8 + 8 * t;
  return b;
}

// Shapes the server runs: h in [1, 20]; SOT n a power of two in [2^10,
// 2^max_log_n]; Ferret n <= 2^max_log_n and 0 < k <= n.
bool valid(const cuot_request &r, int max_log_n) {
  if (r.t < 1 || r.h < 1 || r.h > 20 || r.t > (1ull << 40)) return false;
  const uint64_t n = req_n(r);
  if (n > (1ull << max_log_n)) return false;
  if (r.kind == CUOT_KIND_SOT) return (r.t & (r.t - 1)) == 0 && n >= 1024;
  if (r.kind == CUOT_KIND_FERRET) return r.k > 0 && uint64_t(r.k) <= n;
  return false;
}

struct Slot {
  cuot_ctx *ctx = nullptr;
  cudaStream_t lo = nullptr, hi = nullptr, cur = nullptr;
  cudaEvent_t done = nullptr;
  double dry_end = 0;
};

}  // namespace
}  // namespace cuot

using namespace cuot;

struct cuot_server {
  cuot_server_config cfg;
  int device = 0;
  std::vector<Slot> slots;
  uint64_t reserved = 0;
  std::mutex mu;
  std::set<int> cancelled;
  uint64_t max_used = 0;
};

namespace {

int cuda_fail(cudaError_t e, const char *what) {
  cudaGetLastError();
  return fail(CUOT_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}
#define SV_CUDA(call, what)                       \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

// Scalars of a request: blocks 2^40 + {0, 1, 2} of its seed's AES-CTR stream
// (delta with its LSB set, as Ferret's Delta, ferret_cot.hpp:29-31; the LPN
// seed; the key of the QC polynomial).
void request_scalars(const uint8_t seed[16], cuot_block out[3]) {
  AesKey key;
  host_aes_key_expand(seed, &key);
  for (uint64_t j = 0; j < 3; j++) {
    uint8_t ctr[16] = {0}, blk[16];
    const uint64_t i = (1ull << 40) + j;
    std::memcpy(ctr, &i, 8);
    host_aes_encrypt(key, ctr, blk);
    std::memcpy(&out[j], blk, 16);
  }
  out[0].w[0] |= 1;
}

// Enqueues request r on stream st (no host synchronisation); every device
// buffer it allocates is appended to `bufs`.
int enqueue_request(Slot &s, cudaStream_t st, const cuot_request &r, std::vector<void *> &bufs) {
  const uint64_t n = req_n(r), t = r.t, th = r.t * uint64_t(r.h);
  const int h = r.h;
  auto alloc = [&](void **p, size_t bytes) -> int {
    SV_CUDA(cudaMallocAsync(p, bytes ? bytes : 16, st), "cudaMallocAsync");
    bufs.push_back(*p);
    return CUOT_OK;
  };
  cuot_block sc[3];
  request_scalars(r.seed, sc);
  const cuot_block delta = sc[0], lpn_seed = sc[1], akey = sc[2];
  // inputs from the seed's stream
  uint64_t off = 0;
  cuot_block *roots, *raw, *v, *w;
  uint8_t *choice;
  CUOT_TRY(alloc((void **)&roots, 16 * t));
  CUOT_TRY(alloc((void **)&raw, 16 * ((th + 15) / 16)));
  CUOT_TRY(alloc((void **)&choice, th));
  CUOT_TRY(alloc((void **)&v, 16 * n));
  CUOT_TRY(alloc((void **)&w, 16 * n));
  auto take = [&](cuot_block *dst, uint64_t m) {
    const int rc = cuot_prg_fill(s.ctx, r.seed, off, dst, m, st);
    off += m;
    return rc;
  };
  CUOT_TRY(take(roots, t));
  CUOT_TRY(take(raw, (th + 15) / 16));
  serve_choice_kernel<<<64, 256, 0, st>>>(reinterpret_cast<const uint8_t *>(raw), choice, int64_t(th));
  CUOT_TRY(launch_status());
  uint64_t *cb = nullptr;
  if (r.kind == CUOT_KIND_FERRET) {
    cuot_block *kk_s, *kk_r, *lsum, *rsum, *ss, *mc;
    CUOT_TRY(alloc((void **)&kk_s, 16 * uint64_t(r.k)));
    CUOT_TRY(alloc((void **)&kk_r, 16 * uint64_t(r.k)));
    CUOT_TRY(alloc((void **)&lsum, 16 * th));
    CUOT_TRY(alloc((void **)&rsum, 16 * th));
    CUOT_TRY(alloc((void **)&mc, 16 * th));
    CUOT_TRY(alloc((void **)&ss, 16 * t));
    CUOT_TRY(take(kk_s, uint64_t(r.k)));
    CUOT_TRY(take(kk_r, uint64_t(r.k)));
    CUOT_TRY(cuot_ferret_pprf_sender(s.ctx, roots, t, h, &delta, v, lsum, rsum, ss, st));
    serve_select_kernel<<<64, 256, 0, st>>>(choice, reinterpret_cast<const uint4 *>(lsum),
                                            reinterpret_cast<const uint4 *>(rsum), reinterpret_cast<uint4 *>(mc),
                                            int64_t(th));
    CUOT_TRY(launch_status());
    CUOT_TRY(cuot_ferret_pprf_recver(s.ctx, mc, choice, ss, t, h, w, st));
    const uint8_t *ls = reinterpret_cast<const uint8_t *>(&lpn_seed);
    // both roles' LPN in one launch: they share the request's public seed
    CUOT_TRY(cuot_lpn_primal_dual(s.ctx, ls, kk_s, kk_r, r.k, 10, v, w, int64_t(n), st));
  } else {
    cuot_block *b0, *b1, *m0, *m1, *mc;
    uint64_t *a, *pos;
    CUOT_TRY(alloc((void **)&b0, 16 * th));
    CUOT_TRY(alloc((void **)&b1, 16 * th));
    CUOT_TRY(alloc((void **)&mc, 16 * th));
    CUOT_TRY(alloc((void **)&m0, 16 * (th + t)));
    CUOT_TRY(alloc((void **)&m1, 16 * (th + t)));
    CUOT_TRY(alloc((void **)&a, n / 8));
    CUOT_TRY(alloc((void **)&pos, 8 * t));
    CUOT_TRY(alloc((void **)&cb, n / 8));
    CUOT_TRY(take(b0, th));
    CUOT_TRY(take(b1, th));
    serve_select_kernel<<<64, 256, 0, st>>>(choice, reinterpret_cast<const uint4 *>(b0),
                                            reinterpret_cast<const uint4 *>(b1), reinterpret_cast<uint4 *>(mc),
                                            int64_t(th));
    CUOT_TRY(launch_status());
    CUOT_TRY(cuot_sot_pprf_sender(s.ctx, roots, t, h, &delta, b0, b1, v, m0, m1, st));
    CUOT_TRY(cuot_sot_pprf_recver(s.ctx, m0, m1, mc, choice, t, h, w, st));
    CUOT_TRY(cuot_qc_gen_a(s.ctx, reinterpret_cast<const uint8_t *>(&akey), n, a, st));
    CUOT_TRY(cuot_sot_dual_lpn(s.ctx, a, v, n, st));
    CUOT_TRY(cuot_sot_dual_lpn(s.ctx, a, w, n, st));
    serve_pos_kernel<<<16, 256, 0, st>>>(choice, t, h, pos);
    CUOT_TRY(launch_status());
    CUOT_TRY(cuot_qc_encode_sparse(s.ctx, a, pos, int(t), n, cb, st));
  }
  if (r.v_h) SV_CUDA(cudaMemcpyAsync(r.v_h, v, 16 * n, cudaMemcpyDeviceToHost, st), "D2H v");
  if (r.w_h) SV_CUDA(cudaMemcpyAsync(r.w_h, w, 16 * n, cudaMemcpyDeviceToHost, st), "D2H w");
  if (r.c_h && cb) SV_CUDA(cudaMemcpyAsync(r.c_h, cb, n / 8, cudaMemcpyDeviceToHost, st), "D2H c");
  return CUOT_OK;
}

// Starts request r on slot s: its work, then the stream-ordered frees of its
// buffers (also after a failed enqueue) and the slot's completion event.
int start_request(const cuot_server_config &cfg, Slot &s, const cuot_request &r) {
  const bool hi = cfg.high_priority_below_n && req_n(r) < cfg.high_priority_below_n;
  cudaStream_t st = hi ? s.hi : s.lo;
  s.cur = st;
  std::vector<void *> bufs;
  const int rc = enqueue_request(s, st, r, bufs);
  for (void *p : bufs) cudaFreeAsync(p, st);
  if (rc) return rc;
  SV_CUDA(cudaEventRecord(s.done, st), "cudaEventRecord");
  return CUOT_OK;
}

}  // namespace

extern "C" {

int cuot_server_destroy(cuot_server *sv) {
  if (!sv) return CUOT_OK;
  for (auto &s : sv->slots) {
    if (s.done) cudaEventDestroy(s.done);
    if (s.lo) cudaStreamDestroy(s.lo);
    if (s.hi) cudaStreamDestroy(s.hi);
    if (s.ctx) cuot_ctx_destroy(s.ctx);
  }
  delete sv;
  return CUOT_OK;
}

int cuot_server_create(int device, const cuot_server_config *cfg, cuot_server **out) {
  if (!cfg || !out || cfg->slots < 1 || cfg->slots > 256) return fail(CUOT_EINVAL, "bad argument");
  if (cfg->max_log_n && (cfg->max_log_n < 10 || cfg->max_log_n > 25))
    return fail(CUOT_EINVAL, "max_log_n %d outside [10, 25]", cfg->max_log_n);
  *out = nullptr;
  cuot_server *sv = new cuot_server();
  sv->cfg = *cfg;
  sv->device = device;
  sv->slots.resize(cfg->slots);
  if (cfg->dry_run_service_s > 0) {
    *out = sv;
    return CUOT_OK;
  }
  const int max_log_n = cfg->max_log_n > 0 ? cfg->max_log_n : 24;
  const uint64_t nmax = 1ull << max_log_n;
  // per slot: PPRF levels (16n) or the one-shot dual LPN of any size up to
  // nmax (transform of `a`, blocks or tile words, pass intermediate; the
  // library's own sizing), plus the QC twiddle tables of every size
  uint64_t scratch = 24 * nmax + std::max<uint64_t>(4 * nmax, 512ull << 20) + (64ull << 20);
  uint64_t tables = 0;
  for (int e = 10; e <= max_log_n; e++) tables += 16 * (1ull << e) + 32 * (1ull << (e / 2 + 1));
  int lo_prio = 0, hi_prio = 0;
  cudaSetDevice(device);
  cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
  // keep freed request buffers in the pool between requests
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  int st = CUOT_OK;
  for (auto &s : sv->slots) {
    if ((st = cuot_ctx_create(device, &s.ctx))) break;
    // the slots already overlap their requests: one stream per FFT encode
    if ((st = cuot_ctx_set_tuning(s.ctx, CUOT_TUNE_QC_STREAMS, 1))) break;
    for (int e = 10; e <= max_log_n; e++) scratch = std::max(scratch, qc_one_shot_dual_bytes(s.ctx, e, false));
    if ((st = cuot_ctx_reserve(s.ctx, scratch))) break;
    if (cudaStreamCreateWithPriority(&s.lo, cudaStreamNonBlocking, lo_prio) != cudaSuccess ||
        cudaStreamCreateWithPriority(&s.hi, cudaStreamNonBlocking, hi_prio) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) {
      st = cuda_fail(cudaGetLastError(), "stream/event creation");
      break;
    }
    // build the QC tables of every size now (the first use of a size synchronises)
    for (int e = 10; e <= max_log_n && !st; e++) {
      const uint64_t n = 1ull << e;
      void *a = nullptr, *pl = nullptr;
      if (cudaMalloc(&a, n / 8) != cudaSuccess || cudaMalloc(&pl, n / 8) != cudaSuccess) {
        if (a) cudaFree(a);
        st = cuda_fail(cudaGetLastError(), "QC warm-up allocation");
        break;
      }
      cudaMemset(a, 0, n / 8);
      cudaMemset(pl, 0, n / 8);
      st = cuot_qc_encode(s.ctx, static_cast<uint64_t *>(a), static_cast<uint64_t *>(pl), n, 1, s.lo);
      cudaStreamSynchronize(s.lo);
      cudaFree(a);
      cudaFree(pl);
    }
    if (st) break;
  }
  if (st) {
    cuot_server_destroy(sv);
    return st;
  }
  sv->reserved = uint64_t(cfg->slots) * (scratch + tables);
  *out = sv;
  return CUOT_OK;
}

int cuot_request_scalars(const uint8_t seed[16], cuot_block out[3]) {
  if (!seed || !out) return fail(CUOT_EINVAL, "null argument");
  request_scalars(seed, out);
  return CUOT_OK;
}

int cuot_request_footprint(const cuot_request *r, uint64_t *out) {
  if (!r || !out) return fail(CUOT_EINVAL, "null argument");
  *out = footprint(*r);
  return CUOT_OK;
}

int cuot_server_reserved_bytes(const cuot_server *sv, uint64_t *out) {
  if (!sv || !out) return fail(CUOT_EINVAL, "bad argument");
  *out = sv->reserved;
  return CUOT_OK;
}

int cuot_server_configure(cuot_server *sv, const cuot_server_config *cfg) {
  if (!sv || !cfg) return fail(CUOT_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->cfg.budget_bytes = cfg->budget_bytes;
  sv->cfg.max_queue_wait = cfg->max_queue_wait;
  sv->cfg.big_n = cfg->big_n;
  sv->cfg.max_big = cfg->max_big;
  sv->cfg.high_priority_below_n = cfg->high_priority_below_n;
  return CUOT_OK;
}

int cuot_server_cancel(cuot_server *sv, int index) {
  if (!sv) return fail(CUOT_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->cancelled.insert(index);
  return CUOT_OK;
}

int cuot_server_run(cuot_server *sv, cuot_request *reqs, int count, cuot_server_stats *stats) {
  if (!sv || (count > 0 && !reqs) || count < 0) return fail(CUOT_EINVAL, "bad argument");
  // cuot_server_configure may change the scheduling fields from another
  // thread while this loop runs: every iteration works on a copy taken under
  // the server's mutex.
  cuot_server_config cfg;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    cfg = sv->cfg;
  }
  const bool dry = cfg.dry_run_service_s > 0;
  if (!dry) cudaSetDevice(sv->device);
  const int max_log_n = cfg.max_log_n > 0 ? cfg.max_log_n : 24;
  std::vector<int> order(count);
  for (int i = 0; i < count; i++) {
    order[i] = i;
    reqs[i].status = CUOT_REQ_PENDING;
    reqs[i].t_admit = reqs[i].t_done = -1;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].arrival < reqs[b].arrival; });
  std::deque<int> queue;
  std::vector<int> free_slots;
  for (int s = int(sv->slots.size()) - 1; s >= 0; s--) free_slots.push_back(s);
  std::vector<int> busy(sv->slots.size(), -1);
  double used = 0, max_used = 0;
  int nbusy = 0;
  size_t next = 0;
  const double t0 = now_s();
  auto is_big = [&](const cuot_request &r) { return cfg.big_n && req_n(r) >= cfg.big_n; };
  int rc = CUOT_OK;
  while (next < order.size() || !queue.empty() || nbusy) {
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      cfg = sv->cfg;
    }
    const double budget = cfg.budget_bytes - double(sv->reserved);
    const double now = now_s() - t0;
    while (next < order.size() && reqs[order[next]].arrival <= now) {
      const int i = order[next++];
      if (!valid(reqs[i], max_log_n) || double(footprint(reqs[i])) > budget) {
        reqs[i].status = CUOT_REQ_REJECTED;
        continue;
      }
      reqs[i].status = CUOT_REQ_QUEUED;
      queue.push_back(i);
    }
    // completions
    for (size_t s = 0; s < sv->slots.size(); s++) {
      if (busy[s] < 0) continue;
      bool fin;
      if (dry) {
        fin = now_s() >= sv->slots[s].dry_end;
      } else {
        const cudaError_t e = cudaEventQuery(sv->slots[s].done);
        if (e != cudaSuccess && e != cudaErrorNotReady) {
          rc = cuda_fail(e, "request failed");
          fin = true;
        } else {
          fin = (e == cudaSuccess);
        }
      }
      if (!fin) continue;
      cuot_request &r = reqs[busy[s]];
      r.t_done = now_s() - t0;
      r.status = rc ? CUOT_REQ_FAILED : CUOT_REQ_DONE;
      used -= double(footprint(r));
      busy[s] = -1;
      nbusy--;
      free_slots.push_back(int(s));
    }
    if (rc) break;
    // cancellations and queue timeouts
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      if (!sv->cancelled.empty() || cfg.max_queue_wait > 0) {
        std::deque<int> keep;
        for (int i : queue) {
          if (sv->cancelled.count(i)) reqs[i].status = CUOT_REQ_CANCELLED;
          else if (cfg.max_queue_wait > 0 && now - reqs[i].arrival > cfg.max_queue_wait)
            reqs[i].status = CUOT_REQ_TIMEOUT;
          else keep.push_back(i);
        }
        queue.swap(keep);
      }
    }
    // admission
    while (!queue.empty() && !free_slots.empty()) {
      int nbig = 0;
      for (size_t s = 0; s < sv->slots.size(); s++)
        if (busy[s] >= 0 && is_big(reqs[busy[s]])) nbig++;
      int pick = -1;
      for (size_t j = 0; j < queue.size(); j++) {
        const cuot_request &r = reqs[queue[j]];
        if (used + double(footprint(r)) > budget) break;  // memory is head-of-line
        if (is_big(r) && nbig >= std::max(1, cfg.max_big)) continue;
        pick = int(j);
        break;
      }
      if (pick < 0) break;
      const int i = queue[pick];
      queue.erase(queue.begin() + pick);
      const int s = free_slots.back();
      free_slots.pop_back();
      used += double(footprint(reqs[i]));
      max_used = std::max(max_used, used);
      reqs[i].t_admit = now_s() - t0;
      reqs[i].status = CUOT_REQ_RUNNING;
      busy[s] = i;
      nbusy++;
      if (dry) {
        sv->slots[s].dry_end = now_s() + cfg.dry_run_service_s;
      } else if ((rc = start_request(cfg, sv->slots[s], reqs[i]))) {
        break;
      }
    }
    if (rc) break;
    if (!nbusy && queue.empty() && next < order.size()) {
      const double wait = reqs[order[next]].arrival - (now_s() - t0);
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
    } else if (nbusy) {
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
  }
  if (rc) {
    for (size_t s = 0; s < sv->slots.size(); s++) {
      if (!dry) cudaStreamSynchronize(sv->slots[s].cur ? sv->slots[s].cur : sv->slots[s].lo);
      if (busy[s] >= 0) reqs[busy[s]].status = CUOT_REQ_FAILED;
    }
  }
  if (stats) {
    stats->wall_s = now_s() - t0;
    stats->max_used_bytes = max_used;
  }
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->cancelled.clear();
  }
  return rc;
}

}  // extern "C"
