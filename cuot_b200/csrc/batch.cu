// batch.cu -- the batched engine: many OT-extension instances (Ferret and
// SOT, uneven n and depth, both roles) as one device program.
//
// Two independent branches (run as one chain by default, see cfg.schedule):
//   Ferret branch: a persistent PPRF launch over every Ferret sender tree
//     (each CTA pulls (instance, tree) tasks from an atomic work counter,
//     deepest trees first, and expands one whole tree per task with
//     pprf_tree, in a per-CTA scratch slot for the level ping-pong); one
//     launch selecting the receivers' OT messages (ideal OT of the sender's
//     level sums, as emp-ot's OTIdeal, ideal.h:7-31); the same persistent
//     launch over the receiver trees; one persistent LPN launch over chunks
//     of rows of every instance, both roles of a row from one index
//     computation (the two roles share the public LPN seed).
//   SOT branch: the persistent PPRF launches over the SOT sender and then
//     receiver trees; then per transform size, largest first: blocks into the
//     encode's layout, transform passes that span every instance of that
//     size (each with its own A_hat), back to blocks, and the receivers'
//     choice-bit encodes.
// cfg.schedule: CUOT_BATCH_SERIAL (default) runs every launch in one chain
// on the caller's stream, each role's PPRF as one persistent launch over the
// trees of both branches; CUOT_BATCH_FORK_FERRET runs the Ferret branch on a
// stream of its own beside the SOT branch; CUOT_BATCH_FORK_SIZES also puts
// each transform size on its own stream (sizes that share per-size FFT
// state, qc_lane, on one).  Measured on B200 (the 64-instance mix of
// log2 n in [16, 22], 10 graph replays each): one chain 86.1 ms, Ferret
// beside SOT 88.7 ms, sizes side by side 97.3 ms.  Every part already fills
// the GPU; run together, the persistent PPRF / LPN CTAs take SMs and
// shared memory from the FFT passes, and the sizes' transform passes evict
// each other's intermediate from L2.
// The whole program is captured into a CUDA graph on the first run.
// Spin-free: work queues are atomic counters, reset by a memset node.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "lpn_kernel.cuh"
#include "pprf_kernel.cuh"

namespace cuot {
namespace {

struct PprfTask {
  uint32_t item;
  uint32_t tree;
};

struct PprfBatchArgs {
  const PprfArgs *items;  // one per instance
  const int *modes;       // PprfMode per instance
  const PprfTask *tasks;  // deepest trees first
  uint32_t ntasks;
  unsigned int *counter;
  Blk *scratch;  // gridDim.x slots of 2^hmax blocks
  int hmax;
  const uint32_t *t0;
};

__global__ void __launch_bounds__(kPprfThreads, 3) pprf_batch_kernel(PprfBatchArgs b) {
  extern __shared__ __align__(16) uint32_t smem_tab[];
  __shared__ PprfSmem sm;
  __shared__ uint32_t s_task;
  stage_table(smem_tab, b.t0);
  const TabRef T{reinterpret_cast<const char *>(smem_tab), uint32_t(threadIdx.x & 31) * 4u};
  Blk *slot = b.scratch + (uint64_t(blockIdx.x) << b.hmax);
  for (;;) {
    __syncthreads();  // table staged; previous task finished with s_task
    if (threadIdx.x == 0) s_task = atomicAdd(b.counter, 1u);
    __syncthreads();
    const uint32_t task = s_task;
    if (task >= b.ntasks) break;
    const PprfTask tk = b.tasks[task];
    const PprfArgs &a = b.items[tk.item];
    switch (b.modes[tk.item]) {
      case FERRET_SEND: pprf_tree<FERRET_SEND>(a, tk.tree, slot, T, sm); break;
      case FERRET_RECV: pprf_tree<FERRET_RECV>(a, tk.tree, slot, T, sm); break;
      case SOT_SEND: pprf_tree<SOT_SEND>(a, tk.tree, slot, T, sm); break;
      default: pprf_tree<SOT_RECV>(a, tk.tree, slot, T, sm); break;
    }
  }
}

// mc[i] = choice[i] ? rsum[i] : lsum[i] for every Ferret instance (blockIdx.y).
struct SelItem {
  const uint8_t *choice;
  const Blk *lsum, *rsum;
  Blk *mc;
  uint64_t count;
};
__global__ void ferret_select_kernel(const SelItem *items) {
  const SelItem it = items[blockIdx.y];
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < it.count;
       i += uint64_t(gridDim.x) * blockDim.x)
    st_blk(it.mc + i, ldg_blk((it.choice[i] ? it.rsum : it.lsum) + i));
}

struct LpnTask {
  uint32_t job;
  uint32_t pad;
  int64_t w0, w1;  // work items [w0, w1): 4-row groups, then one-row tail rows
};
struct LpnBatchArgs {
  const LpnArgs *jobs;
  const LpnTask *tasks;
  uint32_t ntasks;
  unsigned int *counter;
  const uint32_t *t0;
};

// Two CTAs per SM: a dual-role group keeps both roles' accumulators live.
__global__ void __launch_bounds__(kLpnThreads, 2) lpn_batch_kernel(LpnBatchArgs b) {
  extern __shared__ __align__(16) uint32_t smem_tab[];
  __shared__ __align__(16) LpnArgs s_job;
  __shared__ uint32_t s_task;
  stage_table(smem_tab, b.t0);
  const TabRef T{reinterpret_cast<const char *>(smem_tab), uint32_t(threadIdx.x & 31) * 4u};
  for (;;) {
    __syncthreads();  // everyone is done with the previous s_job / s_task
    if (threadIdx.x == 0) s_task = atomicAdd(b.counter, 1u);
    __syncthreads();
    const uint32_t task = s_task;
    if (task >= b.ntasks) break;
    const LpnTask tk = b.tasks[task];
    const uint32_t *src = reinterpret_cast<const uint32_t *>(&b.jobs[tk.job]);
    for (int i = threadIdx.x; i < int(sizeof(LpnArgs) / 4); i += blockDim.x)
      reinterpret_cast<uint32_t *>(&s_job)[i] = src[i];
    __syncthreads();
    const LpnArgs &a = s_job;  // every job holds both roles (make_lpn_job)
    for (int64_t w = tk.w0 + threadIdx.x; w < tk.w1; w += blockDim.x) {
      if (w < a.ngroups) {
        if (a.d == 10) lpn_group4<10, true>(a, T, a.g0 + w);
        else lpn_group4_dyn(a, T, a.g0 + w);
      } else {
        lpn_row1(a, T, a.j0 + (w - a.ngroups));
      }
    }
  }
}

// Per-device one-time set-up of this file's constants and kernel attributes.
int batch_setup_device() {
  static std::mutex mu;
  static bool ready[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && ready[dev]) return CUOT_OK;
  cudaError_t e = pprf_upload_keys();
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(pprf_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTableBytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(lpn_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTableBytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "batch set-up failed: %s", cudaGetErrorString(e));
  }
  if (dev >= 0 && dev < 64) ready[dev] = true;
  return CUOT_OK;
}

struct SotClass {
  int e;
  int batch = 1;                  // planes per transform pass group of this size
  std::vector<int> items;         // item indices of this size
  uint8_t *planes = nullptr;      // 2 * items * 16n bytes (jobs: item x role)
  void *Y = nullptr;              // this size's intermediate: qc_y_bytes(batch)
  std::vector<const void *> ahats;  // per job
};

// PPRF branches of the program.
enum { kBrFerret = 0, kBrSot = 1 };
// Work counters: PPRF sender and receiver per branch, LPN.
constexpr int kCounters = 5;
// Events: fork, Ferret branch done, SOT PPRF done, then one per lane.
constexpr int kEvFork = 0, kEvFerret = 1, kEvSotPprf = 2, kEvLane0 = 3;

}  // namespace
}  // namespace cuot

using namespace cuot;

struct cuot_batch {
  cuot_ctx *ctx = nullptr;
  std::vector<cuot_batch_item> items;
  cuot_batch_config cfg{};
  std::vector<void *> allocs;  // every device allocation owned by the batch
  // PPRF per branch (kBrFerret, kBrSot)
  PprfBatchArgs send[2]{}, recv[2]{};
  int pprf_grid[2] = {0, 0};
  int pprf_threads = 256;
  // Ferret selection
  SelItem *sel_d = nullptr;
  int nsel = 0;
  uint64_t sel_max = 0;
  // LPN: one job per Ferret instance, both roles
  LpnBatchArgs lpn{};
  int lpn_grid = 0;
  unsigned int *counters = nullptr;  // [kCounters]
  // SOT: sizes, largest first, grouped into lanes (qc_lane) that run side by side
  std::vector<SotClass> classes;
  std::vector<std::vector<int>> lanes;  // class indices per lane, in order
  std::vector<void *> item_ahat;        // per item (SOT), nullptr otherwise
  std::vector<cuot_qc_plan *> plans;    // plain path, per item (SOT)
  // Ferret per-item sums (batch-owned)
  std::vector<Blk *> lsum, rsum, ss, mc, m0, m1;
  // concurrent schedule: streams[0] for the Ferret branch, streams[j] for
  // lane j >= 1 (lane 0 runs on the caller's stream)
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  // Completion points: group 0 is every Ferret item (after the LPN), group
  // 1 + k the k-th SOT size class in the order the lanes enqueue them (after
  // its sparse encodes).  done_ev[g] is recorded there in every batched run,
  // as an external event node when the run is a graph.
  std::vector<cudaEvent_t> done_ev;
  std::vector<int> class_group;  // per class
  std::vector<int> item_group;   // per item
  int kernels_per_run = 0;  // kernels one batched run launches
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

template <typename T>
int balloc(cuot_batch *b, T **p, uint64_t bytes) {
  void *q = nullptr;
  if (bytes == 0) bytes = 16;
  if (cudaMalloc(&q, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ENOMEM, "batch allocation of %llu bytes failed", (unsigned long long)bytes);
  }
  b->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return CUOT_OK;
}

template <typename T>
int upload(cuot_batch *b, T **dst, const std::vector<T> &v) {
  CUOT_TRY(balloc(b, dst, v.size() * sizeof(T)));
  if (!v.empty() && cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "batch upload failed");
  }
  return CUOT_OK;
}

int check_item(const cuot_batch_item &it, int i) {
  if (it.kind != CUOT_KIND_FERRET && it.kind != CUOT_KIND_SOT) return fail(CUOT_EINVAL, "item %d: bad kind", i);
  if (it.h < 1 || it.h > 20 || it.t < 1 || it.t > (1ull << 31))
    return fail(CUOT_EINVAL, "item %d: t=%llu h=%d out of range", i, (unsigned long long)it.t, it.h);
  if (!it.roots_d || !it.choice_d || !it.v_d || !it.w_d) return fail(CUOT_EINVAL, "item %d: null pointer", i);
  const uint64_t n = it.t << it.h;
  if (it.kind == CUOT_KIND_FERRET) {
    if (it.k < 1 || it.k > 0x7fffffffll || it.d < 1 || it.d > 32 || !it.kk_send_d || !it.kk_recv_d)
      return fail(CUOT_EINVAL, "item %d: bad LPN arguments", i);
    if (it.v_d == it.w_d) return fail(CUOT_EINVAL, "item %d: v and w must not alias", i);
  } else {
    if (n < 1024 || n > (1ull << 25) || (n & (n - 1)))
      return fail(CUOT_EINVAL, "item %d: SOT n=%llu must be a power of two in [2^10, 2^25]", i,
                  (unsigned long long)n);
    if (!it.base0_d || !it.base1_d || !it.mc_d || !it.a_d || !it.punct_d || !it.cbits_d)
      return fail(CUOT_EINVAL, "item %d: null SOT pointer", i);
  }
  return CUOT_OK;
}

// The LPN of both roles of a Ferret item: rows v with kk_send, rows w with
// kk_recv, one index matrix (the item's seed).
LpnArgs make_lpn_job(const cuot_batch_item &it, const uint32_t *t0) {
  LpnArgs a{};
  host_aes_key_expand(it.lpn_seed, &a.key);
  a.t0 = t0;
  a.kk = reinterpret_cast<const Blk *>(it.kk_send_d);
  a.e = reinterpret_cast<Blk *>(it.v_d);
  a.kk2 = reinterpret_cast<const Blk *>(it.kk_recv_d);
  a.e2 = reinterpret_cast<Blk *>(it.w_d);
  const int64_t n = int64_t(it.t << it.h);
  a.n = n;
  a.k = it.k;
  a.d = it.d;
  a.row_lo = 0;
  uint32_t mask = 1;
  while (int64_t(mask) < it.k) mask = (mask << 1) | 1u;  // lpn_f2.h:27-31
  a.mask = mask;
  const int64_t tail = n > 4 ? ((n - 4) + 3) / 4 * 4 : 0;
  a.tail = tail;
  a.g0 = 0;
  a.ngroups = tail / 4;
  a.j0 = tail;
  a.ntail = n - tail;
  return a;
}

int pprf_launch(cuot_batch *b, const PprfBatchArgs &args, int br, cudaStream_t st) {
  if (!args.ntasks) return 0;
  pprf_batch_kernel<<<b->pprf_grid[br], b->pprf_threads, kTableBytes, st>>>(args);
  return 1;
}

int select_launch(cuot_batch *b, cudaStream_t st) {
  if (!b->nsel) return 0;
  const unsigned gx = unsigned(std::min<uint64_t>((b->sel_max + 255) / 256, 1024));
  ferret_select_kernel<<<dim3(gx, b->nsel), 256, 0, st>>>(b->sel_d);
  return 1;
}

int lpn_launch(cuot_batch *b, cudaStream_t st) {
  if (!b->lpn.ntasks) return 0;
  lpn_batch_kernel<<<b->lpn_grid, kLpnThreads, kTableBytes, st>>>(b->lpn);
  return 1;
}

// Records completion group g's event on `st`: under stream capture as an
// external event node, so a wait outside the graph sees it (the flag is
// refused outside capture).
int record_done(cuot_batch *b, int g, cudaStream_t st) {
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "cudaStreamIsCapturing failed");
  }
  const cudaError_t e = cap == cudaStreamCaptureStatusActive
                            ? cudaEventRecordWithFlags(b->done_ev[g], st, cudaEventRecordExternal)
                            : cudaEventRecord(b->done_ev[g], st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "batch completion event record failed");
  }
  return CUOT_OK;
}

// The SOT sizes of one lane, in order, on `st`.
int enqueue_lane(cuot_batch *b, const std::vector<int> &lane, cudaStream_t st) {
  cuot_ctx *ctx = b->ctx;
  for (int ci : lane) {
    SotClass &c = b->classes[ci];
    const uint64_t n = 1ull << c.e;
    const int njobs = int(c.items.size()) * 2;
    for (int j = 0; j < njobs; j++) {
      const cuot_batch_item &it = b->items[c.items[j / 2]];
      CUOT_TRY(qc_job_to_layout(ctx, c.e, j % 2 ? it.w_d : it.v_d, c.planes + uint64_t(j) * n * 16, st));
    }
    CUOT_TRY(qc_encode_jobs(ctx, c.e, reinterpret_cast<uint64_t *>(c.planes), njobs, c.ahats.data(), c.Y,
                            c.batch, st));
    for (int j = 0; j < njobs; j++) {
      const cuot_batch_item &it = b->items[c.items[j / 2]];
      CUOT_TRY(qc_job_from_layout(ctx, c.e, c.planes + uint64_t(j) * n * 16, j % 2 ? it.w_d : it.v_d, st));
    }
    for (int i : c.items) {
      const cuot_batch_item &it = b->items[i];
      CUOT_TRY(cuot_qc_encode_sparse(ctx, it.a_d, it.punct_d, int(it.t), n, it.cbits_d, st));
    }
    CUOT_TRY(record_done(b, b->class_group[ci], st));
  }
  return CUOT_OK;
}

int ev_fail() {
  cudaGetLastError();
  return fail(CUOT_ECUDA, "batch stream fork / join failed");
}

// Enqueues the batched program on `st`.  ev (optional, diagnostic): 5 events
// recorded before the sender PPRF, the receiver PPRF, the LPN, the SOT
// encodes, and at the end; with ev the program runs as one chain (phases in
// order), as it does with CUOT_BATCH_SERIAL.
int enqueue(cuot_batch *b, cudaStream_t st, cudaEvent_t *ev = nullptr) {
  const unsigned long long k0 = cuot_launch_count();
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], st);
  };
  if (cudaMemsetAsync(b->counters, 0, kCounters * sizeof(unsigned int), st) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "counter reset failed");
  }
  const int sched = ev ? CUOT_BATCH_SERIAL : b->cfg.schedule;
  if (sched == CUOT_BATCH_SERIAL) {
    int launches = 0;
    mark(0);
    launches += pprf_launch(b, b->send[kBrSot], kBrSot, st);
    launches += pprf_launch(b, b->send[kBrFerret], kBrFerret, st);
    launches += select_launch(b, st);
    mark(1);
    launches += pprf_launch(b, b->recv[kBrSot], kBrSot, st);
    launches += pprf_launch(b, b->recv[kBrFerret], kBrFerret, st);
    mark(2);
    launches += lpn_launch(b, st);
    CUOT_TRY(launch_status(launches));
    if (b->lpn.ntasks) CUOT_TRY(record_done(b, 0, st));
    mark(3);
    for (const auto &lane : b->lanes) CUOT_TRY(enqueue_lane(b, lane, st));
    mark(4);
  } else {
    cudaEvent_t *E = b->events.data();
    if (cudaEventRecord(E[kEvFork], st) != cudaSuccess) return ev_fail();
    const bool fer = b->send[kBrFerret].ntasks > 0;
    if (fer) {  // Ferret branch on streams[0]
      cudaStream_t sf = b->streams[0];
      if (cudaStreamWaitEvent(sf, E[kEvFork], 0) != cudaSuccess) return ev_fail();
      int launches = pprf_launch(b, b->send[kBrFerret], kBrFerret, sf);
      launches += select_launch(b, sf);
      launches += pprf_launch(b, b->recv[kBrFerret], kBrFerret, sf);
      launches += lpn_launch(b, sf);
      CUOT_TRY(launch_status(launches));
      if (b->lpn.ntasks) CUOT_TRY(record_done(b, 0, sf));
      if (cudaEventRecord(E[kEvFerret], sf) != cudaSuccess) return ev_fail();
    }
    // SOT branch: PPRFs on the caller's stream, then the lanes side by side
    CUOT_TRY(launch_status(pprf_launch(b, b->send[kBrSot], kBrSot, st) +
                           pprf_launch(b, b->recv[kBrSot], kBrSot, st)));
    const bool sizes = sched == CUOT_BATCH_FORK_SIZES;
    if (sizes) {
      if (cudaEventRecord(E[kEvSotPprf], st) != cudaSuccess) return ev_fail();
      for (size_t j = 1; j < b->lanes.size(); j++) {
        cudaStream_t sl = b->streams[j];
        if (cudaStreamWaitEvent(sl, E[kEvSotPprf], 0) != cudaSuccess) return ev_fail();
        CUOT_TRY(enqueue_lane(b, b->lanes[j], sl));
        if (cudaEventRecord(E[kEvLane0 + j], sl) != cudaSuccess) return ev_fail();
      }
      if (!b->lanes.empty()) CUOT_TRY(enqueue_lane(b, b->lanes[0], st));
    } else {
      for (const auto &lane : b->lanes) CUOT_TRY(enqueue_lane(b, lane, st));
    }
    if (fer && cudaStreamWaitEvent(st, E[kEvFerret], 0) != cudaSuccess) return ev_fail();
    if (sizes)
      for (size_t j = 1; j < b->lanes.size(); j++)
        if (cudaStreamWaitEvent(st, E[kEvLane0 + j], 0) != cudaSuccess) return ev_fail();
  }
  b->kernels_per_run = int(cuot_launch_count() - k0);
  return CUOT_OK;
}

}  // namespace

extern "C" {

int cuot_batch_create(cuot_ctx *ctx, const cuot_batch_item *items, int count,
                      const cuot_batch_config *cfg, cuot_batch **out) {
  if (!ctx || !items || count < 1 || !out) return fail(CUOT_EINVAL, "bad argument");
  *out = nullptr;
  for (int i = 0; i < count; i++) CUOT_TRY(check_item(items[i], i));
  DeviceGuard g(ctx);
  CUOT_TRY(batch_setup_device());
  cuot_batch *b = new cuot_batch;
  b->ctx = ctx;
  b->items.assign(items, items + count);
  if (cfg) b->cfg = *cfg;
  int st = CUOT_OK;
  auto cleanup = [&](int s) {
    cuot_batch_destroy(b);
    return s;
  };
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int per_sm = b->cfg.ctas_per_sm > 0 ? b->cfg.ctas_per_sm : 3;
  if (b->cfg.pprf_threads != 0 && b->cfg.pprf_threads != 128 && b->cfg.pprf_threads != 256)
    return cleanup(fail(CUOT_EINVAL, "pprf_threads must be 128 or 256"));
  if (b->cfg.schedule != CUOT_BATCH_SERIAL && b->cfg.schedule != CUOT_BATCH_FORK_FERRET &&
      b->cfg.schedule != CUOT_BATCH_FORK_SIZES)
    return cleanup(fail(CUOT_EINVAL, "schedule must be one of CUOT_BATCH_SERIAL / FORK_FERRET / FORK_SIZES"));
  b->pprf_threads = b->cfg.pprf_threads ? b->cfg.pprf_threads : 256;

  // ---- per-item device state
  b->lsum.assign(count, nullptr); b->rsum.assign(count, nullptr); b->ss.assign(count, nullptr);
  b->mc.assign(count, nullptr); b->m0.assign(count, nullptr); b->m1.assign(count, nullptr);
  b->item_ahat.assign(count, nullptr);
  b->plans.assign(count, nullptr);
  std::vector<PprfArgs> sargs(count), rargs(count);
  std::vector<int> smodes(count), rmodes(count);
  std::vector<SelItem> sel;
  int hmax[2] = {1, 1};
  for (int i = 0; i < count; i++) {
    const cuot_batch_item &it = items[i];
    const uint64_t t = it.t;
    const int h = it.h;
    const int br = it.kind == CUOT_KIND_FERRET ? kBrFerret : kBrSot;
    hmax[br] = std::max(hmax[br], h);
    PprfArgs s{}, r{};
    s.t = r.t = t;
    s.h = r.h = h;
    s.t0 = r.t0 = ctx->t0_d;
    s.roots = reinterpret_cast<const Blk *>(it.roots_d);
    s.leaves = reinterpret_cast<Blk *>(it.v_d);
    r.leaves = reinterpret_cast<Blk *>(it.w_d);
    s.delta = host_load_blk(&it.delta);
    if (it.kind == CUOT_KIND_FERRET) {
      if ((st = balloc(b, &b->lsum[i], t * h * 16)) || (st = balloc(b, &b->rsum[i], t * h * 16)) ||
          (st = balloc(b, &b->ss[i], t * 16)) || (st = balloc(b, &b->mc[i], t * h * 16)))
        return cleanup(st);
      s.lsum = b->lsum[i]; s.rsum = b->rsum[i]; s.ss_out = b->ss[i];
      r.mc = b->mc[i]; r.choice = it.choice_d; r.ss_in = b->ss[i];
      smodes[i] = FERRET_SEND; rmodes[i] = FERRET_RECV;
      sel.push_back(SelItem{it.choice_d, b->lsum[i], b->rsum[i], b->mc[i], t * h});
      b->sel_max = std::max(b->sel_max, t * h);
    } else {
      if ((st = balloc(b, &b->m0[i], (h + 1) * t * 16)) || (st = balloc(b, &b->m1[i], (h + 1) * t * 16)))
        return cleanup(st);
      s.base0 = reinterpret_cast<const Blk *>(it.base0_d);
      s.base1 = reinterpret_cast<const Blk *>(it.base1_d);
      s.m0 = b->m0[i]; s.m1 = b->m1[i];
      r.m0_in = b->m0[i]; r.m1_in = b->m1[i];
      r.mc = reinterpret_cast<const Blk *>(it.mc_d);
      r.choice = it.choice_d;
      smodes[i] = SOT_SEND; rmodes[i] = SOT_RECV;
    }
    sargs[i] = s;
    rargs[i] = r;
  }
  PprfArgs *sd = nullptr, *rd = nullptr;
  int *smd = nullptr, *rmd = nullptr;
  if ((st = upload(b, &sd, sargs)) || (st = upload(b, &rd, rargs)) || (st = upload(b, &smd, smodes)) ||
      (st = upload(b, &rmd, rmodes)) || (st = balloc(b, &b->counters, kCounters * sizeof(unsigned int))))
    return cleanup(st);
  // ---- PPRF tasks: every tree, deepest first.  Concurrent schedules keep
  // one list per branch, each with its own per-CTA scratch slots (the
  // branches run at the same time); the serial schedule puts every tree in
  // one list (slot 0) so each role is a single persistent launch.
  std::vector<int> order(count);
  for (int i = 0; i < count; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return items[x].h > items[y].h; });
  const bool merged = b->cfg.schedule == CUOT_BATCH_SERIAL;
  if (merged) hmax[0] = hmax[1] = std::max(hmax[0], hmax[1]);
  for (int br = 0; br < 2; br++) {
    std::vector<PprfTask> tasks;
    for (int i : order)
      if (merged ? br == 0 : (items[i].kind == CUOT_KIND_FERRET) == (br == kBrFerret))
        for (uint64_t tr = 0; tr < items[i].t; tr++) tasks.push_back(PprfTask{uint32_t(i), uint32_t(tr)});
    if (tasks.empty()) continue;
    b->pprf_grid[br] = int(std::min<uint64_t>(uint64_t(sms) * per_sm, tasks.size()));
    PprfTask *td = nullptr;
    Blk *pscr = nullptr;
    if ((st = upload(b, &td, tasks)) || (st = balloc(b, &pscr, (uint64_t(b->pprf_grid[br]) << hmax[br]) * 16)))
      return cleanup(st);
    b->send[br] = PprfBatchArgs{sd, smd, td, uint32_t(tasks.size()), b->counters + 2 * br, pscr, hmax[br],
                                ctx->t0_d};
    b->recv[br] = PprfBatchArgs{rd, rmd, td, uint32_t(tasks.size()), b->counters + 2 * br + 1, pscr, hmax[br],
                                ctx->t0_d};
  }
  b->nsel = int(sel.size());
  if (b->nsel && (st = upload(b, &b->sel_d, sel))) return cleanup(st);

  // ---- LPN: one job per Ferret item (both roles), tasks of rows_per_task rows
  const int64_t rows_per_task = b->cfg.lpn_rows_per_task > 0 ? (b->cfg.lpn_rows_per_task + 3) / 4 * 4 : 65536;
  std::vector<LpnArgs> jobs;
  std::vector<LpnTask> ltasks;
  for (int i = 0; i < count; i++) {
    const cuot_batch_item &it = items[i];
    if (it.kind != CUOT_KIND_FERRET) continue;
    const LpnArgs a = make_lpn_job(it, ctx->t0_d);
    const uint32_t j = uint32_t(jobs.size());
    jobs.push_back(a);
    const int64_t total = a.ngroups + a.ntail, chunk = rows_per_task / 4;
    for (int64_t w0 = 0; w0 < total; w0 += chunk) ltasks.push_back(LpnTask{j, 0, w0, std::min(total, w0 + chunk)});
  }
  if (!jobs.empty()) {
    LpnArgs *jd = nullptr;
    LpnTask *ltd = nullptr;
    if ((st = upload(b, &jd, jobs)) || (st = upload(b, &ltd, ltasks))) return cleanup(st);
    b->lpn = LpnBatchArgs{jd, ltd, uint32_t(ltasks.size()), b->counters + 4, ctx->t0_d};
    b->lpn_grid = int(std::min<uint64_t>(uint64_t(sms) * per_sm, ltasks.size()));
  }

  // ---- SOT size classes (largest first), their lanes, transforms of every `a`
  for (int i = 0; i < count; i++) {
    const cuot_batch_item &it = items[i];
    if (it.kind != CUOT_KIND_SOT) continue;
    const int e = __builtin_ctzll(it.t << it.h);
    auto c = std::find_if(b->classes.begin(), b->classes.end(), [&](const SotClass &x) { return x.e == e; });
    if (c == b->classes.end()) {
      b->classes.push_back(SotClass{});
      c = b->classes.end() - 1;
      c->e = e;
    }
    c->items.push_back(i);
  }
  std::stable_sort(b->classes.begin(), b->classes.end(),
                   [](const SotClass &x, const SotClass &y) { return x.e > y.e; });
  std::map<int, int> lane_of;  // qc_lane -> index into b->lanes
  for (size_t ci = 0; ci < b->classes.size(); ci++) {
    SotClass &c = b->classes[ci];
    const uint64_t n = 1ull << c.e;
    if ((st = qc_prepare(ctx, c.e))) return cleanup(st);
    if ((st = balloc(b, &c.planes, 2 * c.items.size() * n * 16))) return cleanup(st);
    int pb = b->cfg.qc_planes_per_pass > 0 ? b->cfg.qc_planes_per_pass
                                           : qc_default_batch(n, int(256 * c.items.size()));
    pb = std::min(pb, int(256 * c.items.size()));
    c.batch = pb;
    if ((st = balloc(b, &c.Y, qc_y_bytes(ctx, c.e, pb)))) return cleanup(st);
    const int key = qc_lane(ctx, c.e);
    auto l = lane_of.find(key);
    if (l == lane_of.end()) {
      lane_of[key] = int(b->lanes.size());
      b->lanes.push_back({int(ci)});
    } else {
      b->lanes[l->second].push_back(int(ci));
    }
    for (int i : c.items) {
      if ((st = balloc(b, &b->item_ahat[i], qc_ahat_bytes(ctx, c.e)))) return cleanup(st);
      if ((st = qc_build_ahat(ctx, c.e, items[i].a_d, c.Y, b->item_ahat[i], nullptr))) return cleanup(st);
      c.ahats.push_back(b->item_ahat[i]);  // sender job
      c.ahats.push_back(b->item_ahat[i]);  // receiver job
      if ((st = cuot_qc_plan_create(ctx, items[i].a_d, n, nullptr, &b->plans[i]))) return cleanup(st);
    }
  }
  // ---- streams and events of the concurrent schedule
  const size_t nstreams = std::max<size_t>(1, b->lanes.size());
  for (size_t j = 0; j < nstreams; j++) {
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return cleanup(fail(CUOT_ECUDA, "batch stream creation failed"));
    }
    b->streams.push_back(s);
  }
  for (size_t j = 0; j < kEvLane0 + b->lanes.size(); j++) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return cleanup(fail(CUOT_ECUDA, "batch event creation failed"));
    }
    b->events.push_back(e);
  }
  // ---- completion groups: Ferret items, then the SOT classes in enqueue order
  b->class_group.assign(b->classes.size(), 0);
  int ngroups = 1;
  for (const auto &lane : b->lanes)
    for (int ci : lane) b->class_group[ci] = ngroups++;
  b->item_group.assign(count, 0);
  for (size_t ci = 0; ci < b->classes.size(); ci++)
    for (int i : b->classes[ci].items) b->item_group[i] = b->class_group[ci];
  for (int g = 0; g < ngroups; g++) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return cleanup(fail(CUOT_ECUDA, "batch event creation failed"));
    }
    b->done_ev.push_back(e);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    cudaGetLastError();
    return cleanup(fail(CUOT_ECUDA, "batch set-up kernels failed"));
  }
  *out = b;
  return CUOT_OK;
}

int cuot_batch_run(cuot_batch *b, void *stream) {
  if (!b) return fail(CUOT_EINVAL, "null batch");
  DeviceGuard g(b->ctx);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!b->cfg.use_graph) return enqueue(b, st);
  if (!b->exec) {
    if (st == nullptr) return fail(CUOT_EINVAL, "graph capture needs a non-default stream");
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      return fail(CUOT_ECUDA, "cudaStreamBeginCapture failed");
    }
    int s = enqueue(b, st);
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &gr);
    if (s != CUOT_OK || e != cudaSuccess) {
      cudaGetLastError();
      if (gr) cudaGraphDestroy(gr);
      return s != CUOT_OK ? s : fail(CUOT_ECUDA, "graph capture failed: %s", cudaGetErrorString(e));
    }
    if (cudaGraphInstantiate(&b->exec, gr, 0) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphDestroy(gr);
      return fail(CUOT_ECUDA, "cudaGraphInstantiate failed");
    }
    b->graph = gr;
  }
  if (cudaGraphLaunch(b->exec, st) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "cudaGraphLaunch failed");
  }
  return launch_status(0);
}

int cuot_batch_run_plain(cuot_batch *b, void *stream) {
  if (!b) return fail(CUOT_EINVAL, "null batch");
  DeviceGuard g(b->ctx);
  cuot_ctx *ctx = b->ctx;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (size_t i = 0; i < b->items.size(); i++) {
    const cuot_batch_item &it = b->items[i];
    const uint64_t t = it.t, n = t << it.h;
    const int h = it.h;
    if (it.kind == CUOT_KIND_FERRET) {
      CUOT_TRY(cuot_ferret_pprf_sender(ctx, it.roots_d, t, h, &it.delta, it.v_d,
                                       reinterpret_cast<cuot_block *>(b->lsum[i]),
                                       reinterpret_cast<cuot_block *>(b->rsum[i]),
                                       reinterpret_cast<cuot_block *>(b->ss[i]), st));
      // the selection reads this item's descriptor from the batch's device copy
      size_t k = 0;
      for (size_t j = 0; j < i; j++) k += b->items[j].kind == CUOT_KIND_FERRET;
      ferret_select_kernel<<<dim3(unsigned(std::min<uint64_t>((t * h + 255) / 256, 1024)), 1), 256, 0, st>>>(
          b->sel_d + k);
      CUOT_TRY(launch_status());
      CUOT_TRY(cuot_ferret_pprf_recver(ctx, reinterpret_cast<cuot_block *>(b->mc[i]), it.choice_d,
                                       reinterpret_cast<cuot_block *>(b->ss[i]), t, h, it.w_d, st));
      CUOT_TRY(cuot_lpn_primal_dual(ctx, it.lpn_seed, it.kk_send_d, it.kk_recv_d, it.k, it.d, it.v_d, it.w_d,
                                    int64_t(n), st));
    } else {
      CUOT_TRY(cuot_sot_pprf_sender(ctx, it.roots_d, t, h, &it.delta, it.base0_d, it.base1_d, it.v_d,
                                    reinterpret_cast<cuot_block *>(b->m0[i]),
                                    reinterpret_cast<cuot_block *>(b->m1[i]), st));
      CUOT_TRY(cuot_sot_pprf_recver(ctx, reinterpret_cast<cuot_block *>(b->m0[i]),
                                    reinterpret_cast<cuot_block *>(b->m1[i]), it.mc_d, it.choice_d, t, h,
                                    it.w_d, st));
      CUOT_TRY(cuot_qc_plan_dual_lpn(b->plans[i], it.v_d, st));
      CUOT_TRY(cuot_qc_plan_dual_lpn(b->plans[i], it.w_d, st));
      CUOT_TRY(cuot_qc_encode_sparse(ctx, it.a_d, it.punct_d, int(t), n, it.cbits_d, st));
    }
  }
  return CUOT_OK;
}

int cuot_batch_kernels_per_run(const cuot_batch *b) { return b ? b->kernels_per_run : 0; }

int cuot_batch_item_rank(const cuot_batch *b, int item) {
  if (!b || item < 0 || item >= int(b->items.size())) return -1;
  return b->item_group[item];
}

int cuot_batch_wait_item(cuot_batch *b, int item, void *stream) {
  if (!b || item < 0 || item >= int(b->items.size())) return fail(CUOT_EINVAL, "bad argument");
  DeviceGuard g(b->ctx);
  if (cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), b->done_ev[b->item_group[item]], 0) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUOT_ECUDA, "cudaStreamWaitEvent failed");
  }
  return CUOT_OK;
}

int cuot_batch_run_phases(cuot_batch *b, void *stream, float *phase_ms) {
  if (!b || !phase_ms) return fail(CUOT_EINVAL, "bad argument");
  DeviceGuard g(b->ctx);
  cudaEvent_t ev[5];
  for (auto &e : ev) cudaEventCreate(&e);
  int s = enqueue(b, static_cast<cudaStream_t>(stream), ev);
  if (s == CUOT_OK && cudaEventSynchronize(ev[4]) == cudaSuccess)
    for (int i = 0; i < 4; i++) cudaEventElapsedTime(&phase_ms[i], ev[i], ev[i + 1]);
  for (auto &e : ev) cudaEventDestroy(e);
  return s;
}

int cuot_batch_destroy(cuot_batch *b) {
  if (!b) return CUOT_OK;
  {
    DeviceGuard g(b->ctx);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto *p : b->plans)
      if (p) cuot_qc_plan_destroy(p);
    for (auto s : b->streams) cudaStreamSynchronize(s);
    for (auto s : b->streams) cudaStreamDestroy(s);
    for (auto e : b->events) cudaEventDestroy(e);
    for (auto e : b->done_ev) cudaEventDestroy(e);
    for (void *p : b->allocs) cudaFree(p);
  }
  delete b;
  return CUOT_OK;
}

}  // extern "C"
