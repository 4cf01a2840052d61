// dev_layer_compat.cu -- the reference-signature adapter (include/
// cuot_dev_layer.h) over the C ABI.  One host thread per GPU, as the
// reference's std::async workers (dev_layer.cu:29-58, 94-143), each with its
// own context; calls block until the host outputs are written.
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cuot_dev_layer.h"
#include "ctx.cuh"

namespace {

void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
  }
}
void cuot_check(int st, const char *what) {
  if (st != CUOT_OK)
    throw std::runtime_error(std::string(what) + ": " + cuot_status_string(st) + " " + cuot_last_error());
}

// Per-device context, created on first use.
cuot_ctx *device_ctx(int dev) {
  static std::mutex mu;
  static std::vector<cuot_ctx *> ctxs;
  std::lock_guard<std::mutex> lk(mu);
  if (int(ctxs.size()) <= dev) ctxs.resize(dev + 1, nullptr);
  if (!ctxs[dev]) cuot_check(cuot_ctx_create(dev, &ctxs[dev]), "cuot_ctx_create");
  return ctxs[dev];
}

// Device scratch of at least `bytes`, carved from `m` when it is large
// enough, else from a temporary allocation owned by `tmp`.
struct Scratch {
  void *tmp = nullptr;
  ~Scratch() { if (tmp) cudaFree(tmp); }
  uint8_t *get(Mat *m, uint64_t bytes) {
    if (m && m->data() && m->size_bytes() >= bytes) return reinterpret_cast<uint8_t *>(m->data());
    cuda_check(cudaMalloc(&tmp, bytes), "scratch cudaMalloc");
    return static_cast<uint8_t *>(tmp);
  }
};

template <typename F>
void per_gpu(int ngpu, F f) {
  if (ngpu == 1) { f(0); return; }
  std::vector<std::thread> th;
  std::vector<std::string> err(ngpu);
  for (int g = 0; g < ngpu; g++)
    th.emplace_back([&, g] {
      try { f(g); } catch (const std::exception &e) { err[g] = e.what(); }
    });
  for (auto &t : th) t.join();
  for (auto &e : err)
    if (!e.empty()) throw std::runtime_error(e);
}

}  // namespace

// ---------------------------------------------------------------- Mat
Mat::Mat(std::vector<uint64_t> dim) { resize(std::move(dim)); }
Mat::Mat(const Mat &o) { *this = o; }
Mat::~Mat() {
  if (ptr_) cudaFree(ptr_);
}
uint64_t Mat::size() const {
  if (dim_.empty()) return 0;
  uint64_t s = 1;
  for (auto d : dim_) s *= d;
  return s;
}
blk *Mat::data(std::vector<uint64_t> pos) const {
  uint64_t off = 0, stride = 1;
  for (int i = int(dim_.size()) - 1; i >= 0; i--) {
    off += (i < int(pos.size()) ? pos[i] : 0) * stride;
    stride *= dim_[i];
  }
  return ptr_ + off;
}
void Mat::resize(std::vector<uint64_t> dim) {
  uint64_t need = 1;
  for (auto d : dim) need *= d;
  if (need > cap_) {
    blk *p = nullptr;
    cuda_check(cudaMalloc(&p, need * sizeof(blk)), "Mat cudaMalloc");
    if (ptr_) {
      cuda_check(cudaMemcpy(p, ptr_, size_bytes() < need * sizeof(blk) ? size_bytes() : need * sizeof(blk),
                            cudaMemcpyDeviceToDevice), "Mat resize copy");
      cudaFree(ptr_);
    }
    ptr_ = p;
    cap_ = need;
    cudaGetDevice(&device_);
  }
  dim_ = std::move(dim);
}
void Mat::clear() {
  if (ptr_) cuda_check(cudaMemset(ptr_, 0, size_bytes()), "Mat clear");
}
Mat &Mat::operator=(const Mat &o) {
  if (this == &o) return *this;
  resize(o.dim_);
  if (o.size_bytes())
    cuda_check(cudaMemcpyPeer(ptr_, device_, o.ptr_, o.device_, o.size_bytes()), "Mat copy");
  return *this;
}

// ---------------------------------------------------------------- dev_layer
void cuda_setdev(int gpu) { cuda_check(cudaSetDevice(gpu), "cudaSetDevice"); }

void cuda_mpcot_sender(Mat *expanded, Mat *buffer, Mat *sep, blk *lSum_h, blk *rSum_h,
                       blk *secret_sum, int *t, int depth, blk *delta, int ngpu) {
  std::vector<uint64_t> first(ngpu + 1, 0);
  for (int g = 0; g < ngpu; g++) first[g + 1] = first[g] + uint64_t(t[g]);
  per_gpu(ngpu, [&](int g) {
    cuda_setdev(g);
    cuot_ctx *ctx = device_ctx(g);
    const uint64_t T = uint64_t(t[g]), W = 1ull << depth;
    if (expanded[g].size() < T * W) throw std::runtime_error("cuda_mpcot_sender: expanded too small");
    Scratch s;
    uint8_t *sc = s.get(&sep[g], (2 * T * depth + T) * 16);
    cuot_block *lsum = reinterpret_cast<cuot_block *>(sc);
    cuot_block *rsum = lsum + T * depth, *ss = rsum + T * depth;
    // The roots are the first T blocks of expanded[g]; keep a copy because
    // the leaves overwrite them.
    Scratch sr;
    cuot_block *roots = reinterpret_cast<cuot_block *>(sr.get(&buffer[g], T * 16));
    cuda_check(cudaMemcpy(roots, expanded[g].data(), T * 16, cudaMemcpyDeviceToDevice), "roots");
    cuot_check(cuot_ferret_pprf_sender(ctx, roots, T, depth, reinterpret_cast<const cuot_block *>(delta),
                                       reinterpret_cast<cuot_block *>(expanded[g].data()), lsum, rsum, ss,
                                       nullptr),
               "cuot_ferret_pprf_sender");
    cuda_check(cudaMemcpy(lSum_h + first[g] * depth, lsum, T * depth * 16, cudaMemcpyDeviceToHost), "lsum");
    cuda_check(cudaMemcpy(rSum_h + first[g] * depth, rsum, T * depth * 16, cudaMemcpyDeviceToHost), "rsum");
    cuda_check(cudaMemcpy(secret_sum + first[g], ss, T * 16, cudaMemcpyDeviceToHost), "secret_sum");
  });
}

void cuda_mpcot_recver(Mat *expanded, Mat *buffer, Mat *sep, blk *cSum_h, blk *secret_sum,
                       int *t, int depth, bool *choices, int ngpu) {
  (void)buffer;
  std::vector<uint64_t> first(ngpu + 1, 0);
  for (int g = 0; g < ngpu; g++) first[g + 1] = first[g] + uint64_t(t[g]);
  per_gpu(ngpu, [&](int g) {
    cuda_setdev(g);
    cuot_ctx *ctx = device_ctx(g);
    const uint64_t T = uint64_t(t[g]), W = 1ull << depth;
    if (expanded[g].size() < T * W) throw std::runtime_error("cuda_mpcot_recver: expanded too small");
    Scratch s;
    uint8_t *sc = s.get(&sep[g], T * depth * 16 + T * 16 + T * depth + 16);
    cuot_block *mc = reinterpret_cast<cuot_block *>(sc), *ss = mc + T * depth;
    uint8_t *ch = reinterpret_cast<uint8_t *>(ss + T);
    cuda_check(cudaMemcpy(mc, cSum_h + first[g] * depth, T * depth * 16, cudaMemcpyHostToDevice), "cSum");
    cuda_check(cudaMemcpy(ss, secret_sum + first[g], T * 16, cudaMemcpyHostToDevice), "secret_sum");
    static_assert(sizeof(bool) == 1, "choices are read as bytes");
    cuda_check(cudaMemcpy(ch, choices + first[g] * depth, T * depth, cudaMemcpyHostToDevice), "choices");
    cuot_check(cuot_ferret_pprf_recver(ctx, mc, ch, ss, T, depth,
                                       reinterpret_cast<cuot_block *>(expanded[g].data()), nullptr),
               "cuot_ferret_pprf_recver");
    cuda_check(cudaDeviceSynchronize(), "cuda_mpcot_recver");
  });
}

// `key` is emp's PRP(seed).aes.rd_key (lpn_f2.h:82-86): the expanded AES-128
// schedule, whose round key 0 is the cipher key itself (FIPS-197 5.2: the
// first Nk words of the schedule are the key), so its first 16 bytes are the
// LPN seed that the index AES is keyed with.  Each n[g] must be a multiple of
// 4 except the last GPU's: the row-range LPN starts every range on a 4-row
// group, and FerretCOT's n[g] = trees x 2^h always is (ferret_cot.hpp:55-63).
void cuda_primal_lpn(Role role, Mat *pubMats, int64_t d, int64_t *n, int k, uint32_t *key,
                     Mat *expanded, blk *nn, Mat *kk_d, blk *kk, int ngpu) {
  (void)role;
  (void)pubMats;
  std::vector<int64_t> first(ngpu + 1, 0);
  for (int g = 0; g < ngpu; g++) first[g + 1] = first[g] + n[g];
  const int64_t ntot = first[ngpu];
  per_gpu(ngpu, [&](int g) {
    cuda_setdev(g);
    cuot_ctx *ctx = device_ctx(g);
    if (kk_d[g].size() < uint64_t(k)) kk_d[g].resize({uint64_t(k)});
    if (expanded[g].size() < uint64_t(n[g])) throw std::runtime_error("cuda_primal_lpn: expanded too small");
    cuda_check(cudaMemcpy(kk_d[g].data(), kk, uint64_t(k) * 16, cudaMemcpyHostToDevice), "kk");
    cuot_check(cuot_lpn_primal_range(ctx, reinterpret_cast<const uint8_t *>(key),
                                     reinterpret_cast<const cuot_block *>(kk_d[g].data()), k, int(d),
                                     reinterpret_cast<cuot_block *>(expanded[g].data()), first[g],
                                     first[g] + n[g], ntot, nullptr),
               "cuot_lpn_primal_range");
    cuda_check(cudaMemcpy(nn + first[g], expanded[g].data(), uint64_t(n[g]) * 16, cudaMemcpyDeviceToHost), "nn");
  });
}
