// capi.cpp -- host implementation of the C ABI (include/curplsh_b200.h):
// DeviceResources, IndexBF state, per-stream workspaces and the search
// orchestration (query prep -> fused tensor-core filter -> merge + rerank).
//
// Orchestration replaces searchL2Distance (cuRPLSH src/internal/search.cu:79-216):
// no per-call cudaMalloc of Q x N distance tiles (workspaces are cached per
// stream and only grow), no cudaDeviceSynchronize between tiles, and a single
// persistent launch instead of Q-tile x N-tile loops on alternating streams.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/curplsh_b200.h"
#include "common.cuh"
#include "fused_knn.h"

using namespace curplsh_b200;

// ------------------------------------------------------------------ errors
namespace {
thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CUDA_TRY(call)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                  \
      if (e_ == cudaErrorMemoryAllocation) {                                                  \
        cudaGetLastError();                                                                   \
        return set_error(CURPLSH_ERR_OOM, "%s: %s", #call, cudaGetErrorString(e_));           \
      }                                                                                       \
      return set_error(CURPLSH_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));     \
    }                                                                                         \
  } while (0)

// RAII current-device selection (DeviceScope, include/device_resources.h:13-32)
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) {
      prev = cur;
      cudaSetDevice(dev);
    }
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

// where a pointer lives: -1 host (pageable or pinned), >= 0 device ordinal; managed counts as device
int pointer_device(const void* p, bool* managed = nullptr) {
  cudaPointerAttributes a;
  if (managed) *managed = false;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  if (a.type == cudaMemoryTypeDevice) return a.device;
  if (a.type == cudaMemoryTypeManaged) {
    if (managed) *managed = true;
    return a.device;
  }
  return -1;
}

// Device buffer that only grows.
struct DevBuf {
  void* ptr = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t want = std::max(bytes, (size_t)1 << 20);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

struct PinnedBuf {
  void* ptr = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost(&ptr, std::max(bytes, (size_t)1 << 16));
    if (e == cudaSuccess) cap = std::max(bytes, (size_t)1 << 16);
    return e;
  }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

// Bump allocator over one workspace buffer (256-byte aligned slices).
struct Carve {
  char* base;
  size_t off = 0;
  explicit Carve(void* b) : base(static_cast<char*>(b)) {}
  template <class T>
  T* take(size_t count) {
    off = (size_t)round_up((long long)off, 256);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
};

}  // namespace

// ------------------------------------------------------------------ resources
struct DevRes {
  cudaStream_t def = nullptr;
  bool def_owned = false;
  cudaStream_t alt[2] = {nullptr, nullptr};
  cudaStream_t copy = nullptr;
  int num_sms = 0;
};

// Reference counted: every index holds a reference, so destroying the
// resources while indexes are alive only drops the caller's reference and the
// streams live until the last index is destroyed.
struct curplsh_resources {
  std::mutex mu;
  std::map<int, DevRes> devs;
  std::map<int, cudaStream_t> user_default;
  std::atomic<int> refs{1};
};

namespace {
int init_device(curplsh_resources* r, int device, DevRes** out) {
  std::lock_guard<std::mutex> lk(r->mu);
  auto it = r->devs.find(device);
  if (it != r->devs.end()) {
    *out = &it->second;
    return CURPLSH_OK;
  }
  int ndev = 0;
  CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return set_error(CURPLSH_ERR_INVALID_ARG, "device %d out of range (%d devices)", device, ndev);
  DeviceScope scope(device);
  DevRes d;
  auto u = r->user_default.find(device);
  if (u != r->user_default.end()) {
    d.def = u->second;
  } else {
    CUDA_TRY(cudaStreamCreateWithFlags(&d.def, cudaStreamNonBlocking));
    d.def_owned = true;
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&d.alt[0], cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamCreateWithFlags(&d.alt[1], cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamCreateWithFlags(&d.copy, cudaStreamNonBlocking));
  CUDA_TRY(cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, device));
  auto res = r->devs.emplace(device, d);
  *out = &res.first->second;
  return CURPLSH_OK;
}
}  // namespace

// ------------------------------------------------------------------ index
namespace {
struct StreamWorkspace {
  DevBuf dev;      // query operands, pools, staging
  PinnedBuf host;  // status read-back
};
}  // namespace

struct curplsh_index {
  curplsh_resources* res = nullptr;
  int dim = 0;
  curplsh_bf_config cfg{};
  DevRes* dres = nullptr;
  std::mutex mu;
  // database
  int64_t n = 0;
  long long n_pad = 0;
  long long ld16 = 0, ld8 = 0;
  float* x32 = nullptr;  // [n x dim]
  bool x32_owned = false;
  float* xn = nullptr;            // [n_pad]
  __nv_bfloat16* xh = nullptr;    // [n_pad x ld16]
  __nv_bfloat16* xl = nullptr;    // [n_pad x ld16]
  uint8_t* x8 = nullptr;          // [n_pad x ld8]   (built on first FP8 search)
  float* xs = nullptr;            // [n_pad]
  uint32_t* status = nullptr;     // device words: [0] error status, [1] nonzero if a row is not exactly BF16
  bool bf16_exact = false;        // every stored value is exactly a BF16 value (rerank reads xh)
  long long generation = 0;       // bumped whenever the prepared database changes (add, reset)
  cudaEvent_t order_ev = nullptr; // orders default-stream searches after the legacy stream
  std::map<cudaStream_t, std::unique_ptr<StreamWorkspace>> ws;

  void free_db() {
    if (x32_owned && x32) cudaFree(x32);
    x32 = nullptr;
    x32_owned = false;
    for (void* p : {(void*)xn, (void*)xh, (void*)xl, (void*)x8, (void*)xs})
      if (p) cudaFree(p);
    xn = nullptr;
    xh = xl = nullptr;
    x8 = nullptr;
    xs = nullptr;
    n = 0;
    n_pad = 0;
  }
};

namespace {

int build_fp8(curplsh_index* ix, cudaStream_t st) {
  if (ix->x8 || ix->n == 0) return CURPLSH_OK;
  CUDA_TRY(cudaMalloc(&ix->x8, (size_t)ix->n_pad * ix->ld8));
  CUDA_TRY(cudaMalloc(&ix->xs, (size_t)ix->n_pad * sizeof(float)));
  CUDA_TRY(launch_prep_rows(ix->x32, ix->dim, (int)ix->n, ix->n_pad, ix->dim, nullptr, 0.f, nullptr, nullptr,
                            ix->ld16, ix->x8, ix->xs, ix->ld8, st));
  return CURPLSH_OK;
}

int kprime_for(int form, int k, int rerank_factor, int64_t n) {
  long long kp;
  if (form == kFormExact)
    kp = round_up(k + 16, 32);
  else
    kp = round_up(std::max<long long>((long long)rerank_factor * k, k + 16), 32);
  kp = std::min<long long>(kp, 4096);
  kp = std::max<long long>(kp, k);
  kp = std::min<long long>(kp, n);
  return (int)kp;
}

// Pool capacity: k' kept keys + room for one or two tiles (both halves append
// to the pool; see pool_sync_tiles) + refresh headroom.  A selection runs only when fewer than a tile of
// free slots remain, so each absorbs >= max(k', headroom) survivors.  With the
// default headroom a capacity just above 512 or 1024 keys is trimmed to it
// when that still leaves >= 128 keys of headroom: up to 1024 keys the
// selection holds the whole pool in registers.
int pool_capacity(int kp, int headroom = kTuneDefaultHeadroom) {
  // room for two tiles between selections when the pool still fits registers
  const int P2 = (int)round_up(kp + 2 * kPoolRoom + std::max(kp, headroom), 32);
  if (P2 <= 1024) return P2;
  int P = (int)round_up(kp + kPoolRoom + std::max(kp, headroom), 32);
  if (headroom == kTuneDefaultHeadroom) {
    for (int lim : {512, 1024})
      if (P > lim && kp + kPoolRoom + 128 <= lim && P <= lim + lim / 2) P = lim;
  }
  return P;
}

struct Timing {
  cudaEvent_t ev[5] = {};
  bool on = false;
  int create() {
    for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
    on = true;
    return CURPLSH_OK;
  }
  void rec(int i, cudaStream_t st) {
    if (on) cudaEventRecord(ev[i], st);
  }
  ~Timing() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// The search proper.  Device-side inputs/outputs; `st` orders everything.
int search_device(curplsh_index* ix, int nq, const float* q_dev, int k, int form, int rerank_factor, int* out_idx,
                  float* out_dist, cudaStream_t st, StreamWorkspace& w, char* extra_base, Timing* tm) {
  const int d = ix->dim;
  if (ix->n == 0) {
    CUDA_TRY(launch_fill_results(out_idx, out_dist, (long long)nq * k, st));
    return CURPLSH_OK;
  }
  if (form == kFormFP8) {
    int rc = build_fp8(ix, st);
    if (rc) return rc;
  }
  const int kp = kprime_for(form, k, rerank_factor, ix->n);
  const TuneParams tp = tune_lookup(form, d, k, nq);
  const int P = pool_capacity(kp, tp.headroom);
  FusedPlan plan;
  plan_fused(nq, (int)ix->n, ix->dres->num_sms, &plan, default_split_q4(tp, P));
  const long long nq_pad = round_up(nq, kBM);
  const size_t pool_lists = (size_t)plan.num_qblocks * kBM * plan.units_per_block;

  Carve c(extra_base);
  __nv_bfloat16* qh = c.take<__nv_bfloat16>((size_t)nq_pad * ix->ld16);
  __nv_bfloat16* ql = form == kFormExact ? c.take<__nv_bfloat16>((size_t)nq_pad * ix->ld16) : nullptr;
  uint8_t* q8 = form == kFormFP8 ? c.take<uint8_t>((size_t)nq_pad * ix->ld8) : nullptr;
  float* qn = c.take<float>(nq_pad);
  float* qs = c.take<float>(nq_pad);
  uint32_t* qbound = c.take<uint32_t>(3 * nq_pad);  // [nq_pad] k'-th bounds, then [nq_pad][2] half bounds
  int* counts = c.take<int>(pool_lists);
  uint64_t* pools = c.take<uint64_t>(pool_lists * (size_t)P);
  (void)w;

  tm->rec(1, st);
  CUDA_TRY(launch_prep_rows(q_dev, d, nq, nq_pad, d, qn, 0.f, form == kFormFP8 ? nullptr : qh, ql, ix->ld16,
                            q8, qs, ix->ld8, st, form == kFormFP8 ? kAugNone : kAugQuery));
  CUDA_TRY(cudaMemsetAsync(qbound, 0xFF, (size_t)3 * nq_pad * sizeof(uint32_t), st));
  tm->rec(2, st);
  FusedLaunch f{};
  f.nq = nq;
  f.nb = (int)ix->n;
  f.d = d;
  f.kprime = kp;
  f.pool_cap = P;
  f.form = form;
  f.nq_pad = nq_pad;
  f.nb_pad = ix->n_pad;
  f.ld16 = ix->ld16;
  f.ld8 = ix->ld8;
  f.qh = qh;
  f.ql = ql;
  f.q8 = q8;
  f.qn = qn;
  f.qs = qs;
  f.xh = ix->xh;
  f.xl = ix->xl;
  f.x8 = ix->x8;
  f.xn = ix->xn;
  f.xs = ix->xs;
  f.pools = pools;
  f.pool_counts = counts;
  f.q_bound = qbound;
  f.q_bound_half = qbound + nq_pad;
  f.status = ix->status;
  f.plan = plan;
#ifdef CURPLSH_FUSED_STATS
  // instrumented builds: per-role cycle counters of the fused pass, printed to stderr
  static unsigned long long* stats = nullptr;
  if (!stats) CUDA_TRY(cudaMalloc(&stats, kStatCount * sizeof(unsigned long long)));
  CUDA_TRY(cudaMemsetAsync(stats, 0, kStatCount * sizeof(unsigned long long), st));
  f.stats = stats;
#endif
  CUDA_TRY(launch_fused(f, st));
#ifdef CURPLSH_FUSED_STATS
  {
    unsigned long long h[kStatCount];
    CUDA_TRY(cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    const double ctas = (double)plan.grid;
    fprintf(stderr,
            "[fused-stats] grid %d kp %d P %d | per CTA (Mcycles): total %.2f prod_wait_empty %.2f mma_wait_full %.2f "
            "mma_wait_acc %.2f | per epi warp: wait_acc %.2f filter %.2f refresh %.2f | refreshes %llu survivors %llu\n",
            plan.grid, kp, P, h[kStatCtaCycles] / ctas / 1e6, h[kStatProducerWaitEmpty] / ctas / 1e6,
            h[kStatMmaWaitFull] / ctas / 1e6, h[kStatMmaWaitAccEmpty] / ctas / 1e6,
            h[kStatEpiWaitAccFull] / ctas / 8 / 1e6, h[kStatEpiFilter] / ctas / 8 / 1e6,
            h[kStatEpiRefresh] / ctas / 8 / 1e6, h[kStatRefreshes], h[kStatSurvivors]);
    fprintf(stderr,
            "[fused-stats2] radix passes/refresh %.2f | slow chunks %llu (%.1f%% of warp-chunks) | loop iters/slow "
            "chunk %.2f | tmem Mcycles/warp %.2f | pair barriers Mcycles/warp %.2f\n",
            h[kStatRefreshes] ? (double)h[kStatRadixPasses] / h[kStatRefreshes] : 0.0, h[kStatSlowChunks],
            100.0 * h[kStatSlowChunks] / (ctas * 8 * (double)plan.work_per_cta * 4),
            h[kStatSlowChunks] ? (double)h[kStatLoopIters] / h[kStatSlowChunks] : 0.0,
            h[kStatTmemCycles] / ctas / 8 / 1e6, h[kStatPairBarrier] / ctas / 8 / 1e6);
  }
#endif
  tm->rec(3, st);
  MergeLaunch m{};
  m.nq = nq;
  m.nb = (int)ix->n;
  m.d = d;
  m.k = k;
  m.kprime = kp;
  m.pool_cap = P;
  m.plan = plan;
  m.pools = pools;
  m.pool_counts = counts;
  m.q_bound = qbound;
  m.q_bound_half = qbound + nq_pad;
  m.queries = q_dev;
  m.db = ix->x32;
  m.ld_db = d;
  if (ix->bf16_exact) {
    m.db16 = ix->xh;
    m.ld16 = ix->ld16;
  }
  m.out_idx = out_idx;
  m.out_dist = out_dist;
  m.status = ix->status;
  CUDA_TRY(launch_merge_rerank(m, st));
  tm->rec(4, st);
  return CURPLSH_OK;
}

size_t search_workspace_bytes(const curplsh_index* ix, int nq, int k, int form, int rerank_factor) {
  if (ix->n == 0) return 0;
  const int kp = kprime_for(form, k, rerank_factor, ix->n);
  const TuneParams tp = tune_lookup(form, ix->dim, k, nq);
  const int P = pool_capacity(kp, tp.headroom);
  FusedPlan plan;
  plan_fused(nq, (int)ix->n, ix->dres->num_sms, &plan, default_split_q4(tp, P));
  const long long nq_pad = round_up(nq, kBM);
  const size_t pool_lists = (size_t)plan.num_qblocks * kBM * plan.units_per_block;
  size_t b = 0;
  auto add = [&](size_t bytes) { b = (size_t)round_up((long long)b, 256) + bytes; };
  add((size_t)nq_pad * ix->ld16 * 2);
  if (form == kFormExact) add((size_t)nq_pad * ix->ld16 * 2);
  if (form == kFormFP8) add((size_t)nq_pad * ix->ld8);
  add(nq_pad * 4);
  add(nq_pad * 4);
  add(nq_pad * 12);
  add(pool_lists * 4);
  add(pool_lists * (size_t)P * 8);
  return (size_t)round_up((long long)b, 256) + 256;
}

int do_search(curplsh_index* ix, int64_t num, const float* queries, int k, int precision, int rerank_factor,
              int* indices, float* distances, void* stream, float* pass_ms, bool force_sync) {
  if (!ix) return set_error(CURPLSH_ERR_INVALID_ARG, "null index");
  if (num < 0) return set_error(CURPLSH_ERR_INVALID_ARG, "negative number of queries");
  if (num == 0) return CURPLSH_OK;
  if (!queries || !indices || !distances) return set_error(CURPLSH_ERR_INVALID_ARG, "null pointer argument");
  if (k < 1 || k > 1024) return set_error(CURPLSH_ERR_INVALID_ARG, "k=%d outside [1, 1024]", k);
  if (num > (int64_t)1 << 30) return set_error(CURPLSH_ERR_UNSUPPORTED, "more than 2^30 queries in one call");
  const int form = precision < 0 ? ix->cfg.precision : precision;
  if (form < 0 || form > 2) return set_error(CURPLSH_ERR_INVALID_ARG, "unknown precision %d", precision);
  const int rf = rerank_factor > 0 ? rerank_factor : ix->cfg.rerank_factor;
  std::lock_guard<std::mutex> lk(ix->mu);
  DeviceScope scope(ix->cfg.device);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ix->dres->def;
  if (!stream) {
    // The resources' default stream is non-blocking; a search on it is ordered
    // after the work already queued on the legacy default stream (where device
    // queries are commonly produced), without blocking the host.
    CUDA_TRY(cudaEventRecord(ix->order_ev, cudaStreamLegacy));
    CUDA_TRY(cudaStreamWaitEvent(st, ix->order_ev, 0));
  }
  const int nq = (int)num;
  const int dev = ix->cfg.device;
  const bool q_dev = pointer_device(queries) == dev;
  const bool i_dev = pointer_device(indices) == dev;
  const bool d_dev = pointer_device(distances) == dev;
  const bool sync = force_sync || !(q_dev && i_dev && d_dev);

  auto& slot = ix->ws[st];
  if (!slot) slot.reset(new StreamWorkspace());
  StreamWorkspace& w = *slot;
  const size_t core = search_workspace_bytes(ix, nq, k, form, rf);
  const size_t qbytes = q_dev ? 0 : (size_t)nq * ix->dim * sizeof(float);
  const size_t obytes = (i_dev && d_dev) ? 0 : (size_t)nq * k * (sizeof(int) + sizeof(float));
  const size_t total = (size_t)round_up((long long)qbytes, 256) + (size_t)round_up((long long)obytes, 256) + core;
  cudaError_t e = w.dev.ensure(total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(CURPLSH_ERR_OOM, "workspace of %zu bytes: %s", total, cudaGetErrorString(e));
  }
  CUDA_TRY(w.host.ensure(64));
  char* base = static_cast<char*>(w.dev.ptr);
  const float* qd = queries;
  int* oi = indices;
  float* od = distances;
  size_t off = 0;
  if (!q_dev) {
    qd = reinterpret_cast<const float*>(base + off);
    off += (size_t)round_up((long long)qbytes, 256);
  }
  if (!(i_dev && d_dev)) {
    oi = reinterpret_cast<int*>(base + off);
    od = reinterpret_cast<float*>(base + off + (size_t)nq * k * sizeof(int));
    off += (size_t)round_up((long long)obytes, 256);
  }
  Timing tm;
  if (pass_ms) {
    int rc = tm.create();
    if (rc) return rc;
  }
  tm.rec(0, st);
  if (!q_dev)
    CUDA_TRY(cudaMemcpyAsync(const_cast<float*>(qd), queries, qbytes, cudaMemcpyDefault, st));
  int rc = search_device(ix, nq, qd, k, form, rf, oi, od, st, w, base + off, &tm);
  if (rc) return rc;
  if (!(i_dev && d_dev)) {
    CUDA_TRY(cudaMemcpyAsync(indices, oi, (size_t)nq * k * sizeof(int), cudaMemcpyDefault, st));
    CUDA_TRY(cudaMemcpyAsync(distances, od, (size_t)nq * k * sizeof(float), cudaMemcpyDefault, st));
  }
  if (pass_ms) tm.rec(4, st);  // whole-search end (after copies)
  if (sync) {
    CUDA_TRY(cudaMemcpyAsync(w.host.ptr, ix->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    const uint32_t s = *static_cast<uint32_t*>(w.host.ptr);
    if (s) {
      cudaMemsetAsync(ix->status, 0, sizeof(uint32_t), st);
      cudaStreamSynchronize(st);
      return set_error(CURPLSH_ERR_DEVICE, "device status 0x%x (1: bounded wait expired, 2: pool overflow, 4: schedule)", s);
    }
    if (pass_ms) {
      float t = 0;
      cudaEventElapsedTime(&t, tm.ev[1], tm.ev[2]);
      pass_ms[0] = t;
      cudaEventElapsedTime(&t, tm.ev[2], tm.ev[3]);
      pass_ms[1] = t;
      cudaEventElapsedTime(&t, tm.ev[3], tm.ev[4]);
      pass_ms[2] = t;
      cudaEventElapsedTime(&t, tm.ev[0], tm.ev[4]);
      pass_ms[3] = t;
    }
  }
  return CURPLSH_OK;
}

}  // namespace

// ================================================================== internals
namespace curplsh_b200 {
int index_lock_view(curplsh_index* ix, IndexView* v) {
  if (!ix || !v) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  ix->mu.lock();
  v->device = ix->cfg.device;
  v->dim = ix->dim;
  v->precision = ix->cfg.precision;
  v->rerank_factor = ix->cfg.rerank_factor;
  v->num_sms = ix->dres->num_sms;
  v->n = ix->n;
  v->n_pad = ix->n_pad;
  v->ld16 = ix->ld16;
  v->ld8 = ix->ld8;
  v->x32 = ix->x32;
  v->xn = ix->xn;
  v->xh = ix->xh;
  v->xl = ix->xl;
  v->x8 = ix->x8;
  v->xs = ix->xs;
  v->generation = ix->generation;
  v->bf16_exact = ix->bf16_exact;
  v->stream = ix->dres->def;
  return CURPLSH_OK;
}
void index_unlock(curplsh_index* ix) { ix->mu.unlock(); }
int index_prepare_form(curplsh_index* ix, int form, IndexView* v) {
  if (form != kFormFP8 || ix->x8 || ix->n == 0) return CURPLSH_OK;
  DeviceScope scope(ix->cfg.device);
  int rc = build_fp8(ix, ix->dres->def);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(ix->dres->def));
  v->x8 = ix->x8;
  v->xs = ix->xs;
  return CURPLSH_OK;
}
int search_kprime(int form, int k, int rerank_factor, long long n) { return kprime_for(form, k, rerank_factor, n); }
int search_pool_capacity(int kprime, int headroom) { return pool_capacity(kprime, headroom); }
int record_error(int code, const char* msg) { return set_error(code, "%s", msg); }
}  // namespace curplsh_b200

// ================================================================== C ABI
extern "C" {

void curplsh_bf_config_init(curplsh_bf_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->device = 0;
  cfg->memory_space = CURPLSH_MEMORY_DEVICE;
  cfg->precision = CURPLSH_PRECISION_FP32_EXACT;
  cfg->rerank_factor = 4;
}

const char* curplsh_last_error(void) { return g_last_error.c_str(); }
const char* curplsh_version(void) { return "curplsh_b200 0.1.0 (sm_100a)"; }

int curplsh_get_num_devices(int* out) {
  if (!out) return set_error(CURPLSH_ERR_INVALID_ARG, "null out");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = 0;
    return set_error(CURPLSH_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
  }
  *out = n;
  return CURPLSH_OK;
}

int curplsh_resources_create(curplsh_resources** out) {
  if (!out) return set_error(CURPLSH_ERR_INVALID_ARG, "null out");
  *out = new (std::nothrow) curplsh_resources();
  return *out ? CURPLSH_OK : set_error(CURPLSH_ERR_OOM, "host allocation");
}

static void resources_release(curplsh_resources* r) {
  if (r->refs.fetch_sub(1) != 1) return;
  for (auto& kv : r->devs) {
    DeviceScope scope(kv.first);
    DevRes& d = kv.second;
    if (d.def_owned) cudaStreamDestroy(d.def);
    cudaStreamDestroy(d.alt[0]);
    cudaStreamDestroy(d.alt[1]);
    cudaStreamDestroy(d.copy);
  }
  delete r;
}

int curplsh_resources_destroy(curplsh_resources* r) {
  if (!r) return CURPLSH_OK;
  resources_release(r);
  return CURPLSH_OK;
}

int curplsh_resources_initialize_for_device(curplsh_resources* r, int device) {
  if (!r) return set_error(CURPLSH_ERR_INVALID_ARG, "null resources");
  DevRes* d = nullptr;
  return init_device(r, device, &d);
}

int curplsh_resources_get_default_stream(curplsh_resources* r, int device, void** stream) {
  if (!r || !stream) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  DevRes* d = nullptr;
  int rc = init_device(r, device, &d);
  if (rc) return rc;
  *stream = d->def;
  return CURPLSH_OK;
}

int curplsh_resources_set_default_stream(curplsh_resources* r, int device, void* stream) {
  if (!r) return set_error(CURPLSH_ERR_INVALID_ARG, "null resources");
  std::lock_guard<std::mutex> lk(r->mu);
  if (r->devs.count(device)) return set_error(CURPLSH_ERR_STATE, "device %d already initialised", device);
  r->user_default[device] = static_cast<cudaStream_t>(stream);
  return CURPLSH_OK;
}

int curplsh_resources_get_alternate_streams(curplsh_resources* r, int device, void** streams, int* count) {
  if (!r || !streams || !count) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  DevRes* d = nullptr;
  int rc = init_device(r, device, &d);
  if (rc) return rc;
  const int n = std::min(*count, 2);
  for (int i = 0; i < n; ++i) streams[i] = d->alt[i];
  *count = 2;
  return CURPLSH_OK;
}

int curplsh_resources_get_async_copy_stream(curplsh_resources* r, int device, void** stream) {
  if (!r || !stream) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  DevRes* d = nullptr;
  int rc = init_device(r, device, &d);
  if (rc) return rc;
  *stream = d->copy;
  return CURPLSH_OK;
}

int curplsh_resources_sync_default_stream(curplsh_resources* r, int device) {
  if (!r) return set_error(CURPLSH_ERR_INVALID_ARG, "null resources");
  DevRes* d = nullptr;
  int rc = init_device(r, device, &d);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(d->def));
  return CURPLSH_OK;
}

int curplsh_index_bf_create(curplsh_resources* r, int dim, const curplsh_bf_config* cfg, curplsh_index** out) {
  if (!r || !out) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  if (dim <= 0 || dim > 4096) return set_error(CURPLSH_ERR_INVALID_ARG, "dimension %d outside [1, 4096]", dim);
  curplsh_bf_config c;
  if (cfg)
    c = *cfg;
  else
    curplsh_bf_config_init(&c);
  if (c.memory_space != CURPLSH_MEMORY_DEVICE && c.memory_space != CURPLSH_MEMORY_UNIFIED)
    return set_error(CURPLSH_ERR_INVALID_ARG, "unknown memory space %d", c.memory_space);
  if (c.precision < 0 || c.precision > 2) return set_error(CURPLSH_ERR_INVALID_ARG, "unknown precision %d", c.precision);
  if (c.rerank_factor <= 0) c.rerank_factor = 4;
  DevRes* d = nullptr;
  int rc = init_device(r, c.device, &d);
  if (rc) return rc;
  int major = 0, minor = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, c.device));
  CUDA_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, c.device));
  if (major != 10 || minor != 0)
    return set_error(CURPLSH_ERR_UNSUPPORTED, "device %d is sm_%d%d; this build targets sm_100a (B200)", c.device, major, minor);
  auto* ix = new (std::nothrow) curplsh_index();
  if (!ix) return set_error(CURPLSH_ERR_OOM, "host allocation");
  ix->res = r;
  ix->dim = dim;
  ix->cfg = c;
  ix->dres = d;
  ix->ld16 = round_up(dim + kAugCols, 8);  // BF16 rows carry the augmented norm columns
  ix->ld8 = round_up(dim, 16);
  r->refs.fetch_add(1);
  DeviceScope scope(c.device);
  cudaError_t e = cudaMalloc(&ix->status, 2 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(ix->status, 0, 2 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ix->order_ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete ix;
    resources_release(r);
    return set_error(CURPLSH_ERR_CUDA, "status word: %s", cudaGetErrorString(e));
  }
  *out = ix;
  return CURPLSH_OK;
}

int curplsh_index_destroy(curplsh_index* ix) {
  if (!ix) return CURPLSH_OK;
  {
    DeviceScope scope(ix->cfg.device);
    cudaStreamSynchronize(ix->dres->def);
    for (auto& kv : ix->ws) {
      cudaStreamSynchronize(kv.first);
      kv.second->dev.release();
      kv.second->host.release();
    }
    ix->free_db();
    if (ix->status) cudaFree(ix->status);
    if (ix->order_ev) cudaEventDestroy(ix->order_ev);
  }
  curplsh_resources* r = ix->res;
  delete ix;
  resources_release(r);
  return CURPLSH_OK;
}

int curplsh_index_train(curplsh_index* ix, int64_t num, const float* data) {
  (void)num;
  (void)data;
  if (!ix) return set_error(CURPLSH_ERR_INVALID_ARG, "null index");
  return CURPLSH_OK;  // brute force needs no training (src/index_bf.cpp:13-15)
}

int curplsh_index_add(curplsh_index* ix, int64_t num, const float* data) {
  if (!ix) return set_error(CURPLSH_ERR_INVALID_ARG, "null index");
  if (num <= 0) return CURPLSH_OK;  // as src/index_bf.cpp:29
  if (!data) return set_error(CURPLSH_ERR_INVALID_ARG, "null data");
  if (ix->n + num > ((int64_t)1 << 31) - 1024)
    return set_error(CURPLSH_ERR_UNSUPPORTED, "more than 2^31 - 1024 rows in one index");
  std::lock_guard<std::mutex> lk(ix->mu);
  DeviceScope scope(ix->cfg.device);
  cudaStream_t st = ix->dres->def;
  const int d = ix->dim;
  const int64_t n_old = ix->n, n_new = ix->n + num;
  const long long pad_new = round_up(n_new, kBN);
  const int src_dev = pointer_device(data);
  const bool borrow = ix->cfg.borrow_device_data && src_dev == ix->cfg.device && n_old == 0;
  // Device rows are often produced just before add() by work on the legacy
  // default stream (e.g. a framework's default stream), which the index's
  // non-blocking stream does not wait for: wait for it here (add() is
  // synchronous anyway).  Work on other streams must be complete already.
  if (src_dev >= 0) CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
  // FP32 rows
  float* x32 = nullptr;
  if (borrow) {
    x32 = const_cast<float*>(data);
  } else {
    if (ix->cfg.memory_space == CURPLSH_MEMORY_UNIFIED)
      CUDA_TRY(cudaMallocManaged(&x32, (size_t)n_new * d * sizeof(float)));
    else
      CUDA_TRY(cudaMalloc(&x32, (size_t)n_new * d * sizeof(float)));
    if (n_old) CUDA_TRY(cudaMemcpyAsync(x32, ix->x32, (size_t)n_old * d * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(x32 + (size_t)n_old * d, data, (size_t)num * d * sizeof(float), cudaMemcpyDefault, st));
  }
  float* xn = nullptr;
  __nv_bfloat16 *xh = nullptr, *xl = nullptr;
  CUDA_TRY(cudaMalloc(&xn, (size_t)pad_new * sizeof(float)));
  CUDA_TRY(cudaMalloc(&xh, (size_t)pad_new * ix->ld16 * sizeof(__nv_bfloat16)));
  CUDA_TRY(cudaMalloc(&xl, (size_t)pad_new * ix->ld16 * sizeof(__nv_bfloat16)));
  // rows [0, n_old) keep their prepared copies; rows from n_old on (and padding) are prepared now
  if (n_old) {
    CUDA_TRY(cudaMemcpyAsync(xn, ix->xn, (size_t)n_old * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(xh, ix->xh, (size_t)n_old * ix->ld16 * 2, cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(xl, ix->xl, (size_t)n_old * ix->ld16 * 2, cudaMemcpyDeviceToDevice, st));
  }
  const float inf = __builtin_huge_valf();
  CUDA_TRY(launch_prep_rows(x32 + (size_t)n_old * d, d, (int)num, pad_new - n_old, d, xn + n_old, inf,
                            xh + (size_t)n_old * ix->ld16, xl + (size_t)n_old * ix->ld16, ix->ld16, nullptr,
                            nullptr, ix->ld8, st, kAugDatabase, ix->status + 1));
  uint32_t lo_flag = 1;
  CUDA_TRY(cudaMemcpyAsync(&lo_flag, ix->status + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  // swap in
  float* old_x32 = ix->x32;
  const bool old_owned = ix->x32_owned;
  ix->x32 = nullptr;
  ix->x32_owned = false;
  ix->free_db();
  if (old_owned && old_x32 && old_x32 != x32) cudaFree(old_x32);
  ix->x32 = x32;
  ix->x32_owned = !borrow;
  ix->xn = xn;
  ix->xh = xh;
  ix->xl = xl;
  ix->n = n_new;
  ix->n_pad = pad_new;
  ix->bf16_exact = lo_flag == 0;  // the flag accumulates over every add since creation or reset
  ++ix->generation;
  return CURPLSH_OK;
}

int curplsh_index_search(curplsh_index* ix, int64_t num, const float* queries, int k, int* indices,
                         float* distances) {
  return do_search(ix, num, queries, k, -1, -1, indices, distances, nullptr, nullptr, true);
}

int curplsh_index_search_ex(curplsh_index* ix, int64_t num, const float* queries, int k, int precision,
                            int rerank_factor, int* indices, float* distances, void* stream) {
  return do_search(ix, num, queries, k, precision, rerank_factor, indices, distances, stream, nullptr, false);
}

int curplsh_index_search_profiled(curplsh_index* ix, int64_t num, const float* queries, int k, int precision,
                                  int rerank_factor, int* indices, float* distances, void* stream,
                                  float* pass_ms) {
  if (!pass_ms) return set_error(CURPLSH_ERR_INVALID_ARG, "null pass_ms");
  return do_search(ix, num, queries, k, precision, rerank_factor, indices, distances, stream, pass_ms, true);
}

int curplsh_index_reset(curplsh_index* ix) {
  if (!ix) return set_error(CURPLSH_ERR_INVALID_ARG, "null index");
  std::lock_guard<std::mutex> lk(ix->mu);
  DeviceScope scope(ix->cfg.device);
  cudaStreamSynchronize(ix->dres->def);
  for (auto& kv : ix->ws) cudaStreamSynchronize(kv.first);
  ix->free_db();
  ix->bf16_exact = false;
  CUDA_TRY(cudaMemset(ix->status + 1, 0, sizeof(uint32_t)));
  ++ix->generation;
  return CURPLSH_OK;
}

int curplsh_index_get_dimension(const curplsh_index* ix, int* out) {
  if (!ix || !out) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  *out = ix->dim;
  return CURPLSH_OK;
}
int curplsh_index_get_num_data(const curplsh_index* ix, int64_t* out) {
  if (!ix || !out) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  *out = ix->n;
  return CURPLSH_OK;
}
int curplsh_index_get_device(const curplsh_index* ix, int* out) {
  if (!ix || !out) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  *out = ix->cfg.device;
  return CURPLSH_OK;
}

int curplsh_compute_l2_norm(const float* vectors, int64_t num, int dim, float* norms, int squared, void* stream) {
  if (num < 0 || dim <= 0) return set_error(CURPLSH_ERR_INVALID_ARG, "bad shape");
  if (num == 0) return CURPLSH_OK;
  if (!vectors || !norms) return set_error(CURPLSH_ERR_INVALID_ARG, "null pointer");
  CUDA_TRY(launch_l2_norms(vectors, num, dim, norms, squared, static_cast<cudaStream_t>(stream)));
  return CURPLSH_OK;
}

int curplsh_search_l2_distance(curplsh_resources* res, const float* bases, int64_t nb, const float* base_norms,
                               const float* queries, int64_t nq, int dim, int k, int* indices, float* distances,
                               int exact_distances) {
  (void)base_norms;
  if (!res) return set_error(CURPLSH_ERR_INVALID_ARG, "null resources");
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  curplsh_bf_config cfg;
  curplsh_bf_config_init(&cfg);
  cfg.device = dev;
  cfg.borrow_device_data = 1;
  curplsh_index* ix = nullptr;
  int rc = curplsh_index_bf_create(res, dim, &cfg, &ix);
  if (rc) return rc;
  rc = curplsh_index_add(ix, nb, bases);
  if (!rc) rc = curplsh_index_search(ix, nq, queries, k, indices, distances);
  if (!rc && !exact_distances && nq > 0 && nb > 0) {
    // relative form ||x||^2 - 2 q.x = exact - ||q||^2 (the reference's computeExactDistances=false)
    float* qn = nullptr;
    cudaError_t e = cudaMalloc(&qn, (size_t)nq * sizeof(float));
    if (e == cudaSuccess) e = launch_l2_norms(queries, nq, dim, qn, 1, ix->dres->def);
    std::vector<float> hq(nq), hd((size_t)nq * k);
    std::vector<int> hi((size_t)nq * k);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hq.data(), qn, nq * sizeof(float), cudaMemcpyDeviceToHost, ix->dres->def);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hd.data(), distances, hd.size() * sizeof(float), cudaMemcpyDefault, ix->dres->def);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hi.data(), indices, hi.size() * sizeof(int), cudaMemcpyDefault, ix->dres->def);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ix->dres->def);
    if (e == cudaSuccess) {
      for (int64_t q = 0; q < nq; ++q)
        for (int j = 0; j < k; ++j)
          if (hi[q * k + j] >= 0) hd[q * k + j] -= hq[q];
      e = cudaMemcpy(distances, hd.data(), hd.size() * sizeof(float), cudaMemcpyDefault);
    }
    if (qn) cudaFree(qn);
    if (e != cudaSuccess) rc = set_error(CURPLSH_ERR_CUDA, "relative distances: %s", cudaGetErrorString(e));
  }
  curplsh_index_destroy(ix);
  return rc;
}

}  // extern "C"
