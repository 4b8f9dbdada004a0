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
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <shared_mutex>
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
  explicit Carve(void* b) : base(static_cast<char*>(b)) {}  // null base: only sizes the carve
  template <class T>
  T* take(size_t count) {
    off = (size_t)round_up((long long)off, 256);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
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
  std::mutex mu;   // held for a whole search on this stream (callers sharing a stream take turns)
  DevBuf dev;      // query operands, pools, staging
  DevBuf fb;       // re-search of the queries an estimated bound failed
  PinnedBuf host;  // status read-back
};

// Library-wide switch of the sampled bound estimate (results are identical
// either way; it only changes speed).
std::atomic<int> g_bound_estimate{1};
// Library-wide switch of the coarse-margin check of the BF16/FP8 forms (a
// query whose candidates the coarse distances cannot vouch for is searched
// again in the exact form; see merge_rerank.cu).
std::atomic<int> g_coarse_check{1};
}  // namespace

struct curplsh_index {
  curplsh_resources* res = nullptr;
  int dim = 0;
  curplsh_bf_config cfg{};
  DevRes* dres = nullptr;
  // Searches hold `mu` shared (they run concurrently, each on its own stream's
  // workspace); add, reset and destroy hold it exclusively.
  std::shared_mutex mu;
  std::mutex ws_mu;   // the stream -> workspace map
  std::mutex fp8_mu;  // building the FP8 copy on first use
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
  float xs_uniform = 0.f;         // > 0: every row of the FP8 copy has this scale
  uint32_t* status = nullptr;     // device words: [0] error status, [1] nonzero if a row is not exactly BF16,
                                  // [2..3] 64-bit count of queries whose estimate failed in device-checked searches,
                                  // [4..5] range of the FP8 row scales while the copy is built
  bool bf16_exact = false;        // every stored value is exactly a BF16 value (rerank reads xh)
  long long generation = 0;       // bumped whenever the prepared database changes (add, reset)
  cudaEvent_t order_ev = nullptr; // orders default-stream searches after the legacy stream
  cudaEvent_t fp8_ev = nullptr;   // recorded after the FP8 copy is written; every FP8 reader waits on it
  std::atomic<long long> fallback_queries{0};  // queries re-searched after an estimate failed
  std::atomic<long long> coarse_queries{0};    // queries re-searched after their coarse margin failed
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
    xs_uniform = 0.f;
    n = 0;
    n_pad = 0;
  }
};

namespace {

// Builds the FP8 copy on `st` the first time a search needs it and makes `st`
// wait for it.  The copy is written asynchronously, so a reader on any other
// stream must wait on fp8_ev (recorded right after the write) before it reads
// x8/xs; searches on `st` itself are ordered by the stream.
//
// Row scales: each row's own (max |x| / 448) unless the nonzero rows' scales
// all lie within a factor kFP8UniformSpan of each other; then every row takes
// the largest.  E4M3 is a floating-point format, so a row whose own scale is
// at most 16x smaller keeps its elements in the normal range (2^-6 .. 448)
// either way, and a common scale lets the FP8 pass compare
// ||x||^2 - 2 s_q s acc without loading a scale per database row.  Deciding
// reads two words on the host once per build.
constexpr float kFP8UniformSpan = 16.f;

int build_fp8(curplsh_index* ix, cudaStream_t st) {
  if (ix->n == 0) return CURPLSH_OK;
  std::lock_guard<std::mutex> lk(ix->fp8_mu);  // concurrent searches build it once
  if (!ix->x8) {
    CUDA_TRY(cudaMalloc(&ix->x8, (size_t)ix->n_pad * ix->ld8));
    CUDA_TRY(cudaMalloc(&ix->xs, (size_t)ix->n_pad * sizeof(float)));
    CUDA_TRY(launch_prep_rows(ix->x32, ix->dim, (int)ix->n, ix->n_pad, ix->dim, nullptr, 0.f, nullptr, nullptr,
                              ix->ld16, ix->x8, ix->xs, ix->ld8, st));
    uint32_t range[2] = {0xFFFFFFFFu, 0u};
    CUDA_TRY(launch_positive_range(ix->xs, ix->n, ix->status + 4, st));
    CUDA_TRY(cudaMemcpyAsync(range, ix->status + 4, sizeof(range), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    ix->xs_uniform = 0.f;
    if (range[1] > 0u && range[0] <= range[1]) {
      float lo, hi;
      memcpy(&lo, &range[0], sizeof(float));
      memcpy(&hi, &range[1], sizeof(float));
      if (hi <= kFP8UniformSpan * lo) {
        CUDA_TRY(launch_prep_rows(ix->x32, ix->dim, (int)ix->n, ix->n_pad, ix->dim, nullptr, 0.f, nullptr, nullptr,
                                  ix->ld16, ix->x8, ix->xs, ix->ld8, st, kAugF8Database, nullptr, hi));
        ix->xs_uniform = hi;
      }
    }
    CUDA_TRY(cudaEventRecord(ix->fp8_ev, st));
    return CURPLSH_OK;
  }
  CUDA_TRY(cudaStreamWaitEvent(st, ix->fp8_ev, 0));
  return CURPLSH_OK;
}

// Candidates of a coarse form when no rerank factor is given (<= 0).
// BF16: 2k when the search is verified by the coarse-margin check (a query it
// lists is searched again exactly), else 4k.  On the integer mixture (N = 10^6,
// k = 100), 2^20 uniform rows and two BF16-valued sets, k' = 2k left no query
// short of a true neighbour and the check listed none; k' = k listed 1.7% of
// the uniform queries.  Unverified searches (batch graph, serving loop,
// allocation-free entry) keep the wider 4k margin.
// FP8: 4k and at least 480, verified or not.  E4M3's coarse error (~2% of a
// distance) needs a wider margin than BF16's (~0.4%): on the 10M-row
// unit-sphere mixture (k = 10), k' = 40 left 19 of 10,000 FP8 queries short of
// a true neighbour and the check sent 78% of them to the exact form; from
// k' = 320 up none was short, and the check sent 174 queries at 320, 36 at
// 416, 17 at 480, 1 at 640 (searches 42.8, 41.8, 41.7, 42.4 ms with the
// re-searches).  A fixed factor instead would make k' = 4800 at k = 100,
// where pools that large cost many times the pass.
constexpr long long kFP8MinCandidates = 480;

int kprime_for(int form, int k, int rerank_factor, int64_t n, bool checked) {
  long long kp;
  const int dflt = (form == kFormBF16 && checked) ? 2 : 4;
  long long want = (long long)(rerank_factor > 0 ? rerank_factor : dflt) * k;
  if (rerank_factor <= 0 && form == kFormFP8) want = std::max(want, kFP8MinCandidates);
  if (form == kFormExact)
    kp = round_up(k + 16, 32);
  else
    kp = round_up(std::max<long long>(want, k + 16), 32);
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

// ---- sampled bound estimate
// Without a bound, a candidate pool admits every row until it holds k' keys
// and then tightens as it sees more rows: about k'(1 + ln(rows / k')) rows
// per pool survive the filter, and appending and selecting survivors is most
// of the fused pass's time.  A short first pass over a strided sample of the
// database (rows 0, s, 2s, ...; same form) records, per query, the smallest
// coarse distance of every 128-row block of the sample (no pools, no
// survivors), and the j-th smallest of those B block minima becomes the
// starting bound E of every pool of the full pass.  If a fraction p of the
// database lies under a distance x, a block's minimum is under x with
// probability q(p) = 1 - (1 - p)^128, so the number of block minima under the
// query's k'-th distance is Binomial(B, q(k'/N)); j is the smallest rank whose
// upper tail is <= 1e-6, and E admits about N * (1 - (1 - j/B)^(1/128)) rows.
// E is a guess, not a bound; the merge pass checks it exactly: when at least
// k' candidates lie under the final bound, the k' nearest rows are among them
// (see merge_rerank.cu), otherwise the query is searched again without an
// estimate.  Results never depend on E.

// P(X >= j) for X ~ Binomial(n, q).
double binomial_tail(int n, double q, int j) {
  if (j <= 0) return 1.0;
  if (j > n) return 0.0;
  const double lq = std::log(q), l1q = std::log1p(-q);
  double t = 0.0;
  for (int i = j; i <= n; ++i) {
    const double term =
        std::exp(std::lgamma(n + 1.0) - std::lgamma(i + 1.0) - std::lgamma(n - i + 1.0) + i * lq + (n - i) * l1q);
    t += term;
    if (term < t * 1e-12) break;
  }
  return t;
}

// mu = expected sample rows among a query's k' nearest.  A larger sample gives
// a tighter rank (j / mu falls from ~2.6 at mu = 12 to ~2 at 24) but costs
// more; the sample pass takes at most a tenth of the full pass's tiles.
#ifndef CURPLSH_ESTIMATE_MU
#define CURPLSH_ESTIMATE_MU 12.0
#endif
constexpr double kEstimateMuMax = CURPLSH_ESTIMATE_MU;
constexpr double kEstimateMuMin = 8.0;
constexpr double kEstimateFailure = 1e-6;   // per-query failure probability for a uniform sample
constexpr int kEstimateBlockRows = kHalfN;  // rows per block minimum (one epilogue warp's half tile)

}  // namespace

namespace curplsh_b200 {
// The plan a search of this shape uses when the estimate is enabled (the
// caller reads the process-wide switch once per search).
EstimatePlan plan_estimate(int nq, long long n, int kp, int num_sms) {
  EstimatePlan e;
  if (nq < 1 || kp < 1) return e;
  if (n < (1LL << 16) || n < 64LL * kp) return e;  // a short search gains too little
  const long long T = (n + kBN - 1) / kBN;
  long long tiles = (long long)std::ceil(kEstimateMuMax * (double)n / kp / kBN);
  tiles = std::min(tiles, T / 10);
  if ((double)kp * tiles * kBN / (double)n < kEstimateMuMin) return e;  // too small a sample
  e.rows = (int)(tiles * kBN);
  e.step = (int)(n / e.rows);  // >= 10; rows j * step < n for every j < rows
  e.blocks = e.rows / kEstimateBlockRows;
  const double q0 = -std::expm1(kEstimateBlockRows * std::log1p(-(double)kp / (double)n));
  int j = 1;
  while (j < e.blocks && binomial_tail(e.blocks, q0, j) > kEstimateFailure) ++j;
  if (2 * j > e.blocks) return e;
  e.j = j;
  plan_fused(nq, e.rows, num_sms, &e.plan);
  e.on = true;
  return e;
}
bool bound_estimate_enabled() { return g_bound_estimate.load(std::memory_order_relaxed) != 0; }
}  // namespace curplsh_b200

namespace {

// Sizes and carve of one search's device workspace (search_device and
// search_workspace_bytes use the same layout).
struct SearchShape {
  int kp = 0, P = 0;
  FusedPlan plan;
  long long nq_pad = 0;
  size_t pool_lists = 0;
  EstimatePlan est;
  bool coarse = false;  // the merge checks the coarse margin (needs the failure list)
};

// Whether a search of this form checks the coarse margin (the switch is read
// once per search by the caller and passed down).
bool coarse_check_applies(const curplsh_index* ix, int form, int kp, bool enabled) {
  return enabled && form != kFormExact && ix->n > 0 && kp < ix->n;
}

SearchShape search_shape(const curplsh_index* ix, int nq, int k, int form, int rerank_factor, bool allow_est,
                         bool coarse_on) {
  SearchShape sh;
  sh.kp = kprime_for(form, k, rerank_factor, ix->n, coarse_on);
  const TuneParams tp = tune_lookup(form, ix->dim, k, nq);
  sh.P = pool_capacity(sh.kp, tp.headroom);
  plan_fused(nq, (int)ix->n, ix->dres->num_sms, &sh.plan, default_split_q4(tp, sh.P), form, ix->dim);
  sh.nq_pad = round_up(nq, kBM);
  sh.pool_lists = (size_t)sh.plan.pool_rows() * sh.plan.units_per_block;
  if (allow_est) sh.est = plan_estimate(nq, ix->n, sh.kp, ix->dres->num_sms);
  sh.coarse = coarse_check_applies(ix, form, sh.kp, coarse_on);
  return sh;
}

struct SearchBufs {
  __nv_bfloat16 *qh = nullptr, *ql = nullptr;
  uint8_t* q8 = nullptr;
  float *qn = nullptr, *qs = nullptr;
  uint32_t* qbound = nullptr;   // [nq_pad] bounds of the full pass
  float* minima = nullptr;      // [nq_pad][B] block minima of the sample pass
  int* fail = nullptr;          // [2 + nq]: count, coarse-check count, then query indices
  int* counts = nullptr;
  uint64_t* pools = nullptr;
};

size_t carve_search(Carve& c, const curplsh_index* ix, const SearchShape& sh, int nq, int form, SearchBufs* b) {
  b->qh = c.take<__nv_bfloat16>((size_t)sh.nq_pad * ix->ld16);
  if (form == kFormExact) b->ql = c.take<__nv_bfloat16>((size_t)sh.nq_pad * ix->ld16);
  if (form == kFormFP8) b->q8 = c.take<uint8_t>((size_t)sh.nq_pad * ix->ld8);
  b->qn = c.take<float>(sh.nq_pad);
  b->qs = c.take<float>(sh.nq_pad);
  b->qbound = c.take<uint32_t>(sh.nq_pad);
  if (sh.est.on) b->minima = c.take<float>((size_t)sh.nq_pad * sh.est.blocks);
  if (sh.est.on || sh.coarse) b->fail = c.take<int>(2 + (size_t)nq);
  b->counts = c.take<int>(sh.pool_lists);
  b->pools = c.take<uint64_t>(sh.pool_lists * (size_t)sh.P);
  return (size_t)round_up((long long)c.off, 256);
}

#ifdef CURPLSH_FUSED_STATS
// Instrumented builds: per-role cycle counters of a fused launch, printed to stderr.
cudaError_t fused_stats_begin(FusedLaunch* f, cudaStream_t st) {
  static unsigned long long* stats = nullptr;
  if (!stats) {
    cudaError_t e = cudaMalloc(&stats, kStatCount * sizeof(unsigned long long));
    if (e != cudaSuccess) return e;
  }
  f->stats = stats;
  return cudaMemsetAsync(stats, 0, kStatCount * sizeof(unsigned long long), st);
}

cudaError_t fused_stats_print(const char* label, const FusedLaunch& f, cudaStream_t st) {
  unsigned long long h[kStatCount];
  cudaError_t e = cudaMemcpyAsync(h, f.stats, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  const FusedPlan& plan = f.plan;
  const double ctas = (double)plan.grid;
  fprintf(stderr,
          "[fused-stats %s] grid %d kp %d P %d | per CTA (Mcycles): total %.2f prod_wait_empty %.2f mma_wait_full "
          "%.2f mma_wait_acc %.2f | per epi warp: wait_acc %.2f filter %.2f refresh %.2f | refreshes %llu survivors "
          "%llu\n",
          label, plan.grid, f.kprime, f.pool_cap, h[kStatCtaCycles] / ctas / 1e6, h[kStatProducerWaitEmpty] / ctas / 1e6,
          h[kStatMmaWaitFull] / ctas / 1e6, h[kStatMmaWaitAccEmpty] / ctas / 1e6, h[kStatEpiWaitAccFull] / ctas / 8 / 1e6,
          h[kStatEpiFilter] / ctas / 8 / 1e6, h[kStatEpiRefresh] / ctas / 8 / 1e6, h[kStatRefreshes],
          h[kStatSurvivors]);
  fprintf(stderr,
          "[fused-stats2 %s] radix passes/refresh %.2f | slow chunks %llu (%.1f%% of warp-chunks) | loop iters/slow "
          "chunk %.2f | tmem Mcycles/warp %.2f | pair barriers Mcycles/warp %.2f\n",
          label, h[kStatRefreshes] ? (double)h[kStatRadixPasses] / h[kStatRefreshes] : 0.0, h[kStatSlowChunks],
          100.0 * h[kStatSlowChunks] / (ctas * 8 * (double)plan.work_per_cta * 4),
          h[kStatSlowChunks] ? (double)h[kStatLoopIters] / h[kStatSlowChunks] : 0.0,
          h[kStatTmemCycles] / ctas / 8 / 1e6, h[kStatPairBarrier] / ctas / 8 / 1e6);
  return cudaSuccess;
}
#endif

// The search proper.  Device-side inputs/outputs; `st` orders everything.
// With `allow_est` a sampled bound estimate may be used, with `coarse_on` the
// BF16/FP8 forms check their coarse margin; when either applies, *fail_out
// points at the device list of queries that failed a check ([0] count, then
// indices), which the caller must search again (else *fail_out is null).
// With `dev_recheck` (and no coarse check) a failed estimate is handled on the
// stream instead: when the merge lists any query, the full pass and the merge
// run again from no bound for the whole batch (rare: the estimate fails with
// probability ~1e-6 per query), the failures are counted on the device, and
// *fail_out stays null, so the caller need not synchronise.
int search_device(curplsh_index* ix, int nq, const float* q_dev, int k, int form, int rerank_factor, int* out_idx,
                  float* out_dist, cudaStream_t st, char* extra_base, Timing* tm, bool allow_est, bool coarse_on,
                  int** fail_out, bool dev_recheck) {
  const int d = ix->dim;
  *fail_out = nullptr;
  if (ix->n == 0) {
    CUDA_TRY(launch_fill_results(out_idx, out_dist, (long long)nq * k, st));
    return CURPLSH_OK;
  }
  if (form == kFormFP8) {
    int rc = build_fp8(ix, st);
    if (rc) return rc;
  }
  const SearchShape sh = search_shape(ix, nq, k, form, rerank_factor, allow_est, coarse_on);
  const int kp = sh.kp, P = sh.P;
  const FusedPlan& plan = sh.plan;
  const long long nq_pad = sh.nq_pad;
  Carve c(extra_base);
  SearchBufs b;
  carve_search(c, ix, sh, nq, form, &b);

  tm->rec(1, st);
  CUDA_TRY(launch_prep_rows(q_dev, d, nq, nq_pad, d, b.qn, 0.f, form == kFormFP8 ? nullptr : b.qh, b.ql, ix->ld16,
                            b.q8, b.qs, ix->ld8, st, form == kFormFP8 ? kAugF8Query : kAugQuery));
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
  f.qh = b.qh;
  f.ql = b.ql;
  f.q8 = b.q8;
  f.qn = b.qn;
  f.qs = b.qs;
  f.xh = ix->xh;
  f.xl = ix->xl;
  f.x8 = ix->x8;
  f.xn = ix->xn;
  f.xs = ix->xs;
  f.xs_uniform = ix->xs_uniform;
  f.pools = b.pools;
  f.pool_counts = b.counts;
  f.q_bound = b.qbound;
  f.status = ix->status;
  f.plan = plan;
  if (sh.est.on) {
    // sample pass over rows 0, step, 2 step, ...: block minima, no pools
    FusedLaunch e = f;
    e.nb = sh.est.rows;
    e.nb_pad = sh.est.rows;
    e.db_step = sh.est.step;
    e.kprime = 1;
    e.minima = b.minima;
    e.plan = sh.est.plan;
#ifdef CURPLSH_FUSED_STATS
    CUDA_TRY(fused_stats_begin(&e, st));
#endif
    CUDA_TRY(launch_fused(e, st));
#ifdef CURPLSH_FUSED_STATS
    CUDA_TRY(fused_stats_print("sample", e, st));
#endif
    // the j-th smallest block minimum of every query becomes its starting bound
    CUDA_TRY(launch_estimate_select(b.minima, sh.est.blocks, nq, sh.est.j, b.qbound, st));
  } else {
    CUDA_TRY(cudaMemsetAsync(b.qbound, 0xFF, (size_t)nq_pad * sizeof(uint32_t), st));
  }
  if (b.fail) CUDA_TRY(cudaMemsetAsync(b.fail, 0, 2 * sizeof(int), st));
  tm->rec(2, st);
#ifdef CURPLSH_FUSED_STATS
  CUDA_TRY(fused_stats_begin(&f, st));
#endif
  CUDA_TRY(launch_fused(f, st));
#ifdef CURPLSH_FUSED_STATS
  CUDA_TRY(fused_stats_print("full", f, st));
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
  m.pools = b.pools;
  m.pool_counts = b.counts;
  m.q_bound = b.qbound;
  m.checks = (sh.est.on ? kCheckEstimate : 0) | (sh.coarse ? kCheckCoarse : 0);
  if (m.checks) {
    m.fail_count = b.fail;
    m.coarse_count = b.fail + 1;
    m.fail_list = b.fail + 2;
  }
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
  if (dev_recheck && m.checks == kCheckEstimate) {
    CUDA_TRY(launch_fill_u32_if(b.qbound, nq_pad, 0xFFFFFFFFu, b.fail, st));
    FusedLaunch f2 = f;
    f2.run_if = b.fail;
    CUDA_TRY(launch_fused(f2, st));
    MergeLaunch m2 = m;
    m2.checks = 0;
    m2.fail_count = nullptr;
    m2.coarse_count = nullptr;
    m2.fail_list = nullptr;
    m2.run_if = b.fail;
    CUDA_TRY(launch_merge_rerank(m2, st));
    CUDA_TRY(launch_add_count(reinterpret_cast<unsigned long long*>(ix->status + 2), b.fail, st));
    tm->rec(4, st);
    return CURPLSH_OK;
  }
  tm->rec(4, st);
  if (m.checks) *fail_out = b.fail;
  return CURPLSH_OK;
}

size_t search_workspace_bytes(const curplsh_index* ix, int nq, int k, int form, int rerank_factor,
                              bool allow_est, bool coarse_on) {
  if (ix->n == 0) return 0;
  const SearchShape sh = search_shape(ix, nq, k, form, rerank_factor, allow_est, coarse_on);
  Carve c(nullptr);
  SearchBufs b;
  return carve_search(c, ix, sh, nq, form, &b) + 256;
}

// Searches again the `nf` queries listed at fail_dev + 2 (device) -- in the
// exact form, without an estimate, so no check applies -- and writes their
// results into the full result arrays.
int search_failed(curplsh_index* ix, int nf, const int* fail_dev, const float* q_dev, int k, int rerank_factor,
                  int* out_idx, float* out_dist, cudaStream_t st, StreamWorkspace& w) {
  const int d = ix->dim;
  const int form = kFormExact;
  const size_t qbytes = (size_t)round_up((long long)nf * d * sizeof(float), 256);
  const size_t obytes = (size_t)round_up((long long)nf * k * (sizeof(int) + sizeof(float)), 256);
  const size_t core = search_workspace_bytes(ix, nf, k, form, rerank_factor, false, false);
  cudaError_t e = w.fb.ensure(qbytes + obytes + core);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(CURPLSH_ERR_OOM, "re-search workspace of %zu bytes: %s", qbytes + obytes + core,
                     cudaGetErrorString(e));
  }
  char* base = static_cast<char*>(w.fb.ptr);
  float* qf = reinterpret_cast<float*>(base);
  int* oif = reinterpret_cast<int*>(base + qbytes);
  float* odf = reinterpret_cast<float*>(base + qbytes + (size_t)nf * k * sizeof(int));
  CUDA_TRY(launch_gather_rows(q_dev, d, fail_dev + 2, nf, qf, st));
  Timing none;
  int* again = nullptr;
  int rc = search_device(ix, nf, qf, k, form, rerank_factor, oif, odf, st, base + qbytes + obytes, &none, false,
                         false, &again, false);
  if (rc) return rc;
  CUDA_TRY(launch_scatter_results(oif, odf, fail_dev + 2, nf, k, out_idx, out_dist, st));
  return CURPLSH_OK;
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
  std::shared_lock<std::shared_mutex> lk(ix->mu);
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
  // A search that starts from an estimated bound must check it (a failed
  // query is searched again).  With the caller's buffers on the device and no
  // coarse check, the check runs on the stream (search_device) and the call
  // stays asynchronous; otherwise the host checks it and searches the failed
  // queries again before returning.  The switches are read once here: planning
  // and the checks below agree.  The coarse-margin check of the BF16/FP8 forms
  // is always the host's: a query it lists is searched again in the exact form
  // before the call returns.
  const bool coarse_on = g_coarse_check.load(std::memory_order_relaxed) != 0;
  const int kp = ix->n > 0 ? kprime_for(form, k, rf, ix->n, coarse_on) : 0;
  const bool est = g_bound_estimate.load(std::memory_order_relaxed) && ix->n > 0 &&
                   plan_estimate(nq, ix->n, kp, ix->dres->num_sms).on;
  const bool coarse = coarse_check_applies(ix, form, kp, coarse_on);
  const bool all_dev = q_dev && i_dev && d_dev;
  const bool dev_recheck = est && !coarse && all_dev && !force_sync;
  const bool sync = force_sync || (est && !dev_recheck) || coarse || !all_dev;

  StreamWorkspace* wp;
  {
    std::lock_guard<std::mutex> wl(ix->ws_mu);
    auto& slot = ix->ws[st];
    if (!slot) slot.reset(new StreamWorkspace());
    wp = slot.get();
  }
  StreamWorkspace& w = *wp;
  std::lock_guard<std::mutex> wlk(w.mu);
  const size_t core = search_workspace_bytes(ix, nq, k, form, rf, est, coarse);
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
  int* fail = nullptr;
  int rc = search_device(ix, nq, qd, k, form, rf, oi, od, st, base + off, &tm, est, coarse, &fail, dev_recheck);
  if (rc) return rc;
  auto copy_out = [&]() -> int {
    if (!(i_dev && d_dev)) {
      CUDA_TRY(cudaMemcpyAsync(indices, oi, (size_t)nq * k * sizeof(int), cudaMemcpyDefault, st));
      CUDA_TRY(cudaMemcpyAsync(distances, od, (size_t)nq * k * sizeof(float), cudaMemcpyDefault, st));
    }
    return CURPLSH_OK;
  };
  rc = copy_out();
  if (rc) return rc;
  if (pass_ms) tm.rec(4, st);  // whole-search end (after copies)
  if (sync) {
    uint32_t* hw = static_cast<uint32_t*>(w.host.ptr);
    hw[1] = hw[2] = 0;
    CUDA_TRY(cudaMemcpyAsync(hw, ix->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    if (fail) CUDA_TRY(cudaMemcpyAsync(hw + 1, fail, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    uint32_t s = hw[0];
    const int nf = (int)hw[1], nc = (int)hw[2];
    if (!s && nf > 0) {
      ix->fallback_queries.fetch_add(nf - nc, std::memory_order_relaxed);
      ix->coarse_queries.fetch_add(nc, std::memory_order_relaxed);
      // queries whose estimated bound was too small, or whose coarse margin
      // failed: search them again in the exact form
      rc = search_failed(ix, nf, fail, qd, k, rf, oi, od, st, w);
      if (rc) return rc;
      rc = copy_out();
      if (rc) return rc;
      if (pass_ms) tm.rec(4, st);
      CUDA_TRY(cudaMemcpyAsync(hw, ix->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      CUDA_TRY(cudaStreamSynchronize(st));
      s = hw[0];
    }
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
  ix->mu.lock_shared();
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
  v->xs_uniform = ix->xs_uniform;
  v->generation = ix->generation;
  v->bf16_exact = ix->bf16_exact;
  v->stream = ix->dres->def;
  v->fp8_ready = ix->fp8_ev;
  return CURPLSH_OK;
}
void index_unlock(curplsh_index* ix) { ix->mu.unlock_shared(); }
int index_prepare_form(curplsh_index* ix, int form, IndexView* v) {
  if (form != kFormFP8 || ix->x8 || ix->n == 0) return CURPLSH_OK;
  DeviceScope scope(ix->cfg.device);
  int rc = build_fp8(ix, ix->dres->def);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(ix->dres->def));
  v->x8 = ix->x8;
  v->xs = ix->xs;
  v->xs_uniform = ix->xs_uniform;
  return CURPLSH_OK;
}
int search_kprime(int form, int k, int rerank_factor, long long n) {
  return kprime_for(form, k, rerank_factor, n, false);
}
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
  cfg->rerank_factor = 0;  // the form's default: k' = 4k (FP8: at least 320)
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
  if (c.rerank_factor < 0) c.rerank_factor = 0;  // 0: the form's default
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
  // FP8 rows: the codes, then, when round_up(d, 32) leaves 32 bytes of the
  // last 128-byte K chunk free, the BF16 norm tail there
  ix->ld8 = (round_up(dim, 32) % 128 != 0) ? round_up(dim, 32) + 32 : round_up(dim, 16);
  r->refs.fetch_add(1);
  DeviceScope scope(c.device);
  cudaError_t e = cudaMalloc(&ix->status, 6 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(ix->status, 0, 6 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ix->order_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ix->fp8_ev, cudaEventDisableTiming);
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
    if (ix->fp8_ev) cudaEventDestroy(ix->fp8_ev);
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
  std::unique_lock<std::shared_mutex> lk(ix->mu);
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
  std::unique_lock<std::shared_mutex> lk(ix->mu);
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
int curplsh_set_bound_estimate(int enabled) {
  g_bound_estimate.store(enabled ? 1 : 0, std::memory_order_relaxed);
  return CURPLSH_OK;
}

int curplsh_get_bound_estimate(int* enabled) {
  if (!enabled) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  *enabled = g_bound_estimate.load(std::memory_order_relaxed);
  return CURPLSH_OK;
}

int curplsh_set_coarse_check(int enabled) {
  g_coarse_check.store(enabled ? 1 : 0, std::memory_order_relaxed);
  return CURPLSH_OK;
}

int curplsh_get_coarse_check(int* enabled) {
  if (!enabled) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  *enabled = g_coarse_check.load(std::memory_order_relaxed);
  return CURPLSH_OK;
}

int curplsh_set_cta_pairs(int enabled) {
  if (enabled < 0 || enabled > kPairsAuto) return set_error(CURPLSH_ERR_INVALID_ARG, "CTA pairs mode must be 0, 1 or 2");
  set_cta_pairs(enabled);
  return CURPLSH_OK;
}

int curplsh_get_cta_pairs(int* enabled) {
  if (!enabled) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  *enabled = get_cta_pairs();
  return CURPLSH_OK;
}

int curplsh_set_dual_blocks(int enabled) {
  set_dual_blocks(enabled);
  return CURPLSH_OK;
}

int curplsh_get_dual_blocks(int* enabled) {
  if (!enabled) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  *enabled = get_dual_blocks();
  return CURPLSH_OK;
}

int curplsh_index_estimate_plan(curplsh_index* ix, int64_t num, int k, int precision, int rerank_factor,
                                int* sample_rows, int* step, int* rank) {
  if (!ix || !sample_rows || !step || !rank) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  if (k < 1 || k > 1024 || num < 0 || num > (int64_t)1 << 30)
    return set_error(CURPLSH_ERR_INVALID_ARG, "bad k or number of queries");
  const int form = precision < 0 ? ix->cfg.precision : precision;
  if (form < 0 || form > 2) return set_error(CURPLSH_ERR_INVALID_ARG, "unknown precision %d", precision);
  const int rf = rerank_factor > 0 ? rerank_factor : ix->cfg.rerank_factor;
  std::shared_lock<std::shared_mutex> lk(ix->mu);
  *sample_rows = 0;
  *step = 1;
  *rank = 0;
  if (ix->n == 0 || !g_bound_estimate.load(std::memory_order_relaxed)) return CURPLSH_OK;
  const bool coarse_on = g_coarse_check.load(std::memory_order_relaxed) != 0;
  const EstimatePlan e = plan_estimate((int)num, ix->n, kprime_for(form, k, rf, ix->n, coarse_on), ix->dres->num_sms);
  if (e.on) {
    *sample_rows = e.rows;
    *step = e.step;
    *rank = e.j;
  }
  return CURPLSH_OK;
}

int curplsh_estimate_plan_shape(int64_t num_rows, int64_t num_queries, int kprime, int num_sms, int* sample_rows,
                                int* step, int* rank) {
  if (!sample_rows || !step || !rank) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  if (num_rows < 0 || num_rows > INT32_MAX || num_queries < 0 || num_queries > (int64_t)1 << 30 || kprime < 0 ||
      num_sms < 1)
    return set_error(CURPLSH_ERR_INVALID_ARG, "bad shape");
  *sample_rows = 0;
  *step = 1;
  *rank = 0;
  const EstimatePlan e = plan_estimate((int)num_queries, num_rows, kprime, num_sms);
  if (e.on) {
    *sample_rows = e.rows;
    *step = e.step;
    *rank = e.j;
  }
  return CURPLSH_OK;
}

int curplsh_index_get_fallback_count(curplsh_index* ix, int64_t* count) {
  if (!ix || !count) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  // searches checked on the host count there; searches checked on their stream
  // count on the device (read after everything queued so far has run)
  DeviceScope scope(ix->cfg.device);
  unsigned long long dev = 0;
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(&dev, ix->status + 2, sizeof(dev), cudaMemcpyDeviceToHost));
  *count = ix->fallback_queries.load(std::memory_order_relaxed) + (int64_t)dev;
  return CURPLSH_OK;
}

int curplsh_index_get_coarse_fallback_count(curplsh_index* ix, int64_t* count) {
  if (!ix || !count) return set_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  *count = ix->coarse_queries.load(std::memory_order_relaxed);
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
