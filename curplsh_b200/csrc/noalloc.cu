// noalloc.cu -- a search entry point that allocates no memory.
//
// Why it exists: some callers cannot allocate device memory while they serve
// queries.  Typical cases are a process whose device memory is already owned
// by another allocator (a framework's caching pool that has reserved the GPU),
// and latency-critical loops where cudaMalloc / cudaFree are off limits because
// they synchronise the whole device and stall unrelated streams.  The regular
// search grows a per-stream workspace with cudaMalloc on demand; this variant
// instead runs the same three passes (query prep, fused tensor-core filter,
// merge + exact rerank) out of one fixed scratch array that lives in the
// library's device image.
//
// The scratch: `g_noalloc_scratch`, kNoAllocScratchBytes (64 MiB) per GPU.  It
// belongs to this file's device module, so every GPU on which the module is
// loaded holds it until the process exits; with CUDA's default lazy module
// loading that happens at the first call of this entry point on that device.
// Host code cannot use the array's name as a device address (in host code it
// names a host-side shadow), so each device's address is looked up once with
// cudaGetSymbolAddress, with that device current, during the first call on it.
// That first call should therefore come before any stream capture.
//
// Every call on a device shares the array, and the array keeps whatever the
// last call left in it; everything a call needs zeroed (the device status word,
// the per-query bounds) is cleared by that call with cudaMemsetAsync.  Calls
// whose GPU work overlapped would race on the array; this entry point therefore
// takes a per-device lock and waits for its GPU work before returning, so two
// of its calls never overlap.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/curplsh_b200.h"
#include "common.cuh"
#include "fused_knn.h"

namespace curplsh_b200 {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB per GPU

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
std::mutex g_device_mu[kMaxDevices];
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on `dev` (which must be current);
// looked up once per device.
int scratch_address(int dev, void** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      char msg[256];
      snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the no-alloc scratch on device %d: %s", dev,
               cudaGetErrorString(e));
      return record_error(CURPLSH_ERR_CUDA, msg);
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return CURPLSH_OK;
}

bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

long long rup(long long x, long long m) { return (x + m - 1) / m * m; }

struct Layout {
  size_t status, qh, ql, q8, qn, qs, qbound, counts, pools, total;
};

Layout carve(int form, long long nq_pad, long long ld16, long long ld8, size_t pool_lists, int P) {
  Layout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    off = (size_t)rup((long long)off, 256);
    const size_t at = off;
    off += bytes;
    return at;
  };
  L.status = take(sizeof(uint32_t));
  L.qh = take((size_t)nq_pad * ld16 * 2);
  L.ql = form == kFormExact ? take((size_t)nq_pad * ld16 * 2) : 0;
  L.q8 = form == kFormFP8 ? take((size_t)nq_pad * ld8) : 0;
  L.qn = take((size_t)nq_pad * 4);
  L.qs = take((size_t)nq_pad * 4);
  L.qbound = take((size_t)nq_pad * 4);  // k'-th bounds
  L.counts = take(pool_lists * 4);
  L.pools = take(pool_lists * (size_t)P * 8);
  L.total = off;
  return L;
}

struct DeviceRestore {
  int prev = -1;
  explicit DeviceRestore(int dev) {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) {
      prev = cur;
      cudaSetDevice(dev);
    }
  }
  ~DeviceRestore() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

#define NA_TRY(call)                                                                  \
  do {                                                                                \
    const cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                          \
      char m_[256];                                                                   \
      snprintf(m_, sizeof(m_), "%s: %s", #call, cudaGetErrorString(e_));              \
      return record_error(CURPLSH_ERR_CUDA, m_);                                      \
    }                                                                                 \
  } while (0)

int search_noalloc_locked(const IndexView& v, int nq, const float* q, int k, int* out_idx, float* out_dist,
                          cudaStream_t st) {
  if (v.n == 0) {
    NA_TRY(launch_fill_results(out_idx, out_dist, (long long)nq * k, st));
    return CURPLSH_OK;
  }
  const int form = v.precision;
  if (form == kFormFP8 && !v.x8)
    return record_error(CURPLSH_ERR_STATE,
                        "curplsh_index_search_noalloc: this index has no FP8 copy yet (it is built by the "
                        "index's first regular FP8 search)");
  void* base = nullptr;
  int rc = scratch_address(v.device, &base);
  if (rc) return rc;
  const int kp = search_kprime(form, k, v.rerank_factor, v.n);
  const int P = search_pool_capacity(kp);
  const long long nq_pad = rup(nq, kBM);
  // Widest schedule whose candidate pools fit the scratch (the result does not
  // depend on the schedule, only the speed does).
  FusedPlan plan{};
  Layout L{};
  int cap = v.num_sms;
  for (;;) {
    plan_fused(nq, (int)v.n, cap, &plan, 4, form, v.dim);
    const size_t lists = (size_t)plan.pool_rows() * plan.units_per_block;
    L = carve(form, nq_pad, v.ld16, v.ld8, lists, P);
    if (L.total <= kNoAllocScratchBytes || cap == 1) break;
    cap = cap * 3 / 4 > 1 ? cap * 3 / 4 : 1;
  }
  if (L.total > kNoAllocScratchBytes) {
    char m[320];
    snprintf(m, sizeof(m),
             "curplsh_index_search_noalloc: %d queries with k=%d need %zu bytes of scratch, more than the fixed "
             "%zu-byte (64 MiB) scratch; use fewer queries per call or the regular search",
             nq, k, L.total, kNoAllocScratchBytes);
    return record_error(CURPLSH_ERR_INVALID_ARG, m);
  }
  char* b = static_cast<char*>(base);
  uint32_t* status = reinterpret_cast<uint32_t*>(b + L.status);
  __nv_bfloat16* qh = reinterpret_cast<__nv_bfloat16*>(b + L.qh);
  __nv_bfloat16* ql = form == kFormExact ? reinterpret_cast<__nv_bfloat16*>(b + L.ql) : nullptr;
  uint8_t* q8 = form == kFormFP8 ? reinterpret_cast<uint8_t*>(b + L.q8) : nullptr;
  float* qn = reinterpret_cast<float*>(b + L.qn);
  float* qs = reinterpret_cast<float*>(b + L.qs);
  uint32_t* qbound = reinterpret_cast<uint32_t*>(b + L.qbound);
  int* counts = reinterpret_cast<int*>(b + L.counts);
  uint64_t* pools = reinterpret_cast<uint64_t*>(b + L.pools);

  // From the first enqueue on, an early return (a failed launch or copy) must
  // not release the device lock while work that uses the scratch may still be
  // in flight on `st`: the guard waits for the stream on every return path.
  struct DrainOnReturn {
    cudaStream_t st;
    ~DrainOnReturn() { cudaStreamSynchronize(st); }
  } drain{st};
  // The FP8 copy is written asynchronously by the index's first regular FP8
  // search, possibly on another stream: order this call after that write.
  if (form == kFormFP8 && v.fp8_ready) NA_TRY(cudaStreamWaitEvent(st, v.fp8_ready, 0));
  // state that must start cleared on every call (the array keeps the last call's contents)
  NA_TRY(cudaMemsetAsync(status, 0, sizeof(uint32_t), st));
  NA_TRY(cudaMemsetAsync(qbound, 0xFF, (size_t)nq_pad * sizeof(uint32_t), st));
  NA_TRY(launch_prep_rows(q, v.dim, nq, nq_pad, v.dim, qn, 0.f, form == kFormFP8 ? nullptr : qh, ql, v.ld16, q8,
                          qs, v.ld8, st, form == kFormFP8 ? kAugF8Query : kAugQuery));
  FusedLaunch f{};
  f.nq = nq;
  f.nb = (int)v.n;
  f.d = v.dim;
  f.kprime = kp;
  f.pool_cap = P;
  f.form = form;
  f.nq_pad = nq_pad;
  f.nb_pad = v.n_pad;
  f.ld16 = v.ld16;
  f.ld8 = v.ld8;
  f.qh = qh;
  f.ql = ql;
  f.q8 = q8;
  f.qn = qn;
  f.qs = qs;
  f.xh = v.xh;
  f.xl = v.xl;
  f.x8 = v.x8;
  f.xn = v.xn;
  f.xs = v.xs;
  f.xs_uniform = v.xs_uniform;
  f.pools = pools;
  f.pool_counts = counts;
  f.q_bound = qbound;
  f.status = status;
  f.plan = plan;
  NA_TRY(launch_fused(f, st));
  MergeLaunch m{};
  m.nq = nq;
  m.nb = (int)v.n;
  m.d = v.dim;
  m.k = k;
  m.kprime = kp;
  m.pool_cap = P;
  m.plan = plan;
  m.pools = pools;
  m.pool_counts = counts;
  m.q_bound = qbound;
  m.queries = q;
  m.db = v.x32;
  m.ld_db = v.dim;
  m.out_idx = out_idx;
  m.out_dist = out_dist;
  if (v.bf16_exact) {
    m.db16 = v.xh;
    m.ld16 = v.ld16;
  }
  m.status = status;
  NA_TRY(launch_merge_rerank(m, st));
  uint32_t host_status = 0;
  NA_TRY(cudaMemcpyAsync(&host_status, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  NA_TRY(cudaStreamSynchronize(st));
  if (host_status) {
    char msg[160];
    snprintf(msg, sizeof(msg), "curplsh_index_search_noalloc: device status 0x%x", host_status);
    return record_error(CURPLSH_ERR_DEVICE, msg);
  }
  return CURPLSH_OK;
}

}  // namespace
}  // namespace curplsh_b200

using namespace curplsh_b200;

extern "C" int curplsh_index_search_noalloc(curplsh_index* index, int64_t num, const float* queries, int k,
                                            int* indices, float* distances, void* stream) {
  if (!index) return record_error(CURPLSH_ERR_INVALID_ARG, "curplsh_index_search_noalloc: null index");
  if (num < 0) return record_error(CURPLSH_ERR_INVALID_ARG, "curplsh_index_search_noalloc: negative num");
  if (num == 0) return CURPLSH_OK;
  if (!queries || !indices || !distances)
    return record_error(CURPLSH_ERR_INVALID_ARG, "curplsh_index_search_noalloc: null pointer argument");
  if (k < 1 || k > 1024) return record_error(CURPLSH_ERR_INVALID_ARG, "curplsh_index_search_noalloc: k outside [1, 1024]");
  if (num > (int64_t)1 << 30)
    return record_error(CURPLSH_ERR_INVALID_ARG, "curplsh_index_search_noalloc: too many queries");
  IndexView v{};
  int rc = index_lock_view(index, &v);
  if (rc) return rc;
  if (v.device < 0 || v.device >= kMaxDevices) {
    index_unlock(index);
    return record_error(CURPLSH_ERR_UNSUPPORTED, "curplsh_index_search_noalloc: device ordinal too large");
  }
  {
    std::lock_guard<std::mutex> dev_lock(g_device_mu[v.device]);
    DeviceRestore scope(v.device);
    if (!on_device(queries, v.device) || !on_device(indices, v.device) || !on_device(distances, v.device)) {
      rc = record_error(CURPLSH_ERR_INVALID_ARG,
                        "curplsh_index_search_noalloc: queries, indices and distances must be device memory of "
                        "the index's device (no staging buffers are allocated)");
    } else {
      rc = search_noalloc_locked(v, (int)num, queries, k, indices, distances, static_cast<cudaStream_t>(stream));
    }
  }
  index_unlock(index);
  return rc;
}
