// batch.cpp -- batched search over several indexes as one captured CUDA graph.
//
// No counterpart in cuRPLSH: its IndexBF::search (src/index_bf.cpp:46-74)
// serves one query matrix against one index per call, each call paying its
// own launches and a device synchronisation (src/internal/search.cu:79-216).
//
// Plan (once per batch, and again when an index changes): MultiPlan
// (multi_plan.h) -- requests against one index with one (form, k') share
// query blocks, one prep / fused / merge chain per (form, d) group -- with the
// groups as parallel branches of the graph; each fused launch asks for every
// SM, so a group's tail overlaps the next group's start; items too small to
// spread over many CTAs of a combined launch get launches of their own.
// Run: one cudaGraphLaunch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/curplsh_b200.h"
#include "common.cuh"
#include "fused_knn.h"
#include "multi_plan.h"

using namespace curplsh_b200;

namespace {

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return record_error(code, buf);
}

#define BT_TRY(call)                                                                                  \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) {                                                                          \
      cudaGetLastError();                                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? CURPLSH_ERR_OOM : CURPLSH_ERR_CUDA, "%s: %s", #call, \
                  cudaGetErrorString(e_));                                                            \
    }                                                                                                 \
  } while (0)

bool is_device_ptr(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

}  // namespace

struct curplsh_batch {
  std::vector<curplsh_batch_item> items;
  int precision = -1, rerank_factor = 0;
  int device = 0;
  std::vector<curplsh_index*> uniq;  // sorted by address (lock order)
  std::vector<IndexView> views;
  std::vector<long long> gens;
  MultiPlan plan;
  std::vector<cudaStream_t> branches;  // one per (form, d) group
  std::vector<cudaEvent_t> joins;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  uint32_t* status = nullptr;
  uint32_t* host_status = nullptr;
  cudaStream_t cap = nullptr;
  cudaEvent_t fork = nullptr;
  cudaEvent_t order_ev = nullptr;  // orders NULL-stream runs after the legacy default stream
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int kernels = 0;

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  void drop_plan() {
    drop_graph();
    for (cudaStream_t st : branches) cudaStreamDestroy(st);
    for (cudaEvent_t ev : joins) cudaEventDestroy(ev);
    branches.clear();
    joins.clear();
    if (ws) cudaFree(ws);
    ws = nullptr;
    ws_bytes = 0;
    status = nullptr;
  }
  void lock_all() {
    views.resize(uniq.size());
    for (size_t i = 0; i < uniq.size(); ++i) index_lock_view(uniq[i], &views[i]);
  }
  void unlock_all() {
    for (size_t i = uniq.size(); i-- > 0;) index_unlock(uniq[i]);
  }
};

namespace {

// Builds the plan, the workspace and the graph.  Index locks are held.
int plan_batch(curplsh_batch* b) {
  b->drop_plan();
  int num_sms = 0;
  BT_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, b->device));
  int rc = b->plan.build(b->items.data(), (int)b->items.size(), b->uniq, b->views, b->precision, b->rerank_factor,
                         num_sms);
  if (rc) return rc;
  b->ws_bytes = b->plan.bytes();
  BT_TRY(cudaMalloc(&b->ws, b->ws_bytes));
  b->plan.bind(b->ws);
  b->status = b->plan.status();
  // launch attributes are set before the capture
  for (int form = 0; form < 3; ++form) BT_TRY(prepare_fused_kernels(form));
  BT_TRY(prepare_merge_kernel());
  if (!b->cap) BT_TRY(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  if (!b->fork) BT_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  for (int g = 0; g < b->plan.num_groups(); ++g) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    BT_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->branches.push_back(st);
    BT_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->joins.push_back(ev);
  }
  int kernels = 0;
  BT_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
  rc = b->plan.enqueue(b->cap, &b->branches, &b->joins, b->fork, &kernels);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->cap, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CURPLSH_ERR_CUDA, "stream capture of the batch failed: %s", cudaGetErrorString(e));
  }
  b->graph = graph;
  BT_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->kernels = kernels;
  b->gens.resize(b->uniq.size());
  for (size_t i = 0; i < b->uniq.size(); ++i) b->gens[i] = b->views[i].generation;
  return CURPLSH_OK;
}

struct DevScope {
  int prev = -1;
  explicit DevScope(int dev) {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) {
      prev = cur;
      cudaSetDevice(dev);
    }
  }
  ~DevScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

int curplsh_batch_create(const curplsh_batch_item* items, int count, int precision, int rerank_factor,
                         curplsh_batch** out) {
  if (!out) return fail(CURPLSH_ERR_INVALID_ARG, "null out");
  *out = nullptr;
  if (!items || count <= 0) return fail(CURPLSH_ERR_INVALID_ARG, "empty batch");
  if (precision < -1 || precision > 2) return fail(CURPLSH_ERR_INVALID_ARG, "unknown precision %d", precision);
  std::vector<curplsh_index*> uniq;
  for (int i = 0; i < count; ++i) {
    const curplsh_batch_item& it = items[i];
    if (!it.index) return fail(CURPLSH_ERR_INVALID_ARG, "item %d: null index", i);
    if (it.num < 0) return fail(CURPLSH_ERR_INVALID_ARG, "item %d: negative number of queries", i);
    if (it.k < 1 || it.k > 1024) return fail(CURPLSH_ERR_INVALID_ARG, "item %d: k=%d outside [1, 1024]", i, it.k);
    if (it.num > 0 && (!it.queries || !it.indices || !it.distances))
      return fail(CURPLSH_ERR_INVALID_ARG, "item %d: null pointer", i);
    uniq.push_back(it.index);
  }
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  curplsh_batch* b = new curplsh_batch();
  b->items.assign(items, items + count);
  b->precision = precision;
  b->rerank_factor = rerank_factor;
  b->uniq = uniq;
  b->lock_all();
  int rc = CURPLSH_OK;
  b->device = b->views[0].device;
  for (const IndexView& v : b->views)
    if (v.device != b->device) rc = fail(CURPLSH_ERR_INVALID_ARG, "a batch's indexes must share one device");
  if (!rc) {
    DevScope scope(b->device);
    for (int i = 0; i < count && !rc; ++i) {
      const curplsh_batch_item& it = items[i];
      if (it.num == 0) continue;
      if (!is_device_ptr(it.queries, b->device) || !is_device_ptr(it.indices, b->device) ||
          !is_device_ptr(it.distances, b->device))
        rc = fail(CURPLSH_ERR_INVALID_ARG, "item %d: queries and outputs must be device memory of device %d", i,
                  b->device);
    }
    if (!rc) rc = plan_batch(b);
  }
  b->unlock_all();
  if (rc) {
    curplsh_batch_destroy(b);
    return rc;
  }
  *out = b;
  return CURPLSH_OK;
}

int curplsh_batch_run(curplsh_batch* b, void* stream, int wait) {
  if (!b) return fail(CURPLSH_ERR_INVALID_ARG, "null batch");
  DevScope scope(b->device);
  b->lock_all();
  int rc = CURPLSH_OK;
  bool stale = !b->exec;
  for (size_t i = 0; i < b->uniq.size(); ++i) stale = stale || b->views[i].generation != b->gens[i];
  if (stale) {
    // the old graph may still run on some stream: let it finish before its workspace goes
    cudaDeviceSynchronize();
    rc = plan_batch(b);
  }
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->views[0].stream;
  if (!rc && !stream) {
    cudaError_t e = b->order_ev ? cudaSuccess : cudaEventCreateWithFlags(&b->order_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(b->order_ev, cudaStreamLegacy);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->order_ev, 0);
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = fail(CURPLSH_ERR_CUDA, "ordering after the legacy stream: %s", cudaGetErrorString(e));
    }
  }
  if (!rc) {
    cudaError_t e = cudaGraphLaunch(b->exec, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = fail(CURPLSH_ERR_CUDA, "cudaGraphLaunch: %s", cudaGetErrorString(e));
    }
  }
  b->unlock_all();
  if (rc || !wait) return rc;
  if (!b->host_status) {
    cudaError_t e = cudaMallocHost(&b->host_status, sizeof(uint32_t));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(CURPLSH_ERR_OOM, "cudaMallocHost: %s", cudaGetErrorString(e));
    }
  }
  BT_TRY(cudaMemcpyAsync(b->host_status, b->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  BT_TRY(cudaStreamSynchronize(st));
  if (*b->host_status)
    return fail(CURPLSH_ERR_DEVICE, "device status 0x%x (1: bounded wait expired, 2: pool overflow, 4: schedule)",
                *b->host_status);
  return CURPLSH_OK;
}

int curplsh_batch_get_info(const curplsh_batch* b, int* kernel_launches, int64_t* workspace_bytes) {
  if (!b) return fail(CURPLSH_ERR_INVALID_ARG, "null batch");
  if (kernel_launches) *kernel_launches = b->kernels;
  if (workspace_bytes) *workspace_bytes = (int64_t)b->ws_bytes;
  return CURPLSH_OK;
}

int curplsh_batch_destroy(curplsh_batch* b) {
  if (!b) return CURPLSH_OK;
  {
    DevScope scope(b->device);
    if (b->cap) cudaStreamSynchronize(b->cap);
    cudaDeviceSynchronize();
    b->drop_plan();
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->order_ev) cudaEventDestroy(b->order_ev);
    if (b->host_status) cudaFreeHost(b->host_status);
  }
  delete b;
  return CURPLSH_OK;
}

}  // extern "C"
