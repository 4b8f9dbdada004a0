// server.cpp -- serving loop: continuous batching of search requests against
// one resident index.
//
// No counterpart in cuRPLSH (its IndexBF::search is a blocking call per query
// matrix, src/index_bf.cpp:46-74).  Requests are submitted from any thread
// and return a ticket; a scheduler thread forms "steps" from the waiting
// requests (first come, first served) and issues each step -- query prep,
// fused tensor-core filter, merge + rerank, via MultiPlan -- on one of
// `max_inflight` streams, so a step formed from requests that arrived while
// earlier steps are on the GPU runs concurrently with them.  Admission is by
// device memory: every step's working memory (its MultiPlan plus staging for
// host inputs) is carved from one arena of `memory_budget` bytes allocated at
// creation, and a request waits until its step fits in the free space.
// Completion is signalled by a host function queued behind the step (the
// scheduler sleeps on a condition variable, with a short time-out as a
// safety net rather than a polling loop).
//
// Results: each request resolves k' and the pool capacity exactly as a search
// of that request alone, and a query's candidates and distances do not depend
// on the other queries of its step, so every result equals
// curplsh_index_search_ex of the request alone (same precision and rerank).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/curplsh_b200.h"
#include "fused_knn.h"
#include "multi_plan.h"
#include "server_sched.h"

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

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t rup(size_t x, size_t m) { return (x + m - 1) / m * m; }

int pointer_dev(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ? a.device : -1;
}

enum ReqState { kPending = 0, kRunning = 1, kDone = 2, kFailed = 3 };

struct Request {
  int64_t num = 0;
  const float* queries = nullptr;
  int k = 1;
  int32_t* indices = nullptr;
  float* distances = nullptr;
  bool q_dev = false, o_dev = false;
  // host clock: submitted, issued in a step, the step's completion callback
  // ran, results visible to wait()
  double t_submit = 0, t_issue = 0, t_begin = 0, t_gpu = 0, t_done = 0;
  double gpu_exec = 0;  // seconds between the step's first and last work on its stream (CUDA events)
  int state = kPending;
  int err = CURPLSH_OK;
  std::string msg;
};

struct Step;
struct Slot {
  cudaStream_t st = nullptr;
  char* pinned = nullptr;  // host staging: queries, then outputs, then the status word
  size_t pinned_bytes = 0;
  bool busy = false;
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr;  // bracket the step's device work on st
};

struct Step {
  curplsh_server* srv = nullptr;
  int slot = 0;
  std::vector<int64_t> tickets;
  size_t off = 0, bytes = 0;
  MultiPlan plan;
  // host-output copies to do at completion: (ticket, pinned offset)
  std::vector<std::pair<int64_t, size_t>> host_out;
  double t_begin_seen = 0;  // host clock when the scheduler first saw the step's work begun
  double t_gpu_done = 0;    // host clock when the scheduler saw the step's work complete
};

}  // namespace

struct curplsh_server {
  curplsh_index* index = nullptr;
  curplsh_server_config cfg{};
  int device = 0, num_sms = 0, dim = 0;
  void* arena_mem = nullptr;
  Arena arena;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_done;  // waiters
  std::condition_variable cv_work;  // scheduler
  std::deque<int64_t> pending;
  std::unordered_map<int64_t, Request> reqs;
  std::vector<std::unique_ptr<Step>> inflight;
  int64_t next_ticket = 1;
  bool stop = false;
  std::thread worker;
  curplsh_server_stats stats{};
  double busy_since = -1;
};

namespace {

// Queued behind each step as a wake-up hint only: the scheduler decides that
// a step is complete by querying the CUDA event recorded after its last copy
// (host functions run on a driver thread that was seen to run them tens of
// milliseconds after the work, at low load), and polls every 200 us while
// steps are in flight.  It takes no lock (a host function that blocks would
// stall its stream) and touches nothing but the server, which outlives it
// (destroy synchronises every slot stream before freeing the server).
void CUDART_CB on_step_done(void* p) { static_cast<curplsh_server*>(p)->cv_work.notify_one(); }

// Pinned staging of one slot: [queries][outputs][status word]; every request
// rounds its pieces up to 256 bytes.
size_t pinned_query_bytes(const curplsh_server* s) {
  const size_t m = (size_t)s->cfg.max_step_queries;
  return rup(m * s->dim * sizeof(float) + 256 * m, 256);
}
size_t pinned_bytes_for(const curplsh_server* s) {
  const size_t m = (size_t)s->cfg.max_step_queries;
  const size_t o = m * 1024 * (sizeof(int32_t) + sizeof(float)) + 256 * m;
  return pinned_query_bytes(s) + rup(o, 256) + 256;
}

// Builds the step plan for `tickets` (index locked by the caller).
int build_step(curplsh_server* s, const std::vector<int64_t>& tickets, std::vector<curplsh_index*>& uniq,
               std::vector<IndexView>& views, MultiPlan& plan, std::vector<curplsh_batch_item>& items,
               size_t* staging) {
  items.clear();
  size_t st_bytes = 0;
  for (int64_t t : tickets) {
    const Request& r = s->reqs[t];
    curplsh_batch_item it{};
    it.index = s->index;
    it.num = r.num;
    it.queries = r.queries;  // placeholders for host memory, rebound before launch
    it.k = r.k;
    it.indices = r.indices;
    it.distances = r.distances;
    items.push_back(it);
    if (!r.q_dev) st_bytes += rup((size_t)r.num * s->dim * sizeof(float), 256);
    if (!r.o_dev) st_bytes += rup((size_t)r.num * r.k * (sizeof(int32_t) + sizeof(float)), 256);
  }
  *staging = st_bytes;
  return plan.build(items.data(), (int)items.size(), uniq, views, s->cfg.precision, s->cfg.rerank_factor,
                    s->num_sms);
}

void finish_step(curplsh_server* s, Step& st) {
  // called with the lock held, after the step's stream has completed
  const Slot& slot = s->slots[st.slot];
  const uint32_t status = *reinterpret_cast<const uint32_t*>(slot.pinned + slot.pinned_bytes - 256);
  float exec_ms = 0.f;
  if (cudaEventElapsedTime(&exec_ms, slot.ev_begin, slot.ev_end) != cudaSuccess) {
    cudaGetLastError();
    exec_ms = 0.f;
  }
  for (auto& ho : st.host_out) {
    Request& r = s->reqs[ho.first];
    const size_t ni = (size_t)r.num * r.k;
    memcpy(r.indices, slot.pinned + ho.second, ni * sizeof(int32_t));
    memcpy(r.distances, slot.pinned + ho.second + ni * sizeof(int32_t), ni * sizeof(float));
  }
  const double t = now_s();
  for (int64_t tk : st.tickets) {
    Request& r = s->reqs[tk];
    r.t_done = t;
    r.t_gpu = st.t_gpu_done;
    r.t_begin = st.t_begin_seen;
    r.gpu_exec = exec_ms * 1e-3;
    if (status) {
      r.state = kFailed;
      r.err = CURPLSH_ERR_DEVICE;
      char m[160];
      snprintf(m, sizeof(m), "device status 0x%x (1: bounded wait expired, 2: pool overflow, 4: schedule)", status);
      r.msg = m;
    } else {
      r.state = kDone;
      s->stats.requests_done += 1;
      s->stats.queries_done += r.num;
    }
  }
  s->arena.release(st.off, st.bytes);
  s->slots[st.slot].busy = false;
}

// Forms and issues one step from the head of the queue.  Returns false when
// nothing could be issued (no free slot, or the head does not fit yet).
bool issue_step(curplsh_server* s, std::unique_lock<std::mutex>& lk) {
  int slot_i = -1;
  for (size_t i = 0; i < s->slots.size(); ++i)
    if (!s->slots[i].busy) {
      slot_i = (int)i;
      break;
    }
  if (slot_i < 0 || s->pending.empty()) return false;
  Slot& slot = s->slots[slot_i];
  // take requests first come, first served within the per-step query cap
  std::vector<int64_t> take =
      take_step(s->pending, s->cfg.max_step_queries, [&](int64_t t) { return s->reqs[t].num; });
  std::vector<curplsh_index*> uniq{s->index};
  std::vector<IndexView> views(1);
  if (index_lock_view(s->index, &views[0])) return false;
  std::unique_ptr<Step> st(new Step());
  st->srv = s;
  st->slot = slot_i;
  std::vector<curplsh_batch_item> items;
  size_t staging = 0;
  int rc = CURPLSH_OK;
  // shrink the step until its working memory fits the free arena (the plan
  // and items left behind are those of the admitted requests)
  const int adm = admit_step(take, s->arena, &st->off, &st->bytes,
                             [&](const std::vector<int64_t>& tk, size_t* bytes) -> int {
                               rc = build_step(s, tk, uniq, views, st->plan, items, &staging);
                               if (rc) return rc;
                               *bytes = rup(st->plan.bytes(), 256) + staging;
                               return 0;
                             });
  if (adm == 0) {
    index_unlock(s->index);
    return false;  // admission: wait for running steps to release memory
  }
  if (rc) {
    index_unlock(s->index);
    // the head request cannot be planned: fail it alone
    Request& r = s->reqs[take.front()];
    r.state = kFailed;
    r.err = rc;
    r.msg = curplsh_last_error();
    r.t_done = now_s();
    s->pending.pop_front();
    s->cv_done.notify_all();
    return true;
  }
  for (size_t i = 0; i < take.size(); ++i) s->pending.pop_front();
  const double t_issue = now_s();
  for (int64_t t : take) {
    s->reqs[t].state = kRunning;
    s->reqs[t].t_issue = t_issue;
  }
  st->tickets = take;
  slot.busy = true;
  // ---- bind memory: [plan][staging...]; host inputs go through the pinned slot buffer
  char* dbase = static_cast<char*>(s->arena_mem) + st->off;
  st->plan.bind(dbase);
  size_t doff = rup(st->plan.bytes(), 256);
  size_t pq = 0;                        // pinned query cursor
  size_t po = pinned_query_bytes(s);     // pinned output cursor
  cudaError_t e = cudaEventRecord(slot.ev_begin, slot.st);
  for (size_t i = 0; i < take.size(); ++i) {
    Request& r = s->reqs[take[i]];
    curplsh_batch_item& it = items[i];
    if (!r.q_dev) {
      const size_t qb = (size_t)r.num * s->dim * sizeof(float);
      memcpy(slot.pinned + pq, r.queries, qb);
      float* dq = reinterpret_cast<float*>(dbase + doff);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dq, slot.pinned + pq, qb, cudaMemcpyHostToDevice, slot.st);
      it.queries = dq;
      pq += rup(qb, 256);
      doff += rup(qb, 256);
    }
    if (!r.o_dev) {
      const size_t ni = (size_t)r.num * r.k;
      it.indices = reinterpret_cast<int32_t*>(dbase + doff);
      it.distances = reinterpret_cast<float*>(dbase + doff + ni * sizeof(int32_t));
      doff += rup(ni * (sizeof(int32_t) + sizeof(float)), 256);
    }
  }
  // the plan was built with the caller's pointers: point host-memory
  // requests at their device staging
  for (size_t i = 0; i < take.size(); ++i) st->plan.set_item_pointers((int)i, items[i].queries, items[i].indices,
                                                                         items[i].distances);
  int kernels = 0;
  if (!rc && e == cudaSuccess) rc = st->plan.enqueue(slot.st, nullptr, nullptr, nullptr, &kernels);
  index_unlock(s->index);
  if (!rc && e == cudaSuccess) {
    for (size_t i = 0; i < take.size(); ++i) {
      Request& r = s->reqs[take[i]];
      if (r.o_dev) continue;
      const size_t ni = (size_t)r.num * r.k;
      e = cudaMemcpyAsync(slot.pinned + po, items[i].indices, ni * sizeof(int32_t), cudaMemcpyDeviceToHost, slot.st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(slot.pinned + po + ni * sizeof(int32_t), items[i].distances, ni * sizeof(float),
                            cudaMemcpyDeviceToHost, slot.st);
      st->host_out.emplace_back(take[i], po);
      po += rup(ni * (sizeof(int32_t) + sizeof(float)), 256);
      if (e != cudaSuccess) break;
    }
  }
  if (!rc && e == cudaSuccess)
    e = cudaMemcpyAsync(slot.pinned + slot.pinned_bytes - 256, st->plan.status(), sizeof(uint32_t),
                        cudaMemcpyDeviceToHost, slot.st);
  if (!rc && e == cudaSuccess) e = cudaEventRecord(slot.ev_end, slot.st);
  if (!rc && e == cudaSuccess) e = cudaLaunchHostFunc(slot.st, on_step_done, s);
  if (rc || e != cudaSuccess) {
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = fail(CURPLSH_ERR_CUDA, "serving step: %s", cudaGetErrorString(e));
    }
    // nothing may still read this step's memory: wait for the stream
    lk.unlock();
    cudaStreamSynchronize(slot.st);
    lk.lock();
    const std::string msg = curplsh_last_error();
    for (int64_t t : take) {
      Request& r = s->reqs[t];
      r.state = kFailed;
      r.err = rc;
      r.msg = msg;
      r.t_done = now_s();
    }
    s->arena.release(st->off, st->bytes);
    slot.busy = false;
    s->cv_done.notify_all();
    return true;
  }
  s->stats.steps += 1;
  s->stats.kernel_launches += kernels;
  int64_t q = 0;
  for (int64_t t : take) q += s->reqs[t].num;
  if (q > s->stats.max_step_queries) s->stats.max_step_queries = q;
  s->inflight.push_back(std::move(st));
  if ((int)s->inflight.size() > s->stats.max_inflight_seen) s->stats.max_inflight_seen = (int)s->inflight.size();
  if ((int64_t)s->arena.in_use() > s->stats.peak_bytes_in_use) s->stats.peak_bytes_in_use = (int64_t)s->arena.in_use();
  return true;
}

void scheduler(curplsh_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    bool progressed = false;
    // retire completed steps (their end event has fired; oldest first keeps
    // FIFO completion per slot)
    const double t_poll = now_s();
    for (size_t i = 0; i < s->inflight.size();) {
      Step& stp = *s->inflight[i];
      const Slot& sl = s->slots[stp.slot];
      if (stp.t_begin_seen == 0 && cudaEventQuery(sl.ev_begin) == cudaSuccess) stp.t_begin_seen = t_poll;
      const cudaError_t q = cudaEventQuery(sl.ev_end);
      if (q != cudaErrorNotReady) {
        if (q != cudaSuccess) cudaGetLastError();  // an error: finish_step reports the status word
        stp.t_gpu_done = t_poll;
        if (stp.t_begin_seen == 0) stp.t_begin_seen = t_poll;
        finish_step(s, stp);
        s->inflight.erase(s->inflight.begin() + (long)i);
        progressed = true;
      } else {
        ++i;
      }
    }
    if (progressed) s->cv_done.notify_all();
    while (issue_step(s, lk)) progressed = true;
    const bool busy = !s->inflight.empty();
    const double t = now_s();
    if (busy && s->busy_since < 0) s->busy_since = t;
    if (!busy && s->busy_since >= 0) {
      s->stats.busy_seconds += t - s->busy_since;
      s->busy_since = -1;
    }
    if (s->stop && s->pending.empty() && s->inflight.empty()) break;
    if (!progressed) {
      if (s->inflight.empty())
        s->cv_work.wait(lk);  // submit and destroy notify under the lock
      else
        s->cv_work.wait_for(lk, std::chrono::microseconds(200));
    }
  }
}

}  // namespace

extern "C" {

void curplsh_server_config_init(curplsh_server_config* cfg) {
  if (!cfg) return;
  memset(cfg, 0, sizeof(*cfg));
  cfg->precision = -1;
  cfg->rerank_factor = 0;
  cfg->max_inflight = 3;
  cfg->max_step_queries = 4096;
  cfg->memory_budget = (int64_t)2 << 30;
}

int curplsh_server_create(curplsh_index* index, const curplsh_server_config* cfg, curplsh_server** out) {
  if (!index || !out) return fail(CURPLSH_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  curplsh_server_config c;
  curplsh_server_config_init(&c);
  if (cfg) c = *cfg;
  if (c.max_inflight < 1 || c.max_inflight > 16 || c.max_step_queries < 1 || c.max_step_queries > (1 << 20) ||
      c.memory_budget < ((int64_t)1 << 20) || c.precision < -1 || c.precision > 2)
    return fail(CURPLSH_ERR_INVALID_ARG, "bad server configuration");
  IndexView v;
  if (index_lock_view(index, &v)) return CURPLSH_ERR_INVALID_ARG;
  index_unlock(index);
  std::unique_ptr<curplsh_server> s(new curplsh_server());
  s->index = index;
  s->cfg = c;
  s->device = v.device;
  s->dim = v.dim;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  auto restore = [&]() { cudaSetDevice(prev); };
  cudaError_t e = cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
  if (e == cudaSuccess) e = cudaMalloc(&s->arena_mem, (size_t)c.memory_budget);
  for (int i = 0; i < c.max_inflight && e == cudaSuccess; ++i) {
    Slot sl;
    e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
    sl.pinned_bytes = pinned_bytes_for(s.get());
    if (e == cudaSuccess) e = cudaMallocHost(&sl.pinned, sl.pinned_bytes);
    if (e == cudaSuccess) e = cudaEventCreate(&sl.ev_begin);
    if (e == cudaSuccess) e = cudaEventCreate(&sl.ev_end);
    s->slots.push_back(sl);
  }
  for (int form = 0; form < 3 && e == cudaSuccess; ++form) e = prepare_fused_kernels(form);
  if (e == cudaSuccess) e = prepare_merge_kernel();
  if (e != cudaSuccess) {
    cudaGetLastError();
    for (Slot& sl : s->slots) {
      if (sl.st) cudaStreamDestroy(sl.st);
      if (sl.pinned) cudaFreeHost(sl.pinned);
      if (sl.ev_begin) cudaEventDestroy(sl.ev_begin);
      if (sl.ev_end) cudaEventDestroy(sl.ev_end);
    }
    if (s->arena_mem) cudaFree(s->arena_mem);
    restore();
    return fail(e == cudaErrorMemoryAllocation ? CURPLSH_ERR_OOM : CURPLSH_ERR_CUDA, "server set-up: %s",
                cudaGetErrorString(e));
  }
  restore();
  s->arena.reset((size_t)c.memory_budget);
  curplsh_server* raw = s.release();
  raw->worker = std::thread(scheduler, raw);
  *out = raw;
  return CURPLSH_OK;
}

int curplsh_server_submit(curplsh_server* s, int64_t num, const float* queries, int k, int32_t* indices,
                          float* distances, int64_t* ticket) {
  if (!s || !ticket) return fail(CURPLSH_ERR_INVALID_ARG, "null argument");
  if (num < 1) return fail(CURPLSH_ERR_INVALID_ARG, "a request needs at least one query");
  if (!queries || !indices || !distances) return fail(CURPLSH_ERR_INVALID_ARG, "null pointer argument");
  if (k < 1 || k > 1024) return fail(CURPLSH_ERR_INVALID_ARG, "k=%d outside [1, 1024]", k);
  if (num > s->cfg.max_step_queries)
    return fail(CURPLSH_ERR_INVALID_ARG, "%lld queries in one request, more than max_step_queries=%d",
                (long long)num, s->cfg.max_step_queries);
  Request r;
  r.num = num;
  r.queries = queries;
  r.k = k;
  r.indices = indices;
  r.distances = distances;
  const int qd = pointer_dev(queries), id = pointer_dev(indices), dd = pointer_dev(distances);
  if ((qd >= 0 && qd != s->device) || (id >= 0 && id != s->device) || (dd >= 0 && dd != s->device))
    return fail(CURPLSH_ERR_INVALID_ARG, "device pointers must be on the index's device %d", s->device);
  if ((id >= 0) != (dd >= 0)) return fail(CURPLSH_ERR_INVALID_ARG, "indices and distances must share a memory space");
  r.q_dev = qd >= 0;
  r.o_dev = id >= 0;
  // admission check: the request alone must fit in the whole arena
  {
    std::vector<curplsh_index*> uniq{s->index};
    std::vector<IndexView> views(1);
    if (index_lock_view(s->index, &views[0])) return CURPLSH_ERR_INVALID_ARG;
    curplsh_batch_item it{};
    it.index = s->index;
    it.num = num;
    it.queries = queries;
    it.k = k;
    it.indices = indices;
    it.distances = distances;
    MultiPlan p;
    int rc = p.build(&it, 1, uniq, views, s->cfg.precision, s->cfg.rerank_factor, s->num_sms);
    index_unlock(s->index);
    if (rc) return rc;
    size_t need = rup(p.bytes(), 256);
    if (!r.q_dev) need += rup((size_t)num * s->dim * sizeof(float), 256);
    if (!r.o_dev) need += rup((size_t)num * k * (sizeof(int32_t) + sizeof(float)), 256);
    if (need > (size_t)s->cfg.memory_budget)
      return fail(CURPLSH_ERR_INVALID_ARG, "request needs %zu bytes of working memory, more than the budget %lld",
                  need, (long long)s->cfg.memory_budget);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return fail(CURPLSH_ERR_STATE, "server is shutting down");
  const int64_t t = s->next_ticket++;
  r.t_submit = now_s();
  s->reqs.emplace(t, r);
  s->pending.push_back(t);
  s->cv_work.notify_one();
  *ticket = t;
  return CURPLSH_OK;
}

int curplsh_server_wait_phases(curplsh_server* s, int64_t ticket, double timeout_s, double* latency_s,
                               double* phases) {
  if (!s) return fail(CURPLSH_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(CURPLSH_ERR_INVALID_ARG, "unknown ticket %lld", (long long)ticket);
  auto ready = [&]() { return it->second.state >= kDone; };
  if (timeout_s < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    return fail(CURPLSH_ERR_STATE, "ticket %lld not finished within %.3f s", (long long)ticket, timeout_s);
  }
  const Request r = it->second;
  s->reqs.erase(it);
  if (latency_s) *latency_s = r.t_done - r.t_submit;
  if (phases) {
    const bool ran = r.t_issue > 0 && r.t_gpu > 0;
    phases[0] = r.t_issue > 0 ? r.t_issue - r.t_submit : r.t_done - r.t_submit;  // waiting for a step
    phases[1] = ran ? r.t_gpu - r.t_issue : 0.0;                                 // step issued -> GPU done
    phases[2] = ran ? r.t_done - r.t_gpu : 0.0;                                  // GPU done -> visible
    phases[3] = ran ? r.gpu_exec : 0.0;  // the step's device work itself (CUDA events, inside phases[1])
    phases[4] = ran ? r.t_begin - r.t_issue : 0.0;  // issue -> its first work seen begun (inside phases[1])
  }
  if (r.state == kFailed) return fail(r.err ? r.err : CURPLSH_ERR_DEVICE, "%s", r.msg.c_str());
  return CURPLSH_OK;
}

int curplsh_server_wait(curplsh_server* s, int64_t ticket, double timeout_s, double* latency_s) {
  return curplsh_server_wait_phases(s, ticket, timeout_s, latency_s, nullptr);
}

int curplsh_server_get_stats(curplsh_server* s, curplsh_server_stats* out) {
  if (!s || !out) return fail(CURPLSH_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  if (s->busy_since >= 0) out->busy_seconds += now_s() - s->busy_since;
  return CURPLSH_OK;
}

int curplsh_server_destroy(curplsh_server* s) {
  if (!s) return CURPLSH_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_work.notify_one();
  }
  if (s->worker.joinable()) s->worker.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  for (Slot& sl : s->slots) {
    cudaStreamSynchronize(sl.st);
    cudaStreamDestroy(sl.st);
    cudaFreeHost(sl.pinned);
    cudaEventDestroy(sl.ev_begin);
    cudaEventDestroy(sl.ev_end);
  }
  cudaFree(s->arena_mem);
  cudaSetDevice(prev);
  delete s;
  return CURPLSH_OK;
}

}  // extern "C"
