// batch.cpp -- batched search over several indexes as one captured CUDA graph.
//
// No counterpart in cuRPLSH: its IndexBF::search (src/index_bf.cpp:46-74)
// serves one query matrix against one index per call, each call paying its
// own launches and a device synchronisation (src/internal/search.cu:79-216).
//
// Plan (once per batch, and again when an index changes):
//   * every item resolves its precision form, k' and pool capacity exactly as
//     a single search would (search_kprime / search_pool_capacity), so its
//     results are those of the item searched alone;
//   * items against the same index with the same (form, k') are concatenated
//     into one fused item: their queries share 128-row query blocks, so many
//     small batches stream the database once instead of once each;
//   * fused items are grouped by (form, d) -- one kernel instantiation and one
//     shared-memory layout per group -- and each group gets one segmented prep
//     launch, persistent fused launches of up to kFusedMaxItems items whose
//     balanced schedule spans all of them, and one merge + rerank launch;
//   * groups are parallel branches of the graph; each fused launch asks for
//     every SM, so a group's tail overlaps the next group's start.
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

long long rup(long long x, long long m) { return (x + m - 1) / m * m; }

bool is_device_ptr(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

struct FItem {
  int slot = 0;  // index (into Batch::uniq)
  int form = 0, kp = 0, P = 0, d = 0, k = 1;
  TuneParams tune;
  int nq = 0;
  long long nq_pad = 0;
  std::vector<int> members;  // batch items, in order
  std::vector<int> row0;     // first row of each member
  FusedItemSpec spec{};
  FusedItemPlan plan{};
  long long W = 1;
};

struct FLaunch {
  std::vector<int> fitems;
  FusedBatchPlan bp;
};

struct Group {
  int form = 0, d = 0;
  long long ld16 = 0, ld8 = 0;
  std::vector<int> fitems;
  std::vector<FLaunch> launches;
  long long work = 0;
  int max_ctas = 1;
  cudaStream_t branch = nullptr;
  cudaEvent_t join = nullptr;
};

}  // namespace

struct curplsh_batch {
  std::vector<curplsh_batch_item> items;
  int precision = -1, rerank_factor = 0;
  int device = 0;
  std::vector<curplsh_index*> uniq;  // sorted by address (lock order)
  std::vector<IndexView> views;
  std::vector<long long> gens;
  std::vector<FItem> fitems;
  std::vector<Group> groups;
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
    for (auto& g : groups) {
      if (g.branch) cudaStreamDestroy(g.branch);
      if (g.join) cudaEventDestroy(g.join);
    }
    groups.clear();
    fitems.clear();
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
  const int dev = b->device;
  int num_sms = 0;
  BT_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));

  // ---- fused items
  std::map<std::tuple<int, int, int>, int> fmap;  // (slot, form, kp) -> fitem
  for (size_t i = 0; i < b->items.size(); ++i) {
    const curplsh_batch_item& it = b->items[i];
    if (it.num == 0) continue;
    const int slot = (int)(std::lower_bound(b->uniq.begin(), b->uniq.end(), it.index) - b->uniq.begin());
    IndexView& v = b->views[slot];
    const int form = b->precision < 0 ? v.precision : b->precision;
    const int rf = b->rerank_factor > 0 ? b->rerank_factor : v.rerank_factor;
    int rc = index_prepare_form(b->uniq[slot], form, &v);
    if (rc) return rc;
    const int kp = search_kprime(form, it.k, rf, v.n);
    auto key = std::make_tuple(slot, form, kp);
    auto f = fmap.find(key);
    int fi;
    if (f == fmap.end()) {
      fi = (int)b->fitems.size();
      fmap.emplace(key, fi);
      FItem x;
      x.slot = slot;
      x.form = form;
      x.kp = kp;
      x.d = v.dim;
      x.k = it.k;
      b->fitems.push_back(x);
    } else {
      fi = f->second;
    }
    FItem& x = b->fitems[fi];
    if ((long long)x.nq + it.num > (1LL << 30))
      return fail(CURPLSH_ERR_UNSUPPORTED, "more than 2^30 queries against one index in one batch");
    x.members.push_back((int)i);
    x.row0.push_back(x.nq);
    x.nq += (int)it.num;
  }
  // tuned parameters per fused item, looked up with its concatenated query count
  for (FItem& x : b->fitems) {
    x.tune = tune_lookup(x.form, x.d, x.k, x.nq);
    x.P = search_pool_capacity(x.kp, x.tune.headroom);
  }
  // ---- groups
  std::map<std::pair<int, int>, int> gmap;
  long long total_work = 0;
  for (size_t fi = 0; fi < b->fitems.size(); ++fi) {
    FItem& x = b->fitems[fi];
    const IndexView& v = b->views[x.slot];
    x.nq_pad = rup(x.nq, kBM);
    auto key = std::make_pair(x.form, x.d);
    auto g = gmap.find(key);
    int gi;
    if (g == gmap.end()) {
      gi = (int)b->groups.size();
      gmap.emplace(key, gi);
      Group G;
      G.form = x.form;
      G.d = x.d;
      G.ld16 = v.ld16;
      G.ld8 = v.ld8;
      b->groups.push_back(G);
    } else {
      gi = g->second;
    }
    Group& G = b->groups[gi];
    G.fitems.push_back((int)fi);
    if (v.n > 0) {
      const long long w = (long long)((x.nq + kBM - 1) / kBM) * ((v.n + kBN - 1) / kBN);
      G.work += w;
      total_work += w;
    }
  }
  (void)total_work;
  for (Group& G : b->groups) {
    // Every group's persistent launch asks for all SMs.  The branches are
    // independent, so the hardware starts a later group's CTAs on the SMs an
    // earlier group releases (its tail overlaps the next group's start); a
    // static split of the SMs by tile count would instead leave groups whose
    // tiles are dearer (larger d, larger k') as the long pole.
    G.max_ctas = num_sms;
    // fused launches of up to kFusedMaxItems items with a non-empty database
    FLaunch L;
    for (int fi : G.fitems) {
      if (b->views[b->fitems[fi].slot].n == 0) continue;
      if ((int)L.fitems.size() == kFusedMaxItems) {
        G.launches.push_back(L);
        L.fitems.clear();
      }
      L.fitems.push_back(fi);
    }
    if (!L.fitems.empty()) G.launches.push_back(L);
    for (FLaunch& FL : G.launches) {
      std::vector<FusedItemSpec> specs(FL.fitems.size());
      std::vector<FusedItemPlan> plans(FL.fitems.size());
      for (size_t j = 0; j < FL.fitems.size(); ++j) {
        const FItem& x = b->fitems[FL.fitems[j]];
        specs[j].nq = x.nq;
        specs[j].nb = (int)b->views[x.slot].n;
        // units as long as the item's own CTA ranges would be if it were
        // searched alone (scaled by the tuned split), so its in-pool selection
        // work stays what it is alone
        const long long own = (long long)((x.nq + kBM - 1) / kBM) * ((specs[j].nb + kBN - 1) / kBN);
        // (clamped to the item's own range, as in a search alone, where a
        // unit can never be longer than its CTA range)
        specs[j].split_tiles = split_tiles_for(std::max<long long>(1, (own + num_sms - 1) / num_sms),
                                               std::min(x.tune.split_q4, 4));
      }
      plan_fused_batch(specs.data(), (int)specs.size(), G.max_ctas, plans.data(), &FL.bp);
      for (size_t j = 0; j < FL.fitems.size(); ++j) {
        FItem& x = b->fitems[FL.fitems[j]];
        x.plan = plans[j];
        x.W = FL.bp.work_per_cta;
      }
    }
  }
  // ---- workspace: [status][all bounds][per fused item operands, counts, pools]
  size_t off = 0;
  auto take = [&](size_t bytes) {
    off = (size_t)rup((long long)off, 256);
    const size_t o = off;
    off += bytes;
    return o;
  };
  const size_t o_status = take(sizeof(uint32_t));
  size_t bounds_words = 0;
  for (const FItem& x : b->fitems) bounds_words += 3 * (size_t)x.nq_pad;
  const size_t o_bounds = take(bounds_words * sizeof(uint32_t));
  struct Offs {
    size_t qh, ql, q8, qn, qs, counts, pools, bounds;
  };
  std::vector<Offs> offs(b->fitems.size());
  size_t bcur = 0;
  for (size_t fi = 0; fi < b->fitems.size(); ++fi) {
    const FItem& x = b->fitems[fi];
    const IndexView& v = b->views[x.slot];
    Offs& o = offs[fi];
    o = Offs{};
    o.bounds = o_bounds + bcur * sizeof(uint32_t);
    bcur += 3 * (size_t)x.nq_pad;
    if (v.n == 0) continue;
    const size_t lists = (size_t)x.plan.num_qblocks * kBM * x.plan.units_per_block * 2;
    if (x.form != kFormFP8) o.qh = take((size_t)x.nq_pad * v.ld16 * 2);
    if (x.form == kFormExact) o.ql = take((size_t)x.nq_pad * v.ld16 * 2);
    if (x.form == kFormFP8) o.q8 = take((size_t)x.nq_pad * v.ld8);
    o.qn = take((size_t)x.nq_pad * 4);
    o.qs = take((size_t)x.nq_pad * 4);
    o.counts = take(lists * 4);
    o.pools = take(lists * (size_t)x.P * 8);
  }
  b->ws_bytes = (size_t)rup((long long)off, 256) + 256;
  BT_TRY(cudaMalloc(&b->ws, b->ws_bytes));
  char* base = static_cast<char*>(b->ws);
  b->status = reinterpret_cast<uint32_t*>(base + o_status);
  for (size_t fi = 0; fi < b->fitems.size(); ++fi) {
    FItem& x = b->fitems[fi];
    const IndexView& v = b->views[x.slot];
    const Offs& o = offs[fi];
    FusedItemSpec& s = x.spec;
    s.nq = x.nq;
    s.nb = (int)v.n;
    s.d = v.dim;
    s.kprime = x.kp;
    s.pool_cap = x.P;
    s.nq_pad = x.nq_pad;
    s.nb_pad = v.n_pad;
    s.ld16 = v.ld16;
    s.ld8 = v.ld8;
    s.q_bound = reinterpret_cast<uint32_t*>(base + o.bounds);
    s.q_bound_half = s.q_bound + x.nq_pad;
    if (v.n == 0) continue;
    s.qh = o.qh ? reinterpret_cast<__nv_bfloat16*>(base + o.qh) : nullptr;
    s.ql = o.ql ? reinterpret_cast<__nv_bfloat16*>(base + o.ql) : nullptr;
    s.q8 = o.q8 ? reinterpret_cast<uint8_t*>(base + o.q8) : nullptr;
    s.qn = reinterpret_cast<float*>(base + o.qn);
    s.qs = reinterpret_cast<float*>(base + o.qs);
    s.xh = v.xh;
    s.xl = v.xl;
    s.x8 = v.x8;
    s.xn = v.xn;
    s.xs = v.xs;
    s.pool_counts = reinterpret_cast<int*>(base + o.counts);
    s.pools = reinterpret_cast<uint64_t*>(base + o.pools);
  }

  // ---- capture
  for (const Group& G : b->groups) {
    BT_TRY(prepare_fused_kernels(G.form));
  }
  BT_TRY(prepare_merge_kernel());
  if (!b->cap) BT_TRY(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  if (!b->fork) BT_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  for (Group& G : b->groups) {
    BT_TRY(cudaStreamCreateWithFlags(&G.branch, cudaStreamNonBlocking));
    BT_TRY(cudaEventCreateWithFlags(&G.join, cudaEventDisableTiming));
  }
  int kernels = 0;
  BT_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
  auto enqueue = [&]() -> int {
    BT_TRY(cudaMemsetAsync(b->status, 0, sizeof(uint32_t), b->cap));
    if (bounds_words) BT_TRY(cudaMemsetAsync(base + o_bounds, 0xFF, bounds_words * sizeof(uint32_t), b->cap));
    BT_TRY(cudaEventRecord(b->fork, b->cap));
    for (Group& G : b->groups) {
      cudaStream_t st = G.branch;
      BT_TRY(cudaStreamWaitEvent(st, b->fork, 0));
      // query prep: one segment per member, plus the padding rows of each fused item
      std::vector<PrepSegment> segs;
      auto flush_prep = [&]() -> int {
        if (segs.empty()) return CURPLSH_OK;
        const int aug = G.form == kFormFP8 ? kAugNone : kAugQuery;
        BT_TRY(launch_prep_segments(segs.data(), (int)segs.size(), G.d, G.ld16, G.ld8, 0.f, aug, st));
        ++kernels;
        segs.clear();
        return CURPLSH_OK;
      };
      for (int fi : G.fitems) {
        const FItem& x = b->fitems[fi];
        if (b->views[x.slot].n == 0) continue;
        const FusedItemSpec& s = x.spec;
        auto seg_at = [&](const float* src, int nrows, int rows, long long r0) {
          PrepSegment g{};
          g.x = src;
          g.nrows = nrows;
          g.rows = rows;
          g.norms = const_cast<float*>(s.qn) + r0;
          g.scale = const_cast<float*>(s.qs) + r0;
          g.hi = s.qh ? const_cast<__nv_bfloat16*>(s.qh) + r0 * G.ld16 : nullptr;
          g.lo = s.ql ? const_cast<__nv_bfloat16*>(s.ql) + r0 * G.ld16 : nullptr;
          g.f8 = s.q8 ? const_cast<uint8_t*>(s.q8) + r0 * G.ld8 : nullptr;
          return g;
        };
        for (size_t j = 0; j < x.members.size(); ++j) {
          const curplsh_batch_item& it = b->items[x.members[j]];
          if ((int)segs.size() == kPrepMaxSegments) {
            int rc = flush_prep();
            if (rc) return rc;
          }
          segs.push_back(seg_at(it.queries, (int)it.num, (int)it.num, x.row0[j]));
        }
        if (x.nq_pad > x.nq) {
          if ((int)segs.size() == kPrepMaxSegments) {
            int rc = flush_prep();
            if (rc) return rc;
          }
          segs.push_back(seg_at(nullptr, 0, (int)(x.nq_pad - x.nq), x.nq));
        }
      }
      int rc = flush_prep();
      if (rc) return rc;
      // fused filter
      for (const FLaunch& FL : G.launches) {
        std::vector<FusedItemSpec> specs;
        std::vector<FusedItemPlan> plans;
        for (int fi : FL.fitems) {
          specs.push_back(b->fitems[fi].spec);
          plans.push_back(b->fitems[fi].plan);
        }
        BT_TRY(launch_fused_batch(G.form, specs.data(), plans.data(), (int)specs.size(), FL.bp, b->status, nullptr,
                                  st));
        if (FL.bp.grid > 0) ++kernels;
      }
      // merge + exact rerank: one item per member; one launch per power-of-two
      // class of k' so that small-k items do not reserve the shared memory of
      // the largest k'
      std::map<int, std::vector<MergeItem>> by_class;
      for (int fi : G.fitems) {
        const FItem& x = b->fitems[fi];
        const IndexView& v = b->views[x.slot];
        int cls = 32;
        while (cls < x.kp) cls <<= 1;
        for (size_t j = 0; j < x.members.size(); ++j) {
          const curplsh_batch_item& it = b->items[x.members[j]];
          MergeItem m{};
          m.nq = (int)it.num;
          m.k = it.k;
          m.kprime = x.kp;
          m.pool_cap = x.P;
          m.num_tiles = v.n > 0 ? x.plan.num_tiles : 0;
          m.units_per_block = v.n > 0 ? x.plan.units_per_block : 1;
          m.row0 = x.row0[j];
          m.split_tiles = v.n > 0 ? x.plan.split_tiles : 1;
          m.work_begin = x.plan.work_begin;
          m.work_per_cta = x.W;
          m.pools = x.spec.pools;
          m.pool_counts = x.spec.pool_counts;
          m.q_bound = x.spec.q_bound;
          m.q_bound_half = x.spec.q_bound_half;
          m.queries = it.queries;
          m.db = v.x32;
          m.ld_db = v.dim;
          m.out_idx = it.indices;
          m.out_dist = it.distances;
          by_class[cls].push_back(m);
        }
      }
      for (auto& kv : by_class) {
        std::vector<MergeItem>& all = kv.second;
        for (size_t s0 = 0; s0 < all.size(); s0 += kMergeMaxItems) {
          const int cnt = (int)std::min<size_t>(kMergeMaxItems, all.size() - s0);
          BT_TRY(launch_merge_batch(all.data() + s0, cnt, G.d, b->status, st));
          ++kernels;
        }
      }
      BT_TRY(cudaEventRecord(G.join, st));
      BT_TRY(cudaStreamWaitEvent(b->cap, G.join, 0));
    }
    return CURPLSH_OK;
  };
  int rc = enqueue();
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
