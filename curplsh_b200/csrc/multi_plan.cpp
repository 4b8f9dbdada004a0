// multi_plan.cpp -- see multi_plan.h.
#include "multi_plan.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <map>
#include <tuple>

#include "common.cuh"

namespace curplsh_b200 {
namespace {

// An item whose tiles would span fewer CTA ranges than this in its group's
// combined launch gets a launch of its own.
#ifndef CURPLSH_SOLO_CTAS
#define CURPLSH_SOLO_CTAS 16
#endif
constexpr long long kSoloCtas = CURPLSH_SOLO_CTAS;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return record_error(code, buf);
}

#define MP_TRY(call)                                                                                  \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) {                                                                          \
      cudaGetLastError();                                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? CURPLSH_ERR_OOM : CURPLSH_ERR_CUDA, "%s: %s", #call, \
                  cudaGetErrorString(e_));                                                            \
    }                                                                                                 \
  } while (0)

long long rup(long long x, long long m) { return (x + m - 1) / m * m; }

}  // namespace

int MultiPlan::build(const curplsh_batch_item* items, int n, const std::vector<curplsh_index*>& uniq,
                     std::vector<IndexView>& views, int precision, int rerank_factor, int num_sms) {
  items_.assign(items, items + n);
  fitems_.clear();
  groups_.clear();
  base_ = nullptr;
  status_ = nullptr;
  const bool use_est = bound_estimate_enabled();  // read once: planning and enqueue agree

  // ---- fused items: (index, form, k') -> concatenated queries
  std::map<std::tuple<int, int, int>, int> fmap;
  for (int i = 0; i < n; ++i) {
    const curplsh_batch_item& it = items[i];
    if (it.num == 0) continue;
    const int slot = (int)(std::lower_bound(uniq.begin(), uniq.end(), it.index) - uniq.begin());
    IndexView& v = views[slot];
    const int form = precision < 0 ? v.precision : precision;
    const int rf = rerank_factor > 0 ? rerank_factor : v.rerank_factor;
    int rc = index_prepare_form(uniq[slot], form, &v);
    if (rc) return rc;
    const int kp = search_kprime(form, it.k, rf, v.n);
    auto key = std::make_tuple(slot, form, kp);
    auto f = fmap.find(key);
    int fi;
    if (f == fmap.end()) {
      fi = (int)fitems_.size();
      fmap.emplace(key, fi);
      FItem x;
      x.slot = slot;
      x.form = form;
      x.kp = kp;
      x.d = v.dim;
      x.k = it.k;
      fitems_.push_back(x);
    } else {
      fi = f->second;
    }
    FItem& x = fitems_[fi];
    if ((long long)x.nq + it.num > (1LL << 30))
      return fail(CURPLSH_ERR_UNSUPPORTED, "more than 2^30 queries against one index in one plan");
    x.members.push_back(i);
    x.row0.push_back(x.nq);
    x.nq += (int)it.num;
  }
  // tuned parameters per fused item, looked up with its concatenated query count
  for (FItem& x : fitems_) {
    x.tune = tune_lookup(x.form, x.d, x.k, x.nq);
    x.P = search_pool_capacity(x.kp, x.tune.headroom);
    x.nq_pad = rup(x.nq, kBM);
  }
  // ---- groups by (form, d)
  std::map<std::pair<int, int>, int> gmap;
  for (size_t fi = 0; fi < fitems_.size(); ++fi) {
    const FItem& x = fitems_[fi];
    const IndexView& v = views[x.slot];
    auto key = std::make_pair(x.form, x.d);
    auto g = gmap.find(key);
    int gi;
    if (g == gmap.end()) {
      gi = (int)groups_.size();
      gmap.emplace(key, gi);
      Group G;
      G.form = x.form;
      G.d = x.d;
      G.ld16 = v.ld16;
      G.ld8 = v.ld8;
      groups_.push_back(G);
    } else {
      gi = g->second;
    }
    groups_[gi].fitems.push_back((int)fi);
  }
  for (Group& G : groups_) {
    // Every group's persistent launch asks for all SMs: when groups run as
    // parallel branches the hardware starts a later group's CTAs on the SMs an
    // earlier group releases, while a static split of the SMs by tile count
    // would leave the groups whose tiles are dearer (larger d, larger k') as
    // the long pole.
    //
    // A launch splits its flattened (item, query block, tile) space into equal
    // contiguous CTA ranges by tile count, so an item with few tiles lands on
    // one or two CTAs; when its tiles are dear (a large k' against a small
    // database, where every row survives) those CTAs become the launch's tail.
    // An item whose work would span fewer than kSoloCtas CTA ranges of the
    // combined launch therefore gets a launch of its own (spread over every
    // SM); the larger items share one.
    long long work_all = 0;
    auto work_of = [&](int fi) {
      const FItem& x = fitems_[fi];
      return (long long)((x.nq + kBM - 1) / kBM) * ((views[x.slot].n + kBN - 1) / kBN);
    };
    for (int fi : G.fitems) work_all += work_of(fi);
    const long long w_comb = std::max<long long>(1, (work_all + num_sms - 1) / num_sms);
    FLaunch L;
    for (int fi : G.fitems) {
      if (views[fitems_[fi].slot].n == 0) continue;
      if (work_of(fi) < kSoloCtas * w_comb) {
        FLaunch S;
        S.fitems.push_back(fi);
        G.launches.push_back(S);
        continue;
      }
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
        const FItem& x = fitems_[FL.fitems[j]];
        specs[j].nq = x.nq;
        specs[j].nb = (int)views[x.slot].n;
        specs[j].d = G.d;
        // units as long as the item's own CTA ranges would be if it were
        // searched alone (scaled by the tuned split, at most the whole range,
        // as alone), so its in-pool selection work stays what it is alone
        const long long own = (long long)((x.nq + kBM - 1) / kBM) * ((specs[j].nb + kBN - 1) / kBN);
        specs[j].split_tiles = split_tiles_for(std::max<long long>(1, (own + num_sms - 1) / num_sms),
                                               std::min(default_split_q4(x.tune, x.P), 4));
      }
      plan_fused_batch(specs.data(), (int)specs.size(), num_sms, plans.data(), &FL.bp, G.form);
      for (size_t j = 0; j < FL.fitems.size(); ++j) {
        FItem& x = fitems_[FL.fitems[j]];
        x.plan = plans[j];
        x.W = FL.bp.work_per_cta;
        x.launch = (int)(&FL - G.launches.data());
        if (use_est) x.est = plan_estimate(x.nq, views[x.slot].n, x.kp, num_sms);
        FL.est_any = FL.est_any || x.est.on;
      }
    }
  }
  // ---- working memory: [status][all bounds][per fused item operands, counts, pools]
  size_t off = 0;
  auto take = [&](size_t bytes) {
    off = (size_t)rup((long long)off, 256);
    const size_t o = off;
    off += bytes;
    return o;
  };
  o_status_ = take(sizeof(uint32_t));
  bounds_words_ = 0;
  for (const FItem& x : fitems_) bounds_words_ += (size_t)x.nq_pad;
  o_bounds_ = take(bounds_words_ * sizeof(uint32_t));
  // failure lists of the launches that verify an estimate, in one region
  // (cleared by one memset per run)
  size_t fail_ints = 0;
  for (Group& G : groups_)
    for (FLaunch& FL : G.launches) {
      if (!FL.est_any) continue;
      FL.o_fail = fail_ints * sizeof(int);
      fail_ints += 2;
      for (int fi : FL.fitems) fail_ints += (size_t)fitems_[fi].nq;
      fail_ints = (size_t)rup((long long)fail_ints, 64);
    }
  fails_bytes_ = fail_ints * sizeof(int);
  o_fails_ = take(fails_bytes_);
  for (Group& G : groups_)
    for (FLaunch& FL : G.launches)
      if (FL.est_any) FL.o_fail += o_fails_;
  size_t bcur = 0;
  for (FItem& x : fitems_) {
    const IndexView& v = views[x.slot];
    x.o_bounds = o_bounds_ + bcur * sizeof(uint32_t);
    bcur += (size_t)x.nq_pad;
    if (v.n == 0) continue;
    const size_t lists = (size_t)x.plan.num_qblocks * ((size_t)kBM << (x.plan.pair | x.plan.dual)) *
                         x.plan.units_per_block;
    if (x.form != kFormFP8) x.o_qh = take((size_t)x.nq_pad * v.ld16 * 2);
    if (x.form == kFormExact) x.o_ql = take((size_t)x.nq_pad * v.ld16 * 2);
    if (x.form == kFormFP8) x.o_q8 = take((size_t)x.nq_pad * v.ld8);
    x.o_qn = take((size_t)x.nq_pad * 4);
    x.o_qs = take((size_t)x.nq_pad * 4);
    x.o_counts = take(lists * 4);
    x.o_pools = take(lists * (size_t)x.P * 8);
    if (x.est.on) x.o_minima = take((size_t)x.nq_pad * x.est.blocks * sizeof(float));
  }
  bytes_ = (size_t)rup((long long)off, 256) + 256;
  views_ = views;
  return CURPLSH_OK;
}

void MultiPlan::bind(void* base_v) {
  char* base = static_cast<char*>(base_v);
  base_ = base;
  status_ = reinterpret_cast<uint32_t*>(base + o_status_);
  for (FItem& x : fitems_) {
    const IndexView& v = views_[x.slot];
    FusedItemSpec& s = x.spec;
    s = FusedItemSpec{};
    s.nq = x.nq;
    s.nb = (int)v.n;
    s.d = v.dim;
    s.kprime = x.kp;
    s.pool_cap = x.P;
    s.nq_pad = x.nq_pad;
    s.nb_pad = v.n_pad;
    s.ld16 = v.ld16;
    s.ld8 = v.ld8;
    s.q_bound = reinterpret_cast<uint32_t*>(base + x.o_bounds);
    if (v.n == 0) continue;
    s.qh = x.o_qh ? reinterpret_cast<__nv_bfloat16*>(base + x.o_qh) : nullptr;
    s.ql = x.o_ql ? reinterpret_cast<__nv_bfloat16*>(base + x.o_ql) : nullptr;
    s.q8 = x.o_q8 ? reinterpret_cast<uint8_t*>(base + x.o_q8) : nullptr;
    s.qn = reinterpret_cast<float*>(base + x.o_qn);
    s.qs = reinterpret_cast<float*>(base + x.o_qs);
    s.xh = v.xh;
    s.xl = v.xl;
    s.x8 = v.x8;
    s.xn = v.xn;
    s.xs = v.xs;
    s.xs_uniform = v.xs_uniform;
    s.pool_counts = reinterpret_cast<int*>(base + x.o_counts);
    s.pools = reinterpret_cast<uint64_t*>(base + x.o_pools);
  }
}

int MultiPlan::enqueue(cudaStream_t main, const std::vector<cudaStream_t>* branches,
                       const std::vector<cudaEvent_t>* joins, cudaEvent_t fork, int* kernels_out) const {
  int kernels = 0;
  MP_TRY(cudaMemsetAsync(status_, 0, sizeof(uint32_t), main));
  if (bounds_words_) MP_TRY(cudaMemsetAsync(base_ + o_bounds_, 0xFF, bounds_words_ * sizeof(uint32_t), main));
  if (fails_bytes_) MP_TRY(cudaMemsetAsync(base_ + o_fails_, 0, fails_bytes_, main));
  const bool fan = branches && joins && fork && groups_.size() > 1;
  if (fan) MP_TRY(cudaEventRecord(fork, main));
  for (size_t gi = 0; gi < groups_.size(); ++gi) {
    const Group& G = groups_[gi];
    cudaStream_t st = fan ? (*branches)[gi] : main;
    if (fan) MP_TRY(cudaStreamWaitEvent(st, fork, 0));
    // query prep: one segment per member, plus the padding rows of each fused item
    std::vector<PrepSegment> segs;
    auto flush_prep = [&]() -> int {
      if (segs.empty()) return CURPLSH_OK;
      const int aug = G.form == kFormFP8 ? kAugF8Query : kAugQuery;
      MP_TRY(launch_prep_segments(segs.data(), (int)segs.size(), G.d, G.ld16, G.ld8, 0.f, aug, st));
      ++kernels;
      segs.clear();
      return CURPLSH_OK;
    };
    for (int fi : G.fitems) {
      const FItem& x = fitems_[fi];
      if (views_[x.slot].n == 0) continue;
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
        const curplsh_batch_item& it = items_[x.members[j]];
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
    // sampled bound estimates: the block-minimum pass over the sample and the
    // rank select, which overwrites the item's all-ones bounds
    for (int fi : G.fitems) {
      const FItem& x = fitems_[fi];
      if (!x.est.on) continue;
      const FusedItemSpec& s = x.spec;
      FusedLaunch e{};
      e.nq = s.nq;
      e.nb = x.est.rows;
      e.d = s.d;
      e.kprime = 1;
      e.pool_cap = s.pool_cap;
      e.form = G.form;
      e.nq_pad = s.nq_pad;
      e.nb_pad = x.est.rows;
      e.ld16 = s.ld16;
      e.ld8 = s.ld8;
      e.qh = s.qh;
      e.ql = s.ql;
      e.q8 = s.q8;
      e.qn = s.qn;
      e.qs = s.qs;
      e.xh = s.xh;
      e.xl = s.xl;
      e.x8 = s.x8;
      e.xn = s.xn;
      e.xs = s.xs;
      e.xs_uniform = s.xs_uniform;
      e.db_step = x.est.step;
      e.minima = reinterpret_cast<float*>(base_ + x.o_minima);
      e.pools = s.pools;
      e.pool_counts = s.pool_counts;
      e.q_bound = s.q_bound;
      e.status = status_;
      e.plan = x.est.plan;
      MP_TRY(launch_fused(e, st));
      MP_TRY(launch_estimate_select(e.minima, x.est.blocks, x.nq, x.est.j, s.q_bound, st));
      kernels += 2;
    }
    // fused filter
    auto fused_launch = [&](const FLaunch& FL, const int* run_if) -> int {
      std::vector<FusedItemSpec> specs;
      std::vector<FusedItemPlan> plans;
      for (int fi : FL.fitems) {
        specs.push_back(fitems_[fi].spec);
        plans.push_back(fitems_[fi].plan);
      }
      MP_TRY(launch_fused_batch(G.form, specs.data(), plans.data(), (int)specs.size(), FL.bp, status_, nullptr, st,
                                run_if));
      if (FL.bp.grid > 0) ++kernels;
      return CURPLSH_OK;
    };
    for (const FLaunch& FL : G.launches) {
      rc = fused_launch(FL, nullptr);
      if (rc) return rc;
    }
    // merge + exact rerank: one item per member; one launch per power-of-two
    // class of k' so that small-k requests do not reserve the shared memory
    // of the largest k'.  `only` (>= 0) restricts it to the items of one fused
    // launch, the fallback's merges after a failed estimate (no checks, run
    // only when the launch's failure count is nonzero).
    auto merge_items = [&](int only, std::map<int, std::vector<MergeItem>>& by_class) {
      for (int fi : G.fitems) {
        const FItem& x = fitems_[fi];
        const IndexView& v = views_[x.slot];
        if (only >= 0 && x.launch != only) continue;
        int* fcnt = (x.est.on && only < 0) ? reinterpret_cast<int*>(base_ + G.launches[x.launch].o_fail) : nullptr;
        int cls = 32;
        while (cls < x.kp) cls <<= 1;
        for (size_t j = 0; j < x.members.size(); ++j) {
          const curplsh_batch_item& it = items_[x.members[j]];
          MergeItem m{};
          m.nq = (int)it.num;
          m.k = it.k;
          m.kprime = x.kp;
          m.pool_cap = x.P;
          m.num_tiles = v.n > 0 ? x.plan.num_tiles : 0;
          m.units_per_block = v.n > 0 ? x.plan.units_per_block : 1;
          m.pair = x.plan.pair | x.plan.dual;
          m.row0 = x.row0[j];
          m.split_tiles = v.n > 0 ? x.plan.split_tiles : 1;
          m.work_begin = x.plan.work_begin;
          m.work_per_cta = x.W;
          m.pools = x.spec.pools;
          m.pool_counts = x.spec.pool_counts;
          m.q_bound = x.spec.q_bound;
          m.checks = fcnt ? kCheckEstimate : 0;
          m.nb_total = v.n;
          m.fail_count = fcnt;
          m.fail_list = fcnt ? fcnt + 2 : nullptr;
          m.coarse_count = nullptr;
          m.queries = it.queries;
          m.db = v.x32;
          m.ld_db = v.dim;
          m.db16 = v.bf16_exact ? v.xh : nullptr;
          m.ld16 = v.ld16;
          m.out_idx = it.indices;
          m.out_dist = it.distances;
          by_class[cls].push_back(m);
        }
      }
    };
    auto merge_launches = [&](std::map<int, std::vector<MergeItem>>& by_class, const int* run_if) -> int {
      for (auto& kv : by_class) {
        std::vector<MergeItem>& all = kv.second;
        for (size_t s0 = 0; s0 < all.size(); s0 += kMergeMaxItems) {
          const int cnt = (int)std::min<size_t>(kMergeMaxItems, all.size() - s0);
          MP_TRY(launch_merge_batch(all.data() + s0, cnt, G.d, status_, st, run_if));
          ++kernels;
        }
      }
      return CURPLSH_OK;
    };
    {
      std::map<int, std::vector<MergeItem>> by_class;
      merge_items(-1, by_class);
      rc = merge_launches(by_class, nullptr);
      if (rc) return rc;
    }
    // fallback chains: a launch with a failed estimate runs again without it
    for (size_t li = 0; li < G.launches.size(); ++li) {
      const FLaunch& FL = G.launches[li];
      if (!FL.est_any) continue;
      const int* fcnt = reinterpret_cast<const int*>(base_ + FL.o_fail);
      for (int fi : FL.fitems) {
        const FItem& x = fitems_[fi];
        MP_TRY(launch_fill_u32_if(x.spec.q_bound, x.nq_pad, 0xFFFFFFFFu, fcnt, st));
        ++kernels;
      }
      rc = fused_launch(FL, fcnt);
      if (rc) return rc;
      std::map<int, std::vector<MergeItem>> by_class;
      merge_items((int)li, by_class);
      rc = merge_launches(by_class, fcnt);
      if (rc) return rc;
    }
    if (fan) {
      MP_TRY(cudaEventRecord((*joins)[gi], st));
      MP_TRY(cudaStreamWaitEvent(main, (*joins)[gi], 0));
    }
  }
  if (kernels_out) *kernels_out = kernels;
  return CURPLSH_OK;
}

}  // namespace curplsh_b200
