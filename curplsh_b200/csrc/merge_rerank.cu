// merge_rerank.cu -- per-query merge of the candidate pools and exact rerank.
//
// Replaces the reference's final cross-tile merge and exact-distance epilogue
// (cuRPLSH paths):
//   blockSelect with given indices     src/internal/select.cu:54-96, :275-322
//   broadcastAlongRowsSum (+ ||q||^2)  src/internal/broadcast.cu:15-74
// One CTA per query:
//   1. block radix-select of the k' smallest (coarse distance, row) keys over
//      every pool that covered this query (the union is exact: see the fused
//      pass), so the candidate set does not depend on scheduling;
//   2. exact FP32 rerank: sum_i (q_i - x_i)^2 evaluated directly (no
//      ||q||^2 + ||x||^2 - 2 q.x cancellation), one warp per candidate with a
//      fixed reduction order;
//   3. bitonic sort by (exact distance, row) -- lower row first on ties -- and
//      write the first k; missing results are (-1, FLT_MAX) as in
//      src/internal/search.cu:94-101.
#include <algorithm>
#include <cstring>

#include <cuda_bf16.h>

#include "common.cuh"
#include "fused_knn.h"

namespace curplsh_b200 {

namespace {

// Threads per query's CTA: 128 or 256, chosen per launch (the radix histogram
// has 256 bins, 256 / threads per thread).  128-thread CTAs put twice as many
// queries in flight per SM at the same register budget and win where a
// query's rerank is small (k' x d <= 65536: merge of a 10^4-query BF16 search
// at k' = 224, d = 128, 0.32 -> 0.28 ms); 256 win where it is large (the
// batched workload, d up to 512: 93 -> 74 ms per graph replay).
constexpr int kMergeSmallRerank = 65536;
// Candidates one warp reranks at once: each lane keeps this many database rows
// in flight (a row of d = 128 is one 16-byte load per lane).
#ifndef CURPLSH_RERANK_ROWS
#define CURPLSH_RERANK_ROWS 4
#endif
constexpr int kRerankRows = CURPLSH_RERANK_ROWS;

__device__ __forceinline__ uint32_t block_incl_scan(uint32_t v, uint32_t* warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) warp_tot[warp] = v;
  __syncthreads();
  uint32_t add = 0;
  for (int w = 0; w < warp; ++w) add += warp_tot[w];
  __syncthreads();
  return v + add;
}

struct MergeArgs {
  MergeItem items[kMergeMaxItems];
  int num_items, d;
  int kp2;      // power of two >= the largest kprime
  int pre_cap;  // capacity of the prefiltered key buffer (2 * kp2)
  int lcnt_n;   // room for the largest list count, rounded to 4
  int vec4;     // query and database rows allow 16-byte loads
  uint32_t* status;
  const int* run_if;  // non-null: the launch does nothing unless *run_if != 0
};

// Block-wide radix select: the bound B such that exactly `keep` of the keys
// visited by `each` are <= B (keys are unique).  `each(f)` calls f(key) for
// every key of this thread's share.  8-bit digits from the top; stops as soon
// as the digit bucket holds exactly the remaining rank.
template <int T, class Each>
__device__ uint64_t block_select_bound(Each each, uint32_t keep, uint32_t* hist, uint32_t* warp_tot,
                                       uint32_t* misc) {
  const int tid = threadIdx.x;
  uint64_t prefix = 0, pmask = 0;
  uint32_t rank = keep;
  for (int shift = 56; shift >= 0; shift -= 8) {
#pragma unroll
    for (int b = 0; b < (256 / T); ++b) hist[tid * (256 / T) + b] = 0u;
    __syncthreads();
    each([&](uint64_t key) {
      if ((key & pmask) == prefix) atomicAdd(&hist[(uint32_t)(key >> shift) & 255u], 1u);
    });
    __syncthreads();
    uint32_t cb[(256 / T)], c = 0;
#pragma unroll
    for (int b = 0; b < (256 / T); ++b) {
      cb[b] = hist[tid * (256 / T) + b];
      c += cb[b];
    }
    const uint32_t incl = block_incl_scan(c, warp_tot);
    uint32_t excl = incl - c;
#pragma unroll
    for (int b = 0; b < (256 / T); ++b) {
      if (excl < rank && rank <= excl + cb[b]) {
        misc[1] = (uint32_t)(tid * (256 / T) + b);
        misc[2] = excl;
        misc[3] = cb[b];
      }
      excl += cb[b];
    }
    __syncthreads();
    const uint32_t digit = misc[1], before = misc[2], cnt = misc[3];
    prefix |= (uint64_t)digit << shift;
    pmask |= 0xFFull << shift;
    rank -= before;
    __syncthreads();
    if (cnt == rank || shift == 0) return prefix | ~pmask;
  }
  return ~0ull;
}

// Resident CTAs per SM the register allocation must allow: each query's CTA
// spends most of its time waiting on gathers and barriers, so occupancy hides
// latency.  Unbounded, the 256-thread kernel took 96 registers (2 CTAs per
// SM); at 6 CTAs (40 registers, a few spills) the merge of a 10^4-query search
// dropped from 0.62 to 0.32 ms (BF16, k' = 224).  12 for 128 threads: the same
// 40-register budget.
template <int NT>
__global__ void __launch_bounds__(NT, NT == 128 ? 12 : 6) merge_rerank_kernel(const __grid_constant__ MergeArgs a) {
  if (a.run_if && *a.run_if == 0) return;  // a conditional re-merge whose check passed
  int lo = 0, hi = a.num_items - 1;  // last item with q_begin <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.items[mid].q_begin <= (long long)blockIdx.x)
      lo = mid;
    else
      hi = mid - 1;
  }
  const MergeItem& m = a.items[lo];
  const int q = (int)((long long)blockIdx.x - m.q_begin);
  if (q >= m.nq) return;
  const int d = a.d;
  extern __shared__ __align__(16) uint8_t sm[];
  uint64_t* cand = reinterpret_cast<uint64_t*>(sm);             // [kp2] kept keys, then reranked keys
  uint64_t* pre = cand + a.kp2;                                 // [pre_cap] keys that pass the final bound
  uint32_t* hist = reinterpret_cast<uint32_t*>(pre + a.pre_cap);  // [256]
  uint32_t* warp_tot = hist + 256;                              // [8]
  uint32_t* misc = warp_tot + 8;                                // [8]
  int* lcnt = reinterpret_cast<int*>(misc + 8);                 // [lcnt_n]
  float* qv = reinterpret_cast<float*>(lcnt + a.lcnt_n);        // [d], 16-byte aligned

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int prow = m.row0 + q;  // pool row within the fused item
  const int qb = prow / (kBM << m.pair);  // query block (group of two with CTA pairs)
  const int T = m.num_tiles, U = m.units_per_block;
  const long long W = m.work_per_cta;
  const long long first = (m.work_begin + (long long)qb * T) / W;
  const long long last = (m.work_begin + (long long)(qb + 1) * T - 1) / W;
  // an empty database has no pools; otherwise one list per unit
  const int nlists = T > 0 ? (int)(last - first + 1 + (T - 1) / m.split_tiles) : 0;
  const size_t list0 = (size_t)prow * U;  // pool-list index of unit 0
  // Final bound of the fused pass on this query's k'-th coarse distance: the
  // smallest k'-th of any pool, or the estimate the pass started from.  When
  // it comes from a pool, every key of the k' smallest has a distance <= it.
  uint32_t qbound = 0xFFFFFFFFu;
  if (m.q_bound && T > 0 && a.pre_cap > 0) qbound = m.q_bound[prow];

  for (int i = tid; i < d; i += NT) qv[i] = m.queries[(size_t)q * d + i];
  if (tid == 0) {
    misc[0] = 0;
    misc[4] = 0;
    misc[5] = 0u;            // max over candidates of (coarse - exact), order bits
    misc[6] = 0xFFFFFFFFu;   // min of the same
    misc[7] = 0u;            // largest coarse distance among the candidates, order bits
  }
  for (int l = tid; l < nlists; l += NT) lcnt[l] = m.pool_counts[list0 + l];
  __syncthreads();
  auto list_ptr = [&](int l) { return m.pools + (list0 + (size_t)l) * (size_t)m.pool_cap; };
  auto each_pool_key = [&](auto f) {
    for (int l = 0; l < nlists; ++l) {
      const uint64_t* lp = list_ptr(l);
      for (int o = tid; o < lcnt[l]; o += NT) {
        const uint64_t key = lp[o];
        if ((uint32_t)(key >> 32) <= qbound) f(key);
      }
    }
  };

  // ---- 1. keys under the final bound, compacted into shared memory (when
  // this launch's pools can carry bounds at all)
  int cnt = 0;
  if (a.pre_cap > 0) {
    each_pool_key([&](uint64_t key) {
      const uint32_t pos = atomicAdd(&misc[0], 1u);
      if (pos < (uint32_t)a.pre_cap) pre[pos] = key;
    });
    __syncthreads();
    cnt = (int)misc[0];
  } else {
    for (int l = 0; l < nlists; ++l) cnt += lcnt[l];
  }
  // Started from an estimate E: every row with a key under E was admitted, so
  // k' keys under the final bound (<= E) prove that the k' smallest keys of
  // the whole database are among the candidates (their k'-th is then <= E, and
  // a pool selection never drops one of them).  Fewer: E may have been too
  // small, and the query is listed for a search without the estimate.
  const bool listed = (m.checks & kCheckEstimate) && cnt < m.kprime;  // each query is listed at most once
  if (listed && tid == 0) {
    const int pos = atomicAdd(m.fail_count, 1);
    m.fail_list[pos] = q;
  }
  const int keep = cnt < m.kprime ? cnt : m.kprime;
  // ---- 2. select the k' smallest (in shared memory unless too many passed)
  uint64_t bound = ~0ull;
  if (cnt > keep) {
    if (cnt <= a.pre_cap)
      bound = block_select_bound<NT>(
          [&](auto f) {
            for (int i = tid; i < cnt; i += NT) f(pre[i]);
          },
          (uint32_t)keep, hist, warp_tot, misc);
    else
      bound = block_select_bound<NT>(each_pool_key, (uint32_t)keep, hist, warp_tot, misc);
  }
  if (cnt <= a.pre_cap) {
    for (int i = tid; i < cnt; i += NT) {
      const uint64_t key = pre[i];
      if (key <= bound) {
        const uint32_t pos = atomicAdd(&misc[4], 1u);
        if (pos < (uint32_t)a.kp2) cand[pos] = key;
      }
    }
  } else {
    each_pool_key([&](uint64_t key) {
      if (key <= bound) {
        const uint32_t pos = atomicAdd(&misc[4], 1u);
        if (pos < (uint32_t)a.kp2) cand[pos] = key;
      }
    });
  }
  __syncthreads();
  int kept = (int)misc[4];
  if (kept > a.kp2) {
    if (tid == 0) atomicOr(a.status, kErrPoolOverflow);
    kept = a.kp2;
  }
  // ---- 3. exact FP32 rerank: one warp per group of kRerankRows candidates
  // (that many rows in flight per lane), lane-strided partial sums then a
  // butterfly, in the same fixed order for every row
  constexpr int R = kRerankRows;
  for (int c = R * warp; c < kept; c += R * (NT / 32)) {
    uint32_t ii[R];
    float s[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      ii[r] = (uint32_t)(cand[c + r < kept ? c + r : c] & 0xFFFFFFFFu);
      s[r] = 0.f;
    }
    if (m.db16) {
      // rows exactly representable in BF16: read half the bytes; the same
      // lane-to-element assignment and order as the FP32 path below
      if (a.vec4) {
        const float4* q4 = reinterpret_cast<const float4*>(qv);
        for (int i = lane; i < d / 4; i += 32) {
          const float4 qq = q4[i];
          uint2 u[R];
#pragma unroll
          for (int r = 0; r < R; ++r) u[r] = __ldg(reinterpret_cast<const uint2*>(m.db16 + (size_t)ii[r] * m.ld16) + i);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const float2 u01 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u[r].x));
            const float2 u23 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u[r].y));
            float t;
            t = qq.x - u01.x; s[r] = fmaf(t, t, s[r]);
            t = qq.y - u01.y; s[r] = fmaf(t, t, s[r]);
            t = qq.z - u23.x; s[r] = fmaf(t, t, s[r]);
            t = qq.w - u23.y; s[r] = fmaf(t, t, s[r]);
          }
        }
      } else {
        for (int i = lane; i < d; i += 32) {
          const float qq = qv[i];
          float x[R];
#pragma unroll
          for (int r = 0; r < R; ++r) x[r] = __bfloat162float(m.db16[(size_t)ii[r] * m.ld16 + i]);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const float t = qq - x[r];
            s[r] = fmaf(t, t, s[r]);
          }
        }
      }
    } else if (a.vec4) {
      const float4* q4 = reinterpret_cast<const float4*>(qv);
      for (int i = lane; i < d / 4; i += 32) {
        const float4 qq = q4[i];
        float4 u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = __ldg(reinterpret_cast<const float4*>(m.db + (size_t)ii[r] * m.ld_db) + i);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          float t;
          t = qq.x - u[r].x; s[r] = fmaf(t, t, s[r]);
          t = qq.y - u[r].y; s[r] = fmaf(t, t, s[r]);
          t = qq.z - u[r].z; s[r] = fmaf(t, t, s[r]);
          t = qq.w - u[r].w; s[r] = fmaf(t, t, s[r]);
        }
      }
    } else {
      for (int i = lane; i < d; i += 32) {
        const float qq = qv[i];
        float x[R];
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = __ldg(m.db + (size_t)ii[r] * m.ld_db + i);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const float t = qq - x[r];
          s[r] = fmaf(t, t, s[r]);
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int r = 0; r < R; ++r) s[r] += __shfl_xor_sync(0xffffffffu, s[r], o);
    if (lane == 0) {
      float emax = -3.402823466e38f, emin = 3.402823466e38f, cmax = -3.402823466e38f;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (c + r >= kept) break;
        if (m.checks & kCheckCoarse) {
          const float cr = ord2f((uint32_t)(cand[c + r] >> 32));
          emax = fmaxf(emax, cr - s[r]);
          emin = fminf(emin, cr - s[r]);
          cmax = fmaxf(cmax, cr);
        }
        cand[c + r] = make_key(s[r], ii[r]);
      }
      if (m.checks & kCheckCoarse) {
        atomicMax(&misc[5], f2ord(emax));
        atomicMin(&misc[6], f2ord(emin));
        atomicMax(&misc[7], f2ord(cmax));
      }
    }
  }
  for (int c = kept + tid; c < a.kp2; c += NT) cand[c] = kKeyEmpty;
  __syncthreads();
  // ---- 4. bitonic sort by (exact distance, row)
  int n2 = 1;
  while (n2 < kept) n2 <<= 1;
  for (int size = 2; size <= n2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < n2 / 2; i += NT) {
        const int lo2 = 2 * i - (i & (stride - 1));
        const int hi2 = lo2 + stride;
        const bool asc = (lo2 & size) == 0;
        const uint64_t x = cand[lo2], y = cand[hi2];
        if ((x > y) == asc) {
          cand[lo2] = y;
          cand[hi2] = x;
        }
      }
      __syncthreads();
    }
  }
  // Coarse-margin check.  Every row that is not a candidate has a coarse key
  // above the largest candidate's, cmax.  With e = coarse - exact, such a row
  // can come before the k-th exact result D_k only if its e exceeds
  // cmax - D_k.  The candidates' own errors span [emin, emax]; a query passes
  // when cmax - D_k >= emax + (emax - emin) / 2, i.e. a row outside the
  // candidates would need an error beyond the largest seen by a further half
  // spread.  (emin is pulled down by selection -- rows chosen because their
  // error was negative -- so the spread overstates the error scale, more so
  // for larger k'; half of it catches, in an emulation of E4M3 rounding, every
  // query whose candidates miss a true neighbour on the 10M-row unit-sphere
  // mixture at k' = 4k, where a third of that slack would not.)  This is a
  // check of the data against the form's precision, not a proof: it lists
  // queries whose data is too fine for the coarse form (e.g. FP8 on integer
  // rows) for an exact search again.  Exact coarse distances (spread 0)
  // always pass, since then D_k <= cmax.
  if ((m.checks & kCheckCoarse) && !listed && tid == 0 && kept >= m.kprime && kept > m.k &&
      m.kprime < m.nb_total) {
    const float emax = ord2f(misc[5]), emin = ord2f(misc[6]), cmax = ord2f(misc[7]);
    const float dk = ord2f((uint32_t)(cand[m.k - 1] >> 32));
    if (!(cmax - dk >= emax + 0.5f * (emax - emin))) {
      const int pos = atomicAdd(m.fail_count, 1);
      m.fail_list[pos] = q;
      if (m.coarse_count) atomicAdd(m.coarse_count, 1);
    }
  }
  for (int t = tid; t < m.k; t += NT) {
    int oi = -1;
    float od = 3.402823466e38f;
    if (t < kept) {
      const uint64_t key = cand[t];
      oi = (int)(uint32_t)(key & 0xFFFFFFFFu);
      od = ord2f((uint32_t)(key >> 32));
    }
    m.out_idx[(size_t)q * m.k + t] = oi;
    m.out_dist[(size_t)q * m.k + t] = od;
  }
}

}  // namespace

cudaError_t prepare_merge_kernel() {
  static bool attr_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e =
        cudaFuncSetAttribute(merge_rerank_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(merge_rerank_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    attr_done[dev & 63] = true;
  }
  return cudaSuccess;
}

cudaError_t launch_merge_batch(MergeItem* items, int n, int d, uint32_t* status, cudaStream_t st,
                               const int* run_if) {
  if (n < 1 || n > kMergeMaxItems) return cudaErrorInvalidValue;
  MergeArgs a;
  memset(&a, 0, sizeof(a));
  long long qsum = 0;
  int kpmax = 1, umax = 1;
  for (int i = 0; i < n; ++i) {
    items[i].q_begin = qsum;
    qsum += items[i].nq > 0 ? items[i].nq : 0;
    if (items[i].kprime > kpmax) kpmax = items[i].kprime;
    if (items[i].units_per_block > umax) umax = items[i].units_per_block;
    a.items[i] = items[i];
  }
  if (qsum == 0) return cudaSuccess;
  a.num_items = n;
  a.d = d;
  a.status = status;
  a.run_if = run_if;
  int kp2 = 32;  // >= 32 keeps the shared-memory carve 16-byte aligned
  while (kp2 < kpmax) kp2 <<= 1;
  a.kp2 = kp2;
  // A pool can bound the k'-th distance only if a unit covers at least k'
  // rows; without such pools there is nothing to prefilter with, and the
  // launch keeps the smaller shared-memory footprint (higher occupancy).
  bool bounded = false;
  for (int i = 0; i < n; ++i) {
    long long len = std::min<long long>(items[i].split_tiles, items[i].work_per_cta);
    len = std::min<long long>(len, items[i].num_tiles);
    bounded = bounded || (items[i].q_bound && len * kBN >= items[i].kprime);
    // the estimate check counts the keys under the final bound
    bounded = bounded || (items[i].q_bound && (items[i].checks & kCheckEstimate));
  }
  a.pre_cap = bounded ? 2 * kp2 : 0;
  a.lcnt_n = (umax + 3) & ~3;
  bool vec4 = d % 4 == 0;
  for (int i = 0; i < n; ++i)
    vec4 = vec4 && (reinterpret_cast<uintptr_t>(items[i].queries) & 15) == 0 &&
           (reinterpret_cast<uintptr_t>(items[i].db) & 15) == 0 && items[i].ld_db % 4 == 0;
  a.vec4 = vec4 ? 1 : 0;
  const size_t smem = (size_t)(a.kp2 + a.pre_cap) * 8 + (256 + 8 + 8) * 4 + (size_t)a.lcnt_n * 4 + (size_t)d * 4 + 16;
  cudaError_t e = prepare_merge_kernel();
  if (e != cudaSuccess) return e;
  if (smem > 200 * 1024 || qsum > 0x7fffffffLL) return cudaErrorInvalidValue;
  if ((long long)kpmax * d <= kMergeSmallRerank)
    merge_rerank_kernel<128><<<(unsigned)qsum, 128, smem, st>>>(a);
  else
    merge_rerank_kernel<256><<<(unsigned)qsum, 256, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_merge_rerank(const MergeLaunch& m, cudaStream_t st) {
  if (m.nq <= 0) return cudaSuccess;
  MergeItem it{};
  it.nq = m.nq;
  it.k = m.k;
  it.kprime = m.kprime;
  it.pool_cap = m.pool_cap;
  it.num_tiles = m.plan.num_tiles;
  it.units_per_block = m.plan.units_per_block;
  it.pair = m.plan.pair | m.plan.dual;
  it.row0 = 0;
  it.split_tiles = m.plan.split_tiles > 0 ? m.plan.split_tiles : 1;
  it.work_begin = 0;
  it.work_per_cta = m.plan.work_per_cta;
  it.pools = m.pools;
  it.pool_counts = m.pool_counts;
  it.q_bound = m.q_bound;
  it.checks = m.checks;
  it.nb_total = m.nb;
  it.fail_count = m.fail_count;
  it.coarse_count = m.coarse_count;
  it.fail_list = m.fail_list;
  it.queries = m.queries;
  it.db = m.db;
  it.ld_db = m.ld_db;
  it.db16 = m.db16;
  it.ld16 = m.ld16;
  it.out_idx = m.out_idx;
  it.out_dist = m.out_dist;
  return launch_merge_batch(&it, 1, m.d, m.status, st, m.run_if);
}

}  // namespace curplsh_b200
