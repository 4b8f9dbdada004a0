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
#include <cstring>

#include "common.cuh"
#include "fused_knn.h"

namespace curplsh_b200 {

namespace {

constexpr int kMergeThreads = 256;

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
  int kp2;     // power of two >= the largest kprime
  int lcnt_n;  // room for the largest 2 * units_per_block, rounded to 4
  uint32_t* status;
};

__global__ void __launch_bounds__(kMergeThreads) merge_rerank_kernel(const __grid_constant__ MergeArgs a) {
  int lo = 0, hi = a.num_items - 1;  // last item with q_begin <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.items[mid].q_begin <= (long long)blockIdx.x)
      lo = mid;
    else
      hi = mid - 1;
  }
  const int ii = lo;
  const MergeItem& m = a.items[ii];
  const int q = (int)((long long)blockIdx.x - m.q_begin);
  if (q >= m.nq) return;
  const int d = a.d;
  extern __shared__ __align__(16) uint8_t sm[];
  uint64_t* cand = reinterpret_cast<uint64_t*>(sm);                       // [kp2]
  uint32_t* hist = reinterpret_cast<uint32_t*>(cand + a.kp2);             // [256]
  uint32_t* warp_tot = hist + 256;                                         // [8]
  uint32_t* misc = warp_tot + 8;                                           // [8]
  int* lcnt = reinterpret_cast<int*>(misc + 8);                            // [lcnt_n]
  float* qv = reinterpret_cast<float*>(lcnt + a.lcnt_n);                   // [d]

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int prow = m.row0 + q;  // pool row within the fused item
  const int qb = prow / kBM, row = prow % kBM;
  const int T = m.num_tiles, U = m.units_per_block;
  const long long W = m.work_per_cta;
  const long long first = (m.work_begin + (long long)qb * T) / W;
  const long long last = (m.work_begin + (long long)(qb + 1) * T - 1) / W;
  const int nlists = T > 0 ? 2 * (int)(last - first + 1) : 0;  // an empty database has no pools
  const size_t list0 = ((size_t)qb * kBM + row) * U * 2;  // pool-list index of (u=0, h=0)

  for (int i = tid; i < d; i += kMergeThreads) qv[i] = m.queries[(size_t)q * d + i];
  if (tid == 0) misc[0] = 0;
  for (int l = tid; l < nlists; l += kMergeThreads) lcnt[l] = m.pool_counts[list0 + l];
  __syncthreads();
  int total = 0;
  for (int l = 0; l < nlists; ++l) total += lcnt[l];
  const int keep = total < m.kprime ? total : m.kprime;

  auto list_ptr = [&](int l) { return m.pools + (list0 + (size_t)l) * (size_t)m.pool_cap; };

  // ---- 1. radix-select the k' smallest keys (skipped when everything fits)
  uint64_t bound = ~0ull;
  if (total > keep) {
    uint64_t prefix = 0, pmask = 0;
    uint32_t rank = (uint32_t)keep;
    for (int shift = 56; shift >= 0; shift -= 8) {
      hist[tid] = 0u;  // kMergeThreads == 256 bins
      __syncthreads();
      for (int l = 0; l < nlists; ++l) {
        const uint64_t* lp = list_ptr(l);
        for (int o = tid; o < lcnt[l]; o += kMergeThreads) {
          const uint64_t key = lp[o];
          if ((key & pmask) == prefix) atomicAdd(&hist[(uint32_t)(key >> shift) & 255u], 1u);
        }
      }
      __syncthreads();
      const uint32_t c = hist[tid];
      const uint32_t incl = block_incl_scan(c, warp_tot);
      const uint32_t excl = incl - c;
      if (excl < rank && rank <= incl) {
        misc[1] = (uint32_t)tid;
        misc[2] = excl;
        misc[3] = c;
      }
      __syncthreads();
      const uint32_t digit = misc[1], before = misc[2], cnt = misc[3];
      prefix |= (uint64_t)digit << shift;
      pmask |= 0xFFull << shift;
      rank -= before;
      __syncthreads();
      if (cnt == rank || shift == 0) {
        bound = prefix | ~pmask;
        break;
      }
    }
  }
  // ---- gather the kept keys
  for (int l = 0; l < nlists; ++l) {
    const uint64_t* lp = list_ptr(l);
    for (int o = tid; o < lcnt[l]; o += kMergeThreads) {
      const uint64_t key = lp[o];
      if (key <= bound) {
        const uint32_t pos = atomicAdd(&misc[0], 1u);
        if (pos < (uint32_t)a.kp2) cand[pos] = key;
      }
    }
  }
  __syncthreads();
  int kept = (int)misc[0];
  if (kept > a.kp2) {
    if (tid == 0) atomicOr(a.status, kErrPoolOverflow);
    kept = a.kp2;
  }
  // ---- 2. exact FP32 rerank, one warp per candidate
  for (int c = warp; c < kept; c += kMergeThreads / 32) {
    const uint32_t idx = (uint32_t)(cand[c] & 0xFFFFFFFFu);
    const float* xr = m.db + (size_t)idx * m.ld_db;
    float s = 0.f;
    for (int i = lane; i < d; i += 32) {
      const float t = qv[i] - __ldg(xr + i);
      s = fmaf(t, t, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) cand[c] = make_key(s, idx);
  }
  for (int c = kept + tid; c < a.kp2; c += kMergeThreads) cand[c] = kKeyEmpty;
  __syncthreads();
  // ---- 3. bitonic sort by (exact distance, row)
  int n2 = 1;
  while (n2 < kept) n2 <<= 1;
  for (int size = 2; size <= n2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < n2 / 2; i += kMergeThreads) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool asc = (lo & size) == 0;
        const uint64_t x = cand[lo], y = cand[hi];
        if ((x > y) == asc) {
          cand[lo] = y;
          cand[hi] = x;
        }
      }
      __syncthreads();
    }
  }
  for (int t = tid; t < m.k; t += kMergeThreads) {
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

cudaError_t launch_merge_batch(MergeItem* items, int n, int d, uint32_t* status, cudaStream_t st) {
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
  int kp2 = 1;
  while (kp2 < kpmax) kp2 <<= 1;
  a.kp2 = kp2;
  a.lcnt_n = (2 * umax + 3) & ~3;
  const size_t smem = (size_t)kp2 * 8 + (256 + 8 + 8) * 4 + (size_t)a.lcnt_n * 4 + (size_t)d * 4 + 16;
  static bool attr_done[16] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 15]) {
    cudaError_t e =
        cudaFuncSetAttribute(merge_rerank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    attr_done[dev & 15] = true;
  }
  if (smem > 200 * 1024 || qsum > 0x7fffffffLL) return cudaErrorInvalidValue;
  merge_rerank_kernel<<<(unsigned)qsum, kMergeThreads, smem, st>>>(a);
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
  it.row0 = 0;
  it.work_begin = 0;
  it.work_per_cta = m.plan.work_per_cta;
  it.pools = m.pools;
  it.pool_counts = m.pool_counts;
  it.queries = m.queries;
  it.db = m.db;
  it.ld_db = m.ld_db;
  it.out_idx = m.out_idx;
  it.out_dist = m.out_dist;
  return launch_merge_batch(&it, 1, m.d, m.status, st);
}

}  // namespace curplsh_b200
