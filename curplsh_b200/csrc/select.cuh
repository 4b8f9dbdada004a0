// select.cuh -- warp-cooperative radix selection over 64-bit (distance, row)
// keys for the candidate-pool refresh of the fused pass.
//
// Keys are unique (a database row appears at most once in a pool), so "the r
// smallest keys" is a well-defined set and the result never depends on thread
// timing: ties in distance are broken by the lower row index, the engine's
// deterministic tie rule.
#pragma once
#include <cstdint>
#include "common.cuh"

namespace curplsh_b200 {

#ifdef CURPLSH_FUSED_STATS
// instrumented builds: the fused kernel points this at its pass counter
__device__ unsigned long long* g_radix_pass_counter = nullptr;
#endif

// One radix digit step shared by the register and streaming forms: given the
// warp-private 256-bin histogram of the current digit, find the digit holding
// the element of 1-based `rank`; returns (digit, count of smaller digits,
// count in that digit), identical in every lane.
__device__ __forceinline__ void radix_digit_step(const uint32_t* hist, uint32_t rank, uint32_t& digit,
                                                 uint32_t& before, uint32_t& cnt) {
  const int lane = threadIdx.x & 31;
  uint32_t c[8], tot = 0;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    c[b] = hist[lane * 8 + b];
    tot += c[b];
  }
  uint32_t incl = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const uint32_t excl = incl - tot;
  const uint32_t own = __ballot_sync(0xffffffffu, excl < rank && rank <= incl);
  const int src = __ffs(own) - 1;
  digit = 0;
  before = 0;
  cnt = 0;
  if (lane == src) {
    uint32_t acc = excl;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if (cnt == 0 && acc + c[b] >= rank) {
        digit = (uint32_t)(lane * 8 + b);
        before = acc;
        cnt = c[b];
      }
      acc += c[b];
    }
  }
  digit = __shfl_sync(0xffffffffu, digit, src);
  before = __shfl_sync(0xffffffffu, before, src);
  cnt = __shfl_sync(0xffffffffu, cnt, src);
  __syncwarp();
}

// Warp-wide min / max of 64-bit values.
__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t < v ? t : v;
  }
  return v;
}
__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t > v ? t : v;
  }
  return v;
}

// Radix descent (8 bits per pass) for the key of rank `rank` (1-based) among
// the keys <= `limit` held by the warp (lane L holds key[e] = element e*32+L),
// starting at the highest bit in which the considered keys differ, so bits
// they all share cost no pass.  `hist` is a 256-entry warp-private shared
// buffer.  Returns a key bound B such that exactly `rank` of the considered
// keys are <= B.  Requires 1 <= rank <= number of considered keys.
// Warp-collective.
template <int E>
__device__ __forceinline__ uint64_t warp_radix_bound(const uint64_t (&key)[E], uint64_t limit, uint32_t rank,
                                                     uint32_t* hist) {
  const int lane = threadIdx.x & 31;
  uint64_t lo = ~0ull, hi = 0;
#pragma unroll
  for (int e = 0; e < E; ++e)
    if (key[e] <= limit) {
      lo = key[e] < lo ? key[e] : lo;
      hi = key[e] > hi ? key[e] : hi;
    }
  lo = warp_min_u64(lo);
  hi = warp_max_u64(hi);
  const uint64_t diff = lo ^ hi;
  const int top = diff ? 63 - __clzll((long long)diff) : 0;
  int shift = top >= 7 ? top - 7 : 0;
  // bits at and above shift+8 are common to every considered key
  uint64_t pmask = shift + 8 >= 64 ? 0ull : ~((1ull << (shift + 8)) - 1ull);
  uint64_t prefix = lo & pmask;
  for (;;) {
#pragma unroll
    for (int b = 0; b < 8; ++b) hist[lane * 8 + b] = 0u;
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (key[e] <= limit && (key[e] & pmask) == prefix) atomicAdd(&hist[(uint32_t)(key[e] >> shift) & 255u], 1u);
    __syncwarp();
#ifdef CURPLSH_FUSED_STATS
    if (lane == 0 && g_radix_pass_counter) atomicAdd(g_radix_pass_counter, 1ull);
#endif
    uint32_t digit, before, cnt;
    radix_digit_step(hist, rank, digit, before, cnt);
    prefix |= (uint64_t)digit << shift;
    pmask |= 0xFFull << shift;
    rank -= before;
    if (cnt == rank || shift == 0) break;
    // next 8 bits; a final partial window overlaps bits already fixed, whose
    // values every remaining key shares, so the digit logic is unchanged
    shift = shift >= 8 ? shift - 8 : 0;
  }
  return prefix | ~pmask;
}

template <int E>
__device__ __forceinline__ uint64_t warp_max_key_le(const uint64_t (&key)[E], uint64_t bound) {
  uint64_t m = 0;
#pragma unroll
  for (int e = 0; e < E; ++e)
    if (key[e] <= bound) m = key[e] > m ? key[e] : m;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t v = __shfl_xor_sync(0xffffffffu, m, o);
    m = v > m ? v : m;
  }
  return m;
}

// Count of the warp's keys <= b (every lane gets the total).
template <int E>
__device__ __forceinline__ uint32_t warp_count_le(const uint64_t (&key)[E], uint64_t b) {
  uint32_t c = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) c += key[e] <= b ? 1u : 0u;
  return __reduce_add_sync(0xffffffffu, c);
}

// Smallest sorted-sample index j (lane j of `smp` holds sample j, ascending)
// with count(keys <= sample j) >= rank; starts near the expected position and
// steps, counts being monotone in j.  Returns sample j, count in `cnt`
// (cnt < rank only if even the largest sample is too small).
template <int E>
__device__ __forceinline__ uint64_t warp_sample_find(const uint64_t (&key)[E], uint64_t smp, int n, uint32_t rank,
                                                     uint32_t& cnt) {
  int j = (int)(((long long)rank * 32 + n - 1) / n);
  j = j < 0 ? 0 : (j > 31 ? 31 : j);
  uint64_t b = __shfl_sync(0xffffffffu, smp, j);
  uint32_t c = warp_count_le<E>(key, b);
  if (c >= rank) {
    while (j > 0) {
      const uint64_t b2 = __shfl_sync(0xffffffffu, smp, j - 1);
      const uint32_t c2 = warp_count_le<E>(key, b2);
      if (c2 < rank) break;
      --j;
      b = b2;
      c = c2;
    }
  } else {
    while (c < rank && j < 31) {
      ++j;
      b = __shfl_sync(0xffffffffu, smp, j);
      c = warp_count_le<E>(key, b);
    }
  }
  cnt = c;
  return b;
}

// Contention-free approximate selection for the pool refresh: keeps every key
// <= B where B is the smallest of 32 stratified sample keys with at least
// `keep` keys <= B (so roughly keep + n/32 keys are kept).  B is a genuine
// pool key, so the pool still holds at least `keep` keys <= its bound and the
// bound stays a valid upper bound of the k'-th distance.  Returns B; falls
// back to the exact radix form when the samples cannot free enough room.
template <int E>
__device__ __forceinline__ uint64_t warp_select_keep_sampled(uint64_t* pool, int n, int keep, int cap,
                                                             uint32_t* hist, int& kept) {
  const int lane = threadIdx.x & 31;
  uint64_t key[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int i = e * 32 + lane;
    key[e] = i < n ? pool[i] : kKeyEmpty;
  }
  // one sample per lane: element (lane % E) * 32 + lane, a stride through the pool
  uint64_t smp = key[0];
#pragma unroll
  for (int e = 1; e < E; ++e)
    if ((lane % E) == e) smp = key[e];
  // bitonic sort of the 32 samples across the warp (ascending by lane)
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const uint64_t other = __shfl_xor_sync(0xffffffffu, smp, stride);
      const bool lower = (lane & stride) == 0;
      const bool asc = (lane & size) == 0;
      const uint64_t mn = other < smp ? other : smp, mx = other < smp ? smp : other;
      smp = (lower == asc) ? mn : mx;
    }
  }
  uint32_t c_keep = 0;
  const uint64_t bound = warp_sample_find<E>(key, smp, n, (uint32_t)keep, c_keep);
  if (c_keep < (uint32_t)keep || bound == kKeyEmpty || (int)c_keep > cap - pool_sync_tiles(cap, keep) * kBN) {
    // samples too coarse to free a tile of room: exact selection
    __syncwarp();
    const uint64_t eb = warp_radix_bound<E>(key, kKeyEmpty - 1, (uint32_t)keep, hist);
    int w = 0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const bool take = key[e] <= eb;
      const uint32_t bal = __ballot_sync(0xffffffffu, take);
      if (take) pool[w + __popc(bal & ((1u << lane) - 1u))] = key[e];
      w += __popc(bal);
    }
    kept = w;
    const uint64_t kmax = warp_max_key_le<E>(key, eb);
    __syncwarp();
    return kmax;
  }
  int w = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const bool take = key[e] <= bound;
    const uint32_t bal = __ballot_sync(0xffffffffu, take);
    if (take) pool[w + __popc(bal & ((1u << lane) - 1u))] = key[e];
    w += __popc(bal);
  }
  kept = w;
  __syncwarp();
  return bound;
}

// Streaming form for larger pools (reads global memory on every pass).
__device__ __forceinline__ uint64_t warp_stream_bound(const uint64_t* pool, int n, uint64_t limit, uint32_t rank,
                                                      uint32_t* hist) {
  const int lane = threadIdx.x & 31;
  uint64_t prefix = 0, pmask = 0;
  for (int shift = 56; shift >= 0; shift -= 8) {
#pragma unroll
    for (int b = 0; b < 8; ++b) hist[lane * 8 + b] = 0u;
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
      const uint64_t k = pool[i];
      if (k <= limit && (k & pmask) == prefix) atomicAdd(&hist[(uint32_t)(k >> shift) & 255u], 1u);
    }
    __syncwarp();
    uint32_t digit, before, cnt;
    radix_digit_step(hist, rank, digit, before, cnt);
    prefix |= (uint64_t)digit << shift;
    pmask |= 0xFFull << shift;
    rank -= before;
    if (cnt == rank || shift == 0) break;
  }
  return prefix | ~pmask;
}

__device__ __forceinline__ uint64_t warp_stream_max_le(const uint64_t* pool, int n, uint64_t bound) {
  const int lane = threadIdx.x & 31;
  uint64_t m = 0;
  for (int i = lane; i < n; i += 32) {
    const uint64_t k = pool[i];
    if (k <= bound) m = k > m ? k : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t v = __shfl_xor_sync(0xffffffffu, m, o);
    m = v > m ? v : m;
  }
  return m;
}

__device__ __forceinline__ uint64_t warp_select_keep_stream(uint64_t* pool, int n, int keep, uint32_t* hist,
                                                            int& kept) {
  const int lane = threadIdx.x & 31;
  const uint64_t bound = warp_stream_bound(pool, n, kKeyEmpty - 1, (uint32_t)keep, hist);
  const uint64_t kmax = warp_stream_max_le(pool, n, bound);
  // in-place stable compaction: every read of a 32-entry round completes
  // (ballot) before any lane writes, and writes never pass the reads
  int w = 0;
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const uint64_t k = (i < n) ? pool[i] : kKeyEmpty;
    const bool take = k <= bound;
    const uint32_t bal = __ballot_sync(0xffffffffu, take);
    if (take) pool[w + __popc(bal & ((1u << lane) - 1u))] = k;
    w += __popc(bal);
  }
  __syncwarp();
  kept = w;
  return kmax;
}

// Dispatch on the pool capacity: registers up to 1024 entries, else streaming.
__device__ __forceinline__ uint64_t warp_select_keep_any(uint64_t* pool, int n, int keep, int cap, uint32_t* hist,
                                                         int& kept) {
  if (cap <= 512) return warp_select_keep_sampled<16>(pool, n, keep, cap, hist, kept);
  if (cap <= 1024) return warp_select_keep_sampled<32>(pool, n, keep, cap, hist, kept);
  return warp_select_keep_stream(pool, n, keep, hist, kept);
}

}  // namespace curplsh_b200
