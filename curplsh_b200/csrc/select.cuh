// select.cuh -- warp- and block-cooperative radix selection over 64-bit
// (distance, index) keys.  Keys are unique (every database row appears at most
// once per candidate set), so "the `keep` smallest keys" is a well-defined set
// and the result never depends on thread timing: ties in distance are broken by
// the lower row index, the engine's deterministic tie rule.
#pragma once
#include <cstdint>
#include "common.cuh"

namespace curplsh_b200 {

// Warp-cooperative: among pool[0..n) keep exactly the `keep` smallest keys,
// compacted into pool[0..keep).  Requires n > keep >= 1.  `hist` is a
// 256-entry warp-private shared-memory scratch.  Returns the largest kept key
// and the number kept (== keep for unique keys), same values in every lane.
// All 32 lanes must call with the same arguments.
__device__ __forceinline__ uint64_t warp_select_keep(uint64_t* pool, int n, int keep, uint32_t* hist,
                                                     int& kept) {
  const int lane = threadIdx.x & 31;
  uint64_t prefix = 0, pmask = 0, bound = ~0ull;
  uint32_t rank = (uint32_t)keep;  // 1-based rank among keys matching prefix
  for (int shift = 56; shift >= 0; shift -= 8) {
#pragma unroll
    for (int b = 0; b < 8; ++b) hist[lane * 8 + b] = 0u;
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
      const uint64_t key = pool[i];
      if ((key & pmask) == prefix) atomicAdd(&hist[(uint32_t)(key >> shift) & 255u], 1u);
    }
    __syncwarp();
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
    uint32_t digit = 0, before = 0, cnt = 0;
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
    prefix |= (uint64_t)digit << shift;
    pmask |= 0xFFull << shift;
    rank -= before;
    if (cnt == rank || shift == 0) {
      bound = prefix | ~pmask;
      break;
    }
  }
  // In-place stable compaction of keys <= bound; all reads of a 32-entry round
  // complete (ballot) before any lane writes, and writes never pass the reads.
  int w = 0;
  uint64_t kmax = 0;
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const uint64_t key = (i < n) ? pool[i] : kKeyEmpty;
    const bool take = key <= bound;
    const uint32_t bal = __ballot_sync(0xffffffffu, take);
    if (take) {
      pool[w + __popc(bal & ((1u << lane) - 1u))] = key;
      kmax = key > kmax ? key : kmax;
    }
    w += __popc(bal);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t v = __shfl_xor_sync(0xffffffffu, kmax, o);
    kmax = v > kmax ? v : kmax;
  }
  __syncwarp();
  kept = w;
  return kmax;
}


// Register-resident variant for pools of at most 32*E entries: the pool is read
// once (coalesced, all loads in flight together), the radix passes run on
// registers, and the kept keys are written back compacted.  Same contract as
// warp_select_keep.
template <int E>
__device__ __forceinline__ uint64_t warp_select_keep_reg(uint64_t* pool, int n, int keep, uint32_t* hist,
                                                         int& kept) {
  const int lane = threadIdx.x & 31;
  uint64_t key[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int i = e * 32 + lane;
    key[e] = i < n ? pool[i] : kKeyEmpty;
  }
  uint64_t prefix = 0, pmask = 0, bound = ~0ull;
  uint32_t rank = (uint32_t)keep;
  for (int shift = 56; shift >= 0; shift -= 8) {
#pragma unroll
    for (int b = 0; b < 8; ++b) hist[lane * 8 + b] = 0u;
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (key[e] != kKeyEmpty && (key[e] & pmask) == prefix)
        atomicAdd(&hist[(uint32_t)(key[e] >> shift) & 255u], 1u);
    __syncwarp();
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
    uint32_t digit = 0, before = 0, cnt = 0;
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
    prefix |= (uint64_t)digit << shift;
    pmask |= 0xFFull << shift;
    rank -= before;
    if (cnt == rank || shift == 0) {
      bound = prefix | ~pmask;
      break;
    }
  }
  int w = 0;
  uint64_t kmax = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const bool take = key[e] <= bound && key[e] != kKeyEmpty;
    const uint32_t bal = __ballot_sync(0xffffffffu, take);
    if (take) {
      pool[w + __popc(bal & ((1u << lane) - 1u))] = key[e];
      kmax = key[e] > kmax ? key[e] : kmax;
    }
    w += __popc(bal);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t v = __shfl_xor_sync(0xffffffffu, kmax, o);
    kmax = v > kmax ? v : kmax;
  }
  __syncwarp();
  kept = w;
  return kmax;
}

// Dispatch on the pool capacity: registers up to 1024 entries, else the
// streaming form.
__device__ __forceinline__ uint64_t warp_select_keep_any(uint64_t* pool, int n, int keep, int cap,
                                                         uint32_t* hist, int& kept) {
  if (cap <= 512) return warp_select_keep_reg<16>(pool, n, keep, hist, kept);
  if (cap <= 1024) return warp_select_keep_reg<32>(pool, n, keep, hist, kept);
  return warp_select_keep(pool, n, keep, hist, kept);
}

}  // namespace curplsh_b200
