// shards.cu -- merge of per-shard top-k lists (multi-GPU sharded search).
//
// A database split by rows over G ranks is searched shard by shard; the
// shards' [Q x k] results are exchanged (an all-gather of 8*Q*k bytes per
// shard) and merged here into the global top-k: one CTA per query sorts the
// G*k (distance, global row) keys -- lower row first on equal distances, the
// tie rule of the single-index search -- and writes the first k.  Padding
// slots (-1, FLT_MAX) sort last and stay padding.  No counterpart in the
// reference, which searches one device (include/index.h:18-82).
#include <cfloat>
#include <cstdio>

#include "../../include/curplsh_b200.h"
#include "common.cuh"
#include "fused_knn.h"

namespace curplsh_b200 {
namespace {

constexpr int kShardThreads = 256;

__global__ void __launch_bounds__(kShardThreads) merge_shards_kernel(int nq, int k, int G, const float* __restrict__ dist,
                                                                   const int32_t* __restrict__ idx,
                                                                   const long long* __restrict__ bases, int n2,
                                                                   int32_t* __restrict__ out_idx,
                                                                   float* __restrict__ out_dist) {
  extern __shared__ uint64_t keys[];  // [n2]
  const int q = blockIdx.x;
  const int total = G * k;
  for (int i = threadIdx.x; i < n2; i += kShardThreads) {
    uint64_t key = kKeyEmpty;
    if (i < total) {
      const int s = i / k, j = i - s * k;
      const size_t o = ((size_t)s * nq + q) * k + j;
      const int li = idx[o];
      if (li >= 0) key = make_key(dist[o], (uint32_t)(bases[s] + li));
    }
    keys[i] = key;
  }
  __syncthreads();
  for (int size = 2; size <= n2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < n2 / 2; i += kShardThreads) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool asc = (lo & size) == 0;
        const uint64_t x = keys[lo], y = keys[hi];
        if ((x > y) == asc) {
          keys[lo] = y;
          keys[hi] = x;
        }
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < k; t += kShardThreads) {
    const uint64_t key = keys[t];
    const bool pad = key == kKeyEmpty;
    out_idx[(size_t)q * k + t] = pad ? -1 : (int32_t)(uint32_t)(key & 0xFFFFFFFFu);
    out_dist[(size_t)q * k + t] = pad ? FLT_MAX : ord2f((uint32_t)(key >> 32));
  }
}

}  // namespace
}  // namespace curplsh_b200

using namespace curplsh_b200;

extern "C" int curplsh_merge_shard_results(int64_t num_queries, int k, int num_shards, const float* distances,
                                           const int32_t* indices, const int64_t* shard_bases,
                                           int32_t* out_indices, float* out_distances, void* stream) {
  if (num_queries < 0 || k < 1 || k > 1024 || num_shards < 1 || num_shards > 64)
    return record_error(CURPLSH_ERR_INVALID_ARG, "curplsh_merge_shard_results: bad sizes");
  if (num_queries == 0) return CURPLSH_OK;
  if (!distances || !indices || !shard_bases || !out_indices || !out_distances)
    return record_error(CURPLSH_ERR_INVALID_ARG, "curplsh_merge_shard_results: null pointer");
  if (num_queries > 0x7fffffffLL) return record_error(CURPLSH_ERR_UNSUPPORTED, "too many queries");
  int n2 = 1;
  while (n2 < num_shards * k) n2 <<= 1;
  const size_t smem = (size_t)n2 * sizeof(uint64_t);
  if (smem > 200 * 1024) return record_error(CURPLSH_ERR_UNSUPPORTED, "num_shards * k above 16384");
  cudaError_t e = cudaFuncSetAttribute(merge_shards_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess) {
    merge_shards_kernel<<<(unsigned)num_queries, kShardThreads, smem, static_cast<cudaStream_t>(stream)>>>(
        (int)num_queries, k, num_shards, distances, indices, reinterpret_cast<const long long*>(shard_bases), n2,
        out_indices, out_distances);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    char m[200];
    snprintf(m, sizeof(m), "curplsh_merge_shard_results: %s", cudaGetErrorString(e));
    return record_error(CURPLSH_ERR_CUDA, m);
  }
  return CURPLSH_OK;
}
