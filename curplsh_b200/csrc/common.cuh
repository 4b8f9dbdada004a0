// common.cuh -- definitions shared by the kernels and the host orchestration.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>

namespace curplsh_b200 {

// ------------------------------------------------------------ precision forms
// Form of the coarse (tensor-core) distance pass.  Every form finishes with
// an exact FP32 rerank of its candidates, so returned distances are
// sum_i (q_i - x_i)^2 in FP32 regardless of the coarse precision.
enum Form : int {
  kFormExact = 0,  // 3 x BF16 split products (hi*hi + hi*lo + lo*hi), FP32 accumulate
  kFormBF16 = 1,   // BF16 x BF16, FP32 accumulate, k' = rerank_factor * k candidates
  kFormFP8 = 2,    // FP8-E4M3 with per-vector FP32 scales, k' = rerank_factor * k
};

// ------------------------------------------------------------ device error word
// Bit flags written (atomicOr) to a device status word by kernels that give up.
enum DeviceError : uint32_t {
  kErrNone = 0,
  kErrWaitTimeout = 1u << 0,    // an mbarrier wait exceeded its poll limit
  kErrPoolOverflow = 1u << 1,   // a candidate pool would have overflowed (never expected)
  kErrBadSchedule = 1u << 2,    // unit bookkeeping out of range (never expected)
};

// ------------------------------------------------------------ ordered keys
// Candidates are 64-bit keys: (order-preserving bits of the FP32 distance) << 32
// | database row.  Unsigned comparison of keys is (distance, index)
// lexicographic order, the engine's tie rule (lower index first).
__host__ __device__ __forceinline__ uint32_t f_bits(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(f);
#else
  uint32_t u;
  __builtin_memcpy(&u, &f, 4);
  return u;
#endif
}
__host__ __device__ __forceinline__ float bits_f(uint32_t u) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  __builtin_memcpy(&f, &u, 4);
  return f;
#endif
}
__host__ __device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t u = f_bits(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ord2f(uint32_t o) {
  uint32_t u = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
  return bits_f(u);
}
__host__ __device__ __forceinline__ uint64_t make_key(float d, uint32_t idx) {
  return ((uint64_t)f2ord(d) << 32) | idx;
}
constexpr uint64_t kKeyEmpty = ~0ull;
constexpr uint32_t kOrdInf = 0xFFFFFFFFu;  // "no bound yet" for per-query thresholds

// ------------------------------------------------------------ fused pass geometry
constexpr int kBM = 128;          // queries per block: MMA M, one TMEM lane per query
constexpr int kBN = 256;          // database rows per tile: MMA N (TMEM columns per accumulator)
constexpr int kHalfN = kBN / 2;   // columns of a tile handled by one epilogue warpgroup
constexpr int kChunkBytes = 128;  // K extent of one smem chunk row (one 128-byte swizzle atom)
constexpr int kNumThreads = 320;  // warp 0 TMA producer, warp 1 MMA issuer, warps 2..9 epilogue
// BF16 forms append kAugCols columns to every row so the tensor cores add the
// norms: database rows carry [n1 n2 n3 1 1 1] (||x||^2 = n1+n2+n3, three BF16
// terms), query rows (stored as -2q) carry [1 1 1 m1 m2 m3] (||q||^2 = m1+m2+m3),
// and the accumulator is ||q||^2 + ||x||^2 - 2 q.x directly.
constexpr int kAugCols = 6;
constexpr int kEpiWarps = 8;
// Epilogue warps of the candidate-pool kernel, a build option: 8 or 12 (two or
// three per TMEM lane group; with 12 the block of 14 warps caps registers at
// 128 a thread).  The block-minimum kernel keeps 8.
#ifndef CURPLSH_EPI_WARPS
#define CURPLSH_EPI_WARPS 8
#endif
constexpr int kPoolEpiWarps = CURPLSH_EPI_WARPS;
static_assert(kPoolEpiWarps == 8 || kPoolEpiWarps == 12, "8 or 12 epilogue warps");
constexpr int kMaxEpiWarps = 12;
__host__ __device__ constexpr int epi_warps_for(bool minima) { return minima ? kEpiWarps : kPoolEpiWarps; }
__host__ __device__ constexpr int threads_for(bool minima) { return 64 + 32 * epi_warps_for(minima); }
constexpr int kPoolRoom = kBN;  // free slots a candidate pool keeps for the next tile (both halves)
// Tiles between two selection points of a shared candidate pool: two when the
// capacity leaves room for two tiles of appends above k' + 128, else one.
__host__ __device__ inline int pool_sync_tiles(int cap, int kprime) { return cap >= kprime + 2 * kBN + 128 ? 2 : 1; }

// One work item of the fused pass: a query batch against one resident
// database.  A launch serves a list of items that share the form and the
// dimension; the (item, query block, tile) space of all of them is flattened
// and split evenly across the CTAs.  Items travel in the kernel parameters.
struct FusedItem {
  int nq;                  // real number of queries
  int nb;                  // real number of database rows
  int kprime;              // candidates kept per query (before the FP32 rerank)
  int pool_cap;            // capacity of one candidate pool (entries)
  int num_qblocks;         // G_i = ceil(nq / 128)
  int num_tiles;           // T_i = ceil(nb / 256)
  int units_per_block;     // U_i: max units (pool lists) of one query block of this item
  int split_tiles;         // L_i: a unit never crosses a multiple of L_i tiles within its block
  long long work_begin;    // flattened offset of this item's first (block, tile)
  long long work_end;      // work_begin + G_i * T_i
  const float* db_norms;   // [nb_pad] squared norms, +inf for padding rows (FP8 form)
  const float* db_scale;   // [nb_pad] fp8 per-vector scales (FP8 form)
  const float* q_norms;    // [nq_pad]
  const float* q_scale;    // [nq_pad] (FP8 form)
  uint64_t* pools;         // [G_i*128][U_i][pool_cap]
  int* pool_counts;        // [G_i*128][U_i]
  uint32_t* q_bound;       // [nq_pad] shared per-query bound (ordered bits), init kOrdInf or an estimate
  int db_step;             // database row j of this item is stored row j * db_step (>= 1)
  float db_scale_uniform;  // > 0: every database row has this FP8 scale (db_scale is not read)
  // FP8 form with one database scale s: > 0 is the byte offset of the 32-byte
  // BF16 norm tail of the FP8 rows (query rows [a_h a_h a_l], a = 1/s_q;
  // database rows [b_h b_l b_h], b = -||x||^2 / (2 s)).  One K=16 BF16 MMA over
  // the tails adds ||x||^2 / (-2 s_q s) to the FP8 accumulator, which then is
  // (||x||^2 - 2 q.x) / (-2 s_q s): no database norm is loaded per tile.
  int fp8_tail;
  // Non-null: block-minimum mode (no pools): minima[q * 2 * num_tiles + 2 * t + h]
  // gets the smallest key distance of query q over rows [256 t + 128 h, +128).
  float* minima;
};

// Tensor maps of one item, in this order.
enum FusedMap : int { kMapQHi = 0, kMapQLo, kMapXHi, kMapXLo, kMapQTail, kMapXTail, kMapsPerItem };

struct FusedBatch {
  int num_items;
  int form;
  int d;                   // dimension shared by every item of the launch
  int pair;                // 1: clusters of two CTAs, one 256-row MMA over two query blocks
  int dual;                // 1: each CTA holds two query blocks against 128-row database tiles
  int pad1;
  long long total_work;    // sum of G_i * T_i (G_i: query groups of 128 << pair rows)
  long long work_per_cta;  // W, per CTA (per pair when pair = 1)
  uint32_t* status;        // device error word
  unsigned long long* stats;  // per-role cycle counters, written only by builds with CURPLSH_FUSED_STATS
  const int* run_if;       // non-null: every CTA returns at once unless *run_if != 0
};

// Counter slots of FusedBatch::stats (instrumented builds).
enum FusedStat : int {
  kStatProducerWaitEmpty = 0,  // producer lane: cycles waiting for a free stage
  kStatMmaWaitFull,            // MMA lane: cycles waiting for TMA data
  kStatMmaWaitAccEmpty,        // MMA lane: cycles waiting for the epilogue to free an accumulator
  kStatEpiWaitAccFull,         // epilogue warps (lane 0): cycles waiting for an accumulator
  kStatEpiFilter,              // epilogue warps: cycles filtering tiles
  kStatEpiRefresh,             // epilogue warps: cycles in pool refreshes
  kStatRefreshes,              // number of pool refreshes
  kStatSurvivors,              // candidates appended to pools
  kStatCtaCycles,              // sum over CTAs of kernel cycles
  kStatRadixPasses,            // histogram passes run by pool refreshes
  kStatSlowChunks,             // warp-chunks (32 columns) that entered the survivor path
  kStatLoopIters,              // survivor-append loop iterations executed by warps
  kStatTmemCycles,             // epilogue warps (lane 0): cycles in TMEM loads + waits
  kStatPairBarrier,            // epilogue warps (lane 0): cycles in the pair barriers
  kStatCount
};

}  // namespace curplsh_b200
