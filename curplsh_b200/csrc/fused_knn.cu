// fused_knn.cu -- the fused distance + candidate-filter pass on the 5th-gen
// tensor cores (sm_100a).
//
// Replaces, in one kernel, the reference's per-tile chain (cuRPLSH paths):
//   matrixMultiply / cublasSgemm        src/internal/matrix_ops.cu:8-60   (-2 q.x)
//   l2Select (+ ||x||^2, top-k)         src/internal/select.cu:189-224
//   adjustIndices                       src/internal/search.cu:21-42      (tile -> global row)
// The Q x N distance matrix never leaves the SM: each 128-query x 256-row
// tile is accumulated in TMEM, read back by the epilogue warps, compared with a
// per-query bound and only the survivors are appended to a per-query candidate
// pool in global memory.
//
// Roles (320 threads, one CTA per SM, persistent over a balanced schedule):
//   warp 0      TMA producer: query block (resident, or streamed per K chunk)
//               and database tiles, 128-byte-swizzled, into a stage ring.
//   warp 1      allocates 512 TMEM columns (two 128x256 f32 accumulators) and,
//               from one lane, issues tcgen05.mma; commits release stages and
//               publish accumulators.
//   warps 2..9  epilogue: two warpgroups, each owning one 128-column half of
//               every tile; thread = one query (TMEM lane).  A thread keeps its
//               own pool and bound; a warp refreshes (radix-selects) a pool that
//               is about to overflow, keeping the k' smallest (distance, row)
//               keys, and publishes the tightened bound to the shared per-query
//               bound array so other CTAs working on the same queries filter
//               harder.
//
// Schedule: the (query block, database tile) space is flattened and split into
// equal contiguous ranges, one per CTA, so the work is balanced to one tile for
// any Q, N.  A range covers a few "units" = (query block, tile sub-range).
#include <cuda.h>

#include <cstdio>

#include "common.cuh"
#include <algorithm>
#include <atomic>

#include "fused_knn.h"
#include "ptx.cuh"
#include "select.cuh"

namespace curplsh_b200 {

// ------------------------------------------------------------------ forms
template <int FORM>
struct FormTraits;
template <>
struct FormTraits<kFormExact> {
  static constexpr int kAParts = 2, kBParts = 2, kProducts = 3;
  static constexpr int kChunkElems = 64, kStepElems = 16;  // bf16
  static constexpr bool kFP8 = false;
  static constexpr bool kFolded = true;  // norms ride in the augmented K columns
  // products: hi*hi, hi*lo, lo*hi  (the lo*lo term, O(2^-16) relative, is dropped)
  __device__ static constexpr int a_part(int p) { return p == 2 ? 1 : 0; }
  __device__ static constexpr int b_part(int p) { return p == 1 ? 1 : 0; }
};
template <>
struct FormTraits<kFormBF16> {
  static constexpr int kAParts = 1, kBParts = 1, kProducts = 1;
  static constexpr int kChunkElems = 64, kStepElems = 16;
  static constexpr bool kFP8 = false;
  static constexpr bool kFolded = true;
  __device__ static constexpr int a_part(int) { return 0; }
  __device__ static constexpr int b_part(int) { return 0; }
};
template <>
struct FormTraits<kFormFP8> {
  static constexpr int kAParts = 1, kBParts = 1, kProducts = 1;
  static constexpr int kChunkElems = 128, kStepElems = 32;  // e4m3
  static constexpr bool kFP8 = true;
  static constexpr bool kFolded = false;  // per-row scales: norms are applied in the epilogue
  __device__ static constexpr int a_part(int) { return 0; }
  __device__ static constexpr int b_part(int) { return 0; }
};

constexpr uint32_t kAChunkBytes = kBM * kChunkBytes;  // 16 KB
constexpr uint32_t kBChunkBytes = kBN * kChunkBytes;  // 32 KB
// A narrow tail chunk holds the last <= 16 BF16 columns (the augmented norm
// columns when d is a multiple of 64): 32-byte rows, 32-byte swizzle.
constexpr uint32_t kTailRowBytes = 32;
constexpr uint32_t kATailBytes = kBM * kTailRowBytes;  // 4 KB
constexpr uint32_t kBTailBytes = kBN * kTailRowBytes;  // 8 KB

// ------------------------------------------------------------------ smem layout
struct SmemLayout {
  int kdim;            // K extent of the MMA (d, plus kAugCols for the folded forms)
  int nkc;             // K chunks (128 bytes of K each, except a narrow tail)
  int tail_narrow;     // 1: the last chunk is a 16-column, 32-byte-swizzled tail
  int a_stream;        // 1: query chunks travel with each stage
  uint32_t a_bytes;    // resident query block bytes (0 when streamed)
  uint32_t stage_bytes;
  int stages;
  uint32_t bar_off;    // offset of the barrier block
  uint32_t hist_off;   // warp-private radix histograms
  uint32_t pool_off;   // per-row candidate pool counts and bounds
  uint32_t total;      // dynamic smem bytes requested (includes 1 KB alignment slack)
  uint32_t b_chunk;    // bytes of one B part of a K chunk (this CTA's database rows)
  uint32_t a_block;    // bytes between the two resident query blocks (dual)
  uint32_t b_tail;     // bytes of the B tail chunk
};

// pair = 1: this CTA holds half of each 256-row database tile (CTA pairs);
// epi_warps: epilogue warps (each has a 1 KB histogram / staging area);
// dual = 1: two resident query blocks (a_block bytes apart) and 128-row tiles.
__host__ __device__ inline SmemLayout make_layout(int form, int d, int pair = 0, int epi_warps = kEpiWarps,
                                                  int dual = 0) {
  SmemLayout L{};
  L.b_chunk = (pair || dual) ? kBChunkBytes / 2 : kBChunkBytes;
  L.b_tail = (pair || dual) ? kBTailBytes / 2 : kBTailBytes;
  const bool folded = form != kFormFP8;
  const int chunk_elems = folded ? 64 : 128;
  const int a_parts = (form == kFormExact) ? 2 : 1;
  const int b_parts = (form == kFormExact) ? 2 : 1;
  L.kdim = folded ? d + kAugCols : d;
  L.nkc = (L.kdim + chunk_elems - 1) / chunk_elems;
  // narrow tail only when it holds nothing but the norm columns (d % 64 == 0):
  // the tail runs the hi x hi product alone, which is exact only for those
  L.tail_narrow = folded && (d % 64 == 0);
  // everything below the barrier block must fit the 227 KB opt-in limit
  const uint32_t pool_bytes = dual ? 2048u : 1024u;  // pool counts and bounds of 128 (dual: 256) rows
  const uint32_t budget = 227u * 1024u - 256u - (uint32_t)epi_warps * 256u * 4u - pool_bytes - 1024u;
  const int nreg = L.nkc - (L.tail_narrow ? 1 : 0);
  const uint32_t a_one = (uint32_t)nreg * a_parts * kAChunkBytes + (L.tail_narrow ? kATailBytes : 0u);
  L.a_block = (a_one + 1023u) & ~1023u;
  const uint32_t a_res = dual ? 2u * L.a_block : a_one;
  // a stage = one regular K chunk of the tile; the last one also carries the tail
  const uint32_t b_stage = (uint32_t)b_parts * L.b_chunk + (L.tail_narrow ? L.b_tail : 0u);
  if (((a_res + 1023u) & ~1023u) + 2 * b_stage <= budget) {
    L.a_stream = 0;
    L.a_bytes = (a_res + 1023u) & ~1023u;
    L.stage_bytes = b_stage;
  } else {
    L.a_stream = 1;
    L.a_bytes = 0;
    L.stage_bytes = b_stage + (uint32_t)a_parts * kAChunkBytes + (L.tail_narrow ? kATailBytes : 0u);
  }
  L.stage_bytes = (L.stage_bytes + 1023u) & ~1023u;
  int s = (int)((budget - L.a_bytes) / L.stage_bytes);
  L.stages = s < 2 ? 2 : (s > 8 ? 8 : s);
  L.bar_off = L.a_bytes + (uint32_t)L.stages * L.stage_bytes;
  L.hist_off = L.bar_off + 256;  // barriers: 2*8 + 6 mbarriers + tmem slot + flags < 256 B
  L.pool_off = L.hist_off + epi_warps * 256 * 4;
  L.total = L.pool_off + pool_bytes + 1024;
  return L;
}

// Offset of resident query chunk `kc`, part `part` (0 hi, 1 lo); the narrow
// tail (kc = nkc-1) has a part 0 only.
__device__ __forceinline__ uint32_t a_res_off(const SmemLayout& L, int kc, int part, int a_parts) {
  return (uint32_t)(kc * a_parts + part) * kAChunkBytes;
}

// Offsets inside a stage: B parts, then streamed A parts, then the tail (B, A).
template <int kAP, int kBP>
__device__ __forceinline__ uint32_t stage_a_off(const SmemLayout& L, int part) {
  return (uint32_t)kBP * L.b_chunk + (uint32_t)part * kAChunkBytes;
}
template <int kAP, int kBP>
__device__ __forceinline__ uint32_t stage_tail_off(const SmemLayout& L) {
  return (uint32_t)kBP * L.b_chunk + (L.a_stream ? (uint32_t)kAP * kAChunkBytes : 0u);
}

// ------------------------------------------------------------------ schedule
// Launch arguments: the batch header, then per-item scalars and tensor maps.
template <int MAXI>
struct FusedArgs {
  FusedBatch B;
  FusedItem items[MAXI];
  CUtensorMap maps[MAXI * kMapsPerItem];
};

// Walks the contiguous range [cta*W, min(total,(cta+1)*W)) of the flattened
// (item, query block, tile position) space as units (item, query block,
// [t0, t1)); positions map to database tiles through a per-block rotation.  A
// unit also ends at every multiple of the item's split length L, so no unit
// gathers candidates from more than L tiles (a split-N knob: longer units
// mean fewer pool lists for the merge but more in-pool selections).
// u_ord numbers the units of one query block: the number of cuts (CTA range
// starts and multiples of L) in (0, t0].  A position that is both kinds of
// cut leaves one ordinal unused (`gap`): that unit writes zero counts for it.
// With CTA pairs the space counts query groups of two blocks and a range
// belongs to a pair; each CTA of the pair gets its own block of the group
// (block = 2 * group + rank) and the same tiles.
struct UnitWalk {
  long long pos, end, W;
  int ii, shift, rank;
  __device__ UnitWalk(int cta, const FusedBatch& B, uint32_t cta_rank)
      : W(B.work_per_cta), ii(0), shift(B.pair | B.dual), rank((int)cta_rank) {
    pos = (long long)(cta >> B.pair) * W;
    end = pos + W < B.total_work ? pos + W : B.total_work;
  }
  template <int MAXI>
  __device__ bool next(const FusedArgs<MAXI>& A, int& item, int& qb, int& t0, int& t1, int& u_ord, bool& gap,
                       int& rot) {
    if (pos >= end) return false;
    while (ii < A.B.num_items && A.items[ii].work_end <= pos) ++ii;
    if (ii >= A.B.num_items) return false;
    const FusedItem& it = A.items[ii];
    const long long wb = it.work_begin;
    const int T = it.num_tiles;
    const int Ls = it.split_tiles;
    const long long lp = pos - wb;
    qb = (int)(lp / T);
    t0 = (int)(lp - (long long)qb * T);
    long long len = (end - pos) < (long long)(T - t0) ? (end - pos) : (long long)(T - t0);
    if (len > (long long)(Ls - t0 % Ls)) len = Ls - t0 % Ls;
    t1 = t0 + (int)len;
    const long long base = wb + (long long)qb * T;
    u_ord = (int)(pos / W - base / W) + t0 / Ls;
    gap = t0 > 0 && t0 % Ls == 0 && pos % W == 0;
    // Position j of the block is database tile (j - rot) mod T, where rot is
    // where the first CTA range starting inside this block begins: every such
    // CTA then reads tiles 0, 1, 2, ... from the start, in step with the
    // others, so concurrent CTAs share the database tiles in L2 (a contiguous
    // assignment alone would have them at spread-out offsets).
    {
      const long long first = (base + W - 1) / W * W - base;
      rot = first < T ? (int)first : 0;
    }
    item = ii;
    qb = (qb << shift) + rank;
    pos += len;
    return true;
  }
};

// Bounded wait that also gives up as soon as another role has aborted.
// `cl`: the arrivals come from the other CTA of a pair (acquire at cluster scope).
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                              bool cl = false) {
  auto poll = [&]() { return cl ? mbar_try_wait_cluster(bar, parity) : mbar_try_wait(bar, parity); };
  if (poll()) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 0; i < kWaitPollLimit; ++i) {
    if (poll()) return true;
    if ((i & 255u) == 255u) {
      if (*abort_flag) return false;
      if (globaltimer_ns() - t0 > kWaitTimeoutNs) return false;
    }
  }
  return false;
}

__device__ __forceinline__ void raise_abort(volatile int* abort_flag, uint32_t* status, uint32_t code) {
  *abort_flag = 1;
  atomicOr(status, code);
}

// Filter bound on d' = ||x||^2 - 2 q.x for a pool whose k'-th key distance is
// dstar: keys store fl(d' + ||q||^2), so admit d' <= dstar - ||q||^2 with a
// few-ulp slack; admitting slightly more never changes the selected set, which
// is decided by exact key order.
__device__ __forceinline__ float bound_to_thr(float dstar, float qn) {
  return (dstar - qn) + (fabsf(dstar) + fabsf(qn)) * 4.76837158203125e-7f;  // 2^-21
}

// Filter threshold for a bound `dstar` on the key distance.  The folded forms
// compare the accumulator, which is the key distance itself, so the bound is
// used as is; the FP8 form compares ||x||^2 - 2 q.x and needs bound_to_thr.
template <bool kFolded>
__device__ __forceinline__ float thr_from(float dstar, float qn) {
  return kFolded ? dstar : bound_to_thr(dstar, qn);
}

// Instrumentation (compiled in only with -DCURPLSH_FUSED_STATS): per-role
// cycle counters accumulated in registers and added to B.stats at exit.
#ifdef CURPLSH_FUSED_STATS
#define STAT_DECL(name) unsigned long long name = 0
#define STAT_BEGIN(t) const long long t = clock64()
#define STAT_END(t, acc) acc += (unsigned long long)(clock64() - t)
#define STAT_INC(acc, v) acc += (unsigned long long)(v)
#define STAT_FLUSH(slot, acc) \
  if (B.stats) atomicAdd(&B.stats[slot], acc)
#else
#define STAT_DECL(name)
#define STAT_BEGIN(t)
#define STAT_END(t, acc)
#define STAT_INC(acc, v)
#define STAT_FLUSH(slot, acc)
#endif

// Survivor masks from sign bits.  With u = the float just above thr, a column
// survives iff d < u, i.e. d <= thr.  t = d - u is formed two columns at a time
// by one packed FMA (d * 1 - u: exact product, one rounding), and its sign bit
// is exactly the test: rounding never changes the sign of a nonzero difference,
// d == u gives +0, and a NaN distance gives a NaN with the sign clear, so it
// never survives, as with a compare.  The sign bits enter the mask by funnel
// shifts, four consecutive columns per chain, so bit j belongs to column j: a
// packed FMA per two columns and a shift per column, against a compare, a
// select and an or per column.
__device__ __forceinline__ float next_above(float x) {
  const uint32_t u = __float_as_uint(x);
  if (u == 0x80000000u) return __uint_as_float(1u);  // -0: the smallest positive subnormal
  return __uint_as_float((int32_t)u >= 0 ? u + 1u : u - 1u);
}
// (acc << 1) | (t >> 31)
__device__ __forceinline__ uint32_t shl1_sign(uint32_t acc, uint32_t t) {
  uint32_t r;
  asm("shf.l.wrap.b32 %0, %1, %2, 1;" : "=r"(r) : "r"(t), "r"(acc));
  return r;
}
// bit j set iff km dv[j] < u, computed exactly (one rounding of km dv[j] - u
// keeps its sign); u = next_above(thr) makes it km dv[j] <= thr for km = 1.
// The sign bits are gathered by 32 / L funnel-shift chains of length L and
// joined: fewer instructions beat the extra chain parallelism at two epilogue
// warps per sub-partition (chains of 4 -> 16: BF16 pass 3.48 -> 3.37 ms; the
// FP8 pass gains again from 16 -> 32, 30.1 -> 28.1 ms, BF16 loses 1 %).
template <int L>
__device__ __forceinline__ uint32_t survive_mask32(const float (&dv)[32], float km, float u) {
  float t[32];
#pragma unroll
  for (int i = 0; i < 16; ++i) fma2_f32(t[2 * i], t[2 * i + 1], dv[2 * i], dv[2 * i + 1], km, km, -u, -u);
  // 32 / L independent chains of L funnel shifts, then their L-bit pieces joined
  uint32_t c[32 / L];
#pragma unroll
  for (int p = 0; p < 32 / L; ++p) {
    uint32_t a = __float_as_uint(t[L * p + L - 1]) >> 31;
#pragma unroll
    for (int i = L - 2; i >= 0; --i) a = shl1_sign(a, __float_as_uint(t[L * p + i]));
    c[p] = a;  // bit i = sign of t[L p + i]
  }
#pragma unroll
  for (int w = 1; w < 32 / L; w <<= 1)
#pragma unroll
    for (int p = 0; p + w < 32 / L; p += 2 * w) c[p] |= c[p + w] << (L * w);
  return c[0];
}

// bit j set iff dv[j] <= thr, by compare, select and or: eight independent
// partial masks
__device__ __forceinline__ uint32_t survive_mask32_cmp(const float (&dv)[32], float thr) {
  uint32_t pa[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
  for (int j = 0; j < 32; ++j) pa[j & 7] |= (dv[j] <= thr ? 1u : 0u) << j;
  return ((pa[0] | pa[1]) | (pa[2] | pa[3])) | ((pa[4] | pa[5]) | (pa[6] | pa[7]));
}

// 1: a chunk's masks are built only when some lane's smallest distance of the
// 64 columns (a three-input min tree, 32 instructions) passes.
#ifndef CURPLSH_MIN_FIRST
#define CURPLSH_MIN_FIRST 0
#endif
__device__ __forceinline__ float min64(const float (&a)[32], const float (&b)[32]) {
  float r[22];
#pragma unroll
  for (int i = 0; i < 10; ++i) r[i] = fmin3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
  r[10] = fmin3(a[30], a[31], b[0]);
#pragma unroll
  for (int i = 0; i < 10; ++i) r[11 + i] = fmin3(b[1 + 3 * i], b[2 + 3 * i], b[3 + 3 * i]);
  r[21] = b[31];
  float s[8];
#pragma unroll
  for (int i = 0; i < 7; ++i) s[i] = fmin3(r[3 * i], r[3 * i + 1], r[3 * i + 2]);
  s[7] = r[21];
  return fminf(fmin3(s[0], s[1], s[2]), fmin3(s[3], s[4], fmin3(s[5], s[6], s[7])));
}

// v[j] for a runtime j in [0, 32) without local memory: a 5-level select tree.
__device__ __forceinline__ float select32(const float (&v)[32], int j) {
  float a[16], b[8], c[4], d2[2];
#pragma unroll
  for (int i = 0; i < 16; ++i) a[i] = (j & 16) ? v[i + 16] : v[i];
#pragma unroll
  for (int i = 0; i < 8; ++i) b[i] = (j & 8) ? a[i + 8] : a[i];
#pragma unroll
  for (int i = 0; i < 4; ++i) c[i] = (j & 4) ? b[i + 4] : b[i];
#pragma unroll
  for (int i = 0; i < 2; ++i) d2[i] = (j & 2) ? c[i + 2] : c[i];
  return (j & 1) ? d2[1] : d2[0];
}

// ------------------------------------------------------------------ kernel
// MINIMA selects the block-minimum mode (FusedItem::minima, the sample pass of
// the bound estimate) at compile time, so the candidate-pool kernel carries
// none of its code.
// PAIR selects the CTA-pair kernel: a kernel that contains cta_group::2
// instructions can only be launched as clusters of two, so the single-CTA
// kernel is a separate instance without them.
// DUAL: two query blocks resident per CTA; each 128-row database tile feeds two
// 128 x 128 MMAs (one per block), so a tile crosses L2 -> SM once per 256
// queries without coupling CTAs; warp g of a lane group filters block g.
template <int FORM, int MAXI, bool MINIMA = false, bool PAIR = false, bool DUAL = false>
__global__ void __launch_bounds__(threads_for(MINIMA), 1) fused_knn_kernel(const __grid_constant__ FusedArgs<MAXI> A) {
  static_assert(!(PAIR && DUAL) && !(DUAL && MINIMA), "dual blocks: single CTAs, candidate pools");
  using Tr = FormTraits<FORM>;
  const FusedBatch& B = A.B;
  // a conditional pass (a re-search after a failed check): every thread of
  // every CTA reads the same flag, written by an earlier launch on the stream,
  // and leaves before any barrier or TMEM allocation when it is zero
  if (B.run_if && *B.run_if == 0) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int EW = epi_warps_for(MINIMA);  // epilogue warps
  constexpr int WG = EW / 4;                  // epilogue warps per TMEM lane group
  const SmemLayout L = make_layout(FORM, B.d, PAIR ? 1 : 0, EW, DUAL ? 1 : 0);
  constexpr int kTileRows = DUAL ? kBN / 2 : kBN;  // database rows per tile
  constexpr int kQB = DUAL ? 2 : 1;                // resident query blocks
  const int S = L.stages;
  // CTA pairs: rank 0 issues the MMAs and owns the barriers the pair's loads
  // complete on; each CTA loads and filters its own query block
  constexpr bool pair = PAIR;
  uint32_t rank = 0u;
  if constexpr (PAIR) rank = cluster_ctarank();
  const bool issuer = rank == 0;

  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint64_t* full = bars;            // [8]
  uint64_t* empty = bars + 8;       // [8]
  uint64_t* a_full = bars + 16;
  uint64_t* a_empty = bars + 17;
  uint64_t* acc_full = bars + 18;   // [2]
  uint64_t* acc_empty = bars + 20;  // [2]
  uint64_t* drain = bars + 22;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 23);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 24);
  uint32_t* hist_all = reinterpret_cast<uint32_t*>(smem + L.hist_off);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  STAT_BEGIN(t_kernel);

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(a_full, 1);
    mbar_init(a_empty, 1);
    for (int s = 0; s < 2; ++s) {
      mbar_init(&acc_full[s], 1);
      mbar_init(&acc_empty[s], pair ? 2 * EW : EW);  // both CTAs' epilogue warps
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_barrier_init();
    fence_proxy_async_smem();
  }
  if (warp == 1) {
    if constexpr (PAIR) {
      tmem_alloc_pair(tmem_slot, 512);
      tmem_relinquish_pair();
    } else {
      tmem_alloc(tmem_slot, 512);
      tmem_relinquish();
    }
  }
  tc_fence_before();
  // a pair's barriers must be initialised before the other CTA's loads and
  // arrivals can reach them
  if constexpr (PAIR)
    cluster_sync();
  else
    __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const int KC = Tr::kChunkElems;
  auto maps_of = [&](int ii) { return &A.maps[ii * kMapsPerItem]; };

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      const uint64_t pol_db = l2_policy_evict_first();
      const uint64_t pol_q = l2_policy_evict_last();
      // a pair's loads complete on rank 0's barriers, which expect both CTAs' bytes
      auto load = [&](void* dst, const CUtensorMap* m, uint64_t* bar, int c0, int c1, uint64_t pol) {
        if constexpr (PAIR)
          tma_load_2d_pair(dst, m, bar, c0, c1, pol);
        else
          tma_load_2d(dst, m, bar, c0, c1, pol);
      };
      const uint32_t tx_mul = pair ? 2u : 1u;
      const int half_row = pair ? (int)rank * (kBN / 2) : 0;  // this CTA's rows of a tile
      UnitWalk walk(blockIdx.x, B, rank);
      int ii, qb, t0, t1, u_ord, rot, unit = 0;
      bool gap;
      uint32_t it = 0;
      bool ok = true;
      STAT_DECL(st_wait);
      while (ok && walk.next(A, ii, qb, t0, t1, u_ord, gap, rot)) {
        const CUtensorMap* mp = maps_of(ii);
        const CUtensorMap& tm_q_hi = mp[kMapQHi];
        const CUtensorMap& tm_q_lo = mp[kMapQLo];
        const CUtensorMap& tm_x_hi = mp[kMapXHi];
        const CUtensorMap& tm_x_lo = mp[kMapXLo];
        const CUtensorMap& tm_q_tail = mp[kMapQTail];
        const CUtensorMap& tm_x_tail = mp[kMapXTail];
        if (!L.a_stream) {
          if (unit > 0 && !wait_or_abort(a_empty, (unit - 1) & 1, abort_flag)) {
            raise_abort(abort_flag, B.status, kErrWaitTimeout);
            ok = false;
            break;
          }
          const int nreg = L.nkc - (L.tail_narrow ? 1 : 0);
          if (issuer)
            mbar_arrive_expect_tx(a_full, tx_mul * (uint32_t)kQB *
                                              ((uint32_t)nreg * Tr::kAParts * kAChunkBytes +
                                               (L.tail_narrow ? kATailBytes : 0u)));
          for (int j = 0; j < kQB; ++j) {
            uint8_t* ab = smem + (uint32_t)j * L.a_block;
            const int qrow = (qb + j) * kBM;
            for (int kc = 0; kc < nreg; ++kc)
              for (int part = 0; part < Tr::kAParts; ++part)
                load(ab + a_res_off(L, kc, part, Tr::kAParts), part ? &tm_q_lo : &tm_q_hi, a_full, kc * KC, qrow,
                     pol_q);
            if (L.tail_narrow)
              load(ab + a_res_off(L, nreg, 0, Tr::kAParts), &tm_q_tail, a_full, nreg * KC, qrow, pol_q);
          }
        }
        const int nreg = L.nkc - (L.tail_narrow ? 1 : 0);
        for (int t = t0; t < t1 && ok; ++t) {
          const int T_i = A.items[ii].num_tiles;
          const int tx_row = ((t - rot + T_i) % T_i) * kTileRows + half_row;  // database tile of position t
          for (int kc = 0; kc < nreg; ++kc, ++it) {
            const int s = (int)(it % (uint32_t)S);
            STAT_BEGIN(tw);
            if (!wait_or_abort(&empty[s], ((it / S) & 1u) ^ 1u, abort_flag)) {
              raise_abort(abort_flag, B.status, kErrWaitTimeout);
              ok = false;
              break;
            }
            STAT_END(tw, st_wait);
            uint8_t* st = smem + L.a_bytes + (uint32_t)s * L.stage_bytes;
            const bool with_tail = L.tail_narrow && kc == nreg - 1;
            uint32_t tx = (uint32_t)Tr::kBParts * L.b_chunk + (L.a_stream ? (uint32_t)Tr::kAParts * kAChunkBytes : 0u);
            if (with_tail) tx += L.b_tail + (L.a_stream ? kATailBytes : 0u);
            if (issuer) mbar_arrive_expect_tx(&full[s], tx_mul * tx);
            for (int part = 0; part < Tr::kBParts; ++part)
              load(st + part * L.b_chunk, part ? &tm_x_lo : &tm_x_hi, &full[s], kc * KC, tx_row, pol_db);
            if (L.a_stream)
              for (int part = 0; part < Tr::kAParts; ++part)
                load(st + stage_a_off<Tr::kAParts, Tr::kBParts>(L, part), part ? &tm_q_lo : &tm_q_hi, &full[s],
                     kc * KC, qb * kBM, pol_q);
            if (with_tail) {
              uint8_t* tl = st + stage_tail_off<Tr::kAParts, Tr::kBParts>(L);
              load(tl, &tm_x_tail, &full[s], nreg * KC, tx_row, pol_db);
              if (L.a_stream) load(tl + L.b_tail, &tm_q_tail, &full[s], nreg * KC, qb * kBM, pol_q);
            }
          }
        }
        ++unit;
      }
      STAT_FLUSH(kStatProducerWaitEmpty, st_wait);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0 && issuer) {
      constexpr uint32_t fmt = Tr::kFP8 ? 0u : 1u;  // e4m3 : bf16
      // a pair's MMA is 256 rows: this CTA's query block, then the partner's
      const uint32_t idesc = make_idesc(fmt, fmt, pair ? 2 * kBM : kBM, DUAL ? kBN / 2 : kBN);
      // the FP8 form's BF16 norm tail: the same shape, BF16 operands
      const uint32_t idesc16 = make_idesc(1u, 1u, pair ? 2 * kBM : kBM, DUAL ? kBN / 2 : kBN);
      auto mma = [&](uint32_t d_tmem, uint64_t ad, uint64_t bd, uint32_t acc, bool f8) {
        const uint32_t id = f8 ? idesc : idesc16;
        if constexpr (PAIR) {
          if (f8)
            mma_f8_ss_pair(d_tmem, ad, bd, id, acc);
          else
            mma_f16_ss_pair(d_tmem, ad, bd, id, acc);
        } else {
          if (f8)
            mma_f8_ss(d_tmem, ad, bd, id, acc);
          else
            mma_f16_ss(d_tmem, ad, bd, id, acc);
        }
      };
      // completion goes to the barrier at the same offset in both CTAs of a pair
      auto commit = [&](uint64_t* bar) {
        if constexpr (PAIR)
          mma_commit_pair(bar);
        else
          mma_commit(bar);
      };
      UnitWalk walk(blockIdx.x, B, rank);
      int ii, qb, t0, t1, u_ord, rot, unit = 0;
      bool gap;
      uint32_t it = 0, tc = 0;
      bool ok = true;
      STAT_DECL(st_full);
      STAT_DECL(st_acc);
      while (ok && walk.next(A, ii, qb, t0, t1, u_ord, gap, rot)) {
        if (!L.a_stream) {
          if (!wait_or_abort(a_full, unit & 1, abort_flag)) {
            raise_abort(abort_flag, B.status, kErrWaitTimeout);
            break;
          }
          tc_fence_after();
        }
        for (int t = t0; t < t1 && ok; ++t, ++tc) {
          const uint32_t slot = tc & 1u, use = tc >> 1;
          STAT_BEGIN(ta);
          if (!wait_or_abort(&acc_empty[slot], (use & 1u) ^ 1u, abort_flag, pair)) {
            raise_abort(abort_flag, B.status, kErrWaitTimeout);
            ok = false;
            break;
          }
          STAT_END(ta, st_acc);
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + slot * kBN;
          uint32_t accumulate = 0;
          const int nreg = L.nkc - (L.tail_narrow ? 1 : 0);
          const int fp8_tail = Tr::kFP8 ? A.items[ii].fp8_tail : 0;
          for (int kc = 0; kc < nreg; ++kc, ++it) {
            const int s = (int)(it % (uint32_t)S);
            STAT_BEGIN(tf);
            if (!wait_or_abort(&full[s], (it / S) & 1u, abort_flag)) {
              raise_abort(abort_flag, B.status, kErrWaitTimeout);
              ok = false;
              break;
            }
            STAT_END(tf, st_full);
            tc_fence_after();
            const uint32_t st = smem_u32(smem + L.a_bytes + (uint32_t)s * L.stage_bytes);
            const int rem = L.kdim - kc * KC;
            const int nsteps = rem >= KC ? KC / Tr::kStepElems : (rem + Tr::kStepElems - 1) / Tr::kStepElems;
            for (int j = 0; j < kQB; ++j) {  // dual: block j accumulates into columns j * 128 of the slot
              uint32_t acc_j = accumulate;
#pragma unroll
              for (int pr = 0; pr < Tr::kProducts; ++pr) {
                const uint32_t a_addr =
                    L.a_stream ? st + stage_a_off<Tr::kAParts, Tr::kBParts>(L, Tr::a_part(pr))
                               : smem_u32(smem + (uint32_t)j * L.a_block + a_res_off(L, kc, Tr::a_part(pr), Tr::kAParts));
                const uint32_t b_addr = st + Tr::b_part(pr) * L.b_chunk;
                for (int ks = 0; ks < nsteps; ++ks) {
                  const uint64_t ad = sw128_kmajor_desc(a_addr + ks * 32);
                  const uint64_t bd = sw128_kmajor_desc(b_addr + ks * 32);
                  mma(d_tmem + (uint32_t)j * (kBN / 2), ad, bd, acc_j, Tr::kFP8);
                  acc_j = 1;
                }
              }
            }
            accumulate = 1;
            if (Tr::kFP8 && fp8_tail > 0 && kc == nreg - 1) {
              // the BF16 norm tails: one K=16 step at their byte offset in the
              // last chunk (a 32-byte K step of the 128-byte swizzled rows, as
              // the FP8 steps before it), into the same FP32 accumulator
              const uint32_t toff = (uint32_t)(fp8_tail - kc * KC);
              for (int j = 0; j < kQB; ++j) {
                const uint32_t a_addr =
                    L.a_stream ? st + stage_a_off<Tr::kAParts, Tr::kBParts>(L, 0)
                               : smem_u32(smem + (uint32_t)j * L.a_block + a_res_off(L, kc, 0, Tr::kAParts));
                mma(d_tmem + (uint32_t)j * (kBN / 2), sw128_kmajor_desc(a_addr + toff), sw128_kmajor_desc(st + toff), 1,
                    false);
              }
            }
            if (L.tail_narrow && kc == nreg - 1) {
              // the 16 norm columns: only hi x hi carries them (lo rows are zero
              // there), so one K step of product 0 with the 32-byte-swizzled tiles
              const uint32_t tl = st + stage_tail_off<Tr::kAParts, Tr::kBParts>(L);
              for (int j = 0; j < kQB; ++j) {
                const uint32_t a_addr =
                    L.a_stream ? tl + L.b_tail
                               : smem_u32(smem + (uint32_t)j * L.a_block + a_res_off(L, nreg, 0, Tr::kAParts));
                mma(d_tmem + (uint32_t)j * (kBN / 2), sw32_kmajor_desc(a_addr), sw32_kmajor_desc(tl), 1, false);
              }
            }
            commit(&empty[s]);
          }
          if (!ok) break;
          commit(&acc_full[slot]);
        }
        if (!L.a_stream) commit(a_empty);
        ++unit;
      }
      // Make sure every issued MMA has retired before TMEM is released (in
      // both CTAs of a pair: the commit reaches the partner's drain barrier).
      commit(drain);
      mbar_wait(drain, 0);
      STAT_FLUSH(kStatMmaWaitFull, st_full);
      STAT_FLUSH(kStatMmaWaitAccEmpty, st_acc);
    } else if (lane == 0 && pair) {
      // the partner's MMAs also write this CTA's TMEM and read its shared
      // memory: wait for its final commit before the teardown
      mbar_wait(drain, 0);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    // The WG warps ew, ew + 4, ... read the same TMEM lanes (queries) and split
    // each tile's four 64-column chunks between them: with two warps, warp g
    // takes the 128-column half g; with three, chunk c of the tile counted tc
    // goes to warp (4 tc + c) mod 3.  They share ONE candidate pool per
    // (query, unit): appends reserve slots with a shared-memory counter, and at
    // every S-th tile end the group meets at a named barrier, splits the pools
    // that need a selection between them, and meets again.  A shared pool sees
    // all of a tile's rows, so its bound tightens as one pool over the whole
    // tile would -- about half the survivors and selections of a pool per half.
    const int ew = warp - 2;       // 0..EW-1
    const int g = ew >> 2;         // this warp's index within its lane group
    const int lg = warp & 3;       // TMEM lane group this warp may access
    const int row = lg * 32 + lane;
    const int pair_bar = 1 + lg;   // named barrier of the WG warps of lane group lg
    constexpr int kGroupThreads = 32 * WG;
    uint32_t* hist = hist_all + ew * 256;
    int* cnt_s = reinterpret_cast<int*>(smem + L.pool_off);                   // [128 kQB] pool counts
    float* thr_s = reinterpret_cast<float*>(smem + L.pool_off) + kQB * kBM;   // [128 kQB] pool bounds
    const uint32_t lane_base = (uint32_t)(lg * 32) << 16;
    UnitWalk walk(blockIdx.x, B, rank);
    int ii, qb, t0, t1, u_ord, rot;
    bool gap;
    uint32_t tc = 0;
    bool ok = true;
    STAT_DECL(st_wait);
    STAT_DECL(st_filter);
    STAT_DECL(st_refresh);
    STAT_DECL(st_nref);
    STAT_DECL(st_surv);
    STAT_DECL(st_slow);
    STAT_DECL(st_iters);
    STAT_DECL(st_tmem);
    STAT_DECL(st_bar);
#ifdef CURPLSH_FUSED_STATS
    if (threadIdx.x == 64 && B.stats) g_radix_pass_counter = &B.stats[kStatRadixPasses];
#endif
    while (ok && walk.next(A, ii, qb, t0, t1, u_ord, gap, rot)) {
      const FusedItem& p = A.items[ii];
      const int P = p.pool_cap;
      const int U = p.units_per_block;
      const int S = pool_sync_tiles(P, p.kprime);
      if (u_ord < 0 || u_ord >= U) {  // identical in every epilogue warp: both of a pair leave here
        raise_abort(abort_flag, B.status, kErrBadSchedule);
        break;
      }
      // dual: warp g filters query block qb + g and owns its pools alone
      const int qbw = DUAL ? qb + g : qb;
      const int crow = DUAL ? g * kBM + row : row;  // this lane's pool count / bound slot
      const int q = qbw * kBM + row;
      const bool valid = q < p.nq;
      const float qn = valid ? p.q_norms[q] : 0.f;
      float m2s = -2.f;
      if (Tr::kFP8) m2s = valid ? -2.f * p.q_scale[q] : 0.f;
      // FP8 with one scale s for every database row: d = ||x||^2 + (-2 s_q s) acc
      const bool uniform = Tr::kFP8 && p.db_scale_uniform > 0.f;
      const float ku = m2s * p.db_scale_uniform;
      // with the norm tails the accumulator is d / ku: the filter compares
      // ku acc with the bound and scales only the survivors (km = 1: the
      // accumulator is d itself or is made d below)
      const bool fold = Tr::kFP8 && p.fp8_tail > 0;
      const float km = fold ? ku : 1.f;
      auto key_d = [&](float x) -> float { return Tr::kFolded ? x : fmaf(km, x, qn); };
      const size_t pool_row0 = (size_t)qbw * kBM;  // pool index of lane-group row 0 is added per lane
      auto pool_of = [&](int r) -> uint64_t* {
        return p.pools + ((pool_row0 + (size_t)r) * U + (size_t)u_ord) * (size_t)P;
      };
      uint64_t* pool = pool_of(row);
      // a new unit starts with an empty pool (the previous unit's last barrier
      // ordered every use of the old state before this)
      if (DUAL || g == 0) {
        cnt_s[crow] = 0;
        thr_s[crow] = 3.402823466e38f;
      }
      if constexpr (DUAL)
        __syncwarp();
      else
        bar_sync_named(pair_bar, kGroupThreads);
      float thr = 3.402823466e38f;  // FLT_MAX: admits every finite distance until a pool fills

      // Selections of the pools in `need` (lane bits of this lane group; warp g
      // owns the pools of lanes l with l mod WG = g, so two warps never touch
      // the same pool's state).  Each keeps `keep` keys, records the pool's new
      // count and bound in shared memory and publishes a full set's k'-th
      // distance to q_bound.
      auto refresh = [&](uint32_t need, int keep) {
        STAT_BEGIN(tr);
        while (need) {
          const int src = __ffs(need) - 1;
          need &= need - 1;
          STAT_INC(st_nref, 1);
          const int r = lg * 32 + src;
          const int cr = (DUAL ? g * kBM : 0) + r;
          const int n_src = cnt_s[cr];
          int kept = 0;
          const uint64_t kmax = warp_select_keep_any(pool_of(r), n_src < P ? n_src : P, keep, P, hist, kept);
          if (lane == src) {
            const uint32_t ord = (uint32_t)(kmax >> 32);
            cnt_s[cr] = kept;
            thr_s[cr] = fminf(thr_s[cr], thr_from<Tr::kFolded>(ord2f(ord), qn));
            // only a full set of k' keys bounds the global k'-th distance
            if (kept >= p.kprime) atomicMin(&p.q_bound[q], ord);
          }
        }
        STAT_END(tr, st_refresh);
      };

      // the shared bound is an L2 round trip: load it one tile ahead
      uint32_t nb_ob = kOrdInf;
      if (valid) nb_ob = ld_relaxed_u32(&p.q_bound[q]);
      for (int t = t0; t < t1; ++t, ++tc) {
        const uint32_t slot = tc & 1u, use = tc >> 1;
        const int tphys = (t - rot + p.num_tiles) % p.num_tiles;  // database tile of position t
        thr = fminf(thr, thr_s[crow]);
        if (nb_ob != kOrdInf) thr = fminf(thr, thr_from<Tr::kFolded>(ord2f(nb_ob), qn));
        const float thr_up = next_above(thr);  // d <= thr  <=>  d < thr_up
        if (valid) nb_ob = ld_relaxed_u32(&p.q_bound[q]);
        // this warp's 64-column chunks of the tile (-1: none): 2g and 2g + 1
        // with two warps per lane group; with three, the c with 4 tc + c = g
        // (mod 3), i.e. c1 = (g - tc) mod 3 and, when c1 = 0, also 3
        int my_c[2];
        if constexpr (WG == 2) {
          my_c[0] = 2 * g;
          my_c[1] = 2 * g + 1;
        } else {
          my_c[0] = (int)(((uint32_t)g + 3u - tc % 3u) % 3u);
          my_c[1] = my_c[0] == 0 ? 3 : -1;
        }
        // FP8: the database norms and scales of these columns, loaded before
        // the accumulator wait (their latency overlaps it) and staged in the
        // warp's histogram area, which is free outside a refresh
        float pxn[4], psx[4];
        if (Tr::kFP8 && !fold) {
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int cc = my_c[i >> 1] < 0 ? my_c[0] : my_c[i >> 1];
            // < nb_pad: rows are padded to whole tiles (a strided sample has no padding)
            const int c0 = tphys * kTileRows + (DUAL ? cc - 2 * g : cc) * 64 + lane + 32 * (i & 1);
            const size_t c = MINIMA ? (size_t)c0 * (size_t)p.db_step : (size_t)c0;
            pxn[i] = __ldg(p.db_norms + c);
            psx[i] = uniform ? 0.f : __ldg(p.db_scale + c);
          }
        }
        STAT_BEGIN(tw);
        bool got = wait_or_abort(&acc_full[slot], use & 1u, abort_flag);
        if (!got) raise_abort(abort_flag, B.status, kErrWaitTimeout);
        STAT_END(tw, st_wait);
        // an aborting warp skips the tile but still meets its partner below
        if (got) {
        STAT_BEGIN(tfl);
        tc_fence_after();
        float bmin = 3.402823466e38f;  // block-minimum mode: smallest distance of this half tile
        float* colv = reinterpret_cast<float*>(hist);  // [128] norms, then [128] scales
        if (Tr::kFP8 && !fold) {
          __syncwarp();
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            colv[lane + 32 * i] = pxn[i];
            colv[kHalfN + lane + 32 * i] = psx[i];
          }
          __syncwarp();
        }
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
          const int ch = my_c[h];
          if (ch < 0) break;
          uint32_t v[64];
          STAT_BEGIN(ttm);
          tmem_ld_32x32b_x64(tmem_base + lane_base + slot * kBN + ch * 64, v);
          tmem_ld_wait();
          STAT_END(ttm, st_tmem);
          const int col0 = tphys * kTileRows + (DUAL ? ch - 2 * g : ch) * 64;
          // coarse distances of the 64 columns (two independent 32-column halves)
          float da[32], db[32];
          if (Tr::kFolded || fold) {
            // the accumulator already is ||q||^2 + ||x||^2 - 2 q.x (BF16 and
            // exact forms) or (||x||^2 - 2 q.x) / ku (FP8 with norm tails)
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              da[j] = __uint_as_float(v[j]);
              db[j] = __uint_as_float(v[32 + j]);
            }
            if (MINIMA && fold) {
#pragma unroll
              for (int j = 0; j < 32; j += 2) {
                mul2_f32(da[j], da[j + 1], da[j], da[j + 1], ku, ku);
                mul2_f32(db[j], db[j + 1], db[j], db[j + 1], ku, ku);
              }
            }
          } else {
            const float4* xn4 = reinterpret_cast<const float4*>(colv + h * 64);
            const float4* sx4 = reinterpret_cast<const float4*>(colv + kHalfN + h * 64);
            if (uniform) {
#pragma unroll
              for (int j4 = 0; j4 < 16; ++j4) {
                const float4 xn = xn4[j4];
                float* dst = j4 < 8 ? da : db;
                const int o = (j4 & 7) * 4;
                fma2_f32(dst[o + 0], dst[o + 1], __uint_as_float(v[4 * j4 + 0]), __uint_as_float(v[4 * j4 + 1]), ku,
                         ku, xn.x, xn.y);
                fma2_f32(dst[o + 2], dst[o + 3], __uint_as_float(v[4 * j4 + 2]), __uint_as_float(v[4 * j4 + 3]), ku,
                         ku, xn.z, xn.w);
              }
            } else
#pragma unroll
            for (int j4 = 0; j4 < 16; ++j4) {
              const float4 xn = xn4[j4];
              const float4 sx = sx4[j4];
              float* dst = j4 < 8 ? da : db;
              const int o = (j4 & 7) * 4;
              // fmaf(acc * s_x, -2 s_q, ||x||^2) on column pairs
              float p0, p1, p2, p3;
              mul2_f32(p0, p1, __uint_as_float(v[4 * j4 + 0]), __uint_as_float(v[4 * j4 + 1]), sx.x, sx.y);
              mul2_f32(p2, p3, __uint_as_float(v[4 * j4 + 2]), __uint_as_float(v[4 * j4 + 3]), sx.z, sx.w);
              fma2_f32(dst[o + 0], dst[o + 1], p0, p1, m2s, m2s, xn.x, xn.y);
              fma2_f32(dst[o + 2], dst[o + 3], p2, p3, m2s, m2s, xn.z, xn.w);
            }
          }
          if (MINIMA) {
            // block-minimum mode: no survivors, only the half tile's smallest
            // distance (columns past nb excluded)
            const int lim = p.nb - col0;
            float mm[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {  // a tree, not one dependent chain
              const float a0 = j < lim ? da[j] : 3.402823466e38f;
              const float a1 = 16 + j < lim ? da[16 + j] : 3.402823466e38f;
              const float b0 = 32 + j < lim ? db[j] : 3.402823466e38f;
              const float b1 = 48 + j < lim ? db[16 + j] : 3.402823466e38f;
              mm[j] = fminf(fminf(a0, a1), fminf(b0, b1));
            }
#pragma unroll
            for (int w = 8; w > 0; w >>= 1)
#pragma unroll
              for (int j = 0; j < w; ++j) mm[j] = fminf(mm[j], mm[j + w]);
            bmin = fminf(bmin, mm[0]);
            continue;
          }
#if CURPLSH_MIN_FIRST
          if (!__any_sync(0xffffffffu, valid && min64(da, db) < thr_up)) continue;
#endif
          // survivor masks: bit j of ma / mb for column j of da / db
          uint32_t ma, mb;
          // the FP32-exact form keeps compare masks: with three products per
          // tile it is bound by the tensor pipe, and the packed-FMA masks
          // measured slower there (10M-row sphere: 70.9 vs 77.0 ms)
          if (Tr::kProducts == 3) {
            ma = survive_mask32_cmp(da, thr);
            mb = survive_mask32_cmp(db, thr);
          } else {
            constexpr int kChain = Tr::kFP8 ? 32 : 16;
            ma = survive_mask32<kChain>(da, km, thr_up);
            mb = survive_mask32<kChain>(db, km, thr_up);
          }
          if (!valid) ma = mb = 0u;
          // database rows beyond nb (padding of the last tile) never survive
          if (col0 + 64 > p.nb) {
            const int lim = p.nb - col0;
            ma &= lim <= 0 ? 0u : (lim >= 32 ? ~0u : ((1u << lim) - 1u));
            mb &= lim <= 32 ? 0u : (lim >= 64 ? ~0u : ((1u << (lim - 32)) - 1u));
          }
          if (__any_sync(0xffffffffu, (ma | mb) != 0u)) {
            STAT_INC(st_slow, 1);
#ifdef CURPLSH_FUSED_STATS
            {
              int mx = __popc(ma) + __popc(mb);
#pragma unroll
              for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
              STAT_INC(st_iters, mx);
            }
#endif
            // A lane rarely has more than one survivor per 32 columns: take the
            // first of each half with a register select tree (no local memory),
            // a second one the same way, and stash only for the rare rest.
            // slots for this lane's survivors of the 64 columns, reserved at
            // once by every lane (most add 0): no branch, so the select trees
            // below run while the shared atomic is in flight
            int n = atomicAdd(&cnt_s[crow], __popc(ma) + __popc(mb));
            if ((ma & mb) == ~0u) {
              // every column survives (a pool with no bound yet): append all
              // 64 keys in column order, no extraction
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (n + j < P) pool[n + j] = make_key(key_d(da[j]), (uint32_t)(col0 + j));
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (n + 32 + j < P)
                  pool[n + 32 + j] = make_key(key_d(db[j]), (uint32_t)(col0 + 32 + j));
              n += 64;
              ma = mb = 0u;
              STAT_INC(st_surv, 64);
            }
            // the first survivor of each half, straight-line (j = -1: none)
            auto take2 = [&]() {
              const int ja = __ffs(ma) - 1, jb = __ffs(mb) - 1;
              const float xa = select32(da, ja & 31), xb = select32(db, jb & 31);
              ma &= ma - 1u;
              mb &= mb - 1u;
              const bool ha = ja >= 0, hb = jb >= 0;
              if (ha && n < P) pool[n] = make_key(key_d(xa), (uint32_t)(col0 + ja));
              n += ha ? 1 : 0;
              if (hb && n < P) pool[n] = make_key(key_d(xb), (uint32_t)(col0 + 32 + jb));
              n += hb ? 1 : 0;
              STAT_INC(st_surv, (ha ? 1 : 0) + (hb ? 1 : 0));
            };
            take2();
            if (__any_sync(0xffffffffu, (ma | mb) != 0u)) {
              take2();
              if (__any_sync(0xffffffffu, (ma | mb) != 0u)) {
                float stash[64];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                  stash[j] = da[j];
                  stash[32 + j] = db[j];
                }
                uint64_t mm = ((uint64_t)mb << 32) | ma;
                while (mm) {
                  const int j = __ffsll((long long)mm) - 1;
                  mm &= mm - 1;
                  if (n < P) pool[n] = make_key(key_d(stash[j]), (uint32_t)(col0 + j));
                  ++n;
                  STAT_INC(st_surv, 1);
                }
              }
            }
          }
        }
        if (MINIMA && valid)
          p.minima[(size_t)q * (2 * (size_t)p.num_tiles) + 2 * (size_t)tphys + g] =
              Tr::kFolded ? bmin : bmin + qn;
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          if constexpr (PAIR)
            mbar_arrive_remote(&acc_empty[slot], 0);  // the issuer's barrier counts both CTAs
          else
            mbar_arrive(&acc_empty[slot]);
        }
        STAT_END(tfl, st_filter);
        }  // got
        // every S tiles (and at the unit's end) meet the partner warp; leave
        // together if either aborted
        if ((t - t0 + 1) % S != 0 && t + 1 < t1) continue;
        STAT_BEGIN(tb1);
        bool leave;
        if constexpr (DUAL)
          leave = __any_sync(0xffffffffu, !got || *abort_flag != 0);
        else
          leave = bar_red_or(pair_bar, kGroupThreads, !got || *abort_flag != 0);
        STAT_END(tb1, st_bar);
        if (leave) {
          ok = false;
          break;
        }
        // pools that may not have room for the next S tiles (both halves),
        // or, at the unit's end, every pool above k' (the merge pass reads at
        // most k' keys' worth beyond what it needs)
        const int lim = t + 1 < t1 ? P - S * kTileRows : p.kprime;
        const bool mine = DUAL || (lane % WG) == g;
        const int cn = mine ? cnt_s[crow] : 0;
        if (cn > P) atomicOr(B.status, kErrPoolOverflow);
        refresh(__ballot_sync(0xffffffffu, mine && valid && cn > lim), p.kprime);
        STAT_BEGIN(tb2);
        if constexpr (DUAL)
          __syncwarp();
        else
          bar_sync_named(pair_bar, kGroupThreads);
        STAT_END(tb2, st_bar);
      }
      if (!ok) break;
      // a refresh may keep a few more than k' keys (unsorted): record them all;
      // the merge pass selects exactly
      if (!MINIMA && valid && (DUAL || g == 0)) {
        const int cn = cnt_s[crow];
        p.pool_counts[(pool_row0 + row) * U + u_ord] = cn < P ? cn : P;
        if (gap) p.pool_counts[(pool_row0 + row) * U + u_ord - 1] = 0;
      }
      if constexpr (DUAL)
        __syncwarp();
      else
        bar_sync_named(pair_bar, kGroupThreads);  // the counts are read before the next unit resets them
    }
    if (lane == 0) {
      STAT_FLUSH(kStatEpiWaitAccFull, st_wait);
      STAT_FLUSH(kStatEpiFilter, st_filter);
      STAT_FLUSH(kStatEpiRefresh, st_refresh);
      STAT_FLUSH(kStatRefreshes, st_nref);
      STAT_FLUSH(kStatSlowChunks, st_slow);
      STAT_FLUSH(kStatLoopIters, st_iters);
      STAT_FLUSH(kStatTmemCycles, st_tmem);
      STAT_FLUSH(kStatPairBarrier, st_bar);
    }
    STAT_FLUSH(kStatSurvivors, st_surv);
  }

  tc_fence_before();
  // a pair releases its TMEM together, and neither CTA leaves while the
  // other may still signal its barriers or read its shared memory
  if constexpr (PAIR)
    cluster_sync();
  else
    __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    if constexpr (PAIR)
      tmem_dealloc_pair(tmem_base, 512);
    else
      tmem_dealloc(tmem_base, 512);
  }
#ifdef CURPLSH_FUSED_STATS
  if (threadIdx.x == 0 && B.stats) atomicAdd(&B.stats[kStatCtaCycles], (unsigned long long)(clock64() - t_kernel));
#endif
}

// ------------------------------------------------------------------ host side
namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
  }
  return fn;
}

// 2-D K-major operand map: rows x ld elements, box = (128 bytes of K) x box_rows
// with the 128-byte swizzle, or (narrow) 32 bytes of K with the 32-byte
// swizzle; zero fill out of bounds.  Map row j is stored row j * row_step.
bool make_map(CUtensorMap* m, const void* base, bool fp8, long long rows, long long ld_elems, int box_rows,
              bool narrow = false, int row_step = 1) {
  EncodeTiledFn fn = get_encode_fn();
  if (!fn) return false;
  const int esz = fp8 ? 1 : 2;
  cuuint64_t dims[2] = {(cuuint64_t)ld_elems, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld_elems * esz * (row_step > 1 ? row_step : 1))};
  cuuint32_t box[2] = {(cuuint32_t)((narrow ? kTailRowBytes : kChunkBytes) / esz), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, fp8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                  const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  narrow ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Raises the kernel's dynamic shared memory limit once per device.
template <int FORM, int MAXI, bool MINIMA = false, bool PAIR = false, bool DUAL = false>
cudaError_t ensure_attributes() {
  static bool attr_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_done[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(fused_knn_kernel<FORM, MAXI, MINIMA, PAIR, DUAL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         227 * 1024);
    if (e != cudaSuccess) return e;
    attr_done[dev & 63] = true;
  }
  return cudaSuccess;
}

template <int FORM, int MAXI, bool MINIMA = false, bool PAIR = false, bool DUAL = false>
cudaError_t launch_form(const FusedItemSpec* specs, const FusedItemPlan* plans, int n, const FusedBatchPlan& bp,
                        uint32_t* status, unsigned long long* stats, uint32_t smem, cudaStream_t st,
                        const int* run_if) {
  cudaError_t e = ensure_attributes<FORM, MAXI, MINIMA, PAIR, DUAL>();
  if (e != cudaSuccess) return e;
  smem = make_layout(FORM, specs[0].d, PAIR ? 1 : 0, epi_warps_for(MINIMA), DUAL ? 1 : 0).total;  // this instance's
  FusedArgs<MAXI> a;
  memset(&a, 0, sizeof(a));
  a.B.num_items = n;
  a.B.form = FORM;
  a.B.d = specs[0].d;
  a.B.pair = bp.pair;
  a.B.total_work = bp.total_work;
  a.B.work_per_cta = bp.work_per_cta;
  a.B.dual = bp.dual;
  const int xrows = kBN >> (bp.pair | bp.dual);  // database rows one CTA loads per tile
  a.B.status = status;
  a.B.stats = stats;
  a.B.run_if = run_if;
  const bool fp8 = FORM == kFormFP8;
  for (int i = 0; i < n; ++i) {
    const FusedItemSpec& f = specs[i];
    const FusedItemPlan& pl = plans[i];
    FusedItem& it = a.items[i];
    it.nq = f.nq;
    it.nb = f.nb;
    it.kprime = f.kprime;
    it.pool_cap = f.pool_cap;
    it.num_qblocks = pl.num_qblocks;
    it.num_tiles = pl.num_tiles;
    it.units_per_block = pl.units_per_block;
    it.split_tiles = pl.split_tiles;
    it.work_begin = pl.work_begin;
    it.work_end = pl.work_end;
    it.db_norms = f.xn;
    it.db_scale = f.xs;
    it.q_norms = f.qn;
    it.q_scale = f.qs;
    it.pools = f.pools;
    it.pool_counts = f.pool_counts;
    it.q_bound = f.q_bound;
    it.db_step = f.db_step > 1 ? f.db_step : 1;
    it.db_scale_uniform = f.xs_uniform;
    it.fp8_tail = (fp8 && f.xs_uniform > 0.f) ? (int)fp8_tail_offset(f.d, f.ld8) : 0;
    it.minima = f.minima;
    CUtensorMap* m = &a.maps[i * kMapsPerItem];
    const void* qh = fp8 ? (const void*)f.q8 : (const void*)f.qh;
    const void* xh = fp8 ? (const void*)f.x8 : (const void*)f.xh;
    const long long ldq = fp8 ? f.ld8 : f.ld16;
    const int step = it.db_step;
    if (!make_map(&m[kMapQHi], qh, fp8, f.nq_pad, ldq, kBM) ||
        !make_map(&m[kMapXHi], xh, fp8, f.nb_pad, ldq, xrows, false, step))
      return cudaErrorInvalidValue;
    if (FORM == kFormExact) {
      if (!make_map(&m[kMapQLo], f.ql, false, f.nq_pad, f.ld16, kBM) ||
          !make_map(&m[kMapXLo], f.xl, false, f.nb_pad, f.ld16, xrows, false, step))
        return cudaErrorInvalidValue;
    } else {
      m[kMapQLo] = m[kMapQHi];
      m[kMapXLo] = m[kMapXHi];
    }
    if (FORM != kFormFP8) {
      if (!make_map(&m[kMapQTail], f.qh, false, f.nq_pad, f.ld16, kBM, true) ||
          !make_map(&m[kMapXTail], f.xh, false, f.nb_pad, f.ld16, xrows, true, step))
        return cudaErrorInvalidValue;
    } else {
      m[kMapQTail] = m[kMapQHi];
      m[kMapXTail] = m[kMapXHi];
    }
  }
  if (!PAIR) {
    fused_knn_kernel<FORM, MAXI, MINIMA, PAIR, DUAL><<<bp.grid, threads_for(MINIMA), smem, st>>>(a);
    return cudaGetLastError();
  }
  if (bp.grid % 2) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)bp.grid, 1, 1);
  cfg.blockDim = dim3(threads_for(MINIMA), 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, fused_knn_kernel<FORM, MAXI, MINIMA, PAIR, DUAL>, a);
}

template <int FORM>
cudaError_t launch_form_any(const FusedItemSpec* specs, const FusedItemPlan* plans, int n, const FusedBatchPlan& bp,
                            uint32_t* status, unsigned long long* stats, uint32_t smem, cudaStream_t st,
                            const int* run_if) {
  if (n == 1 && specs[0].minima)
    return bp.pair ? launch_form<FORM, 1, true, true>(specs, plans, n, bp, status, stats, smem, st, run_if)
                   : launch_form<FORM, 1, true>(specs, plans, n, bp, status, stats, smem, st, run_if);
  for (int i = 0; i < n; ++i)
    if (specs[i].minima) return cudaErrorInvalidValue;  // block-minimum mode is single-item
  if constexpr (FORM != kFormExact) {
    if (bp.dual)
      return n == 1 ? launch_form<FORM, 1, false, false, true>(specs, plans, n, bp, status, stats, smem, st, run_if)
                    : launch_form<FORM, kFusedMaxItems, false, false, true>(specs, plans, n, bp, status, stats, smem,
                                                                          st, run_if);
  } else {
    if (bp.dual) return cudaErrorInvalidValue;  // dual blocks are planned for BF16 / FP8 only
  }
  if (n == 1)
    return bp.pair ? launch_form<FORM, 1, false, true>(specs, plans, n, bp, status, stats, smem, st, run_if)
                   : launch_form<FORM, 1>(specs, plans, n, bp, status, stats, smem, st, run_if);
  return bp.pair ? launch_form<FORM, kFusedMaxItems, false, true>(specs, plans, n, bp, status, stats, smem, st, run_if)
                 : launch_form<FORM, kFusedMaxItems>(specs, plans, n, bp, status, stats, smem, st, run_if);
}

}  // namespace

#ifndef CURPLSH_DUAL_DEFAULT
#define CURPLSH_DUAL_DEFAULT 1
#endif
namespace {
std::atomic<int> g_cta_pairs{kPairsAuto};
std::atomic<int> g_dual{CURPLSH_DUAL_DEFAULT};
// Automatic CTA pairs: from these dimensions on, the MMAs of a tile are heavy
// enough that halving each SM's database bytes per query pays.  Measured on
// 10^6 N(0,1) BF16-valued rows, 4,096 queries (k = 10) and 2,048 (k = 100),
// single CTAs -> pairs: BF16 d = 128 2.33 -> 2.93 ms, 256 3.15 -> 3.44, 320
// 3.59 -> 3.48, 384 4.67 -> 3.83, 512 5.98 -> 4.54; FP32-exact d = 128 3.44 ->
// 3.43, 192 4.75 -> 4.36, 256 6.10 -> 5.55, 512 11.5 -> 9.9 (identical results).
constexpr int kPairMinDimBF16 = 320;
constexpr int kPairMinDimExact = 192;
}  // namespace

void set_cta_pairs(int mode) {
  g_cta_pairs.store(mode == kPairsAuto ? kPairsAuto : (mode ? 1 : 0), std::memory_order_relaxed);
}
int get_cta_pairs() { return g_cta_pairs.load(std::memory_order_relaxed); }
void set_dual_blocks(int on) { g_dual.store(on ? 1 : 0, std::memory_order_relaxed); }
int get_dual_blocks() { return g_dual.load(std::memory_order_relaxed); }

void plan_fused_batch(const FusedItemSpec* specs, int n, int max_ctas, FusedItemPlan* plans, FusedBatchPlan* out,
                      int form) {
  // Query groups of two blocks (dual blocks in one CTA for BF16/FP8, else CTA
  // pairs when on) when there are enough query blocks and few groups would be
  // half empty (an item with an odd block count leaves its last group one
  // block short)
  long long blocks = 0, odd = 0;
  for (int i = 0; i < n; ++i) {
    const long long g = specs[i].nb > 0 ? (specs[i].nq + kBM - 1) / kBM : 0;
    blocks += g;
    odd += g & 1;
  }
  const bool grouped = blocks >= 4 && odd * 8 <= blocks;
  // dual blocks need both query blocks resident in shared memory
  const bool dual_fits = n > 0 && specs[0].d > 0 && !make_layout(form, specs[0].d, 0, kPoolEpiWarps, 1).a_stream;
  // FP8 only: its MMAs are light, so halving the tile bytes per query pays
  // (sphere 39.6 -> 37.7 ms); the BF16 pass got slower (3.50 -> 4.52 ms on the
  // integer mixture: twice the MMA instructions and shared-memory A reads)
  const int dual = (grouped && dual_fits && get_dual_blocks() && form == kFormFP8) ? 1 : 0;
  const int pm = get_cta_pairs();
  const int d0 = n > 0 ? specs[0].d : 0;
  const bool want_pair = pm == 1 || (pm == kPairsAuto && ((form == kFormBF16 && d0 >= kPairMinDimBF16) ||
                                                          (form == kFormExact && d0 >= kPairMinDimExact)));
  const int pair = (!dual && grouped && want_pair && max_ctas >= 2) ? 1 : 0;
  const int rows = kBM << (pair | dual);
  const int tile_rows = dual ? kBN / 2 : kBN;
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    FusedItemPlan& pl = plans[i];
    pl.num_qblocks = specs[i].nb > 0 ? (specs[i].nq + rows - 1) / rows : 0;
    pl.num_tiles = (specs[i].nb + tile_rows - 1) / tile_rows;
    pl.split_tiles = specs[i].split_tiles > 0 && specs[i].split_tiles < pl.num_tiles ? specs[i].split_tiles
                                                                                      : std::max(pl.num_tiles, 1);
    pl.work_begin = total;
    total += (long long)pl.num_qblocks * pl.num_tiles;
    pl.work_end = total;
    pl.pair = pair;
    pl.dual = dual;
  }
  const long long units = max_ctas >> pair;  // CTAs, or pairs of CTAs
  long long grid = units < total ? units : total;
  if (grid < 1) grid = 1;
  out->pair = pair;
  out->dual = dual;
  out->total_work = total;
  out->work_per_cta = total > 0 ? (total + grid - 1) / grid : 1;
  out->grid = total > 0 ? (int)((total + out->work_per_cta - 1) / out->work_per_cta) << pair : 0;
  const long long W = out->work_per_cta;
  for (int i = 0; i < n; ++i) {
    FusedItemPlan& pl = plans[i];
    int U = 1;
    for (int qb = 0; qb < pl.num_qblocks; ++qb) {
      const long long base = pl.work_begin + (long long)qb * pl.num_tiles;
      const long long u = (base + pl.num_tiles - 1) / W - base / W + (pl.num_tiles - 1) / pl.split_tiles + 1;
      if (u > U) U = (int)u;
    }
    pl.units_per_block = U;
  }
}

void plan_fused(int nq, int nb, int num_sms, FusedPlan* out, int split_q4, int form, int d) {
  FusedItemSpec s{};
  s.nq = nq;
  s.nb = nb;
  s.d = d;
  FusedItemPlan ip;
  FusedBatchPlan bp;
  plan_fused_batch(&s, 1, num_sms, &ip, &bp, form);
  if (split_q4 < 4 && bp.grid > 0) {
    s.split_tiles = split_tiles_for(bp.work_per_cta, split_q4);
    plan_fused_batch(&s, 1, num_sms, &ip, &bp, form);
  }
  out->num_qblocks = ip.num_qblocks;
  out->num_tiles = ip.num_tiles;
  out->work_per_cta = bp.work_per_cta;
  out->grid = bp.grid;
  out->pair = bp.pair;
  out->dual = bp.dual;
  out->units_per_block = ip.units_per_block;
  out->split_tiles = ip.split_tiles;
}

uint32_t fused_smem_bytes(int form, int d) { return make_layout(form, d).total; }

cudaError_t prepare_fused_kernels(int form) {
  cudaError_t e;
  switch (form) {
    case kFormExact:
      e = ensure_attributes<kFormExact, 1>();
      if (e == cudaSuccess) e = ensure_attributes<kFormExact, 1, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormExact, 1, false, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormExact, 1, true, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormExact, kFusedMaxItems, false, true>();
      return e != cudaSuccess ? e : ensure_attributes<kFormExact, kFusedMaxItems>();
    case kFormBF16:
      e = ensure_attributes<kFormBF16, 1>();
      if (e == cudaSuccess) e = ensure_attributes<kFormBF16, 1, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormBF16, 1, false, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormBF16, 1, true, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormBF16, kFusedMaxItems, false, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormBF16, 1, false, false, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormBF16, kFusedMaxItems, false, false, true>();
      return e != cudaSuccess ? e : ensure_attributes<kFormBF16, kFusedMaxItems>();
    case kFormFP8:
      e = ensure_attributes<kFormFP8, 1>();
      if (e == cudaSuccess) e = ensure_attributes<kFormFP8, 1, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormFP8, 1, false, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormFP8, 1, true, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormFP8, kFusedMaxItems, false, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormFP8, 1, false, false, true>();
      if (e == cudaSuccess) e = ensure_attributes<kFormFP8, kFusedMaxItems, false, false, true>();
      return e != cudaSuccess ? e : ensure_attributes<kFormFP8, kFusedMaxItems>();
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fused_batch(int form, const FusedItemSpec* specs, const FusedItemPlan* plans, int n,
                               const FusedBatchPlan& bp, uint32_t* status, unsigned long long* stats,
                               cudaStream_t st, const int* run_if) {
  if (n < 1 || n > kFusedMaxItems) return cudaErrorInvalidValue;
  for (int i = 1; i < n; ++i)
    if (specs[i].d != specs[0].d) return cudaErrorInvalidValue;
  if (bp.grid == 0) return cudaSuccess;
  const uint32_t smem = make_layout(form, specs[0].d, bp.pair).total;
  if (smem > 227u * 1024u) return cudaErrorInvalidConfiguration;  // a layout bug, not a caller error
  switch (form) {
    case kFormExact:
      return launch_form_any<kFormExact>(specs, plans, n, bp, status, stats, smem, st, run_if);
    case kFormBF16:
      return launch_form_any<kFormBF16>(specs, plans, n, bp, status, stats, smem, st, run_if);
    case kFormFP8:
      return launch_form_any<kFormFP8>(specs, plans, n, bp, status, stats, smem, st, run_if);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fused(const FusedLaunch& f, cudaStream_t st) {
  FusedItemSpec s{};
  s.nq = f.nq;
  s.nb = f.nb;
  s.d = f.d;
  s.kprime = f.kprime;
  s.pool_cap = f.pool_cap;
  s.nq_pad = f.nq_pad;
  s.nb_pad = f.nb_pad;
  s.ld16 = f.ld16;
  s.ld8 = f.ld8;
  s.qh = f.qh;
  s.ql = f.ql;
  s.q8 = f.q8;
  s.qn = f.qn;
  s.qs = f.qs;
  s.xh = f.xh;
  s.xl = f.xl;
  s.x8 = f.x8;
  s.xn = f.xn;
  s.xs = f.xs;
  s.xs_uniform = f.xs_uniform;
  s.pools = f.pools;
  s.pool_counts = f.pool_counts;
  s.q_bound = f.q_bound;
  s.db_step = f.db_step;
  s.minima = f.minima;
  FusedItemPlan ip;
  ip.num_qblocks = f.plan.num_qblocks;
  ip.num_tiles = f.plan.num_tiles;
  ip.units_per_block = f.plan.units_per_block;
  ip.split_tiles = f.plan.split_tiles > 0 ? f.plan.split_tiles : std::max(f.plan.num_tiles, 1);
  ip.work_begin = 0;
  ip.work_end = (long long)f.plan.num_qblocks * f.plan.num_tiles;
  ip.pair = f.plan.pair;
  ip.dual = f.plan.dual;
  FusedBatchPlan bp;
  bp.total_work = ip.work_end;
  bp.work_per_cta = f.plan.work_per_cta;
  bp.grid = f.plan.grid;
  bp.pair = f.plan.pair;
  bp.dual = f.plan.dual;
  return launch_fused_batch(f.form, &s, &ip, 1, bp, f.status, f.stats, st, f.run_if);
}

}  // namespace curplsh_b200
