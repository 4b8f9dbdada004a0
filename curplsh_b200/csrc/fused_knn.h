// fused_knn.h -- host-side interface of the device passes (fused filter,
// merge + rerank, row preparation).  Internal to libcurplsh_b200.so.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

namespace curplsh_b200 {

struct FusedPlan {
  int num_qblocks = 0;        // G = ceil(nq / (128 << pair)): query blocks, or groups of two with CTA pairs
  int num_tiles = 0;          // T = ceil(nb / 256)
  long long work_per_cta = 0; // W
  int grid = 0;               // CTAs launched
  int units_per_block = 0;    // U: max units (pool lists) of one query block
  int split_tiles = 1;        // L: resolved unit length limit
  int pair = 0;               // 1: clusters of two CTAs share each 256-row MMA (two query blocks)
  int dual = 0;               // 1: one CTA holds two query blocks against 128-row database tiles
  // pool rows of the plan (pools and counts are indexed by query row)
  long long pool_rows() const { return (long long)num_qblocks * (128LL << (pair | dual)); }
};

// Tuned launch parameters for one (form, d, k, Q) bucket (tuning.cpp).
constexpr int kTuneDefaultHeadroom = 256;
constexpr int kTuneMinHeadroom = 128;
constexpr int kTuneMaxHeadroom = 8192;
struct TuneParams {
  int split_q4 = 4;                      // unit length limit in quarters of the search's own CTA range W
  int headroom = kTuneDefaultHeadroom;   // pool capacity = k' + room + max(k', headroom), rounded to 32
  bool tuned = false;                    // set by the autotuner (else the defaults below apply)
};
TuneParams tune_lookup(int form, int d, int k, long long nq);
// Split used when a bucket was never tuned: pools above 1024 keys take the
// streaming selection (several passes over global memory), so their units are
// halved, leaving more of the selection to the merge pass.
inline int default_split_q4(const TuneParams& t, int pool_cap) {
  return t.tuned ? t.split_q4 : (pool_cap > 1024 ? 2 : 4);
}
// Unit length limit for an item whose own CTA range is w_own tiles (>= 1).
inline int split_tiles_for(long long w_own, int split_q4) {
  const long long s = (w_own * split_q4 + 3) / 4;
  return (int)(s < 1 ? 1 : (s > (1LL << 30) ? (1LL << 30) : s));
}

struct FusedLaunch {
  int nq, nb, d, kprime, pool_cap, form;
  long long nq_pad, nb_pad, ld16, ld8;
  // query operands (device)
  const __nv_bfloat16* qh;
  const __nv_bfloat16* ql;
  const uint8_t* q8;
  const float* qn;
  const float* qs;
  // database operands (device)
  const __nv_bfloat16* xh;
  const __nv_bfloat16* xl;
  const uint8_t* x8;
  const float* xn;
  const float* xs;
  float xs_uniform = 0.f;   // > 0: one FP8 scale for every database row
  // database row j of this pass is stored row j * db_step (a strided sample when > 1)
  int db_step = 1;
  // non-null: block-minimum mode, see FusedItem::minima (pools are not used)
  float* minima = nullptr;
  // outputs / scratch
  uint64_t* pools;
  int* pool_counts;
  uint32_t* q_bound;
  uint32_t* status;
  unsigned long long* stats = nullptr;  // instrumented builds only
  const int* run_if = nullptr;          // non-null: the launch does nothing unless *run_if != 0
  FusedPlan plan;
};

// One search over at most num_sms CTAs.  split_q4 < 4 cuts units shorter than
// the CTA ranges (split_tiles_for(W, split_q4)); >= 4 leaves the ranges whole.
// `form` (-1: unknown) decides whether dual blocks may be used (BF16 and FP8).
void plan_fused(int nq, int nb, int num_sms, FusedPlan* out, int split_q4 = 4, int form = -1, int d = 0);
uint32_t fused_smem_bytes(int form, int d);
cudaError_t launch_fused(const FusedLaunch& f, cudaStream_t st);

// ---- batched form: several (queries, database) items of one form and one
// dimension in a single persistent launch.  The flattened work space is the
// concatenation of every item's (query block, tile) grid; each CTA takes a
// contiguous range of W units, so the load is balanced across items of any
// size.  A single search is the one-item case.
constexpr int kFusedMaxItems = 16;

struct FusedItemSpec {
  int nq, nb, d, kprime, pool_cap;
  int split_tiles;  // max tiles per unit (<= 0: no limit beyond the CTA ranges)
  long long nq_pad, nb_pad, ld16, ld8;
  const __nv_bfloat16* qh;
  const __nv_bfloat16* ql;
  const uint8_t* q8;
  const float* qn;
  const float* qs;
  const __nv_bfloat16* xh;
  const __nv_bfloat16* xl;
  const uint8_t* x8;
  const float* xn;
  const float* xs;
  float xs_uniform;         // > 0: one FP8 scale for every database row
  uint64_t* pools;          // [G*128][U][pool_cap]
  int* pool_counts;         // [G*128][U]
  uint32_t* q_bound;        // [nq_pad], initialised to all ones (or to estimated bounds)
  int db_step;              // database row j is stored row j * db_step (0 or 1: contiguous)
  float* minima;            // non-null: block-minimum mode (FusedItem::minima)
};
struct FusedItemPlan {
  int num_qblocks, num_tiles, units_per_block;  // num_qblocks: groups of 128 << pair query rows
  int split_tiles;  // resolved split length L (>= 1)
  long long work_begin, work_end;
  int pair;         // the launch's FusedBatchPlan::pair
  int dual;         // the launch's FusedBatchPlan::dual
};
struct FusedBatchPlan {
  long long total_work = 0, work_per_cta = 1;
  int grid = 0;
  int pair = 0;  // 1: clusters of two CTAs; work_per_cta is per pair and grid counts CTAs
  int dual = 0;  // 1: each CTA takes query groups of two blocks and 128-row database tiles
};
// CTA pairs on (1) or off (0, default) for the plans made after the call.
// CTA pairs: 0 off, 1 on (every grouped pass), kPairsAuto (the default): on
// for BF16 passes with d >= 320 and FP32-exact passes with d >= 192
constexpr int kPairsAuto = 2;
void set_cta_pairs(int mode);
int get_cta_pairs();
// Dual query blocks (BF16 / FP8) on or off for the plans made after the call.
void set_dual_blocks(int on);
int get_dual_blocks();
// Plans `n` items over at most `max_ctas` CTAs.  Only nq, nb and split_tiles
// of the specs are read, so pool sizes (which depend on units_per_block) can be computed
// from the plan before the pools are carved.
void plan_fused_batch(const FusedItemSpec* specs, int n, int max_ctas, FusedItemPlan* plans, FusedBatchPlan* out,
                      int form = -1);
// Sets the kernels' launch attributes on the current device (done lazily by
// the launches; call it before a stream capture).
cudaError_t prepare_fused_kernels(int form);
// `run_if` (optional, device): every CTA returns at once unless *run_if != 0
// (a pass that must run only after a failed check, decided on the device).
cudaError_t launch_fused_batch(int form, const FusedItemSpec* specs, const FusedItemPlan* plans, int n,
                               const FusedBatchPlan& bp, uint32_t* status, unsigned long long* stats,
                               cudaStream_t st, const int* run_if = nullptr);

// ---- sampled bound estimate (capi.cpp): a short fused pass over a strided
// sample of the database records per query the smallest distance of every
// 128-row block of the sample; the j-th smallest of those B block minima is
// the starting bound of every candidate pool of the full pass.
struct EstimatePlan {
  bool on = false;
  int rows = 0;    // sample rows (a multiple of 256)
  int step = 1;    // sample row j is database row j * step
  int blocks = 0;  // B = rows / 128 block minima per query
  int j = 0;       // rank of the estimate among the block minima
  FusedPlan plan;
};
// The estimate a search of nq queries with k' candidates against n rows uses
// (on == false: none), whatever the process-wide switch says.
EstimatePlan plan_estimate(int nq, long long n, int kp, int num_sms);
// The process-wide switch (curplsh_set_bound_estimate).
bool bound_estimate_enabled();

// Row preparation: squared norms (FP32), BF16 hi/lo split, FP8-E4M3 with a
// per-row FP32 scale.  Rows in [nrows, nrows_pad) are written as zeros with
// norm `pad_norm`.  Any of the output pointers may be null.  `aug` selects the
// augmented BF16 row layout (kAugNone / kAugDatabase / kAugQuery, see kAugCols):
// database rows get [n1 n2 n3 1 1 1] after column d, query rows are stored as -2q
// followed by [1 1 1 m1 m2 m3]; lo rows get zeros there.  kAugF8Query /
// kAugF8Database write the FP8 rows' BF16 norm tail (see fp8_tail_offset):
// query rows [a_h a_h a_l] with a = 1/s_q (a zero row takes scale 1), database
// rows [b_h b_l b_h] with b = -||x||^2 / (2 fixed_scale) (zeros without a
// fixed scale).
enum AugMode : int { kAugNone = 0, kAugDatabase = 1, kAugQuery = 2, kAugF8Query = 3, kAugF8Database = 4 };
// Byte offset of the FP8 rows' 32-byte BF16 norm tail, round_up(d, 32), when
// a row of stride ld8 has room for it inside its last 128-byte K chunk; else 0.
__host__ __device__ inline long long fp8_tail_offset(long long d, long long ld8) {
  const long long t8 = (d + 31) / 32 * 32;
  return (t8 % 128 != 0 && t8 + 32 <= ld8) ? t8 : 0;
}
// `lo_nonzero` (optional) gets a nonzero value when some real row element is
// not exactly representable in BF16 (its lo part is nonzero).
cudaError_t launch_prep_rows(const float* x, long long ldx, int nrows, long long nrows_pad, int d, float* norms,
                             float pad_norm, __nv_bfloat16* hi, __nv_bfloat16* lo, long long ld16, uint8_t* f8,
                             float* scale, long long ld8, cudaStream_t st, int aug = kAugNone,
                             uint32_t* lo_nonzero = nullptr, float fixed_scale = 0.f);
// out[0] / out[1] = order bits of the smallest / largest positive s[i], i < n
// (0xFFFFFFFF / 0 when there is none)
cudaError_t launch_positive_range(const float* s, long long n, uint32_t* out, cudaStream_t st);

// The same preparation for several row ranges of one dimension in a single
// launch.  Every pointer points at the segment's first row; source rows have
// stride d; rows [nrows, rows) are written as padding.
constexpr int kPrepMaxSegments = 128;
struct PrepSegment {
  const float* x;
  int nrows;              // real rows
  int rows;               // rows written (real + padding)
  long long block_begin;  // filled by launch_prep_segments
  float* norms;
  __nv_bfloat16* hi;
  __nv_bfloat16* lo;
  uint8_t* f8;
  float* scale;
};
cudaError_t launch_prep_segments(PrepSegment* segs, int n, int d, long long ld16, long long ld8, float pad_norm,
                                 int aug, cudaStream_t st);

// Plain squared (or not) L2 norms, as computeL2Norm.
cudaError_t launch_l2_norms(const float* x, long long n, int d, float* norms, int squared, cudaStream_t st);

// Checks of the merge pass that list a query for a search again (MergeItem::checks).
constexpr int kCheckEstimate = 1;  // the fused pass started from estimated bounds: verify them
constexpr int kCheckCoarse = 2;    // coarse (BF16/FP8) distances: verify the candidate margin

struct MergeLaunch {
  int nq, nb, d, k, kprime, pool_cap;
  const int* run_if = nullptr;   // non-null: the launch does nothing unless *run_if != 0
  int checks = 0;                // kCheck* bits; any bit needs fail_count / fail_list
  int* coarse_count = nullptr;   // kCheckCoarse: queries listed by that check (may be null)
  FusedPlan plan;
  const uint64_t* pools;
  const int* pool_counts;
  const uint32_t* q_bound;       // final bounds of the fused pass (may be null)
  int* fail_count = nullptr;     // see MergeItem
  int* fail_list = nullptr;
  const float* queries;   // [nq x d] fp32, row stride d
  const float* db;        // [nb x d] fp32, row stride ld_db
  long long ld_db;
  const __nv_bfloat16* db16 = nullptr;  // see MergeItem
  long long ld16 = 0;
  int* out_idx;
  float* out_dist;
  uint32_t* status;
};
cudaError_t launch_merge_rerank(const MergeLaunch& m, cudaStream_t st);

// Batched merge: one CTA per query of every item; items share d.  An item is
// a run of `nq` consecutive pool rows [row0, row0 + nq) of one fused item, so
// several query batches that were concatenated into one fused item each keep
// their own query and output pointers and their own k.
constexpr int kMergeMaxItems = 128;
struct MergeItem {
  int nq, k, kprime, pool_cap, num_tiles, units_per_block;
  int pair;                // the fused launch ran CTA pairs (query groups of 256 rows)
  int row0;                // first pool row of this item within its fused item
  int split_tiles;         // the fused item's resolved split length L
  long long work_begin;    // the fused item's offset in its launch's flattened work space
  long long work_per_cta;  // W of that launch
  long long q_begin;       // first CTA of this item (filled by launch_merge_batch)
  const uint64_t* pools;   // the fused item's pools and counts
  const int* pool_counts;
  const uint32_t* q_bound;       // the fused item's final bounds by pool row (may be null)
  // kCheck* bits.  kCheckEstimate: the fused pass started from estimated
  // bounds, and a query with fewer than k' candidates under its final bound
  // may miss rows.  kCheckCoarse: the candidates were chosen by coarse
  // (BF16/FP8) distances, and a query whose candidate margin does not cover
  // the coarse error seen among its candidates may miss rows.  Either way the
  // query's index within the item is appended to fail_list (count in
  // *fail_count) for a search again.
  int checks;
  long long nb_total;      // database rows (kCheckCoarse: nothing to check when k' covers them all)
  int* fail_count;
  int* fail_list;
  int* coarse_count;       // kCheckCoarse: counts the queries that check listed (may be null)
  const float* queries;    // [nq x d] fp32, row stride d
  const float* db;         // database rows fp32, row stride ld_db
  long long ld_db;
  const __nv_bfloat16* db16;  // non-null: every row is exactly BF16; rerank reads these rows (stride ld16)
  long long ld16;
  int* out_idx;            // [nq x k]
  float* out_dist;
};
cudaError_t launch_merge_batch(MergeItem* items, int n, int d, uint32_t* status, cudaStream_t st,
                               const int* run_if = nullptr);
cudaError_t prepare_merge_kernel();

// Fill [n] ints / floats (N == 0 results, padding).
cudaError_t launch_fill_results(int* idx, float* dist, long long n, cudaStream_t st);
// p[i] = v for i < n, only when *cond != 0 (decided on the device).
cudaError_t launch_fill_u32_if(uint32_t* p, long long n, uint32_t v, const int* cond, cudaStream_t st);
// *acc += *cnt on the stream (one thread)
cudaError_t launch_add_count(unsigned long long* acc, const int* cnt, cudaStream_t st);
// out[q] = order bits of the j-th smallest (1-based) of minima[q * count ..
// q * count + count) for q < nq (all ones when count < j).
cudaError_t launch_estimate_select(const float* minima, int count, int nq, int j, uint32_t* out, cudaStream_t st);
// dst[i] = src[rows[i]] for i < n (rows of d floats).
cudaError_t launch_gather_rows(const float* src, int d, const int* rows, int n, float* dst, cudaStream_t st);
// out[rows[i]] = in[i] for i < n (result rows of k indices and distances).
cudaError_t launch_scatter_results(const int* in_idx, const float* in_dist, const int* rows, int n, int k,
                                   int* out_idx, float* out_dist, cudaStream_t st);

}  // namespace curplsh_b200

// ---------------------------------------------------------------- index internals
// Read-only view of an index's prepared database, for library code outside
// capi.cpp (the allocation-free search).  Implemented in capi.cpp.
struct curplsh_index;
namespace curplsh_b200 {
struct IndexView {
  int device, dim, precision, rerank_factor, num_sms;
  long long n, n_pad, ld16, ld8;
  const float* x32;
  const float* xn;
  const __nv_bfloat16* xh;
  const __nv_bfloat16* xl;
  const uint8_t* x8;
  const float* xs;
  float xs_uniform;      // > 0: every row of the FP8 copy has this scale
  long long generation;  // changes whenever add()/reset() replace the prepared database
  bool bf16_exact;       // every stored value is exactly a BF16 value (xl is all zero)
  cudaStream_t stream;   // the index's default stream
  cudaEvent_t fp8_ready; // recorded after the FP8 copy (x8, xs) was written; wait on it before reading them
};
// Locks the index (same lock as search/add) and fills `out`; unlock with index_unlock.
int index_lock_view(curplsh_index* index, IndexView* out);
void index_unlock(curplsh_index* index);
// With the lock held: builds the FP8 copy if `form` needs it and it is missing
// (synchronous), updating `v`.
int index_prepare_form(curplsh_index* index, int form, IndexView* v);
// Candidate count k' and pool capacity used by every search of this library.
int search_kprime(int form, int k, int rerank_factor, long long n);
int search_pool_capacity(int kprime, int headroom = kTuneDefaultHeadroom);
// Records a message for curplsh_last_error() and returns `code`.
int record_error(int code, const char* msg);
}  // namespace curplsh_b200
