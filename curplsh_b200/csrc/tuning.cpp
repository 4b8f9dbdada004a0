// tuning.cpp -- per-shape launch parameters of the fused pass.
//
// No counterpart in cuRPLSH (its tile sizes are fixed by chooseTileSize,
// src/internal/search.cu:12-77).  Two knobs of the persistent kernel are
// free -- neither changes any result, only the speed:
//   * split (quarters of the CTA range W the search gets alone): the longest
//     run of database tiles one candidate pool covers.  Shorter runs mean more
//     pools per query (more merge work) and fewer in-pool selections; longer
//     runs the reverse.  The tile itself stays 128 x 256 (the largest single-CTA
//     MMA shape, double-buffered in 512 TMEM columns).
//   * pool headroom (the k-select width): pool capacity is
//     k' + 128 + max(k', headroom) keys; a pool is reduced back to ~k' keys
//     only when it is full, so a larger headroom means rarer but longer
//     selections.
// The table is filled by the project's autotuner (curplsh_b200/autotune.py)
// through the C ABI and read at plan time by every search path except the
// allocation-free one (which keeps the defaults).
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>

#include "../../include/curplsh_b200.h"
#include "fused_knn.h"

namespace curplsh_b200 {
namespace {

std::mutex g_mu;
std::map<std::tuple<int, int, int, int>, TuneParams> g_table;

int log2_floor(long long v) {
  int r = 0;
  while (v > 1) {
    v >>= 1;
    ++r;
  }
  return r;
}
int log2_ceil(long long v) {
  int r = 0;
  while ((1LL << r) < v) ++r;
  return r;
}
std::tuple<int, int, int, int> key_of(int form, int d, int k, long long nq) {
  return std::make_tuple(form, d, log2_ceil(k < 1 ? 1 : k), log2_floor(nq < 1 ? 1 : nq));
}

}  // namespace

TuneParams tune_lookup(int form, int d, int k, long long nq) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_table.find(key_of(form, d, k, nq));
  return it == g_table.end() ? TuneParams{} : it->second;
}

}  // namespace curplsh_b200

using namespace curplsh_b200;

extern "C" {

int curplsh_tuning_set(int precision, int dim, int k, int64_t num_queries, int split_q4, int pool_headroom) {
  if (precision < 0 || precision > 2 || dim < 1 || k < 1 || k > 1024 || num_queries < 1)
    return record_error(CURPLSH_ERR_INVALID_ARG, "curplsh_tuning_set: bad shape");
  if (split_q4 < 1 || split_q4 > 64 || pool_headroom < kTuneMinHeadroom || pool_headroom > kTuneMaxHeadroom)
    return record_error(CURPLSH_ERR_INVALID_ARG,
                        "curplsh_tuning_set: split_q4 must be in [1, 64], pool_headroom in [128, 8192]");
  std::lock_guard<std::mutex> lk(g_mu);
  g_table[key_of(precision, dim, k, num_queries)] = TuneParams{split_q4, pool_headroom, true};
  return CURPLSH_OK;
}

int curplsh_tuning_get(int precision, int dim, int k, int64_t num_queries, int* split_q4, int* pool_headroom) {
  if (!split_q4 || !pool_headroom) return record_error(CURPLSH_ERR_INVALID_ARG, "null argument");
  const TuneParams t = tune_lookup(precision, dim, k, num_queries);
  *split_q4 = t.split_q4;
  *pool_headroom = t.headroom;
  return CURPLSH_OK;
}

int curplsh_tuning_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
  return CURPLSH_OK;
}

}  // extern "C"
