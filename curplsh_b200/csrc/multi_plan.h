// multi_plan.h -- planning and launching of several searches at once, shared
// by the batch graph (batch.cpp) and the serving loop (server.cpp).
// Internal to libcurplsh_b200.so.
//
// A plan covers a list of requests (index, queries, k, outputs):
//   * every request resolves its precision form, k' and pool capacity exactly
//     as a single search would, so its results are those of the request
//     searched alone;
//   * requests against the same index with the same (form, k') are
//     concatenated into one fused item whose queries share 128-row blocks;
//   * fused items are grouped by (form, d): per group one segmented prep
//     launch, persistent fused launches of up to kFusedMaxItems items, and one
//     merge + rerank launch per power-of-two class of k';
//   * a fused item large enough for the sampled bound estimate starts its
//     pools from it, exactly as a single search does; the merge verifies the
//     estimate on the device, and when any query of a fused launch failed,
//     a fallback chain enqueued behind it (bounds reset, the fused launch and
//     its merges again, without the estimate) runs -- every kernel of it reads
//     the launch's failure count first and does nothing when it is zero, so
//     the plan needs no host round trip and can be captured in a graph.
// build() sizes everything without allocating; bind() places the working
// memory in a caller-provided range; enqueue() issues the launches.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/curplsh_b200.h"
#include "fused_knn.h"

namespace curplsh_b200 {

class MultiPlan {
 public:
  // `uniq` are the distinct indexes (sorted by address), `views` their locked
  // views (updated when an FP8 copy has to be built).  Requests with num == 0
  // are skipped.
  int build(const curplsh_batch_item* items, int n, const std::vector<curplsh_index*>& uniq,
            std::vector<IndexView>& views, int precision, int rerank_factor, int num_sms);
  size_t bytes() const { return bytes_; }
  void bind(void* base);
  uint32_t* status() const { return status_; }
  // Replaces the query and output pointers of request i (same shapes).
  void set_item_pointers(int i, const float* queries, int32_t* indices, float* distances) {
    items_[i].queries = queries;
    items_[i].indices = indices;
    items_[i].distances = distances;
  }
  int num_groups() const { return (int)groups_.size(); }
  // Issues the memsets and launches on `main`.  With `branches` (one stream
  // and one join event per group, plus the `fork` event) the groups run as
  // parallel branches that rejoin `main`; otherwise they run in order on it.
  int enqueue(cudaStream_t main, const std::vector<cudaStream_t>* branches, const std::vector<cudaEvent_t>* joins,
              cudaEvent_t fork, int* kernels) const;

 private:
  struct FItem {
    int slot = 0;
    int form = 0, kp = 0, P = 0, d = 0, k = 1;
    TuneParams tune;
    int nq = 0;
    long long nq_pad = 0;
    std::vector<int> members;
    std::vector<int> row0;
    FusedItemSpec spec{};
    FusedItemPlan plan{};
    long long W = 1;
    EstimatePlan est;   // est.on: the full pass starts from the sampled bound estimate
    int launch = -1;    // index of its fused launch within its group
    size_t o_qh = 0, o_ql = 0, o_q8 = 0, o_qn = 0, o_qs = 0, o_counts = 0, o_pools = 0, o_bounds = 0;
    size_t o_minima = 0;
  };
  struct FLaunch {
    std::vector<int> fitems;
    FusedBatchPlan bp;
    bool est_any = false;  // some item uses the estimate: verification and the fallback chain
    size_t o_fail = 0;     // [2 + queries]: failure count, (unused), failed query indices
  };
  struct Group {
    int form = 0, d = 0;
    long long ld16 = 0, ld8 = 0;
    std::vector<int> fitems;
    std::vector<FLaunch> launches;
  };
  std::vector<curplsh_batch_item> items_;
  std::vector<IndexView> views_;
  std::vector<FItem> fitems_;
  std::vector<Group> groups_;
  size_t bytes_ = 0, o_status_ = 0, o_bounds_ = 0, bounds_words_ = 0, o_fails_ = 0, fails_bytes_ = 0;
  char* base_ = nullptr;
  uint32_t* status_ = nullptr;
};

}  // namespace curplsh_b200
