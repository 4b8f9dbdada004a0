// server_sched.h -- the serving loop's admission and step-forming rules, free
// of CUDA so they can be tested on the host (tests/cpp/test_server_sched.cpp).
// Internal to libcurplsh_b200.so.
//
// No counterpart in cuRPLSH (its IndexBF::search is one blocking call per
// query matrix, src/index_bf.cpp:46-74).
#pragma once
#include <cstddef>
#include <cstdint>
#include <deque>
#include <functional>
#include <iterator>
#include <map>
#include <vector>

namespace curplsh_b200 {

inline size_t sched_round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

// First-fit allocator over [0, size) with coalescing of free neighbours;
// every block is rounded up to 256-byte granules.  It only does the
// bookkeeping: the memory itself is one device allocation made at creation.
class Arena {
 public:
  void reset(size_t size) {
    free_.clear();
    if (size) free_[0] = size;
    size_ = size;
    in_use_ = 0;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = sched_round_up(bytes ? bytes : 1, 256);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes, start = it->first + bytes;
        free_.erase(it);
        if (rest) free_[start] = rest;
        in_use_ += bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = sched_round_up(bytes ? bytes : 1, 256);
    in_use_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t in_use() const { return in_use_; }
  size_t size() const { return size_; }
  size_t free_blocks() const { return free_.size(); }
  size_t largest_free() const {
    size_t m = 0;
    for (const auto& kv : free_) m = kv.second > m ? kv.second : m;
    return m;
  }

 private:
  std::map<size_t, size_t> free_;
  size_t size_ = 0, in_use_ = 0;
};

// The requests of the next step, first come first served: the longest prefix
// of `pending` whose query counts sum to at most max_step_queries (always at
// least the head request).  `num_of(ticket)` gives a request's query count.
inline std::vector<int64_t> take_step(const std::deque<int64_t>& pending, int64_t max_step_queries,
                                      const std::function<int64_t(int64_t)>& num_of) {
  std::vector<int64_t> take;
  int64_t q = 0;
  for (int64_t t : pending) {
    const int64_t n = num_of(t);
    if (!take.empty() && q + n > max_step_queries) break;
    take.push_back(t);
    q += n;
  }
  return take;
}

// Admission by device memory: shrinks `take` (halving it, always keeping its
// head, so requests still run in arrival order) until the step's working
// memory, bytes_for(take), fits in the arena; on success *off holds the
// step's block.  Returns the outcome: 1 admitted, 0 the head alone does not
// fit now (wait for running steps to release memory), < 0 bytes_for failed.
inline int admit_step(std::vector<int64_t>& take, Arena& arena, size_t* off, size_t* bytes,
                      const std::function<int(const std::vector<int64_t>&, size_t*)>& bytes_for) {
  while (!take.empty()) {
    size_t b = 0;
    const int rc = bytes_for(take, &b);
    if (rc) return rc < 0 ? rc : -rc;
    if (arena.alloc(b, off)) {
      *bytes = b;
      return 1;
    }
    if (take.size() == 1) return 0;
    take.resize(take.size() / 2);
  }
  return 0;
}

}  // namespace curplsh_b200
