// index_bf.h -- IndexBFConfig and IndexBF (cuRPLSH include/index_bf.h:8-46,
// src/index_bf.cpp) over the C ABI, plus tensor overloads of add/search.
#pragma once
#include <utility>

#include "device_tensor.h"
#include "host_tensor.h"
#include "index.h"

namespace curplsh {

struct IndexBFConfig : public IndexConfig {
  IndexBFConfig()
      : storeTransposed(false), computeExactDistances(false), precision(CURPLSH_PRECISION_FP32_EXACT),
        rerankFactor(0), borrowDeviceData(false) {}
  /// accepted; the engine always keeps its own K-major tiled copy
  bool storeTransposed;
  /// accepted; search always returns exact squared distances, like
  /// IndexBF::search (src/index_bf.cpp:68-69)
  bool computeExactDistances;
  /// coarse form: CURPLSH_PRECISION_FP32_EXACT / _BF16_RERANK / _FP8_RERANK
  int precision;
  /// k' = rerankFactor * k candidates for the BF16 / FP8 forms (0: the form's default -- BF16 2k
  /// when the coarse-margin check is on, else 4k; FP8 4k and at least 480)
  int rerankFactor;
  /// keep a reference to device rows passed to add() instead of copying them
  bool borrowDeviceData;
};

class IndexBF : public Index {
 public:
  IndexBF(DeviceResources* resources, int dim, IndexBFConfig config = IndexBFConfig())
      : Index(resources, dim, config), config_(config) {
    curplsh_bf_config c;
    curplsh_bf_config_init(&c);
    c.device = config.device;
    c.memory_space = static_cast<int32_t>(config.memorySpace);
    c.store_transposed = config.storeTransposed;
    c.compute_exact_distances = config.computeExactDistances;
    c.precision = config.precision;
    c.rerank_factor = config.rerankFactor;
    c.borrow_device_data = config.borrowDeviceData;
    check(curplsh_index_bf_create(resources->handle(), dim, &c, &h_));
  }
  ~IndexBF() override { curplsh_index_destroy(h_); }
  IndexBF(const IndexBF&) = delete;
  IndexBF& operator=(const IndexBF&) = delete;

  void train(int num, const float* data) override { check(curplsh_index_train(h_, num, data)); }

  void add(int num, const float* data) override {
    check(curplsh_index_add(h_, num, data));
    sync_count_();
  }
  void add(const DeviceTensor<float, 2>& data) {
    check(curplsh_index_add(h_, data.getSize(0), data.data()));
    sync_count_();
  }
  void add(const HostTensor<float, 2>& data) {
    check(curplsh_index_add(h_, data.getSize(0), data.data()));
    sync_count_();
  }

  void search(int num, const float* queries, int k, int* indices, float* distances) override {
    check(curplsh_index_search(h_, num, queries, k, indices, distances));
  }
  /// Search a [num x dim] query tensor; returns (distances, indices) on the device.
  std::pair<DeviceTensor<float, 2>, DeviceTensor<int, 2>> search(const Tensor<float, 2>& queries, int k) {
    DeviceTensor<float, 2> dist({queries.getSize(0), k});
    DeviceTensor<int, 2> idx({queries.getSize(0), k});
    check(curplsh_index_search(h_, queries.getSize(0), queries.data(), k, idx.data(), dist.data()));
    return {std::move(dist), std::move(idx)};
  }

  void reset() override {
    check(curplsh_index_reset(h_));
    numData_ = 0;
  }

  curplsh_index* handle() { return h_; }

 protected:
  void sync_count_() {
    int64_t n = 0;
    check(curplsh_index_get_num_data(h_, &n));
    numData_ = static_cast<int>(n);
  }
  const IndexBFConfig config_;
  curplsh_index* h_ = nullptr;
};

}  // namespace curplsh
