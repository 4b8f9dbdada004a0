// index.h -- IndexConfig and the abstract Index (cuRPLSH include/index.h:8-82).
#pragma once
#include "device_resources.h"
#include "memory_space.h"

namespace curplsh {

struct IndexConfig {
  IndexConfig() : device(0), memorySpace(MemorySpace::Device) {}
  /// GPU device on which the index is resident
  int device;
  /// memory space of the primary storage
  MemorySpace memorySpace;
};

class Index {
 public:
  Index(DeviceResources* resources, int dimension, IndexConfig config)
      : dimension_(dimension), numData_(0), verbose_(false), isTrained_(true), resources_(resources),
        memorySpace_(config.memorySpace), device_(config.device) {}
  virtual ~Index() = default;

  /// Train on representative vectors (include/index.h:24-29).
  virtual void train(int num, const float* data) = 0;
  /// Add num vectors with sequential labels (include/index.h:31-38).
  virtual void add(int num, const float* data) = 0;
  /// k nearest neighbours of each query; missing results are padded with -1
  /// (include/index.h:40-53).
  virtual void search(int num, const float* queries, int k, int* indices, float* distances) = 0;
  /// Remove all data (include/index.h:55-56).
  virtual void reset() = 0;

  int getDimension() const { return dimension_; }
  int getNumData() const { return numData_; }
  DeviceResources* getResources() { return resources_; }
  int getDevice() const { return device_; }

 protected:
  const int dimension_;
  int numData_;
  bool verbose_;
  bool isTrained_;
  DeviceResources* resources_;
  const MemorySpace memorySpace_;
  const int device_;
};

}  // namespace curplsh
