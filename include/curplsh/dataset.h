// dataset.h -- TEXMEX .fvecs/.ivecs files and recall evaluation, the
// reference's include/dataset.h (helper::loadXvecsData :14-45, Dataset
// :50-167, DatasetIrisa :169-192, DatasetSIFT :194-198, DatasetGIST
// :200-204), header-only.
//
// Same file semantics: each row is a 4-byte dimension followed by the row's
// values; the dimension comes from the first row and the row count is
// file size / (dim * sizeof(T) + sizeof(IndexT)).  Differences: errors throw
// curplsh::Error instead of asserting; evaluate() leaves the caller's result
// and ground-truth rows unsorted (the reference sorts them in place); a
// saveXvecsData writer is provided (a TODO in the reference).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "error.h"
#include "memory_space.h"

namespace curplsh {

namespace helper {

template <typename T, typename IndexT>
void loadXvecsData(const char* filename, T*& data, IndexT& num, IndexT& dim, MemorySpace space) {
  FILE* f = std::fopen(filename, "rb");
  if (!f) throw Error(CURPLSH_ERR_INVALID_ARG, std::string("cannot open ") + filename);
  int32_t d = 0;
  if (std::fread(&d, sizeof(d), 1, f) != 1 || d <= 0) {
    std::fclose(f);
    throw Error(CURPLSH_ERR_INVALID_ARG, std::string("bad header in ") + filename);
  }
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  const size_t row_bytes = sizeof(int32_t) + (size_t)d * sizeof(T);
  const size_t n = (size_t)size / row_bytes;
  std::fseek(f, 0, SEEK_SET);
  std::vector<T> host(n * (size_t)d);
  for (size_t i = 0; i < n; ++i) {
    int32_t rd = 0;
    if (std::fread(&rd, sizeof(rd), 1, f) != 1 || rd != d ||
        std::fread(host.data() + i * d, sizeof(T), (size_t)d, f) != (size_t)d) {
      std::fclose(f);
      throw Error(CURPLSH_ERR_INVALID_ARG, std::string("truncated or inconsistent rows in ") + filename);
    }
  }
  std::fclose(f);
  num = (IndexT)n;
  dim = (IndexT)d;
  const size_t bytes = host.size() * sizeof(T);
  cudaError_t e = space == MemorySpace::Unified ? cudaMallocManaged((void**)&data, bytes ? bytes : 1)
                                                 : cudaMalloc((void**)&data, bytes ? bytes : 1);
  if (e != cudaSuccess) throw Error(CURPLSH_ERR_OOM, cudaGetErrorString(e));
  if (bytes) {
    e = cudaMemcpy(data, host.data(), bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) throw Error(CURPLSH_ERR_CUDA, cudaGetErrorString(e));
  }
}

// Writes host rows [num x dim] in the same layout.
template <typename T, typename IndexT>
void saveXvecsData(const char* filename, const T* data, IndexT num, IndexT dim) {
  FILE* f = std::fopen(filename, "wb");
  if (!f) throw Error(CURPLSH_ERR_INVALID_ARG, std::string("cannot create ") + filename);
  const int32_t d = (int32_t)dim;
  for (IndexT i = 0; i < num; ++i) {
    if (std::fwrite(&d, sizeof(d), 1, f) != 1 ||
        std::fwrite(data + (size_t)i * dim, sizeof(T), (size_t)dim, f) != (size_t)dim) {
      std::fclose(f);
      throw Error(CURPLSH_ERR_INVALID_ARG, std::string("write failed: ") + filename);
    }
  }
  std::fclose(f);
}

}  // namespace helper

template <typename T, typename IndexT>
class Dataset {
 public:
  typedef T DataType;
  typedef IndexT IndexType;

  Dataset() : Dataset(0, 0, 0, 0, nullptr, nullptr, nullptr, "", MemorySpace::Device) {}
  Dataset(IndexT dimension, IndexT gtK, IndexT numBase, IndexT numQuery, T* base, T* query, IndexT* gt,
          const char* name, MemorySpace space)
      : dimension_(dimension), gtK_(gtK), numBase_(numBase), numQuery_(numQuery), base_(base), query_(query),
        gt_(gt), name_(name), space_(space), isMemOwner(false) {}
  Dataset(const Dataset&) = delete;
  Dataset& operator=(const Dataset&) = delete;
  virtual ~Dataset() {
    if (isMemOwner) {
      cudaFree(base_);
      cudaFree(query_);
      cudaFree(gt_);
    }
  }

  IndexT getDimension() const { return dimension_; }
  IndexT getGroundTruthK() const { return gtK_; }
  IndexT getNumBase() const { return numBase_; }
  IndexT getNumQuery() const { return numQuery_; }
  const T* getBase() const { return base_; }
  const T* getQuery() const { return query_; }
  const IndexT* getGroundTruth() const { return gt_; }
  std::string getName() const { return name_; }
  MemorySpace getMemorySpace() const { return space_; }

  // Mean over queries of |result ∩ ground truth| / gtK (sorted multisets).
  // `indices` holds gtK results per query, host or device; `diff` (host,
  // optional) gets gtK - |intersection| per query.
  virtual float evaluate(const IndexT* indices, IndexT* diff = nullptr) const {
    const size_t n = (size_t)numQuery_ * gtK_;
    std::vector<IndexT> res(n), gt(n);
    cudaError_t e = cudaMemcpy(res.data(), indices, n * sizeof(IndexT), cudaMemcpyDefault);
    if (e == cudaSuccess) e = cudaMemcpy(gt.data(), gt_, n * sizeof(IndexT), cudaMemcpyDefault);
    if (e != cudaSuccess) throw Error(CURPLSH_ERR_CUDA, cudaGetErrorString(e));
    float recall = 0.f;
    std::vector<IndexT> common((size_t)gtK_);
    for (IndexT i = 0; i < numQuery_; ++i) {
      IndexT* r = res.data() + (size_t)i * gtK_;
      IndexT* g = gt.data() + (size_t)i * gtK_;
      std::sort(r, r + gtK_);
      std::sort(g, g + gtK_);
      const IndexT num = (IndexT)(std::set_intersection(r, r + gtK_, g, g + gtK_, common.begin()) - common.begin());
      recall += num / (float)gtK_;
      if (diff) diff[i] = gtK_ - num;
    }
    return numQuery_ ? recall / numQuery_ : 0.f;
  }

 protected:
  IndexT dimension_ = 0, gtK_ = 0, numBase_ = 0, numQuery_ = 0;
  T* base_ = nullptr;
  T* query_ = nullptr;
  IndexT* gt_ = nullptr;
  std::string name_;
  MemorySpace space_ = MemorySpace::Device;
  bool isMemOwner = false;
};

template <typename IndexT>
class DatasetIrisa : public Dataset<float, IndexT> {
 public:
  DatasetIrisa(const char* name, const char* datadir, MemorySpace space = MemorySpace::Device) {
    this->name_ = name;
    this->space_ = space;
    this->isMemOwner = true;
    std::string dir(datadir);
    if (dir.empty() || dir.back() != '/') dir += '/';
    helper::loadXvecsData<float, IndexT>((dir + name + "_base.fvecs").c_str(), this->base_, this->numBase_,
                                         this->dimension_, space);
    helper::loadXvecsData<float, IndexT>((dir + name + "_query.fvecs").c_str(), this->query_, this->numQuery_,
                                         this->dimension_, space);
    helper::loadXvecsData<IndexT, IndexT>((dir + name + "_groundtruth.ivecs").c_str(), this->gt_,
                                          this->numQuery_, this->gtK_, space);
  }
};

class DatasetSIFT : public DatasetIrisa<int> {
 public:
  explicit DatasetSIFT(const char* basedir, MemorySpace space = MemorySpace::Device)
      : DatasetIrisa<int>("sift", basedir, space) {}
};

class DatasetGIST : public DatasetIrisa<int> {
 public:
  explicit DatasetGIST(const char* basedir, MemorySpace space = MemorySpace::Device)
      : DatasetIrisa<int>("gist", basedir, space) {}
};

}  // namespace curplsh
