// tensor.h -- Tensor<T, Dim, IndexT>: non-owning row-major view with sizes and
// strides (cuRPLSH include/tensor.h:17-114), host-side subset: construction
// from (data, sizes) or (data, sizes, strides), getters, narrow(), view checks.
#pragma once
#include <cstddef>
#include <initializer_list>
#include <stdexcept>

namespace curplsh {

template <typename T, int Dim, typename IndexT = int>
class Tensor {
 public:
  typedef T DataType;
  typedef IndexT IndexType;

  Tensor() : data_(nullptr) {
    for (int i = 0; i < Dim; ++i) {
      sizes_[i] = 0;
      strides_[i] = 1;
    }
  }
  Tensor(T* data, const IndexT sizes[Dim]) : data_(data) {
    for (int i = 0; i < Dim; ++i) sizes_[i] = sizes[i];
    contiguous_strides_();
  }
  Tensor(T* data, std::initializer_list<IndexT> sizes) : data_(data) {
    if ((int)sizes.size() != Dim) throw std::invalid_argument("Tensor: wrong number of sizes");
    int i = 0;
    for (auto s : sizes) sizes_[i++] = s;
    contiguous_strides_();
  }
  Tensor(T* data, const IndexT sizes[Dim], const IndexT strides[Dim]) : data_(data) {
    for (int i = 0; i < Dim; ++i) {
      sizes_[i] = sizes[i];
      strides_[i] = strides[i];
    }
  }

  T* data() const { return data_; }
  T* end() const { return data_ + getNumElements(); }
  IndexT getSize(int i) const { return sizes_[i]; }
  IndexT getStride(int i) const { return strides_[i]; }
  const IndexT* sizes() const { return sizes_; }
  const IndexT* strides() const { return strides_; }
  size_t getNumElements() const {
    size_t n = 1;
    for (int i = 0; i < Dim; ++i) n *= (size_t)sizes_[i];
    return n;
  }
  size_t getDataMemSize() const { return getNumElements() * sizeof(T); }
  bool isContiguous() const {
    IndexT s = 1;
    for (int i = Dim - 1; i >= 0; --i) {
      if (sizes_[i] != 1 && strides_[i] != s) return false;
      s *= sizes_[i];
    }
    return true;
  }
  template <typename Other>
  bool isSameSizes(const Other& o) const {
    for (int i = 0; i < Dim; ++i)
      if (sizes_[i] != o.getSize(i)) return false;
    return true;
  }
  /// Sub-tensor [start, start+num) along `dim` (include/tensor.h narrow()).
  Tensor<T, Dim, IndexT> narrow(int dim, IndexT start, IndexT num) const {
    IndexT sz[Dim], st[Dim];
    for (int i = 0; i < Dim; ++i) {
      sz[i] = sizes_[i];
      st[i] = strides_[i];
    }
    sz[dim] = num;
    return Tensor<T, Dim, IndexT>(data_ + (size_t)start * strides_[dim], sz, st);
  }

 protected:
  void contiguous_strides_() {
    strides_[Dim - 1] = 1;
    for (int i = Dim - 2; i >= 0; --i) strides_[i] = strides_[i + 1] * sizes_[i + 1];
  }
  T* data_;
  IndexT sizes_[Dim];
  IndexT strides_[Dim];
};

}  // namespace curplsh
