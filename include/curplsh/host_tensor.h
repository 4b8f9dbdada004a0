// host_tensor.h -- HostTensor (cuRPLSH include/host_tensor.h:16-92): owning
// (new[]) or referencing host tensor.
#pragma once
#include <cstring>
#include <utility>

#include "tensor.h"

namespace curplsh {

template <typename T, int Dim, typename IndexT = int>
class HostTensor : public Tensor<T, Dim, IndexT> {
 public:
  HostTensor() : Tensor<T, Dim, IndexT>(), owner_(false) {}
  explicit HostTensor(std::initializer_list<IndexT> sizes) : Tensor<T, Dim, IndexT>(nullptr, sizes), owner_(true) {
    this->data_ = new T[this->getNumElements()];
  }
  HostTensor(T* data, std::initializer_list<IndexT> sizes) : Tensor<T, Dim, IndexT>(data, sizes), owner_(false) {}
  HostTensor(T* data, const IndexT sizes[Dim]) : Tensor<T, Dim, IndexT>(data, sizes), owner_(false) {}
  HostTensor(HostTensor&& o) noexcept : Tensor<T, Dim, IndexT>(o), owner_(o.owner_) {
    o.owner_ = false;
    o.data_ = nullptr;
  }
  HostTensor& operator=(HostTensor&& o) noexcept {
    if (this != &o) {
      release_();
      Tensor<T, Dim, IndexT>::operator=(o);
      owner_ = o.owner_;
      o.owner_ = false;
      o.data_ = nullptr;
    }
    return *this;
  }
  HostTensor(const HostTensor&) = delete;
  HostTensor& operator=(const HostTensor&) = delete;
  ~HostTensor() { release_(); }

  HostTensor& zero() {
    if (this->data_) std::memset(this->data_, 0, this->getDataMemSize());
    return *this;
  }

 private:
  void release_() {
    if (owner_ && this->data_) delete[] this->data_;
    this->data_ = nullptr;
    owner_ = false;
  }
  bool owner_;
};

}  // namespace curplsh
