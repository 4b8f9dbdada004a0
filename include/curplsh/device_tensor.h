// device_tensor.h -- DeviceTensor (cuRPLSH include/device_tensor.h:16-135):
// owning (cudaMalloc / cudaMallocManaged) or referencing device tensor.  The
// constructor from a host pointer + stream copies to the device, as the
// reference's ctorAllocCopy_ does (device_tensor.h:173-185).
#pragma once
#include <cuda_runtime.h>

#include <utility>

#include "error.h"
#include "memory_space.h"
#include "tensor.h"

namespace curplsh {

template <typename T, int Dim, typename IndexT = int>
class DeviceTensor : public Tensor<T, Dim, IndexT> {
 public:
  DeviceTensor() : Tensor<T, Dim, IndexT>(), owner_(false), space_(MemorySpace::Device) {}
  /// Allocate (include/device_tensor.h:74-80).
  explicit DeviceTensor(std::initializer_list<IndexT> sizes, MemorySpace space = MemorySpace::Device)
      : Tensor<T, Dim, IndexT>(nullptr, sizes), owner_(true), space_(space) {
    allocate_();
  }
  /// Reference existing device memory (include/device_tensor.h:82-94).
  DeviceTensor(T* data, std::initializer_list<IndexT> sizes, MemorySpace space)
      : Tensor<T, Dim, IndexT>(data, sizes), owner_(false), space_(space) {}
  /// Copy from host memory on `stream` (include/device_tensor.h:117-123).
  DeviceTensor(const T* host, std::initializer_list<IndexT> sizes, cudaStream_t stream)
      : Tensor<T, Dim, IndexT>(nullptr, sizes), owner_(true), space_(MemorySpace::Device) {
    allocate_();
    if (this->getDataMemSize()) {
      cudaError_t e = cudaMemcpyAsync(this->data_, host, this->getDataMemSize(), cudaMemcpyDefault, stream);
      if (e != cudaSuccess) throw Error(CURPLSH_ERR_CUDA, cudaGetErrorString(e));
    }
  }
  DeviceTensor(DeviceTensor&& o) noexcept : Tensor<T, Dim, IndexT>(o), owner_(o.owner_), space_(o.space_) {
    o.owner_ = false;
    o.data_ = nullptr;
  }
  DeviceTensor& operator=(DeviceTensor&& o) noexcept {
    if (this != &o) {
      release_();
      Tensor<T, Dim, IndexT>::operator=(o);
      owner_ = o.owner_;
      space_ = o.space_;
      o.owner_ = false;
      o.data_ = nullptr;
    }
    return *this;
  }
  DeviceTensor(const DeviceTensor&) = delete;
  DeviceTensor& operator=(const DeviceTensor&) = delete;
  ~DeviceTensor() { release_(); }

  DeviceTensor& zero(cudaStream_t stream = 0) {
    if (this->data_) cudaMemsetAsync(this->data_, 0, this->getDataMemSize(), stream);
    return *this;
  }
  /// Copy to host (include/device_tensor.h:125-129); synchronous.
  void toHost(T* host, cudaStream_t stream = 0) const {
    cudaError_t e = cudaMemcpyAsync(host, this->data_, this->getDataMemSize(), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) throw Error(CURPLSH_ERR_CUDA, cudaGetErrorString(e));
  }
  MemorySpace space() const { return space_; }

 private:
  void allocate_() {
    const size_t bytes = this->getDataMemSize();
    if (!bytes) return;
    cudaError_t e = space_ == MemorySpace::Unified ? cudaMallocManaged((void**)&this->data_, bytes)
                                                   : cudaMalloc((void**)&this->data_, bytes);
    if (e != cudaSuccess) throw Error(CURPLSH_ERR_OOM, cudaGetErrorString(e));
  }
  void release_() {
    if (owner_ && this->data_) cudaFree(this->data_);
    this->data_ = nullptr;
    owner_ = false;
  }
  bool owner_;
  MemorySpace space_;
};

}  // namespace curplsh
