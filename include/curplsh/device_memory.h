// device_memory.h -- the reference's temporary-memory interface
// (include/device_memory.h:10-89: DeviceMemory, DeviceMemoryReservation),
// which it declares but never implements, with one implementation:
// StreamOrderedDeviceMemory, backed by a CUDA stream-ordered memory pool
// (cudaMallocFromPoolAsync / cudaFreeAsync).  A reservation is usable on its
// stream as soon as getMemory returns, and its memory is reused by later
// reservations in stream order without device-wide synchronisation; the pool
// keeps freed memory cached up to `release_threshold` bytes.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <sstream>
#include <string>
#include <utility>

#include "error.h"

namespace curplsh {

class DeviceMemoryReservation;

class DeviceMemory {
 public:
  virtual ~DeviceMemory() = default;
  /// Returns the device we are managing memory for
  virtual int getDevice() const = 0;
  /// Obtains a temporary allocation for our device, ordered on `stream`
  virtual DeviceMemoryReservation getMemory(cudaStream_t stream, size_t size) = 0;
  /// Returns the size available without a new device allocation
  virtual size_t getSizeAvailable() const = 0;
  /// Returns a string describing the manager's state
  virtual std::string toString() const = 0;
  /// Returns the high-water mark of device memory reserved
  virtual size_t getHighWaterCudaMalloc() const = 0;

 protected:
  friend class DeviceMemoryReservation;
  virtual void returnAllocation(DeviceMemoryReservation& m) = 0;
};

class DeviceMemoryReservation {
 public:
  DeviceMemoryReservation() = default;
  DeviceMemoryReservation(DeviceMemory* state, int device, void* data, size_t size, cudaStream_t stream)
      : state_(state), device_(device), data_(data), size_(size), stream_(stream) {}
  DeviceMemoryReservation(DeviceMemoryReservation&& other) noexcept { *this = std::move(other); }
  DeviceMemoryReservation& operator=(DeviceMemoryReservation&& other) noexcept {
    if (this != &other) {
      release();
      state_ = other.state_;
      device_ = other.device_;
      data_ = other.data_;
      size_ = other.size_;
      stream_ = other.stream_;
      other.data_ = nullptr;
    }
    return *this;
  }
  DeviceMemoryReservation(const DeviceMemoryReservation&) = delete;
  DeviceMemoryReservation& operator=(const DeviceMemoryReservation&) = delete;
  ~DeviceMemoryReservation() { release(); }

  int device() const { return device_; }
  void* get() const { return data_; }
  size_t size() const { return size_; }
  cudaStream_t stream() const { return stream_; }

 private:
  void release() {
    if (data_ && state_) state_->returnAllocation(*this);
    data_ = nullptr;
  }
  DeviceMemory* state_ = nullptr;
  int device_ = 0;
  void* data_ = nullptr;
  size_t size_ = 0;
  cudaStream_t stream_ = nullptr;
};

// DeviceMemory over a dedicated CUDA memory pool of one device.
class StreamOrderedDeviceMemory : public DeviceMemory {
 public:
  explicit StreamOrderedDeviceMemory(int device, size_t release_threshold = SIZE_MAX) : device_(device) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    check(cudaMemPoolCreate(&pool_, &props));
    uint64_t thr = release_threshold;
    check(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &thr));
  }
  ~StreamOrderedDeviceMemory() override {
    if (pool_) cudaMemPoolDestroy(pool_);
  }
  StreamOrderedDeviceMemory(const StreamOrderedDeviceMemory&) = delete;
  StreamOrderedDeviceMemory& operator=(const StreamOrderedDeviceMemory&) = delete;

  int getDevice() const override { return device_; }

  DeviceMemoryReservation getMemory(cudaStream_t stream, size_t size) override {
    void* p = nullptr;
    if (size) check(cudaMallocFromPoolAsync(&p, size, pool_, stream));
    return DeviceMemoryReservation(this, device_, p, size, stream);
  }

  size_t getSizeAvailable() const override {
    const uint64_t reserved = attr(cudaMemPoolAttrReservedMemCurrent), used = attr(cudaMemPoolAttrUsedMemCurrent);
    return reserved > used ? (size_t)(reserved - used) : 0;
  }

  std::string toString() const override {
    std::ostringstream s;
    s << "StreamOrderedDeviceMemory(device " << device_ << "): reserved " << attr(cudaMemPoolAttrReservedMemCurrent)
      << " B, used " << attr(cudaMemPoolAttrUsedMemCurrent) << " B, high water "
      << attr(cudaMemPoolAttrReservedMemHigh) << " B";
    return s.str();
  }

  size_t getHighWaterCudaMalloc() const override { return (size_t)attr(cudaMemPoolAttrReservedMemHigh); }

 protected:
  void returnAllocation(DeviceMemoryReservation& m) override {
    if (m.get()) cudaFreeAsync(m.get(), m.stream());
  }

 private:
  static void check(cudaError_t e) {
    if (e != cudaSuccess) throw Error(e == cudaErrorMemoryAllocation ? CURPLSH_ERR_OOM : CURPLSH_ERR_CUDA,
                                      cudaGetErrorString(e));
  }
  uint64_t attr(cudaMemPoolAttr a) const {
    uint64_t v = 0;
    cudaMemPoolGetAttribute(pool_, a, &v);
    return v;
  }
  int device_;
  cudaMemPool_t pool_ = nullptr;
};

}  // namespace curplsh
