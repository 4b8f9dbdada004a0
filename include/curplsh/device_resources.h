// device_resources.h -- DeviceScope and DeviceResources
// (cuRPLSH include/device_resources.h:13-32, :60-263) over the C ABI.
// Streams only: the engine needs no cuBLAS or cuRAND handle, so
// getBlasHandle()/getRandGenerator() return nullptr.
#pragma once
#include <cuda_runtime.h>

#include <initializer_list>
#include <vector>

#include "error.h"

namespace curplsh {

/// RAII: select a device, restore the previous one on destruction.
class DeviceScope {
 public:
  explicit DeviceScope(int device) {
    cudaGetDevice(&prev_);
    if (prev_ != device) {
      cudaSetDevice(device);
    } else {
      prev_ = -1;
    }
  }
  ~DeviceScope() {
    if (prev_ != -1) cudaSetDevice(prev_);
  }

 private:
  int prev_ = -1;
};

inline int getCurrentDevice() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

inline int getNumDevices() {
  int n = 0;
  check(curplsh_get_num_devices(&n));
  return n;
}

class DeviceResources {
 public:
  DeviceResources() { check(curplsh_resources_create(&h_)); }
  explicit DeviceResources(int device) : DeviceResources() { initializeForDevice(device); }
  DeviceResources(std::initializer_list<int> devices) : DeviceResources() {
    for (int d : devices) initializeForDevice(d);
  }
  ~DeviceResources() { curplsh_resources_destroy(h_); }
  DeviceResources(const DeviceResources&) = delete;
  DeviceResources& operator=(const DeviceResources&) = delete;

  void initializeForDevice(int device) { check(curplsh_resources_initialize_for_device(h_, device)); }

  /// Use `stream` as the default stream of `device` (before the device is initialised).
  void setDefaultStream(int device, cudaStream_t stream) {
    check(curplsh_resources_set_default_stream(h_, device, stream));
  }

  void* getBlasHandle(int) { return nullptr; }
  void* getRandGenerator(int) { return nullptr; }

  cudaStream_t getDefaultStream(int device) {
    void* s = nullptr;
    check(curplsh_resources_get_default_stream(h_, device, &s));
    return static_cast<cudaStream_t>(s);
  }
  std::vector<cudaStream_t> getAlternateStreams(int device) {
    void* s[2] = {nullptr, nullptr};
    int n = 2;
    check(curplsh_resources_get_alternate_streams(h_, device, s, &n));
    return {static_cast<cudaStream_t>(s[0]), static_cast<cudaStream_t>(s[1])};
  }
  cudaStream_t getAsyncCopyStream(int device) {
    void* s = nullptr;
    check(curplsh_resources_get_async_copy_stream(h_, device, &s));
    return static_cast<cudaStream_t>(s);
  }
  void syncDefaultStream(int device) { check(curplsh_resources_sync_default_stream(h_, device)); }

  void* getBlasHandleCurrentDevice() { return nullptr; }
  cudaStream_t getDefaultStreamCurrentDevice() { return getDefaultStream(getCurrentDevice()); }
  std::vector<cudaStream_t> getAlternateStreamsCurrentDevice() { return getAlternateStreams(getCurrentDevice()); }
  cudaStream_t getAsyncCopyStreamCurrentDevice() { return getAsyncCopyStream(getCurrentDevice()); }
  void syncDefaultStreamCurrentDevice() { syncDefaultStream(getCurrentDevice()); }

  curplsh_resources* handle() { return h_; }

 private:
  curplsh_resources* h_ = nullptr;
};

}  // namespace curplsh
