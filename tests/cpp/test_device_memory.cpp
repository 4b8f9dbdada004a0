// DeviceMemory / DeviceMemoryReservation over StreamOrderedDeviceMemory.
// Prints "cpp device memory ok" on success.
#include <cstdio>
#include <vector>

#include "curplsh/device_memory.h"

int main() {
  curplsh::StreamOrderedDeviceMemory mem(0);
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  {
    curplsh::DeviceMemoryReservation a = mem.getMemory(st, 1 << 20);
    curplsh::DeviceMemoryReservation b = mem.getMemory(st, 3 << 20);
    if (!a.get() || !b.get() || a.size() != (1u << 20) || a.stream() != st || a.device() != 0) return 1;
    cudaMemsetAsync(a.get(), 7, a.size(), st);
    std::vector<unsigned char> h(16);
    cudaMemcpyAsync(h.data(), a.get(), h.size(), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    if (h[0] != 7 || h[15] != 7) return 2;
    curplsh::DeviceMemoryReservation c = std::move(b);  // moved-from b must not free twice
    if (b.get() != nullptr || !c.get()) return 3;
    if (mem.getHighWaterCudaMalloc() < (4u << 20)) return 4;
  }
  cudaStreamSynchronize(st);
  // both returned: their memory is available without a new device allocation
  if (mem.getSizeAvailable() < (4u << 20)) return 5;
  {
    curplsh::DeviceMemoryReservation d = mem.getMemory(st, 2 << 20);
    if (!d.get()) return 6;
  }
  cudaStreamSynchronize(st);
  std::printf("%s\n", mem.toString().c_str());
  cudaStreamDestroy(st);
  std::printf("cpp device memory ok\n");
  return 0;
}
