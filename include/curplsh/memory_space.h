// memory_space.h -- MemorySpace (cuRPLSH include/memory_space.h:12-17).
#pragma once
#include "../curplsh_b200.h"

namespace curplsh {

enum class MemorySpace {
  /// plain device memory (cudaMalloc)
  Device = CURPLSH_MEMORY_DEVICE,
  /// unified memory (cudaMallocManaged)
  Unified = CURPLSH_MEMORY_UNIFIED,
};

}  // namespace curplsh
