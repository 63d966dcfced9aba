// Highway-API shim, aligned allocation (TEST INFRASTRUCTURE ONLY).
#ifndef HWY_SHIM_ALIGNED_ALLOCATOR_H_
#define HWY_SHIM_ALIGNED_ALLOCATOR_H_

#include <stdlib.h>

#include <memory>
#include <type_traits>

#include "hwy/base.h"

namespace hwy {

struct AlignedFreer {
  void operator()(void* p) const { free(p); }
};

template <typename T>
using AlignedFreeUniquePtr = std::unique_ptr<T, AlignedFreer>;

// n elements of T, 64-byte aligned; the memory is uninitialised.
template <typename T>
AlignedFreeUniquePtr<T[]> AllocateAligned(size_t n) {
  const size_t bytes = RoundUpTo<size_t>(n * sizeof(T) + (n == 0), 64);
  return AlignedFreeUniquePtr<T[]>(static_cast<T*>(aligned_alloc(64, bytes)));
}

}  // namespace hwy

#endif  // HWY_SHIM_ALIGNED_ALLOCATOR_H_
