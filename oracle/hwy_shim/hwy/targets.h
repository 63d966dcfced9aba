// Highway-API shim, target queries (TEST INFRASTRUCTURE ONLY): the one
// static target is reported as supported on every host; the operations of
// highway.h are plain C++ and run anywhere.
#ifndef HWY_SHIM_TARGETS_H_
#define HWY_SHIM_TARGETS_H_

#include <stdint.h>

#include "hwy/base.h"

namespace hwy {

inline int64_t SupportedTargets() { return HWY_AVX3; }
inline void SetSupportedTargetsForTest(int64_t) {}
inline const char* TargetName(int64_t target) {
  return target == HWY_AVX3 ? "AVX3" : "unknown";
}

}  // namespace hwy

#endif  // HWY_SHIM_TARGETS_H_
