// Highway-API shim, base macros (TEST INFRASTRUCTURE ONLY).
//
// The reference's hot-path sources are written against Google Highway, which
// is not available here. This directory restates, from Highway's documented
// API, the handful of macros, tags and operations those sources use, for one
// static target: an AVX-512-class target (HWY_AVX3) with 64-byte vectors, so
// that the sources take their AVX-512 code paths (32 vector registers, 8
// doubles or 16 floats a vector). Each operation is the lane-wise IEEE
// operation its name documents; MulAdd is a fused multiply-add per lane.
// Nothing here is Highway's code.
#ifndef HWY_SHIM_BASE_H_
#define HWY_SHIM_BASE_H_

#include <stddef.h>
#include <stdint.h>

#define HWY_RESTRICT __restrict__
#define HWY_INLINE inline __attribute__((always_inline))
#define HWY_NOINLINE __attribute__((noinline))
#define HWY_ATTR
#define HWY_MIN(a, b) ((a) < (b) ? (a) : (b))
#define HWY_MAX(a, b) ((a) > (b) ? (a) : (b))
#define HWY_LIKELY(x) __builtin_expect(!!(x), 1)
#define HWY_UNLIKELY(x) __builtin_expect(!!(x), 0)
#define HWY_ALIGN alignas(64)
#define HWY_PRAGMA(tokens) _Pragma(#tokens)
#define HWY_UNROLL(factor) HWY_PRAGMA(GCC unroll factor)

// Target bits: a better target has a smaller value, as in Highway.
#define HWY_AVX3_SPR (1LL << 4)
#define HWY_AVX3_ZEN4 (1LL << 6)
#define HWY_AVX3 (1LL << 8)
#define HWY_AVX2 (1LL << 9)
#define HWY_SSE4 (1LL << 11)
#define HWY_SCALAR (1LL << 62)
#define HWY_STATIC_TARGET HWY_AVX3
#define HWY_TARGET HWY_AVX3
#define HWY_TARGETS HWY_AVX3
#define HWY_DISABLED_TARGETS 0
#define HWY_ARCH_X86 1
#define HWY_ARCH_ARM 0
#define HWY_HAVE_SCALABLE 0
#define HWY_NAMESPACE N_AVX3

namespace hwy {

template <typename T>
constexpr T RoundUpTo(T what, T align) {
  return (what + align - 1) / align * align;
}

}  // namespace hwy

#endif  // HWY_SHIM_BASE_H_
