// Device helpers that fix the reference's rounding in the LU kernels (shared
// by the single-problem and the batched factorizations).
#pragma once

#include <cfloat>

namespace hb {
namespace {

template <typename T>
__device__ __forceinline__ T Sfmin();
template <>
__device__ __forceinline__ double Sfmin<double>() { return DBL_MIN; }
template <>
__device__ __forceinline__ float Sfmin<float>() { return FLT_MIN; }

// y + alpha*x in the reference's rounding for a column of length len: shorter
// than one SIMD vector of the reference's target, two roundings; otherwise
// one FMA (src/lapack/factor_kernels.cc:79-118).
template <typename T>
__device__ __forceinline__ T Axpy(T y, T alpha, T x, int len, int lanes) {
  if (len < lanes) {
    const T p = alpha * x;
    return y + p;
  }
  return fma(x, alpha, y);
}

// (value, index) candidates: larger value wins, then the smaller index.
// value < 0 marks "no candidate" (no rows, or only NaNs).
template <typename T>
__device__ __forceinline__ bool Better(T v, int i, T bv, int bi) {
  return v > bv || (v == bv && v >= T(0) && i < bi);
}

}  // namespace
}  // namespace hb
