// Highway-API shim, vectors and operations (TEST INFRASTRUCTURE ONLY).
//
// One static target (HWY_AVX3: 64-byte vectors). A vector is an array of its
// lanes and every operation is written lane by lane with the IEEE operation
// Highway documents for it, so results do not depend on the host's SIMD
// width: MulAdd(a, b, c) = fma(a, b, c), NegMulAdd(a, b, c) = fma(-a, b, c),
// AddSub(a, b) = a - b in even lanes and a + b in odd lanes, OddEven(o, e)
// takes odd lanes from o and even lanes from e, Reverse2 swaps adjacent
// lanes. ReduceSum adds the two halves of the vector lane-wise, then the
// halves of that, down to one lane (the x86 order: for 8 lanes
// ((v0 + v4) + (v2 + v6)) + ((v1 + v5) + (v3 + v7))). Dispatch is static:
// HWY_DYNAMIC_DISPATCH(f) names N_AVX3::f.
#ifndef HWY_SHIM_HIGHWAY_H_
#define HWY_SHIM_HIGHWAY_H_

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#include <cmath>
#include <type_traits>

#if defined(__AVX2__) && defined(__FMA__)
#include <immintrin.h>
#endif

#include "hwy/base.h"
#include "hwy/targets.h"

#define HWY_ONCE 1
#define HWY_BEFORE_NAMESPACE()
#define HWY_AFTER_NAMESPACE()
#define HWY_EXPORT(FUNC) static_assert(true, #FUNC)
#define HWY_DYNAMIC_DISPATCH(FUNC) N_AVX3::FUNC

namespace hwy {
namespace N_AVX3 {

constexpr size_t kVectorBytes = 64;

template <typename T, size_t N>
struct Simd {
  using T_ = T;
  static constexpr size_t kLanes = N;
};

template <typename T>
using ScalableTag = Simd<T, kVectorBytes / sizeof(T)>;

template <class D>
using TFromD = typename std::remove_const_t<D>::T_;

// A descriptor of the same lane count with lanes of type T.
template <typename T, class D>
using Rebind = Simd<T, std::remove_const_t<D>::kLanes>;

template <class D>
struct VecT {
  TFromD<D> raw[D::kLanes];
};
// Descriptors are often declared const (decltype keeps it): the vector type
// is that of the unqualified descriptor.
template <class D>
using Vec = VecT<std::remove_const_t<D>>;

template <class D>
struct MaskT {
  bool raw[D::kLanes];
};

template <class D>
constexpr size_t MaxLanes(D) {
  return D::kLanes;
}
template <class D>
constexpr size_t Lanes(D) {
  return D::kLanes;
}

#define HWY_SHIM_LANES for (size_t i = 0; i < D::kLanes; ++i)

template <class D>
HWY_INLINE VecT<D> Zero(D) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = TFromD<D>(0);
  return r;
}
template <class D>
HWY_INLINE VecT<D> Set(D, TFromD<D> t) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = t;
  return r;
}
template <class D>
HWY_INLINE VecT<D> LoadU(D, const TFromD<D>* HWY_RESTRICT p) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = p[i];
  return r;
}
template <class D>
HWY_INLINE VecT<D> Load(D d, const TFromD<D>* HWY_RESTRICT p) {
  return LoadU(d, p);
}
// The first `count` lanes from p, the others zero (p is not read there).
template <class D>
HWY_INLINE VecT<D> LoadN(D, const TFromD<D>* HWY_RESTRICT p, size_t count) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = i < count ? p[i] : TFromD<D>(0);
  return r;
}
template <class D>
HWY_INLINE void StoreU(const VecT<D>& v, D, TFromD<D>* HWY_RESTRICT p) {
  HWY_SHIM_LANES p[i] = v.raw[i];
}
template <class D>
HWY_INLINE void Store(const VecT<D>& v, D d, TFromD<D>* HWY_RESTRICT p) {
  StoreU(v, d, p);
}
template <class D>
HWY_INLINE void StoreN(const VecT<D>& v, D, TFromD<D>* HWY_RESTRICT p, size_t count) {
  HWY_SHIM_LANES if (i < count) p[i] = v.raw[i];
}
// p[4 i + k] = v_k[i].
template <class D>
HWY_INLINE void StoreInterleaved4(const VecT<D>& v0, const VecT<D>& v1, const VecT<D>& v2,
                                  const VecT<D>& v3, D, TFromD<D>* HWY_RESTRICT p) {
  HWY_SHIM_LANES {
    p[4 * i + 0] = v0.raw[i];
    p[4 * i + 1] = v1.raw[i];
    p[4 * i + 2] = v2.raw[i];
    p[4 * i + 3] = v3.raw[i];
  }
}

// Lane-wise arithmetic on vectors of descriptor D (deduced from the vector).
#define HWY_SHIM_BINARY(NAME, EXPR)                                 \
  template <class D>                                                \
  HWY_INLINE VecT<D> NAME(const VecT<D>& a, const VecT<D>& b) {        \
    VecT<D> r;                                                       \
    HWY_SHIM_LANES r.raw[i] = (EXPR);                               \
    return r;                                                       \
  }
HWY_SHIM_BINARY(Add, a.raw[i] + b.raw[i])
HWY_SHIM_BINARY(Sub, a.raw[i] - b.raw[i])
HWY_SHIM_BINARY(Mul, a.raw[i] * b.raw[i])
HWY_SHIM_BINARY(Div, a.raw[i] / b.raw[i])
HWY_SHIM_BINARY(Min, a.raw[i] < b.raw[i] ? a.raw[i] : b.raw[i])
HWY_SHIM_BINARY(Max, a.raw[i] > b.raw[i] ? a.raw[i] : b.raw[i])
// a - b in even lanes, a + b in odd lanes.
HWY_SHIM_BINARY(AddSub, (i & 1) ? a.raw[i] + b.raw[i] : a.raw[i] - b.raw[i])
// Odd lanes from a, even lanes from b.
HWY_SHIM_BINARY(OddEven, (i & 1) ? a.raw[i] : b.raw[i])
#undef HWY_SHIM_BINARY

template <class D>
HWY_INLINE VecT<D> MulAdd(const VecT<D>& mul, const VecT<D>& x, const VecT<D>& add) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = std::fma(mul.raw[i], x.raw[i], add.raw[i]);
  return r;
}
// add - mul * x, fused.
template <class D>
HWY_INLINE VecT<D> NegMulAdd(const VecT<D>& mul, const VecT<D>& x, const VecT<D>& add) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = std::fma(-mul.raw[i], x.raw[i], add.raw[i]);
  return r;
}
template <class D>
HWY_INLINE VecT<D> Neg(const VecT<D>& v) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = -v.raw[i];
  return r;
}
template <class D>
HWY_INLINE VecT<D> Abs(const VecT<D>& v) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = std::fabs(v.raw[i]);
  return r;
}
template <class D>
HWY_INLINE VecT<D> Reverse2(D, const VecT<D>& v) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = v.raw[i ^ 1];
  return r;
}
// Each lane converted to the wider type of descriptor DW (same lane count).
template <class DW, class DN>
HWY_INLINE VecT<DW> PromoteTo(DW, const VecT<DN>& v) {
  static_assert(DW::kLanes == DN::kLanes, "PromoteTo keeps the lane count");
  VecT<DW> r;
  for (size_t i = 0; i < DW::kLanes; ++i) r.raw[i] = static_cast<TFromD<DW>>(v.raw[i]);
  return r;
}

// Halving reduction: lanes i and i + h are added for h = N/2, N/4, ..., 1.
template <class D>
HWY_INLINE TFromD<D> ReduceSum(D, const VecT<D>& v) {
  TFromD<D> t[D::kLanes];
  HWY_SHIM_LANES t[i] = v.raw[i];
  for (size_t h = D::kLanes / 2; h >= 1; h /= 2)
    for (size_t i = 0; i < h; ++i) t[i] = t[i] + t[i + h];
  return t[0];
}
template <class D>
HWY_INLINE TFromD<D> ReduceMin(D, const VecT<D>& v) {
  TFromD<D> m = v.raw[0];
  HWY_SHIM_LANES m = v.raw[i] < m ? v.raw[i] : m;
  return m;
}
template <class D>
HWY_INLINE TFromD<D> ReduceMax(D, const VecT<D>& v) {
  TFromD<D> m = v.raw[0];
  HWY_SHIM_LANES m = v.raw[i] > m ? v.raw[i] : m;
  return m;
}

// Comparisons (false for NaN) and masks.
#define HWY_SHIM_COMPARE(NAME, OP)                                   \
  template <class D>                                                 \
  HWY_INLINE MaskT<D> NAME(const VecT<D>& a, const VecT<D>& b) {       \
    MaskT<D> m;                                                      \
    HWY_SHIM_LANES m.raw[i] = a.raw[i] OP b.raw[i];                  \
    return m;                                                        \
  }
HWY_SHIM_COMPARE(Eq, ==)
HWY_SHIM_COMPARE(Lt, <)
HWY_SHIM_COMPARE(Gt, >)
HWY_SHIM_COMPARE(Le, <=)
HWY_SHIM_COMPARE(Ge, >=)
#undef HWY_SHIM_COMPARE

template <class D>
HWY_INLINE MaskT<D> Or(const MaskT<D>& a, const MaskT<D>& b) {
  MaskT<D> m;
  HWY_SHIM_LANES m.raw[i] = a.raw[i] || b.raw[i];
  return m;
}
template <class D>
HWY_INLINE MaskT<D> And(const MaskT<D>& a, const MaskT<D>& b) {
  MaskT<D> m;
  HWY_SHIM_LANES m.raw[i] = a.raw[i] && b.raw[i];
  return m;
}
template <class D>
HWY_INLINE MaskT<D> FirstN(D, size_t n) {
  MaskT<D> m;
  HWY_SHIM_LANES m.raw[i] = i < n;
  return m;
}
template <class D>
HWY_INLINE VecT<D> IfThenElse(const MaskT<D>& m, const VecT<D>& yes, const VecT<D>& no) {
  VecT<D> r;
  HWY_SHIM_LANES r.raw[i] = m.raw[i] ? yes.raw[i] : no.raw[i];
  return r;
}
template <class D>
HWY_INLINE bool AllFalse(D, const MaskT<D>& m) {
  HWY_SHIM_LANES if (m.raw[i]) return false;
  return true;
}
template <class D>
HWY_INLINE intptr_t FindFirstTrue(D, const MaskT<D>& m) {
  HWY_SHIM_LANES if (m.raw[i]) return static_cast<intptr_t>(i);
  return -1;
}

#undef HWY_SHIM_LANES

#if defined(__AVX2__) && defined(__FMA__)
// The hot operations of the real 64-byte vectors as pairs of 256-bit AVX2
// operations (the same lane-wise IEEE results as the loops above, faster).
#define HWY_SHIM_X86_PAIR(TYPE, N, VT, SUF)                                        \
  HWY_INLINE VecT<Simd<TYPE, N>> LoadU(Simd<TYPE, N>, const TYPE* HWY_RESTRICT p) { \
    VecT<Simd<TYPE, N>> r;                                                        \
    _mm256_storeu_##SUF(r.raw, _mm256_loadu_##SUF(p));                            \
    _mm256_storeu_##SUF(r.raw + N / 2, _mm256_loadu_##SUF(p + N / 2));            \
    return r;                                                                     \
  }                                                                               \
  HWY_INLINE VecT<Simd<TYPE, N>> MulAdd(const VecT<Simd<TYPE, N>>& m,              \
                                        const VecT<Simd<TYPE, N>>& x,              \
                                        const VecT<Simd<TYPE, N>>& a) {            \
    VecT<Simd<TYPE, N>> r;                                                        \
    _mm256_storeu_##SUF(r.raw, _mm256_fmadd_##SUF(_mm256_loadu_##SUF(m.raw),      \
                                                  _mm256_loadu_##SUF(x.raw),      \
                                                  _mm256_loadu_##SUF(a.raw)));    \
    _mm256_storeu_##SUF(r.raw + N / 2,                                            \
                        _mm256_fmadd_##SUF(_mm256_loadu_##SUF(m.raw + N / 2),     \
                                           _mm256_loadu_##SUF(x.raw + N / 2),     \
                                           _mm256_loadu_##SUF(a.raw + N / 2)));   \
    return r;                                                                     \
  }
HWY_SHIM_X86_PAIR(double, 8, __m256d, pd)
HWY_SHIM_X86_PAIR(float, 16, __m256, ps)
#undef HWY_SHIM_X86_PAIR
#endif

}  // namespace N_AVX3
}  // namespace hwy

#endif  // HWY_SHIM_HIGHWAY_H_
