// Project-written stand-in for the small subset of the Google Highway API that
// scl-core's diffusion translation units use (scl/core/simd.hpp:15-30 include
// <hwy/highway.h> and inject hwy::HWY_NAMESPACE into scl::simd).
//
// This is ORACLE infrastructure: it exists only so that the reference's own
// C++ sources under the reference tree compile into oracle/_ref/ for parity
// checks and the CPU baseline. It contains no Highway source. Every op is a
// plain per-lane loop over a fixed-width lane array, written so that GCC
// auto-vectorises it at the width chosen by SCL_SHIM_VEC_BYTES.
//
// Arithmetic contract that matters for parity:
//   MulAdd(a, b, c) == fma(a, b, c) per lane (single rounding), which is what
//   Highway's MulAdd lowers to on every x86 target with FMA (AVX2 and up).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <type_traits>

#ifndef SCL_SHIM_VEC_BYTES
#if defined(__AVX512F__)
#define SCL_SHIM_VEC_BYTES 64
#elif defined(__AVX__)
#define SCL_SHIM_VEC_BYTES 32
#else
#define SCL_SHIM_VEC_BYTES 16
#endif
#endif

#define HWY_NAMESPACE N_SCL_SHIM
#define HWY_INLINE inline __attribute__((always_inline))
#define HWY_ATTR
#define HWY_RESTRICT __restrict__

namespace hwy {

struct SortAscending {};
struct SortDescending {};

namespace N_SCL_SHIM {

template <class T>
struct Simd {
  using T_ = T;
  static constexpr size_t kLanes = SCL_SHIM_VEC_BYTES / sizeof(T) ? SCL_SHIM_VEC_BYTES / sizeof(T) : 1;
};

template <class T>
using ScalableTag = Simd<T>;

template <class D>
using TFromD = typename D::T_;

template <class T>
struct Vec {
  static constexpr size_t N = Simd<T>::kLanes;
  alignas(SCL_SHIM_VEC_BYTES) T v[N];
};

template <class T>
struct Mask {
  static constexpr size_t N = Simd<T>::kLanes;
  bool m[N];
};

namespace detail {
template <size_t S> struct UnsignedOfSize;
template <> struct UnsignedOfSize<1> { using type = uint8_t; };
template <> struct UnsignedOfSize<2> { using type = uint16_t; };
template <> struct UnsignedOfSize<4> { using type = uint32_t; };
template <> struct UnsignedOfSize<8> { using type = uint64_t; };
}  // namespace detail

template <class D>
using RebindToUnsigned = Simd<typename detail::UnsignedOfSize<sizeof(TFromD<D>)>::type>;

template <class D>
using VFromD = Vec<TFromD<D>>;

template <class T>
HWY_INLINE constexpr size_t Lanes(Simd<T>) { return Simd<T>::kLanes; }

template <class T>
HWY_INLINE Vec<T> Zero(Simd<T>) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = T(0);
  return r;
}

template <class T>
HWY_INLINE Vec<T> Undefined(Simd<T> d) { return Zero(d); }

template <class T, class U>
HWY_INLINE Vec<T> Set(Simd<T>, U x) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = static_cast<T>(x);
  return r;
}

template <class T, class U>
HWY_INLINE Vec<T> Iota(Simd<T>, U start) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = static_cast<T>(static_cast<T>(start) + static_cast<T>(i));
  return r;
}

template <class T>
HWY_INLINE Vec<T> Load(Simd<T>, const T* HWY_RESTRICT p) {
  Vec<T> r;
  std::memcpy(r.v, p, sizeof(r.v));
  return r;
}

template <class T>
HWY_INLINE Vec<T> LoadU(Simd<T> d, const T* HWY_RESTRICT p) { return Load(d, p); }

template <class T>
HWY_INLINE void Store(Vec<T> a, Simd<T>, T* HWY_RESTRICT p) { std::memcpy(p, a.v, sizeof(a.v)); }

template <class T>
HWY_INLINE void StoreU(Vec<T> a, Simd<T> d, T* HWY_RESTRICT p) { Store(a, d, p); }

template <class T>
HWY_INLINE void Stream(Vec<T> a, Simd<T> d, T* HWY_RESTRICT p) { Store(a, d, p); }

template <class T>
HWY_INLINE void StoreInterleaved2(Vec<T> a, Vec<T> b, Simd<T>, T* HWY_RESTRICT p) {
  for (size_t i = 0; i < Vec<T>::N; ++i) {
    p[2 * i] = a.v[i];
    p[2 * i + 1] = b.v[i];
  }
}

template <class T>
HWY_INLINE void LoadInterleaved2(Simd<T>, const T* HWY_RESTRICT p, Vec<T>& a, Vec<T>& b) {
  for (size_t i = 0; i < Vec<T>::N; ++i) {
    a.v[i] = p[2 * i];
    b.v[i] = p[2 * i + 1];
  }
}

#define SCL_SHIM_BINOP(NAME, EXPR)                         \
  template <class T>                                       \
  HWY_INLINE Vec<T> NAME(Vec<T> a, Vec<T> b) {             \
    Vec<T> r;                                              \
    for (size_t i = 0; i < Vec<T>::N; ++i) {               \
      const T x = a.v[i];                                  \
      const T y = b.v[i];                                  \
      r.v[i] = (EXPR);                                     \
    }                                                      \
    return r;                                              \
  }

SCL_SHIM_BINOP(Add, x + y)
SCL_SHIM_BINOP(Sub, x - y)
SCL_SHIM_BINOP(Mul, x * y)
SCL_SHIM_BINOP(Div, x / y)
SCL_SHIM_BINOP(Min, (y < x) ? y : x)
SCL_SHIM_BINOP(Max, (x < y) ? y : x)
#undef SCL_SHIM_BINOP

// Single-rounding fused multiply-add per lane.
template <class T>
HWY_INLINE Vec<T> MulAdd(Vec<T> a, Vec<T> b, Vec<T> c) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = std::fma(a.v[i], b.v[i], c.v[i]);
  return r;
}

template <class T>
HWY_INLINE Vec<T> NegMulAdd(Vec<T> a, Vec<T> b, Vec<T> c) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = std::fma(-a.v[i], b.v[i], c.v[i]);
  return r;
}

template <class T>
HWY_INLINE Vec<T> Abs(Vec<T> a) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = a.v[i] < T(0) ? T(-a.v[i]) : a.v[i];
  return r;
}

template <class T>
HWY_INLINE Vec<T> Neg(Vec<T> a) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = -a.v[i];
  return r;
}

template <class T>
HWY_INLINE Vec<T> Sqrt(Vec<T> a) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = std::sqrt(a.v[i]);
  return r;
}

template <class T>
HWY_INLINE Vec<T> Exp(Simd<T>, Vec<T> a) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = std::exp(a.v[i]);
  return r;
}

template <class T>
HWY_INLINE Vec<T> Log(Simd<T>, Vec<T> a) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = std::log(a.v[i]);
  return r;
}

template <class T>
HWY_INLINE Vec<T> Reverse(Simd<T>, Vec<T> a) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = a.v[Vec<T>::N - 1 - i];
  return r;
}

template <class T>
HWY_INLINE T GetLane(Vec<T> a) { return a.v[0]; }

// Horizontal reductions return the result broadcast to every lane.
template <class T>
HWY_INLINE Vec<T> SumOfLanes(Simd<T> d, Vec<T> a) {
  T s = T(0);
  for (size_t i = 0; i < Vec<T>::N; ++i) s += a.v[i];
  return Set(d, s);
}

template <class T>
HWY_INLINE T ReduceSum(Simd<T> d, Vec<T> a) { return GetLane(SumOfLanes(d, a)); }

template <class T>
HWY_INLINE Vec<T> MinOfLanes(Simd<T> d, Vec<T> a) {
  T s = a.v[0];
  for (size_t i = 1; i < Vec<T>::N; ++i) s = a.v[i] < s ? a.v[i] : s;
  return Set(d, s);
}

template <class T>
HWY_INLINE Vec<T> MaxOfLanes(Simd<T> d, Vec<T> a) {
  T s = a.v[0];
  for (size_t i = 1; i < Vec<T>::N; ++i) s = s < a.v[i] ? a.v[i] : s;
  return Set(d, s);
}

#define SCL_SHIM_CMP(NAME, OP)                           \
  template <class T>                                     \
  HWY_INLINE Mask<T> NAME(Vec<T> a, Vec<T> b) {          \
    Mask<T> r;                                           \
    for (size_t i = 0; i < Vec<T>::N; ++i) r.m[i] = (a.v[i] OP b.v[i]); \
    return r;                                            \
  }

SCL_SHIM_CMP(Eq, ==)
SCL_SHIM_CMP(Ne, !=)
SCL_SHIM_CMP(Lt, <)
SCL_SHIM_CMP(Gt, >)
SCL_SHIM_CMP(Le, <=)
SCL_SHIM_CMP(Ge, >=)
#undef SCL_SHIM_CMP

template <class T>
HWY_INLINE size_t CountTrue(Simd<T>, Mask<T> m) {
  size_t c = 0;
  for (size_t i = 0; i < Mask<T>::N; ++i) c += m.m[i] ? 1 : 0;
  return c;
}

template <class T>
HWY_INLINE bool AllTrue(Simd<T>, Mask<T> m) {
  for (size_t i = 0; i < Mask<T>::N; ++i)
    if (!m.m[i]) return false;
  return true;
}

template <class T>
HWY_INLINE bool AllFalse(Simd<T>, Mask<T> m) {
  for (size_t i = 0; i < Mask<T>::N; ++i)
    if (m.m[i]) return false;
  return true;
}

template <class T>
HWY_INLINE Vec<T> IfThenElse(Mask<T> m, Vec<T> a, Vec<T> b) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = m.m[i] ? a.v[i] : b.v[i];
  return r;
}

template <class T>
HWY_INLINE Vec<T> IfThenElseZero(Mask<T> m, Vec<T> a) {
  Vec<T> r;
  for (size_t i = 0; i < Vec<T>::N; ++i) r.v[i] = m.m[i] ? a.v[i] : T(0);
  return r;
}

template <class T>
HWY_INLINE void VQSortStatic(T* HWY_RESTRICT p, size_t n, SortAscending) {
  std::sort(p, p + n);
}

template <class T>
HWY_INLINE void VQSortStatic(T* HWY_RESTRICT p, size_t n, SortDescending) {
  std::sort(p, p + n, std::greater<T>());
}

}  // namespace N_SCL_SHIM

template <class T>
inline void VQSort(T* HWY_RESTRICT p, size_t n, SortAscending o) { N_SCL_SHIM::VQSortStatic(p, n, o); }

template <class T>
inline void VQSort(T* HWY_RESTRICT p, size_t n, SortDescending o) { N_SCL_SHIM::VQSortStatic(p, n, o); }

}  // namespace hwy
