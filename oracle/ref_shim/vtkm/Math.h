// Stand-in for vtkm/Math.h (VTK-m 1.9.0): the math functions RBMD's force path calls, each the
// C++ standard library overload of its argument's type (float or double).  Test infrastructure.
#pragma once
#include <algorithm>
#include <cmath>

#include "Types.h"

namespace vtkm {

inline Float64 Pi() { return 3.14159265358979323846264338327950288; }
inline Float32 Pif() { return 3.14159265358979323846264338327950288f; }
inline Float64 TwoPi() { return 2.0 * Pi(); }

#define RBMD_SHIM_MATH1(NAME, STD)                                                            \
  inline Float32 NAME(Float32 x) { return std::STD(x); }                                      \
  inline Float64 NAME(Float64 x) { return std::STD(x); }                                      \
  template <typename T, typename = typename std::enable_if<std::is_integral<T>::value>::type> \
  inline Float64 NAME(T x) { return std::STD(static_cast<Float64>(x)); }                      \
  template <typename T, IdComponent N>                                                        \
  inline Vec<T, N> NAME(Vec<T, N> v) {                                                        \
    for (IdComponent i = 0; i < N; ++i) v[i] = NAME(v[i]);                                    \
    return v;                                                                                 \
  }
RBMD_SHIM_MATH1(Sqrt, sqrt)
RBMD_SHIM_MATH1(Exp, exp)
RBMD_SHIM_MATH1(Log, log)
RBMD_SHIM_MATH1(Cos, cos)
RBMD_SHIM_MATH1(Sin, sin)
RBMD_SHIM_MATH1(Round, round)
RBMD_SHIM_MATH1(Floor, floor)
RBMD_SHIM_MATH1(Ceil, ceil)
#undef RBMD_SHIM_MATH1

inline Float32 Pow(Float32 x, Float32 y) { return std::pow(x, y); }
inline Float64 Pow(Float64 x, Float64 y) { return std::pow(x, y); }

inline Int32 Abs(Int32 x) { return x < 0 ? -x : x; }
inline Int64 Abs(Int64 x) { return x < 0 ? -x : x; }
inline Float32 Abs(Float32 x) { return std::fabs(x); }
inline Float64 Abs(Float64 x) { return std::fabs(x); }

template <typename T>
inline T Min(const T& a, const T& b) { return (a < b) ? a : b; }
template <typename T>
inline T Max(const T& a, const T& b) { return (a < b) ? b : a; }
// component-wise on Vecs
template <typename T, IdComponent N>
inline Vec<T, N> Min(const Vec<T, N>& a, const Vec<T, N>& b) {
  Vec<T, N> r;
  for (IdComponent i = 0; i < N; ++i) r[i] = Min(a[i], b[i]);
  return r;
}
template <typename T, IdComponent N>
inline Vec<T, N> Max(const Vec<T, N>& a, const Vec<T, N>& b) {
  Vec<T, N> r;
  for (IdComponent i = 0; i < N; ++i) r[i] = Max(a[i], b[i]);
  return r;
}

}  // namespace vtkm
