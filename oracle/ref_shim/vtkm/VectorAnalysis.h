// Stand-in for vtkm/VectorAnalysis.h (VTK-m 1.9.0): Dot, MagnitudeSquared, Magnitude.
#pragma once
#include "Math.h"

namespace vtkm {

template <typename T>
inline T Dot(const Vec<T, 2>& a, const Vec<T, 2>& b) { return a[0] * b[0] + a[1] * b[1]; }
template <typename T>
inline T Dot(const Vec<T, 3>& a, const Vec<T, 3>& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
template <typename T, IdComponent N>
inline T MagnitudeSquared(const Vec<T, N>& x) { return Dot(x, x); }
template <typename T, IdComponent N>
inline T Magnitude(const Vec<T, N>& x) { return Sqrt(MagnitudeSquared(x)); }

}  // namespace vtkm
