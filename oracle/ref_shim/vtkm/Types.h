// Minimal stand-in for the parts of VTK-m 1.9.0 (https://gitlab.kitware.com/vtk/vtk-m, tag
// v1.9.0) that RBMD's force-path headers use, so that those headers compile on the host with
// gcc and can be executed as the oracle's reference.  Test infrastructure only: nothing in the
// library links it.
//
// Semantics restated from VTK-m's published API (vtkm/Types.h, vtkm/VecTraits.h,
// vtkm/VectorAnalysis.h, vtkm/Math.h):
//   * vtkm::Id and vtkm::IdComponent are 32-bit: RBMD builds VTK-m with VTKm_USE_64BIT_IDS=OFF
//     (rbmd/README.md:94); vtkm::FloatDefault is Float32 (the default precision);
//   * Vec<T, N> arithmetic is component-wise in T; a Vec converts to a Vec of another component
//     type component by component with static_cast (float -> int truncates toward zero);
//   * a Float64 scalar times (or dividing) a Vec of Float32 is evaluated in double per component
//     and rounded back to float;
//   * Dot(a, b) = a[0]*b[0] + a[1]*b[1] + a[2]*b[2] (left to right); MagnitudeSquared = Dot(x, x);
//     Magnitude = Sqrt(MagnitudeSquared);
//   * the math functions call the C++ standard library overload of the argument's type.
#pragma once
#include <cmath>
#include <cstdint>
#include <initializer_list>
#include <type_traits>

#define VTKM_EXEC
#define VTKM_CONT
#define VTKM_EXEC_CONT
#define VTKM_ALWAYS_EXPORT
#define VTKM_SUPPRESS_EXEC_WARNINGS
#define VTKM_DEPRECATED(...)

namespace vtkm {

using Int8 = int8_t;
using UInt8 = uint8_t;
using Int16 = int16_t;
using UInt16 = uint16_t;
using Int32 = int32_t;
using UInt32 = uint32_t;
using Int64 = int64_t;
using UInt64 = uint64_t;
using Float32 = float;
using Float64 = double;
using Id = Int32;
using IdComponent = Int32;
using FloatDefault = Float32;
using HashType = UInt32;

template <typename T, IdComponent N>
class Vec {
 public:
  using ComponentType = T;
  static constexpr IdComponent NUM_COMPONENTS = N;
  T Components[N];

  Vec() = default;
  Vec(const T& fill) {                       // NOLINT: implicit, as in VTK-m ("Vec3f H = 0.0;")
    for (IdComponent i = 0; i < N; ++i) Components[i] = fill;
  }
  template <typename... Ts, typename = typename std::enable_if<(sizeof...(Ts) == N && N > 1)>::type>
  Vec(const Ts&... vals) : Components{static_cast<T>(vals)...} {}   // NOLINT
  template <typename U>
  Vec(const Vec<U, N>& src) {                // NOLINT: implicit component-wise conversion
    for (IdComponent i = 0; i < N; ++i) Components[i] = static_cast<T>(src[i]);
  }
  T& operator[](IdComponent i) { return Components[i]; }
  const T& operator[](IdComponent i) const { return Components[i]; }
  IdComponent GetNumberOfComponents() const { return N; }

  Vec& operator+=(const Vec& b) { for (IdComponent i = 0; i < N; ++i) Components[i] += b[i]; return *this; }
  Vec& operator-=(const Vec& b) { for (IdComponent i = 0; i < N; ++i) Components[i] -= b[i]; return *this; }
  Vec& operator*=(const Vec& b) { for (IdComponent i = 0; i < N; ++i) Components[i] *= b[i]; return *this; }
  Vec& operator/=(const Vec& b) { for (IdComponent i = 0; i < N; ++i) Components[i] /= b[i]; return *this; }
  Vec& operator*=(const T& s) { for (IdComponent i = 0; i < N; ++i) Components[i] *= s; return *this; }
  Vec& operator/=(const T& s) { for (IdComponent i = 0; i < N; ++i) Components[i] /= s; return *this; }
  bool operator==(const Vec& b) const {
    for (IdComponent i = 0; i < N; ++i) if (!(Components[i] == b[i])) return false;
    return true;
  }
  bool operator!=(const Vec& b) const { return !(*this == b); }
};

// element-wise Vec (op) Vec; a second operand of another component type is converted first
#define RBMD_SHIM_VEC_BINOP(OP)                                                              \
  template <typename T, typename U, IdComponent N>                                           \
  inline Vec<T, N> operator OP(Vec<T, N> a, const Vec<U, N>& b) {                            \
    for (IdComponent i = 0; i < N; ++i) a[i] = a[i] OP static_cast<T>(b[i]);                 \
    return a;                                                                                \
  }                                                                                          \
  template <typename T, IdComponent N>                                                       \
  inline Vec<T, N> operator OP(Vec<T, N> a, const T& s) {                                    \
    for (IdComponent i = 0; i < N; ++i) a[i] = a[i] OP s;                                    \
    return a;                                                                                \
  }                                                                                          \
  template <typename T, IdComponent N>                                                       \
  inline Vec<T, N> operator OP(const T& s, Vec<T, N> a) {                                    \
    for (IdComponent i = 0; i < N; ++i) a[i] = s OP a[i];                                    \
    return a;                                                                                \
  }                                                                                          \
  template <typename T, IdComponent N,                                                       \
            typename = typename std::enable_if<!std::is_same<T, Float64>::value>::type>      \
  inline Vec<T, N> operator OP(Vec<T, N> a, Float64 s) {                                     \
    for (IdComponent i = 0; i < N; ++i) a[i] = static_cast<T>(a[i] OP s);                   \
    return a;                                                                                \
  }                                                                                          \
  template <typename T, IdComponent N,                                                       \
            typename = typename std::enable_if<!std::is_same<T, Float64>::value>::type>      \
  inline Vec<T, N> operator OP(Float64 s, Vec<T, N> a) {                                     \
    for (IdComponent i = 0; i < N; ++i) a[i] = static_cast<T>(s OP a[i]);                   \
    return a;                                                                                \
  }
RBMD_SHIM_VEC_BINOP(+)
RBMD_SHIM_VEC_BINOP(-)
RBMD_SHIM_VEC_BINOP(*)
RBMD_SHIM_VEC_BINOP(/)
#undef RBMD_SHIM_VEC_BINOP

template <typename T, IdComponent N>
inline Vec<T, N> operator-(Vec<T, N> a) {
  for (IdComponent i = 0; i < N; ++i) a[i] = -a[i];
  return a;
}

using Id2 = Vec<Id, 2>;
using Id3 = Vec<Id, 3>;
using Vec2i = Vec<Id, 2>;
using Vec3i = Vec<Id, 3>;
using Vec2i_32 = Vec<Int32, 2>;
using Vec3i_32 = Vec<Int32, 3>;
using Vec2f = Vec<FloatDefault, 2>;
using Vec3f = Vec<FloatDefault, 3>;
using Vec4f = Vec<FloatDefault, 4>;
using Vec2f_32 = Vec<Float32, 2>;
using Vec3f_32 = Vec<Float32, 3>;
using Vec3f_64 = Vec<Float64, 3>;

template <typename T1, typename T2>
struct Pair {
  T1 first;
  T2 second;
};

// component access used by the reference's math header
template <typename T>
struct VecTraits {
  using ComponentType = T;
  static constexpr IdComponent NUM_COMPONENTS = 1;
};
template <typename T, IdComponent N>
struct VecTraits<Vec<T, N>> {
  using ComponentType = T;
  static constexpr IdComponent NUM_COMPONENTS = N;
};
template <typename T>
struct TypeTraits {};

// a view of a portal's range [offset, offset + n) (ArrayHandleGroupVecVariable entries)
template <typename PortalType>
class VecFromPortal {
 public:
  using ComponentType = typename std::remove_const<typename PortalType::ValueType>::type;
  VecFromPortal() = default;
  VecFromPortal(const PortalType& p, IdComponent n, Id offset) : portal_(p), n_(n), offset_(offset) {}
  IdComponent GetNumberOfComponents() const { return n_; }
  ComponentType operator[](IdComponent i) const { return portal_.Get(offset_ + i); }

 private:
  PortalType portal_{};
  IdComponent n_ = 0;
  Id offset_ = 0;
};

}  // namespace vtkm
