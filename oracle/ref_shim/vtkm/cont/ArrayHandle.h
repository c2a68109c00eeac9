// Stand-in for vtkm/cont/ArrayHandle.h (VTK-m 1.9.0): an array handle is a host vector, its
// read portal a (pointer, size) view with Get(i).  Test infrastructure.
#pragma once
#include <vector>

#include "../Types.h"

namespace vtkm {
namespace cont {

template <typename T>
struct ReadPortalT {
  using ValueType = T;
  const T* data = nullptr;
  Id size = 0;
  T Get(Id i) const { return data[i]; }
  Id GetNumberOfValues() const { return size; }
};

template <typename T>
struct WritePortalT {
  using ValueType = T;
  T* data = nullptr;
  Id size = 0;
  T Get(Id i) const { return data[i]; }
  void Set(Id i, const T& v) const { data[i] = v; }
  Id GetNumberOfValues() const { return size; }
};

template <typename T, typename Storage = void>
class ArrayHandle {
 public:
  using ValueType = T;
  using ReadPortalType = ReadPortalT<T>;
  using WritePortalType = WritePortalT<T>;
  void Allocate(Id n) { v_.resize((size_t)n); }
  Id GetNumberOfValues() const { return (Id)v_.size(); }
  ReadPortalType ReadPortal() const { return {v_.data(), (Id)v_.size()}; }
  WritePortalType WritePortal() { return {v_.data(), (Id)v_.size()}; }
  std::vector<T>& Vector() { return v_; }

 private:
  std::vector<T> v_;
};

struct ExecutionObjectBase {};
struct DeviceAdapterId {};
struct Token {};

}  // namespace cont
}  // namespace vtkm
