// Stand-in for vtkm/cont/ArrayHandleIndex.h (VTK-m 1.9.0): the implicit array 0, 1, ..., n-1.
#pragma once
#include "ArrayHandle.h"

namespace vtkm {
namespace cont {
struct ArrayHandleIndex {
  explicit ArrayHandleIndex(Id n) : size(n) {}
  Id size;
};
}  // namespace cont
}  // namespace vtkm
