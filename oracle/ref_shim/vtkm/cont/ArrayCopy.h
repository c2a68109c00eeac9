// Stand-in for vtkm/cont/ArrayCopy.h (VTK-m 1.9.0): copy an index array into an array handle.
#pragma once
#include "ArrayHandleIndex.h"

namespace vtkm {
namespace cont {
inline void ArrayCopy(const ArrayHandleIndex& src, ArrayHandle<Id>& dst) {
  dst.Allocate(src.size);
  for (Id i = 0; i < src.size; ++i) dst.Vector()[(size_t)i] = i;
}
}  // namespace cont
}  // namespace vtkm
