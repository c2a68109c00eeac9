// Stand-in for vtkm/cont/ArrayHandleGroupVec.h (VTK-m 1.9.0): fixed-size groups (type name only).
#pragma once
#include "ArrayHandle.h"

namespace vtkm {
namespace cont {
template <typename ComponentsHandle, IdComponent N>
class ArrayHandleGroupVec {};
}  // namespace cont
}  // namespace vtkm
