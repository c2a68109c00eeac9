// Stand-in for vtkm/cont/ArrayHandleGroupVecVariable.h (VTK-m 1.9.0): entry i of the grouped
// array is the range [offsets[i], offsets[i+1]) of the components array.
#pragma once
#include "ArrayHandle.h"

namespace vtkm {
namespace cont {

template <typename ComponentsHandle, typename OffsetsHandle>
class ArrayHandleGroupVecVariable {
 public:
  using ComponentsPortal = typename ComponentsHandle::ReadPortalType;
  using OffsetsPortal = typename OffsetsHandle::ReadPortalType;
  struct ReadPortalType {
    using ValueType = vtkm::VecFromPortal<ComponentsPortal>;
    ComponentsPortal components;
    OffsetsPortal offsets;
    ValueType Get(Id i) const {
      const Id b = offsets.Get(i);
      return ValueType(components, (IdComponent)(offsets.Get(i + 1) - b), b);
    }
    Id GetNumberOfValues() const { return offsets.GetNumberOfValues() - 1; }
  };
};

}  // namespace cont
}  // namespace vtkm
