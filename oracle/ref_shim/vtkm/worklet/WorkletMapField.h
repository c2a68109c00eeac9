// Stand-in for vtkm/worklet/WorkletMapField.h and WorkletMapTopology.h (VTK-m 1.9.0): the tag
// types a worklet names in its ControlSignature / ExecutionSignature.  The oracle's reference
// harness calls a worklet's operator() directly with the arguments its ExecutionSignature lists.
#pragma once
#include <stdexcept>

#include "../cont/ArrayHandle.h"

namespace vtkm {
namespace worklet {

struct WorkletBase {
  struct FieldIn {};
  struct FieldOut {};
  struct FieldInOut {};
  struct WholeArrayIn {};
  struct WholeArrayOut {};
  struct WholeArrayInOut {};
  struct ExecObject {};
  struct AtomicArrayInOut {};
  struct InputIndex {};
  struct WorkIndex {};
  struct OutputIndex {};
  struct ThreadIndices {};
  struct Device {};
  struct _1 {}; struct _2 {}; struct _3 {}; struct _4 {}; struct _5 {}; struct _6 {}; struct _7 {};
  struct _8 {}; struct _9 {}; struct _10 {}; struct _11 {}; struct _12 {}; struct _13 {};
  struct _14 {}; struct _15 {}; struct _16 {}; struct _17 {}; struct _18 {}; struct _19 {};
  struct _20 {};
  // a worklet's error report ends the reference call with an exception
  void RaiseError(const char* msg) const { throw std::runtime_error(msg); }
};
struct WorkletMapField : WorkletBase {};
struct WorkletVisitCellsWithPoints : WorkletBase {
  struct CellSetIn {};
  struct FieldInPoint {};
  struct FieldInCell {};
  struct FieldOutCell {};
  struct FieldOutPoint {};
  struct FieldInOutCell {};
  struct PointCount {};
  struct PointIndices {};
  struct CellShape {};
};

}  // namespace worklet
}  // namespace vtkm
