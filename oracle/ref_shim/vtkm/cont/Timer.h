// Stand-in for vtkm/cont/Timer.h (VTK-m 1.9.0): a timer that measures nothing (type name only).
#pragma once
#include "ArrayHandle.h"

namespace vtkm {
namespace cont {
struct Timer {
  void Start() {}
  void Stop() {}
  double GetElapsedTime() const { return 0.0; }
};
}  // namespace cont
}  // namespace vtkm
