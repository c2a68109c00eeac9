// Stand-in for vtkm/worklet/WorkletMapTopology.h (VTK-m 1.9.0).
#pragma once
#include "WorkletMapField.h"
