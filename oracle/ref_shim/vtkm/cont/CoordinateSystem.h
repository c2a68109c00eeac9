// Stand-in for vtkm/cont/CoordinateSystem.h (VTK-m 1.9.0): nothing of it is used on the path compiled here.
#pragma once
#include "ArrayHandle.h"
