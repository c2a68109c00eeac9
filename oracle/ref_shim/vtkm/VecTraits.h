// Stand-in for vtkm/VecTraits.h (VTK-m 1.9.0): everything RBMD uses from it lives in Types.h.
#pragma once
#include "Types.h"
