// Declaration-only stand-in (see vtkSmartPointer.h).  ORACLE TEST INFRASTRUCTURE ONLY.
#pragma once
#include "vtkSmartPointer.h"
class vtkXMLUnstructuredGridReader {};
