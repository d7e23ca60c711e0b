// Declaration-only stand-ins for the VTK types named in the reference's
// reader/writer headers.  VTK is used by the reference only for .vtu file
// I/O, which oracle runs switch off; any call into it aborts.
// ORACLE TEST INFRASTRUCTURE ONLY.
#pragma once
template <class T> class vtkSmartPointer {
public:
  vtkSmartPointer() = default;
  T *operator->() const { return p_; }
  T *Get() const { return p_; }
  static vtkSmartPointer New() { return vtkSmartPointer(); }
private:
  T *p_ = nullptr;
};
