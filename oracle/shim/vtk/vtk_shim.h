// Minimal stand-in for the VTK classes that Geometry::loadGeometryVTK names
// (oracle/_ref reference build only; VTK is not installed here).  The classes
// only let the reference source compile: every method that would read a file
// reports that VTK input is unavailable.  The reference build loads
// geometries from the txt format only.
#ifndef LBIB_SHIM_VTK_H
#define LBIB_SHIM_VTK_H
#include <cstddef>
#include <stdexcept>
#include <string>

typedef long long vtkIdType;
typedef std::string vtkStdString;

[[noreturn]] inline void lbib_vtk_unavailable() {
    throw std::runtime_error("VTK geometry input is unavailable in this build");
}

struct vtkObjectShim {
    virtual ~vtkObjectShim() {}
    const char* GetClassName() const { return "vtkObject"; }
};
struct vtkDataObject : vtkObjectShim {};
struct vtkAbstractArray : vtkObjectShim {};
struct vtkDataArray : vtkAbstractArray {};
struct vtkDoubleArray : vtkDataArray {
    void DeepCopy(vtkDataArray*) { lbib_vtk_unavailable(); }
    double GetValue(vtkIdType) const { lbib_vtk_unavailable(); }
    vtkIdType GetSize() const { lbib_vtk_unavailable(); }
};
struct vtkStringArray : vtkAbstractArray {
    void DeepCopy(vtkAbstractArray*) { lbib_vtk_unavailable(); }
    vtkStdString GetValue(vtkIdType) const { lbib_vtk_unavailable(); }
};
struct vtkPointData : vtkObjectShim {
    vtkDataArray* GetArray(const char*) { lbib_vtk_unavailable(); }
    vtkAbstractArray* GetAbstractArray(const char*) { lbib_vtk_unavailable(); }
};
struct vtkCellData : vtkObjectShim {};
struct vtkPoints : vtkObjectShim {
    vtkIdType GetNumberOfPoints() const { lbib_vtk_unavailable(); }
    double* GetPoint(vtkIdType) { lbib_vtk_unavailable(); }
};
struct vtkCellArray : vtkObjectShim {
    vtkIdType GetNumberOfCells() const { lbib_vtk_unavailable(); }
    void GetCell(vtkIdType, vtkIdType&, vtkIdType*&) { lbib_vtk_unavailable(); }
};
struct vtkPolygon : vtkObjectShim {};
struct vtkPolyData : vtkDataObject {
    void ShallowCopy(vtkDataObject*) { lbib_vtk_unavailable(); }
    vtkCellArray* GetPolys() { lbib_vtk_unavailable(); }
    vtkPoints* GetPoints() { lbib_vtk_unavailable(); }
    vtkPointData* GetPointData() { lbib_vtk_unavailable(); }
};
struct vtkMultiBlockDataSet : vtkDataObject {
    void ShallowCopy(vtkDataObject*) { lbib_vtk_unavailable(); }
    unsigned GetNumberOfBlocks() const { lbib_vtk_unavailable(); }
    vtkDataObject* GetBlock(unsigned) { lbib_vtk_unavailable(); }
};
struct vtkXMLMultiBlockDataReader : vtkObjectShim {
    void SetFileName(const char*) {}
    void Update() { lbib_vtk_unavailable(); }
    vtkMultiBlockDataSet* GetOutput() { lbib_vtk_unavailable(); }
};
struct vtkXMLMultiBlockDataWriter : vtkObjectShim {};

template <typename T>
class vtkSmartPointer {
 public:
    vtkSmartPointer() : p_(nullptr) {}
    vtkSmartPointer(T* p) : p_(p) {}
    template <typename U> vtkSmartPointer(const vtkSmartPointer<U>& o) : p_(o.Get()) {}
    static vtkSmartPointer<T> New() { return vtkSmartPointer<T>(nullptr); }
    T* operator->() const { lbib_vtk_unavailable(); }
    T* Get() const { return p_; }
    operator T*() const { return p_; }
 private:
    T* p_;
};
#endif
