// vtk_io.h — VTK XML files without VTK: the ASCII multiblock (.vtm) geometry
// reader of Geometry::loadGeometryVTK (Geometry.cpp:162-306) and the writers
// behind the vtk*Reporter functors (vtkCellReporter.cpp, vtkForceReporter.cpp,
// vtkCDEReporter.cpp, vtkFluidReporter.cpp), in the layout VTK's
// vtkXMLMultiBlockDataWriter gives them in ASCII mode: <name>.vtm lists the
// blocks, block k lives in <name>/<name>_k.{vtp,vti}.  Host code only.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace lbib {
namespace vtk {

struct Conn {
    uint32_t id1, id2, dom;
    std::string desc;  // "\t<bsolver>\t<cdesolver>" per pair
};

// What loadGeometryVTK builds: nodes with ids 0..n-1 in point order, the
// connections polygon by polygon, and each domain's cell type.
struct Geometry {
    std::vector<double> x, y;
    std::vector<Conn> conns;
    std::map<uint32_t, uint32_t> cellType;
};

// Throws std::runtime_error with the reference's message where it has one.
void read_vtm_geometry(const std::string& path, Geometry& g);

// One data array of a block: name, components, values (tuple-major), VTK type
// ("Float64", "Float32", "UInt32", "Int64").
struct Array {
    std::string name;
    int components;
    std::string type;
    std::vector<double> values;
};

// Poly data: points (x, y; z = 0), cells as a CSR (offsets after each cell, as
// VTK stores them), point arrays, cell arrays, point string arrays.
struct PolyData {
    std::vector<double> px, py;          // written as Float32 (vtkPoints' default type)
    std::vector<int64_t> connectivity;
    std::vector<int64_t> offsets;
    bool lines = false;                  // cells are lines (else polygons)
    std::vector<Array> pointData;
    std::vector<Array> cellData;
    std::vector<std::pair<std::string, std::vector<std::string>>> pointStrings;
};

// Image data of X x Y points, origin 0, spacing s.
struct ImageData {
    int X = 0, Y = 0;
    double spacing = 1.0;
    std::vector<Array> pointData;
};

// Appends one block to <vtm> (created when absent), as a reporter does when
// it reads the file back and adds its block at the end.
void append_block(const std::string& vtm, const PolyData& pd);
void append_block(const std::string& vtm, const ImageData& id);

}  // namespace vtk
}  // namespace lbib
