// LbmLib::nodes::PhysicalNode (libs/LbmLib/include/nodes/PhysicalNode.hpp):
// a lattice node as host plugins and reporters see it.  The lattice lives on
// the device; this is a read-only view of one node of the last downloaded
// snapshot (domain id, cell type, fluid velocity and density, species
// concentrations), taken when a host plugin first reads the lattice in a
// step.  Writes (FluidSolver::addMass, distributions) have no host path:
// mass and species sources are the device bio solvers' per-domain tables.
#ifndef LBIBCELL_DROPIN_PHYSICALNODE_HPP
#define LBIBCELL_DROPIN_PHYSICALNODE_HPP

#include <LbmLib/include/Field.hpp>

#include <string>

namespace LbmLib {
namespace geometry {
class GeometryHandler;
}
namespace nodes {

class PhysicalNode;

// FluidSolver's read accessors (FluidSolver.cpp:196-257)
class FluidSolverView {
 public:
    explicit FluidSolverView(const PhysicalNode& n) : node_(n) {}
    Field<double> getVelocity() const;
    double getRho() const;
    void addMass(double mass);  // not available on the host: throws

 private:
    const PhysicalNode& node_;
};

// CDE solvers' getC (CDESolverD2Q5.cpp: the sum of the five distributions)
class CDESolverView {
 public:
    CDESolverView(const PhysicalNode& n, int species) : node_(n), k_(species) {}
    double getC() const;

 private:
    const PhysicalNode& node_;
    int k_;
};

class PhysicalNode {
 public:
    PhysicalNode(int x, int y, const geometry::GeometryHandler* owner) : x_(x), y_(y), owner_(owner) {}
    int getXPos() const { return x_; }
    int getYPos() const { return y_; }
    unsigned int getDomainIdentifier() const;
    unsigned int getCellType() const;
    FluidSolverView getFluidSolver() const { return FluidSolverView(*this); }
    CDESolverView getCDESolverSlow(const std::string& name) const;
    const geometry::GeometryHandler* owner() const { return owner_; }

 private:
    int x_, y_;
    const geometry::GeometryHandler* owner_;
};

}  // namespace nodes
}  // namespace LbmLib

#endif
