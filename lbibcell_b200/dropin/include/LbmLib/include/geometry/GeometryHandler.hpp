// LbmLib::geometry::GeometryHandler (libs/LbmLib/include/geometry/GeometryHandler.hpp):
// the lattice of a geometry.  Here the lattice is the device simulation that
// SimulationRunner builds; this object answers host plugins' questions about
// it (cell areas, per-domain concentrations, cell types) through the C ABI,
// and forwards their topology edits (createGeometryNode, createConnection,
// eraseConnection, cureLattice).
#ifndef LBIBCELL_DROPIN_GEOMETRYHANDLER_HPP
#define LBIBCELL_DROPIN_GEOMETRYHANDLER_HPP

#include <LbmLib/include/geometry/Geometry.hpp>
#include <LbmLib/include/nodes/PhysicalNode.hpp>

#include <map>
#include <memory>
#include <string>
#include <vector>

struct lbib_handle;

namespace LbmLib {
namespace geometry {

class GeometryHandler {
 public:
    explicit GeometryHandler(const Geometry& geometry);
    ~GeometryHandler();

    // ny rows of nx nodes ([y][x], GeometryHandler.cpp:463-474): read-only
    // views of the device lattice, created on the first call
    const std::vector<std::vector<nodes::PhysicalNode*>>& getPhysicalNodes() const;
    const Geometry& getGeometry() const { return geometry_; }
    // GeometryHandler::computeAreas (GeometryHandler.cpp:101-134)
    const std::map<unsigned int, double> computeAreas() const;
    // GeometryHandler::computeAccumulatedDomainConcentrations (:136-147)
    std::map<unsigned int, double> computeAccumulatedDomainConcentrations(const std::string& name) const;
    // GeometryHandler::cureLattice (:149-170), after the mirror's edits reach the device
    void cureLattice();
    unsigned int createGeometryNode(const double xpos, const double ypos);
    void createConnection(std::shared_ptr<nodes::GeometryNode> const p1, std::shared_ptr<nodes::GeometryNode> const p2,
                          const std::map<std::string, std::vector<std::string>> boundaryconditiondescriptor,
                          const unsigned int domainidentifier);
    void eraseConnection(std::shared_ptr<Connection> toErase);
    const std::shared_ptr<nodes::GeometryNode> returnGeometryNode(const unsigned int nodeID) const;
    // getCellTypeTrackerMap / copyCellTypeToPhysicalNodes (:267-319)
    std::map<unsigned int, unsigned int>& getCellTypeTrackerMap();
    void copyCellTypeToPhysicalNodes(std::map<unsigned int, unsigned int>& celltrackermap);
    void copyCellTypeToPhysicalNodes(unsigned int domainidentifier, unsigned int celltype);
    bool checkGeometryIntegrity(void) const { return geometry_.checkGeometryIntegrity(); }

    // --- not in the reference: the device simulation and its lattice snapshot
    void attach(lbib_handle* h);
    lbib_handle* handle() const { return h_; }
    void invalidate() const;           // the device moved on
    struct Snapshot;
    const Snapshot& snapshot() const;  // the lattice fields the views read
    int species(const std::string& name) const;

 private:
    const Geometry& geometry_;
    lbib_handle* h_;
    std::map<unsigned int, unsigned int> cellTypes_;
    bool cellTypesSet_;  // the application copied cell types (replayed when the simulation is built)
    mutable std::vector<nodes::PhysicalNode> views_;
    mutable std::vector<std::vector<nodes::PhysicalNode*>> grid_;
    mutable std::shared_ptr<Snapshot> snap_;
};

}  // namespace geometry
}  // namespace LbmLib

#endif
