// LbmLib::geometry::Geometry (libs/LbmLib/include/geometry/Geometry.hpp):
// the membrane read from a geometry file (.txt, or .vtm as written by the
// cell reporter).  Once a simulation runs, the nodes and connections live on
// the device; the maps returned here are a host mirror, refreshed from the
// device when a host plugin or reporter asks for them, and edits made through
// GeometryHandler are sent back after the plugin call.
#ifndef LBIBCELL_DROPIN_GEOMETRY_HPP
#define LBIBCELL_DROPIN_GEOMETRY_HPP

#include <LbmLib/include/geometry/Connection.hpp>
#include <LbmLib/include/nodes/GeometryNode.hpp>

#include <map>
#include <memory>
#include <string>
#include <vector>

struct lbib_handle;

namespace LbmLib {
namespace geometry {

class Geometry {
 public:
    explicit Geometry(const std::string& filename);
    ~Geometry();

    // Geometry::writeGeometry (Geometry.cpp:77-95)
    void writeGeometry(const std::string& fileName) const;
    const std::map<unsigned int, std::shared_ptr<nodes::GeometryNode>>& getGeometryNodes() const;
    const std::vector<std::shared_ptr<Connection>>& getConnections() const;

    // range queries in the reference's cell-list order (Geometry.cpp:306-374);
    // they run on the device and need a running simulation
    const std::vector<std::shared_ptr<nodes::GeometryNode>> getGeometryNodesWithinRadius(const double x,
                                                                                          const double y,
                                                                                          const double radius) const;
    const std::vector<std::shared_ptr<nodes::GeometryNode>> getGeometryNodesWithinRadiusWithAvoidance(
        const double x, const double y, const double radius, const unsigned int domainIdentifier) const;
    std::shared_ptr<nodes::GeometryNode> getGeometryNodesWithinRadiusWithAvoidanceClosest(
        const double x, const double y, const double radius, const unsigned int domainIdentifier) const;

    // topology edits (Geometry.cpp:381-452): applied to the mirror, sent to the
    // device after the plugin call
    unsigned int addGeometryNode(const double x, const double y);
    unsigned int removeGeometryNode(const unsigned int nodeid);
    void eraseConnection(std::shared_ptr<Connection> toDelete);
    void addConnection(std::shared_ptr<nodes::GeometryNode> p1, std::shared_ptr<nodes::GeometryNode> p2,
                       const std::map<std::string, std::vector<std::string>>& descriptor,
                       const unsigned int domainIdentifier);
    bool checkGeometryIntegrity() const;
    // every connection's domain with cell type 1 and domain 0 with type 0
    std::map<unsigned int, unsigned int> getCellTypeTrackerMap(void) const;

    // --- not in the reference: the link to the device simulation
    const std::string& sourceFile() const { return file_; }
    void attach(lbib_handle* h) const;      // the running simulation, or nullptr
    void invalidate() const { stale_ = true; }   // the device moved on: refresh before the next read
    void markEdited() const { edited_ = true; }
    bool edited() const { return edited_; }
    void pushEdits() const;                 // send the mirror's topology and positions to the device

 private:
    void load(const std::string& filename);
    void refresh() const;
    std::shared_ptr<nodes::GeometryNode> mirrorNode(unsigned int id, double x, double y) const;

    std::string file_;
    mutable lbib_handle* h_;
    mutable bool stale_, edited_;
    mutable std::map<unsigned int, std::shared_ptr<nodes::GeometryNode>> nodes_;
    mutable std::vector<std::shared_ptr<Connection>> connections_;
    // boundary-condition descriptors by (first id, second id), from the file;
    // a connection a plugin creates carries the one it was given
    mutable std::map<std::pair<unsigned int, unsigned int>, Connection::Descriptor> descriptors_;
};

}  // namespace geometry
}  // namespace LbmLib

#endif
