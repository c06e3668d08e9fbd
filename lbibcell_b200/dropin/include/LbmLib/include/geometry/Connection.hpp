// LbmLib::geometry::Connection (libs/LbmLib/include/geometry/Connection.hpp):
// a membrane connection from its first to its second node, with the cell's
// domain id and the boundary-condition descriptor of its geometry-file line.
#ifndef LBIBCELL_DROPIN_CONNECTION_HPP
#define LBIBCELL_DROPIN_CONNECTION_HPP

#include <LbmLib/include/nodes/GeometryNode.hpp>

#include <cmath>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace LbmLib {
namespace geometry {

class Connection {
 public:
    typedef std::map<std::string, std::vector<std::string>> Descriptor;
    Connection(std::shared_ptr<nodes::GeometryNode> p1, std::shared_ptr<nodes::GeometryNode> p2,
               const Descriptor& descriptor, unsigned int domainIdentifier)
        : nodes_(p1, p2), descriptor_(descriptor), domain_(domainIdentifier) {}

    const std::pair<std::shared_ptr<nodes::GeometryNode> const, std::shared_ptr<nodes::GeometryNode> const>
    getGeometryNodes() const {
        return std::pair<std::shared_ptr<nodes::GeometryNode> const, std::shared_ptr<nodes::GeometryNode> const>(
            nodes_.first, nodes_.second);
    }
    double getLength() const {
        const double dx = nodes_.first->getXPos() - nodes_.second->getXPos();
        const double dy = nodes_.first->getYPos() - nodes_.second->getYPos();
        return std::sqrt(dx * dx + dy * dy);
    }
    unsigned int getDomainIdentifier() const { return domain_; }
    const Descriptor getBoundaryConditionDescriptor() const { return descriptor_; }
    void setDomainIdentifier(const unsigned int domainIdentifier) { domain_ = domainIdentifier; }

 private:
    std::pair<std::shared_ptr<nodes::GeometryNode>, std::shared_ptr<nodes::GeometryNode>> nodes_;
    Descriptor descriptor_;
    unsigned int domain_;
};

}  // namespace geometry
}  // namespace LbmLib

#endif
