// LbmLib::nodes::GeometryNode (libs/LbmLib/include/nodes/GeometryNode.hpp):
// a membrane node as host plugins see it.  The node lives on the device;
// this object mirrors its id, position, velocity, force and its two
// connections (incoming [0], outgoing [1]).  The mirror is refreshed from the
// device before host plugins and reporters run; a position set here is sent
// back to the device after the plugin returns.
#ifndef LBIBCELL_DROPIN_GEOMETRYNODE_HPP
#define LBIBCELL_DROPIN_GEOMETRYNODE_HPP

#include <LbmLib/include/Field.hpp>
#include <LbmLib/include/GlobalSimulationParameters.hpp>
#include <UtilLib/include/Exception.hpp>
#include <UtilLib/include/Log.hpp>

#include <array>
#include <memory>
#include <string>

namespace LbmLib {
namespace geometry {
class Connection;
class Geometry;
}  // namespace geometry
namespace nodes {

class GeometryNode {
 public:
    GeometryNode(double x, double y, unsigned int id) : pos_(x, y), id_(id), owner_(nullptr) {}
    virtual ~GeometryNode() {}

    unsigned int getId() const { return id_; }
    double getXPos() const { return pos_.x; }
    double getYPos() const { return pos_.y; }
    Field<double> getPos() const { return pos_; }
    double getXVelocity() const { return vel_.x; }
    double getYVelocity() const { return vel_.y; }
    Field<double> getVelocity() const { return vel_; }
    Field<double> getForce() const { return force_; }
    virtual std::string getType() const { return "GeometryNode"; }

    // LagrangianPoint::setPos: the device node takes the position after the
    // plugin call (GeometryNode::isUpdateNeeded then decides the rebinding)
    virtual void setPos(double x, double y);
    void setXPos(double x) { setPos(x, pos_.y); }
    void setYPos(double y) { setPos(pos_.x, y); }

    template <int Index>
    void setConnection(const std::shared_ptr<geometry::Connection> connection) {
        connections_[Index] = connection;
    }
    template <int Index>
    const std::shared_ptr<geometry::Connection> getConnection() const {
        return connections_[Index];
    }
    // the domain of the adjacent connections (GeometryNode.cpp:273-286)
    unsigned int getDomainIdOfAdjacentConnections() const;

    // mirror bookkeeping (not in the reference)
    void mirrorState(double x, double y, double vx, double vy, double fx, double fy) {
        pos_ = Field<double>(x, y);
        vel_ = Field<double>(vx, vy);
        force_ = Field<double>(fx, fy);
    }
    void setOwner(geometry::Geometry* owner) { owner_ = owner; }

 private:
    Field<double> pos_, vel_, force_;
    unsigned int id_;
    geometry::Geometry* owner_;
    std::array<std::shared_ptr<geometry::Connection>, 2> connections_;
};

}  // namespace nodes
}  // namespace LbmLib

#endif
