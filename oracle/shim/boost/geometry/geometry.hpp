// Minimal stand-in for the Boost.Geometry symbols that the LBIBCell sources
// name (oracle/_ref reference build only; Boost is not installed here).
// Only what the lattice hot path executes is functional: point_xy, an open
// counter-clockwise polygon, append/make and a shoelace area.  The R-tree and
// point-registration machinery are declared so the headers compile; the hot
// path never calls them.
#ifndef LBIB_SHIM_BOOST_GEOMETRY_HPP
#define LBIB_SHIM_BOOST_GEOMETRY_HPP
#include <cassert>
#include <cmath>
#include <iomanip>
#include <mutex>
#include <sstream>
#include <vector>

#define BOOST_GEOMETRY_REGISTER_POINT_2D_GET_SET(Point, Coord, Cs, Get0, Get1, Set0, Set1)

namespace boost {
namespace geometry {
namespace cs { struct cartesian {}; }
namespace index {
template <typename Value> struct indexable {};
}
namespace model {
namespace d2 {
template <typename T>
struct point_xy {
    T xv = 0, yv = 0;
    point_xy() {}
    point_xy(T a, T b) : xv(a), yv(b) {}
    T x() const { return xv; }
    T y() const { return yv; }
};
}  // namespace d2
template <typename T, std::size_t D, typename CS>
struct point {
    T v[D];
};
template <typename P, bool ClockWise = true, bool Closed = true>
struct polygon {
    std::vector<P> ring;
};
}  // namespace model

template <typename P>
P make(double x, double y) { return P(x, y); }

template <typename P, bool CW, bool CL>
void append(model::polygon<P, CW, CL>& poly, const P& p) { poly.ring.push_back(p); }

// Shoelace area over the ring in stored order (open ring: the closing edge
// is implied).  Counter-clockwise rings give a positive area.
template <typename P, bool CW, bool CL>
double area(const model::polygon<P, CW, CL>& poly) {
    const std::vector<P>& r = poly.ring;
    const std::size_t n = r.size();
    double sum = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        const std::size_t j = (i + 1 == n) ? 0 : i + 1;
        sum += r[i].x() * r[j].y() - r[j].x() * r[i].y();
    }
    return sum / 2.0;
}

template <typename A, typename B>
double distance(const A& a, const B& b) {
    return std::sqrt((a.x() - b.x()) * (a.x() - b.x()) + (a.y() - b.y()) * (a.y() - b.y()));
}
}  // namespace geometry
}  // namespace boost
#endif
