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

// Point registration: records the two getters, so that distance() works on a
// registered type (the cell-division plugins measure GeometryNode distances).
namespace boost {
namespace geometry {
namespace lbib_traits {
template <typename P>
struct access {};
}  // namespace lbib_traits
}  // namespace geometry
}  // namespace boost
#define BOOST_GEOMETRY_REGISTER_POINT_2D_GET_SET(Point, Coord, Cs, Get0, Get1, Set0, Set1)   \
    namespace boost {                                                                    \
    namespace geometry {                                                                 \
    namespace lbib_traits {                                                              \
    template <>                                                                          \
    struct access<Point> {                                                               \
        static Coord x(const Point& p) { return p.Get0(); }                             \
        static Coord y(const Point& p) { return p.Get1(); }                             \
    };                                                                                   \
    }                                                                                    \
    }                                                                                    \
    }

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
    template <std::size_t I>
    T get() const { return v[I]; }
    template <std::size_t I>
    void set(T a) { v[I] = a; }
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

// Coordinates of a point: a registered type through its getters, point_xy
// through x() / y().
template <typename P>
auto coord_x(const P& p, int) -> decltype(lbib_traits::access<P>::x(p)) { return lbib_traits::access<P>::x(p); }
template <typename P>
auto coord_x(const P& p, long) -> decltype(p.x()) { return p.x(); }
template <typename P>
auto coord_y(const P& p, int) -> decltype(lbib_traits::access<P>::y(p)) { return lbib_traits::access<P>::y(p); }
template <typename P>
auto coord_y(const P& p, long) -> decltype(p.y()) { return p.y(); }

// Cartesian (Pythagoras) distance: the squared differences summed by
// dimension, then the root.
template <typename A, typename B>
double distance(const A& a, const B& b) {
    const double dx = coord_x(a, 0) - coord_x(b, 0), dy = coord_y(a, 0) - coord_y(b, 0);
    return std::sqrt(dx * dx + dy * dy);
}
}  // namespace geometry
}  // namespace boost
#endif
