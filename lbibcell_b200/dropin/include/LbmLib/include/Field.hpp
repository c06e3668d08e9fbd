// LbmLib::Field (libs/LbmLib/include/Field.hpp): a 2-vector with the
// arithmetic plugins use (positions, velocities, forces).
#ifndef LBIBCELL_DROPIN_FIELD_HPP
#define LBIBCELL_DROPIN_FIELD_HPP

namespace LbmLib {

template <class T>
struct Field {
    T x, y;
    Field() : x(0), y(0) {}
    Field(T x_, T y_) : x(x_), y(y_) {}
    Field& operator+=(const Field& o) { x += o.x; y += o.y; return *this; }
    Field& operator-=(const Field& o) { x -= o.x; y -= o.y; return *this; }
    Field& operator*=(T s) { x *= s; y *= s; return *this; }
    Field& operator/=(T s) { x /= s; y /= s; return *this; }
    Field operator+(const Field& o) const { return Field(x + o.x, y + o.y); }
    Field operator-(const Field& o) const { return Field(x - o.x, y - o.y); }
    Field operator*(T s) const { return Field(x * s, y * s); }
    Field operator/(T s) const { return Field(x / s, y / s); }
};

template <class T>
Field<T> operator*(T s, const Field<T>& f) { return Field<T>(s * f.x, s * f.y); }

}  // namespace LbmLib

#endif
