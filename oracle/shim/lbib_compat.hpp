// Force-included into every reference translation unit of the oracle/_ref
// build.  It supplies what older standard libraries pulled in transitively
// (<cstring>, <algorithm>, <random>) and the stream-to-stream insertion that pre-C++11
// libraries accepted through the void* conversion; the message text is
// written instead of a pointer value.
#ifndef LBIB_COMPAT_HPP
#define LBIB_COMPAT_HPP
#include <algorithm>
#include <cstring>
#include <ostream>
#include <random>
#include <sstream>
// Declared in namespace std so that argument-dependent lookup finds it from
// inside the reference's namespaces, which declare operator<< of their own.
namespace std {
inline ostream& operator<<(ostream& os, const stringstream& ss) { return os << ss.str(); }
}
#endif
