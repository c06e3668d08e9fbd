// Stand-in header (oracle/_ref reference build only).
#include <boost/geometry/geometry.hpp>
