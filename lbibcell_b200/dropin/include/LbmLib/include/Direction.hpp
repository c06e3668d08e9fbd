// LbmLib::Direction (libs/LbmLib/include/Direction.hpp:34-44): the lattice
// directions in the reference's order.
#ifndef LBIBCELL_DROPIN_DIRECTION_HPP
#define LBIBCELL_DROPIN_DIRECTION_HPP

namespace LbmLib {
enum Direction { T, E, N, W, S, NE, NW, SW, SE };
}

#endif
