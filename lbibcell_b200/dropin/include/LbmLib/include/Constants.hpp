// Constants of LBIBCell (libs/LbmLib/include/Constants.hpp) that plugins use.
#ifndef LBIBCELL_DROPIN_CONSTANTS_HPP
#define LBIBCELL_DROPIN_CONSTANTS_HPP

#include <cmath>

namespace LbmLib {
const double PI = std::atan(1) * 4;
const double CS = 1.0 / std::sqrt(3.0);  // the lattice speed of sound
const double EPSILON = 1e-9;             // positions this close to a lattice line are perturbed
const double MAXLENGTH = 0.5;            // remeshing splits longer connections
const double MINLENGTH = 0.5;            // coarsening joins closer neighbours
}  // namespace LbmLib

#endif
