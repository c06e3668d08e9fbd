// LbmLib::solver::BioAbstractSolver (libs/LbmLib/include/solver/BioSolver/BioAbstractSolver.hpp):
// the interface of a bio solver plugin.
#ifndef LBIBCELL_DROPIN_BIOABSTRACTSOLVER_HPP
#define LBIBCELL_DROPIN_BIOABSTRACTSOLVER_HPP

#include <string>

namespace LbmLib {
namespace geometry {
class GeometryHandler;
}
namespace solver {
class ForceSolver;

class BioAbstractSolver {
 public:
    virtual ~BioAbstractSolver() {}
    virtual void applyBioProcess(geometry::GeometryHandler& geometryhandler, solver::ForceSolver& forcesolver) = 0;
    virtual std::string getName() = 0;
};

}  // namespace solver
}  // namespace LbmLib

#endif
