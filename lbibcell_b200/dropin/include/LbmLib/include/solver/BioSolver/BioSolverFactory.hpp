// The bio solvers' name registry (libs/LbmLib/include/solver/BioSolver/BioSolverFactory.hpp).
#ifndef LBIBCELL_DROPIN_BIOSOLVERFACTORY_HPP
#define LBIBCELL_DROPIN_BIOSOLVERFACTORY_HPP

#include <LbmLib/include/solver/BioSolver/BioAbstractSolver.hpp>
#include <UtilLib/include/Factory.hpp>
#include <UtilLib/include/Singleton.hpp>

#include <string>

namespace LbmLib {
namespace solver {
typedef UtilLib::Singleton<UtilLib::Factory<BioAbstractSolver, std::string>> BioSolverFactory;
}
}  // namespace LbmLib

#endif
