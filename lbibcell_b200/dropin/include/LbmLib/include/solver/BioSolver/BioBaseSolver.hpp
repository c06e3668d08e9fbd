// LbmLib::solver::BioBaseSolver<T> (libs/LbmLib/include/solver/BioSolver/BioBaseSolver.hpp:45-96):
// derive a plugin T from it, give T a `static const std::string name` and a
// constructor that calls this one: T registers itself under its name at
// static-initialisation time, and SimulationRunner::addBioSolver(name)
// creates it.  Plugins registered this way run on the host after the device
// step, in registration order; the names of the reference's own solvers run
// on the device.
#ifndef LBIBCELL_DROPIN_BIOBASESOLVER_HPP
#define LBIBCELL_DROPIN_BIOBASESOLVER_HPP

#include <LbmLib/include/solver/BioSolver/BioSolverFactory.hpp>

#include <string>

namespace LbmLib {
namespace solver {

template <class T>
struct BioBaseSolver : BioAbstractSolver {
 public:
    std::string getName() { return T::name; }

 protected:
    BioBaseSolver() { reg = reg; }  // instantiates the registration below
    virtual ~BioBaseSolver() {}
    static BioAbstractSolver* create() { return new T; }
    static bool reg;
    static bool init() { return BioSolverFactory::instance().registerType(T::name, BioBaseSolver::create); }
};

template <class T>
bool BioBaseSolver<T>::reg = BioBaseSolver<T>::init();

}  // namespace solver
}  // namespace LbmLib

#endif
