// LbmLib::SimulationRunner (libs/LbmLib/include/SimulationRunner.hpp:43-231):
// the time loop of SimulationRunner::runSimulation (SimulationRunner.cpp:72-110)
// on one GPU.  The runner builds the device simulation (liblbibcuda.so, the
// C ABI in include/lbibcell.h) from the parameter file, the geometry, the
// force file and the registered solvers:
//   * mass and bio solvers whose names the device runtime knows (the
//     reference's own and the configuration plugins) run on the device
//     inside the step;
//   * any other bio solver name is created through BioSolverFactory, as the
//     reference does, and its applyBioProcess runs on the host after each
//     device step, in registration order, against this library's
//     GeometryHandler and ForceSolver (they must be registered after the
//     device's bio solvers, whose step they follow);
//   * an unknown name throws std::bad_typeid (Factory.hpp:45-47).
// The lattice precision is FP64 unless LBIB_PRECISION=fp32 selects the
// FP32-shifted storage; LBIB_DEVICE selects the CUDA device; LBIB_PLUGIN_FILE
// names a plugin file (lbibcell_b200/configs.py) with the parameters of the
// configuration plugins and species, which the reference hard-codes.
#ifndef LBIBCELL_DROPIN_SIMULATIONRUNNER_HPP
#define LBIBCELL_DROPIN_SIMULATIONRUNNER_HPP

#include <LbmLib/include/Field.hpp>
#include <LbmLib/include/geometry/GeometryHandler.hpp>
#include <LbmLib/include/solver/BioSolver/BioAbstractSolver.hpp>
#include <LbmLib/include/solver/ForceSolver.hpp>

#include <memory>
#include <string>
#include <vector>

struct lbib_handle;

namespace LbmLib {
namespace geometry {
class GeometryHandler;
}
namespace reportHandler {
class ReportHandler;
}
namespace solver {
class BioAbstractSolver;
}

class SimulationRunner {
 public:
    SimulationRunner(const geometry::GeometryHandler& geometry, const reportHandler::ReportHandler& reportHandler);
    ~SimulationRunner();

    void runSimulation();
    // SimulationRunner::writeSimulation (SimulationRunner.cpp:112-149), with
    // 17 significant digits so that a restart continues with the same values
    void writeSimulation(const std::string& forceFileName, const std::string& geometryFileName,
                         const std::string& parameterFileName, const std::string& solverFileName);
    void initSolvers(Field<double> fluidVelocity);  // SimulationRunner.cpp:308-320
    void initSolvers();                             // SimulationRunner.cpp:290-306
    void initSolvers(const std::string& filename);  // SimulationRunner.cpp:151-182
    void addMassSolver(const std::string& name);
    void addBioSolver(const std::string& name);
    void initForceSolver(const std::string& fileName);
    const solver::ForceSolver& getForceSolver(void) { return forceSolver_; }

    // --- not in the reference: the device simulation (built on first need)
    lbib_handle* deviceHandle();

 private:
    void build();
    void requireDevice();
    void stepDevice(unsigned int n);
    void runHostBio();

    geometry::GeometryHandler& geometryHandler_;
    const reportHandler::ReportHandler& reportHandler_;
    solver::ForceSolver forceSolver_;
    std::vector<std::string> massSolvers_;
    std::vector<std::string> deviceBio_;
    std::vector<std::unique_ptr<solver::BioAbstractSolver>> hostBio_;
    lbib_handle* h_;
    bool configChanged_;  // solvers or forces registered since the device simulation was built
    // what was done to the lattice before the configuration changed, replayed
    // when the simulation is built again
    bool velocityInit_;
    Field<double> velocity_;
    std::string restartFile_;
    std::string workDir_;
};

}  // namespace LbmLib

#endif
