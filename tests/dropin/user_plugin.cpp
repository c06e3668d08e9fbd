// A user bio solver written against LBIBCell's plugin API
// (libs/LbmLib/include/solver/BioSolver/BioBaseSolver.hpp), of the kind an
// application adds without changing the library.  TEST INFRASTRUCTURE: the
// same source is compiled into the reference build (oracle/Makefile) and
// into an application linked against lbibcell_b200's drop-in libLbmLib, where
// the device does not know the solver and runs it on the host between steps.
//
// UserPullSolver: every 5th iteration it drops the type-2 forces, then pulls
// the nodes of each cell that lie right of the cell's mean x outward with a
// constant force proportional to their distance from the mean, scaled down
// as the cell's area grows past its first area (computeAreas).
#include <LbmLib/include/GlobalSimulationParameters.hpp>
#include <LbmLib/include/geometry/GeometryHandler.hpp>
#include <LbmLib/include/nodes/GeometryNode.hpp>
#include <LbmLib/include/solver/BioSolver/BioBaseSolver.hpp>
#include <LbmLib/include/solver/ForceSolver.hpp>

#include <map>
#include <sstream>
#include <string>

namespace LbmLib {
namespace solver {

class UserPullSolver : public BioBaseSolver<UserPullSolver> {
 public:
    UserPullSolver();
    virtual void applyBioProcess(geometry::GeometryHandler& gh, solver::ForceSolver& fs) {
        if (Parameters.getCurrentIteration() % 5 != 0) return;
        fs.deleteForceType(2);
        const std::map<unsigned int, double> areas = gh.computeAreas();
        std::map<unsigned int, double> sumX, count;
        for (const auto& kv : gh.getGeometry().getGeometryNodes()) {
            const unsigned int d = kv.second->getDomainIdOfAdjacentConnections();
            sumX[d] += kv.second->getXPos();
            count[d] += 1.0;
        }
        std::stringstream line;
        for (const auto& kv : gh.getGeometry().getGeometryNodes()) {
            const auto& n = kv.second;
            const unsigned int d = n->getDomainIdOfAdjacentConnections();
            const double cx = sumX[d] / count[d];
            if (first_.find(d) == first_.end()) first_[d] = areas.at(d);
            const double scale = first_[d] / areas.at(d);
            if (n->getXPos() <= cx) continue;
            line.str(std::string());
            line.clear();
            line << "2\t" << n->getId() << "\t" << 1e-4 * scale * (n->getXPos() - cx) << "\t" << 0.0;
            fs.addForce(&line);
        }
    }
    static const std::string name;

 private:
    std::map<unsigned int, double> first_;
};

const std::string UserPullSolver::name = "UserPullSolver";
UserPullSolver::UserPullSolver() : BioBaseSolver() {}

}  // namespace solver
}  // namespace LbmLib
