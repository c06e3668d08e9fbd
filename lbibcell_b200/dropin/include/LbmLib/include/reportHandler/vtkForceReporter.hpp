// LbmLib::reportHandler::vtkForceReporter (libs/LbmLib/include/reportHandler/vtkForceReporter.hpp):
// forces: one line per force with a partner node, and its type (vtkForceReporter.cpp).
// The constructor takes the reference's arguments; the data come from the
// running simulation at report time.
#ifndef LBIBCELL_DROPIN_VTKFORCEREPORTER_HPP
#define LBIBCELL_DROPIN_VTKFORCEREPORTER_HPP

#include <LbmLib/include/geometry/Connection.hpp>
#include <LbmLib/include/nodes/GeometryNode.hpp>
#include <LbmLib/include/nodes/PhysicalNode.hpp>
#include <LbmLib/include/reportHandler/AbstractReportFunctor.hpp>
#include <LbmLib/include/reportHandler/vtkReporterBlock.hpp>
#include <LbmLib/include/solver/ForceSolver.hpp>

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace LbmLib {
namespace reportHandler {

class vtkForceReporter : public AbstractReportFunctor {
 public:
    vtkForceReporter(const std::map<unsigned int, std::shared_ptr<nodes::GeometryNode>>& geometryNodes,
                     const solver::ForceSolver& forcesolver, const std::string& filename)
        : AbstractReportFunctor(filename) {
        (void)geometryNodes;
        (void)forcesolver;
    }
    virtual void operator()(unsigned int time) const { writeVtkBlock(filename_, time, 2, 1); }
};

}  // namespace reportHandler
}  // namespace LbmLib

#endif
