// LbmLib::reportHandler::vtkCellPNGReporter (libs/LbmLib/include/reportHandler/vtkCellPNGReporter.hpp):
// a PNG picture of the cells through VTK's rendering (vtkCellPNGReporter.cpp:38-43,70-72); no graphics stack here: writes nothing.
// The constructor takes the reference's arguments; the data come from the
// running simulation at report time.
#ifndef LBIBCELL_DROPIN_VTKCELLPNGREPORTER_HPP
#define LBIBCELL_DROPIN_VTKCELLPNGREPORTER_HPP

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

class vtkCellPNGReporter : public AbstractReportFunctor {
 public:
    vtkCellPNGReporter(const std::vector<std::shared_ptr<geometry::Connection>>& connections,
                       const std::string& filename)
        : AbstractReportFunctor(filename) {
        (void)connections;
    }
    virtual void operator()(unsigned int time) const { writeVtkBlock(filename_, time, 5, 1); }
};

}  // namespace reportHandler
}  // namespace LbmLib

#endif
