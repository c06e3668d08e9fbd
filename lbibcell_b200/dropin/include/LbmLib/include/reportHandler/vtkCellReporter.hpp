// LbmLib::reportHandler::vtkCellReporter (libs/LbmLib/include/reportHandler/vtkCellReporter.hpp):
// cells: the membrane polygons with domain_identifier, cell_type and boundarydescriptors (vtkCellReporter.cpp).
// The constructor takes the reference's arguments; the data come from the
// running simulation at report time.
#ifndef LBIBCELL_DROPIN_VTKCELLREPORTER_HPP
#define LBIBCELL_DROPIN_VTKCELLREPORTER_HPP

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

class vtkCellReporter : public AbstractReportFunctor {
 public:
    vtkCellReporter(const std::vector<std::shared_ptr<geometry::Connection>>& connections,
                    const std::map<unsigned int, unsigned int>& celltypetrackermap, const std::string& filename)
        : AbstractReportFunctor(filename) {
        (void)connections;
        (void)celltypetrackermap;
    }
    virtual void operator()(unsigned int time) const { writeVtkBlock(filename_, time, 1, 1); }
};

}  // namespace reportHandler
}  // namespace LbmLib

#endif
