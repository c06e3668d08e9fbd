// LbmLib::reportHandler::vtkFluidReporter (libs/LbmLib/include/reportHandler/vtkFluidReporter.hpp):
// density and velocity on the (coarsened) lattice (vtkFluidReporter.cpp:44-106).
// The constructor takes the reference's arguments; the data come from the
// running simulation at report time.
#ifndef LBIBCELL_DROPIN_VTKFLUIDREPORTER_HPP
#define LBIBCELL_DROPIN_VTKFLUIDREPORTER_HPP

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

class vtkFluidReporter : public AbstractReportFunctor {
 public:
    vtkFluidReporter(const std::vector<std::vector<nodes::PhysicalNode*>>& physicalNodes,
                     const unsigned int cdecoarseningfactor, const std::string& filename)
        : AbstractReportFunctor(filename), coarsening_(cdecoarseningfactor) {
        (void)physicalNodes;
    }
    virtual void operator()(unsigned int time) const { writeVtkBlock(filename_, time, 4, coarsening_); }

 private:
    unsigned int coarsening_;
};

}  // namespace reportHandler
}  // namespace LbmLib

#endif
