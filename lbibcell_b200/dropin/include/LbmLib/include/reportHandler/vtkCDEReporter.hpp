// LbmLib::reportHandler::vtkCDEReporter (libs/LbmLib/include/reportHandler/vtkCDEReporter.hpp):
// the concentration of every CDE solver on the (coarsened) lattice (vtkCDEReporter.cpp).
// The constructor takes the reference's arguments; the data come from the
// running simulation at report time.
#ifndef LBIBCELL_DROPIN_VTKCDEREPORTER_HPP
#define LBIBCELL_DROPIN_VTKCDEREPORTER_HPP

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

class vtkCDEReporter : public AbstractReportFunctor {
 public:
    vtkCDEReporter(const std::vector<std::vector<nodes::PhysicalNode*>>& physicalNodes,
                   const unsigned int cdecoarseningfactor, const std::string& filename)
        : AbstractReportFunctor(filename), coarsening_(cdecoarseningfactor) {
        (void)physicalNodes;
    }
    virtual void operator()(unsigned int time) const { writeVtkBlock(filename_, time, 3, coarsening_); }

 private:
    unsigned int coarsening_;
};

}  // namespace reportHandler
}  // namespace LbmLib

#endif
