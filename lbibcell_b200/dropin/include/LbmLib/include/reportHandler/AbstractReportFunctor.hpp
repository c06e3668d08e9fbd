// LbmLib::reportHandler::AbstractReportFunctor (libs/LbmLib/include/reportHandler/AbstractReportFunctor.hpp).
#ifndef LBIBCELL_DROPIN_ABSTRACTREPORTFUNCTOR_HPP
#define LBIBCELL_DROPIN_ABSTRACTREPORTFUNCTOR_HPP

#include <string>

namespace LbmLib {
namespace reportHandler {

class AbstractReportFunctor {
 public:
    explicit AbstractReportFunctor(const std::string& filename) : filename_(filename) {}
    virtual ~AbstractReportFunctor() {}
    virtual void operator()(unsigned int time) const = 0;

 protected:
    const std::string filename_;
};

}  // namespace reportHandler
}  // namespace LbmLib

#endif
