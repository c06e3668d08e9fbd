// LbmLib::reportHandler::ReportHandler (libs/LbmLib/include/reportHandler/ReportHandler.hpp,
// ReportHandler.cpp:31-56): the registered reporters, called every
// reportStep-th time.
#ifndef LBIBCELL_DROPIN_REPORTHANDLER_HPP
#define LBIBCELL_DROPIN_REPORTHANDLER_HPP

#include <LbmLib/include/reportHandler/AbstractReportFunctor.hpp>

#include <memory>
#include <vector>

namespace LbmLib {
namespace reportHandler {

class ReportHandler {
 public:
    explicit ReportHandler(unsigned int reportStep = 1) : reportStep_(reportStep ? reportStep : 1) {}
    void registerReporter(std::unique_ptr<AbstractReportFunctor> reporter) {
        reporters_.push_back(std::move(reporter));
    }
    void writeReport(unsigned int time) const {
        if (time % reportStep_ == 0) writeCrashReport(time);
    }
    void writeCrashReport(unsigned int time) const {
        for (const auto& r : reporters_) (*r)(time);
    }

 private:
    unsigned int reportStep_;
    std::vector<std::unique_ptr<AbstractReportFunctor>> reporters_;
};

}  // namespace reportHandler
}  // namespace LbmLib

#endif
