// LbmLib::Parameters (libs/LbmLib/include/GlobalSimulationParameters.hpp):
// the global parameter file's values.  The runner reads them when it builds
// the device simulation and advances the current iteration after each step.
#ifndef LBIBCELL_DROPIN_GLOBALSIMULATIONPARAMETERS_HPP
#define LBIBCELL_DROPIN_GLOBALSIMULATIONPARAMETERS_HPP

#include <UtilLib/include/Singleton.hpp>

#include <map>
#include <string>

namespace LbmLib {

class GlobalSimulationParameters_ {
 public:
    GlobalSimulationParameters_();
    // GlobalSimulationParameters.cpp:34-72: "Key:\tvalue" lines, CDESolvers:
    // followed by name tau pairs; lines starting with # are comments
    void loadGlobalSimulationParameters(const std::string& fileName);
    void writeGlobalSimulationParameters(const std::string& fileName) const;
    void printParameters() const;

    unsigned int getCurrentIteration() const { return currentIteration_; }
    unsigned int getIterations() const { return iterations_; }
    unsigned int getReportSteps() const { return reportSteps_; }
    void setReportSteps(unsigned int steps) { reportSteps_ = steps; }
    double getTauFluid() const { return tauFluid_; }
    unsigned int getSizeX() const { return sizeX_; }
    unsigned int getSizeY() const { return sizeY_; }
    const std::map<std::string, double>& getCdeSolvers() const { return cdeSolvers_; }
    unsigned int operator++(int) { return currentIteration_++; }

    // not in the reference: the file the values came from ("" if none)
    const std::string& sourceFile() const { return file_; }

 private:
    unsigned int currentIteration_, iterations_, reportSteps_, sizeX_, sizeY_;
    double tauFluid_;
    std::map<std::string, double> cdeSolvers_;
    std::string file_;
};

typedef UtilLib::Singleton<GlobalSimulationParameters_> globalSimulationParametersSingleton_;

static GlobalSimulationParameters_& Parameters = globalSimulationParametersSingleton_::instance();

}  // namespace LbmLib

#endif
