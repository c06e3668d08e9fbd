// LbmLib::solver::ForceSolver (libs/LbmLib/include/solver/ForceSolver.hpp):
// the force list of the membrane nodes.  The list lives on the device and
// the device evaluates it every step; this object takes host plugins' edits
// in the reference's text format and forwards them in order (records added
// within one plugin call go to the device together, before any delete and
// before the call returns).
#ifndef LBIBCELL_DROPIN_FORCESOLVER_HPP
#define LBIBCELL_DROPIN_FORCESOLVER_HPP

#include <sstream>
#include <string>
#include <vector>

struct lbib_handle;

namespace LbmLib {
namespace solver {

class ForceSolver {
 public:
    ForceSolver() : h_(nullptr) {}
    // ForceSolver::loadForceFile (ForceSolver.cpp:87-105): the file is read
    // when the simulation is built
    void loadForceFile(const std::string& filename) { file_ = filename; }
    // ForceSolver::addForce (ForceSolver.cpp:107-139): "type id1 [id2] parameters"
    void addForce(std::stringstream* const forcedescriptor);
    // ForceSolver::writeForceSolver (ForceSolver.cpp:141-156)
    void writeForceSolver(const std::string& filename) const;
    void deleteAllForces();
    void deleteForceType(const unsigned int forcetype);

    // --- not in the reference
    const std::string& forceFile() const { return file_; }
    void attach(lbib_handle* h) { h_ = h; }
    void flush();  // sends the buffered records to the device

 private:
    lbib_handle* h_;
    std::string file_;
    std::vector<int> type_;
    std::vector<unsigned> id1_, id2_;
    std::vector<double> par_;
};

}  // namespace solver
}  // namespace LbmLib

#endif
