// The VTK XML writers behind the vtk*Reporter classes: each reporter adds
// its block to <filename>_<time>.vtm for the simulation that is running
// (the one SimulationRunner is stepping or reporting), written by the
// device runtime without VTK (lbib_write_vtk).  Not a reference header.
#ifndef LBIBCELL_DROPIN_VTKREPORTERBLOCK_HPP
#define LBIBCELL_DROPIN_VTKREPORTERBLOCK_HPP

#include <string>

namespace LbmLib {
namespace reportHandler {
// kind: 1 cells, 2 forces, 3 CDE fields, 4 fluid fields, 5 cell PNG (no graphics stack: nothing written)
void writeVtkBlock(const std::string& filename, unsigned int time, int kind, unsigned int coarsening);
}  // namespace reportHandler
}  // namespace LbmLib

#endif
