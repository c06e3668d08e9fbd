// Parameters of the lbibcell_b200 configuration plugins in the reference
// build (oracle/_ref).  TEST INFRASTRUCTURE ONLY.
#ifndef LBIB_REF_REGISTRY_HPP
#define LBIB_REF_REGISTRY_HPP
#include <map>
#include <string>

namespace lbibref {
struct CdeParams {
    double init = 0.0;
    double decay = 0.0;
    std::map<unsigned int, double> source;
};
struct TensionParams { double force = 0.01; unsigned int frequency = 10; };
struct AreaParams { double factor = 1.2; double strength = 0.01; double maxsource = 0.004; };
struct JunctionParams { double radius = 1.0; double k = 0.02; double l0 = 0.5; };
struct DivisionParams { double factor = 2.0; unsigned int frequency = 100; };
struct Registry {
    std::map<std::string, CdeParams> cde;
    TensionParams tension;
    AreaParams area;
    JunctionParams junction;
    DivisionParams division;
    long long diagonalReinit = 0;
    long long failedReinit = 0;
};
Registry& registry();
}  // namespace lbibref
#endif
