// An application written against LBIBCell's API, as apps/tutorial_01.cpp is,
// linked against lbibcell_b200's drop-in libLbmLib.  TEST INFRASTRUCTURE:
// it runs the configuration given on the command line and, at every report
// step, writes the state in the binary dump format of oracle/ref_driver.cpp
// (read by oracle/oracle.py read_dump), so that the run compares with the
// reference build's bit for bit.
//
//   dropin_app parameters geometry force plugins outdir
//
// The plugin file's "MassSolver <name>" and "BioSolver <name>" lines are
// registered by name, in file order (their parameters, if any, are ignored:
// the reference's addBioSolver takes a name only).
#include <LbmLib/include/GlobalSimulationParameters.hpp>
#include <LbmLib/include/SimulationRunner.hpp>
#include <LbmLib/include/geometry/Geometry.hpp>
#include <LbmLib/include/geometry/GeometryHandler.hpp>
#include <LbmLib/include/reportHandler/AbstractReportFunctor.hpp>
#include <LbmLib/include/reportHandler/ReportHandler.hpp>

#include <lbibcell.h>

#include <cstdint>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace {

class DeviceDump : public LbmLib::reportHandler::AbstractReportFunctor {
 public:
    DeviceDump(LbmLib::SimulationRunner& runner, const std::string& dir)
        : AbstractReportFunctor(dir), runner_(runner) {}

    void operator()(unsigned int time) const override {
        lbib_handle* h = runner_.deviceHandle();
        long long sz[10];
        lbib_get_sizes(h, sz);
        const int64_t nx = sz[0], ny = sz[1], S = sz[2], M = sz[3], C = sz[4];
        const size_t L = (size_t)nx * ny;
        std::vector<double> f(9 * L), g(5 * L * (S ? S : 1)), vel(2 * L), force(2 * L), node(6 * M);
        std::vector<unsigned> dom(L), ctype(L), ids(M), conn(3 * C);
        lbib_download_lattice(h, f.data(), S ? g.data() : nullptr, vel.data(), force.data(), dom.data(), ctype.data());
        lbib_download_membrane(h, ids.data(), node.data());
        lbib_download_connections(h, conn.data());
        std::ofstream out(filename_ + "/dump_" + std::to_string(time) + ".bin", std::ios::binary);
        const int64_t hdr[8] = {0x4c424942, (int64_t)time, nx, ny, S, M, C,
                                (int64_t)LbmLib::Parameters.getCurrentIteration()};
        out.write((const char*)hdr, sizeof hdr);
        out.write((const char*)f.data(), sizeof(double) * f.size());
        out.write((const char*)g.data(), sizeof(double) * 5 * L * S);
        out.write((const char*)vel.data(), sizeof(double) * vel.size());
        out.write((const char*)force.data(), sizeof(double) * force.size());
        out.write((const char*)dom.data(), sizeof(unsigned) * dom.size());
        out.write((const char*)ctype.data(), sizeof(unsigned) * ctype.size());
        out.write((const char*)ids.data(), sizeof(unsigned) * ids.size());
        out.write((const char*)node.data(), sizeof(double) * node.size());
        out.write((const char*)conn.data(), sizeof(unsigned) * conn.size());
        const int64_t counters[2] = {0, 0};
        out.write((const char*)counters, sizeof counters);
    }

 private:
    LbmLib::SimulationRunner& runner_;
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 6) {
        std::cerr << "usage: dropin_app parameters geometry force plugins outdir\n";
        return 2;
    }
    try {
        LbmLib::Parameters.loadGlobalSimulationParameters(argv[1]);
        LbmLib::geometry::Geometry geo(argv[2]);
        LbmLib::geometry::GeometryHandler geohandler(geo);
        LbmLib::reportHandler::ReportHandler reporter(LbmLib::Parameters.getReportSteps());
        LbmLib::SimulationRunner simRunner(geohandler, reporter);
        reporter.registerReporter(std::unique_ptr<LbmLib::reportHandler::AbstractReportFunctor>(
            new DeviceDump(simRunner, argv[5])));
        simRunner.initSolvers();
        simRunner.initForceSolver(argv[3]);
        std::ifstream in(argv[4]);
        std::string line;
        while (std::getline(in, line)) {
            if (line.empty() || line[0] == '#') continue;
            std::stringstream ls(line);
            std::string kind, name;
            ls >> kind >> name;
            if (kind == "MassSolver") simRunner.addMassSolver(name);
            else if (kind == "BioSolver") simRunner.addBioSolver(name);
        }
        simRunner.runSimulation();
    } catch (const std::exception& e) {
        std::cerr << "dropin_app failed: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
