// ref_driver.cpp — runs the reference LBIBCell code (built into oracle/_ref by
// oracle/build_ref.sh) on a configuration and writes binary state dumps.
// TEST INFRASTRUCTURE ONLY.
//
// The application body follows apps/tutorial_01.cpp:38-152: parameters,
// Geometry(txt), GeometryHandler, ReportHandler, SimulationRunner, then
// initSolvers, initForceSolver, mass and bio solvers by name, runSimulation.
// A report functor (the reference's own reporter API,
// AbstractReportFunctor.hpp) dumps the state every ReportStep iterations.
//
// usage: ref_driver params.txt geometry.txt force.txt plugins.txt outdir
//                   [timing W K] [restart SOLVERFILE] [write PREFIX] [edit ITER FILE] [run N]
//                   [celltype DOMAIN TYPE]...
//   With "timing W K" no reporter is registered: runSimulation() runs W
//   untimed iterations, then K iterations whose wall time is printed as JSON
//   (the CPU baseline).  "restart SOLVERFILE" loads the distributions with
//   SimulationRunner::initSolvers(file) after initSolvers(); "write PREFIX"
//   calls SimulationRunner::writeSimulation at the end, into PREFIX_force.txt,
//   PREFIX_geometry.txt, PREFIX_parameters.txt and PREFIX_solver.txt.  "edit
//   ITER FILE" stops at iteration ITER, applies the topology edit in FILE
//   through GeometryHandler (applyEdit), cures the lattice and runs on.  "run N"
//   runs N iterations where the parameter file's Iterations count is larger
//   (the solvers' initSolver still sees the file's count).  "celltype D T"
//   sets the cell type of domain D in GeometryHandler's cell-type tracker map
//   and copies the map to the lattice (copyCellTypeToPhysicalNodes) after
//   initSolvers, as a host bio solver does.  The log
//   goes to outdir/log.txt as in apps/tutorial_01.cpp:47-57.
//
// Dump file outdir/dump_<t>.bin (little endian):
//   int64 hdr[8] = {0x4c424942, t, nx, ny, S, M, C, currentIteration}
//   f[L][9] double (reference slot convention), g[S][L][5] double,
//   vel[L][2] double, force[L][2] double, dom[L] u32, ctype[L] u32,
//   ids[M] u32, node[M][6] double (x, y, vx, vy, fx, fy), conn[C][3] u32,
//   int64 counters[2] = {diagonal reinit, failed reinit}

// Standard headers first, so that only the reference's own headers see the
// access override below.
#include <array>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <unordered_set>
#include <vector>
#include <omp.h>

// Reading the force_ members needs access past `private`, as the
// reference's own tests do (libs/UtilLib/test/geometry/FastNeighborList_test.cpp).
#define private public
#define protected public
#include <LbmLib/include/GlobalSimulationParameters.hpp>
#include <LbmLib/include/SimulationRunner.hpp>
#include <LbmLib/include/geometry/Connection.hpp>
#include <LbmLib/include/geometry/Geometry.hpp>
#include <LbmLib/include/geometry/GeometryHandler.hpp>
#include <LbmLib/include/nodes/GeometryNode.hpp>
#include <LbmLib/include/nodes/PhysicalNode.hpp>
#include <LbmLib/include/reportHandler/AbstractReportFunctor.hpp>
#include <LbmLib/include/reportHandler/ReportHandler.hpp>
#include <LbmLib/include/solver/CDESolver/CDEAbstractSolver.hpp>
#include <LbmLib/include/solver/FluidSolver/FluidSolver.hpp>
#include <UtilLib/include/Log.hpp>
#undef private
#undef protected

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>

#include "ref_registry.hpp"

namespace {

struct PluginList {
    bool outlet = false;
    std::vector<std::string> bio;
};

PluginList loadPlugins(const std::string& fn) {
    PluginList pl;
    std::ifstream in(fn);
    if (!in.is_open()) throw std::runtime_error("cannot open plugin file " + fn);
    std::string line;
    auto& reg = lbibref::registry();
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ls(line);
        std::string kind, name;
        ls >> kind >> name;
        if (kind == "MassSolver") {
            if (name == "MassSolverBoxOutlet") pl.outlet = true;
        } else if (kind == "BioSolver") {
            pl.bio.push_back(name);
            std::string k; double v;
            while (ls >> k >> v) {
                if (name == "LbibMembraneTension") {
                    if (k == "force") reg.tension.force = v;
                    if (k == "frequency") reg.tension.frequency = (unsigned)v;
                } else if (name == "LbibAreaRegulator") {
                    if (k == "factor") reg.area.factor = v;
                    if (k == "strength") reg.area.strength = v;
                    if (k == "maxsource") reg.area.maxsource = v;
                } else if (name == "LbibCellJunction") {
                    if (k == "radius") reg.junction.radius = v;
                    if (k == "k") reg.junction.k = v;
                    if (k == "l0") reg.junction.l0 = v;
                } else if (name == "LbibCellDivision") {
                    if (k == "factor") reg.division.factor = v;
                    if (k == "frequency") reg.division.frequency = (unsigned)v;
                }
            }
        } else if (kind == "CDE") {
            std::string k; double v;
            while (ls >> k >> v) {
                if (k == "init") reg.cde[name].init = v;
                if (k == "decay") reg.cde[name].decay = v;
            }
        } else if (kind == "CDESource") {
            unsigned d; double r;
            while (ls >> d >> r) reg.cde[name].source[d] = r;
        }
    }
    return pl;
}

class DumpReporter : public LbmLib::reportHandler::AbstractReportFunctor {
 public:
    DumpReporter(const LbmLib::geometry::GeometryHandler& gh, const std::string& dir)
        : AbstractReportFunctor(dir), gh_(gh) {}

    void operator()(unsigned int time) const override {
        using namespace LbmLib;
        const auto& grid = gh_.getPhysicalNodes();
        const int64_t ny = grid.size(), nx = grid[0].size();
        const int64_t S = grid[0][0]->getCDESolvers().size();
        const auto& nodes = gh_.getGeometry().getGeometryNodes();
        const auto& conns = gh_.getGeometry().getConnections();
        std::ofstream out(filename_ + "/dump_" + std::to_string(time) + ".bin", std::ios::binary);
        int64_t hdr[8] = {0x4c424942, (int64_t)time, nx, ny, S, (int64_t)nodes.size(), (int64_t)conns.size(),
                          (int64_t)Parameters.getCurrentIteration()};
        out.write((const char*)hdr, sizeof(hdr));
        std::vector<double> buf;
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x)
                for (int d = 0; d < 9; ++d)
                    buf.push_back(grid[y][x]->getFluidSolver().distributions_[d]);
        write(out, buf);
        for (int64_t k = 0; k < S; ++k)
            for (int64_t y = 0; y < ny; ++y)
                for (int64_t x = 0; x < nx; ++x)
                    for (int d = 0; d < 5; ++d)
                        buf.push_back(grid[y][x]->getCDESolver(k).accessDistribution((Direction)d));
        write(out, buf);
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                buf.push_back(grid[y][x]->getFluidSolver().velocity_.x);
                buf.push_back(grid[y][x]->getFluidSolver().velocity_.y);
            }
        write(out, buf);
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                buf.push_back(grid[y][x]->getFluidSolver().force_.x);
                buf.push_back(grid[y][x]->getFluidSolver().force_.y);
            }
        write(out, buf);
        std::vector<uint32_t> ub;
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) ub.push_back(grid[y][x]->getDomainIdentifier());
        writeU(out, ub);
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) ub.push_back(grid[y][x]->getCellType());
        writeU(out, ub);
        for (const auto& kv : nodes) ub.push_back(kv.first);
        writeU(out, ub);
        for (const auto& kv : nodes) {
            const auto& g = *kv.second;
            buf.push_back(g.getXPos()); buf.push_back(g.getYPos());
            buf.push_back(g.getXVelocity()); buf.push_back(g.getYVelocity());
            buf.push_back(g.force_.x); buf.push_back(g.force_.y);
        }
        write(out, buf);
        for (const auto& c : conns) {
            ub.push_back(c->getGeometryNodes().first->getId());
            ub.push_back(c->getGeometryNodes().second->getId());
            ub.push_back(c->getDomainIdentifier());
        }
        writeU(out, ub);
        int64_t cnt[2] = {lbibref::registry().diagonalReinit, lbibref::registry().failedReinit};
        out.write((const char*)cnt, sizeof(cnt));
    }

 private:
    static void write(std::ofstream& o, std::vector<double>& b) {
        o.write((const char*)b.data(), b.size() * sizeof(double));
        b.clear();
    }
    static void writeU(std::ofstream& o, std::vector<uint32_t>& b) {
        o.write((const char*)b.data(), b.size() * sizeof(uint32_t));
        b.clear();
    }
    const LbmLib::geometry::GeometryHandler& gh_;
};

}  // namespace

// A topology edit between steps, as a host bio solver (a cell division) makes
// it through GeometryHandler: lines "erase id1 id2" (eraseConnection), "node x
// y" (createGeometryNode, ids in order), "conn id1 id2 domain"
// (createConnection with no boundary descriptor), applied in file order.
void applyEdit(LbmLib::geometry::GeometryHandler& gh, const std::string& file) {
    std::ifstream in(file);
    if (!in.is_open()) throw std::runtime_error("cannot open edit file " + file);
    std::string line;
    while (std::getline(in, line)) {
        std::stringstream ls(line);
        std::string k;
        ls >> k;
        if (k == "erase") {
            unsigned a, b;
            ls >> a >> b;
            std::shared_ptr<LbmLib::geometry::Connection> hit;
            for (const auto& c : gh.getGeometry().getConnections())
                if (c->getGeometryNodes().first->getId() == a && c->getGeometryNodes().second->getId() == b) hit = c;
            if (!hit) throw std::runtime_error("edit: no connection to erase");
            gh.eraseConnection(hit);
        } else if (k == "node") {
            double x, y;
            ls >> x >> y;
            gh.createGeometryNode(x, y);
        } else if (k == "conn") {
            unsigned a, b, d;
            ls >> a >> b >> d;
            gh.createConnection(gh.returnGeometryNode(a), gh.returnGeometryNode(b),
                                std::map<std::string, std::vector<std::string>>(), d);
        }
    }
}

int main(int argc, char** argv) {
    if (argc < 6) {
        std::cerr << "usage: ref_driver params geometry force plugins outdir [timing]\n";
        return 2;
    }
    bool timing = false;
    unsigned warm = 0, steps = 0;
    std::string restartFile, writePrefix, editFile;
    unsigned editIter = 0, runIters = 0;
    bool withVelocity = false;
    double velX = 0.0, velY = 0.0;
    std::vector<std::pair<unsigned, unsigned>> cellTypes;
    for (int a = 6; a < argc; ++a) {
        const std::string k = argv[a];
        if (k == "timing" && a + 2 < argc) {
            timing = true;
            warm = (unsigned)std::stoul(argv[a + 1]);
            steps = (unsigned)std::stoul(argv[a + 2]);
            a += 2;
        } else if (k == "restart" && a + 1 < argc) {
            restartFile = argv[++a];
        } else if (k == "write" && a + 1 < argc) {
            writePrefix = argv[++a];
        } else if (k == "run" && a + 1 < argc) {
            runIters = (unsigned)std::stoul(argv[++a]);
        } else if (k == "celltype" && a + 2 < argc) {
            cellTypes.emplace_back((unsigned)std::stoul(argv[a + 1]), (unsigned)std::stoul(argv[a + 2]));
            a += 2;
        } else if (k == "velocity" && a + 2 < argc) {
            withVelocity = true;
            velX = std::stod(argv[a + 1]);
            velY = std::stod(argv[a + 2]);
            a += 2;
        } else if (k == "edit" && a + 2 < argc) {
            editIter = (unsigned)std::stoul(argv[a + 1]);
            editFile = argv[a + 2];
            a += 2;
        } else {
            std::cerr << "unknown argument " << k << "\n";
            return 2;
        }
    }
    try {
        std::shared_ptr<std::ostream> logStream(new std::ofstream(std::string(argv[5]) + "/log.txt"));
        UtilLib::Log::setStream(logStream);
        PluginList pl = loadPlugins(argv[4]);
        LbmLib::Parameters.loadGlobalSimulationParameters(argv[1]);
        LbmLib::geometry::Geometry geo(argv[2]);
        LbmLib::geometry::GeometryHandler geohandler(geo);
        LbmLib::reportHandler::ReportHandler reporter(LbmLib::Parameters.getReportSteps());
        LbmLib::SimulationRunner simRunner(geohandler, reporter);
        if (!timing)
            reporter.registerReporter(std::unique_ptr<LbmLib::reportHandler::AbstractReportFunctor>(
                new DumpReporter(geohandler, argv[5])));
        simRunner.initSolvers();
        // SimulationRunner::initSolvers(Field<double>): the lattice again, at a uniform velocity
        if (withVelocity) simRunner.initSolvers(LbmLib::Field<double>(velX, velY));
        if (!restartFile.empty()) simRunner.initSolvers(restartFile);
        if (!cellTypes.empty()) {
            for (const auto& ct : cellTypes) geohandler.getCellTypeTrackerMap()[ct.first] = ct.second;
            geohandler.copyCellTypeToPhysicalNodes(geohandler.getCellTypeTrackerMap());
        }
        simRunner.initForceSolver(argv[3]);
        if (pl.outlet) simRunner.addMassSolver("MassSolverBoxOutlet");
        for (const auto& b : pl.bio) simRunner.addBioSolver(b);
        if (runIters) LbmLib::Parameters.iterations_ = runIters;
        if (!timing && !editFile.empty()) {
            // run to the edit's iteration, edit, run the rest
            const unsigned total = LbmLib::Parameters.iterations_;
            const unsigned first = editIter - LbmLib::Parameters.getCurrentIteration();
            LbmLib::Parameters.iterations_ = first;
            simRunner.runSimulation();
            applyEdit(geohandler, editFile);
            // then what a division plugin does after its edits
            // (tutorial_01_BioSolverCellDivision.cpp:84-91)
            geohandler.cureLattice();
            geohandler.copyCellTypeToPhysicalNodes(geohandler.getCellTypeTrackerMap());
            LbmLib::Parameters.iterations_ = total - first;
            simRunner.runSimulation();
        } else if (!timing) {
            simRunner.runSimulation();
            if (!writePrefix.empty())
                simRunner.writeSimulation(writePrefix + "_force.txt", writePrefix + "_geometry.txt",
                                          writePrefix + "_parameters.txt", writePrefix + "_solver.txt");
        } else {
            LbmLib::Parameters.iterations_ = warm;
            if (warm) simRunner.runSimulation();
            LbmLib::Parameters.iterations_ = steps;
            const auto t0 = std::chrono::steady_clock::now();
            simRunner.runSimulation();
            const auto t1 = std::chrono::steady_clock::now();
            const double sec = std::chrono::duration<double>(t1 - t0).count();
            std::fprintf(stderr, "{\"seconds\": %.6f, \"iterations\": %u, \"warmup\": %u, \"nx\": %u, \"ny\": %u, \"threads\": %d}\n",
                         sec, steps, warm, LbmLib::Parameters.getSizeX(), LbmLib::Parameters.getSizeY(),
                         omp_get_max_threads());
        }
    } catch (const std::exception& e) {
        std::cerr << "reference run failed: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
