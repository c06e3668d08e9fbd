// lbib_oracle.cpp — CPU restatement of LBIBCell's lattice hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// implementation in lbibcell_b200/.  Only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline leg may load it.  It is never linked into, called by
// or used as a fallback for the product path.
//
// It restates, function by function, the serial (OMP_NUM_THREADS=1) behaviour
// of the reference C++ code (wyq977/LBIBCell).  Citations are
// path:line relative to the reference project root.  Floating-point
// expressions keep the reference's evaluation order; the file is compiled
// with -O2 -ffp-contract=off so that no FMA contraction changes a rounding.
//
// Pinning: the restatement is checked bit for bit against the reference
// itself, compiled from its own sources by oracle/build_ref.sh into
// oracle/_ref/ (tests/test_oracle_pin.py, golden fixtures in tests/golden/).
//
// Layout: distributions are kept in the reference's own slot convention
// (swap-scheme streaming, post-collision values stored under the inverse
// direction after FluidSolver::localSwap), so dumps compare slot by slot
// with the reference's solver dump format (SimulationRunner.cpp:112-149).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <numeric>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

// libs/LbmLib/include/Direction.hpp:34-44
enum Dir { T = 0, E = 1, N = 2, W = 3, S = 4, NE = 5, NW = 6, SW = 7, SE = 8 };
// libs/LbmLib/src/Direction.cpp:27-61
static const int INV[9] = {T, W, S, E, N, SW, SE, NE, NW};
static const int CX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int CY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};

// libs/LbmLib/include/Constants.hpp:31-49
static const double CS = 1 / std::sqrt(3);
static const double EPSILON = 10E-10;
static const double PERTURBATION = 10E-7;
static const double MAXLENGTH = 0.5;

// libs/LbmLib/src/solver/FluidSolver/FluidSolver.cpp:39-47
static const double W0 = 4.0 / 9.0;
static const double W1 = 1.0 / 9.0;
static const double W2 = 1.0 / 36.0;

// libs/LbmLib/src/nodes/GeometryNode.cpp:47-48
static const double halfPi = M_PI / 2.0;
static const double doublePi = 2.0 * M_PI;

// Error codes shared with the product's C ABI (include/lbibcell.h).
enum Err {
    OK = 0,
    ERR_EDGE_W = 10, ERR_EDGE_S = 11, ERR_EDGE_E = 12, ERR_EDGE_N = 13,
    ERR_SPEED = 20,
    ERR_LEFT_DOMAIN = 30,
    ERR_VERTICAL = 40,
    ERR_FORCE_NODE = 50,
    ERR_INPUT = 90,
};

struct Fail {
    int code;
    std::string msg;
};

// ---------------------------------------------------------------------------
// fastCos and the 4-point Dirac weight: libs/LbmLib/src/nodes/GeometryNode.cpp:55-94
inline double fastCos(const double x) {
    double cos;
    double tempx = x + halfPi;
    if (tempx > M_PI) {
        tempx -= doublePi;
    }
    if (tempx < .00) {
        cos = 1.27323954 * tempx + 0.405284735 * tempx * tempx;
        if (cos < 0.0) {
            cos = 0.225 * (cos * -cos - cos) + cos;
        } else {
            cos = 0.225 * (cos * cos - cos) + cos;
        }
    } else {
        cos = 1.27323954 * tempx - 0.405284735 * tempx * tempx;
        if (cos < 0.0) {
            cos = 0.225 * (cos * -cos - cos) + cos;
        } else {
            cos = 0.225 * (cos * cos - cos) + cos;
        }
    }
    return cos;
}

inline double delta(const double dx, const double dy) {
    return ((1.0 + fastCos(halfPi * dx)) * (1.0 + fastCos(halfPi * dy))) / 16.0;
}

// ---------------------------------------------------------------------------
// Plugin parameters (the lbibcell_b200 plugin file, see lbibcell_b200/configs.py)

struct CdeSpec {
    std::string name;
    double tau = 1.0;
    int kind = 1;           // 0 base CDESolverD2Q5, 1 Lbib linear source/decay, 2 tutorial_01 SIGNAL
    double init = 0.0;      // initial concentration (kind 1)
    double decay = 0.0;     // linear decay rate (kind 1)
    std::map<unsigned, double> source;  // per-domain production per step (kind 1)
};

struct TensionSpec { double force = 0.01; unsigned frequency = 10; };
struct AreaSpec { double factor = 1.2; double strength = 0.01; double maxsource = 0.004; };

struct Force {
    unsigned type;
    unsigned id1, id2;
    double a, b, c, d;   // type-dependent parameters in file order
};

struct GNode {
    double x, y;       // LagrangianPoint::position_
    double vx = 0, vy = 0;
    double fx = 0, fy = 0;
    double ox, oy;     // GeometryNode::oldPosition_
    int stencil[16];
    int conn0 = -1, conn1 = -1;   // incoming / outgoing connection (pool index)
};

struct Conn {
    unsigned id1, id2, domain;
    std::string descriptor;   // boundary-solver pairs, kept verbatim
};

struct BNode {
    double x, y;
    unsigned domain;
};

struct Sim {
    // Parameters (libs/LbmLib/src/GlobalSimulationParameters.cpp:34-72)
    unsigned currentIteration = 0, iterations = 0, reportStep = 1;
    int nx = 0, ny = 0;
    double tauF = 1.0;
    std::vector<CdeSpec> cde;       // in the parameter map's (alphabetical) order
    int S = 0;
    size_t L = 0;

    // Lattice state
    std::vector<double> f;          // L*9, reference slot convention
    std::vector<double> g;          // S*L*5
    std::vector<double> ux, uy;     // FluidSolver::velocity_
    std::vector<double> frx, fry;   // FluidSolver::force_
    std::vector<double> rhoToAdd;   // FluidSolver::rhoToAdd_
    std::vector<unsigned> dom, ctype;
    std::vector<int> bn;            // L*5 boundary-node slots (index into bnodes or -1)
    std::vector<BNode> bnodes;

    // Membrane
    std::map<unsigned, GNode> nodes;
    std::vector<Conn> pool;
    std::vector<int> conns;         // Geometry::connections_ order (pool indices)
    std::map<unsigned, unsigned> cellTypeTracker;  // GeometryHandler::cellTypeTrackerMap_

    // ForceSolver::forcemap_
    std::map<unsigned, std::vector<Force>> forcemap;

    // Solvers
    bool outlet = false;
    // FluidSolver's force model (its base class, FluidSolver.hpp:41): 0 Luo 1993,
    // 1 Guo, Zheng & Shi 2002 as GuoZhengShi2002ForceModel.cpp writes it,
    // 2 the same with the NE coefficient of the model's expansion (+6 u_y, :51)
    int forceModel = 0;
    std::vector<int> bioOrder;      // 1 tension, 2 area regulator, in registration order
    TensionSpec tension;
    AreaSpec area;
    std::map<unsigned, double> targetArea;

    // Perturbation generators: GeometryNode.cpp:153-158, Connection.cpp:332-337
    std::mt19937 genNode{1};
    std::mt19937 genConn{1};
    std::uniform_real_distribution<> dis{-PERTURBATION, PERTURBATION};

    bool cellTypesCopied = false;   // copyCellTypeToPhysicalNodes has run at least once
    unsigned long long perturbCount = 0;
    unsigned long long reinitCount = 0;

    inline size_t idx(int x, int y) const { return (size_t)y * nx + x; }
    inline size_t nbr(size_t n, int d) const {
        int x = (int)(n % nx), y = (int)(n / nx);
        x += CX[d]; y += CY[d];
        if (x < 0) x += nx; if (x >= nx) x -= nx;
        if (y < 0) y += ny; if (y >= ny) y -= ny;
        return idx(x, y);
    }
};

[[noreturn]] static void fail(int code, const std::string& m) { throw Fail{code, m}; }

// ---------------------------------------------------------------------------
// File loaders (reference formats)

// libs/LbmLib/src/GlobalSimulationParameters.cpp:34-72
static void loadParameters(Sim& s, const std::string& fn) {
    std::ifstream in(fn);
    if (!in.is_open()) fail(ERR_INPUT, "Cannot find the parameter file.");
    std::string line;
    std::map<std::string, double> cdes;
    while (std::getline(in, line)) {
        if (line.empty() || line.at(0) == '#') continue;
        std::stringstream ls(line);
        std::string id;
        ls >> id;
        if (id == "CurrentIterations:") ls >> s.currentIteration;
        else if (id == "Iterations:") ls >> s.iterations;
        else if (id == "ReportStep:") ls >> s.reportStep;
        else if (id == "SizeX:") ls >> s.nx;
        else if (id == "SizeY:") ls >> s.ny;
        else if (id == "tauFluid:") ls >> s.tauF;
        else if (id == "CDESolvers:") {
            std::string nm; double tau;
            while (ls >> nm >> tau) cdes[nm] = tau;
        } else fail(ERR_INPUT, "An unknown parameter was passed in the global Parameter file");
    }
    for (auto& kv : cdes) {
        CdeSpec c; c.name = kv.first; c.tau = kv.second;
        if (kv.first == "CDESolverD2Q5") c.kind = 0;
        else if (kv.first == "tutorial_01_CDESolverD2Q5_SIGNAL") c.kind = 2;
        else c.kind = 1;
        s.cde.push_back(c);
    }
    s.S = (int)s.cde.size();
}

// lbibcell_b200 plugin file: lbibcell_b200/configs.py documents the format.
static void loadPlugins(Sim& s, const std::string& fn) {
    if (fn.empty()) return;
    std::ifstream in(fn);
    if (!in.is_open()) fail(ERR_INPUT, "Cannot find the plugin file.");
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line.at(0) == '#') continue;
        std::stringstream ls(line);
        std::string kind, name;
        ls >> kind >> name;
        std::map<std::string, double> kv;
        if (kind == "MassSolver") {
            if (name == "MassSolverBoxOutlet") s.outlet = true;
            else fail(ERR_INPUT, "unknown mass solver " + name);
        } else if (kind == "ForceModel") {
            if (name == "Luo1993ForceModel") s.forceModel = 0;
            else if (name == "GuoZhengShi2002ForceModel") s.forceModel = 1;
            else if (name == "GuoZhengShi2002ForceModelCorrected") s.forceModel = 2;
            else fail(ERR_INPUT, "unknown force model " + name);
        } else if (kind == "BioSolver") {
            std::string k; double v;
            while (ls >> k >> v) kv[k] = v;
            if (name == "LbibMembraneTension") {
                s.bioOrder.push_back(1);
                if (kv.count("force")) s.tension.force = kv["force"];
                if (kv.count("frequency")) s.tension.frequency = (unsigned)kv["frequency"];
            } else if (name == "LbibAreaRegulator") {
                s.bioOrder.push_back(2);
                if (kv.count("factor")) s.area.factor = kv["factor"];
                if (kv.count("strength")) s.area.strength = kv["strength"];
                if (kv.count("maxsource")) s.area.maxsource = kv["maxsource"];
            } else fail(ERR_INPUT, "unknown bio solver " + name);
        } else if (kind == "CDE") {
            std::string k; double v;
            while (ls >> k >> v) kv[k] = v;
            for (auto& c : s.cde) if (c.name == name) {
                if (kv.count("init")) c.init = kv["init"];
                if (kv.count("decay")) c.decay = kv["decay"];
            }
        } else if (kind == "CDESource") {
            unsigned d; double r;
            while (ls >> d >> r)
                for (auto& c : s.cde) if (c.name == name) c.source[d] = r;
        } else fail(ERR_INPUT, "unknown plugin line " + kind);
    }
}

// GeometryNode::perturbatePosition — libs/LbmLib/src/nodes/GeometryNode.cpp:153-214.
// The two draws in one setPos(x + dis(gen), y + dis(gen)) call are taken
// y-first: g++ evaluates those arguments right to left (checked against the
// reference build in oracle/_ref).
static void perturbatePosition(Sim& s, GNode& p) {
    double temprand;
    if (std::abs(static_cast<int>(p.x) - p.x) <= EPSILON) {
        temprand = 0.0;
        while (std::abs(temprand) < 5.0 * EPSILON) temprand = s.dis(s.genNode);
        p.x = p.x + temprand;
        s.perturbCount++;
    }
    if (std::abs(static_cast<int>(p.y) - p.y) <= EPSILON) {
        temprand = 0.0;
        while (std::abs(temprand) < 5.0 * EPSILON) temprand = s.dis(s.genNode);
        p.y = p.y + temprand;
        s.perturbCount++;
    }
    if (std::abs(p.y - std::floor(p.y) - (p.x - std::floor(p.x))) <= EPSILON) {
        double ry = s.dis(s.genNode);
        double rx = s.dis(s.genNode);
        p.x = p.x + rx; p.y = p.y + ry;
        s.perturbCount++;
    }
    if (std::abs(std::ceil(p.y) - p.y - (p.x - std::floor(p.x))) <= EPSILON) {
        double ry = s.dis(s.genNode);
        double rx = s.dis(s.genNode);
        p.x = p.x + rx; p.y = p.y + ry;
        s.perturbCount++;
    }
}

// GeometryNode(x, y, id): libs/LbmLib/src/nodes/GeometryNode.cpp:98-117
static GNode makeNode(Sim& s, double x, double y) {
    GNode p;
    p.x = x; p.y = y;
    p.ox = x - 5.0; p.oy = y - 5.0;
    for (int k = 0; k < 16; ++k) p.stencil[k] = -1;
    perturbatePosition(s, p);
    return p;
}

// Geometry::loadGeometryTXT — libs/LbmLib/src/geometry/Geometry.cpp:99-160
static void loadGeometry(Sim& s, const std::string& fn) {
    std::ifstream in(fn);
    if (!in.is_open()) fail(ERR_INPUT, "Cannot find the geometry.txt file.");
    s.cellTypeTracker[0] = 0;
    std::string line;
    bool nodes = true;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        if (line.find("#Connection") != std::string::npos) nodes = false;
        if (line.at(0) == '#') continue;
        std::stringstream ls(line);
        if (nodes) {
            unsigned id; double x, y;
            ls >> id >> x >> y;
            s.nodes[id] = makeNode(s, x, y);
        } else {
            unsigned id1, id2, d;
            ls >> id1 >> id2 >> d;
            s.cellTypeTracker[d] = 1;
            std::string rest, a, b;
            while (ls >> a >> b) rest += "\t" + a + "\t" + b;
            Conn c{id1, id2, d, rest};
            s.pool.push_back(c);
            int ci = (int)s.pool.size() - 1;
            s.conns.push_back(ci);
            s.nodes.at(id1).conn1 = ci;
            s.nodes.at(id2).conn0 = ci;
        }
    }
}

// ForceStructs loaders: libs/LbmLib/include/solver/ForceStructs.hpp:49-588
static void addForceLine(Sim& s, const std::string& line) {
    std::stringstream ls(line);
    Force f{};
    unsigned type;
    ls >> type;
    f.type = type;
    switch (type) {
        case 0: case 7: ls >> f.id1 >> f.id2 >> f.a >> f.b; break;        // k l0
        case 1: ls >> f.id1 >> f.a >> f.b >> f.c >> f.d; break;            // x y k l0
        case 2: ls >> f.id1 >> f.a >> f.b; break;                          // fx fy
        case 3: case 4: ls >> f.id1 >> f.a >> f.b >> f.c; break;           // y|x k l0
        case 5: case 6: ls >> f.id1 >> f.id2 >> f.a; break;                // f
        default: fail(ERR_INPUT, "Invalid force solver type found.");
    }
    s.forcemap[f.id1].push_back(f);
}

// ForceSolver::loadForceFile — libs/LbmLib/src/solver/ForceSolver.cpp:89-105
static void loadForces(Sim& s, const std::string& fn) {
    if (fn.empty()) return;
    std::ifstream in(fn);
    if (!in.is_open()) fail(ERR_INPUT, "Cannot find the force solver file.");
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line.at(0) == '#') continue;
        addForceLine(s, line);
    }
}

// ---------------------------------------------------------------------------
// Fluid solver (D2Q9 BGK, Luo 1993 forcing)

// FluidSolver::getRho — FluidSolver.cpp:248-251 (std::accumulate in slot order)
static inline double sumSlots9(const double* f) {
    double r = 0.0;
    for (int i = 0; i < 9; ++i) r += f[i];
    return r;
}

// Luo1993ForceModel::computeVelocity — Luo1993ForceModel.cpp:51-70
static inline void computeVelocity(double rho, const double* fi, double& uxo, double& uyo) {
    const double rhoI = 1.0 / rho;
    uxo = (fi[E] + fi[NE] + fi[SE] - (fi[NW] + fi[W] + fi[SW])) * rhoI;
    uyo = (fi[NE] + fi[N] + fi[NW] - (fi[SW] + fi[S] + fi[SE])) * rhoI;
}

// GuoZhengShi2002ForceModel::computeVelocity — GuoZhengShi2002ForceModel.cpp:60-78
static inline void computeVelocityGuo(double rho, const double* fi, double fx, double fy, double& uxo, double& uyo) {
    const double rhoI = 1.0 / rho;
    uxo = (fi[E] + fi[NE] + fi[SE] - (fi[NW] + fi[W] + fi[SW]) + 0.5 * fx) * rhoI;
    uyo = (fi[NE] + fi[N] + fi[NW] - (fi[SW] + fi[S] + fi[SE]) + 0.5 * fy) * rhoI;
}

// The force contribution of FluidSolver::collide (FluidSolver.cpp:140-145):
// Luo1993ForceModel::computeForce (Luo1993ForceModel.cpp:29-49) from getRho()
// without rhoToAdd, or GuoZhengShi2002ForceModel::computeForce
// (GuoZhengShi2002ForceModel.cpp:29-58) from tau and the stored velocity
// getVelocity() (velocity_ of the previous collide).
static void forceContribution(const Sim& s, size_t n, const double* fi, double* fc) {
    const double fx = s.frx[n], fy = s.fry[n];
    if (s.forceModel == 0) {
        const double rhoF = sumSlots9(fi);
        const double W1rho3 = rhoF * 3.0 / 9.0;
        const double W2rho3 = rhoF * 3.0 / 36.0;
        fc[T] = 0.0;
        fc[E] = W1rho3 * fx;
        fc[N] = W1rho3 * fy;
        fc[W] = -W1rho3 * fx;
        fc[S] = -W1rho3 * fy;
        fc[NE] = W2rho3 * (fx + fy);
        fc[NW] = W2rho3 * (-fx + fy);
        fc[SW] = W2rho3 * (-fx - fy);
        fc[SE] = W2rho3 * (fx - fy);
        return;
    }
    const double vx = s.ux[n], vy = s.uy[n];
    const double tau = s.tauF;
    const double G0 = (1.0 - 0.5 / tau) * 4.0 / 9.0;
    const double G1 = (1.0 - 0.5 / tau) / 9.0;
    const double G2 = (1.0 - 0.5 / tau) / 36.0;
    // the NE term's F_y factor: 9 v_x - 3 v_y + 3 as written at :51; 9 v_x + 6 v_y + 3 corrected
    const double neY = s.forceModel == 1 ? -3.0 : 6.0;
    fc[T] = G0 * (-3.0 * vx * fx - 3.0 * vy * fy);
    fc[E] = G1 * ((6.0 * vx + 3.0) * fx - 3.0 * vy * fy);
    fc[N] = G1 * (-3.0 * vx * fx + (6.0 * vy + 3.0) * fy);
    fc[W] = G1 * ((6.0 * vx - 3.0) * fx - 3.0 * vy * fy);
    fc[S] = G1 * (-3.0 * vx * fx + (6.0 * vy - 3.0) * fy);
    fc[NE] = G2 * ((6.0 * vx + 9.0 * vy + 3.0) * fx + (9.0 * vx + neY * vy + 3.0) * fy);
    fc[NW] = G2 * ((6.0 * vx - 9.0 * vy - 3.0) * fx + (-9.0 * vx + 6.0 * vy + 3.0) * fy);
    fc[SW] = G2 * ((6.0 * vx + 9.0 * vy - 3.0) * fx + (9.0 * vx + 6.0 * vy - 3.0) * fy);
    fc[SE] = G2 * ((6.0 * vx - 9.0 * vy + 3.0) * fx + (-9.0 * vx + 6.0 * vy - 3.0) * fy);
}

// FluidSolver::collide — FluidSolver.cpp:103-183, with the force model's
// velocity and force contribution, and localSwap (:259-264).
static void fluidCollide(Sim& s, size_t n) {
    double* fi = &s.f[n * 9];
    double rho = sumSlots9(fi);
    if (std::isfinite(s.rhoToAdd[n])) rho += s.rhoToAdd[n];
    const double fx = s.frx[n], fy = s.fry[n];
    double ux, uy;
    if (s.forceModel == 0) computeVelocity(rho, fi, ux, uy);
    else computeVelocityGuo(rho, fi, fx, fy, ux, uy);
    const double ux2 = ux * ux;
    const double uy2 = uy * uy;
    const double lastTerm = 3.0 / 2.0 * (ux2 + uy2);
    const double tauI = 1.0 / s.tauF;
    const double W3 = 9.0 / 2.0;
    const double W1rho = W1 * rho;
    const double W2rho = W2 * rho;
    double fc[9];
    forceContribution(s, n, fi, fc);
    double temp[9];
    temp[T] = W0 * rho * (1.0 - lastTerm) * tauI + fc[T];
    temp[E] = W1rho * (1.0 + 3.0 * ux + W3 * ux2 - lastTerm) * tauI + fc[E];
    temp[NE] = W2rho * (1.0 + 3.0 * (ux + uy) + W3 * (ux + uy) * (ux + uy) - lastTerm) * tauI + fc[NE];
    temp[N] = W1rho * (1.0 + 3.0 * uy + W3 * uy2 - lastTerm) * tauI + fc[N];
    temp[NW] = W2rho * (1.0 + 3.0 * (-ux + uy) + W3 * (-ux + uy) * (-ux + uy) - lastTerm) * tauI + fc[NW];
    temp[W] = W1rho * (1.0 + 3.0 * (-ux) + W3 * ux2 - lastTerm) * tauI + fc[W];
    temp[SW] = W2rho * (1.0 + 3.0 * (-ux - uy) + W3 * (-ux - uy) * (-ux - uy) - lastTerm) * tauI + fc[SW];
    temp[S] = W1rho * (1.0 + 3.0 * (-uy) + W3 * uy2 - lastTerm) * tauI + fc[S];
    temp[SE] = W2rho * (1.0 + 3.0 * (ux - uy) + W3 * (ux - uy) * (ux - uy) - lastTerm) * tauI + fc[SE];
    for (int d = 0; d < 9; ++d) {
        const double tempD = fi[d];
        fi[d] = tempD - tempD * tauI + temp[d];
    }
    if (s.forceModel == 0) computeVelocity(rho, fi, ux, uy);
    else computeVelocityGuo(rho, fi, fx, fy, ux, uy);
    s.ux[n] = ux; s.uy[n] = uy;
    s.rhoToAdd[n] = 0.0;
    std::swap(fi[E], fi[W]); std::swap(fi[NE], fi[SW]);
    std::swap(fi[N], fi[S]); std::swap(fi[NW], fi[SE]);
}

// FluidSolver::advect — FluidSolver.cpp:185-194 (swap with the W, SW, S, SE neighbours)
static void fluidAdvect(Sim& s, size_t n) {
    std::swap(s.f[n * 9 + E], s.f[s.nbr(n, W) * 9 + W]);
    std::swap(s.f[n * 9 + NE], s.f[s.nbr(n, SW) * 9 + SW]);
    std::swap(s.f[n * 9 + N], s.f[s.nbr(n, S) * 9 + S]);
    std::swap(s.f[n * 9 + NW], s.f[s.nbr(n, SE) * 9 + SE]);
}

// ---------------------------------------------------------------------------
// CDE solvers (D2Q5)

static inline double sumSlots5(const double* g) {
    double r = 0.0;
    for (int i = 0; i < 5; ++i) r += g[i];
    return r;
}

// Reaction term R for species k at node n.
//   kind 1 (Lbib linear): R = source[domain] - decay * C
//   kind 2 (tutorial_01 SIGNAL): tutorial_01_CDESolverD2Q5_SIGNAL.cpp:92-100
static inline double reaction(const Sim& s, int k, size_t n, double C) {
    const CdeSpec& c = s.cde[k];
    if (c.kind == 1) {
        auto it = c.source.find(s.dom[n]);
        const double src = it == c.source.end() ? 0.0 : it->second;
        return src - c.decay * C;
    }
    if (c.kind == 2) {
        if (s.dom[n] == 1 && s.currentIteration < 5000) return 0.0001;
        return -0.00001 * C;
    }
    return 0.0;
}

// CDESolverD2Q5::collide — CDESolverD2Q5.cpp:75-107; with the reaction source
// added as dt*R/3 (rest) and dt*R/6 (moving) as in
// tutorial_01_CDESolverD2Q5_SIGNAL.cpp:102-135.
static void cdeCollide(Sim& s, int k, size_t n) {
    double* gi = &s.g[((size_t)k * s.L + n) * 5];
    const double C = sumSlots5(gi);
    const double ux = s.ux[n], uy = s.uy[n];
    const double w0 = C / 3.0;
    const double w1 = C / 6.0;
    const double tauI = 1.0 / s.cde[k].tau;
    double temp[5];
    temp[T] = w0;
    temp[E] = w1 * (1.0 + ux * 3.0);
    temp[N] = w1 * (1.0 + uy * 3.0);
    temp[W] = w1 * (1.0 + (-ux) * 3.0);
    temp[S] = w1 * (1.0 + (-uy) * 3.0);
    if (s.cde[k].kind == 0) {
        for (int d = 0; d < 5; ++d) {
            double tempD = gi[d];
            gi[d] = tempD - tempD * tauI + temp[d] * tauI;
        }
    } else {
        const double R = reaction(s, k, n, C);
        const double deltaT = 1.0;
        const double r0 = deltaT * R / 3.0;
        const double r1 = deltaT * R / 6.0;
        gi[T] = gi[T] - gi[T] * tauI + temp[T] * tauI + r0;
        gi[E] = gi[E] - gi[E] * tauI + temp[E] * tauI + r1;
        gi[N] = gi[N] - gi[N] * tauI + temp[N] * tauI + r1;
        gi[W] = gi[W] - gi[W] * tauI + temp[W] * tauI + r1;
        gi[S] = gi[S] - gi[S] * tauI + temp[S] * tauI + r1;
    }
    std::swap(gi[E], gi[W]);
    std::swap(gi[N], gi[S]);
}

// CDESolverD2Q5::advect — CDESolverD2Q5.cpp:141-149
static void cdeAdvect(Sim& s, int k, size_t n) {
    double* base = &s.g[(size_t)k * s.L * 5];
    std::swap(base[n * 5 + E], base[s.nbr(n, W) * 5 + W]);
    std::swap(base[n * 5 + N], base[s.nbr(n, S) * 5 + S]);
}

// CDESolverD2Q5::reinitialise — CDESolverD2Q5.cpp:156-228.
// The diagonal fallback reads PhysicalNode::boundaryNodes_ (a 5-element
// array) at indices NE..SE, past its end (PhysicalNode.hpp:200-210).  Index
// NE aliases the (domainIdentifier_, cellType_) pair, which is "non-null"
// unless both are zero; indices NW..SE read past the object and are treated
// as non-null.  This is what the reference build does with glibc's heap.
static void cdeReinit(Sim& s, int k, size_t n) {
    double sumC = 0.0;
    int counter = 0;
    const unsigned my = s.dom[n];
    const int dir1[4] = {E, N, W, S};
    for (int d : dir1) {
        size_t m = s.nbr(n, d);
        if (s.bn[n * 5 + d] < 0 && my == s.dom[m]) {
            sumC += sumSlots5(&s.g[((size_t)k * s.L + m) * 5]);
            counter++;
        }
    }
    if (counter == 0) {
        const bool neNull = (s.dom[n] == 0 && s.ctype[n] == 0);
        if (neNull) {
            size_t m = s.nbr(n, NE);
            if (my == s.dom[m]) {
                sumC += sumSlots5(&s.g[((size_t)k * s.L + m) * 5]);
                counter++;
            }
        }
    }
    sumC /= static_cast<double>(counter);
    double* gi = &s.g[((size_t)k * s.L + n) * 5];
    for (int d = 0; d < 5; ++d) gi[d] = sumC / 5.0;
    cdeCollide(s, k, n);
}

// CDE initial conditions
static void cdeInit(Sim& s, int k, size_t n) {
    double* gi = &s.g[((size_t)k * s.L + n) * 5];
    const CdeSpec& c = s.cde[k];
    if (c.kind == 0) {
        // CDESolverD2Q5::initSolver — CDESolverD2Q5.cpp:37-40
        gi[T] = 1.0;
        cdeCollide(s, k, n);
    } else if (c.kind == 2) {
        // tutorial_01_CDESolverD2Q5_SIGNAL::initSolver — :46-57
        for (int d = 0; d < 5; ++d) gi[d] = s.dom[n] == 0 ? 0.0 : 1.0 / 5.0;
    } else {
        for (int d = 0; d < 5; ++d) gi[d] = c.init / 5.0;
    }
}

// ---------------------------------------------------------------------------
// Geometry: forces, spreading, interpolation, motion, crossings, domain ids

// ForceSolver::calculateForce — ForceSolver.cpp:42-85; force kinds per
// ForceStructs.hpp:49-588.  Each force adds to its own node id1, in the
// node's insertion order.
static void calculateForce(Sim& s) {
    for (auto& kv : s.nodes) { kv.second.fx = 0.0; kv.second.fy = 0.0; }
    for (auto& kv : s.forcemap) {
        for (const Force& f : kv.second) {
            auto it1 = s.nodes.find(f.id1);
            if (it1 == s.nodes.end()) fail(ERR_FORCE_NODE, "Could not compute and set the forces.");
            GNode& p1 = it1->second;
            switch (f.type) {
                case 0: case 7: {
                    auto it2 = s.nodes.find(f.id2);
                    if (it2 == s.nodes.end()) fail(ERR_FORCE_NODE, "Could not compute and set the forces.");
                    GNode& p2 = it2->second;
                    const double dist = std::sqrt((p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y));
                    const double fm = f.a * (dist - f.b);
                    const double ddx = p2.x - p1.x, ddy = p2.y - p1.y;
                    const double dist2 = std::sqrt((p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y));
                    p1.fx += (ddx * fm) / dist2;
                    p1.fy += (ddy * fm) / dist2;
                    break;
                }
                case 1: {
                    // anchor at (x, y): ForceStructs.hpp ForceType1
                    const double tx = f.a, ty = f.b;
                    const double dist = std::sqrt((tx - p1.x) * (tx - p1.x) + (ty - p1.y) * (ty - p1.y));
                    const double fm = f.c * (dist - f.d);
                    if (dist != 0.0) {
                        p1.fx += ((tx - p1.x) * fm) / dist;
                        p1.fy += ((ty - p1.y) * fm) / dist;
                    }
                    break;
                }
                case 2:
                    p1.fx += f.a; p1.fy += f.b;
                    break;
                case 3: {
                    const double dist = std::sqrt((p1.x - p1.x) * (p1.x - p1.x) + (f.a - p1.y) * (f.a - p1.y));
                    const double fm = f.b * (dist - f.c);
                    const double fy = p1.y < f.a ? fm : -fm;
                    p1.fx += 0.0; p1.fy += fy;
                    break;
                }
                case 4: {
                    const double dist = std::sqrt((f.a - p1.x) * (f.a - p1.x) + (p1.y - p1.y) * (p1.y - p1.y));
                    const double fm = f.b * (dist - f.c);
                    const double fx = p1.x < f.a ? fm : -fm;
                    p1.fx += fx; p1.fy += 0.0;
                    break;
                }
                case 5: case 6: {
                    auto it2 = s.nodes.find(f.id2);
                    if (it2 == s.nodes.end()) fail(ERR_FORCE_NODE, "Could not compute and set the forces.");
                    GNode& p2 = it2->second;
                    const double ddx = p2.x - p1.x, ddy = p2.y - p1.y;
                    const double dist = std::sqrt((p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y));
                    p1.fx += (ddx * f.a) / dist;
                    p1.fy += (ddy * f.a) / dist;
                    break;
                }
            }
        }
    }
}

// SimulationRunner::distributeForce — SimulationRunner.cpp:425-453 and
// GeometryNode::distributeForce — GeometryNode.cpp:228-235.
static void distributeForce(Sim& s) {
    std::fill(s.frx.begin(), s.frx.end(), 0.0);
    std::fill(s.fry.begin(), s.fry.end(), 0.0);
    for (auto& kv : s.nodes) {
        GNode& p = kv.second;
        for (int k = 0; k < 16; ++k) {
            const int m = p.stencil[k];
            const double dx = (double)(m % s.nx) - p.x;
            const double dy = (double)(m / s.nx) - p.y;
            const double dl = delta(dx, dy);
            s.frx[m] += p.fx * dl;
            s.fry[m] += p.fy * dl;
        }
    }
}

// GeometryNode::collectVelocity — GeometryNode.cpp:216-226 (slot order 0..15)
// and LagrangianPoint::setVelocity's speed check — LagrangianPoint.cpp:92-103.
static void collectVelocity(Sim& s) {
    for (auto& kv : s.nodes) {
        GNode& p = kv.second;
        double vx = 0.0, vy = 0.0;
        for (int k = 0; k < 16; ++k) {
            const int m = p.stencil[k];
            const double dx = (double)(m % s.nx) - p.x;
            const double dy = (double)(m / s.nx) - p.y;
            const double dl = delta(dx, dy);
            vx += s.ux[m] * dl;
            vy += s.uy[m] * dl;
        }
        p.vx = vx; p.vy = vy;
        if (((vx * vx) + (vy * vy)) > CS) fail(ERR_SPEED, "The magnitude of velocity is too high");
    }
}

// GeometryHandler::connectGeometryNodesToPhysicalNodes(pt) — GeometryHandler.cpp:608-644
// with GeometryNode::isUpdateNeeded — GeometryNode.cpp:256-261 and
// Rectangle::pointWithinBounds — libs/UtilLib/src/geometry/Rectangle.cpp.
static void connectNode(Sim& s, GNode& p) {
    const double north = std::ceil(p.oy), south = std::floor(p.oy);
    const double west = std::floor(p.ox), east = std::ceil(p.ox);
    const bool within = (p.x >= west) && (p.x < east) && (p.y <= north) && (p.y > south);
    if (within) return;
    const double minX = p.x - 2.0, maxX = p.x + 2.0, minY = p.y - 2.0, maxY = p.y + 2.0;
    if (minX < 0) fail(ERR_EDGE_W, "geometry point moved too close to the west boundary");
    if (minY < 0) fail(ERR_EDGE_S, "geometry point moved too close to the south boundary");
    if (maxX > s.nx) fail(ERR_EDGE_E, "geometry point moved too close to the east boundary");
    if (maxY > s.ny) fail(ERR_EDGE_N, "geometry point moved too close to the north boundary");
    for (int x = (int)std::ceil(minX); x <= (int)std::floor(maxX); x++)
        for (int y = (int)std::ceil(minY); y <= (int)std::floor(maxY); y++)
            p.stencil[(x * 4 + y) % 16] = (int)s.idx(x, y);
}

static void connectAll(Sim& s) {
    for (auto& kv : s.nodes) connectNode(s, kv.second);
}

// Connection::perturbConnection — Connection.cpp:332-387
static void perturbConnection(Sim& s, Conn& c) {
    GNode& p1 = s.nodes.at(c.id1);
    GNode& p2 = s.nodes.at(c.id2);
    double temprand;
    if (std::abs(p1.x - p2.x) < EPSILON) {
        temprand = 0.0;
        while (std::abs(temprand) < 5.0 * EPSILON) temprand = s.dis(s.genConn);
        p1.x = p1.x + temprand;
        perturbatePosition(s, p1);
        s.perturbCount++;
    }
    if (std::abs(p1.y - p2.y) < EPSILON) {
        temprand = 0.0;
        while (std::abs(temprand) < 5.0 * EPSILON) temprand = s.dis(s.genConn);
        p1.y = p1.y + temprand;
        perturbatePosition(s, p1);
        s.perturbCount++;
    }
}

// GeometryHandler::perturbConnections — GeometryHandler.cpp:326-356
static void perturbConnections(Sim& s) {
    std::map<unsigned, int> first;
    for (int ci : s.conns)
        if (first.find(s.pool[ci].domain) == first.end()) first[s.pool[ci].domain] = ci;
    for (auto& kv : first) {
        int start = kv.second, c = start;
        do {
            perturbConnection(s, s.pool[c]);
            c = s.nodes.at(s.pool[c].id2).conn1;
        } while (c != start);
    }
}

// Connection::insertBoundaryNode — Connection.cpp:181-222 (closest wins,
// strict <, so ties keep the earlier one).
static void insertBN(Sim& s, const BNode& b, size_t node, int d) {
    const int slot = INV[d];
    int& cur = s.bn[node * 5 + slot];
    const double px = (double)(node % s.nx), py = (double)(node / s.nx);
    if (cur < 0) {
        s.bnodes.push_back(b);
        cur = (int)s.bnodes.size() - 1;
    } else {
        const BNode& o = s.bnodes[cur];
        const double dn = (px - b.x) * (px - b.x) + (py - b.y) * (py - b.y);
        const double dold = (px - o.x) * (px - o.x) + (py - o.y) * (py - o.y);
        if (dn < dold) {
            s.bnodes.push_back(b);
            cur = (int)s.bnodes.size() - 1;
        }
    }
}

// Connection::generateBoundaryNodes — Connection.cpp:224-324
static void generateBoundaryNodes(Sim& s) {
    s.bnodes.clear();
    std::fill(s.bn.begin(), s.bn.end(), -1);
    for (int ci : s.conns) {
        const Conn& c = s.pool[ci];
        const GNode& p1 = s.nodes.at(c.id1);
        const GNode& p2 = s.nodes.at(c.id2);
        const double maxX = std::max(p1.x, p2.x), maxY = std::max(p1.y, p2.y);
        const double minX = std::min(p1.x, p2.x), minY = std::min(p1.y, p2.y);
        const double m = (p2.y - p1.y) / (p2.x - p1.x);
        const double n = p1.y - (p2.y - p1.y) / (p2.x - p1.x) * p1.x;
        if (!std::isfinite(m)) fail(ERR_VERTICAL, "This can only happen if something went wrong with the perturbation of the connection.");
        for (int i = (int)std::ceil(minX); i <= (int)std::floor(maxX); i++) {
            const double yc = m * i + n;
            BNode bS{(double)i, yc, 0}, bN{(double)i, yc, 0};
            if (p1.x < p2.x) bN.domain = c.domain; else bS.domain = c.domain;
            const size_t fS = s.idx(i, (int)std::floor(m * i + n));
            const size_t fN = s.idx(i, (int)std::ceil(m * i + n));
            insertBN(s, bS, fS, S);
            insertBN(s, bN, fN, N);
        }
        for (int i = (int)std::ceil(minY); i <= (int)std::floor(maxY); i++) {
            const double xc = (i - n) / m;
            BNode bW{xc, (double)i, 0}, bE{xc, (double)i, 0};
            if (p1.y > p2.y) bE.domain = c.domain; else bW.domain = c.domain;
            const size_t fW = s.idx((int)std::floor((i - n) / m), i);
            const size_t fE = s.idx((int)std::ceil((i - n) / m), i);
            insertBN(s, bW, fW, W);
            insertBN(s, bE, fE, E);
        }
    }
}

// GeometryHandler::updateDomainIdentifier — GeometryHandler.cpp:58-66 and
// PhysicalNode::updateDomainIdentifier — PhysicalNode.cpp:109-124.
static void updateDomainIdentifier(Sim& s) {
    for (size_t n = 0; n < s.L; ++n) {
        unsigned t = s.dom[n];
        for (int d = 0; d < 5; ++d)
            if (s.bn[n * 5 + d] >= 0) t = s.bnodes[s.bn[n * 5 + d]].domain;
        if (s.dom[n] != t) {
            s.dom[n] = t;
            for (int k = 0; k < s.S; ++k) cdeReinit(s, k, n);
            s.reinitCount++;
        }
    }
}

// GeometryHandler::updateAllDomainIdentifiers — GeometryHandler.cpp:68-85
static void updateAllDomainIdentifiers(Sim& s) {
    for (int y = 0; y < s.ny; ++y) {
        unsigned cur = s.dom[s.idx(0, y)];
        if (cur != 0) fail(ERR_LEFT_DOMAIN, "domainID at the left boundary must be 0.");
        for (int x = 1; x < s.nx; ++x) {
            const size_t n = s.idx(x, y);
            if (s.bn[n * 5 + W] >= 0) cur = s.bnodes[s.bn[n * 5 + W]].domain;
            s.dom[n] = cur;
        }
    }
}

// GeometryHandler::copyCellTypeToPhysicalNodes(map) — GeometryHandler.cpp:267-301
static void copyCellType(Sim& s) {
    for (size_t n = 0; n < s.L; ++n) {
        auto it = s.cellTypeTracker.find(s.dom[n]);
        if (it == s.cellTypeTracker.end()) s.cellTypeTracker[s.dom[n]] = 1;
        s.ctype[n] = s.cellTypeTracker[s.dom[n]];
    }
    s.cellTypesCopied = true;
}

// GeometryHandler::cureLattice — GeometryHandler.cpp:149-170
static void cureLattice(Sim& s) {
    perturbConnections(s);
    connectAll(s);
    generateBoundaryNodes(s);
    updateAllDomainIdentifiers(s);
}

// GeometryHandler::moveLattice — GeometryHandler.cpp:358-383, with
// Geometry::moveGeometryNodes — Geometry.cpp:454-469 and GeometryNode::move —
// GeometryNode.cpp:245-254.
static void moveLattice(Sim& s) {
    for (auto& kv : s.nodes) {
        GNode& p = kv.second;
        p.ox = p.x; p.oy = p.y;
        p.x = p.x + p.vx;
        p.y = p.y + p.vy;
        perturbatePosition(s, p);
    }
    perturbConnections(s);
    generateBoundaryNodes(s);
    connectAll(s);
    updateDomainIdentifier(s);
    updateAllDomainIdentifiers(s);
    copyCellType(s);
}

static double connLength(const Sim& s, const Conn& c) {
    const GNode& a = s.nodes.at(c.id1);
    const GNode& b = s.nodes.at(c.id2);
    return std::sqrt((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y));
}

static void eraseConn(Sim& s, int ci) {
    Conn& c = s.pool[ci];
    GNode& a = s.nodes.at(c.id1);
    GNode& b = s.nodes.at(c.id2);
    if (a.conn1 == ci) a.conn1 = -1;
    if (b.conn0 == ci) b.conn0 = -1;
    s.conns.erase(std::remove(s.conns.begin(), s.conns.end(), ci), s.conns.end());
}

static void addConn(Sim& s, unsigned id1, unsigned id2, const std::string& desc, unsigned dom) {
    s.pool.push_back(Conn{id1, id2, dom, desc});
    int ci = (int)s.pool.size() - 1;
    s.conns.push_back(ci);
    s.nodes.at(id1).conn1 = ci;
    s.nodes.at(id2).conn0 = ci;
}

// GeometryHandler::remeshBoundary — GeometryHandler.cpp:385-431 with
// Geometry::addGeometryNode — Geometry.cpp:382-400.
static unsigned remeshOnce(Sim& s) {
    std::vector<int> copy = s.conns;
    unsigned counter = 0;
    for (int ci : copy) {
        if (connLength(s, s.pool[ci]) > MAXLENGTH) {
            const Conn c = s.pool[ci];
            const GNode& a = s.nodes.at(c.id1);
            const GNode& b = s.nodes.at(c.id2);
            const double x1 = a.x, y1 = a.y, x2 = b.x, y2 = b.y;
            const unsigned nid = s.nodes.rbegin()->first + 1;
            s.nodes[nid] = makeNode(s, (x1 + x2) / 2, (y1 + y2) / 2);
            eraseConn(s, ci);
            addConn(s, c.id1, nid, c.descriptor, c.domain);
            addConn(s, nid, c.id2, c.descriptor, c.domain);
            counter++;
        }
    }
    connectAll(s);
    return counter;
}

// GeometryHandler::coarsenBoundary — GeometryHandler.cpp:433-461 with
// Geometry::removeGeometryNode — Geometry.cpp:402-431.
static void coarsen(Sim& s) {
    for (auto it = s.nodes.begin(); it != s.nodes.end();) {
        const GNode& p = it->second;
        const GNode& P1 = s.nodes.at(s.pool[p.conn0].id1);
        const GNode& P2 = s.nodes.at(s.pool[p.conn1].id2);
        const double length = std::sqrt((P2.x - P1.x) * (P2.x - P1.x) + (P2.y - P1.y) * (P2.y - P1.y));
        if (length < MAXLENGTH) {
            const unsigned id = it->first;
            ++it;
            const int C1 = s.nodes.at(id).conn0, C2 = s.nodes.at(id).conn1;
            const unsigned N1 = s.pool[C1].id1, N2 = s.pool[C2].id2;
            const std::string desc = s.pool[C1].descriptor;
            const unsigned dom = s.pool[C1].domain;
            eraseConn(s, C1);
            eraseConn(s, C2);
            s.nodes.erase(id);
            addConn(s, N1, N2, desc, dom);
        } else {
            ++it;
        }
    }
}

// GeometryHandler::computeAreas — GeometryHandler.cpp:101-134.  The polygon
// area is the shoelace sum over the ring in ring order (the stand-in for
// boost::geometry::area used by the reference build too).
static std::map<unsigned, double> computeAreas(const Sim& s) {
    std::map<unsigned, int> first;
    for (int ci : s.conns)
        if (first.find(s.pool[ci].domain) == first.end()) first[s.pool[ci].domain] = ci;
    std::map<unsigned, double> areas;
    for (auto& kv : first) {
        std::vector<double> xs, ys;
        int start = kv.second, c = start;
        do {
            const GNode& p = s.nodes.at(s.pool[c].id2);
            xs.push_back(p.x); ys.push_back(p.y);
            c = p.conn1;
        } while (c != start);
        double sum = 0.0;
        const size_t np = xs.size();
        for (size_t i = 0; i < np; ++i) {
            const size_t j = (i + 1 == np) ? 0 : i + 1;
            sum += xs[i] * ys[j] - xs[j] * ys[i];
        }
        areas[kv.first] = sum / 2.0;
    }
    return areas;
}

// MassSolverBoxOutlet::calculateMass — MassSolverBoxOutlet.cpp:42-72
static void boxOutlet(Sim& s) {
    auto rescale = [&](size_t n) {
        const double sc = 1.0 / sumSlots9(&s.f[n * 9]);
        for (int d = 0; d < 9; ++d) s.f[n * 9 + d] *= sc;
        for (int k = 0; k < s.S; ++k)
            for (int d = 0; d < 5; ++d) s.g[((size_t)k * s.L + n) * 5 + d] *= sc;
    };
    for (int y = 0; y < s.ny; ++y) rescale(s.idx(0, y));
    for (int x = 0; x < s.nx; ++x) rescale(s.idx(x, 0));
}

// LbibMembraneTension: tutorial_01_BioSolverMembraneTension.cpp:40-74 with
// the force magnitude and frequency as parameters.
static void bioTension(Sim& s) {
    if (s.currentIteration % s.tension.frequency != 0) return;
    for (auto& kv : s.forcemap) {
        auto& v = kv.second;
        v.erase(std::remove_if(v.begin(), v.end(), [](const Force& f) { return f.type == 6; }), v.end());
    }
    for (int ci : s.conns) {
        const Conn& c = s.pool[ci];
        Force a{6, c.id1, c.id2, s.tension.force, 0, 0, 0};
        Force b{6, c.id2, c.id1, s.tension.force, 0, 0, 0};
        s.forcemap[c.id1].push_back(a);
        s.forcemap[c.id2].push_back(b);
    }
}

// LbibAreaRegulator: tutorial_01_BioSolverAreaRegulator.cpp:44-99 with a
// per-cell target of factor x the first measured area and a proportional
// gain relative to the target.
static void bioArea(Sim& s) {
    std::map<unsigned, double> areas = computeAreas(s);
    for (auto& kv : areas)
        if (s.targetArea.find(kv.first) == s.targetArea.end()) s.targetArea[kv.first] = s.area.factor * kv.second;
    std::map<unsigned, double> src;
    for (auto& kv : areas) {
        const double tgt = s.targetArea[kv.first];
        double r = s.area.strength * (tgt - kv.second) / tgt;
        if (r > s.area.maxsource) r = s.area.maxsource;
        else if (r < -s.area.maxsource) r = -s.area.maxsource;
        src[kv.first] = r;
    }
    for (size_t n = 0; n < s.L; ++n) {
        const unsigned d = s.dom[n];
        if (d != 0) {
            auto it = src.find(d);
            s.rhoToAdd[n] = 0.0;
            s.rhoToAdd[n] += (it == src.end() ? 0.0 : it->second);
        }
    }
}

// ---------------------------------------------------------------------------
// Construction and the time step

static void init(Sim& s, const std::string& params, const std::string& geom,
                 const std::string& force, const std::string& plugins) {
    loadParameters(s, params);
    if (s.nx <= 0 || s.ny <= 0) fail(ERR_INPUT, "bad lattice size");
    s.L = (size_t)s.nx * s.ny;
    s.f.assign(s.L * 9, 0.0);
    s.g.assign((size_t)s.S * s.L * 5, 0.0);
    s.ux.assign(s.L, 0.0); s.uy.assign(s.L, 0.0);
    s.frx.assign(s.L, 0.0); s.fry.assign(s.L, 0.0);
    s.rhoToAdd.assign(s.L, 0.0);
    s.dom.assign(s.L, 0); s.ctype.assign(s.L, 0);
    s.bn.assign(s.L * 5, -1);
    loadPlugins(s, plugins);
    // Geometry(file) then GeometryHandler(geometry): GeometryHandler.cpp:51-56
    loadGeometry(s, geom);
    cureLattice(s);
    // SimulationRunner::initSolvers — SimulationRunner.cpp:290-306
    for (size_t n = 0; n < s.L; ++n) {
        s.f[n * 9 + T] = 1.0;   // FluidSolver::initSolver — FluidSolver.cpp:50-60
        fluidCollide(s, n);
        for (int k = 0; k < s.S; ++k) cdeInit(s, k, n);
    }
    loadForces(s, force);
}

// SimulationRunner::runSimulation loop body — SimulationRunner.cpp:72-99
static void step(Sim& s) {
    calculateForce(s);
    distributeForce(s);
    for (size_t n = 0; n < s.L; ++n) {
        fluidAdvect(s, n);
        for (int k = 0; k < s.S; ++k) cdeAdvect(s, k, n);
    }
    for (size_t n = 0; n < s.L; ++n) {
        fluidCollide(s, n);
        for (int k = 0; k < s.S; ++k) cdeCollide(s, k, n);
    }
    collectVelocity(s);
    moveLattice(s);
    while (remeshOnce(s)) {}
    if (s.currentIteration % 10 == 0) {
        s.forcemap.clear();
        coarsen(s);
    }
    if (s.outlet) boxOutlet(s);
    for (int b : s.bioOrder) {
        if (b == 1) bioTension(s);
        else if (b == 2) bioArea(s);
    }
    s.currentIteration++;
}

}  // namespace orc

// ---------------------------------------------------------------------------
// C ABI for the test harness (ctypes).

using orc::Sim;

struct OrcHandle {
    Sim s;
    int err = 0;
    std::string msg;
};

extern "C" {

void* orc_create(const char* params, const char* geom, const char* force, const char* plugins) {
    OrcHandle* h = new OrcHandle();
    try {
        orc::init(h->s, params, geom, force ? force : "", plugins ? plugins : "");
    } catch (const orc::Fail& f) {
        h->err = f.code; h->msg = f.msg;
    } catch (const std::exception& e) {
        h->err = orc::ERR_INPUT; h->msg = e.what();
    }
    return h;
}

void orc_destroy(void* p) { delete static_cast<OrcHandle*>(p); }

int orc_error(void* p, char* buf, int len) {
    OrcHandle* h = static_cast<OrcHandle*>(p);
    if (buf && len > 0) { std::snprintf(buf, len, "%s", h->msg.c_str()); }
    return h->err;
}

int orc_step(void* p, int nsteps) {
    OrcHandle* h = static_cast<OrcHandle*>(p);
    if (h->err) return h->err;
    try {
        for (int i = 0; i < nsteps; ++i) orc::step(h->s);
    } catch (const orc::Fail& f) {
        h->err = f.code; h->msg = f.msg;
    } catch (const std::exception& e) {
        h->err = orc::ERR_INPUT; h->msg = e.what();
    }
    return h->err;
}

// sizes[0..7] = nx, ny, S, M (membrane nodes), C (connections), currentIteration, perturbCount, reinitCount
void orc_sizes(void* p, long long* sizes) {
    const Sim& s = static_cast<OrcHandle*>(p)->s;
    sizes[0] = s.nx; sizes[1] = s.ny; sizes[2] = s.S;
    sizes[3] = (long long)s.nodes.size(); sizes[4] = (long long)s.conns.size();
    sizes[5] = s.currentIteration; sizes[6] = (long long)s.perturbCount; sizes[7] = (long long)s.reinitCount;
}

// Lattice fields in the reference's layout: f[L][9] slots, g[S][L][5] slots,
// vel/force[L][2], dom/ctype[L], rhoToAdd[L].
void orc_get_lattice(void* p, double* f, double* g, double* vel, double* force,
                     unsigned* dom, unsigned* ctype, double* rhoToAdd) {
    const Sim& s = static_cast<OrcHandle*>(p)->s;
    if (f) std::memcpy(f, s.f.data(), s.f.size() * sizeof(double));
    if (g) std::memcpy(g, s.g.data(), s.g.size() * sizeof(double));
    for (size_t n = 0; n < s.L; ++n) {
        if (vel) { vel[2 * n] = s.ux[n]; vel[2 * n + 1] = s.uy[n]; }
        if (force) { force[2 * n] = s.frx[n]; force[2 * n + 1] = s.fry[n]; }
        if (dom) dom[n] = s.dom[n];
        if (ctype) ctype[n] = s.ctype[n];
        if (rhoToAdd) rhoToAdd[n] = s.rhoToAdd[n];
    }
}

// Membrane nodes in id order: ids[M], state[M][6] = x, y, vx, vy, fx, fy.
void orc_get_membrane(void* p, unsigned* ids, double* state) {
    const Sim& s = static_cast<OrcHandle*>(p)->s;
    size_t i = 0;
    for (auto& kv : s.nodes) {
        ids[i] = kv.first;
        const orc::GNode& g = kv.second;
        double* o = state + 6 * i;
        o[0] = g.x; o[1] = g.y; o[2] = g.vx; o[3] = g.vy; o[4] = g.fx; o[5] = g.fy;
        ++i;
    }
}

// Connections in vector order: conn[C][3] = id1, id2, domain.
void orc_get_connections(void* p, unsigned* conn) {
    const Sim& s = static_cast<OrcHandle*>(p)->s;
    size_t i = 0;
    for (int ci : s.conns) {
        conn[3 * i] = s.pool[ci].id1; conn[3 * i + 1] = s.pool[ci].id2; conn[3 * i + 2] = s.pool[ci].domain;
        ++i;
    }
}

// Cell areas (shoelace over each ring): dom[k], area[k]; returns the count.
int orc_areas(void* p, unsigned* dom, double* area, int cap) {
    const Sim& s = static_cast<OrcHandle*>(p)->s;
    auto a = orc::computeAreas(s);
    int i = 0;
    for (auto& kv : a) {
        if (i < cap) { dom[i] = kv.first; area[i] = kv.second; }
        ++i;
    }
    return i;
}

// Overwrite lattice state (for stage-level parity tests).
void orc_set_lattice(void* p, const double* f, const double* g, const double* force) {
    Sim& s = static_cast<OrcHandle*>(p)->s;
    if (f) std::memcpy(s.f.data(), f, s.f.size() * sizeof(double));
    if (g) std::memcpy(s.g.data(), g, s.g.size() * sizeof(double));
    if (force)
        for (size_t n = 0; n < s.L; ++n) { s.frx[n] = force[2 * n]; s.fry[n] = force[2 * n + 1]; }
}

// Lattice-only step with the current force field and domain ids held fixed:
// advect, collide (fluid then species), optional box outlet, iteration++.
int orc_lattice_step(void* p, int nsteps, int outlet) {
    OrcHandle* h = static_cast<OrcHandle*>(p);
    Sim& s = h->s;
    for (int i = 0; i < nsteps; ++i) {
        for (size_t n = 0; n < s.L; ++n) {
            orc::fluidAdvect(s, n);
            for (int k = 0; k < s.S; ++k) orc::cdeAdvect(s, k, n);
        }
        for (size_t n = 0; n < s.L; ++n) {
            orc::fluidCollide(s, n);
            for (int k = 0; k < s.S; ++k) orc::cdeCollide(s, k, n);
        }
        if (outlet) orc::boxOutlet(s);
        s.currentIteration++;
    }
    return 0;
}

double orc_fastcos(double x) { return orc::fastCos(x); }
double orc_delta(double dx, double dy) { return orc::delta(dx, dy); }

}  // extern "C"
