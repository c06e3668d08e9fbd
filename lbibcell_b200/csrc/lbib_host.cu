// lbib_host.cu — host runtime of lbibcell_b200: loaders for the reference's
// text formats, the device-resident simulation handle, the staged time step
// and the C ABI declared in include/lbibcell.h.
//
// The time step is a fixed sequence of stage kernels on one stream (the order
// of SimulationRunner::runSimulation, SimulationRunner.cpp:72-99).  Events that
// only the host can handle — the reference's random perturbation of
// positions (two std::mt19937(1) streams, GeometryNode.cpp:153-158 and
// Connection.cpp:332-337), remeshing, coarsening — are detected on the device,
// which then sets a halt word: every later stage kernel returns at once, the
// host reads the status after the batch, applies the event in the reference's
// order and resumes the step at the stage after the one that halted.  Steps
// without such events run with no host round trip.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <cub/cub.cuh>

#include "../../include/lbibcell.h"
#include "kernels.cuh"
#include "lattice_math.cuh"
#include "vtk_io.h"

namespace lbib {


struct HostFail {
    int code;
    std::string msg;
    long long index;
};

[[noreturn]] static void fail(int code, const std::string& m, long long index = -1) {
    throw HostFail{code, m, index};
}

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) ::lbib::fail(::lbib::ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct HConn {
    uint32_t id1, id2, dom;
    std::string desc;
};

// Position of each node id in a node array: a dense table over the ids when
// they are compact (the usual case: ids 1..n growing by remeshing), else a
// binary search over the sorted (id, position) pairs.  at() throws
// std::out_of_range for an absent id, as std::map::at does.
struct IdIndex {
    std::vector<int> dense;
    std::vector<std::pair<uint32_t, int>> sorted;
    explicit IdIndex(const std::vector<uint32_t>& ids) {
        uint32_t mx = 0;
        for (uint32_t id : ids) mx = std::max(mx, id);
        if ((size_t)mx <= 8 * ids.size() + 1024) {
            dense.assign((size_t)mx + 1, -1);
            for (size_t i = 0; i < ids.size(); ++i) dense[ids[i]] = (int)i;
        } else {
            sorted.resize(ids.size());
            for (size_t i = 0; i < ids.size(); ++i) sorted[i] = {ids[i], (int)i};
            std::sort(sorted.begin(), sorted.end());
        }
    }
    // position of id, or -1
    int find(uint32_t id) const {
        if (sorted.empty()) return id < dense.size() ? dense[id] : -1;
        auto it = std::lower_bound(sorted.begin(), sorted.end(), std::make_pair(id, -1));
        return it != sorted.end() && it->first == id ? it->second : -1;
    }
    int at(uint32_t id) const {
        if (sorted.empty()) {
            if (id < dense.size() && dense[id] >= 0) return dense[id];
        } else {
            auto it = std::lower_bound(sorted.begin(), sorted.end(), std::make_pair(id, -1));
            if (it != sorted.end() && it->first == id) return it->second;
        }
        throw std::out_of_range("node id");
    }
};

struct HForce {
    uint32_t type, id1, id2;
    double p[4];
};

// Initial conditions set on the host (the rest by the init kernels).
enum InitStyle {
    INIT_KERNEL = 0,  // init64 / init32
    INIT_ZERO,        // CDESolverD2Q5BMP.cpp:45-50
    INIT_T2,          // tutorial_02_CDESolverD2Q5_R.cpp:44-59: (1 + U(-0.01, 0.01)) / 5 per slot, 0 outside cells
    INIT_SCHNAK,      // SchnakenbergD2Q5u.cpp:43-58: 0.2 (1 + U(-0.01, 0.01)) per node, 0 outside cells
    INIT_DIRAC        // DiracD2Q5.cpp:39-66: the 2D heat kernel at t = 50, D = 0.04, centred at (32, 32)
};

struct Species {
    std::string name;
    SpeciesConst c;
    double init = 0.0;
    std::map<uint32_t, double> source;
    std::string partnerName;
    int initStyle = INIT_KERNEL;
};

template <typename T>
static T* dalloc(size_t n) {
    T* p = nullptr;
    if (n == 0) n = 1;
    CK(cudaMalloc(&p, n * sizeof(T)));
    return p;
}

// Device state of a differentiated run (lbib_diff_*): the snapshot it starts
// from, the checkpoints of the forward pass, one segment of recomputed states,
// the adjoint planes and the gradient accumulators.  A "state" is the fluid
// planes (9*L) followed by the species planes (S*5*L), FP64.
struct DiffCtx {
    int T = 0, K = 0, nSeg = 0;
    size_t stateBytes = 0;    // (9 + 5 S) L values of the lattice precision
    int rs = 8;               // bytes of a stored value: 8 (FP64) or 4 (FP32-shifted)
    char* x0 = nullptr;       // state at step 0
    char* u0 = nullptr;       // velocity and force planes at step 0 (restored by lbib_diff_end), 4*L values
    char* ck = nullptr;       // states at steps K, 2K, ... (nSeg - 1 of them)
    char* seg = nullptr;      // states base+1 .. base+K-1 of the segment being reversed
    // A second segment buffer for FP32 states, when the device has room for
    // it: the reverse pass then recomputes the next segment on `recStream`
    // while the adjoint steps of the current one run on `adjStream` (higher
    // priority).  adjoint_512, T = 2000, K = 100: FP32 states 58.5 -> 52.6 ms
    // per reverse pass; FP64 states 72.7 -> 76.5 ms (the FP64 recompute slows
    // the FP64 adjoint steps more than it saves), so FP64 runs stay serial.
    char* seg2 = nullptr;
    cudaStream_t recStream = nullptr, adjStream = nullptr;
    cudaEvent_t evRec[2] = {nullptr, nullptr}, evAdj[2] = {nullptr, nullptr}, evFork = nullptr, evJoin[2] = {nullptr, nullptr};
    char* fin = nullptr;      // the final state of the forward pass
    float* P[2] = {nullptr, nullptr};  // adjoint planes, (9 + 5 S) L each
    double* G = nullptr;      // 2*L
    double* force = nullptr;  // 2*L spread of the parameter forces
    float* force32 = nullptr; // 2*L the same for the FP32-shifted forward
    double* fxp = nullptr;    // membrane forces (parameters), Mcap each
    double* fyp = nullptr;
    double* gfx = nullptr;
    double* gfy = nullptr;
    double* srcTab = nullptr; // S*nDomains
    double* seed = nullptr;   // S*L
    double* grad = nullptr;   // 1 + S + S*nDomains
    double* racc = nullptr;   // S*L
    double* part = nullptr;   // adjoint blocks * (1 + S)
    double* massTab = nullptr;  // nDomains: the run's per-domain mass source (rhoToAdd)
    double* macc = nullptr;     // L: dL/d rhoToAdd per node
    double* seedF = nullptr;    // 9*L: dL/d(final fluid state), natural direction order
    bool massUsed = false;      // the run applies massTab (an area regulator, or lbib_diff_mass)
    bool haveSeedF = false;
    std::vector<double> gmass;  // dL/d massTab of the last backward pass
    Status* st = nullptr;
    double tauF = 1.0;
    double tau[kMaxSpecies] = {1.0, 1.0, 1.0};
    int outlet = 0;
    unsigned it0 = 0;
    bool forwardDone = false;
    bool lastSegKept = false;   // the forward left the last segment's states in seg
    bool backwardDone = false;  // gfx / gfy hold the last reverse pass's membrane-force gradient
    // Moving membrane nodes (lbib_diff_motion): the positions after every
    // step, pos + t * 2 * M = X after step t then Y (t = 0: the snapshot's),
    // and the reverse pass's per-node and per-step planes.
    bool motion = false;
    int M = 0;                  // the membrane's node count at lbib_diff_begin
    double* pos = nullptr;      // (T + 1) * 2 * M
    double* lam = nullptr;      // 2 * M: dL/dX after the step being reversed
    double* seedX = nullptr;    // 2 * M: dL/dX after the final step
    bool haveSeedX = false;
    double* gu = nullptr;       // 2 * L: dL/d(post-collision velocity) of one step
    double* uo = nullptr;       // 2 * L: the post-collision velocity of one step
    double* posAt(int t) const { return pos + (size_t)t * 2 * M; }
    char* state(int i) const { return i == 0 ? x0 : ck + (size_t)(i - 1) * stateBytes; }
    ~DiffCtx() {
        auto fr = [](void* p) { if (p) cudaFree(p); };
        fr(x0); fr(u0); fr(ck); fr(seg); fr(fin); fr(P[0]); fr(P[1]); fr(G); fr(force); fr(force32); fr(fxp);
        fr(fyp); fr(gfx); fr(gfy);
        fr(srcTab); fr(seed); fr(grad); fr(racc); fr(part); fr(st); fr(massTab); fr(macc); fr(seedF); fr(seg2);
        fr(pos); fr(lam); fr(seedX); fr(gu); fr(uo);
        for (cudaEvent_t e : {evRec[0], evRec[1], evAdj[0], evAdj[1], evFork, evJoin[0], evJoin[1]})
            if (e) cudaEventDestroy(e);
        if (recStream) cudaStreamDestroy(recStream);
        if (adjStream) cudaStreamDestroy(adjStream);
    }
};

// The status allocation (device, and its pinned host copy): the status word,
// the membrane counts (Topo) and the per-cell areas, so that one copy reads
// all three back after a step.
constexpr size_t kTopoOffset = (sizeof(Status) + 63) / 64 * 64;
constexpr size_t kAreaOffset = kTopoOffset + (sizeof(Topo) + 63) / 64 * 64;

struct Handle {
    // parameters
    int nx = 0, ny = 0, S = 0;
    size_t L = 0;
    int precision = 0;
    int device = 0;
    double tauF = 1.0;
    int forceModel = FM_LUO;  // the fluid's force model (plugin file line "ForceModel <name>")
    unsigned iteration = 0, iterations = 0, reportStep = 1;
    std::vector<Species> sp;
    bool outlet = false;
    // 1 tension, 2 area regulator, 3 cell junctions, 4 cell division (host),
    // 5 differentiation (host), 6 growth
    std::vector<int> bio;
    double tensionForce = 0.01;
    unsigned tensionFreq = 10;
    // tutorial_01_BioSolverCellJunction.cpp:37-41
    double junctionRadius = 1.0, junctionK = 0.02, junctionL0 = 0.5;
    double areaFactor = 1.2, areaStrength = 0.01, areaMax = 0.004;
    bool areaTutorial = false;   // tutorial_01_BioSolverAreaRegulator's rule
    int diffSpecies = -1;        // the species differentiation reads
    bool diffInit = false;       // its one-time reset of the cell-type map done
    int growthR = -1, growthL = -1;
    bool growthConst = false;    // BioSolverGrowth (constant source) rather than tutorial_02's
    double* massNode = nullptr;  // per-node mass source (growth)

    // lattice buffers
    void* f[2] = {nullptr, nullptr};
    void* g[2] = {nullptr, nullptr};
    void* u = nullptr;
    void* force = nullptr;
    uint32_t* dom = nullptr;
    int cur = 0;
    int nDomains = 1;
    double* massTab = nullptr;
    double* srcTab = nullptr;
    uint32_t* ctypeTab = nullptr;
    std::vector<uint32_t> ctypeHost;
    bool cellTypesCopied = false;

    // membrane (host mirror of the topology; positions live on the device)
    std::vector<uint32_t> ids;
    std::vector<HConn> conns;
    std::map<uint32_t, std::vector<HForce>> forcemap;
    // The force list as loaded (from the force file or a restart) holds no
    // records: until the first deleteAllForces, tension renewals may rebuild it
    // whole.  forceListIt: the iteration of the first step on that list.
    bool forcesPureAtLoad = true;
    unsigned forceListIt = 0;
    ForceScratch fs{};
    int fsMcap = 0, fsFcap = 0;  // capacities the scratch was allocated for
    bool fsQuery = false;        // the scratch holds the cell-list buffers
    int keepRecords = 0;         // force records the host re-uploads after a topology upload
    MembraneDev m{};
    int Mcap = 0, Ccap = 0, Fcap = 0, cellCap = 0;
    int* outPos = nullptr;
    int* inPos = nullptr;
    double* area = nullptr;
    double* target = nullptr;
    unsigned long long* areaAcc = nullptr;  // fixed-point area sums of FP32-shifted runs
    std::vector<double> targetHost;  // per cell, survives ring rebuilds
    std::vector<uint32_t> ringDomHost;

    TileDev tiles{};
    CrossDev cross{};
    TopoDev td{};
    std::vector<std::string> descTable;  // boundary-descriptor strings of the connections
    NfSpec* nfTabDev = nullptr;          // boundary solvers per descriptor (device), nullptr: none
    Status* st = nullptr;
    Status* stHost = nullptr;
    Topo* topoHost = nullptr;   // pinned copy of the device counts, read with the status word
    bool ringsCurrent = false;  // the device's ring order matches the topology (no rebuild needed)
    // per-cell areas read back with the status word at the end of lbib_step
    // when its bio stage formed them (the area regulator): the host copy's
    // area part; areaFresh: they are the areas of the current state (any
    // other API call clears it); statusWithAreas: the next status read takes
    // the areas along
    double* areaPinned = nullptr;
    bool areaFresh = false;
    bool statusWithAreas = false;
    // LBIB_FULL_HOST_EVENTS=1 at creation: host events take the whole
    // membrane to the host (the reference's algorithms on a full copy) instead
    // of the listed nodes and connections only (a cross-check of the latter)
    bool fullHostEvents = false;
    bool workAfterEvB = false;  // GPU work was issued after the step loop's last timing event
    // the device status word carries on from the last batch of steps (no
    // halt, nothing wrote it since): the next batch needs no reset; its
    // first step counts the batch's last step (pad[0] was lastPad0)
    bool statusContinues = false;
    int lastPad0 = 0;
    cudaStream_t stream = nullptr;

    std::mt19937 genNode{1};
    std::mt19937 genConn{1};
    std::uniform_real_distribution<> dis{-kPERTURBATION, kPERTURBATION};
    // cell division (bio kind 4, the last bio solver): every divisionFreq-th
    // iteration, cells larger than divisionMax split; policy 0 = across the
    // longest axis, 1 = along a random direction (generator seeded 1)
    int divisionPolicy = 0;
    unsigned divisionFreq = 100;
    double divisionMax = 380.0;
    // LbibCellDivision: threshold divisionFactor x the cell's reference area
    // (its area at the solver's first look; daughters inherit it); 0 = the
    // fixed divisionMax of the reference's plugins
    double divisionFactor = 0.0;
    std::map<uint32_t, double> divisionRef;
    std::mt19937 genDiv{1};

    long long hostEvents = 0;
    long long launches = 0;
    // CUDA graphs of one step, keyed by (buffer parity, coarsening step, bio
    // solvers' force-list operations); rebuilt when a buffer is reallocated
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;
    };
    std::map<int, StepGraph> graphs;
    bool useGraphs = true;
    long long graphEpoch = 0, graphBuiltEpoch = 0;  // kernels launched by the last lbib_step / lbib_lattice_step
    long long stepsDone = 0;

    // errors
    int err = 0;
    std::string msg;
    long long errIndex = -1;

    // timing
    bool profiling = false;
    cudaEvent_t evA = nullptr, evB = nullptr;
    std::vector<cudaEvent_t> kEvents;
    double lastTotalMs = 0, lastCollideMs = 0;
    long long lastCollideLaunches = 0;

    DiffCtx* diff = nullptr;

    ~Handle();
};

Handle::~Handle() {
    cudaSetDevice(device);
    delete diff;
    auto fr = [](void* p) { if (p) cudaFree(p); };
    for (int i = 0; i < 2; ++i) { fr(f[i]); fr(g[i]); }
    fr(u); fr(force); fr(dom); fr(massTab); fr(massNode); fr(srcTab); fr(ctypeTab);
    fr(m.x); fr(m.y); fr(m.ox); fr(m.oy); fr(m.vx); fr(m.vy); fr(m.fx); fr(m.fy); fr(m.id); fr(m.bx); fr(m.by);
    fr(m.prev); fr(m.next); fr(m.ca); fr(m.cb); fr(m.cdom); fr(m.foff); fr(m.ftype); fr(m.fpartner); fr(m.fpar);
    fr(m.ringStart); fr(m.ringNode); fr(m.ringDom);
    fr(outPos); fr(inPos); fr(target); fr(areaAcc);  // area lives in the status allocation
    fr(tiles.count); fr(tiles.fill); fr(tiles.start); fr(tiles.list); fr(tiles.scanTmp); fr(tiles.slots);
    fr(cross.bnDist); fr(cross.bnConn); fr(cross.bnDom); fr(cross.wDom); fr(cross.mark);
    fr(cross.changedNode); fr(cross.changedDom); fr(cross.perturbList); fr(cross.reinitDone); fr(cross.waitList);
    fr(cross.nWait);
    fr(cross.recKey); fr(cross.recConn); fr(cross.recDom); fr(cross.recDist); fr(cross.nfKeys); fr(cross.nfD);
    fr(cross.nfSpec); fr(cross.nfU); fr(cross.nfN); fr(nfTabDev);
    fr(cross.bounceW); fr(cross.bounceS); fr(cross.bounceKeys); fr(cross.bounceN);
    fr(m.cdesc);  // m.topo lives in the status allocation
    fr(td.flag); fr(td.rank); fr(td.nflag); fr(td.nrank); fr(td.ca2); fr(td.cb2); fr(td.cdom2); fr(td.cdesc2);
    fr(td.dalt); fr(td.id2); fr(td.prev2); fr(td.next2); fr(td.inConn); fr(td.outConn); fr(td.removed);
    fr(td.connAlive); fr(td.ncA); fr(td.ncB); fr(td.ncDom); fr(td.ncDesc); fr(td.ncAlive); fr(td.cellOfDom);
    fr(td.firstConn); fr(td.cellCount); fr(td.cellStart); fr(td.cellFill); fr(td.members); fr(td.succ); fr(td.rngList);
    fr(td.dist); fr(td.startNode); fr(td.scanTmp);
    fr(st);
    if (stHost) cudaFreeHost(stHost);  // topoHost lives in the same block
    if (evA) cudaEventDestroy(evA);
    if (evB) cudaEventDestroy(evB);
    for (auto e : kEvents) cudaEventDestroy(e);
    for (auto& kv : graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    fr(fs.foffS); fr(fs.ftypeS); fr(fs.fpartnerS); fr(fs.fparS); fr(fs.cnt); fr(fs.scanTmp);
    fr(fs.binKey); fr(fs.binKeySorted); fr(fs.binIdx); fr(fs.binIdxSorted); fr(fs.sortTmp); fr(fs.closest);
    fr(fs.binStart); fr(fs.binHead); fr(fs.binNext); fr(fs.linkKey); fr(fs.linkPrevM);
    fr(fs.inCnt); fr(fs.inOff); fr(fs.inList); fr(fs.inFill);
    if (stream) cudaStreamDestroy(stream);
}

// ---------------------------------------------------------------------------
// Loaders for the reference formats.

// GlobalSimulationParameters::loadGlobalSimulationParameters (GlobalSimulationParameters.cpp:34-72).
// Species are kept in the parameter map's (alphabetical) order.
static void load_parameters(Handle& h, const std::string& fn) {
    std::ifstream in(fn);
    if (!in.is_open()) fail(ERR_INPUT, "Cannot find the parameter file.");
    std::string line;
    std::map<std::string, double> cdes;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ls(line);
        std::string key;
        ls >> key;
        if (key == "CurrentIterations:") ls >> h.iteration;
        else if (key == "Iterations:") ls >> h.iterations;
        else if (key == "ReportStep:") ls >> h.reportStep;
        else if (key == "SizeX:") ls >> h.nx;
        else if (key == "SizeY:") ls >> h.ny;
        else if (key == "tauFluid:") ls >> h.tauF;
        else if (key == "CDESolvers:") {
            std::string nm; double tau;
            while (ls >> nm >> tau) cdes[nm] = tau;
        } else fail(ERR_INPUT, "An unknown parameter was passed in the global Parameter file");
    }
    // The reference's CDE solvers by name (libs/LbmLib/src/solver/CDESolver),
    // and the Lbib species plugins (any other name): reaction kind, partner
    // species, reinitialise() variant, deltaT and initial condition.
    for (auto& kv : cdes) {
        Species s;
        s.name = kv.first;
        s.c.tau = kv.second;
        s.c.decay = 0.0;
        s.c.partner = -1;
        s.c.reinit = RI_BASE;
        s.c.dt = 1.0;
        s.c.hill = 0.0;
        s.c.bounce = 0;
        const std::string& nm = kv.first;
        if (nm == "CDESolverD2Q5") {
            s.c.kind = RX_NONE;
        } else if (nm == "tutorial_01_CDESolverD2Q5_SIGNAL" || nm == "CDESolverD2Q5HH") {
            s.c.kind = RX_SIGNAL;
            s.c.reinit = RI_ALL4;
        } else if (nm == "tutorial_02_CDESolverD2Q5_R" || nm == "tutorial_02_CDESolverD2Q5_L") {
            s.c.kind = nm.back() == 'R' ? RX_T2_R : RX_T2_L;
            s.c.reinit = RI_ALL4;
            s.partnerName = nm.back() == 'R' ? "tutorial_02_CDESolverD2Q5_L" : "tutorial_02_CDESolverD2Q5_R";
            s.initStyle = INIT_T2;
        } else if (nm == "SchnakenbergD2Q5u" || nm == "SchnakenbergD2Q5v") {
            s.c.kind = nm.back() == 'u' ? RX_SCHNAK_U : RX_SCHNAK_V;
            s.c.reinit = RI_DIAG;
            s.c.dt = 20.0 / (double)h.iterations;  // SchnakenbergD2Q5u.cpp:57
            s.partnerName = nm.back() == 'u' ? "SchnakenbergD2Q5v" : "SchnakenbergD2Q5u";
            s.initStyle = INIT_SCHNAK;
        } else if (nm == "CDESolverD2Q5BMP") {
            s.c.kind = RX_BMP;
            s.c.reinit = RI_ALL4;
            s.c.hill = std::pow(0.01, 4.0);  // pow(k_hill, n_hill), CDESolverD2Q5BMP.cpp:113-117
            s.partnerName = "CDESolverD2Q5HH";
            s.initStyle = INIT_ZERO;
        } else if (nm == "DiracD2Q5") {
            // DiracD2Q5.cpp: CDESolverD2Q5's collide without reaction; advect
            // keeps the populations of links with a boundary node (:166-180);
            // reinitialise from E,N,W,S without a boundary node, else the four
            // diagonals, C/4 per slot (:182-228)
            s.c.kind = RX_NONE;
            s.c.reinit = RI_DIAG;
            s.c.bounce = 1;
            s.initStyle = INIT_DIRAC;
        } else if (nm.compare(0, 4, "Lbib") == 0) {
            s.c.kind = RX_LINEAR;
        } else {
            // the D2Q4 solvers are not built
            fail(ERR_INPUT, "unknown or unsupported CDE solver " + nm);
        }
        h.sp.push_back(s);
    }
    h.S = (int)h.sp.size();
    if (h.S > kMaxSpecies) fail(ERR_INPUT, "at most 3 CDE species are supported");
    for (auto& s : h.sp) {
        if (s.partnerName.empty()) continue;
        for (int j = 0; j < h.S; ++j)
            if (h.sp[j].name == s.partnerName) s.c.partner = j;
        // PhysicalNode::getCDESolverSlow throws for a solver the node lacks
        if (s.c.partner < 0) fail(ERR_INPUT, s.name + " needs the CDE solver " + s.partnerName);
    }
    if (h.nx < 8 || h.ny < 8) fail(ERR_INPUT, "lattice too small");
}

static void load_plugins(Handle& h, const std::string& fn) {
    if (fn.empty()) return;
    std::ifstream in(fn);
    if (!in.is_open()) fail(ERR_INPUT, "Cannot find the plugin file.");
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ls(line);
        std::string kind, name;
        ls >> kind >> name;
        std::map<std::string, double> kv;
        if (kind == "MassSolver") {
            if (name == "MassSolverBoxOutlet") h.outlet = true;
            else fail(ERR_INPUT, "unknown mass solver " + name);
        } else if (kind == "ForceModel") {
            // FluidSolver's force model, a base class chosen when the
            // reference is compiled (FluidSolver.hpp:41); here per handle
            if (name == "Luo1993ForceModel") h.forceModel = FM_LUO;
            else if (name == "GuoZhengShi2002ForceModel") h.forceModel = FM_GUO;
            else if (name == "GuoZhengShi2002ForceModelCorrected") h.forceModel = FM_GUO_CORRECTED;
            else fail(ERR_INPUT, "unknown force model " + name);
        } else if (kind == "BioSolver") {
            std::string k; double v;
            while (ls >> k >> v) kv[k] = v;
            if (name == "LbibMembraneTension") {
                h.bio.push_back(1);
                if (kv.count("force")) h.tensionForce = kv["force"];
                if (kv.count("frequency")) h.tensionFreq = (unsigned)kv["frequency"];
                if (h.tensionFreq == 0) fail(ERR_INPUT, "tension frequency must be positive");
            } else if (name == "tutorial_01_BioSolverMembraneTension" ||
                       name == "tutorial_02_BioSolverMembraneTension" || name == "BioSolverMembraneTension") {
                // the same renewal with the constants of each file (FREQUENCY 10; FORCE
                // 0.01, 0.005, 0.02: tutorial_01_BioSolverMembraneTension.cpp:34-35,
                // tutorial_02_...:34-35, BioSolverMembraneTension.cpp:34-35)
                h.bio.push_back(1);
                h.tensionFreq = 10;
                h.tensionForce = name == "tutorial_01_BioSolverMembraneTension"   ? 0.01
                                 : name == "tutorial_02_BioSolverMembraneTension" ? 0.005
                                                                                  : 0.02;
            } else if (name == "tutorial_01_BioSolverAreaRegulator") {
                // tutorial_01_BioSolverAreaRegulator.cpp:34-37: TARGETAREA 200, KP 1e-5, MAXSOURCE 0.004
                h.bio.push_back(2);
                h.areaTutorial = true;
                h.areaFactor = 200.0;
                h.areaStrength = 0.00001;
                h.areaMax = 0.004;
            } else if (name == "tutorial_01_BioSolverDifferentiation" || name == "BioSolverDifferentiation") {
                // tutorial_01_BioSolverDifferentiation.cpp:33-84 (host, every 100th iteration)
                h.bio.push_back(5);
            } else if (name == "tutorial_02_BioSolverGrowth" || name == "BioSolverGrowth") {
                // BioSolverGrowth.cpp:33-64: every node inside a cell gets 0.0025
                h.bio.push_back(6);
                h.growthConst = name == "BioSolverGrowth";
            } else if (name == "BioSolverEmpty") {
                // BioSolverEmpty.cpp:36-45 does nothing
            } else if (name == "tutorial_01_BioSolverCellJunction" || name == "tutorial_02_BioSolverCellJunction" ||
                       name == "BioSolverCellJunction" || name == "LbibCellJunction") {
                // the reference's solvers take no parameters; LbibCellJunction is
                // the same solver with radius, k and l0 from the plugin file
                h.bio.push_back(3);
                if (kv.count("radius")) h.junctionRadius = kv["radius"];
                if (kv.count("k")) h.junctionK = kv["k"];
                if (kv.count("l0")) h.junctionL0 = kv["l0"];
            } else if (name == "tutorial_01_BioSolverCellDivision" || name == "tutorial_02_BioSolverCellDivision" ||
                       name == "BioSolverCellDivision") {
                // tutorial_01_BioSolverCellDivision.cpp:33-36 (the plain one
                // divides along a random direction, BioSolverCellDivision.cpp:100-101)
                h.bio.push_back(4);
                h.divisionPolicy = name == "BioSolverCellDivision" ? 1 : 0;
            } else if (name == "LbibCellDivision") {
                // the tutorial_01 division (longest axis) with a per-cell
                // threshold: factor x the cell's reference area, every
                // `frequency` iterations
                h.bio.push_back(4);
                h.divisionPolicy = 0;
                h.divisionFactor = kv.count("factor") ? kv["factor"] : 2.0;
                h.divisionFreq = kv.count("frequency") ? (unsigned)kv["frequency"] : 100u;
                if (h.divisionFreq == 0 || !(h.divisionFactor > 0.0))
                    fail(ERR_INPUT, "LbibCellDivision needs a positive factor and frequency");
            } else if (name == "LbibAreaRegulator") {
                h.bio.push_back(2);
                h.areaTutorial = false;
                if (kv.count("factor")) h.areaFactor = kv["factor"];
                if (kv.count("strength")) h.areaStrength = kv["strength"];
                if (kv.count("maxsource")) h.areaMax = kv["maxsource"];
            } else fail(ERR_INPUT, "unknown bio solver " + name);
            if (h.bio.size() > 8) fail(ERR_INPUT, "more than 8 bio solvers");
            for (size_t q = 0; q + 1 < h.bio.size(); ++q)
                if (h.bio[q] == 4) fail(ERR_INPUT, "the cell-division solver must be the last bio solver");
            // the host bio solvers run after the device's step: none may precede a device one
            bool host = false;
            for (int b : h.bio) {
                if (b == 4 || b == 5) host = true;
                else if (host) fail(ERR_INPUT, "differentiation and cell division must follow the other bio solvers");
            }
        } else if (kind == "CDE") {
            std::string k; double v;
            while (ls >> k >> v) kv[k] = v;
            for (auto& s : h.sp)
                if (s.name == name) {
                    if (kv.count("init")) s.init = kv["init"];
                    if (kv.count("decay")) s.c.decay = kv["decay"];
                }
        } else if (kind == "CDESource") {
            uint32_t d; double r;
            while (ls >> d >> r)
                for (auto& s : h.sp)
                    if (s.name == name) s.source[d] = r;
        } else fail(ERR_INPUT, "unknown plugin line " + kind);
    }
}

// Checks of the bio solvers that read species or share state, once the
// parameter and plugin files are both read.
static void check_bio(Handle& h) {
    auto species = [&](const char* nm) {
        for (int k = 0; k < h.S; ++k)
            if (h.sp[k].name == nm) return k;
        // PhysicalNode::getCDESolverSlow throws for a solver the node lacks
        fail(ERR_INPUT, std::string("a bio solver needs the CDE solver ") + nm);
        return -1;
    };
    int count[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int b : h.bio) count[b]++;
    if (count[1] > 1 || count[2] > 1)
        fail(ERR_INPUT, "one membrane-tension and one area-regulator solver at most");
    if (count[5]) h.diffSpecies = species("tutorial_01_CDESolverD2Q5_SIGNAL");
    if (count[6]) {
        if (!h.growthConst) {
            h.growthR = species("tutorial_02_CDESolverD2Q5_R");
            h.growthL = species("tutorial_02_CDESolverD2Q5_L");
        }
        // FluidSolver::addMass overwrites: two mass sources would depend on their order
        if (count[2] || count[6] > 1) fail(ERR_INPUT, "two bio solvers set the mass source (growth, area regulator)");
    }
}

static bool has_junctions(const Handle& h) {
    return std::find(h.bio.begin(), h.bio.end(), 3) != h.bio.end();
}

// ForceSolver::addForce text format (ForceSolver.cpp:107-139; ForceStructs.hpp).
static void add_force_line(Handle& h, const std::string& line) {
    std::stringstream ls(line);
    HForce f{};
    ls >> f.type;
    switch (f.type) {
        case 0: case 7: ls >> f.id1 >> f.id2 >> f.p[0] >> f.p[1]; break;
        case 1: ls >> f.id1 >> f.p[0] >> f.p[1] >> f.p[2] >> f.p[3]; break;
        case 2: ls >> f.id1 >> f.p[0] >> f.p[1]; break;
        case 3: case 4: ls >> f.id1 >> f.p[0] >> f.p[1] >> f.p[2]; break;
        case 5: case 6: ls >> f.id1 >> f.id2 >> f.p[0]; break;
        default: fail(ERR_INPUT, "Invalid force solver type found.");
    }
    h.forcemap[f.id1].push_back(f);
}

// ---------------------------------------------------------------------------
// Host copies of the membrane arrays (used by the host-side events).

struct HostMembrane {
    std::vector<double> x, y, ox, oy, vx, vy, fx, fy;
    std::vector<double> bx, by;  // position at the last stencil binding
};

static void download_membrane(Handle& h, HostMembrane& hm) {
    const int M = h.m.M;
    hm.x.resize(M); hm.y.resize(M); hm.ox.resize(M); hm.oy.resize(M);
    hm.vx.resize(M); hm.vy.resize(M); hm.fx.resize(M); hm.fy.resize(M);
    hm.bx.resize(M); hm.by.resize(M);
    if (M == 0) return;
    const size_t b = sizeof(double) * M;
    CK(cudaMemcpyAsync(hm.x.data(), h.m.x, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.y.data(), h.m.y, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.ox.data(), h.m.ox, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.oy.data(), h.m.oy, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.vx.data(), h.m.vx, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.vy.data(), h.m.vy, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.fx.data(), h.m.fx, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.fy.data(), h.m.fy, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.bx.data(), h.m.bx, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(hm.by.data(), h.m.by, b, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
}

static void ensure_capacity(Handle& h, int M, int C, int F, int cells);

// Uploads node arrays, connections, ring order, neighbour indices and the
// force records, after any change of the host topology mirror.
static void upload_topology(Handle& h, const HostMembrane& hm, bool uploadForces) {
    const int M = (int)h.ids.size();
    const int C = (int)h.conns.size();
    const IdIndex index(h.ids);
    std::vector<int> ca(C), cb(C), prev(M, -1), next(M, -1), cdesc(C);
    std::vector<uint32_t> cdom(C);
    for (int c = 0; c < C; ++c) {
        ca[c] = index.at(h.conns[c].id1);
        cb[c] = index.at(h.conns[c].id2);
        cdom[c] = h.conns[c].dom;
        auto dt = std::find(h.descTable.begin(), h.descTable.end(), h.conns[c].desc);
        if (dt == h.descTable.end()) { h.descTable.push_back(h.conns[c].desc); dt = h.descTable.end() - 1; }
        cdesc[c] = (int)(dt - h.descTable.begin());
        next[ca[c]] = cb[c];
        prev[cb[c]] = ca[c];
    }
    for (int i = 0; i < M; ++i)
        if (prev[i] < 0 || next[i] < 0) fail(ERR_INPUT, "Geometry::checkGeometryIntegrity: open membrane", i);
    // rings: GeometryHandler::computeAreas (GeometryHandler.cpp:112-126):
    // per domain (ascending), start at the first connection with that domain
    // and follow the second node's outgoing connection.
    std::map<uint32_t, int> first;
    for (int c = 0; c < C; ++c)
        if (!first.count(cdom[c])) first[cdom[c]] = c;
    std::vector<int> outConn(M, -1);
    for (int c = 0; c < C; ++c) outConn[ca[c]] = c;
    std::vector<int> ringStart, ringNode;
    std::vector<uint32_t> ringDom;
    for (auto& kv : first) {
        ringStart.push_back((int)ringNode.size());
        ringDom.push_back(kv.first);
        int c = kv.second;
        int guard = 0;
        do {
            ringNode.push_back(cb[c]);
            c = outConn[cb[c]];
            if (++guard > C) fail(ERR_INPUT, "broken ring", kv.first);
        } while (c != kv.second);
    }
    ringStart.push_back((int)ringNode.size());
    const int cells = (int)ringDom.size();
    // force records
    std::vector<int> foff(M + 1, 0), ftype, fpart;
    std::vector<double> fpar;
    if (uploadForces) {
        for (int i = 0; i < M; ++i) {
            foff[i] = (int)ftype.size();
            auto it = h.forcemap.find(h.ids[i]);
            if (it == h.forcemap.end()) continue;
            for (const HForce& f : it->second) {
                ftype.push_back((int)f.type);
                int j = -1;
                if (f.type == 0 || f.type == 7 || f.type == 5 || f.type == 6) {
                    j = index.find(f.id2);
                }
                fpart.push_back(j);
                for (int q = 0; q < 4; ++q) fpar.push_back(f.p[q]);
            }
        }
        foff[M] = (int)ftype.size();
        // forces on ids that are not membrane nodes fail like nodes.at() would
        for (auto& kv : h.forcemap)
            if (!kv.second.empty() && index.find(kv.first) < 0) fail(ERR_FORCE_NODE, "Could not compute and set the forces.", kv.first);
    }
    ensure_capacity(h, M, C, 1, cells);
    // room for the loaded records plus the bio solvers' own: two tension records
    // per node, and with junctions up to two springs per node
    const int F = std::max((int)ftype.size(), h.keepRecords) + (has_junctions(h) ? 4 : 2) * h.Mcap;
    ensure_capacity(h, M, C, F, cells);
    h.m.M = M;
    h.m.C = C;
    h.m.nCells = cells;
    const size_t bd = sizeof(double) * M;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h.stream));
    };
    up(h.m.x, hm.x.data(), bd); up(h.m.y, hm.y.data(), bd);
    up(h.m.ox, hm.ox.data(), bd); up(h.m.oy, hm.oy.data(), bd);
    up(h.m.vx, hm.vx.data(), bd); up(h.m.vy, hm.vy.data(), bd);
    up(h.m.fx, hm.fx.data(), bd); up(h.m.fy, hm.fy.data(), bd);
    up(h.m.bx, hm.bx.data(), bd); up(h.m.by, hm.by.data(), bd);
    up(h.m.id, h.ids.data(), sizeof(uint32_t) * M);
    up(h.m.prev, prev.data(), sizeof(int) * M);
    up(h.m.next, next.data(), sizeof(int) * M);
    up(h.m.ca, ca.data(), sizeof(int) * C);
    up(h.m.cb, cb.data(), sizeof(int) * C);
    up(h.m.cdom, cdom.data(), sizeof(uint32_t) * C);
    up(h.m.cdesc, cdesc.data(), sizeof(int) * C);
    {
        // device counts, domain -> cell table, ring bookkeeping
        Topo tp{};
        tp.M = M; tp.C = C; tp.maxId = M ? h.ids.back() : 0u; tp.changed = 0;
        up(h.m.topo, &tp, sizeof(Topo));
        std::vector<int> cellOf(h.nDomains, -1);
        for (int c = 0; c < cells; ++c)
            if (ringDom[c] < (uint32_t)h.nDomains) cellOf[ringDom[c]] = c;
        if (!h.td.cellOfDom) {
            h.td.cellOfDom = dalloc<int>(h.nDomains);
            h.td.firstConn = dalloc<int>(h.nDomains);
            h.td.nDomains = h.nDomains;
        }
        up(h.td.cellOfDom, cellOf.data(), sizeof(int) * h.nDomains);
        std::vector<int> big(h.nDomains, 0x7fffffff);
        up(h.td.firstConn, big.data(), sizeof(int) * h.nDomains);
        h.td.nCellsCap = cells;
    }
    up(h.m.ringStart, ringStart.data(), sizeof(int) * ringStart.size());
    up(h.m.ringNode, ringNode.data(), sizeof(int) * ringNode.size());
    up(h.m.ringDom, ringDom.data(), sizeof(uint32_t) * cells);
    if (uploadForces) {
        up(h.m.foff, foff.data(), sizeof(int) * (M + 1));
        up(h.m.ftype, ftype.data(), sizeof(int) * ftype.size());
        up(h.m.fpartner, fpart.data(), sizeof(int) * fpart.size());
        up(h.m.fpar, fpar.data(), sizeof(double) * fpar.size());
    }
    // per-cell area targets follow their domain across ring rebuilds
    std::map<uint32_t, double> tgt;
    for (size_t c = 0; c < h.ringDomHost.size(); ++c) tgt[h.ringDomHost[c]] = h.targetHost[c];
    std::vector<double> tnew(cells);
    for (int c = 0; c < cells; ++c) tnew[c] = tgt.count(ringDom[c]) ? tgt[ringDom[c]] : NAN;
    h.ringDomHost = ringDom;
    h.targetHost = tnew;
    up(h.target, tnew.data(), sizeof(double) * cells);
    CK(cudaStreamSynchronize(h.stream));
    h.ringsCurrent = true;  // the rings were uploaded with the topology
}

// Refreshes the host mirror of the topology (node ids, connection vector)
// from the device, which edits it when remeshing and coarsening.
static void pull_topology(Handle& h) {
    Topo tp{};
    CK(cudaMemcpyAsync(&tp, h.m.topo, sizeof(Topo), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    const int M = tp.M, C = tp.C;
    std::vector<int> ca(C), cb(C), cdesc(C);
    std::vector<uint32_t> cdom(C);
    h.ids.resize(M);
    if (M) CK(cudaMemcpyAsync(h.ids.data(), h.m.id, sizeof(uint32_t) * M, cudaMemcpyDeviceToHost, h.stream));
    if (C) {
        CK(cudaMemcpyAsync(ca.data(), h.m.ca, sizeof(int) * C, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaMemcpyAsync(cb.data(), h.m.cb, sizeof(int) * C, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaMemcpyAsync(cdom.data(), h.m.cdom, sizeof(uint32_t) * C, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaMemcpyAsync(cdesc.data(), h.m.cdesc, sizeof(int) * C, cudaMemcpyDeviceToHost, h.stream));
    }
    CK(cudaStreamSynchronize(h.stream));
    h.conns.resize(C);
    for (int c = 0; c < C; ++c)
        h.conns[c] = HConn{h.ids[ca[c]], h.ids[cb[c]], cdom[c],
                           cdesc[c] >= 0 && cdesc[c] < (int)h.descTable.size() ? h.descTable[cdesc[c]] : std::string()};
    h.m.M = M;
    h.m.C = C;
}

// Copies the device's area targets to the host mirror (they are set on the
// device by the first area-regulator call).
static void sync_targets(Handle& h) {
    if (h.m.nCells == 0) return;
    h.targetHost.resize(h.m.nCells);
    CK(cudaMemcpyAsync(h.targetHost.data(), h.target, sizeof(double) * h.m.nCells, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
}

// Scratch of the device force-list edits (membrane tension on a list with other
// forces, cell junctions), sized for the node and record capacities.
// `need`: allocate even without a tension or junction solver (the force-list and
// range-query calls of the C ABI).
static void ensure_force_scratch(Handle& h, bool need = false) {
    const bool tension = std::find(h.bio.begin(), h.bio.end(), 1) != h.bio.end();
    const bool junction = has_junctions(h) || need || h.fsQuery;
    h.fs.outPos = h.outPos;
    h.fs.inPos = h.inPos;
    if (!(tension || junction)) return;
    if (h.fsMcap == h.Mcap && h.fsFcap == h.Fcap && (h.fs.binKey != nullptr) == junction) return;
    auto fr = [](void* p) { if (p) cudaFree(p); };
    ForceScratch& fs = h.fs;
    fr(fs.foffS); fr(fs.ftypeS); fr(fs.fpartnerS); fr(fs.fparS); fr(fs.cnt); fr(fs.scanTmp);
    fr(fs.binKey); fr(fs.binKeySorted); fr(fs.binIdx); fr(fs.binIdxSorted); fr(fs.sortTmp); fr(fs.closest);
    fr(fs.binStart); fr(fs.binHead); fr(fs.binNext); fr(fs.linkKey); fr(fs.linkPrevM);
    fr(fs.inCnt); fr(fs.inOff); fr(fs.inList); fr(fs.inFill);
    fs = ForceScratch{};
    fs.outPos = h.outPos;
    fs.inPos = h.inPos;
    const int n = h.Mcap;
    fs.Fcap = h.Fcap;
    fs.foffS = dalloc<int>(n + 1);
    fs.cnt = dalloc<int>(n + 1);
    fs.ftypeS = dalloc<int>(h.Fcap);
    fs.fpartnerS = dalloc<int>(h.Fcap);
    fs.fparS = dalloc<double>(4 * (size_t)h.Fcap);
    fs.scanTmpBytes = force_scan_bytes(n + 1);
    CK(cudaMalloc(&fs.scanTmp, fs.scanTmpBytes));
    if (junction) {
        fs.binKey = dalloc<unsigned>(n); fs.binKeySorted = dalloc<unsigned>(n);
        fs.binIdx = dalloc<int>(n); fs.binIdxSorted = dalloc<int>(n);
        fs.sortBits = 1;
        while ((1ull << fs.sortBits) <= (unsigned long long)h.L && fs.sortBits < 32) ++fs.sortBits;
        fs.sortTmpBytes = junction_sort_bytes(n, fs.sortBits);
        CK(cudaMalloc(&fs.sortTmp, fs.sortTmpBytes));
        fs.binCap = (unsigned)h.L;
        fs.binStart = dalloc<int>(h.L);
        CK(cudaMemsetAsync(fs.binStart, 0xff, sizeof(int) * h.L, h.stream));
        fs.binHead = dalloc<int>(h.L);
        CK(cudaMemsetAsync(fs.binHead, 0xff, sizeof(int) * h.L, h.stream));
        fs.binNext = dalloc<int>(n);
        fs.linkKey = dalloc<unsigned>(n);
        fs.linkPrevM = dalloc<int>(1);
        CK(cudaMemsetAsync(fs.linkPrevM, 0, sizeof(int), h.stream));
        fs.closest = dalloc<int>(n);
        fs.inCnt = dalloc<int>(n + 1); fs.inOff = dalloc<int>(n + 1);
        fs.inList = dalloc<int>(n); fs.inFill = dalloc<int>(n);
    }
    h.fsMcap = h.Mcap;
    h.fsFcap = h.Fcap;
    h.fsQuery = junction;
    h.graphEpoch++;
}

// Sizes the status allocation for cellCap areas, keeping the status word and
// the counts (device and host copies).
static void resize_status_block(Handle& h) {
    const size_t bytes = kAreaOffset + sizeof(double) * (size_t)h.cellCap;
    char* dev = dalloc<char>(bytes);
    char* host = nullptr;
    CK(cudaMallocHost(&host, bytes));
    std::memset(host, 0, bytes);
    if (h.st) {
        CK(cudaMemcpyAsync(dev, h.st, kAreaOffset, cudaMemcpyDeviceToDevice, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        std::memcpy(host, h.stHost, kAreaOffset);
        cudaFree(h.st);
        cudaFreeHost(h.stHost);
    } else {
        CK(cudaMemsetAsync(dev, 0, kAreaOffset, h.stream));
    }
    h.st = (Status*)dev;
    h.m.topo = (Topo*)(dev + kTopoOffset);
    h.area = (double*)(dev + kAreaOffset);
    h.stHost = (Status*)host;
    h.topoHost = (Topo*)(host + kTopoOffset);
    h.areaPinned = (double*)(host + kAreaOffset);
    h.graphEpoch++;  // kernels captured with the old addresses
}

static void ensure_capacity(Handle& h, int M, int C, int F, int cells) {
    // headroom for remeshing on the device: node and connection buffers hold
    // twice the current counts before the host has to grow them
    auto grow = [&](int need, int& cap) {
        if (need <= cap) return false;
        cap = std::max(2 * need + 1024, 64);
        h.graphEpoch++;
        return true;
    };
    if (grow(M, h.Mcap)) {
        // membrane arrays are rewritten by every upload_topology; no copy needed
        auto fr = [](void* p) { if (p) cudaFree(p); };
        fr(h.m.x); fr(h.m.y); fr(h.m.ox); fr(h.m.oy); fr(h.m.vx); fr(h.m.vy); fr(h.m.fx); fr(h.m.fy); fr(h.m.bx); fr(h.m.by);
        fr(h.m.id); fr(h.m.prev); fr(h.m.next); fr(h.outPos); fr(h.inPos); fr(h.cross.perturbList);
        fr(h.m.foff); fr(h.m.ringNode); fr(h.tiles.list);
        fr(h.td.nflag); fr(h.td.nrank); fr(h.td.dalt); fr(h.td.id2); fr(h.td.prev2); fr(h.td.next2);
        fr(h.td.inConn); fr(h.td.outConn); fr(h.td.removed); fr(h.td.ncA); fr(h.td.ncB); fr(h.td.ncDom);
        fr(h.td.ncDesc); fr(h.td.ncAlive); fr(h.td.members); fr(h.td.succ); fr(h.td.dist); fr(h.td.rngList);
        const int n = h.Mcap;
        h.td.nflag = dalloc<int>(n + 1); h.td.nrank = dalloc<int>(n + 1);
        h.td.dalt = dalloc<double>(10 * (size_t)n);
        h.td.id2 = dalloc<uint32_t>(n); h.td.prev2 = dalloc<int>(n); h.td.next2 = dalloc<int>(n);
        h.td.inConn = dalloc<int>(n); h.td.outConn = dalloc<int>(n);
        h.td.removed = dalloc<unsigned char>(n);
        CK(cudaMemsetAsync(h.td.removed, 0, n, h.stream));
        h.td.ncA = dalloc<int>(n); h.td.ncB = dalloc<int>(n); h.td.ncDom = dalloc<uint32_t>(n);
        h.td.ncDesc = dalloc<int>(n); h.td.ncAlive = dalloc<int>(n + 1);
        CK(cudaMemsetAsync(h.td.ncAlive, 0, sizeof(int) * (n + 1), h.stream));
        h.td.members = dalloc<int>(n); h.td.succ = dalloc<int>(n + 1); h.td.dist = dalloc<int>(n + 1);
        h.td.rngList = dalloc<int>(n);
        h.m.x = dalloc<double>(n); h.m.y = dalloc<double>(n); h.m.ox = dalloc<double>(n); h.m.oy = dalloc<double>(n);
        h.m.bx = dalloc<double>(n); h.m.by = dalloc<double>(n);
        h.m.vx = dalloc<double>(n); h.m.vy = dalloc<double>(n); h.m.fx = dalloc<double>(n); h.m.fy = dalloc<double>(n);
        h.m.id = dalloc<uint32_t>(n); h.m.prev = dalloc<int>(n); h.m.next = dalloc<int>(n);
        h.outPos = dalloc<int>(n); h.inPos = dalloc<int>(n);
        h.cross.perturbList = dalloc<int>(n); h.cross.perturbCap = n;
        h.m.foff = dalloc<int>(n + 1);
        h.m.ringNode = dalloc<int>(n);
        h.tiles.cap = 4 * n;
        h.tiles.list = dalloc<int>(h.tiles.cap);
    }
    if (grow(C, h.Ccap)) {
        auto fr = [](void* p) { if (p) cudaFree(p); };
        fr(h.m.ca); fr(h.m.cb); fr(h.m.cdom); fr(h.m.cdesc); fr(h.cross.changedNode); fr(h.cross.reinitDone); fr(h.cross.waitList);
        fr(h.cross.recKey); fr(h.cross.recConn); fr(h.cross.recDom); fr(h.cross.recDist);
        fr(h.cross.changedDom);
        // the boundary-node list of the last crossings is still to be used by
        // the next stream-collide and cleared after it: carried over
        uint32_t* oldKeys = h.cross.nfKeys;
        double* oldD = h.cross.nfD;
        const int oldCap = h.cross.nfCap;
        fr(h.td.flag); fr(h.td.rank); fr(h.td.ca2); fr(h.td.cb2); fr(h.td.cdom2); fr(h.td.cdesc2); fr(h.td.connAlive);
        const int n = h.Ccap;
        h.m.ca = dalloc<int>(n); h.m.cb = dalloc<int>(n); h.m.cdom = dalloc<uint32_t>(n); h.m.cdesc = dalloc<int>(n);
        h.td.flag = dalloc<int>(n + 1); h.td.rank = dalloc<int>(n + 1);
        h.td.ca2 = dalloc<int>(n); h.td.cb2 = dalloc<int>(n); h.td.cdom2 = dalloc<uint32_t>(n);
        h.td.cdesc2 = dalloc<int>(n); h.td.connAlive = dalloc<int>(n);
        // each connection of length <= MAXLENGTH crosses at most one line per axis
        // (two records each); longer ones exist only between the move and the remesh
        h.cross.changedCap = 8 * n + 1024;
        h.cross.recCap = 16 * n + 1024;
        h.cross.recKey = dalloc<uint32_t>(h.cross.recCap);
        h.cross.nfKeys = dalloc<uint32_t>(h.cross.recCap);  // no more boundary nodes than records
        h.cross.nfD = dalloc<double>(2 * (size_t)h.cross.recCap);
        h.cross.nfCap = h.cross.recCap;
        if (oldKeys != nullptr && oldCap > 0)
            CK(cudaMemcpyAsync(h.cross.nfKeys, oldKeys, sizeof(uint32_t) * oldCap, cudaMemcpyDeviceToDevice, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        fr(oldKeys); fr(oldD);
        h.cross.recConn = dalloc<uint32_t>(h.cross.recCap);
        h.cross.recDom = dalloc<uint32_t>(h.cross.recCap);
        h.cross.recDist = dalloc<unsigned long long>(h.cross.recCap);
        h.cross.changedNode = dalloc<uint32_t>(h.cross.changedCap);
        h.cross.reinitDone = dalloc<int>(h.cross.changedCap);
        h.cross.waitList = dalloc<int>(h.cross.changedCap);
        if (!h.cross.nWait) {
            h.cross.nWait = dalloc<int>(1);
            CK(cudaMemsetAsync(h.cross.nWait, 0, sizeof(int), h.stream));
        }
        h.cross.changedDom = dalloc<uint32_t>(h.cross.changedCap);
    }
    if (grow(F, h.Fcap)) {
        auto fr = [](void* p) { if (p) cudaFree(p); };
        fr(h.m.ftype); fr(h.m.fpartner); fr(h.m.fpar);
        h.m.ftype = dalloc<int>(h.Fcap); h.m.fpartner = dalloc<int>(h.Fcap); h.m.fpar = dalloc<double>(4 * (size_t)h.Fcap);
    }
    if (grow(cells, h.cellCap)) {
        auto fr = [](void* p) { if (p) cudaFree(p); };
        fr(h.m.ringStart); fr(h.m.ringDom); fr(h.target); fr(h.areaAcc);
        fr(h.td.cellCount); fr(h.td.cellStart); fr(h.td.cellFill); fr(h.td.startNode);
        h.m.ringStart = dalloc<int>(h.cellCap + 1); h.m.ringDom = dalloc<uint32_t>(h.cellCap);
        resize_status_block(h);
        h.target = dalloc<double>(h.cellCap);
        h.areaAcc = dalloc<unsigned long long>(h.cellCap);
        CK(cudaMemset(h.areaAcc, 0, sizeof(unsigned long long) * h.cellCap));
        h.td.cellCount = dalloc<int>(h.cellCap + 1); h.td.cellStart = dalloc<int>(h.cellCap + 1);
        h.td.cellFill = dalloc<int>(h.cellCap); h.td.startNode = dalloc<int>(h.cellCap);
    }
    ensure_force_scratch(h);
    // scan scratch for the largest scan (nodes, connections or cells)
    const size_t need = topo_scan_bytes(std::max(std::max(h.Mcap, h.Ccap), h.cellCap) + 1);
    if (need > h.td.scanTmpBytes) {
        if (h.td.scanTmp) cudaFree(h.td.scanTmp);
        CK(cudaMalloc(&h.td.scanTmp, need));
        h.td.scanTmpBytes = need;
    }
    h.m.Mcap = h.Mcap;
    h.m.Ccap = h.Ccap;
}

// ---------------------------------------------------------------------------
// Host-side events, in the reference's order.

// GeometryNode::perturbatePosition (GeometryNode.cpp:153-214).  The two draws
// of one setPos(x + dis(gen), y + dis(gen)) are taken y-first: g++ evaluates
// those arguments right to left, which is what the reference build does.
static void perturbate(Handle& h, double& x, double& y) {
    double r;
    if (std::abs(static_cast<int>(x) - x) <= kEPSILON) {
        r = 0.0;
        while (std::abs(r) < 5.0 * kEPSILON) r = h.dis(h.genNode);
        x = x + r;
    }
    if (std::abs(static_cast<int>(y) - y) <= kEPSILON) {
        r = 0.0;
        while (std::abs(r) < 5.0 * kEPSILON) r = h.dis(h.genNode);
        y = y + r;
    }
    if (std::abs(y - std::floor(y) - (x - std::floor(x))) <= kEPSILON) {
        const double ry = h.dis(h.genNode);
        const double rx = h.dis(h.genNode);
        x = x + rx; y = y + ry;
    }
    if (std::abs(std::ceil(y) - y - (x - std::floor(x))) <= kEPSILON) {
        const double ry = h.dis(h.genNode);
        const double rx = h.dis(h.genNode);
        x = x + rx; y = y + ry;
    }
}

// GeometryHandler::perturbConnections + Connection::perturbConnection
// (GeometryHandler.cpp:326-356, Connection.cpp:332-387) on the host copy.
static void perturb_connections(Handle& h, HostMembrane& hm) {
    const IdIndex index(h.ids);
    std::map<uint32_t, int> first;
    for (size_t c = 0; c < h.conns.size(); ++c)
        if (!first.count(h.conns[c].dom)) first[h.conns[c].dom] = (int)c;
    std::vector<int> outConn(h.ids.size(), -1);
    for (size_t c = 0; c < h.conns.size(); ++c) outConn[index.at(h.conns[c].id1)] = (int)c;
    for (auto& kv : first) {
        int c = kv.second;
        do {
            const int a = index.at(h.conns[c].id1), b = index.at(h.conns[c].id2);
            double r;
            if (std::abs(hm.x[a] - hm.x[b]) < kEPSILON) {
                r = 0.0;
                while (std::abs(r) < 5.0 * kEPSILON) r = h.dis(h.genConn);
                hm.x[a] = hm.x[a] + r;
                perturbate(h, hm.x[a], hm.y[a]);
            }
            if (std::abs(hm.y[a] - hm.y[b]) < kEPSILON) {
                r = 0.0;
                while (std::abs(r) < 5.0 * kEPSILON) r = h.dis(h.genConn);
                hm.y[a] = hm.y[a] + r;
                perturbate(h, hm.x[a], hm.y[a]);
            }
            c = outConn[b];
        } while (c != kv.second);
    }
}

// GeometryHandler::remeshBoundary loop (GeometryHandler.cpp:385-431,
// SimulationRunner.cpp:190-199) with Geometry::addGeometryNode /
// eraseConnection / addConnection (Geometry.cpp:382-452).  One pass visits
// the connections present at its start, in vector order; each long one gets a
// new node at its midpoint (next id, perturbed on creation) and is replaced by
// two connections appended at the end of the vector.
static bool remesh(Handle& h, HostMembrane& hm) {
    bool any = false;
    for (;;) {
        const IdIndex index(h.ids);
        std::vector<HConn> kept, added;
        kept.reserve(h.conns.size());
        for (const HConn& c : h.conns) {
            const int a = index.at(c.id1), b = index.at(c.id2);
            const double len = std::sqrt((hm.x[a] - hm.x[b]) * (hm.x[a] - hm.x[b]) +
                                         (hm.y[a] - hm.y[b]) * (hm.y[a] - hm.y[b]));
            if (len > kMAXLENGTH) {
                const uint32_t nid = h.ids.back() + 1;
                double nx = (hm.x[a] + hm.x[b]) / 2, ny = (hm.y[a] + hm.y[b]) / 2;
                const double ox = nx - 5.0, oy = ny - 5.0;
                perturbate(h, nx, ny);
                h.ids.push_back(nid);
                hm.x.push_back(nx); hm.y.push_back(ny);
                hm.ox.push_back(ox); hm.oy.push_back(oy);
                hm.bx.push_back(nx); hm.by.push_back(ny);  // bound by the edge check after the upload
                hm.vx.push_back(0.0); hm.vy.push_back(0.0);
                hm.fx.push_back(0.0); hm.fy.push_back(0.0);
                added.push_back(HConn{c.id1, nid, c.dom, c.desc});
                added.push_back(HConn{nid, c.id2, c.dom, c.desc});
            } else {
                kept.push_back(c);
            }
        }
        if (added.empty()) break;
        kept.insert(kept.end(), added.begin(), added.end());
        h.conns.swap(kept);
        any = true;
    }
    return any;
}

// ---------------------------------------------------------------------------
// Stage launcher

template <typename Real>
static LatticeArgs<Real> lattice_args(Handle& h, unsigned iteration, int parity) {
    LatticeArgs<Real> a{};
    a.nx = h.nx; a.ny = h.ny; a.L = h.L; a.S = h.S;
    a.fin = (const Real*)h.f[parity];
    a.fout = (Real*)h.f[1 - parity];
    a.gin = (const Real*)h.g[parity];
    a.gout = (Real*)h.g[1 - parity];
    a.u = (Real*)h.u;
    a.force = (const Real*)h.force;
    a.tileCount = h.tiles.count;
    a.tilesX = h.tiles.tilesX;
    a.dom = h.dom;
    bool area = false;
    for (int b : h.bio) area |= (b == 2);
    a.massTab = area ? h.massTab : nullptr;
    a.massNode = h.massNode;
    a.nDomains = h.nDomains;
    a.srcTab = h.srcTab;
    a.ctypeTab = h.ctypeTab;
    a.tauF = h.tauF;
    a.forceModel = h.forceModel;
    for (int k = 0; k < h.S; ++k) {
        a.sp[k] = h.sp[k].c;
        a.coupled |= coupled_kind(h.sp[k].c.kind) ? 1 : 0;
    }
    a.status = h.st;
    a.outlet = h.outlet ? 1 : 0;
    a.bounceW = h.cross.bounceW;
    a.bounceS = h.cross.bounceS;
    if (h.cross.nfTab != nullptr) {
        a.nfSpec = h.cross.nfSpec;
        a.nfU = h.cross.nfU;
        a.nfTab = h.cross.nfTab;
        a.nfKeys = h.cross.nfKeys;
        a.nfN = h.cross.nfN;
        a.nfCap = h.cross.nfCap;
        a.nfD = h.cross.nfD;
    }
    return a;
}

// The first kernel of a step without a membrane (with one, the force kernel).
__global__ void step_begin_kernel(Status* st) {
    pdl_wait();
    if (st->halt) return;
    begin_step(st);
}

__global__ void iteration_inc_kernel(Status* st) {
    pdl_wait(); st->iteration += 1; }

// Launches the stage kernels of one step from `fromStage` on.  `coarsenStep`
// (Parameters' iteration % 10 == 0) and `bioOps` (which bio solvers change the
// force list, step_bio_ops) are the only host decisions; everything else reads
// device state.  Returns the number of kernels launched.
template <typename Real>
static long long launch_stages(Handle& h, bool coarsenStep, int bioOps, int parity, int fromStage,
                               cudaEvent_t evCollideA, cudaEvent_t evCollideB) {
    cudaStream_t s = h.stream;
    Real* gcur = (Real*)h.g[1 - parity];
    const bool hasM = h.m.Mcap > 0;
    const unsigned it = 0;  // kernels read the iteration from the status word
    long long nl = 0;
    if (fromStage <= ST_FORCE) {
        // the step's counters are reset by the force kernel, or alone without a
        // membrane; in FP32-shifted runs the force kernel also fills the
        // spread's per-tile lists
        if (hasM) launch_force_eval<Real>(h.m, h.st, it, s, true, sizeof(Real) == 4 ? &h.tiles : nullptr, h.nx, h.ny);
        else launch_pdl(step_begin_kernel, 1, 1, 0, s, h.st);
        nl += 1;
    }
    if (fromStage <= ST_SPREAD) {
        const bool filled = sizeof(Real) == 4 && hasM && fromStage <= ST_FORCE;
        launch_spread<Real>(h.m, h.tiles, (Real*)h.force, h.nx, h.ny, h.L, h.st, it, s, filled);
        nl += hasM ? (sizeof(Real) == 8 ? 6 : (filled ? 1 : 2)) : 0;
    }
    if (fromStage <= ST_COLLIDE) {
        if (evCollideA) cudaEventRecord(evCollideA, s);
        if (sizeof(Real) == 8) {
            const LatticeArgs<double> a = lattice_args<double>(h, it, parity);
            launch_stream_collide64(a, s);
        } else {
            const LatticeArgs<float> a = lattice_args<float>(h, it, parity);
            launch_stream_collide32(a, s);
        }
        if (evCollideB) cudaEventRecord(evCollideB, s);
        nl += 1 + (h.cross.nfTab != nullptr ? 2 : 0);
    }
    if (fromStage <= ST_INTERP_MOVE) {
        launch_interp_move<Real>(h.m, (const Real*)h.u, h.nx, h.ny, h.L, h.cross, h.st, it, s);
        nl += hasM;
    }
    if (fromStage <= ST_PERTURB_CONN) {
        launch_perturb_conn_check(h.m, h.st, it, s, h.td.rngList, h.Mcap);
        nl += hasM;
    }
    if (fromStage <= ST_CROSSINGS) {
        launch_crossings<Real>(h.m, h.cross, h.dom, h.nx, h.ny, h.L, h.st, it, s);
        nl += hasM ? 3 : 0;
    }
    if (fromStage <= ST_REINIT) {
        SpeciesConst spc[kMaxSpecies] = {};
        for (int k = 0; k < h.S; ++k) spc[k] = h.sp[k].c;
        launch_reinit<Real>(h.cross, h.dom, gcur, (const Real*)h.u, h.S, spc, h.srcTab, h.nDomains, h.ctypeTab, 0,
                            h.nx, h.ny, h.L, h.st, it, s);
        nl += 2;
    }
    if (fromStage <= ST_DOMAIN) {
        launch_domain_fill(h.cross, h.dom, h.nx, h.ny, h.L, h.st, it, s);
        nl += 1;
    }
    if (fromStage <= ST_REMESH_COMMIT)
        nl += launch_remesh(h.m, h.td, h.nx, h.ny, h.st, s, fromStage == ST_REMESH_COMMIT);
    if (fromStage <= ST_COARSEN && coarsenStep) {
        // SimulationRunner.cpp:84-87: ForceSolver::deleteAllForces, then coarsenBoundary
        launch_clear_forces(h.m, s);
        nl += 1 + launch_coarsen(h.m, h.td, h.st, s);
    }
    // ST_OUTLET: MassSolverBoxOutlet runs inside the stream-collide kernel
    if (fromStage <= ST_BIO) {
        // FP64 runs sum the areas in ring order (the reference's order), so the
        // rings are re-ranked after any topology change; FP32-shifted runs sum
        // in exact fixed point and need no ring order here
        if (sizeof(Real) == 8) nl += launch_rings(h.m, h.td, h.st, s);
        for (size_t q = 0; q < h.bio.size(); ++q) {
            const int b = h.bio[q], op = (bioOps >> (2 * q)) & 3;
            if (b == 2) {
                const uint32_t* ct = h.areaTutorial ? h.ctypeTab : nullptr;
                if (sizeof(Real) == 8) {
                    launch_area_regulator(h.m, h.area, h.target, h.massTab, h.nDomains, h.areaFactor,
                                          h.areaStrength, h.areaMax, ct, h.st, s);
                    nl += h.m.nCells > 0 ? 2 : 0;
                } else {
                    launch_area_regulator_fixed(h.m, h.td.cellOfDom, h.areaAcc, h.area, h.target, h.massTab,
                                                h.nDomains, h.areaFactor, h.areaStrength, h.areaMax, ct, h.st, s);
                    nl += h.m.nCells > 0 ? 2 : 0;
                }
                if (h.massNode != nullptr) {
                    launch_mass_expand(h.dom, h.L, h.massTab, h.nDomains, h.massNode, h.st, s);
                    nl += 1;
                }
            } else if (b == 6) {
                launch_growth<Real>(gcur, h.dom, h.L, h.growthR, h.growthL, h.massNode, h.st, s);
                nl += 1;
            } else if (b == 1 && op == BIO_TENSION_FILL) {
                launch_tension_renewal(h.m, h.outPos, h.inPos, h.tensionForce, s);
                nl += hasM ? 2 : 0;
            } else if (b == 1 && op == BIO_TENSION_EDIT) {
                nl += launch_tension_edit(h.m, h.fs, h.tensionForce, h.st, s);
            } else if (b == 3 && op == BIO_JUNCTIONS) {
                nl += launch_junctions(h.m, h.fs, h.nx, h.ny, h.junctionRadius, h.junctionK, h.junctionL0, h.st, s);
            }
        }
    }
    return nl;
}

// The stage the host resumes at after handling the halt of `stage`.
static int resume_stage(int stage) {
    switch (stage) {
        case ST_INTERP_MOVE: return ST_PERTURB_CONN;
        case ST_PERTURB_CONN: return ST_CROSSINGS;
        case ST_REMESH: return ST_COARSEN;
        case ST_REMESH_RNG: return ST_REMESH_COMMIT;
        default: return -1;
    }
}

// Reads the status word and, in the same synchronisation, the device counts:
// their `changed` flag says whether the ring order of the cell areas is stale
// (remeshing or coarsening on the device set it; a ring rebuild clears it).
static void read_status(Handle& h) {
    const size_t areas = h.statusWithAreas ? sizeof(double) * (size_t)h.m.nCells : 0;
    h.statusWithAreas = false;
    CK(cudaMemcpyAsync(h.stHost, h.st, kAreaOffset + areas, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    if (h.m.topo) h.ringsCurrent = h.topoHost->changed == 0;
}

static void write_status(Handle& h) {
    h.statusContinues = false;
    CK(cudaMemcpyAsync(h.st, h.stHost, sizeof(Status), cudaMemcpyHostToDevice, h.stream));
}

// The bio stage of a step leaves the cell areas of the new state in h.area
// when the area regulator is registered: in ring order in FP64 runs, from
// the exact fixed-point sums in FP32-shifted runs (the values lbib_areas
// forms).  Their read-back rides on the status word's.
static bool step_leaves_areas(const Handle& h) {
    if (h.m.nCells == 0 || h.m.Ccap == 0 || h.areaPinned == nullptr) return false;
    for (int b : h.bio)
        if (b == 2) return true;
    return false;
}

// GeometryHandler::computeAreas into the device array `area`: in ring order in
// FP64 runs (the ring order is rebuilt only when the topology changed since
// it was last built), from the fixed-point sums in FP32-shifted runs.
static void queue_areas(Handle& h, double* area) {
    if (h.precision == LBIB_FP64) {
        if (!h.ringsCurrent) launch_rings(h.m, h.td, h.st, h.stream);
        launch_areas(h.m, area, h.st, h.stream);
    } else {
        launch_areas_fixed(h.m, h.td.cellOfDom, h.nDomains, h.areaAcc, area, h.stream);
    }
}

static void queue_step_areas(Handle& h) {
    if (step_leaves_areas(h)) h.statusWithAreas = true;
}

// Clears the status word for a run that starts at Parameters' iteration `it`.
static void reset_status(Handle& h, unsigned it, bool cellTypesCopied) {
    std::memset(h.stHost, 0, sizeof(Status));
    h.stHost->iteration = it;
    h.stHost->cellTypesCopied = cellTypesCopied ? 1 : 0;
    h.stHost->pad[3] = 1;  // the next step begins a run
    write_status(h);
}

// Bookkeeping the host does for a step it launches: the loaded force list is
// gone after the step's ForceSolver::deleteAllForces.
static void host_step_bookkeeping(Handle& h, unsigned iteration) {
    if (iteration % 10 == 0) h.forcemap.clear();
}

// What the bio solvers of step `it` do to the force list, 2 bits per solver in
// registration order (SimulationRunner::applyBioSolvers):
//   BIO_TENSION_FILL  the membrane-tension renewal on a list of tension records
//                     only (or none): the list is rebuilt whole;
//   BIO_TENSION_EDIT  the same renewal on a list that holds other forces:
//                     deleteForceType(6), then the new records appended;
//   BIO_JUNCTIONS     the cell-junction solver (every 10th iteration).
// Before the bio stage, the list holds only tension records when the step's
// own coarsening stage cleared it (iteration % 10 == 0), or when it was
// cleared at an earlier multiple of 10 and no junction solver added springs,
// or, before any clearing, when it was loaded empty.
// The list holds only tension records (or none) at the start of step `it`:
// after the last clearing since the list was set (a multiple of 10 in
// [forceListIt, it - 1]) the junction solver, if registered, added springs;
// before any clearing the list is as set.
static bool pure_at_start(const Handle& h, unsigned it) {
    if (it > 0) {
        const unsigned c = (it - 1) - (it - 1) % 10;
        if (c >= h.forceListIt) return !has_junctions(h);
    }
    return h.forcesPureAtLoad;
}

static int step_bio_ops(const Handle& h, unsigned it) {
    bool pure = it % 10 == 0 ? true : pure_at_start(h, it);
    int ops = 0;
    for (size_t q = 0; q < h.bio.size(); ++q) {
        int op = 0;
        if (h.bio[q] == 1 && it % h.tensionFreq == 0) {
            op = pure ? BIO_TENSION_FILL : BIO_TENSION_EDIT;
        } else if (h.bio[q] == 3 && it % 10 == 0) {
            op = BIO_JUNCTIONS;
            pure = false;
        }
        ops |= op << (2 * q);
    }
    return ops;
}

// The new nodes of a remesh pass that were made on a lattice line or
// diagonal: GeometryNode's constructor perturbs them when remeshBoundary
// creates them (GeometryNode.cpp:98-117, GeometryHandler.cpp:385-431), drawing
// from the node generator in creation (= id) order.  The device made the
// pass's nodes and listed these; the host draws their perturbation from the
// same generator and the device then commits the pass.  Only the pass's new
// positions cross the bus.
static void perturb_new_nodes(Handle& h) {
    const Topo tp = *h.topoHost;  // read back with the status word
    const int M = tp.M, K = tp.K, n = tp.rngFill;
    if (K <= 0 || n <= 0 || n > K || M + K > h.Mcap) fail(ERR_STATE, "remesh: bad list of new nodes to perturb");
    std::vector<int> list(n);
    std::vector<double> x(K), y(K);
    CK(cudaMemcpyAsync(list.data(), h.td.rngList, sizeof(int) * n, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(x.data(), h.m.x + M, sizeof(double) * K, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(y.data(), h.m.y + M, sizeof(double) * K, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    std::sort(list.begin(), list.end());
    for (int j : list) {
        if (j < M || j >= M + K) fail(ERR_STATE, "remesh: new node index out of the pass", j);
        perturbate(h, x[j - M], y[j - M]);
    }
    CK(cudaMemcpyAsync(h.m.x + M, x.data(), sizeof(double) * K, cudaMemcpyHostToDevice, h.stream));
    CK(cudaMemcpyAsync(h.m.y + M, y.data(), sizeof(double) * K, cudaMemcpyHostToDevice, h.stream));
    const int zero[2] = {0, 0};  // nRng, rngFill: the commit goes ahead
    static_assert(offsetof(Topo, rngFill) == offsetof(Topo, nRng) + sizeof(int), "Topo field order");
    CK(cudaMemcpyAsync((char*)h.m.topo + offsetof(Topo, nRng), zero, sizeof zero, cudaMemcpyHostToDevice, h.stream));
    CK(cudaStreamSynchronize(h.stream));
}

// GeometryHandler::perturbConnections (GeometryHandler.cpp:326-356) from the
// device's list of connections that need it, without the whole membrane.  A
// perturbation moves only the first node of its connection, which is the
// second node of the connection before it in the ring walk: that one was
// visited already, except for the walk's last connection (into the walk's
// first node), which is tested again here when the first one moved.  So the
// listed connections, visited in (domain, walk) order, with the ring-closing
// test, draw exactly what the reference's full walk draws.  Returns false
// (the caller takes the full path) when the list overflowed or a connection's
// ring was not found.
static bool perturb_listed_connections(Handle& h) {
    const int n = h.stHost->nPerturbConn;
    if (n <= 0 || n > h.Mcap) return false;
    launch_rings(h.m, h.td, h.st, h.stream);  // a no-op when they are current
    // the records go to the coarsening's node scratch (10 doubles per node of
    // capacity), free until this step's coarsening
    static_assert(sizeof(ConnPerturbRec) <= 10 * sizeof(double), "record larger than the scratch per node");
    ConnPerturbRec* dev = reinterpret_cast<ConnPerturbRec*>(h.td.dalt);
    launch_conn_perturb_gather(h.m, h.td, n, dev, h.stream);
    CK(cudaGetLastError());
    std::vector<ConnPerturbRec> rec(n);
    CK(cudaMemcpyAsync(rec.data(), dev, sizeof(ConnPerturbRec) * n, cudaMemcpyDeviceToHost, h.stream));
    read_status(h);
    if (h.stHost->err) fail(h.stHost->err, "ring order for the connection perturbation", h.stHost->errIndex);
    for (const ConnPerturbRec& r : rec)
        if (r.walk < 0) return false;
    std::sort(rec.begin(), rec.end(), [](const ConnPerturbRec& p, const ConnPerturbRec& q) {
        return p.dom != q.dom ? p.dom < q.dom : p.walk < q.walk;
    });
    std::map<int, std::pair<double, double>> pos;  // node index -> current position
    for (const ConnPerturbRec& r : rec) {
        pos.emplace(r.a, std::make_pair(r.xa, r.ya));
        pos.emplace(r.b, std::make_pair(r.xb, r.yb));
        pos.emplace(r.z, std::make_pair(r.xz, r.yz));
    }
    std::map<int, std::pair<double, double>> moved;
    auto perturb = [&](int a, int b) {  // Connection::perturbConnection (Connection.cpp:332-387)
        auto& pa = pos.at(a);
        const auto& pb = pos.at(b);
        double r;
        if (std::abs(pa.first - pb.first) < kEPSILON) {
            r = 0.0;
            while (std::abs(r) < 5.0 * kEPSILON) r = h.dis(h.genConn);
            pa.first = pa.first + r;
            perturbate(h, pa.first, pa.second);
            moved[a] = pa;
        }
        if (std::abs(pa.second - pos.at(b).second) < kEPSILON) {
            r = 0.0;
            while (std::abs(r) < 5.0 * kEPSILON) r = h.dis(h.genConn);
            pa.second = pa.second + r;
            perturbate(h, pa.first, pa.second);
            moved[a] = pa;
        }
    };
    for (size_t i = 0; i < rec.size();) {
        size_t j = i;
        bool closingListed = false;
        while (j < rec.size() && rec[j].dom == rec[i].dom) {
            perturb(rec[j].a, rec[j].b);
            closingListed |= rec[j].walk == rec[j].len - 1;
            ++j;
        }
        // the walk's last connection (z -> first node), when the first moved
        if (rec[i].walk == 0 && !closingListed && moved.count(rec[i].a)) perturb(rec[i].z, rec[i].a);
        i = j;
    }
    for (const auto& kv : moved) {
        CK(cudaMemcpyAsync(h.m.x + kv.first, &kv.second.first, sizeof(double), cudaMemcpyHostToDevice, h.stream));
        CK(cudaMemcpyAsync(h.m.y + kv.first, &kv.second.second, sizeof(double), cudaMemcpyHostToDevice, h.stream));
    }
    CK(cudaStreamSynchronize(h.stream));
    return true;
}

// LBIB_LOG_HOST_EVENTS=1 prints each host event's stage and duration to
// stderr (a diagnostic, off by default).
static bool log_host_events() {
    const char* e = std::getenv("LBIB_LOG_HOST_EVENTS");
    return e && e[0] == '1';
}

// The host side of a halted stage, in the reference's order.  Returns true
// when only the listed nodes or connections crossed the bus.
static bool handle_halt(Handle& h, int stage) {
    h.hostEvents++;
    if (stage == ST_REMESH_RNG) {
        perturb_new_nodes(h);
        return true;
    }
    if (stage == ST_PERTURB_CONN && !h.fullHostEvents && perturb_listed_connections(h)) return true;
    if (stage == ST_INTERP_MOVE) {
        // positions that need GeometryNode::perturbatePosition, in id order;
        // only those nodes' positions cross the bus
        const int cnt = h.stHost->nPerturbNode;
        if (cnt > h.cross.perturbCap) fail(ERR_CAPACITY, "perturbation list overflow");
        std::vector<int> list(cnt);
        if (cnt) CK(cudaMemcpyAsync(list.data(), h.cross.perturbList, sizeof(int) * cnt, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        std::sort(list.begin(), list.end());
        std::vector<double> xy(2 * (size_t)cnt);
        for (int k = 0; k < cnt; ++k) {
            if (list[k] < 0 || list[k] >= h.Mcap) fail(ERR_STATE, "perturbation list entry out of range", list[k]);
            CK(cudaMemcpyAsync(&xy[2 * k], h.m.x + list[k], sizeof(double), cudaMemcpyDeviceToHost, h.stream));
            CK(cudaMemcpyAsync(&xy[2 * k + 1], h.m.y + list[k], sizeof(double), cudaMemcpyDeviceToHost, h.stream));
        }
        CK(cudaStreamSynchronize(h.stream));
        for (int k = 0; k < cnt; ++k) perturbate(h, xy[2 * k], xy[2 * k + 1]);
        for (int k = 0; k < cnt; ++k) {
            CK(cudaMemcpyAsync(h.m.x + list[k], &xy[2 * k], sizeof(double), cudaMemcpyHostToDevice, h.stream));
            CK(cudaMemcpyAsync(h.m.y + list[k], &xy[2 * k + 1], sizeof(double), cudaMemcpyHostToDevice, h.stream));
        }
        CK(cudaStreamSynchronize(h.stream));
        return true;
    }
    pull_topology(h);
    HostMembrane hm;
    if (stage == ST_PERTURB_CONN) {
        download_membrane(h, hm);
        perturb_connections(h, hm);
        CK(cudaMemcpyAsync(h.m.x, hm.x.data(), sizeof(double) * hm.x.size(), cudaMemcpyHostToDevice, h.stream));
        CK(cudaMemcpyAsync(h.m.y, hm.y.data(), sizeof(double) * hm.y.size(), cudaMemcpyHostToDevice, h.stream));
    } else if (stage == ST_REMESH) {
        download_membrane(h, hm);
        sync_targets(h);
        const int Mold = (int)h.ids.size();
        // the force list keeps its records; new nodes have none
        std::vector<int> foff(Mold + 1);
        CK(cudaMemcpyAsync(foff.data(), h.m.foff, sizeof(int) * (Mold + 1), cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        const int nrec = foff[Mold];
        std::vector<int> ftype(nrec), fpart(nrec);
        std::vector<double> fpar(4 * (size_t)nrec);
        if (nrec) {
            CK(cudaMemcpyAsync(ftype.data(), h.m.ftype, sizeof(int) * nrec, cudaMemcpyDeviceToHost, h.stream));
            CK(cudaMemcpyAsync(fpart.data(), h.m.fpartner, sizeof(int) * nrec, cudaMemcpyDeviceToHost, h.stream));
            CK(cudaMemcpyAsync(fpar.data(), h.m.fpar, sizeof(double) * 4 * nrec, cudaMemcpyDeviceToHost, h.stream));
            CK(cudaStreamSynchronize(h.stream));
        }
        remesh(h, hm);
        h.keepRecords = nrec;
        upload_topology(h, hm, false);
        h.keepRecords = 0;
        foff.resize(h.m.M + 1, nrec);
        CK(cudaMemcpyAsync(h.m.foff, foff.data(), sizeof(int) * foff.size(), cudaMemcpyHostToDevice, h.stream));
        if (nrec) {
            CK(cudaMemcpyAsync(h.m.ftype, ftype.data(), sizeof(int) * nrec, cudaMemcpyHostToDevice, h.stream));
            CK(cudaMemcpyAsync(h.m.fpartner, fpart.data(), sizeof(int) * nrec, cudaMemcpyHostToDevice, h.stream));
            CK(cudaMemcpyAsync(h.m.fpar, fpar.data(), sizeof(double) * 4 * nrec, cudaMemcpyHostToDevice, h.stream));
        }
        // new nodes are bound to the lattice now (GeometryHandler.cpp:427-428)
        reset_status(h, h.iteration, true);
        launch_edge_check(h.m, h.nx, h.ny, h.st, 0, h.stream);
        read_status(h);
        if (h.stHost->err) fail(h.stHost->err, "geometry point moved too close to the boundary", h.stHost->errIndex);
    } else {
        fail(ERR_STATE, "unexpected halt stage");
    }
    return false;
}

template <typename Real>
static void launch_step_graph(Handle& h, int parity, bool coarsenStep, int bioOps) {
    const int key = (bioOps << 2) | (coarsenStep ? 2 : 0) | parity;
    if (h.graphEpoch != h.graphBuiltEpoch) {
        for (auto& kv : h.graphs)
            if (kv.second.exec) { cudaGraphExecDestroy(kv.second.exec); kv.second.exec = nullptr; }
        h.graphBuiltEpoch = h.graphEpoch;
    }
    Handle::StepGraph& g = h.graphs[key];
    if (!g.exec) {
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
        g.launches = launch_stages<Real>(h, coarsenStep, bioOps, parity, ST_FORCE, nullptr, nullptr);
        CK(cudaStreamEndCapture(h.stream, &graph));
        CK(cudaGraphInstantiate(&g.exec, graph, 0));
        CK(cudaGraphDestroy(graph));
    }
    CK(cudaGraphLaunch(g.exec, h.stream));
    if (check_launches()) {
        const cudaError_t e = cudaStreamSynchronize(h.stream);
        if (e != cudaSuccess)
            std::fprintf(stderr, "lbib: step graph (parity %d, coarsen %d, bio ops %d) at iteration %u failed: %s\n",
                         parity, coarsenStep ? 1 : 0, bioOps, h.iteration, cudaGetErrorString(e));
    }
    h.launches += g.launches;
}

// Bio solvers that run on the host after the device's step: cell division
// (kind 4) and differentiation (kind 5), each every 100th iteration.
static bool host_bio_at(const Handle& h, unsigned it) {
    for (int b : h.bio) {
        if (b == 4 && it % h.divisionFreq == 0) return true;
        if (b == 5 && it % 100u == 0) return true;
    }
    return false;
}
static void run_division(Handle& h);
static void run_differentiation(Handle& h);
static std::map<uint32_t, double> accumulated_concentrations(Handle& h, int k);
static void grow_domains(Handle& h, int nd);
// The host bio solvers of iteration `it` (the step just run), in list order.
static void run_host_bio(Handle& h, unsigned it) {
    for (int b : h.bio) {
        if (b == 5 && it % 100u == 0) run_differentiation(h);
        if (b == 4 && it % h.divisionFreq == 0) run_division(h);
    }
}

template <typename Real>
static void run_steps(Handle& h, int n) {
    const int kBatch = 64;
    const bool hostBio = std::find_if(h.bio.begin(), h.bio.end(), [](int b) { return b == 4 || b == 5; }) !=
                         h.bio.end();
    while (n > 0) {
        int B = std::min(n, kBatch);
        if (hostBio) {
            // the batch ends with the next step that has host bio solvers; they follow it
            for (int b = 0; b < B; ++b)
                if (host_bio_at(h, h.iteration + b)) {
                    B = b + 1;
                    break;
                }
        }
        // a status word that carries on from the last batch needs no reset
        // (one host-to-device copy less per call); its steps' count starts
        // at lastPad0 and the first step counts the last batch's last step
        int pad0 = -1;
        if (h.statusContinues) pad0 = h.lastPad0;
        else reset_status(h, h.iteration, h.cellTypesCopied);
        const bool prof = h.profiling;
        while ((int)h.kEvents.size() < 2 * B) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            h.kEvents.push_back(e);
        }
        for (int b = 0; b < B; ++b) {
            const unsigned it = h.iteration + b;
            host_step_bookkeeping(h, it);
            const int parity = (h.cur + b) & 1;
            if (prof || !h.useGraphs)
                h.launches += launch_stages<Real>(h, it % 10 == 0, step_bio_ops(h, it), parity, ST_FORCE,
                                                  prof ? h.kEvents[2 * b] : nullptr,
                                                  prof ? h.kEvents[2 * b + 1] : nullptr);
            else
                launch_step_graph<Real>(h, parity, it % 10 == 0, step_bio_ops(h, it));
        }
        CK(cudaGetLastError());
        queue_step_areas(h);
        CK(cudaEventRecord(h.evB, h.stream));  // the end of the call's GPU work, unless more follows
        h.workAfterEvB = false;
        read_status(h);
        const Status st = *h.stHost;
        // the first kernel of each step counted the step before it; the last
        // step of the batch completed unless a halt is pending
        const int done = pad0 < 0 ? st.pad[0] + (st.halt ? 0 : 1) : st.pad[0] - pad0 - (st.halt ? 1 : 0);
        if (!st.halt) {
            h.statusContinues = true;
            h.lastPad0 = st.pad[0];
        }
        if (prof) {
            for (int b = 0; b < std::min(done, B); ++b) {
                float ms = 0;
                if (cudaEventElapsedTime(&ms, h.kEvents[2 * b], h.kEvents[2 * b + 1]) == cudaSuccess) {
                    h.lastCollideMs += ms;
                    h.lastCollideLaunches += 1;
                }
            }
        }
        h.cur = (h.cur + done) & 1;
        h.iteration += done;
        h.stepsDone += done;
        if (done > 0) h.cellTypesCopied = true;
        n -= done;
        if (hostBio && done > 0) {
            run_host_bio(h, h.iteration - 1);
            h.workAfterEvB = true;
        }
        if (!st.halt) continue;
        if (st.err) {
            h.err = st.err;
            h.errIndex = st.errIndex;
            char buf[128];
            std::snprintf(buf, sizeof buf, "device error %d at stage %d, iteration %u", st.err, st.haltStage, h.iteration);
            h.msg = buf;
            fail(st.err, h.msg, st.errIndex);
        }
        // the halted step ran up to st.haltStage: serve the host event, resume
        int stage = st.haltStage;
        const unsigned it = h.iteration;
        for (;;) {
            const auto t0 = std::chrono::steady_clock::now();
            const bool listed = handle_halt(h, stage);
            if (log_host_events())
                std::fprintf(stderr, "lbib: host event at stage %d, iteration %u (%s): %.3f ms\n", stage, it,
                             listed ? "listed" : "full membrane",
                             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
            const int from = resume_stage(stage);
            if (from < 0) fail(ERR_STATE, "unexpected halt stage");
            reset_status(h, it, h.cellTypesCopied);
            h.launches += launch_stages<Real>(h, it % 10 == 0, step_bio_ops(h, it), h.cur, from, nullptr, nullptr);
            queue_step_areas(h);
            CK(cudaEventRecord(h.evB, h.stream));
            h.workAfterEvB = false;
            read_status(h);
            if (h.stHost->err) {
                h.err = h.stHost->err;
                h.errIndex = h.stHost->errIndex;
                fail(h.stHost->err, "device error after a host event", h.stHost->errIndex);
            }
            if (!h.stHost->halt) break;
            stage = h.stHost->haltStage;
        }
        h.cur = (h.cur + 1) & 1;
        h.iteration += 1;
        h.stepsDone += 1;
        h.cellTypesCopied = true;
        n -= 1;
        if (hostBio) {
            run_host_bio(h, h.iteration - 1);
            h.workAfterEvB = true;
        }
    }
}

// ---------------------------------------------------------------------------
// Construction

static void cure_lattice(Handle& h, HostMembrane& hm);
static void setup_boundary_solvers(Handle& h);

// The initial conditions of the species whose initSolver the init kernels do
// not cover, set on the host in SimulationRunner::initSolvers' node order
// (rows, then columns; SimulationRunner.cpp:290-306).  The reference seeds its
// generators from std::random_device, so no two of its runs agree; here each
// solver type has one std::mt19937 with the default seed, drawn in that order.
static void init_species_host(Handle& h, const double* vel) {
    bool any = false;
    for (const auto& s : h.sp) any |= s.initStyle != INIT_KERNEL;
    if (!any) return;
    const size_t L = h.L;
    std::vector<uint32_t> dom(L);
    CK(cudaMemcpyAsync(dom.data(), h.dom, sizeof(uint32_t) * L, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    std::map<int, std::mt19937> gens;  // one generator per solver type
    for (int k = 0; k < h.S; ++k) {
        const Species& s = h.sp[k];
        if (s.initStyle == INIT_KERNEL) continue;
        std::mt19937& gen = gens[s.c.kind];
        std::uniform_real_distribution<> dis(-0.01, 0.01);
        std::vector<double> g(5 * L);
        for (size_t n = 0; n < L; ++n) {
            double gi[5];
            switch (s.initStyle) {
                case INIT_T2:
                    for (int q = 0; q < 5; ++q) gi[q] = dom[n] == 0 ? 0.0 : (1.0 + dis(gen)) / 5.0;
                    break;
                case INIT_SCHNAK: {
                    const double temp = 0.2 * (1.0 + dis(gen));
                    for (int q = 0; q < 5; ++q) gi[q] = dom[n] == 0 ? 0.0 : temp;
                    break;
                }
                case INIT_DIRAC: {
                    // DiracD2Q5::initSolver (DiracD2Q5.cpp:39-66) on the host, with
                    // the host's exp: every slot 0.2 x the heat kernel at the
                    // node's distance from (32, 32), then collide at the
                    // fluid's velocity (zero after FluidSolver::initSolver)
                    const double pos = 32, D = 0.04, t = 50;
                    const double PI = std::atan(1) * 4;
                    const double px = (double)(n % (size_t)h.nx), py = (double)(n / (size_t)h.nx);
                    const double dist = std::sqrt((pos - px) * (pos - px) + (pos - py) * (pos - py));
                    const double kernel = std::exp(-dist * dist / (4.0 * D * t)) / (4.0 * PI * D * t);
                    for (int q = 0; q < 5; ++q) gi[q] = kernel * 0.2;
                    collide_cde64(gi, vel ? vel[0] : 0.0, vel ? vel[1] : 0.0, s.c, 0.0, 0.0, dom[n], 0u, 0u);
                    break;
                }
                default:
                    for (int q = 0; q < 5; ++q) gi[q] = 0.0;
            }
            for (int q = 0; q < 5; ++q) g[(size_t)q * L + n] = gi[q];
        }
        if (h.precision == LBIB_FP64) {
            CK(cudaMemcpyAsync((double*)h.g[0] + (size_t)k * 5 * L, g.data(), sizeof(double) * 5 * L,
                               cudaMemcpyHostToDevice, h.stream));
        } else {
            std::vector<float> gf(g.begin(), g.end());
            CK(cudaMemcpyAsync((float*)h.g[0] + (size_t)k * 5 * L, gf.data(), sizeof(float) * 5 * L,
                               cudaMemcpyHostToDevice, h.stream));
        }
        CK(cudaStreamSynchronize(h.stream));
    }
}

// SimulationRunner::initSolvers (SimulationRunner.cpp:290-306), or with a
// velocity initSolvers(Field<double>) (:308-320): every node's FluidSolver
// initSolver (FluidSolver.cpp:50-101) and then its CDE solvers' initSolver.
static void init_lattice(Handle& h, const double* vel) {
    SpeciesConst spc[kMaxSpecies] = {};
    double init[kMaxSpecies] = {0, 0, 0};
    for (int k = 0; k < h.S; ++k) { spc[k] = h.sp[k].c; init[k] = h.sp[k].init; }
    if (h.precision == LBIB_FP64)
        launch_init64((double*)h.f[0], (double*)h.g[0], (double*)h.u, h.S, h.L, h.tauF, h.dom, vel, spc, init,
                      h.stream);
    else
        launch_init32((float*)h.f[0], (float*)h.g[0], (float*)h.u, h.S, h.L, h.tauF, h.dom, vel, spc, init,
                      h.stream);
    init_species_host(h, vel);
    h.cur = 0;
}

static void create(Handle& h, const std::string& params, const std::string& geom, const std::string& forceFile,
                   const std::string& plugins) {
    CK(cudaSetDevice(h.device));
    CK(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h.evA));
    CK(cudaEventCreate(&h.evB));
    load_parameters(h, params);
    load_plugins(h, plugins);
    check_bio(h);
    for (const auto& sp : h.sp) h.cross.diag8 |= sp.c.reinit == RI_DIAG ? 1 : 0;
    h.L = (size_t)h.nx * h.ny;
    const size_t rs = h.precision == LBIB_FP64 ? sizeof(double) : sizeof(float);
    for (int i = 0; i < 2; ++i) {
        CK(cudaMalloc(&h.f[i], 9 * h.L * rs));
        CK(cudaMalloc(&h.g[i], std::max(1, h.S) * 5 * h.L * rs));
    }
    CK(cudaMalloc(&h.u, 2 * h.L * rs));
    CK(cudaMalloc(&h.force, 2 * h.L * rs));
    CK(cudaMemsetAsync(h.force, 0, 2 * h.L * rs, h.stream));
    h.dom = dalloc<uint32_t>(h.L);
    CK(cudaMemsetAsync(h.dom, 0, sizeof(uint32_t) * h.L, h.stream));
    // the status word and the membrane counts share one allocation (and one
    // pinned host copy), so that one copy reads both back after a step
    resize_status_block(h);
    init_kernel_attributes();
    if (const char* e = std::getenv("LBIB_FULL_HOST_EVENTS")) h.fullHostEvents = e[0] == '1';
    // LBIB_NO_GRAPHS=1 launches every stage kernel directly (no CUDA graphs)
    if (const char* e = std::getenv("LBIB_NO_GRAPHS")) h.useGraphs = !(e[0] == '1');
    std::memset(h.stHost, 0, sizeof(Status));
    write_status(h);

    // tiles
    h.tiles.tilesX = (h.nx + kTile - 1) / kTile;
    h.tiles.tilesY = (h.ny + kTile - 1) / kTile;
    h.tiles.nTiles = h.tiles.tilesX * h.tiles.tilesY;
    // count has one extra zero entry: the exclusive scan over nTiles + 1
    // items yields start[nTiles] = total
    h.tiles.count = dalloc<int>(h.tiles.nTiles + 1);
    h.tiles.fill = dalloc<int>(h.tiles.nTiles);
    h.tiles.start = dalloc<int>(h.tiles.nTiles + 1);
    CK(cudaMemsetAsync(h.tiles.count, 0, sizeof(int) * (h.tiles.nTiles + 1), h.stream));
    cub::DeviceScan::ExclusiveSum(nullptr, h.tiles.scanTmpBytes, h.tiles.count, h.tiles.start, h.tiles.nTiles + 1, h.stream);
    CK(cudaMalloc(&h.tiles.scanTmp, std::max<size_t>(h.tiles.scanTmpBytes, 16)));
    if (h.precision == LBIB_FP32_SHIFTED) h.tiles.slots = dalloc<int>((size_t)h.tiles.nTiles * kTileSlots);

    // crossing planes
    h.cross.bnDist = dalloc<unsigned long long>(4 * h.L);
    h.cross.bnConn = dalloc<uint32_t>(4 * h.L);
    h.cross.bnDom = dalloc<uint32_t>(4 * h.L);
    h.cross.wDom = dalloc<uint32_t>(h.L);
    h.cross.mark = dalloc<int>(h.L);
    CK(cudaMemsetAsync(h.cross.mark, 0, sizeof(int) * h.L, h.stream));
    CK(cudaMemsetAsync(h.cross.bnDist, 0xff, sizeof(unsigned long long) * 4 * h.L, h.stream));
    CK(cudaMemsetAsync(h.cross.bnConn, 0xff, sizeof(uint32_t) * 4 * h.L, h.stream));
    CK(cudaMemsetAsync(h.cross.wDom, 0, sizeof(uint32_t) * h.L, h.stream));
    bool bounce = false;
    for (const auto& s : h.sp) bounce |= s.c.bounce != 0;
    if (bounce) {
        // DiracD2Q5: the W / S boundary-node marks its advect reads
        h.cross.bounceW = dalloc<uint8_t>(h.L);
        h.cross.bounceS = dalloc<uint8_t>(h.L);
        CK(cudaMemsetAsync(h.cross.bounceW, 0, h.L, h.stream));
        CK(cudaMemsetAsync(h.cross.bounceS, 0, h.L, h.stream));
        h.cross.bounceCap = (int)std::min<size_t>(2 * h.L, 0x7fffffff);
        h.cross.bounceKeys = dalloc<uint32_t>(h.cross.bounceCap);
        h.cross.bounceN = dalloc<int>(1);
        CK(cudaMemsetAsync(h.cross.bounceN, 0, sizeof(int), h.stream));
    }

    // (h.m.topo points into the status allocation, set with it)

    // geometry: Geometry::loadGeometryTXT (Geometry.cpp:99-160), or for a
    // ".vtm" file loadGeometryVTK (Geometry.cpp:162-306, the choice made at
    // Geometry.cpp:61-71); each new GeometryNode runs perturbatePosition
    // (GeometryNode.cpp:98-117), in the order the nodes are created.
    std::map<uint32_t, std::pair<double, double>> nodes;
    std::map<uint32_t, uint32_t> ctypes;
    ctypes[0] = 0;
    std::string line;
    bool readingNodes = true;
    uint32_t maxDom = 0;
    const bool vtm = geom.size() >= 4 && geom.compare(geom.size() - 4, 4, ".vtm") == 0;
    std::ifstream in;
    if (vtm) {
        vtk::Geometry vg;
        try {
            vtk::read_vtm_geometry(geom, vg);
        } catch (const std::runtime_error& e) {
            fail(ERR_INPUT, e.what());
        }
        for (size_t k = 0; k < vg.x.size(); ++k) {
            double x = vg.x[k], y = vg.y[k];
            perturbate(h, x, y);
            nodes[(uint32_t)k] = {x, y};
        }
        for (const auto& c : vg.conns) {
            h.conns.push_back(HConn{c.id1, c.id2, c.dom, c.desc});
            maxDom = std::max(maxDom, c.dom);
        }
        for (const auto& kv : vg.cellType) ctypes[kv.first] = kv.second;
    } else {
        in.open(geom);
        if (!in.is_open()) fail(ERR_INPUT, "Cannot find the geometry.txt file.");
    }
    while (!vtm && std::getline(in, line)) {
        if (line.empty()) continue;
        if (line.find("#Connection") != std::string::npos) readingNodes = false;
        if (line[0] == '#') continue;
        std::stringstream ls(line);
        if (readingNodes) {
            uint32_t id; double x, y;
            ls >> id >> x >> y;
            perturbate(h, x, y);
            nodes[id] = {x, y};
        } else {
            HConn c;
            ls >> c.id1 >> c.id2 >> c.dom;
            std::string a, b;
            while (ls >> a >> b) c.desc += "\t" + a + "\t" + b;
            ctypes[c.dom] = 1;
            maxDom = std::max(maxDom, c.dom);
            h.conns.push_back(c);
        }
    }
    HostMembrane hm;
    for (auto& kv : nodes) {
        h.ids.push_back(kv.first);
        hm.x.push_back(kv.second.first);
        hm.y.push_back(kv.second.second);
        hm.ox.push_back(kv.second.first - 5.0);
        hm.oy.push_back(kv.second.second - 5.0);
        hm.bx.push_back(kv.second.first);   // bound by cureLattice's edge check
        hm.by.push_back(kv.second.second);
        hm.vx.push_back(0.0); hm.vy.push_back(0.0); hm.fx.push_back(0.0); hm.fy.push_back(0.0);
    }
    // tables indexed by domain id
    for (auto& s : h.sp)
        for (auto& kv : s.source) maxDom = std::max(maxDom, kv.first);
    h.nDomains = (int)maxDom + 1;
    h.massTab = dalloc<double>(h.nDomains);
    CK(cudaMemsetAsync(h.massTab, 0, sizeof(double) * h.nDomains, h.stream));
    // per-node sources: growth, or an area regulator in a run whose cell
    // division changes domains after the bio step
    const bool areaDiv = std::count(h.bio.begin(), h.bio.end(), 2) && std::count(h.bio.begin(), h.bio.end(), 4);
    const bool growth = std::count(h.bio.begin(), h.bio.end(), 6) > 0;
    if (growth || areaDiv) {
        h.massNode = dalloc<double>(h.L);
        CK(cudaMemsetAsync(h.massNode, 0, sizeof(double) * h.L, h.stream));
    }
    std::vector<double> src((size_t)std::max(1, h.S) * h.nDomains, 0.0);
    for (int k = 0; k < h.S; ++k)
        for (auto& kv : h.sp[k].source) src[(size_t)k * h.nDomains + kv.first] = kv.second;
    h.srcTab = dalloc<double>(src.size());
    CK(cudaMemcpyAsync(h.srcTab, src.data(), sizeof(double) * src.size(), cudaMemcpyHostToDevice, h.stream));
    h.ctypeHost.assign(h.nDomains, 1);
    for (auto& kv : ctypes)
        if (kv.first < (uint32_t)h.nDomains) h.ctypeHost[kv.first] = kv.second;
    h.ctypeTab = dalloc<uint32_t>(h.nDomains);
    CK(cudaMemcpyAsync(h.ctypeTab, h.ctypeHost.data(), sizeof(uint32_t) * h.nDomains, cudaMemcpyHostToDevice, h.stream));

    if (!forceFile.empty()) {
        std::ifstream fin(forceFile);
        if (!fin.is_open()) fail(ERR_INPUT, "Cannot find the force solver file.");
        while (std::getline(fin, line)) {
            if (line.empty()) fail(ERR_INPUT, "empty line in the force file");
            if (line[0] == '#') continue;
            add_force_line(h, line);
        }
    }
    h.forcesPureAtLoad = h.forcemap.empty();
    h.forceListIt = h.iteration;

    upload_topology(h, hm, false);
    {
        std::vector<int> z(h.m.M + 1, 0);
        CK(cudaMemcpyAsync(h.m.foff, z.data(), sizeof(int) * z.size(), cudaMemcpyHostToDevice, h.stream));
    }
    setup_boundary_solvers(h);
    cure_lattice(h, hm);

    if (h.cross.bounceW != nullptr) {
        // the lattice kernels carry DiracD2Q5's advect for the plain fluid only
        if (h.forceModel != FM_LUO || h.massNode != nullptr || h.cross.nfTab != nullptr)
            fail(ERR_INPUT, "DiracD2Q5 runs with the Luo force model, without per-node mass sources and "
                            "without boundary solvers on connections");
        for (const auto& s : h.sp)
            if (coupled_kind(s.c.kind)) fail(ERR_INPUT, "DiracD2Q5 runs without coupled reactions");
    }
    // SimulationRunner::initSolvers (SimulationRunner.cpp:290-306)
    init_lattice(h, nullptr);
    // SimulationRunner::initForceSolver: the force list
    if (!h.forcemap.empty()) upload_topology(h, hm, true);
    CK(cudaStreamSynchronize(h.stream));
    CK(cudaGetLastError());
}

// GeometryHandler::cureLattice (GeometryHandler.cpp:149-170): perturb the
// connections, bind the stencils (edge test), generate the crossings and set
// every domain id by the row scan.  No species reinitialisation happens here.
// The boundary solvers named on the connections ("bsolver cdesolver" pairs,
// Geometry.cpp:122-151; Connection::connectionType_ is a map from solver name
// to the CDE solvers in file order; BoundaryNode creates the solvers in the
// map's name order, BoundaryNode.cpp:35-46).  Unknown names fail like the
// reference's factories and getCDESolverSlow.
static void setup_boundary_solvers(Handle& h) {
    std::vector<NfSpec> tab(h.descTable.size());
    bool any = false;
    for (size_t i = 0; i < h.descTable.size(); ++i) {
        std::map<std::string, std::vector<std::string>> type;
        std::stringstream ls(h.descTable[i]);
        std::string bs, cde;
        while (ls >> bs >> cde) type[bs].push_back(cde);
        NfSpec sp{};
        for (const auto& kv : type) {
            if (sp.nSolvers == 2) fail(ERR_INPUT, "more than two boundary solvers on a connection");
            NfSolver& so = sp.s[sp.nSolvers++];
            if (kv.first == "BoundarySolverNoFlux") so.kind = NF_NOFLUX;
            else if (kv.first == "BoundarySolverNoFluxD2Q5") so.kind = NF_NOFLUX_D2Q5;
            else fail(ERR_INPUT, "unknown boundary solver " + kv.first);
            if (kv.second.size() > 4) fail(ERR_INPUT, "more than four CDE solvers for one boundary solver");
            for (const auto& name : kv.second) {
                int k = -1;
                for (int j = 0; j < h.S; ++j)
                    if (h.sp[j].name == name) k = j;
                if (k < 0) fail(ERR_INPUT, "boundary solver for an unknown CDE solver " + name);
                so.cde[so.nCde++] = k;
            }
        }
        any |= sp.nSolvers > 0;
        tab[i] = sp;
    }
    if (!any) return;
    if (tab.size() > 255) fail(ERR_INPUT, "more than 255 distinct connection descriptors");
    h.nfTabDev = dalloc<NfSpec>(tab.size());
    CK(cudaMemcpyAsync(h.nfTabDev, tab.data(), sizeof(NfSpec) * tab.size(), cudaMemcpyHostToDevice, h.stream));
    h.cross.nfTab = h.nfTabDev;
    h.cross.nfSpec = dalloc<uint8_t>(4 * h.L);
    CK(cudaMemsetAsync(h.cross.nfSpec, 0, 4 * h.L, h.stream));
    h.cross.nfU = dalloc<double>(8 * h.L);
    h.cross.nfN = dalloc<int>(1);
    CK(cudaMemsetAsync(h.cross.nfN, 0, sizeof(int), h.stream));
}

static void cure_lattice(Handle& h, HostMembrane& hm) {
    perturb_connections(h, hm);
    CK(cudaMemcpyAsync(h.m.x, hm.x.data(), sizeof(double) * hm.x.size(), cudaMemcpyHostToDevice, h.stream));
    CK(cudaMemcpyAsync(h.m.y, hm.y.data(), sizeof(double) * hm.y.size(), cudaMemcpyHostToDevice, h.stream));
    std::memset(h.stHost, 0, sizeof(Status));
    write_status(h);
    launch_edge_check(h.m, h.nx, h.ny, h.st, 0, h.stream);
    if (h.precision == LBIB_FP64) launch_crossings<double>(h.m, h.cross, h.dom, h.nx, h.ny, h.L, h.st, 0, h.stream);
    else launch_crossings<float>(h.m, h.cross, h.dom, h.nx, h.ny, h.L, h.st, 0, h.stream);
    launch_domain_fill(h.cross, h.dom, h.nx, h.ny, h.L, h.st, 0, h.stream);
    // the crossings mark the nodes whose domain they change; at set-up no
    // re-initialisation follows to clear the marks
    CK(cudaMemsetAsync(h.cross.mark, 0, sizeof(int) * h.L, h.stream));
    read_status(h);
    if (h.stHost->err) fail(h.stHost->err, "lattice set-up failed", h.stHost->errIndex);
    std::memset(h.stHost, 0, sizeof(Status));
    write_status(h);
}

// ---------------------------------------------------------------------------
// Differentiated runs (lbib_diff_*): frozen geometry, FP64, checkpoints every
// K steps and segment-by-segment recomputation in the backward pass.

static void diff_begin(Handle& h, int T, int K) {
    delete h.diff;
    h.diff = nullptr;
    pull_topology(h);
    const size_t L = h.L;
    const int S = h.S;
    const int nSeg = (T + K - 1) / K;
    const int rs = h.precision == LBIB_FP64 ? 8 : 4;
    const size_t stateElems = (size_t)(9 + 5 * S) * L;
    const size_t stateBytes = stateElems * rs;
    const size_t states = 1 + (size_t)(nSeg - 1) + (size_t)(K - 1) + 1;
    const size_t nPart = (size_t)adjoint_blocks(h.nx, h.ny) * (1 + S);
    const size_t bytes = states * stateBytes + 2 * stateElems * sizeof(float) +
                         sizeof(double) * (22 * L + 2 * (size_t)S * L + nPart + 4 * (size_t)h.Mcap +
                                           2 * (size_t)S * h.nDomains + 2 * (size_t)h.nDomains + 1 + S);
    size_t freeB = 0, totalB = 0;
    CK(cudaMemGetInfo(&freeB, &totalB));
    if (bytes + (256u << 20) > freeB)
        fail(ERR_CAPACITY, "differentiated run needs " + std::to_string(bytes >> 20) + " MiB of device memory, " +
                               std::to_string(freeB >> 20) + " MiB free (raise K or lower T)");
    std::unique_ptr<DiffCtx> d(new DiffCtx());
    d->T = T; d->K = K; d->nSeg = nSeg; d->stateBytes = stateBytes; d->rs = rs;
    d->x0 = dalloc<char>(stateBytes);
    d->u0 = dalloc<char>(4 * L * rs);
    d->ck = dalloc<char>((size_t)(nSeg - 1) * stateBytes);
    d->seg = dalloc<char>((size_t)(K - 1) * stateBytes);
    d->fin = dalloc<char>(stateBytes);
    d->P[0] = dalloc<float>(stateElems);
    d->P[1] = dalloc<float>(stateElems);
    d->G = dalloc<double>(2 * L);
    d->force = dalloc<double>(2 * L);
    if (rs == 4) d->force32 = dalloc<float>(2 * L);
    d->fxp = dalloc<double>(h.Mcap); d->fyp = dalloc<double>(h.Mcap);
    d->gfx = dalloc<double>(h.Mcap); d->gfy = dalloc<double>(h.Mcap);
    d->srcTab = dalloc<double>((size_t)S * h.nDomains);
    d->seed = dalloc<double>((size_t)S * L);
    d->grad = dalloc<double>(1 + S + (size_t)(S + 1) * h.nDomains);
    d->racc = dalloc<double>((size_t)S * L);
    d->massTab = dalloc<double>(h.nDomains);
    d->macc = dalloc<double>(L);
    d->seedF = dalloc<double>(9 * L);
    {
        // the frozen mass table: the area regulator's last rates, or none
        bool area = false;
        for (int b : h.bio) area |= (b == 2);
        d->massUsed = area;
        if (area) CK(cudaMemcpyAsync(d->massTab, h.massTab, sizeof(double) * h.nDomains, cudaMemcpyDeviceToDevice,
                                     h.stream));
        else CK(cudaMemsetAsync(d->massTab, 0, sizeof(double) * h.nDomains, h.stream));
    }
    d->part = dalloc<double>(nPart);
    d->st = dalloc<Status>(1);
    const char* serial = std::getenv("LBIB_DIFF_SERIAL");  // diagnostic: one segment buffer
    if (rs == 4 && nSeg >= 2 && K >= 2 && !(serial && serial[0] == '1')) {
        // the second segment buffer only where it leaves 2 GiB free
        const size_t segBytes = (size_t)(K - 1) * stateBytes;
        CK(cudaMemGetInfo(&freeB, &totalB));
        if (segBytes + (size_t(2) << 30) <= freeB) {
            d->seg2 = dalloc<char>(segBytes);
            int least = 0, greatest = 0;
            CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
            CK(cudaStreamCreateWithPriority(&d->recStream, cudaStreamNonBlocking, least));
            CK(cudaStreamCreateWithPriority(&d->adjStream, cudaStreamNonBlocking, greatest));
            for (cudaEvent_t* e : {&d->evRec[0], &d->evRec[1], &d->evAdj[0], &d->evAdj[1], &d->evFork, &d->evJoin[0],
                                   &d->evJoin[1]})
                CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        }
    }
    CK(cudaMemsetAsync(d->st, 0, sizeof(Status), h.stream));
    CK(cudaMemsetAsync(d->force, 0, sizeof(double) * 2 * L, h.stream));
    // snapshot of the lattice and the run's default parameters
    CK(cudaMemcpyAsync(d->x0, h.f[h.cur], 9 * L * rs, cudaMemcpyDeviceToDevice, h.stream));
    if (S) CK(cudaMemcpyAsync(d->x0 + 9 * L * rs, h.g[h.cur], 5 * S * L * rs, cudaMemcpyDeviceToDevice, h.stream));
    CK(cudaMemcpyAsync(d->u0, h.u, 2 * L * rs, cudaMemcpyDeviceToDevice, h.stream));
    CK(cudaMemcpyAsync(d->u0 + 2 * L * rs, h.force, 2 * L * rs, cudaMemcpyDeviceToDevice, h.stream));
    if (S) CK(cudaMemcpyAsync(d->srcTab, h.srcTab, sizeof(double) * S * h.nDomains, cudaMemcpyDeviceToDevice, h.stream));
    if (h.m.M) {
        CK(cudaMemcpyAsync(d->fxp, h.m.fx, sizeof(double) * h.m.M, cudaMemcpyDeviceToDevice, h.stream));
        CK(cudaMemcpyAsync(d->fyp, h.m.fy, sizeof(double) * h.m.M, cudaMemcpyDeviceToDevice, h.stream));
    }
    d->tauF = h.tauF;
    for (int k = 0; k < S; ++k) d->tau[k] = h.sp[k].c.tau;
    d->outlet = h.outlet ? 1 : 0;
    d->it0 = h.iteration;
    CK(cudaStreamSynchronize(h.stream));
    h.diff = d.release();
}

static bool diff_needs_iteration(const Handle& h) {
    for (int k = 0; k < h.S; ++k)
        if (h.sp[k].c.kind == RX_SIGNAL) return true;
    return false;
}

// Forward step t of the differentiated run: state `in` (after step t-1) to
// `out`, in the handle's lattice precision.
template <typename Real>
static void diff_forward_step_t(Handle& h, DiffCtx& d, const char* in, char* out, int t, cudaStream_t stream) {
    const unsigned it = d.it0 + (unsigned)(t - 1);
    if (diff_needs_iteration(h)) launch_set_iteration(d.st, it, stream);
    LatticeArgs<Real> a = lattice_args<Real>(h, it, h.cur);
    a.fin = (const Real*)in; a.fout = (Real*)out;
    a.gin = (const Real*)in + 9 * h.L; a.gout = (Real*)out + 9 * h.L;
    a.force = sizeof(Real) == 8 ? (const Real*)d.force : (const Real*)d.force32;
    a.srcTab = d.srcTab;
    a.massTab = d.massUsed ? d.massTab : nullptr;
    a.tauF = d.tauF;
    for (int k = 0; k < h.S; ++k) a.sp[k].tau = d.tau[k];
    a.status = d.st;
    a.outlet = d.outlet;
    if (sizeof(Real) == 8) launch_stream_collide64(*(const LatticeArgs<double>*)&a, stream);
    else launch_stream_collide32(*(const LatticeArgs<float>*)&a, stream);
}

// Step t of a run with moving membrane nodes: the node forces spread from
// the positions after step t-1, the lattice step, then (move) the positions
// after step t.  The reverse pass replays it without the move: the positions
// of every step are stored.
static void diff_motion_spread(Handle& h, DiffCtx& d, int t, cudaStream_t stream) {
    const double* X = d.posAt(t - 1);
    CK(cudaMemsetAsync(d.force, 0, sizeof(double) * 2 * h.L, stream));
    launch_motion_spread(X, X + d.M, d.fxp, d.fyp, d.M, h.nx, h.ny, h.L, d.force, d.st, stream);
    if (d.rs == 4) launch_to_float(d.force, d.force32, 2 * h.L, stream);
}

static void diff_forward_step(Handle& h, DiffCtx& d, const char* in, char* out, int t, cudaStream_t stream,
                              bool move = false) {
    if (d.motion) diff_motion_spread(h, d, t, stream);
    if (d.rs == 8) diff_forward_step_t<double>(h, d, in, out, t, stream);
    else diff_forward_step_t<float>(h, d, in, out, t, stream);
    if (d.motion && move) {
        const double* X0 = d.posAt(t - 1);
        double* X1 = d.posAt(t);
        if (d.rs == 8)
            launch_motion_move<double>(X0, X0 + d.M, X1, X1 + d.M, d.M, (const double*)h.u, h.nx, h.ny, h.L, d.st,
                                       stream);
        else
            launch_motion_move<float>(X0, X0 + d.M, X1, X1 + d.M, d.M, (const float*)h.u, h.nx, h.ny, h.L, d.st,
                                      stream);
    }
}

static void diff_check_status(Handle& h, DiffCtx& d) {
    Status st{};
    CK(cudaMemcpyAsync(&st, d.st, sizeof(Status), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    if (st.err) fail(st.err, "differentiated run: device error in the force spread", st.errIndex);
}

static void diff_forward(Handle& h, DiffCtx& d) {
    const size_t L = h.L;
    MembraneDev mp = h.m;
    mp.fx = d.fxp;
    mp.fy = d.fyp;
    if (!d.motion) {
        // after a moving-node pass the field holds values outside the force tiles
        if (d.pos != nullptr) CK(cudaMemsetAsync(d.force, 0, sizeof(double) * 2 * L, h.stream));
        launch_spread<double>(mp, h.tiles, d.force, h.nx, h.ny, L, d.st, d.it0, h.stream);
        if (d.rs == 4) launch_to_float(d.force, d.force32, 2 * L, h.stream);
    }
    // two scratch states for the steps between checkpoints (the segment
    // buffer, free during the forward pass; with K = 2 one is enough, with
    // K = 1 every state but the last is a checkpoint)
    char* scratch[2] = {d.seg, d.K > 2 ? d.seg + d.stateBytes : d.seg};
    // the last segment's states go where the reverse pass reads them, so that
    // it need not recompute that segment
    const int lastBase = (d.nSeg - 1) * d.K;
    const char* in = d.x0;
    char* out = nullptr;
    for (int t = 1; t <= d.T; ++t) {
        if (t % d.K == 0 && t < d.T) out = d.state(t / d.K);
        else if (t == d.T) out = d.fin;
        else if (t > lastBase) out = d.seg + (size_t)(t - lastBase - 1) * d.stateBytes;
        else out = scratch[t & 1];
        diff_forward_step(h, d, in, out, t, h.stream, true);
        in = out;
    }
    d.lastSegKept = true;
    // the final state and the force field become the handle's lattice, for
    // lbib_download_lattice
    if (d.rs == 8) CK(cudaMemcpyAsync(h.force, d.force, sizeof(double) * 2 * L, cudaMemcpyDeviceToDevice, h.stream));
    else CK(cudaMemcpyAsync(h.force, d.force32, sizeof(float) * 2 * L, cudaMemcpyDeviceToDevice, h.stream));
    CK(cudaMemcpyAsync(h.f[h.cur], in, 9 * L * d.rs, cudaMemcpyDeviceToDevice, h.stream));
    if (h.S)
        CK(cudaMemcpyAsync(h.g[h.cur], in + 9 * L * d.rs, 5 * h.S * L * d.rs, cudaMemcpyDeviceToDevice, h.stream));
    CK(cudaGetLastError());
    diff_check_status(h, d);
    d.forwardDone = true;
}

static void diff_backward(Handle& h, DiffCtx& d) {
    const size_t L = h.L;
    const int S = h.S;
    CK(cudaMemsetAsync(d.G, 0, sizeof(double) * 2 * L, h.stream));
    CK(cudaMemsetAsync(d.grad, 0, sizeof(double) * (1 + S + (size_t)(S + 1) * h.nDomains), h.stream));
    if (S) CK(cudaMemsetAsync(d.racc, 0, sizeof(double) * S * L, h.stream));
    CK(cudaMemsetAsync(d.macc, 0, sizeof(double) * L, h.stream));
    CK(cudaMemsetAsync(d.part, 0, sizeof(double) * adjoint_blocks(h.nx, h.ny) * (1 + S), h.stream));
    AdjointArgs a{};
    a.nx = h.nx; a.ny = h.ny; a.L = L; a.S = S;
    a.force = d.force;
    a.dom = h.dom;
    a.massTab = d.massUsed ? d.massTab : nullptr;
    a.macc = d.massUsed ? d.macc : nullptr;
    a.nDomains = h.nDomains;
    a.srcTab = d.srcTab;
    a.tauIF = 1.0 / d.tauF;
    for (int k = 0; k < S; ++k) {
        a.sp[k] = h.sp[k].c;
        a.sp[k].tau = d.tau[k];
        a.tauI[k] = 1.0 / d.tau[k];
    }
    a.outlet = d.outlet;
    a.G = d.G;
    a.racc = d.racc;
    a.part = d.part;
    a.grad = d.grad;
    // Segment s (steps base+1 .. base+len) is reversed from the states
    // base .. base+len-1: the checkpoint, then its recomputed states in a
    // segment buffer (d.seg always, or alternately d.seg and d.seg2).
    // (a run with moving nodes refills the one force field every step: serial)
    const bool two = d.seg2 != nullptr && !d.motion;
    if (d.motion) {
        if (d.haveSeedX)
            CK(cudaMemcpyAsync(d.lam, d.seedX, sizeof(double) * 2 * d.M, cudaMemcpyDeviceToDevice, h.stream));
        else CK(cudaMemsetAsync(d.lam, 0, sizeof(double) * 2 * d.M, h.stream));
        if (d.M) {
            CK(cudaMemsetAsync(d.gfx, 0, sizeof(double) * d.M, h.stream));
            CK(cudaMemsetAsync(d.gfy, 0, sizeof(double) * d.M, h.stream));
        }
    }
    auto bufOf = [&](int s) -> char* { return two && ((d.nSeg - 1 - s) & 1) ? d.seg2 : d.seg; };
    auto segState = [&](int s, int j) -> char* {  // state s*K + j, 0 <= j < len
        return j == 0 ? d.state(s) : bufOf(s) + (size_t)(j - 1) * d.stateBytes;
    };
    auto segLen = [&](int s) { return std::min(d.K, d.T - s * d.K); };
    auto recompute = [&](int s, cudaStream_t stream) {
        for (int j = 1; j < segLen(s); ++j)
            diff_forward_step(h, d, segState(s, j - 1), segState(s, j), s * d.K + j, stream);
    };
    auto reverse = [&](int s, cudaStream_t stream) {
        const int base = s * d.K;
        for (int t = base + segLen(s); t > base; --t) {
            const char* prev = segState(s, t - 1 - base);
            a.fprev = prev;
            a.gprev = prev + 9 * L * d.rs;
            a.fp32 = d.rs == 4;
            const bool seedStep = t == d.T;
            // the adjoint planes are FP32 (in the first half of the state-sized buffers)
            const float* pin = d.P[(t + 1) & 1];
            a.pf = seedStep ? nullptr : pin;
            a.pg = seedStep ? nullptr : pin + 9 * L;
            a.seed = seedStep ? d.seed : nullptr;
            a.seedF = seedStep && d.haveSeedF ? d.seedF : nullptr;
            a.qf = d.P[t & 1];
            a.qg = d.P[t & 1] + 9 * L;
            a.iteration = d.it0 + (unsigned)(t - 1);
            a.chained = t < base + segLen(s);  // the segment's first step follows its recompute
            if (!d.motion) {
                launch_adjoint_step64(a, stream);
                continue;
            }
            // moving nodes: dL/du of this step is the spread of dL/dX after
            // it (the interpolation's transpose), the force field is the one
            // spread from the step-start positions, and the step's G and
            // velocity then carry dL/dX back to those positions
            const double* X = d.posAt(t - 1);
            CK(cudaMemsetAsync(d.gu, 0, sizeof(double) * 2 * L, stream));
            launch_motion_spread(X, X + d.M, d.lam, d.lam + d.M, d.M, h.nx, h.ny, L, d.gu, d.st, stream);
            CK(cudaMemsetAsync(d.force, 0, sizeof(double) * 2 * L, stream));
            launch_motion_spread(X, X + d.M, d.fxp, d.fyp, d.M, h.nx, h.ny, L, d.force, d.st, stream);
            a.gu = d.gu;
            a.uo = d.uo;
            a.chained = 0;
            launch_adjoint_step64_motion(a, stream);
            launch_motion_adjoint(X, X + d.M, d.fxp, d.fyp, d.lam, d.lam + d.M, d.uo, d.G, d.gfx, d.gfy, d.M, h.nx,
                                  h.ny, L, stream);
        }
    };
    const bool keptLast = d.lastSegKept;
    if (!two) {
        for (int s = d.nSeg - 1; s >= 0; --s) {
            if (!(s == d.nSeg - 1 && keptLast)) recompute(s, h.stream);
            if (s < d.nSeg - 1) d.lastSegKept = false;  // seg now holds an earlier segment
            reverse(s, h.stream);
        }
    } else {
        // Segment s-1 is recomputed while segment s is reversed.  Its buffer
        // was last read by the reverse pass of segment s+1, which it waits for.
        CK(cudaEventRecord(d.evFork, h.stream));
        CK(cudaStreamWaitEvent(d.recStream, d.evFork, 0));
        CK(cudaStreamWaitEvent(d.adjStream, d.evFork, 0));
        auto issueRecompute = [&](int s) {
            const int b = (d.nSeg - 1 - s) & 1;
            if (s + 2 <= d.nSeg - 1) CK(cudaStreamWaitEvent(d.recStream, d.evAdj[b], 0));
            if (!(s == d.nSeg - 1 && keptLast)) recompute(s, d.recStream);
            CK(cudaEventRecord(d.evRec[b], d.recStream));
        };
        issueRecompute(d.nSeg - 1);
        issueRecompute(d.nSeg - 2);
        for (int s = d.nSeg - 1; s >= 0; --s) {
            const int b = (d.nSeg - 1 - s) & 1;
            CK(cudaStreamWaitEvent(d.adjStream, d.evRec[b], 0));
            reverse(s, d.adjStream);
            CK(cudaEventRecord(d.evAdj[b], d.adjStream));
            if (s - 2 >= 0) issueRecompute(s - 2);
        }
        CK(cudaEventRecord(d.evJoin[0], d.recStream));
        CK(cudaEventRecord(d.evJoin[1], d.adjStream));
        CK(cudaStreamWaitEvent(h.stream, d.evJoin[0], 0));
        CK(cudaStreamWaitEvent(h.stream, d.evJoin[1], 0));
        // d.seg holds the last segment unless an earlier one went there
        d.lastSegKept = d.nSeg < 3;
    }
    launch_adjoint_finish(a, h.stream);
    if (!d.motion) launch_force_adjoint(h.m, d.G, h.nx, h.ny, L, d.gfx, d.gfy, h.stream);
    CK(cudaGetLastError());
}

// Switches a differentiated run to moving membrane nodes (lbib_diff_motion).
static void diff_set_motion(Handle& h, DiffCtx& d, bool on) {
    if (!on) {
        d.motion = false;
        return;
    }
    if (d.motion) return;
    if (d.pos != nullptr) {  // switched on before: the buffers and the snapshot positions are kept
        d.motion = true;
        d.forwardDone = false;
        return;
    }
    const size_t L = h.L;
    const int M = h.m.M;
    const size_t bytes = sizeof(double) * ((size_t)(d.T + 1) * 2 * M + 4 * (size_t)M + 4 * L);
    size_t freeB = 0, totalB = 0;
    CK(cudaMemGetInfo(&freeB, &totalB));
    if (bytes + (256u << 20) > freeB)
        fail(ERR_CAPACITY, "moving-node differentiated run needs " + std::to_string(bytes >> 20) +
                               " MiB of device memory, " + std::to_string(freeB >> 20) + " MiB free");
    d.M = M;
    d.pos = dalloc<double>((size_t)(d.T + 1) * 2 * M + 1);
    d.lam = dalloc<double>(2 * (size_t)M + 1);
    d.seedX = dalloc<double>(2 * (size_t)M + 1);
    d.gu = dalloc<double>(2 * L);
    d.uo = dalloc<double>(2 * L);
    if (M) {
        CK(cudaMemcpyAsync(d.pos, h.m.x, sizeof(double) * M, cudaMemcpyDeviceToDevice, h.stream));
        CK(cudaMemcpyAsync(d.pos + M, h.m.y, sizeof(double) * M, cudaMemcpyDeviceToDevice, h.stream));
    }
    CK(cudaStreamSynchronize(h.stream));
    d.motion = true;
    d.forwardDone = false;
}

}  // namespace lbib

// ---------------------------------------------------------------------------
// C ABI

using lbib::Handle;
using lbib::HostFail;

struct lbib_handle {
    Handle h;
};

#define API_BEGIN(hh)                                    \
    if (!(hh)) return LBIB_ERR_STATE;                    \
    Handle& h = (hh)->h;                                 \
    if (h.err) return h.err;                             \
    h.areaFresh = false;                                 \
    try {                                                \
        cudaSetDevice(h.device);
#define API_END                                          \
    } catch (const HostFail& e) {                        \
        h.err = e.code; h.msg = e.msg; h.errIndex = e.index; \
        return e.code;                                   \
    } catch (const std::exception& e) {                  \
        h.err = LBIB_ERR_INPUT; h.msg = e.what();        \
        return h.err;                                    \
    }                                                    \
    return LBIB_OK;

extern "C" {

int lbib_create_from_files(const char* parameters, const char* geometry, const char* force, const char* plugins,
                           int precision, int device, lbib_handle** out) {
    if (!out || !parameters || !geometry) return LBIB_ERR_INPUT;
    if (precision != LBIB_FP64 && precision != LBIB_FP32_SHIFTED) return LBIB_ERR_INPUT;
    lbib_handle* hh = new lbib_handle();
    *out = hh;
    Handle& h = hh->h;
    h.precision = precision;
    h.device = device;
    try {
        lbib::create(h, parameters, geometry, force ? force : "", plugins ? plugins : "");
    } catch (const HostFail& e) {
        h.err = e.code; h.msg = e.msg; h.errIndex = e.index;
        return e.code;
    } catch (const std::exception& e) {
        h.err = LBIB_ERR_INPUT; h.msg = e.what();
        return h.err;
    }
    return LBIB_OK;
}

int lbib_destroy(lbib_handle* hh) {
    delete hh;
    return LBIB_OK;
}

int lbib_step(lbib_handle* hh, int n) {
    API_BEGIN(hh)
    if (n < 0) lbib::fail(LBIB_ERR_INPUT, "negative step count");
    h.lastCollideMs = 0;
    h.lastCollideLaunches = 0;
    h.launches = 0;
    CK(cudaEventRecord(h.evA, h.stream));
    if (h.precision == LBIB_FP64) lbib::run_steps<double>(h, n);
    else lbib::run_steps<float>(h, n);
    // the areas read back with the last status word are those of the state
    // now, unless a host bio solver edited the geometry after the last step
    h.areaFresh = n > 0 && lbib::step_leaves_areas(h) && !lbib::host_bio_at(h, h.iteration - 1);
    // evB was recorded before the last status read (whose synchronisation
    // completed it) unless host work followed
    if (n == 0 || h.workAfterEvB) {
        CK(cudaEventRecord(h.evB, h.stream));
        CK(cudaEventSynchronize(h.evB));
    }
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h.evA, h.evB));
    h.lastTotalMs = ms;
    API_END
}

int lbib_lattice_step(lbib_handle* hh, int n, int outlet) {
    API_BEGIN(hh)
    if (n < 0) lbib::fail(LBIB_ERR_INPUT, "negative step count");
    lbib::reset_status(h, h.iteration, h.cellTypesCopied);
    h.lastCollideMs = 0;
    h.lastCollideLaunches = 0;
    h.launches = (long long)n * 2;
    while ((int)h.kEvents.size() < 2 * n) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        h.kEvents.push_back(e);
    }
    CK(cudaEventRecord(h.evA, h.stream));
    for (int i = 0; i < n; ++i) {
        const int p = h.cur;
        if (h.profiling) CK(cudaEventRecord(h.kEvents[2 * i], h.stream));
        if (h.precision == LBIB_FP64) {
            auto a = lbib::lattice_args<double>(h, h.iteration, p);
            a.outlet = outlet ? 1 : 0;
            lbib::launch_stream_collide64(a, h.stream);
        } else {
            auto a = lbib::lattice_args<float>(h, h.iteration, p);
            a.outlet = outlet ? 1 : 0;
            lbib::launch_stream_collide32(a, h.stream);
        }
        if (h.profiling) CK(cudaEventRecord(h.kEvents[2 * i + 1], h.stream));
        h.cur = 1 - p;
        launch_pdl(lbib::iteration_inc_kernel, 1, 1, 0, h.stream, h.st);
        h.iteration++;
    }
    CK(cudaEventRecord(h.evB, h.stream));
    CK(cudaEventSynchronize(h.evB));
    CK(cudaGetLastError());
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h.evA, h.evB));
    h.lastTotalMs = ms;
    if (h.profiling)
        for (int i = 0; i < n; ++i) {
            float k = 0;
            CK(cudaEventElapsedTime(&k, h.kEvents[2 * i], h.kEvents[2 * i + 1]));
            h.lastCollideMs += k;
            h.lastCollideLaunches++;
        }
    API_END
}

int lbib_get_sizes(lbib_handle* hh, long long* s) {
    if (!hh || !s) return LBIB_ERR_STATE;
    Handle& h = hh->h;
    if (!h.err) {
        // the counts only: one small read, not the whole topology
        lbib::Topo tp{};
        if (cudaSetDevice(h.device) == cudaSuccess &&
            cudaMemcpyAsync(&tp, h.m.topo, sizeof(tp), cudaMemcpyDeviceToHost, h.stream) == cudaSuccess &&
            cudaStreamSynchronize(h.stream) == cudaSuccess) {
            h.m.M = tp.M;
            h.m.C = tp.C;
        } else {
            h.err = LBIB_ERR_CUDA;
            h.msg = "lbib_get_sizes: reading the membrane counts failed";
        }
    }
    s[0] = h.nx; s[1] = h.ny; s[2] = h.S; s[3] = h.m.M; s[4] = h.m.C;
    s[5] = h.iteration; s[6] = h.precision; s[7] = h.hostEvents; s[8] = h.stepsDone; s[9] = h.m.nCells;
    return LBIB_OK;
}

int lbib_download_lattice(lbib_handle* hh, double* f, double* g, double* vel, double* force, unsigned* dom,
                          unsigned* ctype) {
    API_BEGIN(hh)
    const size_t L = h.L;
    const int S = h.S;
    const bool fp64 = h.precision == LBIB_FP64;
    const size_t rs = fp64 ? 8 : 4;
    std::vector<char> buf;
    auto fetch = [&](const void* src, size_t count) {
        buf.resize(count * rs);
        CK(cudaMemcpyAsync(buf.data(), src, count * rs, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
    };
    auto val = [&](size_t i) -> double {
        return fp64 ? ((const double*)buf.data())[i] : (double)((const float*)buf.data())[i];
    };
    static const int INV9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    static const int INV5[5] = {0, 3, 4, 1, 2};
    static const double W9[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                                 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
    if (f) {
        fetch(h.f[h.cur], 9 * L);
        for (size_t n = 0; n < L; ++n)
            for (int d = 0; d < 9; ++d) {
                const int q = INV9[d];
                f[n * 9 + d] = fp64 ? val(q * L + n) : val(q * L + n) + W9[q];
            }
    }
    if (g && S > 0) {
        fetch(h.g[h.cur], (size_t)S * 5 * L);
        for (int k = 0; k < S; ++k)
            for (size_t n = 0; n < L; ++n)
                for (int d = 0; d < 5; ++d) g[((size_t)k * L + n) * 5 + d] = val(((size_t)k * 5 + INV5[d]) * L + n);
    }
    if (vel) {
        fetch(h.u, 2 * L);
        for (size_t n = 0; n < L; ++n) { vel[2 * n] = val(n); vel[2 * n + 1] = val(L + n); }
    }
    if (force) {
        fetch(h.force, 2 * L);
        std::vector<int> tc(h.tiles.nTiles);
        CK(cudaMemcpyAsync(tc.data(), h.tiles.count, sizeof(int) * tc.size(), cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        for (size_t n = 0; n < L; ++n) {
            const int x = (int)(n % h.nx), y = (int)(n / h.nx);
            const bool act = tc[(y / lbib::kTile) * h.tiles.tilesX + x / lbib::kTile] > 0;
            force[2 * n] = act ? val(n) : 0.0;
            force[2 * n + 1] = act ? val(L + n) : 0.0;
        }
    }
    if (dom || ctype) {
        std::vector<uint32_t> d(L);
        CK(cudaMemcpyAsync(d.data(), h.dom, sizeof(uint32_t) * L, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        for (size_t n = 0; n < L; ++n) {
            if (dom) dom[n] = d[n];
            if (ctype) ctype[n] = h.cellTypesCopied ? (d[n] < h.ctypeHost.size() ? h.ctypeHost[d[n]] : 1u) : 0u;
        }
    }
    API_END
}

int lbib_upload_lattice(lbib_handle* hh, const double* f, const double* g, const double* force) {
    API_BEGIN(hh)
    const size_t L = h.L;
    const bool fp64 = h.precision == LBIB_FP64;
    static const int INV9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    static const int INV5[5] = {0, 3, 4, 1, 2};
    static const double W9[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                                 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
    auto put = [&](void* dst, const std::vector<double>& v) {
        if (fp64) {
            CK(cudaMemcpyAsync(dst, v.data(), v.size() * 8, cudaMemcpyHostToDevice, h.stream));
            CK(cudaStreamSynchronize(h.stream));
        } else {
            std::vector<float> fv(v.begin(), v.end());
            CK(cudaMemcpyAsync(dst, fv.data(), fv.size() * 4, cudaMemcpyHostToDevice, h.stream));
            CK(cudaStreamSynchronize(h.stream));
        }
    };
    if (f) {
        std::vector<double> v(9 * L);
        for (size_t n = 0; n < L; ++n)
            for (int d = 0; d < 9; ++d) {
                const int q = INV9[d];
                v[q * L + n] = fp64 ? f[n * 9 + d] : f[n * 9 + d] - W9[q];
            }
        put(h.f[h.cur], v);
    }
    if (g && h.S > 0) {
        std::vector<double> v((size_t)h.S * 5 * L);
        for (int k = 0; k < h.S; ++k)
            for (size_t n = 0; n < L; ++n)
                for (int d = 0; d < 5; ++d) v[((size_t)k * 5 + INV5[d]) * L + n] = g[((size_t)k * L + n) * 5 + d];
        put(h.g[h.cur], v);
    }
    if (force) {
        std::vector<double> v(2 * L);
        for (size_t n = 0; n < L; ++n) { v[n] = force[2 * n]; v[L + n] = force[2 * n + 1]; }
        put(h.force, v);
        // mark every tile active so that the lattice kernels read the field
        std::vector<int> ones(h.tiles.nTiles, 1);
        CK(cudaMemcpyAsync(h.tiles.count, ones.data(), sizeof(int) * ones.size(), cudaMemcpyHostToDevice, h.stream));
        CK(cudaStreamSynchronize(h.stream));
    }
    API_END
}

int lbib_init_velocity(lbib_handle* hh, double ux, double uy) {
    API_BEGIN(hh)
    if (!std::isfinite(ux) || !std::isfinite(uy)) lbib::fail(LBIB_ERR_INPUT, "lbib_init_velocity: non-finite velocity");
    const double vel[2] = {ux, uy};
    lbib::init_lattice(h, vel);
    CK(cudaStreamSynchronize(h.stream));
    CK(cudaGetLastError());
    API_END
}

int lbib_download_membrane(lbib_handle* hh, unsigned* ids, double* state) {
    API_BEGIN(hh)
    lbib::pull_topology(h);
    lbib::HostMembrane hm;
    lbib::download_membrane(h, hm);
    for (size_t i = 0; i < h.ids.size(); ++i) {
        if (ids) ids[i] = h.ids[i];
        if (state) {
            double* o = state + 6 * i;
            o[0] = hm.x[i]; o[1] = hm.y[i]; o[2] = hm.vx[i]; o[3] = hm.vy[i]; o[4] = hm.fx[i]; o[5] = hm.fy[i];
        }
    }
    API_END
}

int lbib_download_connections(lbib_handle* hh, unsigned* conn) {
    API_BEGIN(hh)
    lbib::pull_topology(h);
    for (size_t c = 0; c < h.conns.size(); ++c) {
        conn[3 * c] = h.conns[c].id1; conn[3 * c + 1] = h.conns[c].id2; conn[3 * c + 2] = h.conns[c].dom;
    }
    API_END
}

int lbib_areas(lbib_handle* hh, unsigned* dom, double* area, int cap) {
    if (!hh) return -LBIB_ERR_STATE;
    Handle& h = hh->h;
    if (h.err) return -h.err;
    if (cap < 0 || (cap > 0 && (!dom || !area))) {
        h.msg = "lbib_areas: bad output buffers";
        return -LBIB_ERR_INPUT;
    }
    try {
        CK(cudaSetDevice(h.device));
        // after lbib_step, the areas its bio stage formed are already on the
        // host; otherwise one round trip forms and reads them
        if (!h.areaFresh && h.m.nCells > 0) {
            lbib::reset_status(h, h.iteration, h.cellTypesCopied);
            lbib::queue_areas(h, h.area);
            CK(cudaGetLastError());
            h.statusWithAreas = true;
            lbib::read_status(h);
            if (h.stHost->err) {
                const long long idx = h.stHost->errIndex;
                lbib::reset_status(h, h.iteration, h.cellTypesCopied);
                h.msg = "lbib_areas: cell " + std::to_string(idx) + " has more membrane nodes than one ring may hold";
                h.errIndex = idx;
                return -LBIB_ERR_CAPACITY;
            }
            h.areaFresh = true;
        }
        for (int c = 0; c < h.m.nCells && c < cap; ++c) {
            dom[c] = h.ringDomHost[c];
            area[c] = h.areaPinned[c];
        }
        return h.m.nCells;
    } catch (const HostFail& e) {
        h.err = e.code; h.msg = e.msg;
        return -e.code;
    } catch (const std::exception& e) {
        h.err = LBIB_ERR_INPUT; h.msg = e.what();
        return -h.err;
    }
}

}  // extern "C"

namespace {

// Address of the fixed area array on each device, looked up once per device
// with that device current.
constexpr int kStaticDevices = 64;
std::mutex g_staticMu;
double* g_staticArea[kStaticDevices] = {};

cudaError_t static_area_address(int device, double** out) {
    if (device < 0 || device >= kStaticDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_staticMu);
    if (!g_staticArea[device]) {
        double* p = nullptr;
        const cudaError_t e = lbib::static_area_scratch(&p);
        if (e != cudaSuccess) return e;
        g_staticArea[device] = p;
    }
    *out = g_staticArea[device];
    return cudaSuccess;
}

}  // namespace

extern "C" {

int lbib_areas_static(lbib_handle* hh, unsigned* dom, double* area, int cap) {
    if (!hh) return -LBIB_ERR_STATE;
    Handle& h = hh->h;
    if (h.err) return -h.err;
    if (h.m.nCells > lbib::kStaticAreaCells) {
        h.msg = "lbib_areas_static: " + std::to_string(h.m.nCells) + " cells exceed the fixed device array of " +
                std::to_string(lbib::kStaticAreaCells) + " cells (use lbib_areas)";
        return -LBIB_ERR_CAPACITY;
    }
    if (cap < 0 || (cap > 0 && (!dom || !area))) {
        h.msg = "lbib_areas_static: bad output buffers";
        return -LBIB_ERR_INPUT;
    }
    try {
        CK(cudaSetDevice(h.device));
        double* scratch = nullptr;
        CK(static_area_address(h.device, &scratch));
        lbib::reset_status(h, h.iteration, h.cellTypesCopied);
        // all-ones bytes read back as NaN: a cell the kernel leaves out shows
        // no value of an earlier call (or of another handle sharing the array)
        if (h.m.nCells > 0) CK(cudaMemsetAsync(scratch, 0xFF, sizeof(double) * h.m.nCells, h.stream));
        lbib::queue_areas(h, scratch);
        CK(cudaGetLastError());
        const int n = std::min(h.m.nCells, cap);
        if (n > 0) CK(cudaMemcpyAsync(area, scratch, sizeof(double) * n, cudaMemcpyDeviceToHost, h.stream));
        lbib::read_status(h);
        if (h.stHost->err) {
            const long long idx = h.stHost->errIndex;
            lbib::reset_status(h, h.iteration, h.cellTypesCopied);
            h.msg = "lbib_areas_static: a cell has more membrane nodes than one ring may hold";
            h.errIndex = idx;
            return -LBIB_ERR_CAPACITY;
        }
        for (int c = 0; c < n; ++c) dom[c] = h.ringDomHost[c];
        return h.m.nCells;
    } catch (const HostFail& e) {
        h.err = e.code; h.msg = e.msg;
        return -e.code;
    } catch (const std::exception& e) {
        h.err = LBIB_ERR_INPUT; h.msg = e.what();
        return -h.err;
    }
}

// GeometryHandler::computeAccumulatedDomainConcentrations(name)
// (GeometryHandler.cpp:136-147).
int lbib_accumulated_concentrations(lbib_handle* hh, const char* species, unsigned* dom, double* acc, int cap) {
    if (!hh) return -LBIB_ERR_STATE;
    Handle& h = hh->h;
    if (h.err) return -h.err;
    int count = 0;
    try {
        cudaSetDevice(h.device);
        if (species == nullptr || dom == nullptr || acc == nullptr) lbib::fail(LBIB_ERR_INPUT, "null argument");
        int k = -1;
        for (int j = 0; j < h.S; ++j)
            if (h.sp[j].name == species) k = j;
        if (k < 0) lbib::fail(LBIB_ERR_INPUT, std::string("no CDE solver ") + species);
        const auto m = lbib::accumulated_concentrations(h, k);
        if ((int)m.size() > cap) lbib::fail(LBIB_ERR_CAPACITY, "accumulated concentrations: buffer too small");
        for (const auto& kv : m) {
            dom[count] = kv.first;
            acc[count] = kv.second;
            ++count;
        }
    } catch (const HostFail& e) {
        h.err = e.code; h.msg = e.msg; h.errIndex = e.index;
        return -e.code;
    } catch (const std::exception& e) {
        h.err = LBIB_ERR_INPUT; h.msg = e.what();
        return -h.err;
    }
    return count;
}

// GeometryHandler::getCellTypeTrackerMap()[dom] = type, then
// copyCellTypeToPhysicalNodes (GeometryHandler.cpp:267-314).
int lbib_set_cell_types(lbib_handle* hh, const unsigned* dom, const unsigned* type, int n) {
    API_BEGIN(hh)
    if (n < 0 || (n > 0 && (dom == nullptr || type == nullptr))) lbib::fail(LBIB_ERR_INPUT, "bad cell-type list");
    unsigned top = 0;
    for (int i = 0; i < n; ++i) top = std::max(top, dom[i]);
    if (n > 0) lbib::grow_domains(h, (int)top + 1);
    for (int i = 0; i < n; ++i) h.ctypeHost[dom[i]] = type[i];
    CK(cudaMemcpyAsync(h.ctypeTab, h.ctypeHost.data(), sizeof(uint32_t) * h.nDomains, cudaMemcpyHostToDevice,
                       h.stream));
    CK(cudaStreamSynchronize(h.stream));
    h.cellTypesCopied = true;
    API_END
}

// GeometryHandler::getCellTypeTrackerMap (GeometryHandler.cpp:316-319): the
// type of every domain id below the handle's domain count.
int lbib_get_cell_types(lbib_handle* hh, unsigned* dom, unsigned* type, int cap) {
    if (!hh) return -LBIB_ERR_STATE;
    Handle& h = hh->h;
    if (h.err) return -h.err;
    int count = 0;
    try {
        cudaSetDevice(h.device);
        if (dom == nullptr || type == nullptr) lbib::fail(LBIB_ERR_INPUT, "null argument");
        if ((int)h.ctypeHost.size() > cap) lbib::fail(LBIB_ERR_CAPACITY, "cell types: buffer too small");
        for (size_t d = 0; d < h.ctypeHost.size(); ++d) {
            dom[count] = (unsigned)d;
            type[count] = h.ctypeHost[d];
            ++count;
        }
    } catch (const HostFail& e) {
        h.err = e.code; h.msg = e.msg; h.errIndex = e.index;
        return -e.code;
    } catch (const std::exception& e) {
        h.err = LBIB_ERR_INPUT; h.msg = e.what();
        return -h.err;
    }
    return count;
}

int lbib_set_species_source(lbib_handle* hh, int k, const double* rates, int n) {
    API_BEGIN(hh)
    if (k < 0 || k >= h.S || n < 0 || n > h.nDomains || (n > 0 && !rates))
        lbib::fail(LBIB_ERR_INPUT, "bad species index or table size");
    if (n > 0)
        CK(cudaMemcpyAsync(h.srcTab + (size_t)k * h.nDomains, rates, sizeof(double) * n, cudaMemcpyHostToDevice,
                           h.stream));
    API_END
}

int lbib_set_species_sources(lbib_handle* hh, const double* rates, int n) {
    API_BEGIN(hh)
    if (n != h.nDomains || (h.S > 0 && !rates)) lbib::fail(LBIB_ERR_INPUT, "rates must be S x domain count");
    if (h.S > 0)
        CK(cudaMemcpyAsync(h.srcTab, rates, sizeof(double) * (size_t)h.S * h.nDomains, cudaMemcpyHostToDevice,
                           h.stream));
    API_END
}

int lbib_last_error(lbib_handle* hh, char* buf, int len, long long* index) {
    if (!hh) return LBIB_ERR_STATE;
    Handle& h = hh->h;
    if (buf && len > 0) std::snprintf(buf, len, "%s", h.msg.c_str());
    if (index) *index = h.errIndex;
    return h.err;
}

int lbib_last_timing(lbib_handle* hh, double* out) {
    if (!hh || !out) return LBIB_ERR_STATE;
    out[0] = hh->h.lastTotalMs;
    out[1] = hh->h.lastCollideMs;
    out[2] = (double)hh->h.lastCollideLaunches;
    out[3] = (double)hh->h.launches;
    return LBIB_OK;
}

int lbib_set_profiling(lbib_handle* hh, int on) {
    if (!hh) return LBIB_ERR_STATE;
    hh->h.profiling = on != 0;
    return LBIB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Differentiated runs.

extern "C" {

int lbib_get_domain_count(lbib_handle* hh, int* n) {
    API_BEGIN(hh)
    if (!n) lbib::fail(LBIB_ERR_INPUT, "lbib_get_domain_count: NULL output");
    *n = h.nDomains;
    API_END
}

int lbib_diff_begin(lbib_handle* hh, int T, int K) {
    API_BEGIN(hh)
    if (h.cross.nfTab != nullptr)
        lbib::fail(LBIB_ERR_STATE, "differentiated runs do not cover boundary solvers on connections");
    if (h.massNode != nullptr) lbib::fail(LBIB_ERR_STATE, "differentiated runs do not cover per-node mass sources");
    if (h.forceModel != lbib::FM_LUO) lbib::fail(LBIB_ERR_STATE, "differentiated runs cover the Luo force model only");
    if (h.cross.bounceW != nullptr) lbib::fail(LBIB_ERR_STATE, "differentiated runs do not cover DiracD2Q5");
    for (int k = 0; k < h.S; ++k)
        if (lbib::coupled_kind(h.sp[k].c.kind))
            lbib::fail(LBIB_ERR_STATE, "differentiated runs do not cover the coupled reaction of " + h.sp[k].name);
    if (T < 1) lbib::fail(LBIB_ERR_INPUT, "differentiated run: T must be at least 1");
    if (K <= 0) K = (int)std::ceil(std::sqrt((double)T));
    if (K > T) K = T;
    lbib::diff_begin(h, T, K);
    API_END
}

int lbib_diff_forward(lbib_handle* hh, const double* memForce, const double* tau, const double* rates, int outlet) {
    API_BEGIN(hh)
    if (!h.diff) lbib::fail(LBIB_ERR_STATE, "lbib_diff_forward before lbib_diff_begin");
    lbib::DiffCtx& d = *h.diff;
    if (tau) {
        for (int k = 0; k <= h.S; ++k)
            if (!(tau[k] > 0.5)) lbib::fail(LBIB_ERR_INPUT, "relaxation times must exceed 0.5", k);
        d.tauF = tau[0];
        for (int k = 0; k < h.S; ++k) d.tau[k] = tau[1 + k];
    }
    if (rates && h.S)
        CK(cudaMemcpyAsync(d.srcTab, rates, sizeof(double) * h.S * h.nDomains, cudaMemcpyHostToDevice, h.stream));
    const int M = h.m.M;
    if (memForce && M) {
        std::vector<double> fx(M), fy(M);
        for (int i = 0; i < M; ++i) { fx[i] = memForce[2 * i]; fy[i] = memForce[2 * i + 1]; }
        CK(cudaMemcpyAsync(d.fxp, fx.data(), sizeof(double) * M, cudaMemcpyHostToDevice, h.stream));
        CK(cudaMemcpyAsync(d.fyp, fy.data(), sizeof(double) * M, cudaMemcpyHostToDevice, h.stream));
        CK(cudaStreamSynchronize(h.stream));
    }
    d.outlet = outlet ? 1 : 0;
    d.backwardDone = false;
    CK(cudaEventRecord(h.evA, h.stream));
    lbib::diff_forward(h, d);
    CK(cudaEventRecord(h.evB, h.stream));
    CK(cudaEventSynchronize(h.evB));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h.evA, h.evB));
    h.lastTotalMs = ms;
    API_END
}

int lbib_diff_backward(lbib_handle* hh, const double* dLdC, double* gForce, double* gTau, double* gRates) {
    API_BEGIN(hh)
    if (!h.diff || !h.diff->forwardDone) lbib::fail(LBIB_ERR_STATE, "lbib_diff_backward before lbib_diff_forward");
    if (!dLdC && h.S) lbib::fail(LBIB_ERR_INPUT, "lbib_diff_backward: dLdC is NULL");
    lbib::DiffCtx& d = *h.diff;
    const size_t L = h.L;
    if (h.S) CK(cudaMemcpyAsync(d.seed, dLdC, sizeof(double) * h.S * L, cudaMemcpyHostToDevice, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    CK(cudaEventRecord(h.evA, h.stream));
    lbib::diff_backward(h, d);
    CK(cudaEventRecord(h.evB, h.stream));
    CK(cudaEventSynchronize(h.evB));
    d.backwardDone = true;
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h.evA, h.evB));
    h.lastTotalMs = ms;
    const size_t nG = 1 + h.S + (size_t)(h.S + 1) * h.nDomains;
    std::vector<double> grad(nG);
    CK(cudaMemcpy(grad.data(), d.grad, sizeof(double) * nG, cudaMemcpyDeviceToHost));
    d.gmass.assign(grad.begin() + 1 + h.S + (size_t)h.S * h.nDomains, grad.end());
    if (gTau) {
        gTau[0] = -grad[0] / (d.tauF * d.tauF);
        for (int k = 0; k < h.S; ++k) gTau[1 + k] = -grad[1 + k] / (d.tau[k] * d.tau[k]);
    }
    if (gRates)
        for (size_t i = 0; i < (size_t)h.S * h.nDomains; ++i) gRates[i] = grad[1 + h.S + i];
    const int M = h.m.M;
    if (gForce && M) {
        std::vector<double> gx(M), gy(M);
        CK(cudaMemcpy(gx.data(), d.gfx, sizeof(double) * M, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(gy.data(), d.gfy, sizeof(double) * M, cudaMemcpyDeviceToHost));
        for (int i = 0; i < M; ++i) { gForce[2 * i] = gx[i]; gForce[2 * i + 1] = gy[i]; }
    }
    API_END
}

int lbib_diff_force_params(lbib_handle* hh, double* gPar, int cap) {
    if (!hh) return -LBIB_ERR_STATE;
    Handle& h = hh->h;
    if (h.err) return -h.err;
    try {
        CK(cudaSetDevice(h.device));
        if (!h.diff || !h.diff->backwardDone)
            lbib::fail(LBIB_ERR_STATE, "lbib_diff_force_params before lbib_diff_backward");
        if (h.diff->motion)
            lbib::fail(LBIB_ERR_STATE, "lbib_diff_force_params: the records' positions move in this run");
        if (cap < 0 || (cap > 0 && !gPar)) lbib::fail(LBIB_ERR_INPUT, "lbib_diff_force_params: bad output buffer");
        lbib::pull_topology(h);
        const int M = h.m.M;
        int nrec = 0;
        if (M) CK(cudaMemcpy(&nrec, h.m.foff + M, sizeof(int), cudaMemcpyDeviceToHost));
        const int n = std::min(nrec, cap);
        if (n > 0) {
            double* g = nullptr;
            CK(cudaMallocAsync((void**)&g, sizeof(double) * 4 * (size_t)nrec, h.stream));
            lbib::launch_force_param_grad(h.m, h.diff->gfx, h.diff->gfy, g, h.stream);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(gPar, g, sizeof(double) * 4 * (size_t)n, cudaMemcpyDeviceToHost, h.stream));
            CK(cudaFreeAsync(g, h.stream));
            CK(cudaStreamSynchronize(h.stream));
        }
        return nrec;
    } catch (const HostFail& e) {
        h.err = e.code; h.msg = e.msg; h.errIndex = e.index;
        return -e.code;
    } catch (const std::exception& e) {
        h.err = LBIB_ERR_INPUT; h.msg = e.what();
        return -h.err;
    }
}

int lbib_download_forces(lbib_handle* hh, int* type, unsigned* id1, unsigned* id2, double* par, int cap) {
    if (!hh) return -LBIB_ERR_STATE;
    Handle& h = hh->h;
    if (h.err) return -h.err;
    try {
        CK(cudaSetDevice(h.device));
        if (cap < 0 || (cap > 0 && (!type || !id1 || !id2 || !par)))
            lbib::fail(LBIB_ERR_INPUT, "lbib_download_forces: bad output buffers");
        lbib::pull_topology(h);
        const int M = h.m.M;
        std::vector<int> foff(M + 1, 0);
        if (M) CK(cudaMemcpy(foff.data(), h.m.foff, sizeof(int) * (M + 1), cudaMemcpyDeviceToHost));
        const int nrec = foff[M];
        const int n = std::min(nrec, cap);
        if (n > 0) {
            std::vector<int> part(n);
            CK(cudaMemcpy(type, h.m.ftype, sizeof(int) * n, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(part.data(), h.m.fpartner, sizeof(int) * n, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(par, h.m.fpar, sizeof(double) * 4 * (size_t)n, cudaMemcpyDeviceToHost));
            for (int i = 0, r = 0; i < M && r < n; ++i)
                for (; r < foff[i + 1] && r < n; ++r) {
                    id1[r] = h.ids[i];
                    id2[r] = part[r] >= 0 && part[r] < M ? h.ids[part[r]] : 0u;
                }
        }
        return nrec;
    } catch (const HostFail& e) {
        h.err = e.code; h.msg = e.msg; h.errIndex = e.index;
        return -e.code;
    } catch (const std::exception& e) {
        h.err = LBIB_ERR_INPUT; h.msg = e.what();
        return -h.err;
    }
}

int lbib_diff_mass(lbib_handle* hh, const double* mass, double* gMass, int n) {
    API_BEGIN(hh)
    if (!h.diff) lbib::fail(LBIB_ERR_STATE, "lbib_diff_mass outside a differentiated run");
    if (n != h.nDomains) lbib::fail(LBIB_ERR_INPUT, "lbib_diff_mass: n must be the domain count");
    lbib::DiffCtx& d = *h.diff;
    if (mass) {
        CK(cudaMemcpyAsync(d.massTab, mass, sizeof(double) * n, cudaMemcpyHostToDevice, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        d.massUsed = true;
        d.forwardDone = false;
        d.backwardDone = false;
    }
    if (gMass)
        for (int i = 0; i < n; ++i) gMass[i] = d.massUsed && i < (int)d.gmass.size() ? d.gmass[i] : 0.0;
    API_END
}

int lbib_diff_fluid_seed(lbib_handle* hh, const double* dLdf) {
    API_BEGIN(hh)
    if (!h.diff) lbib::fail(LBIB_ERR_STATE, "lbib_diff_fluid_seed outside a differentiated run");
    lbib::DiffCtx& d = *h.diff;
    d.haveSeedF = dLdf != nullptr;
    if (dLdf) {
        // lbib_download_lattice's slot layout [L][9] to the device's direction planes
        static const int INV9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
        const size_t L = h.L;
        std::vector<double> nat(9 * L);
        for (size_t n = 0; n < L; ++n)
            for (int q = 0; q < 9; ++q) nat[(size_t)q * L + n] = dLdf[n * 9 + INV9[q]];
        CK(cudaMemcpyAsync(d.seedF, nat.data(), sizeof(double) * 9 * L, cudaMemcpyHostToDevice, h.stream));
        CK(cudaStreamSynchronize(h.stream));
    }
    API_END
}

int lbib_diff_motion(lbib_handle* hh, int on, const double* dLdX) {
    API_BEGIN(hh)
    if (!h.diff) lbib::fail(LBIB_ERR_STATE, "lbib_diff_motion before lbib_diff_begin");
    lbib::DiffCtx& d = *h.diff;
    if (on && h.m.M == 0) lbib::fail(LBIB_ERR_STATE, "lbib_diff_motion: the geometry has no membrane nodes");
    lbib::diff_set_motion(h, d, on != 0);
    d.haveSeedX = false;
    if (on && dLdX) {
        const int M = d.M;
        std::vector<double> v(2 * (size_t)M);
        for (int i = 0; i < M; ++i) { v[i] = dLdX[2 * i]; v[M + i] = dLdX[2 * i + 1]; }
        CK(cudaMemcpyAsync(d.seedX, v.data(), sizeof(double) * 2 * M, cudaMemcpyHostToDevice, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        d.haveSeedX = true;
    }
    API_END
}

int lbib_diff_positions(lbib_handle* hh, double* xT, double* gX0, int n) {
    API_BEGIN(hh)
    if (!h.diff || !h.diff->motion) lbib::fail(LBIB_ERR_STATE, "lbib_diff_positions outside a moving-node run");
    lbib::DiffCtx& d = *h.diff;
    if (n != d.M) lbib::fail(LBIB_ERR_INPUT, "lbib_diff_positions: n must be the membrane's node count");
    if (xT && !d.forwardDone) lbib::fail(LBIB_ERR_STATE, "lbib_diff_positions: no forward pass yet");
    if (gX0 && !d.backwardDone) lbib::fail(LBIB_ERR_STATE, "lbib_diff_positions: no reverse pass yet");
    std::vector<double> v(2 * (size_t)n);
    auto put = [&](const double* dev, double* out) {
        CK(cudaMemcpy(v.data(), dev, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i) { out[2 * i] = v[i]; out[2 * i + 1] = v[n + i]; }
    };
    if (n && xT) put(d.posAt(d.T), xT);
    if (n && gX0) put(d.lam, gX0);
    API_END
}

int lbib_diff_end(lbib_handle* hh) {
    API_BEGIN(hh)
    if (h.diff) {
        lbib::DiffCtx& d = *h.diff;
        const size_t L = h.L;
        const size_t rs = d.rs;
        CK(cudaMemcpyAsync(h.f[h.cur], d.x0, 9 * L * rs, cudaMemcpyDeviceToDevice, h.stream));
        if (h.S)
            CK(cudaMemcpyAsync(h.g[h.cur], d.x0 + 9 * L * rs, 5 * h.S * L * rs, cudaMemcpyDeviceToDevice, h.stream));
        CK(cudaMemcpyAsync(h.u, d.u0, 2 * L * rs, cudaMemcpyDeviceToDevice, h.stream));
        CK(cudaMemcpyAsync(h.force, d.u0 + 2 * L * rs, 2 * L * rs, cudaMemcpyDeviceToDevice, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        delete h.diff;
        h.diff = nullptr;
    }
    API_END
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Checkpoint files in the reference's formats.

namespace {

std::string g17(double v) {
    char b[40];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

}  // namespace

extern "C" {

int lbib_write_simulation(lbib_handle* hh, const char* forceFile, const char* geometryFile, const char* parameterFile,
                          const char* solverFile) {
    API_BEGIN(hh)
    lbib::pull_topology(h);
    const int M = (int)h.ids.size();
    const size_t L = h.L;
    if (geometryFile && *geometryFile) {
        // Geometry::writeGeometry (Geometry.cpp:77-95), nodes in id order
        std::vector<double> x(M), y(M);
        if (M) {
            CK(cudaMemcpyAsync(x.data(), h.m.x, sizeof(double) * M, cudaMemcpyDeviceToHost, h.stream));
            CK(cudaMemcpyAsync(y.data(), h.m.y, sizeof(double) * M, cudaMemcpyDeviceToHost, h.stream));
        }
        CK(cudaStreamSynchronize(h.stream));
        std::ofstream o(geometryFile);
        if (!o.is_open()) lbib::fail(LBIB_ERR_INPUT, std::string("cannot open ") + geometryFile);
        o << "#Nodes (id\txPos\tyPos)\n";
        for (int i = 0; i < M; ++i) o << h.ids[i] << '\t' << g17(x[i]) << '\t' << g17(y[i]) << '\n';
        o << "#Connection (nodeId1\tnodeId2\tdomainId\tbsolver\tcdesolver\t...)\n";
        for (const auto& c : h.conns) o << c.id1 << '\t' << c.id2 << '\t' << c.dom << c.desc << '\n';
    }
    if (forceFile && *forceFile) {
        // ForceSolver::writeForceSolver (ForceSolver.cpp:141-156): per node in id
        // order, its forces in insertion order, each as ForceStructs.hpp writes it
        std::vector<int> foff(M + 1, 0);
        if (M) CK(cudaMemcpyAsync(foff.data(), h.m.foff, sizeof(int) * (M + 1), cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        const int nrec = foff[M];
        std::vector<int> ftype(nrec), fpart(nrec);
        std::vector<double> fpar(4 * (size_t)nrec);
        if (nrec) {
            CK(cudaMemcpyAsync(ftype.data(), h.m.ftype, sizeof(int) * nrec, cudaMemcpyDeviceToHost, h.stream));
            CK(cudaMemcpyAsync(fpart.data(), h.m.fpartner, sizeof(int) * nrec, cudaMemcpyDeviceToHost, h.stream));
            CK(cudaMemcpyAsync(fpar.data(), h.m.fpar, sizeof(double) * 4 * nrec, cudaMemcpyDeviceToHost, h.stream));
            CK(cudaStreamSynchronize(h.stream));
        }
        std::ofstream o(forceFile);
        if (!o.is_open()) lbib::fail(LBIB_ERR_INPUT, std::string("cannot open ") + forceFile);
        for (int i = 0; i < M; ++i)
            for (int r = foff[i]; r < foff[i + 1]; ++r) {
                const int t = ftype[r];
                const double* p = &fpar[4 * (size_t)r];
                const unsigned partner = fpart[r] >= 0 && fpart[r] < M ? h.ids[fpart[r]] : 0u;
                o << t << '\t' << h.ids[i];
                switch (t) {
                    case 0: case 7: o << '\t' << partner << '\t' << g17(p[0]) << '\t' << g17(p[1]); break;
                    case 1: o << '\t' << g17(p[0]) << '\t' << g17(p[1]) << '\t' << g17(p[2]) << '\t' << g17(p[3]); break;
                    case 2: o << '\t' << g17(p[0]) << '\t' << g17(p[1]); break;
                    case 3: case 4: o << '\t' << g17(p[0]) << '\t' << g17(p[1]) << '\t' << g17(p[2]); break;
                    default: o << '\t' << partner << '\t' << g17(p[0]); break;  // 5, 6
                }
                o << '\n';
            }
    }
    if (parameterFile && *parameterFile) {
        // GlobalSimulationParameters::writeGlobalSimulationParameters (GlobalSimulationParameters.cpp:74-97)
        std::ofstream o(parameterFile);
        if (!o.is_open()) lbib::fail(LBIB_ERR_INPUT, std::string("cannot open ") + parameterFile);
        o << "#Global Parameter file\n";
        o << "CurrentIterations:\t" << h.iteration << "\n";
        o << "Iterations:\t" << h.iterations << "\n";
        o << "ReportStep:\t" << h.reportStep << "\n";
        o << "SizeX:\t" << h.nx << "\n";
        o << "SizeY:\t" << h.ny << "\n";
        o << "tauFluid:\t" << g17(h.tauF) << "\n";
        o << "CDESolvers:";
        for (const auto& sp : h.sp) o << '\t' << sp.name << '\t' << g17(sp.c.tau);
        o << "\n";
    }
    if (solverFile && *solverFile) {
        // SimulationRunner::writeSimulation's solver dump (SimulationRunner.cpp:121-145):
        // rows y, then x; distributions in the stored (post-swap) slot order
        std::vector<double> f(9 * L), g(5 * (size_t)h.S * L);
        const int rc = lbib_download_lattice(hh, f.data(), h.S ? g.data() : nullptr, nullptr, nullptr, nullptr, nullptr);
        if (rc) return rc;
        std::ofstream o(solverFile);
        if (!o.is_open()) lbib::fail(LBIB_ERR_INPUT, std::string("cannot open ") + solverFile);
        o << "#Solvers (xPos\tyPos\tDistributions...)\n";
        o << "#BEGIN FluidSolver\n";
        for (int y = 0; y < h.ny; ++y)
            for (int x = 0; x < h.nx; ++x) {
                const size_t n = (size_t)y * h.nx + x;
                o << x << '\t' << y;
                for (int q = 0; q < 9; ++q) o << '\t' << g17(f[9 * n + q]);
                o << '\n';
            }
        o << "#END FluidSolver\n";
        for (int k = 0; k < h.S; ++k) {
            o << "#BEGIN " << h.sp[k].name << "\n";
            for (int y = 0; y < h.ny; ++y)
                for (int x = 0; x < h.nx; ++x) {
                    const size_t n = (size_t)y * h.nx + x;
                    o << x << '\t' << y;
                    for (int q = 0; q < 5; ++q) o << '\t' << g17(g[((size_t)k * L + n) * 5 + q]);
                    o << '\n';
                }
            o << "#END " << h.sp[k].name << "\n";
        }
    }
    API_END
}

int lbib_load_solvers(lbib_handle* hh, const char* solverFile) {
    API_BEGIN(hh)
    // SimulationRunner::initSolvers(file) (SimulationRunner.cpp:151-182): nodes
    // listed in the file take its distributions, the others keep theirs
    std::ifstream in(solverFile ? solverFile : "");
    if (!in.is_open()) lbib::fail(LBIB_ERR_INPUT, "Cannot find the solver file.");
    const size_t L = h.L;
    std::vector<double> f(9 * L), g(5 * (size_t)h.S * L);
    int rc = lbib_download_lattice(hh, f.data(), h.S ? g.data() : nullptr, nullptr, nullptr, nullptr, nullptr);
    if (rc) return rc;
    std::string line, solver;
    int k = -1;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        std::stringstream ls(line);
        if (line[0] == '#') {
            std::string tag;
            if (line.find("#BEGIN") != std::string::npos) {
                ls >> tag >> solver;
                k = -1;
                if (solver != "FluidSolver") {
                    for (int j = 0; j < h.S; ++j)
                        if (h.sp[j].name == solver) k = j;
                    if (k < 0) lbib::fail(LBIB_ERR_INPUT, "unknown CDE solver in the solver file: " + solver);
                }
            } else if (line.find("#END") != std::string::npos) {
                solver.clear();
            }
            continue;
        }
        int x, y;
        ls >> x >> y;
        if (!ls || x < 0 || y < 0 || x >= h.nx || y >= h.ny) lbib::fail(LBIB_ERR_INPUT, "bad node in the solver file: " + line);
        const size_t n = (size_t)y * h.nx + x;
        if (solver == "FluidSolver") {
            for (int q = 0; q < 9; ++q) ls >> f[9 * n + q];
        } else if (k >= 0) {
            for (int q = 0; q < 5; ++q) ls >> g[((size_t)k * L + n) * 5 + q];
        } else {
            lbib::fail(LBIB_ERR_INPUT, "solver file line outside a #BEGIN/#END block: " + line);
        }
        if (!ls) lbib::fail(LBIB_ERR_INPUT, "bad distributions in the solver file: " + line);
    }
    rc = lbib_upload_lattice(hh, f.data(), h.S ? g.data() : nullptr, nullptr);
    if (rc) return rc;
    API_END
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The force list and the node range queries for host plugins: the calls a
// bio solver makes on ForceSolver (addForce, deleteForceType, deleteAllForces;
// ForceSolver.cpp:107-139,170-215) and Geometry
// (getGeometryNodesWithinRadius[WithAvoidance][Closest], Geometry.cpp:306-374)
// between steps, in bulk.

namespace lbib {

// Runs one edit of the force list now (between steps) and checks its status.
static void run_force_edit(Handle& h, int delType, int gen) {
    ensure_force_scratch(h, true);
    reset_status(h, h.iteration, h.cellTypesCopied);
    launch_force_edit(h.m, h.fs, delType, gen, 0.0, 0.0, 0.0, h.st, h.stream);
    CK(cudaGetLastError());
    read_status(h);
    if (h.stHost->err) fail(h.stHost->err, "force list edit failed", h.stHost->errIndex);
}

// Makes room for `extra` more records, keeping the list.
static void reserve_force_records(Handle& h, int extra) {
    const int M = h.m.M;
    int R = 0;
    CK(cudaMemcpyAsync(&R, h.m.foff + M, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    if (R + extra <= h.Fcap) return;
    std::vector<int> ftype(R), fpart(R);
    std::vector<double> fpar(4 * (size_t)R);
    if (R) {
        CK(cudaMemcpyAsync(ftype.data(), h.m.ftype, sizeof(int) * R, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaMemcpyAsync(fpart.data(), h.m.fpartner, sizeof(int) * R, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaMemcpyAsync(fpar.data(), h.m.fpar, sizeof(double) * fpar.size(), cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
    }
    ensure_capacity(h, h.m.M, h.m.C, R + extra + 2 * h.Mcap, h.m.nCells);
    if (R) {
        CK(cudaMemcpyAsync(h.m.ftype, ftype.data(), sizeof(int) * R, cudaMemcpyHostToDevice, h.stream));
        CK(cudaMemcpyAsync(h.m.fpartner, fpart.data(), sizeof(int) * R, cudaMemcpyHostToDevice, h.stream));
        CK(cudaMemcpyAsync(h.m.fpar, fpar.data(), sizeof(double) * fpar.size(), cudaMemcpyHostToDevice, h.stream));
    }
}

// Index of node `id` in the id-ordered node arrays, -1 if absent.
static int node_index(const Handle& h, uint32_t id) {
    auto it = std::lower_bound(h.ids.begin(), h.ids.end(), id);
    return it != h.ids.end() && *it == id ? (int)(it - h.ids.begin()) : -1;
}

// The list as it stands between steps, set by a host call: later steps treat
// it like a list loaded at this iteration.
static void set_list_state(Handle& h, bool pure) {
    h.forcesPureAtLoad = pure;
    h.forceListIt = h.iteration;
    h.forcemap.clear();
}

template <typename T>
static T* upload(Handle& h, const std::vector<T>& v) {
    T* d = dalloc<T>(std::max<size_t>(v.size(), 1));
    if (!v.empty()) CK(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, h.stream));
    return d;
}

}  // namespace lbib

extern "C" {

int lbib_add_forces(lbib_handle* hh, const int* type, const unsigned* id1, const unsigned* id2, const double* par,
                    int n) {
    if (n < 0 || (n > 0 && (!type || !id1 || !par))) return LBIB_ERR_INPUT;
    API_BEGIN(hh)
    if (n == 0) return LBIB_OK;
    lbib::pull_topology(h);
    std::vector<int> node(n), partner(n, -1);
    for (int k = 0; k < n; ++k) {
        const int t = type[k];
        if (t < 0 || t > 7) lbib::fail(LBIB_ERR_INPUT, "Invalid force solver type found.", k);
        node[k] = lbib::node_index(h, id1[k]);
        if (node[k] < 0) lbib::fail(LBIB_ERR_FORCE_NODE, "Could not compute and set the forces.", (long long)id1[k]);
        if (t == 0 || t == 5 || t == 6 || t == 7) {
            if (!id2) lbib::fail(LBIB_ERR_INPUT, "forces of types 0, 5, 6, 7 need a second node", k);
            partner[k] = lbib::node_index(h, id2[k]);
            if (partner[k] < 0)
                lbib::fail(LBIB_ERR_FORCE_NODE, "Could not compute and set the forces.", (long long)id2[k]);
        }
    }
    // per node, in call order (ForceSolver::addForce appends to forcemap_[id1])
    std::vector<int> off(h.Mcap + 1, 0);
    for (int k = 0; k < n; ++k) off[node[k] + 1]++;
    for (int i = 0; i < h.Mcap; ++i) off[i + 1] += off[i];
    std::vector<int> fill(off.begin(), off.end() - 1), ltype(n), lpart(n);
    std::vector<double> lpar(4 * (size_t)n);
    for (int k = 0; k < n; ++k) {
        const int r = fill[node[k]]++;
        ltype[r] = type[k];
        lpart[r] = partner[k];
        for (int q = 0; q < 4; ++q) lpar[4 * (size_t)r + q] = par[4 * (size_t)k + q];
    }
    lbib::reserve_force_records(h, n);
    lbib::ensure_force_scratch(h, true);
    h.fs.listOff = lbib::upload(h, off);
    h.fs.listType = lbib::upload(h, ltype);
    h.fs.listPartner = lbib::upload(h, lpart);
    h.fs.listPar = lbib::upload(h, lpar);
    struct Free {
        lbib::ForceScratch& fs;
        ~Free() {
            cudaFree(fs.listOff); cudaFree(fs.listType); cudaFree(fs.listPartner); cudaFree(fs.listPar);
            fs.listOff = fs.listType = fs.listPartner = nullptr;
            fs.listPar = nullptr;
        }
    } freeList{h.fs};
    lbib::run_force_edit(h, -1, lbib::GEN_LIST);
    lbib::set_list_state(h, false);
    API_END
}

int lbib_delete_force_type(lbib_handle* hh, int type) {
    API_BEGIN(hh)
    const bool pure = lbib::pure_at_start(h, h.iteration);
    lbib::run_force_edit(h, type, lbib::GEN_NONE);
    lbib::set_list_state(h, pure);
    API_END
}

int lbib_delete_all_forces(lbib_handle* hh) {
    API_BEGIN(hh)
    lbib::launch_clear_forces(h.m, h.stream);
    CK(cudaStreamSynchronize(h.stream));
    lbib::set_list_state(h, true);
    API_END
}

int lbib_nodes_within_radius(lbib_handle* hh, double x, double y, double radius, long long avoidDomain,
                             unsigned* ids, int cap) {
    if (!hh) return -LBIB_ERR_STATE;
    if (cap < 0 || (cap > 0 && !ids) || !(radius >= 0.0)) return -LBIB_ERR_INPUT;
    Handle& h = hh->h;
    if (h.err) return -h.err;
    try {
        cudaSetDevice(h.device);
        lbib::ensure_force_scratch(h, true);
        lbib::launch_cell_list(h.m, h.fs, h.nx, h.ny, h.stream);
        const std::vector<double> q = {x, y};
        const std::vector<long long> av = {avoidDomain};
        double* dq = lbib::upload(h, q);
        long long* dav = lbib::upload(h, av);
        unsigned* dids = lbib::dalloc<unsigned>(std::max(cap, 1));
        int* dcount = lbib::dalloc<int>(1);
        lbib::launch_range_query(h.m, h.fs, h.nx, h.ny, dq, dq + 1, dav, 1, radius, 0, dids, cap, dcount, nullptr,
                                 h.stream);
        int count = 0;
        CK(cudaMemcpyAsync(&count, dcount, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
        if (cap > 0) CK(cudaMemcpyAsync(ids, dids, sizeof(unsigned) * cap, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        cudaFree(dq); cudaFree(dav); cudaFree(dids); cudaFree(dcount);
        return count;
    } catch (const HostFail& e) {
        h.err = e.code; h.msg = e.msg;
        return -e.code;
    }
}

int lbib_closest_nodes(lbib_handle* hh, const double* x, const double* y, const long long* avoidDomain, int n,
                       double radius, long long* closest) {
    if (n < 0 || (n > 0 && (!x || !y || !closest)) || !(radius >= 0.0)) return LBIB_ERR_INPUT;
    API_BEGIN(hh)
    if (n == 0) return LBIB_OK;
    lbib::ensure_force_scratch(h, true);
    lbib::launch_cell_list(h.m, h.fs, h.nx, h.ny, h.stream);
    double* dx = lbib::upload(h, std::vector<double>(x, x + n));
    double* dy = lbib::upload(h, std::vector<double>(y, y + n));
    long long* dav = avoidDomain ? lbib::upload(h, std::vector<long long>(avoidDomain, avoidDomain + n)) : nullptr;
    long long* dout = lbib::dalloc<long long>(n);
    lbib::launch_range_query(h.m, h.fs, h.nx, h.ny, dx, dy, dav, n, radius, 1, nullptr, 0, nullptr, dout, h.stream);
    CK(cudaMemcpyAsync(closest, dout, sizeof(long long) * n, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    cudaFree(dx); cudaFree(dy); if (dav) cudaFree(dav); cudaFree(dout);
    API_END
}

}  // extern "C"

// ---------------------------------------------------------------------------
// VTK reporters without VTK (vtkCellReporter, vtkForceReporter,
// vtkCDEReporter, vtkFluidReporter): each call appends the functor's block to
// <prefix>_<time>.vtm.

namespace lbib {

// The reporter's boundary descriptor string: "\t", then "<bsolver>\t<cde>\t"
// for every pair of the connection's descriptor map (vtkCellReporter.cpp).
static std::string reporter_descriptor(const std::string& desc) {
    std::stringstream ls(desc);
    std::map<std::string, std::vector<std::string>> type;
    std::string a, b;
    while (ls >> a >> b) type[a].push_back(b);
    std::string out = "\t";
    for (const auto& kv : type)
        for (const auto& c : kv.second) out += kv.first + "\t" + c + "\t";
    return out;
}

static void vtk_cells(lbib_handle* hh, Handle& h, const std::string& vtm) {
    pull_topology(h);
    std::vector<unsigned> ids(h.m.M);
    std::vector<double> st(6 * (size_t)h.m.M);
    if (int rc = lbib_download_membrane(hh, ids.data(), st.data())) fail(rc, "membrane download failed");
    std::map<uint32_t, int> index;
    for (int i = 0; i < h.m.M; ++i) index[ids[i]] = i;
    std::map<uint32_t, int> outConn;  // node id -> its connection<1> (outgoing)
    std::map<uint32_t, std::vector<int>> cells;  // domain -> connections in vector order
    for (size_t c = 0; c < h.conns.size(); ++c) {
        outConn[h.conns[c].id1] = (int)c;
        cells[h.conns[c].dom].push_back((int)c);
    }
    vtk::PolyData pd;
    vtk::Array domA{"domain_identifier", 1, "Float64", {}}, typeA{"cell_type", 1, "Float64", {}};
    std::vector<std::string> descs;
    for (const auto& kv : cells) {
        const int start = kv.second[0];
        int c = start;
        do {
            const int n = index.at(h.conns[c].id2);
            pd.px.push_back(st[6 * (size_t)n]);
            pd.py.push_back(st[6 * (size_t)n + 1]);
            pd.connectivity.push_back((int64_t)pd.connectivity.size());
            domA.values.push_back((double)h.conns[c].dom);
            const uint32_t d = h.conns[c].dom;
            if (d >= h.ctypeHost.size()) fail(ERR_STATE, "domainIdentifier not found in the cellTrackerMap.");
            typeA.values.push_back((double)h.ctypeHost[d]);
            descs.push_back(reporter_descriptor(h.conns[c].desc));
            c = outConn.at(h.conns[c].id2);
        } while (c != start);
        pd.offsets.push_back((int64_t)pd.connectivity.size());
    }
    pd.pointData = {domA, typeA};
    pd.pointStrings.push_back({"boundarydescriptors", descs});
    vtk::append_block(vtm, pd);
}

static void vtk_forces(lbib_handle* hh, Handle& h, const std::string& vtm) {
    pull_topology(h);
    const int M = h.m.M;
    std::vector<unsigned> ids(M);
    std::vector<double> st(6 * (size_t)M);
    if (int rc = lbib_download_membrane(hh, ids.data(), st.data())) fail(rc, "membrane download failed");
    std::vector<int> foff(M + 1);
    CK(cudaMemcpyAsync(foff.data(), h.m.foff, sizeof(int) * (M + 1), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    const int R = foff[M];
    std::vector<int> ftype(R), fpart(R);
    if (R) {
        CK(cudaMemcpyAsync(ftype.data(), h.m.ftype, sizeof(int) * R, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaMemcpyAsync(fpart.data(), h.m.fpartner, sizeof(int) * R, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
    }
    vtk::PolyData pd;
    pd.lines = true;
    vtk::Array typeA{"ForceType", 1, "UInt32", {}};
    for (int i = 0; i < M; ++i)
        for (int r = foff[i]; r < foff[i + 1]; ++r) {
            const int t = ftype[r];
            const bool paired = t == 0 || t == 5 || t == 6 || t == 7;
            // getPartnerGeometryNode() != 0: forces without a partner report 0,
            // and so does a partner whose id is 0 (vtkForceReporter.cpp)
            const uint32_t pid = paired && fpart[r] >= 0 && fpart[r] < M ? ids[fpart[r]] : 0u;
            if (pid == 0) continue;
            pd.px.push_back(st[6 * (size_t)i]);
            pd.py.push_back(st[6 * (size_t)i + 1]);
            pd.px.push_back(st[6 * (size_t)fpart[r]]);
            pd.py.push_back(st[6 * (size_t)fpart[r] + 1]);
            pd.connectivity.push_back((int64_t)pd.px.size() - 2);
            pd.connectivity.push_back((int64_t)pd.px.size() - 1);
            pd.offsets.push_back((int64_t)pd.connectivity.size());
            typeA.values.push_back((double)t);
        }
    pd.cellData = {typeA};
    vtk::append_block(vtm, pd);
}

// vtkCDEReporter / vtkFluidReporter: a uniform grid of nx/f x ny/f points,
// spacing f, filled by rows y = 0, f, 2f, .. and columns x = 0, f, .. (the
// functors' loops; when f does not divide the lattice they produce more values
// than the grid's points, and so does this writer).
static void vtk_grid(lbib_handle* hh, Handle& h, const std::string& vtm, int f, bool fluid) {
    const size_t L = h.L;
    std::vector<double> fd, g, vel;
    if (fluid) {
        fd.resize(9 * L);
        vel.resize(2 * L);
    } else {
        g.resize((size_t)std::max(1, h.S) * 5 * L);
    }
    if (int rc = lbib_download_lattice(hh, fluid ? fd.data() : nullptr, fluid ? nullptr : g.data(),
                                       fluid ? vel.data() : nullptr, nullptr, nullptr, nullptr))
        fail(rc, "lattice download failed");
    vtk::ImageData im;
    im.X = h.nx / f;
    im.Y = h.ny / f;
    im.spacing = f;
    if (fluid) {
        vtk::Array rho{"density", 1, "Float64", {}}, u{"velocity", 3, "Float64", {}};
        for (int y = 0; y < h.ny; y += f)
            for (int x = 0; x < h.nx; x += f) {
                const size_t n = (size_t)y * h.nx + x;
                double r = 0.0;  // FluidSolver::getRho: accumulate over the slots
                for (int q = 0; q < 9; ++q) r += fd[9 * n + q];
                rho.values.push_back(r);
                u.values.push_back(vel[2 * n]);
                u.values.push_back(vel[2 * n + 1]);
                u.values.push_back(0.0);
            }
        im.pointData = {rho, u};
    } else {
        std::map<std::string, int> byName;  // the functor's map: arrays in name order
        for (int k = 0; k < h.S; ++k) byName[h.sp[k].name] = k;
        for (const auto& kv : byName) {
            vtk::Array c{kv.first, 1, "Float64", {}};
            for (int y = 0; y < h.ny; y += f)
                for (int x = 0; x < h.nx; x += f) {
                    const size_t n = (size_t)y * h.nx + x;
                    double sum = 0.0;  // CDESolverD2Q5::getC
                    for (int q = 0; q < 5; ++q) sum += g[((size_t)kv.second * L + n) * 5 + q];
                    c.values.push_back(sum);
                }
            im.pointData.push_back(c);
        }
    }
    vtk::append_block(vtm, im);
}

}  // namespace lbib

extern "C" {

int lbib_read_vtm_geometry(const char* path, unsigned* ids, double* xy, int capNodes, unsigned* conns,
                           int capConns, int* counts) {
    if (!path || !counts || capNodes < 0 || capConns < 0) return LBIB_ERR_INPUT;
    lbib::vtk::Geometry g;
    try {
        lbib::vtk::read_vtm_geometry(path, g);
    } catch (const std::exception&) {
        return LBIB_ERR_INPUT;
    }
    counts[0] = (int)g.x.size();
    counts[1] = (int)g.conns.size();
    for (int k = 0; k < counts[0] && k < capNodes; ++k) {
        if (ids) ids[k] = (unsigned)k;
        if (xy) { xy[2 * k] = g.x[k]; xy[2 * k + 1] = g.y[k]; }
    }
    for (int c = 0; c < counts[1] && c < capConns; ++c)
        if (conns) {
            conns[3 * c] = g.conns[c].id1;
            conns[3 * c + 1] = g.conns[c].id2;
            conns[3 * c + 2] = g.conns[c].dom;
        }
    return LBIB_OK;
}

int lbib_write_vtk(lbib_handle* hh, const char* prefix, unsigned time, int kind, int coarsening) {
    if (!prefix || kind < LBIB_VTK_CELLS || kind > LBIB_VTK_CELL_PNG || coarsening < 1) return LBIB_ERR_INPUT;
    API_BEGIN(hh)
    const std::string vtm = std::string(prefix) + "_" + std::to_string(time) + ".vtm";
    try {
        switch (kind) {
            case LBIB_VTK_CELLS: lbib::vtk_cells(hh, h, vtm); break;
            case LBIB_VTK_FORCES: lbib::vtk_forces(hh, h, vtm); break;
            case LBIB_VTK_CDE: lbib::vtk_grid(hh, h, vtm, coarsening, false); break;
            case LBIB_VTK_FLUID: lbib::vtk_grid(hh, h, vtm, coarsening, true); break;
            default: break;  // vtkCellPNGReporter renders through a graphics stack: nothing is written
        }
    } catch (const std::runtime_error& e) {
        lbib::fail(LBIB_ERR_INPUT, e.what());
    }
    API_END
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Topology edits by a host bio solver (a cell division, a growth step):
// the Geometry calls addGeometryNode / removeGeometryNode / addConnection /
// eraseConnection (Geometry.cpp:381-452) made between steps, given as the
// resulting node and connection lists.

namespace lbib {

// Widens the per-domain tables to nd domains (new domains: no mass source, no
// species production, cell type 1 as the text geometry loader gives).
static void grow_domains(Handle& h, int nd) {
    if (nd <= h.nDomains) return;
    const int old = h.nDomains;
    double* mt = dalloc<double>(nd);
    CK(cudaMemsetAsync(mt, 0, sizeof(double) * nd, h.stream));
    CK(cudaMemcpyAsync(mt, h.massTab, sizeof(double) * old, cudaMemcpyDeviceToDevice, h.stream));
    const int S = std::max(1, h.S);
    double* st = dalloc<double>((size_t)S * nd);
    CK(cudaMemsetAsync(st, 0, sizeof(double) * S * nd, h.stream));
    for (int k = 0; k < S; ++k)
        CK(cudaMemcpyAsync(st + (size_t)k * nd, h.srcTab + (size_t)k * old, sizeof(double) * old,
                           cudaMemcpyDeviceToDevice, h.stream));
    h.ctypeHost.resize(nd, 1u);
    uint32_t* ct = dalloc<uint32_t>(nd);
    CK(cudaMemcpyAsync(ct, h.ctypeHost.data(), sizeof(uint32_t) * nd, cudaMemcpyHostToDevice, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    cudaFree(h.massTab); cudaFree(h.srcTab); cudaFree(h.ctypeTab);
    h.massTab = mt; h.srcTab = st; h.ctypeTab = ct;
    cudaFree(h.td.cellOfDom); cudaFree(h.td.firstConn);  // re-made for nd by upload_topology
    h.td.cellOfDom = nullptr; h.td.firstConn = nullptr;
    h.nDomains = nd;
    h.graphEpoch++;
}

// The device table of boundary solvers has one entry per descriptor string; a
// string first seen now gets an entry with no solvers.
static void ensure_descriptor(Handle& h, const std::string& desc) {
    if (std::find(h.descTable.begin(), h.descTable.end(), desc) != h.descTable.end()) return;
    h.descTable.push_back(desc);
    if (!h.nfTabDev) return;
    const size_t n = h.descTable.size();
    NfSpec* t = dalloc<NfSpec>(n);
    CK(cudaMemsetAsync(t, 0, sizeof(NfSpec) * n, h.stream));
    CK(cudaMemcpyAsync(t, h.nfTabDev, sizeof(NfSpec) * (n - 1), cudaMemcpyDeviceToDevice, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    cudaFree(h.nfTabDev);
    h.nfTabDev = t;
    h.cross.nfTab = t;
    h.graphEpoch++;
}

}  // namespace lbib

extern "C" {

int lbib_upload_membrane(lbib_handle* hh, const unsigned* ids, const double* xy, int M, const unsigned* conns,
                         int C) {
    if (M < 0 || C < 0 || (M > 0 && (!ids || !xy)) || (C > 0 && !conns)) return LBIB_ERR_INPUT;
    API_BEGIN(hh)
    if (h.diff) lbib::fail(LBIB_ERR_STATE, "topology edits are not possible during a differentiated run");
    for (int k = 1; k < M; ++k)
        if (ids[k] <= ids[k - 1]) lbib::fail(LBIB_ERR_INPUT, "node ids must ascend", k);
    lbib::pull_topology(h);
    lbib::HostMembrane old;
    lbib::download_membrane(h, old);
    lbib::sync_targets(h);
    const lbib::IdIndex oldIdx(h.ids);
    const std::vector<uint32_t> oldIds = h.ids;
    // the force list, remapped by node id; records of removed nodes go
    std::vector<int> foff(h.m.M + 1);
    CK(cudaMemcpyAsync(foff.data(), h.m.foff, sizeof(int) * (h.m.M + 1), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    const int R = foff[h.m.M];
    std::vector<int> ftype(R), fpart(R);
    std::vector<double> fpar(4 * (size_t)R);
    if (R) {
        CK(cudaMemcpyAsync(ftype.data(), h.m.ftype, sizeof(int) * R, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaMemcpyAsync(fpart.data(), h.m.fpartner, sizeof(int) * R, cudaMemcpyDeviceToHost, h.stream));
        CK(cudaMemcpyAsync(fpar.data(), h.m.fpar, sizeof(double) * fpar.size(), cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
    }
    // the new node arrays: kept nodes keep their state, new ones start like a
    // GeometryNode created at (x, y) (perturbed, old position 5 lu away, at rest)
    std::vector<uint32_t> newIds(ids, ids + M);
    lbib::HostMembrane hm;
    for (int k = 0; k < M; ++k) {
        double x = xy[2 * k], y = xy[2 * k + 1];
        const int o = oldIdx.find(newIds[k]);
        if (o >= 0) {
            hm.ox.push_back(old.ox[o]); hm.oy.push_back(old.oy[o]);
            hm.bx.push_back(old.bx[o]); hm.by.push_back(old.by[o]);
            hm.vx.push_back(old.vx[o]); hm.vy.push_back(old.vy[o]);
            hm.fx.push_back(old.fx[o]); hm.fy.push_back(old.fy[o]);
        } else {
            lbib::perturbate(h, x, y);
            hm.ox.push_back(x - 5.0); hm.oy.push_back(y - 5.0);
            hm.bx.push_back(x); hm.by.push_back(y);
            hm.vx.push_back(0.0); hm.vy.push_back(0.0); hm.fx.push_back(0.0); hm.fy.push_back(0.0);
        }
        hm.x.push_back(x);
        hm.y.push_back(y);
    }
    const lbib::IdIndex newIdx(newIds);
    std::vector<int> nfoff(M + 1, 0), nftype, nfpart;
    std::vector<double> nfpar;
    for (int k = 0; k < M; ++k) {
        const int o = oldIdx.find(newIds[k]);
        if (o >= 0)
            for (int r = foff[o]; r < foff[o + 1]; ++r) {
                int p = fpart[r];
                if (p >= 0) {
                    p = p < (int)oldIds.size() ? newIdx.find(oldIds[p]) : -1;
                    if (p < 0) continue;  // its partner was removed
                }
                nftype.push_back(ftype[r]);
                nfpart.push_back(p);
                for (int q = 0; q < 4; ++q) nfpar.push_back(fpar[4 * (size_t)r + q]);
            }
        nfoff[k + 1] = (int)nftype.size();
    }
    // connections keep their boundary descriptor; new ones have none
    std::map<std::pair<uint32_t, uint32_t>, std::string> oldDesc;
    for (const auto& c : h.conns) oldDesc[{c.id1, c.id2}] = c.desc;
    std::vector<lbib::HConn> nc(C);
    uint32_t maxDom = 0;
    for (int c = 0; c < C; ++c) {
        nc[c].id1 = conns[3 * c];
        nc[c].id2 = conns[3 * c + 1];
        nc[c].dom = conns[3 * c + 2];
        if (newIdx.find(nc[c].id1) < 0 || newIdx.find(nc[c].id2) < 0)
            lbib::fail(LBIB_ERR_INPUT, "a connection names a node that is not in the list", c);
        auto it = oldDesc.find({nc[c].id1, nc[c].id2});
        nc[c].desc = it == oldDesc.end() ? std::string() : it->second;
        lbib::ensure_descriptor(h, nc[c].desc);
        maxDom = std::max(maxDom, nc[c].dom);
    }
    lbib::grow_domains(h, (int)maxDom + 1);
    h.ids = newIds;
    h.conns = nc;
    h.keepRecords = (int)nftype.size();
    lbib::upload_topology(h, hm, false);
    h.keepRecords = 0;
    CK(cudaMemcpyAsync(h.m.foff, nfoff.data(), sizeof(int) * (M + 1), cudaMemcpyHostToDevice, h.stream));
    if (!nftype.empty()) {
        CK(cudaMemcpyAsync(h.m.ftype, nftype.data(), sizeof(int) * nftype.size(), cudaMemcpyHostToDevice, h.stream));
        CK(cudaMemcpyAsync(h.m.fpartner, nfpart.data(), sizeof(int) * nfpart.size(), cudaMemcpyHostToDevice,
                           h.stream));
        CK(cudaMemcpyAsync(h.m.fpar, nfpar.data(), sizeof(double) * nfpar.size(), cudaMemcpyHostToDevice,
                           h.stream));
    }
    // new nodes are bound to the lattice at once: the edge test of
    // connectGeometryNodesToPhysicalNodes (GeometryHandler.cpp:618-636)
    lbib::reset_status(h, h.iteration, h.cellTypesCopied);
    lbib::launch_edge_check(h.m, h.nx, h.ny, h.st, 0, h.stream);
    lbib::read_status(h);
    if (h.stHost->err) lbib::fail(h.stHost->err, "geometry point moved too close to the boundary", h.stHost->errIndex);
    h.graphEpoch++;
    API_END
}

int lbib_cure_lattice(lbib_handle* hh) {
    API_BEGIN(hh)
    if (h.diff) lbib::fail(LBIB_ERR_STATE, "topology edits are not possible during a differentiated run");
    lbib::pull_topology(h);
    lbib::HostMembrane hm;
    lbib::download_membrane(h, hm);
    lbib::cure_lattice(h, hm);
    API_END
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The cell-division bio solver (tutorial_01_BioSolverCellDivision.cpp:42-140,
// the same in tutorial_02; BioSolverCellDivision.cpp with a random direction),
// run on the host after the step of every FREQUENCY-th iteration: it is the
// last bio solver of its run, so nothing on the device follows it in the step.

namespace lbib {

// The two connections of a cell that a division line crosses
// (getTwoConnectionsLongestAxis / getTwoConnectionsRandomDirection,
// tutorial_01_BioSolverCellDivision.cpp:151-248): connection (p, q) is cut
// when p lies above the line and q below it, or p on or below and q on or
// above.
static std::vector<int> cut_connections(const Handle& h, const HostMembrane& hm, const IdIndex& idx,
                                        const std::vector<int>& cell, double slope, double intercept) {
    std::vector<int> cut;
    for (int c : cell) {
        const int p = idx.at(h.conns[c].id1), q = idx.at(h.conns[c].id2);
        const bool c1 = hm.y[p] > slope * hm.x[p] + intercept;
        const bool c2 = hm.y[q] < slope * hm.x[q] + intercept;
        if ((c1 && c2) || (!c1 && !c2)) cut.push_back(c);
    }
    return cut;
}

static std::map<std::string, std::vector<std::string>> descriptor_map(const std::string& desc) {
    std::stringstream ls(desc);
    std::map<std::string, std::vector<std::string>> m;
    std::string a, b;
    while (ls >> a >> b) m[a].push_back(b);
    return m;
}

// divideCell (tutorial_01_BioSolverCellDivision.cpp:94-149) on the host
// mirror; returns the new cell's domain id.
static uint32_t divide_cell(Handle& h, const HostMembrane& hm, uint32_t dom,
                            const std::map<uint32_t, std::vector<int>>& cells) {
    const uint32_t newId = cells.rbegin()->first + 1;
    const IdIndex idx(h.ids);
    const std::vector<int>& cell = cells.at(dom);
    std::vector<int> cut;
    if (h.divisionPolicy == 0) {
        // the furthest pair of the connections' first nodes (the first found
        // of equal distance), then the perpendicular bisector
        double dist = 0.0;
        int n1 = -1, n2 = -1;
        for (int c1 : cell)
            for (int c2 : cell) {
                const int a = idx.at(h.conns[c1].id1), b = idx.at(h.conns[c2].id1);
                const double dx = hm.x[a] - hm.x[b], dy = hm.y[a] - hm.y[b];
                const double d = std::sqrt(dx * dx + dy * dy);
                if (d > dist) {
                    dist = d;
                    n1 = a;
                    n2 = b;
                }
            }
        if (n1 < 0) fail(ERR_STATE, "cell division: degenerate cell", dom);
        const double mx = 0.5 * (hm.x[n1] + hm.x[n2]), my = 0.5 * (hm.y[n1] + hm.y[n2]);
        const double slope = -(hm.x[n2] - hm.x[n1]) / (hm.y[n2] - hm.y[n1]);
        const double intercept = my - slope * mx;
        cut = cut_connections(h, hm, idx, cell, slope, intercept);
    } else {
        // a random direction through the centre of the first nodes
        double cx = 0.0, cy = 0.0;
        for (int c : cell) {
            const int a = idx.at(h.conns[c].id1);
            cx += hm.x[a];
            cy += hm.y[a];
        }
        cx /= (double)cell.size();
        cy /= (double)cell.size();
        std::uniform_real_distribution<> angle(0.0, 2.0 * M_PI);
        for (int tries = 1;; ++tries) {
            const double slope = std::tan(angle(h.genDiv));
            const double intercept = cy - slope * cx;
            cut = cut_connections(h, hm, idx, cell, slope, intercept);
            if (cut.size() == 2) break;
            if (tries > 10) fail(ERR_STATE, "could not find cell division plane", dom);
        }
    }
    if (cut.size() != 2) fail(ERR_STATE, "More or less than 2 connections found in the cell division", dom);
    const HConn c0 = h.conns[cut[0]], c1 = h.conns[cut[1]];
    if (descriptor_map(c0.desc) != descriptor_map(c1.desc))
        fail(ERR_STATE, "The method cannot handle cell division cases with heterogeneous boundary conditions.", dom);
    // the two new connections are appended, the two cut ones erased
    std::vector<HConn> next;
    next.reserve(h.conns.size());
    for (size_t c = 0; c < h.conns.size(); ++c)
        if ((int)c != cut[0] && (int)c != cut[1]) next.push_back(h.conns[c]);
    next.push_back(HConn{c0.id1, c1.id2, dom, c0.desc});
    next.push_back(HConn{c1.id1, c0.id2, dom, c0.desc});
    h.conns.swap(next);
    // the ring through c1's second node becomes the new cell
    std::map<uint32_t, int> out;
    for (size_t c = 0; c < h.conns.size(); ++c) out[h.conns[c].id1] = (int)c;
    const int start = out.at(c1.id2);
    int c = start;
    do {
        h.conns[c].dom = newId;
        c = out.at(h.conns[c].id2);
    } while (c != start);
    return newId;
}

static void run_division(Handle& h) {
    // GeometryHandler::computeAreas, in ring order
    launch_rings(h.m, h.td, h.st, h.stream);
    launch_areas(h.m, h.area, nullptr, h.stream);
    std::vector<double> a(h.m.nCells);
    if (h.m.nCells) CK(cudaMemcpyAsync(a.data(), h.area, sizeof(double) * a.size(), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    h.ringsCurrent = true;
    std::map<uint32_t, double> areas;
    for (int c = 0; c < h.m.nCells; ++c) areas[h.ringDomHost[c]] = a[c];
    areas[0] = 0.0;
    // LbibCellDivision: a cell's threshold is divisionFactor times its
    // reference area, the area at the solver's first look at it
    if (h.divisionFactor > 0.0)
        for (const auto& kv : areas)
            if (kv.first != 0 && !h.divisionRef.count(kv.first)) h.divisionRef[kv.first] = kv.second;
    auto divides = [&](uint32_t dom, double area) {
        return h.divisionFactor > 0.0 ? area > h.divisionFactor * h.divisionRef[dom] : area > h.divisionMax;
    };
    bool any = false;
    for (auto it = std::next(areas.begin()); it != areas.end(); ++it) any |= divides(it->first, it->second);
    HostMembrane hm;
    if (any) {
        // the host mirror of the membrane, only when a cell divides
        pull_topology(h);
        download_membrane(h, hm);
        sync_targets(h);
    }
    auto cellsOf = [&]() {
        std::map<uint32_t, std::vector<int>> cells;
        for (size_t c = 0; c < h.conns.size(); ++c) cells[h.conns[c].dom].push_back((int)c);
        return cells;
    };
    for (auto it = std::next(areas.begin()); it != areas.end(); ++it) {
        if (!divides(it->first, it->second)) continue;
        const uint32_t newId = divide_cell(h, hm, it->first, cellsOf());
        if (h.divisionFactor > 0.0) h.divisionRef[newId] = h.divisionRef[it->first];
        grow_domains(h, (int)newId + 1);
        h.ctypeHost[newId] = it->first < h.ctypeHost.size() ? h.ctypeHost[it->first] : 1u;
        // the daughter's nodes keep the mass source the step's area regulator
        // gave them (FluidSolver::addMass ran before the division)
        if (it->first < (uint32_t)h.nDomains)
            CK(cudaMemcpyAsync(h.massTab + newId, h.massTab + it->first, sizeof(double), cudaMemcpyDeviceToDevice,
                               h.stream));
        // the edited topology on the device (the force list stays: no node
        // changed), then GeometryHandler::cureLattice
        std::vector<int> foff(h.m.M + 1);
        CK(cudaMemcpyAsync(foff.data(), h.m.foff, sizeof(int) * (h.m.M + 1), cudaMemcpyDeviceToHost, h.stream));
        CK(cudaStreamSynchronize(h.stream));
        h.keepRecords = foff[h.m.M];
        upload_topology(h, hm, false);
        h.keepRecords = 0;
        cure_lattice(h, hm);
        h.graphEpoch++;
    }
    // copyCellTypeToPhysicalNodes: the cell-type table
    CK(cudaMemcpyAsync(h.ctypeTab, h.ctypeHost.data(), sizeof(uint32_t) * h.nDomains, cudaMemcpyHostToDevice,
                       h.stream));
    CK(cudaStreamSynchronize(h.stream));
}

// GeometryHandler::computeAccumulatedDomainConcentrations (GeometryHandler.cpp:
// 136-147): per domain, the sum of species k's getC() over the lattice, rows
// in order and columns from x = 1 (column 0 is left out, as there).
static std::map<uint32_t, double> accumulated_concentrations(Handle& h, int k) {
    const size_t L = h.L;
    std::vector<uint32_t> dom(L);
    const size_t rs = h.precision == LBIB_FP64 ? sizeof(double) : sizeof(float);
    std::vector<unsigned char> raw(5 * L * rs);
    CK(cudaMemcpyAsync(dom.data(), h.dom, sizeof(uint32_t) * L, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaMemcpyAsync(raw.data(), (const unsigned char*)h.g[h.cur] + (size_t)k * 5 * L * rs, 5 * L * rs,
                       cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    auto val = [&](int q, size_t n) {
        return rs == 8 ? ((const double*)raw.data())[(size_t)q * L + n] : (double)((const float*)raw.data())[(size_t)q * L + n];
    };
    std::map<uint32_t, double> acc;
    for (int y = 0; y < h.ny; ++y)
        for (int x = 1; x < h.nx; ++x) {
            const size_t n = (size_t)y * h.nx + x;
            double C = 0.0;  // getC(): slots T, W, S, E, N after localSwap
            C += val(0, n);
            C += val(3, n);
            C += val(4, n);
            C += val(1, n);
            C += val(2, n);
            acc[dom[n]] += C;
        }
    return acc;
}

// tutorial_01_BioSolverDifferentiation::applyBioProcess
// (tutorial_01_BioSolverDifferentiation.cpp:42-84): the first call resets the
// cell-type map (domain 0 type 0, every cell type 1); each call marks the
// cells whose accumulated signal is below THRESHOLD 1.6 as type 2 (the map's
// first domain, the extracellular one, is skipped) and copies the map to the
// lattice.  The reference's reset runs once per process (a std::once_flag);
// here it runs once per handle.
static void run_differentiation(Handle& h) {
    const std::map<uint32_t, double> acc = accumulated_concentrations(h, h.diffSpecies);
    if (!h.diffInit) {
        h.diffInit = true;
        std::fill(h.ctypeHost.begin(), h.ctypeHost.end(), 1u);
        if (!h.ctypeHost.empty()) h.ctypeHost[0] = 0;
    }
    for (auto it = std::next(acc.begin()); it != acc.end(); ++it)
        if (it->second < 1.6 && it->first < h.ctypeHost.size()) h.ctypeHost[it->first] = 2;
    CK(cudaMemcpyAsync(h.ctypeTab, h.ctypeHost.data(), sizeof(uint32_t) * h.nDomains, cudaMemcpyHostToDevice,
                       h.stream));
    CK(cudaStreamSynchronize(h.stream));
    h.cellTypesCopied = true;
}

}  // namespace lbib
