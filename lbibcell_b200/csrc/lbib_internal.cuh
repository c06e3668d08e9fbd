// lbib_internal.cuh — shared definitions of the lbibcell_b200 device runtime.
//
// Lattice layout in HBM (structure of arrays, one plane per direction):
//   distributions  f[q][n], q = 0..8 in the reference's D2Q9 order
//                  T,E,N,W,S,NE,NW,SW,SE (libs/LbmLib/include/Direction.hpp:34-44),
//                  n = y*nx + x.  Two copies (A/B) for the pull scheme; each
//                  copy holds the post-collision values of one step in natural
//                  direction order (the reference stores them under the
//                  inverse direction after FluidSolver::localSwap).
//   species        g[k][q][n], q = 0..4 (T,E,N,W,S), two copies.
//   velocity       u[2][n]  (post-collision fluid velocity, FluidSolver::velocity_)
//   force          F[2][n]  (spread IBM force, FluidSolver::force_), written and
//                  read only inside tiles that hold membrane stencils.
//   domain         dom[n] (u32, PhysicalNode::domainIdentifier_)
// FP64 mode stores f; FP32-shifted mode stores f - w_q (rest state rho0 = 1).
//
// Membrane (nodes kept in ascending id order, the reference's std::map order):
//   x, y, ox, oy, vx, vy, fx, fy (FP64), id (u32)
// Connections in Geometry::connections_ order: a[c], b[c] node indices, dom[c].
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <utility>
#include <cuda_runtime.h>

namespace lbib {

// Programmatic dependent launch.  The stage kernels of a step are short and
// many; launching each with programmatic stream serialization lets the
// launch and block scheduling of a kernel overlap the end of the previous
// one.  Every kernel except the adjoint step begins with griddepcontrol.wait,
// which returns once the previous grid has completed and its memory
// operations are visible, and none of those triggers its dependents early, so
// their blocks start only once every block of the previous kernel has exited.
// The adjoint step (k_adjoint.cu) triggers its dependents right after its own
// wait, and loads the inputs that no kernel of the reverse pass writes before
// that wait; a kernel launched after it therefore starts during its last wave,
// while every kernel before it has completed.  Ordering is the same as plain
// stream order.  LBIB_NO_PDL=1 launches without the attribute.
// Early triggers inside the time step were measured and are not used: the
// spread triggering the FP32 stream-collide kernel (which then loaded its
// planes before its wait) 0.1696 -> 0.1755 ms per step on tissue_1024, and
// every kernel triggering after its wait 0.201 ms.

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

inline bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("LBIB_NO_PDL");
        return !(e && e[0] == '1');
    }();
    return on;
}

// LBIB_CHECK_LAUNCHES=1, a fault diagnostic (off by default): every stage
// kernel launched outside a graph (all of them with LBIB_NO_GRAPHS=1), and
// every step graph, is waited for where it is launched, and a failure names
// the kernel or the step on stderr.
inline bool check_launches() {
    static const bool on = [] {
        const char* e = std::getenv("LBIB_CHECK_LAUNCHES");
        return e && e[0] == '1';
    }();
    return on;
}

// A launch with (programmatic) or without programmatic stream serialization.
template <typename... KArgs, typename... Args>
inline void launch_ex(bool programmatic, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                      cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = programmatic && pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
    if (check_launches()) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(s, &cs);
        if (cs == cudaStreamCaptureStatusNone) {
            const cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                const char* name = "?";
                cudaFuncGetName(&name, (const void*)kernel);
                std::fprintf(stderr, "lbib: kernel %s (grid %u x %u, block %u) failed: %s\n", name, grid.x, grid.y,
                             block.x, cudaGetErrorString(e));
            }
        }
    }
}

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
    launch_ex(true, kernel, grid, block, smem, s, std::forward<Args>(args)...);
}

// Direction tables: libs/LbmLib/include/Direction.hpp:34-44 and
// libs/LbmLib/src/Direction.cpp:27-61.
enum Dir { T = 0, E = 1, N = 2, W = 3, S = 4, NE = 5, NW = 6, SW = 7, SE = 8 };

// Constants: libs/LbmLib/include/Constants.hpp:31-49.
constexpr double kEPSILON = 10E-10;
constexpr double kPERTURBATION = 10E-7;
constexpr double kMAXLENGTH = 0.5;

// Status word shared by all stage kernels (device memory, one per handle).
struct Status {
    int halt;          // non-zero: later stage kernels return immediately
    int haltStage;     // stage that raised the halt
    int err;           // LBIB_ERR_* (0 = none)
    int errIndex;      // node / connection index of the first error
    int nPerturbNode;  // membrane nodes whose position needs the host RNG
    int nPerturbConn;  // connections that need Connection::perturbConnection
    int nChanged;      // lattice nodes whose domain id changed (reinit list)
    int nRecords;      // crossing records this step
    int remesh;        // a connection is longer than MAXLENGTH
    int coarsen;       // a node is a coarsening candidate
    int nDiagReinit;   // reinit from diagonal neighbours
    int nFailedReinit; // reinit without any neighbour (division by zero)
    unsigned iteration;   // Parameters' current iteration of the step being run
    int cellTypesCopied;  // copyCellTypeToPhysicalNodes has run (after the first step)
    int pad[4];           // [0] steps of a run completed before its current one, [2] crossing records of the step, [3] first step of a run
};

// Stage numbers (halt points), in the reference's order of
// SimulationRunner::runSimulation (SimulationRunner.cpp:72-99).
enum Stage {
    ST_FORCE = 1,
    ST_SPREAD = 2,
    ST_COLLIDE = 3,
    ST_INTERP_MOVE = 4,
    ST_PERTURB_CONN = 5,
    ST_CROSSINGS = 6,
    ST_REINIT = 7,
    ST_DOMAIN = 8,
    ST_REMESH = 9,
    ST_REMESH_COMMIT = 10,  // the remesh pass's commit (resumed at after the host perturbed its new nodes)
    ST_COARSEN = 11,
    ST_OUTLET = 12,
    ST_BIO = 13,
    ST_DONE = 14,
    ST_REMESH_RNG = 15,     // halt only: new nodes of the remesh pass need the host's random perturbation
};

// Error codes (also returned through the C ABI, include/lbibcell.h).
enum Err {
    ERR_OK = 0,
    ERR_EDGE_W = 10, ERR_EDGE_S = 11, ERR_EDGE_E = 12, ERR_EDGE_N = 13,
    ERR_SPEED = 20,
    ERR_LEFT_DOMAIN = 30,
    ERR_VERTICAL = 40,
    ERR_FORCE_NODE = 50,
    ERR_STENCIL = 60,
    ERR_CAPACITY = 70,
    ERR_CUDA = 80,
    ERR_INPUT = 90,
    ERR_STATE = 91,
};

__device__ __forceinline__ void raise_error(Status* st, int code, int index, int stage) {
    if (atomicCAS(&st->err, 0, code) == 0) st->errIndex = index;
    atomicExch(&st->halt, 1);
    atomicCAS(&st->haltStage, 0, stage);
}

// The start of a step, run by thread 0 of the step's first kernel when no halt
// is pending: the step before it in the same run is then complete, so it is
// counted (Parameters++, SimulationRunner.cpp:98) before this step's kernels
// read the iteration; then the step's counters are cleared.  pad[3], set with
// the status word, marks the first step of a run, which has no predecessor
// there.  (The host counts the run's last step itself: it completed unless a
// halt is pending.)
__device__ __forceinline__ void begin_step(Status* st) {
    if (st->pad[3]) {
        st->pad[3] = 0;
    } else {
        st->pad[0] += 1;
        st->iteration += 1;
        st->cellTypesCopied = 1;
    }
    st->pad[2] = 0;
    st->nPerturbNode = 0;
    st->nPerturbConn = 0;
    st->nChanged = 0;
    st->nRecords = 0;
    st->remesh = 0;
    st->coarsen = 0;
}

__device__ __forceinline__ void raise_halt(Status* st, int stage) {
    atomicExch(&st->halt, 1);
    atomicCAS(&st->haltStage, 0, stage);
}

// Reaction kinds of the CDE species (the reaction term of each solver's collide):
//   RX_NONE      CDESolverD2Q5
//   RX_LINEAR    source[domain] - decay*C (the Lbib species plugins)
//   RX_SIGNAL    tutorial_01_CDESolverD2Q5_SIGNAL.cpp:92-100; CDESolverD2Q5HH.cpp:113-129
//                computes the same terms with the same constants
//   RX_T2_R/L    tutorial_02_CDESolverD2Q5_R.cpp:94-105 / _L.cpp:94-106 (partner L / R)
//   RX_SCHNAK_U/V SchnakenbergD2Q5u.cpp:114-121 / v.cpp:110-117 (partner v / u)
//   RX_BMP       CDESolverD2Q5BMP.cpp:107-120 (partner CDESolverD2Q5HH, cell type 2)
enum Reaction {
    RX_NONE = 0, RX_LINEAR = 1, RX_SIGNAL = 2, RX_T2_R = 3, RX_T2_L = 4, RX_SCHNAK_U = 5, RX_SCHNAK_V = 6,
    RX_BMP = 7
};
// The kinds whose reaction reads another species or the cell type.
__host__ __device__ __forceinline__ bool coupled_kind(int kind) { return kind >= RX_T2_R; }

// reinitialise() variants (domain change of a lattice node):
//   RI_BASE  CDESolverD2Q5.cpp:156-228: E,N,W,S, then the diagonals, else 0/0
//   RI_ALL4  tutorial_01_CDESolverD2Q5_SIGNAL.cpp:184-250 (and tutorial_02 R/L,
//            BMP, HH): as RI_BASE, then all of E,N,W,S whatever their domain
//   RI_DIAG  SchnakenbergD2Q5u.cpp:190-231 and v: the four diagonals
//            of the same domain without the boundary-node test, C/4 per slot
enum Reinit { RI_BASE = 0, RI_ALL4 = 1, RI_DIAG = 2 };

constexpr int kMaxSpecies = 3;

// Per-species constants for the lattice kernels.
struct SpeciesConst {
    int kind;
    double tau;
    double decay;
    int partner;    // species index the reaction reads (-1: none)
    int reinit;     // Reinit
    double dt;      // the solver's deltaT (SchnakenbergD2Q5u/v: 20 / Iterations; BMP: 1)
    double hill;    // RX_BMP: pow(k_hill, n_hill) as the host's pow gives it
    int bounce;     // DiracD2Q5: advect keeps the populations of links with a boundary node
    // FP32 forms for the FP32-shifted kernel, set by its launcher from the
    // fields above: (float)(1 / tau), (float)decay, (float)dt, (float)hill
    float tIf, decayf, dtf, hillf;
};

// Boundary solvers on connections (the "bsolver cdesolver" pairs of a
// geometry file's connection lines, Geometry.cpp:122-151), per distinct list
// of pairs: the solvers in name order (BoundaryNode's std::map), each with its
// CDE solvers in file order.
enum NoFluxKind { NF_NOFLUX = 1, NF_NOFLUX_D2Q5 = 2 };  // BoundarySolverNoFlux, BoundarySolverNoFluxD2Q5
struct NfSolver {
    int kind;
    int nCde;
    int cde[4];  // species indices
};
struct NfSpec {
    int nSolvers;
    NfSolver s[2];
};

// Everything the fused stream-collide kernel reads besides the planes.
template <typename Real>
struct LatticeArgs {
    int nx, ny;
    size_t L;
    int S;
    const Real* fin;      // 9*L
    Real* fout;           // 9*L
    const Real* gin;      // S*5*L
    Real* gout;           // S*5*L
    Real* u;              // 2*L
    const Real* force;    // 2*L (valid where tileCount > 0)
    const int* tileCount; // per 16x16 tile: membrane stencils overlapping it
    int tilesX;
    const uint32_t* dom;  // L
    const double* massTab;     // per-domain rhoToAdd (nullptr: none)
    const double* massNode;    // per-node rhoToAdd (nullptr: none; replaces massTab)
    int nDomains;              // entries in massTab / srcTab rows
    const double* srcTab;      // [S][nDomains] production per step
    const uint32_t* ctypeTab;  // per-domain cell type (read by RX_BMP)
    double tauF;
    float tauIf, gff;          // FP32-shifted kernel: (float)(1 / tauF), (float)(1 - 1 / (2 tauF)), set by its launcher
    int forceModel;            // FM_LUO, FM_GUO (as the reference writes it), FM_GUO_CORRECTED
    SpeciesConst sp[kMaxSpecies];
    int coupled;               // some species has a coupled_kind reaction
    const Status* status;
    int outlet;                // MassSolverBoxOutlet registered: rescale x=0 / y=0 nodes
    // no-flux boundary nodes of the previous step's crossings (nullptr: none)
    const uint8_t* nfSpec;     // 4*L: descriptor index + 1 per (node, slot E,N,W,S), 0 none
    const double* nfU;         // 8*L: the boundary node's velocity per (node, slot)
    const NfSpec* nfTab;
    const uint32_t* nfKeys;    // the (node, slot) keys set in nfSpec
    const int* nfN;            // number of nfKeys
    int nfCap;
    double* nfD;               // 2 per key: preAdvect's value of each solver
    // links with a boundary node, for species whose advect keeps their
    // populations (DiracD2Q5): per node, a boundary node in the W / S slot
    // (nullptr: no such species)
    const uint8_t* bounceW;
    const uint8_t* bounceS;
};

constexpr int kTile = 16;  // force tiles are 16x16 lattice nodes

// Force models of FluidSolver (its base class, FluidSolver.hpp:41):
// Luo1993ForceModel (compiled in by the reference), GuoZhengShi2002ForceModel
// as the reference writes it (NE term with -3 u_y, GuoZhengShi2002ForceModel.cpp:51)
// and with the coefficient of the model's expansion (+6 u_y).
enum ForceModel { FM_LUO = 0, FM_GUO = 1, FM_GUO_CORRECTED = 2 };
__host__ __device__ __forceinline__ double guo_ne_y(int forceModel) { return forceModel == FM_GUO ? -3.0 : 6.0; }

}  // namespace lbib
