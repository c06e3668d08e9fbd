// kernels.cuh — launch wrappers of the lbibcell_b200 device kernels.
#pragma once

#include "lbib_internal.cuh"

namespace lbib {

// Membrane counts live in device memory: remeshing and coarsening change them
// on the device, and kernels launched ahead of time size their work from here.
struct Topo {
    int M;            // membrane nodes
    int C;            // connections
    unsigned maxId;   // id of the last node (ids ascend with the index)
    int changed;      // the topology changed: rings must be rebuilt
    int K;            // connections split by the current remesh pass
    int removed;      // nodes removed by the current coarsening
    int nCand;        // coarsening candidates
    unsigned done;    // blocks of the remesh count / copy that have finished (the last one decides / commits)
    int nRng;         // new nodes of the remesh pass that need the random perturbation
    int rngFill;      // entries of TopoDev::rngList (those nodes' indices)
};

// Membrane state on the device (nodes in ascending id order).
struct MembraneDev {
    Topo* topo;     // device counts
    int Mcap, Ccap; // capacities (launch grids)
    int M;          // host view of the node count (valid after a pull)
    int C;          // host view of the connection count
    double* x; double* y;       // LagrangianPoint::position_
    double* ox; double* oy;     // GeometryNode::oldPosition_
    // position at the node's last stencil binding: GeometryNode::
    // neighbourPhysicalNodes_ is rebound only when isUpdateNeeded fires
    // (GeometryNode.cpp:256-261), from the position of that moment
    // (GeometryHandler.cpp:608-644); the stencil ranges derive from it
    double* bx; double* by;
    double* vx; double* vy;     // LagrangianPoint::velocity_
    double* fx; double* fy;     // GeometryNode::force_
    uint32_t* id;
    int* prev; int* next;       // ring neighbours (node indices)
    int* ca; int* cb;           // connection endpoints (node indices), vector order
    uint32_t* cdom;             // connection domain ids
    int* cdesc;                 // connection boundary-descriptor index (host string table)
    // force records (CSR by node, insertion order)
    int* foff;                  // M+1
    int* ftype; int* fpartner;  // records
    double* fpar;               // 4 parameters per record
    // rings for the area computation (GeometryHandler::computeAreas order)
    int nCells;
    int* ringStart;             // nCells+1
    int* ringNode;              // node indices, ring order
    uint32_t* ringDom;          // domain of each ring
};

// Scratch of the device force-list edits and of the cell-junction search.
enum ForceGen { GEN_NONE = 0, GEN_TENSION = 1, GEN_JUNCTION = 2, GEN_LIST = 3 };
// Force-list operations of one bio solver in one step (2 bits per solver).
enum BioOp { BIO_NONE = 0, BIO_TENSION_FILL = 1, BIO_TENSION_EDIT = 2, BIO_JUNCTIONS = 3 };
struct ForceScratch {
    int Fcap;                   // capacity of the force records
    int* foffS;                 // Mcap+1: offsets before the edit
    int* ftypeS; int* fpartnerS; double* fparS;  // Fcap: records before the edit
    int* cnt;                   // Mcap+1: records per node after the edit
    void* scanTmp; size_t scanTmpBytes;
    int* outPos; int* inPos;    // Mcap: a node's outgoing / incoming connection
    // cell junctions
    unsigned* binKey; unsigned* binKeySorted;  // Mcap: cell-list bin of each node
    int* binIdx; int* binIdxSorted;            // Mcap: node index
    void* sortTmp; size_t sortTmpBytes;
    int sortBits;               // key bits: bins 0..nx*ny-1, nx*ny for unused slots
    int* binStart;              // nx*ny: first sorted position of each bin (checked on use)
    unsigned binCap;            // nx*ny
    // the junction step's own cell list: per bin a linked list of its nodes
    int* binHead;               // nx*ny: first node of the bin's list, -1 empty
    int* binNext;               // Mcap: next node of the same bin, -1 end
    unsigned* linkKey;          // Mcap: the bin each node was linked into
    int* linkPrevM;             // 1: nodes linked by the last call (their heads are cleared by the next)
    int* closest;               // Mcap: closest node of another cell within the radius, -1: none
    int* inCnt; int* inOff;     // Mcap+1: nodes that found node i, and their offsets
    int* inList; int* inFill;   // Mcap
    // records added through the C ABI: CSR by node (Mcap+1 offsets), in call order
    int* listOff; int* listType; int* listPartner; double* listPar;
    int listCap;
};

// Crossing resolution buffers (dense per lattice node and slot E,N,W,S).
struct CrossDev {
    unsigned long long* bnDist;  // 4*L, EMPTY = ~0ull
    uint32_t* bnConn;            // 4*L, ~0u
    uint32_t* bnDom;             // 4*L
    uint32_t* wDom;              // L, W-slot winner domain + 1 (0: none)
    int* mark;                   // L, position + 1 of a node in this step's changed list (0: none)
    int* reinitDone;             // changedCap: 1 = re-initialised by the wide pass, 2 + w = waiting at waitList[w]
    int* waitList;               // changedCap: list positions of the nodes that wait for another
    int* nWait;                  // entries of waitList
    uint32_t* changedNode;       // capacity: nodes whose domain changes
    uint32_t* changedDom;
    int changedCap;
    int diag8;                   // a species re-initialises from all four diagonals (RI_DIAG)
    int* perturbList;            // membrane node indices flagged for the host RNG
    int perturbCap;
    // crossing records of this step (one per candidate node-slot pair)
    uint32_t* recKey; uint32_t* recConn; uint32_t* recDom; unsigned long long* recDist;
    int recCap;
    // boundary nodes with boundary solvers, for the next step's stream-collide
    // (nfTab == nullptr when no connection has one)
    const NfSpec* nfTab;         // per connection descriptor index
    uint8_t* nfSpec;             // 4*L, descriptor index + 1 (0: none)
    double* nfU;                 // 8*L, boundary node velocity (x, y)
    uint32_t* nfKeys;            // keys set in nfSpec, for the reset
    double* nfD;                 // 2 per key, scratch of the boundary solvers
    int* nfN;                    // number of nfKeys
    int nfCap;
    // the W- and S-slot boundary nodes of this step's crossings, for the next
    // step's advect of DiracD2Q5 species (nullptr when none is registered)
    uint8_t* bounceW;            // L
    uint8_t* bounceS;            // L
    uint32_t* bounceKeys;        // keys set, for the reset
    int* bounceN;
    int bounceCap;
};

// Tiles for force spreading.
struct TileDev {
    int tilesX, tilesY, nTiles;
    int* count;     // nTiles
    int* fill;      // nTiles
    int* start;     // nTiles + 1
    int* list;      // capacity entries
    int cap;
    void* scanTmp;  // CUB temporary storage
    size_t scanTmpBytes;
    int* slots;     // FP32-shifted runs: nTiles x kTileSlots membrane indices (unordered)
};

// Entries a tile's slot list holds (the fixed-point spread's 32-bit low parts
// cannot overflow below 1024 contributions per lattice node either).
constexpr int kTileSlots = 1024;

// Scratch of the device-side topology edits and the ring ranking.
struct TopoDev {
    int* flag;          // Ccap + 1
    int* rank;          // Ccap + 1
    int* nflag;         // Mcap + 1
    int* nrank;         // Mcap + 1
    int* ca2; int* cb2; uint32_t* cdom2; int* cdesc2;    // Ccap
    double* dalt;       // 10 * Mcap node doubles
    uint32_t* id2; int* prev2; int* next2;                // Mcap
    int* inConn; int* outConn;                            // Mcap
    unsigned char* removed;                               // Mcap
    int* connAlive;                                       // Ccap
    int* ncA; int* ncB; uint32_t* ncDom; int* ncDesc; int* ncAlive;  // Mcap
    int nCellsCap;
    int* cellOfDom;     // nDomains (cell index of a domain id, -1 none)
    int* firstConn;     // nDomains
    int* cellCount;     // nCells + 1
    int* cellStart;     // nCells + 1
    int* cellFill;      // nCells
    int* members;       // Mcap
    int* succ; int* dist;                                 // Mcap
    int* rngList;       // Mcap: new nodes of a remesh pass that need the host's random perturbation
    int* startNode;     // nCells
    void* scanTmp; size_t scanTmpBytes;
    int nDomains;
};

void launch_stream_collide64(const LatticeArgs<double>& a, cudaStream_t s);
// The membrane boundary solvers (2 launches, before the stream-collide kernel
// of the same state); the stream-collide launchers call it when a.nfTab is set.
template <typename Real>
void launch_noflux(const LatticeArgs<Real>& a, cudaStream_t s);
void launch_outlet64(double* f, double* g, int nS, int nx, int ny, size_t L, const Status* st, cudaStream_t s);
// vel == nullptr: FluidSolver::initSolver (f_T = 1, then collide); else
// FluidSolver::initWithVelocity at the uniform velocity vel[0], vel[1].
void launch_init64(double* f, double* g, double* u, int nS, size_t L, double tauF, const uint32_t* dom,
                   const double* vel, const SpeciesConst* sp, const double* init, cudaStream_t s);

void launch_stream_collide32(const LatticeArgs<float>& a, cudaStream_t s);
void launch_outlet32(float* f, float* g, int nS, int nx, int ny, size_t L, const Status* st, cudaStream_t s);
void launch_init32(float* f, float* g, float* u, int nS, size_t L, double tauF, const uint32_t* dom,
                   const double* vel, const SpeciesConst* sp, const double* init, cudaStream_t s);

// Membrane pipeline.  `Real` is the lattice precision (velocity / force planes).
template <typename Real>
// `tiles`: also fill the FP32-shifted spread's per-tile slot lists (then call
// launch_spread with slotsFilled).
void launch_force_eval(const MembraneDev& m, Status* st, unsigned iteration, cudaStream_t s, bool begin = false,
                       TileDev* tiles = nullptr, int nx = 0, int ny = 0);
template <typename Real>
void launch_spread(const MembraneDev& m, TileDev& t, Real* force, int nx, int ny, size_t L, Status* st,
                   unsigned iteration, cudaStream_t s, bool slotsFilled = false);
template <typename Real>
void launch_interp_move(const MembraneDev& m, const Real* u, int nx, int ny, size_t L, CrossDev& c, Status* st,
                        unsigned iteration, cudaStream_t s);
void launch_perturb_conn_check(const MembraneDev& m, Status* st, unsigned iteration, cudaStream_t s, int* list,
                               int cap);
template <typename Real>
void launch_crossings(const MembraneDev& m, CrossDev& c, const uint32_t* dom, int nx, int ny, size_t L, Status* st,
                      unsigned iteration, cudaStream_t s);
template <typename Real>
void launch_reinit(CrossDev& c, uint32_t* dom, Real* g, const Real* u, int nS, const SpeciesConst* sp,
                   const double* srcTab, int nDomains, const uint32_t* ctypeTab, int cellTypesCopied, int nx,
                   int ny, size_t L, Status* st, unsigned iteration, cudaStream_t s);
void launch_domain_fill(CrossDev& c, uint32_t* dom, int nx, int ny, size_t L, Status* st, unsigned iteration,
                        cudaStream_t s);
void launch_edge_check(const MembraneDev& m, int nx, int ny, Status* st, unsigned iteration, cudaStream_t s);
void launch_remesh_check(Status* st, unsigned iteration, cudaStream_t s);
void launch_coarsen_check(const MembraneDev& m, Status* st, unsigned iteration, cudaStream_t s);
void launch_clear_forces(MembraneDev& m, cudaStream_t s);
// ForceSolver::deleteForceType(6) + the membrane-tension records, on a list that
// holds other forces too (launches returned).
int launch_tension_edit(MembraneDev& m, ForceScratch& fs, double force, Status* st, cudaStream_t s);
// The cell-junction bio solver (launches returned).
int launch_junctions(MembraneDev& m, ForceScratch& fs, int nx, int ny, double radius, double K, double L0,
                     Status* st, cudaStream_t s);
size_t force_scan_bytes(int n);
// ForceSolver::deleteForceType(delType) (delType < 0: none) followed by the
// records of `gen` (GEN_NONE, GEN_LIST) appended per node (launches returned).
int launch_force_edit(MembraneDev& m, ForceScratch& fs, int delType, int gen, double tensionForce, double K,
                      double L0, Status* st, cudaStream_t s);
// The cell list of the nodes (1-lu bins, id order within a bin) and each
// node's outgoing/incoming connection, for the range queries.
int launch_cell_list(MembraneDev& m, ForceScratch& fs, int nx, int ny, cudaStream_t s);
// Geometry::getGeometryNodesWithinRadius[WithAvoidance][Closest] for nq query
// points (mode 0: the ids of all hits of query 0, up to cap, count in *count;
// mode 1: the id of the closest hit of each query, or -1, in closest[q]).
void launch_range_query(MembraneDev& m, ForceScratch& fs, int nx, int ny, const double* qx, const double* qy,
                        const long long* avoid, int nq, double radius, int mode, unsigned* ids, int cap, int* count,
                        long long* closest, cudaStream_t s);
size_t junction_sort_bytes(int n, int bits);
void launch_tension_renewal(MembraneDev& m, int* outPos, int* inPos, double force, cudaStream_t s);
// ctypeTab != nullptr selects tutorial_01_BioSolverAreaRegulator's rule (fixed
// target, cell type 1 at maxsource); nullptr the LbibAreaRegulator rule.
void launch_area_regulator(const MembraneDev& m, double* area, double* target, double* massTab, int nDomains,
                           double factor, double strength, double maxsource, const uint32_t* ctypeTab,
                           const Status* st, cudaStream_t s);
// st != nullptr: a ring longer than the kernel's limit raises ERR_CAPACITY there.
void launch_areas(const MembraneDev& m, double* area, Status* st, cudaStream_t s);
// dL/d of each force record's 4 parameters from the node-force gradient (gfx, gfy).
void launch_force_param_grad(const MembraneDev& m, const double* gfx, const double* gfy, double* gpar,
                             cudaStream_t s);
// GeometryHandler::computeAreas from exact fixed-point shoelace sums (FP32-shifted
// runs): independent of the summation order, so no ring order is needed.
void launch_areas_fixed(const MembraneDev& m, const int* cellOfDom, int nDomains, unsigned long long* acc,
                        double* area, cudaStream_t s);
// FP32-shifted runs: areas from the connections in fixed point (no ring order
// needed), then the regulator.  acc (nCells) must start at zero; it is left zero.
void launch_area_regulator_fixed(const MembraneDev& m, const int* cellOfDom, unsigned long long* acc, double* area,
                                 double* target, double* massTab, int nDomains, double factor, double strength,
                                 double maxsource, const uint32_t* ctypeTab, const Status* st, cudaStream_t s);
// massNode[n] = massTab[dom[n]] (0 outside cells).
void launch_mass_expand(const uint32_t* dom, size_t L, const double* massTab, int nDomains, double* massNode,
                        const Status* st, cudaStream_t s);
// tutorial_02_BioSolverGrowth: the per-node mass source from species iR, iL.
template <typename Real>
void launch_growth(const Real* g, const uint32_t* dom, size_t L, int iR, int iL, double* massNode, const Status* st,
                   cudaStream_t s);

// Cells that fit the fixed device array of lbib_areas_static (16384 doubles,
// 128 KB), and the address of that array on the current device.
constexpr int kStaticAreaCells = 16384;
cudaError_t static_area_scratch(double** ptr);

// Device-side topology edits (k_topology.cu).  Each returns the number of
// kernels it launched.
// A connection to perturb (Connection::perturbConnection), with what the host
// needs to do it in GeometryHandler::perturbConnections' order
// (GeometryHandler.cpp:326-356): its cell's ring walk starts at the domain's
// first connection in vector order and follows the second node's outgoing
// connection; walk = the connection's place in that walk (-1: no ring found),
// len = the ring's length, z = the first node of the walk's last connection
// (whose second node is the walk's first node).
struct ConnPerturbRec {
    int dom, walk, len, a, b, z;
    double xa, ya, xb, yb, xz, yz;
};
void launch_conn_perturb_gather(const MembraneDev& m, const TopoDev& t, int n, ConnPerturbRec* out, cudaStream_t s);

// A remesh pass (count, apply, commit); commitOnly: the commit alone, after
// the host perturbed the pass's new nodes (halt ST_REMESH_RNG).
int launch_remesh(MembraneDev& m, TopoDev& t, int nx, int ny, Status* st, cudaStream_t s, bool commitOnly = false);
int launch_coarsen(MembraneDev& m, TopoDev& t, Status* st, cudaStream_t s);
int launch_rings(MembraneDev& m, TopoDev& t, Status* st, cudaStream_t s);
size_t topo_scan_bytes(int n);

// Adjoint of one FP64 lattice step of a differentiated run (k_adjoint.cu).
struct AdjointArgs {
    int nx, ny;
    size_t L;
    int S;
    const void* fprev;     // 9*L      state after step t-1 (FP64, or FP32 deviations from rest with fp32)
    const void* gprev;     // S*5*L
    int fp32;              // the states are FP32-shifted (f = stored value + w_q)
    const float* pf;       // 9*L      adjoint planes of step t+1 (unused with seed), FP32
    const float* pg;       // S*5*L
    const double* seed;    // S*L      dL/dC_k at the final step, or nullptr
    const double* seedF;   // 9*L      dL/d(stored fluid state) at the final step (natural order), or nullptr
    float* qf;             // 9*L      adjoint planes of step t (output), FP32
    float* qg;             // S*5*L
    const double* force;   // 2*L      spread force field (zero outside the force tiles)
    const uint32_t* dom;
    const double* massTab; // per-domain rhoToAdd, or nullptr
    int nDomains;
    const double* srcTab;  // [S][nDomains]
    double tauIF;              // 1 / tauFluid
    double tauI[kMaxSpecies];  // 1 / tau of each species
    SpeciesConst sp[kMaxSpecies];
    unsigned iteration;    // iteration counter during step t
    int outlet;
    int chained;           // the previous launch on the stream is an adjoint step of the same pass
                           // (programmatic launch); 0: a plain launch after whatever came before
    double* G;             // 2*L      dL/dF(x), summed over steps
    double* racc;          // S*L      dL/d source at each node, summed over steps
    double* macc;          // L        dL/d rhoToAdd at each node, summed over steps (with massTab)
    double* part;          // adjoint_blocks * (1 + S): per-block relaxation-time partials
    double* grad;          // 1 + S + S*nDomains + nDomains (written by launch_adjoint_finish)
    // moving-membrane runs only (the kernel is launched in its motion form):
    const double* gu;      // 2*L      dL/d(post-collision velocity) of step t
    double* uo;            // 2*L      the post-collision velocity of step t (output)
};
void launch_adjoint_step64(const AdjointArgs& a, cudaStream_t s);
// The same step in its motion form (a.gu, a.uo; G overwritten), a plain launch.
void launch_adjoint_step64_motion(const AdjointArgs& a, cudaStream_t s);
// Converts n doubles to floats (the force field of an FP32-shifted run).
void launch_to_float(const double* in, float* out, size_t n, cudaStream_t s);
// Thread blocks of one adjoint launch (the rows of AdjointArgs::part).
int adjoint_blocks(int nx, int ny);
// Reduces the per-block and per-node partials into grad.
void launch_adjoint_finish(const AdjointArgs& a, cudaStream_t s);
void launch_set_iteration(Status* st, unsigned it, cudaStream_t s);

// Transpose of the spread under fixed positions: gf[i] = sum over node i's 16
// stencil slots of dirac * G(x) (k_membrane.cu).
void launch_force_adjoint(const MembraneDev& m, const double* G, int nx, int ny, size_t L, double* gfx,
                          double* gfy, cudaStream_t s);

// Differentiated runs with moving membrane nodes (k_membrane.cu).  The
// stencil of each node follows from its position at the step (the 4x4
// lattice nodes within 2 lu), its weights are calculateDiscreteDeltaDirac's.
// out[n] += dirac(x_n - X_i) * (ax_i, ay_i) over every node's stencil (FP64
// atomics: the spread of the node forces, or of dL/dX onto dL/du).
void launch_motion_spread(const double* X, const double* Y, const double* ax, const double* ay, int M, int nx,
                          int ny, size_t L, double* out, Status* st, cudaStream_t s);
// X1 = X0 + the velocity interpolated from u at X0 (GeometryNode::collectVelocity
// then move, GeometryNode.cpp:216-226, 245-254, without the perturbation).
template <typename Real>
void launch_motion_move(const double* X0, const double* Y0, double* X1, double* Y1, int M, const Real* u, int nx,
                        int ny, size_t L, Status* st, cudaStream_t s);
// Reverse of one step's spread, interpolation and move for node i at its
// step-start position X: with lambda = dL/dX_after,
//   lambda += sum_n grad_X dirac * (lambda . uo(n) + F_i . G(n)),
//   gF_i   += sum_n dirac * G(n),
// G = dL/d(force field) of the step, uo its post-collision velocity.
void launch_motion_adjoint(const double* X, const double* Y, const double* fx, const double* fy, double* lx,
                           double* ly, const double* uo, const double* G, double* gfx, double* gfy, int M, int nx,
                           int ny, size_t L, cudaStream_t s);

// Opt-in shared-memory sizes of the kernels that need more than 48 KB; called
// once before any launch (and so before any stream capture).
void init_kernel_attributes();
void init_kernel_attributes_topology();

}  // namespace lbib
