/* lbibcell.h — C ABI of the lbibcell_b200 device runtime (liblbibcuda.so).
 *
 * One handle owns one simulation: the lattice (D2Q9 fluid + up to three D2Q5
 * species), the membrane (immersed-boundary nodes and connections), the force
 * list and the registered mass/bio solvers, all resident on one GPU.  Host
 * code (the Python mirror in lbibcell_b200/, or a C++ host) drives it through
 * these calls.  All calls return 0 or an LBIB_ERR_* code and never throw or
 * abort across the ABI; lbib_last_error() gives the message and the index of
 * the node or connection involved.  The caller owns every host buffer; the
 * handle owns every device buffer.  A handle uses one CUDA stream and is not
 * thread-safe.
 *
 * The comment of each call names the reference interface it replaces (paths
 * relative to the LBIBCell project root).
 */
#ifndef LBIBCELL_H
#define LBIBCELL_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbib_handle lbib_handle;

/* Precision of the lattice. */
#define LBIB_FP64 0          /* plain: bit-identical to the reference's double run */
#define LBIB_FP32_SHIFTED 1  /* FP32 storage of f - w (deviation from rest), FP32 collision */

/* Error codes. */
#define LBIB_OK 0
#define LBIB_ERR_EDGE_W 10        /* "geometry point moved too close to the west boundary" */
#define LBIB_ERR_EDGE_S 11
#define LBIB_ERR_EDGE_E 12
#define LBIB_ERR_EDGE_N 13
#define LBIB_ERR_SPEED 20         /* membrane speed^2 > CS (LagrangianPoint.cpp:96-102) */
#define LBIB_ERR_LEFT_DOMAIN 30   /* "domainID at the left boundary must be 0." */
#define LBIB_ERR_VERTICAL 40      /* non-finite connection slope (Connection.cpp:315-323) */
#define LBIB_ERR_FORCE_NODE 50    /* force refers to a missing node (ForceStructs.hpp) */
#define LBIB_ERR_STENCIL 60       /* membrane node stencil leaves the lattice */
#define LBIB_ERR_CAPACITY 70      /* a per-step device list overflowed */
#define LBIB_ERR_CUDA 80          /* CUDA runtime error */
#define LBIB_ERR_INPUT 90         /* bad file or argument */
#define LBIB_ERR_STATE 91         /* call not valid in the handle's state */

/* Creates a simulation from the reference's own text files (parameter,
 * geometry and force files) plus the plugin file that names the mass/bio
 * solvers and species parameters (format: lbibcell_b200/configs.py).
 * Replaces the set-up of apps/tutorial_01.cpp:59-143:
 *   Parameters.loadGlobalSimulationParameters  (GlobalSimulationParameters.cpp:34-72)
 *   geometry::Geometry(file) txt loader        (Geometry.cpp:99-160)
 *   geometry::GeometryHandler(geo)             (GeometryHandler.cpp:51-56, cureLattice :149-170)
 *   SimulationRunner(geohandler, reporter)     (SimulationRunner.cpp:50-64)
 *   SimulationRunner::initSolvers()            (SimulationRunner.cpp:290-306)
 *   SimulationRunner::initForceSolver(file)    (SimulationRunner.cpp:392-394)
 *   SimulationRunner::addMassSolver / addBioSolver (SimulationRunner.cpp:401-408)
 * `device` is the CUDA device ordinal. */
int lbib_create_from_files(const char* parameters, const char* geometry, const char* force, const char* plugins,
                           int precision, int device, lbib_handle** out);

/* Releases every device and host resource of the handle. */
int lbib_destroy(lbib_handle* h);

/* Advances n time steps: the body of SimulationRunner::runSimulation
 * (SimulationRunner.cpp:72-99) — force evaluation, spreading, fused
 * stream-collide of fluid and species, interpolation and motion, crossings,
 * domain ids and species reinitialisation, remeshing, coarsening every 10
 * iterations, mass solvers, bio solvers.  Returns after the GPU finished. */
int lbib_step(lbib_handle* h, int n);

/* Lattice-only steps with the geometry held fixed: pull-stream + collide of
 * fluid and species (FluidSolver/CDESolver advect+collide), then the box
 * outlet when `outlet` is non-zero.  The force field, domain ids and mass
 * sources stay as they are.  Stage-level parity and bandwidth measurement. */
int lbib_lattice_step(lbib_handle* h, int n, int outlet);

/* sizes[0..9] = nx, ny, S, M (membrane nodes), C (connections), iteration,
 * precision, host interventions (perturbation/remesh/coarsen), steps done,
 * number of cells. */
int lbib_get_sizes(lbib_handle* h, long long* sizes);

/* Lattice state in the reference's layout (SimulationRunner::writeSimulation's
 * solver dump order, SimulationRunner.cpp:112-149): f[L][9] and g[S][L][5]
 * in the slot convention after FluidSolver::localSwap, vel[L][2]
 * (FluidSolver::velocity_), force[L][2] (FluidSolver::force_), dom[L]
 * (PhysicalNode::domainIdentifier_), ctype[L] (PhysicalNode::cellType_).
 * Any pointer may be NULL.  FP32-shifted state is converted to f = h + w. */
int lbib_download_lattice(lbib_handle* h, double* f, double* g, double* vel, double* force, unsigned* dom,
                          unsigned* ctype);

/* Overwrites the distributions (reference slot layout) and, if non-NULL, the
 * spread force field.  Replaces SimulationRunner::initSolvers(file)
 * (SimulationRunner.cpp:151-182) for restarts and stage-level tests. */
int lbib_upload_lattice(lbib_handle* h, const double* f, const double* g, const double* force);

/* SimulationRunner::initSolvers(Field<double>) (SimulationRunner.cpp:308-320):
 * every node's fluid at the equilibrium of density 1 and the uniform
 * velocity (ux, uy) (FluidSolver::setVelocity + initWithVelocity,
 * FluidSolver.cpp:62-101, 233-240), its stored velocity set to (ux, uy),
 * then each CDE solver's initSolver (which collides at that velocity).
 * Replaces the lattice state; the membrane and force list are unchanged. */
int lbib_init_velocity(lbib_handle* h, double ux, double uy);

/* Membrane nodes in ascending id order (Geometry::getGeometryNodes):
 * ids[M], state[M][6] = x, y, vx, vy, fx, fy. */
int lbib_download_membrane(lbib_handle* h, unsigned* ids, double* state);

/* Connections in Geometry::getConnections order: conn[C][3] = id1, id2, domain. */
int lbib_download_connections(lbib_handle* h, unsigned* conn);

/* Cell areas (GeometryHandler::computeAreas, GeometryHandler.cpp:101-134):
 * dom[k], area[k] for k < return value (capped at cap).  FP64 handles sum each
 * ring in the reference's order; FP32-shifted handles sum each shoelace term
 * rounded to 2^-24 in any order (exact, so deterministic; at most n 2^-26 from
 * the ring-order sum for a cell of n nodes).  Right after lbib_step with an
 * area regulator registered, the areas its bio stage formed were read back
 * with the step's status word and the call does no device work.  Negative on
 * error: -LBIB_ERR_CAPACITY (the handle stays usable) when, on an FP64
 * handle, a cell's ring holds more than 4096 membrane nodes, the most one
 * ring sum takes. */
int lbib_areas(lbib_handle* h, unsigned* dom, double* area, int cap);

/* The same cell areas as lbib_areas, computed without any allocation: no
 * cudaMalloc, no host heap.  No counterpart in the reference.  For callers
 * that must not allocate while a run is under way, such as a host that
 * reserved the device memory for itself, or a tight per-step loop where an
 * allocator call (and the synchronisation it can bring) is not acceptable.
 * The per-cell sums go to one fixed array in device memory of 16384 doubles
 * (128 KB); a simulation with more cells is rejected with
 * -LBIB_ERR_CAPACITY, its message readable by lbib_last_error, and the
 * handle stays usable.  Every call on a device, from any handle, shares
 * that one array: each call first sets the entries it will read to NaN, so
 * no value of an earlier call can come back, but calls that overlap in time
 * (two threads, or two handles on different streams) race on it and must be
 * serialised by the caller.  A cell whose ring holds more than 4096 nodes
 * gives -LBIB_ERR_CAPACITY on an FP64 handle, with the cell's index in
 * lbib_last_error (the handle stays usable; area[] may then hold NaN).  The first call on a
 * device looks up the array's address; make that call before any stream
 * capture.  Returns the number of cells, as lbib_areas. */
int lbib_areas_static(lbib_handle* h, unsigned* dom, double* area, int cap);

/* GeometryHandler::computeAccumulatedDomainConcentrations(species)
 * (libs/LbmLib/src/geometry/GeometryHandler.cpp:136-147): per domain id
 * (ascending), the sum of the named CDE solver's concentration over the
 * lattice nodes of that domain, rows in order and columns from x = 1 (the
 * reference leaves column 0 out).  Returns the number of domains, or the
 * negated error code (LBIB_ERR_INPUT for an unknown species,
 * LBIB_ERR_CAPACITY when cap is too small). */
int lbib_accumulated_concentrations(lbib_handle* h, const char* species, unsigned* dom, double* acc, int cap);

/* GeometryHandler::getCellTypeTrackerMap()[dom[i]] = type[i] for n entries,
 * then copyCellTypeToPhysicalNodes (GeometryHandler.cpp:267-314): the
 * lattice nodes of those domains take the new types from the next step on
 * (a bio solver that reads them in the same step sees them at once). */
int lbib_set_cell_types(lbib_handle* h, const unsigned* dom, const unsigned* type, int n);

/* GeometryHandler::getCellTypeTrackerMap (GeometryHandler.cpp:316-319): the
 * cell type of every domain id below the handle's domain count.  Returns the
 * count, or the negated error code. */
int lbib_get_cell_types(lbib_handle* h, unsigned* dom, unsigned* type, int cap);

/* Sets species k's production rate per domain id (rates[0..n), n <= number of
 * domain ids), taking effect at the next step.  This is the per-domain table
 * that a host BioSolver plugin would otherwise write node by node through
 * CDESolver state (e.g. tutorial_01_CDESolverD2Q5_SIGNAL.cpp:92-100, where the
 * production depends on the node's domain id). */
int lbib_set_species_source(lbib_handle* h, int k, const double* rates, int n);

/* The same for every species at once, in one host-to-device copy:
 * rates[k * n + d] for species k (parameter-file order) and domain id d,
 * n = lbib_get_domain_count. */
int lbib_set_species_sources(lbib_handle* h, const double* rates, int n);

/* Writes the simulation in the reference's four text formats, as
 * SimulationRunner::writeSimulation does (SimulationRunner.cpp:112-149):
 * the force list (ForceSolver::writeForceSolver, ForceSolver.cpp:141-156),
 * the geometry (Geometry::writeGeometry, Geometry.cpp:77-95), the global
 * parameters with the current iteration (GlobalSimulationParameters.cpp:74-97)
 * and the solver dump (distributions per node, rows y then x, in the stored
 * slot order).  Numbers are written with 17 significant digits, so a restart
 * from these files continues with the same values; the reference's loaders
 * read them unchanged.  Any file name may be NULL or empty to skip it. */
int lbib_write_simulation(lbib_handle* h, const char* forceFile, const char* geometryFile, const char* parameterFile,
                          const char* solverFile);

/* Loads the distributions of a solver dump (SimulationRunner::initSolvers(file),
 * SimulationRunner.cpp:151-182) into the lattice: the nodes the file lists take
 * its values, the others keep theirs.  With lbib_create_from_files on the
 * written parameter, geometry and force files this restarts a run, from a
 * dump of this library or of the reference. */
int lbib_load_solvers(lbib_handle* h, const char* solverFile);

/* Number of domain ids (rows of the per-domain source and mass tables). */
int lbib_get_domain_count(lbib_handle* h, int* n);

/* Differentiated runs (no counterpart in the reference).  An FP64 handle
 * runs them in FP64; an FP32-shifted handle runs the forward steps in its
 * FP32 kernel and stores the checkpoints in FP32 (half the memory), while the
 * reverse step computes in FP64 from those states and the parameter
 * gradients accumulate in FP64.
 *
 * A differentiated run advances the lattice T steps with the geometry frozen
 * (unless lbib_diff_motion moves the nodes) at its state when lbib_diff_begin
 * is called: the membrane positions (so the
 * Dirac weights of the spread), the domain ids and the per-domain mass table
 * stay fixed, exactly as in lbib_lattice_step.  Each step is the pull-stream
 * + collide of the fluid (Luo force) and the species (with their reaction),
 * then the box outlet when enabled.  Its parameters are the membrane node
 * forces F_i (spread once into the force field), the relaxation times
 * (tauFluid and each species' tau) and the per-domain production rates of the
 * linear-source species.  The reverse pass gives the gradients of a scalar
 * loss L of the final concentrations C_k(x) = sum of species k's five
 * distributions, from the caller's dL/dC_k(x).
 *
 * lbib_diff_begin snapshots the current lattice as the run's initial state
 * and allocates the checkpoints: one state every K steps (K <= 0 picks
 * ceil(sqrt(T))) plus K-1 states of the segment being reversed; each state is
 * (9 + 5 S) * Nx * Ny values of the lattice precision.  The defaults of the parameters are the
 * handle's: the membrane forces of the last force evaluation, the relaxation
 * times and source rates of the files. */
int lbib_diff_begin(lbib_handle* h, int T, int K);

/* Runs the T forward steps from the snapshot, storing the checkpoints.
 * memForce[M][2] (node order of lbib_download_membrane), tau[1 + S]
 * (tauFluid, then the species in parameter-file order) and rates[S][n_domains]
 * replace the current parameters when non-NULL and stay in effect for later
 * calls.  outlet != 0 applies the box outlet after each step.  The final state
 * and the spread force field become the handle's lattice
 * (lbib_download_lattice). */
int lbib_diff_forward(lbib_handle* h, const double* memForce, const double* tau, const double* rates, int outlet);

/* Reverse pass of the last lbib_diff_forward: recomputes each segment of K
 * steps from its checkpoint and runs the adjoint steps backwards.  dLdC[S][L]
 * (L = Nx * Ny, node y * Nx + x) is dL/dC_k(x) at the final step.  Outputs
 * (any may be NULL): gForce[M][2] = dL/dF_i, gTau[1 + S] = dL/dtau,
 * gRates[S][n_domains] = dL/d rate (zero for species without a linear source).
 * Per-domain and relaxation-time gradients are sums of atomic adds: their
 * last bits can differ between calls. */
int lbib_diff_backward(lbib_handle* h, const double* dLdC, double* gForce, double* gTau, double* gRates);

/* The per-domain mass source as a parameter of a differentiated run: the
 * rhoToAdd that FluidSolver::addMass sets (FluidSolver.cpp:141-145, 196-257)
 * and the collide adds to the density, frozen for the run (the area
 * regulator's rates of the last step, or none).  mass[n], when non-NULL,
 * replaces that table for the following lbib_diff_forward calls (a run
 * without an area regulator then gets one); gMass[n], when non-NULL,
 * receives dL/d mass[d] of the last lbib_diff_backward (zeros when the run
 * has no mass table).  n must be the domain count (lbib_get_domain_count).
 * With frozen cell areas an area regulator's rate is linear in its strength
 * below the clamp, so dL/d strength = dL/d mass times the rate's factor. */
int lbib_diff_mass(lbib_handle* h, const double* mass, double* gMass, int n);

/* dL/d of the final fluid distributions, dLdf[L][9] in lbib_download_lattice's
 * layout, joined to the species' seed of the following lbib_diff_backward
 * calls (for a loss of the flow, such as its kinetic energy); NULL removes
 * it.  Must be called after lbib_diff_begin. */
int lbib_diff_fluid_seed(lbib_handle* h, const double* dLdf);

/* dL/d of the force records' parameters, through the node forces
 * (ForceSolver::calculateForce, ForceSolver.cpp:42-85 with the forces of
 * ForceStructs.hpp:49-588): after lbib_diff_backward, with its dL/dF_i and
 * the handle's current records and positions.  Each record adds to its own
 * node's force only, so dL/dp = dL/dF_i . dF_i/dp.  gPar[4 r + q] for record
 * r (lbib_download_forces' order) and parameter q (lbib_add_forces' meaning;
 * 0 for parameters the type does not read; the spring's k and l0, the
 * anchor's x, y, k, l0, the constant force, the slider's position, k, l0 and
 * the tension's f).  The gradient is that of the run's loss when the run's
 * node forces are these records' forces (memForce of lbib_diff_forward, or
 * the default when the records did not change since the last force
 * evaluation).  Returns the record count (fills min(count, cap) records) or
 * a negative LBIB_ERR_*. */
int lbib_diff_force_params(lbib_handle* h, double* gPar, int cap);

/* Differentiated runs with moving membrane nodes (the adjoint of
 * GeometryNode::collectVelocity + move, GeometryNode.cpp:216-226, 245-254;
 * no counterpart in the reference).  on != 0, after lbib_diff_begin, makes
 * every following lbib_diff_forward move the nodes: step t spreads the node
 * forces F_i from the positions after step t-1, runs the lattice step, and
 * moves each node by the post-collision velocity interpolated at those
 * positions.  The stencil of a node is the 4x4 lattice nodes within 2 lu of
 * its position at the step; the perturbation of nodes on lattice lines
 * (GeometryNode.cpp:155-214) is left out (its random jumps have no
 * derivative).  The domain ids, the boundary nodes and the mass table stay
 * those of lbib_diff_begin.  The positions of every step are stored:
 * (T + 1) * M * 16 bytes more device memory.  dLdX[M][2], when non-NULL, is
 * dL/dX of the final positions (a loss of the membrane's shape), joined to
 * dLdC in lbib_diff_backward; the reverse pass then also carries dL/dX back
 * through each step (the Dirac weights' derivative included), its gForce is
 * dL/dF_i through both the lattice and the motion, and lbib_diff_positions
 * gives dL/dX at the start.  Spreads use FP64 atomic adds: the last bits of
 * the fields can differ between calls.  lbib_diff_force_params is refused in
 * such a run.  on = 0 switches the motion off again. */
int lbib_diff_motion(lbib_handle* h, int on, const double* dLdX);

/* Of a run with moving nodes: xT[M][2] = the positions after the last
 * lbib_diff_forward's final step, gX0[M][2] = dL/dX of the positions at the
 * start from the last lbib_diff_backward (either may be NULL).  n must be the
 * node count M. */
int lbib_diff_positions(lbib_handle* h, double* xT, double* gX0, int n);

/* Restores the snapshot taken by lbib_diff_begin (distributions, velocity and
 * force planes) and frees the run's device memory. */
int lbib_diff_end(lbib_handle* h);

/* The ForceSolver's records in the device's order: by node (ascending id),
 * each node's records in insertion order (forcemap_[id] order, ForceSolver.cpp:
 * 42-85).  type[r], id1[r] (the node), id2[r] (the partner's id for types 0,
 * 5, 6, 7; 0 otherwise), par[4 r .. 4 r + 3] as lbib_add_forces takes them.
 * Returns the record count (fills min(count, cap)) or a negative LBIB_ERR_*. */
int lbib_download_forces(lbib_handle* h, int* type, unsigned* id1, unsigned* id2, double* par, int cap);

/* ForceSolver::addForce for n records at once (ForceSolver.cpp:107-139), in
 * place of one text line each.  Record k has type[k] (0-7, ForceStructs.hpp),
 * node id1[k], for types 0, 5, 6, 7 the partner node id2[k] (id2 may be NULL
 * when no record needs one) and four parameters par[4k..4k+3]:
 *   0, 7  k, l0            1  x, y, k, l0      2  fx, fy
 *   3, 4  position, k, l0  5, 6  f             (unused ones are ignored)
 * Each node's new records follow its existing ones in call order, as
 * forcemap_[id1].push_back does.  An unknown node id fails with
 * LBIB_ERR_FORCE_NODE (the reference fails when the force is next evaluated,
 * ForceStructs.hpp "Could not compute and set the forces.").  The records stay
 * until a deleteForceType of their type or the deleteAllForces of every 10th
 * iteration (SimulationRunner.cpp:84-87), as in the reference. */
int lbib_add_forces(lbib_handle* h, const int* type, const unsigned* id1, const unsigned* id2, const double* par,
                    int n);

/* ForceSolver::deleteForceType (ForceSolver.cpp:183-215): removes every record
 * of that type, keeping the others in order. */
int lbib_delete_force_type(lbib_handle* h, int type);

/* ForceSolver::deleteAllForces (ForceSolver.cpp:170-181). */
int lbib_delete_all_forces(lbib_handle* h);

/* The membrane after a host bio solver's topology edits between steps (a cell
 * division, growth): Geometry::addGeometryNode / removeGeometryNode /
 * addConnection / eraseConnection (Geometry.cpp:381-452), given as the
 * resulting lists.  ids[M] ascend; xy[2M] are the positions; conns[3C] hold
 * (id1, id2, domain) per connection in vector order, each closed ring one
 * cell.  Nodes that existed keep their velocity, force and old position; new
 * ones start as a new GeometryNode does (perturbed, GeometryNode.cpp:98-117,
 * at rest).  Force records of removed nodes, or toward them, are dropped; the
 * others keep their order.  A connection keeps its boundary descriptor when
 * one with the same (id1, id2) existed, else has none.  New domain ids get
 * cell type 1 and no species production (lbib_set_species_source sets it).
 * Domain ids of the lattice follow at the next step's crossings, or at once
 * after lbib_cure_lattice, as after the reference plugin's cureLattice. */
int lbib_upload_membrane(lbib_handle* h, const unsigned* ids, const double* xy, int M, const unsigned* conns,
                         int C);

/* GeometryHandler::cureLattice (GeometryHandler.cpp:149-170), which a host
 * plugin calls after its topology edits (tutorial_01_BioSolverCellDivision.cpp
 * :84): perturbConnections, the edge test of every node, new boundary nodes,
 * and every lattice node's domain id set at once (no species
 * re-initialisation, as in the reference). */
int lbib_cure_lattice(lbib_handle* h);

/* Geometry::getGeometryNodesWithinRadius (Geometry.cpp:306-323), or with
 * avoidDomain >= 0 getGeometryNodesWithinRadiusWithAvoidance (:325-348): the
 * ids of the membrane nodes within `radius` of (x, y) (distance <= radius),
 * leaving out nodes whose adjacent connections carry domain avoidDomain, in
 * the order of the reference's cell list (1-lu bins by row, then column,
 * ascending id within a bin; FastNeighborList.hpp:400-444, 494-520).  Writes
 * up to cap ids; returns the number of hits, or a negated LBIB_ERR_* code. */
int lbib_nodes_within_radius(lbib_handle* h, double x, double y, double radius, long long avoidDomain,
                             unsigned* ids, int cap);

/* Geometry::getGeometryNodesWithinRadiusWithAvoidanceClosest
 * (Geometry.cpp:350-374) for n query points at once: closest[q] = the id of the
 * first hit of smallest distance in the order above, or -1 when none.
 * avoidDomain may be NULL (no domain left out) or hold one domain per query. */
int lbib_closest_nodes(lbib_handle* h, const double* x, const double* y, const long long* avoidDomain, int n,
                       double radius, long long* closest);

/* VTK output without VTK: the block that vtkCellReporter (cells: polygons of
 * the membrane with domain_identifier, cell_type, boundarydescriptors),
 * vtkForceReporter (forces: a line per force with a partner, ForceType),
 * vtkCDEReporter (one concentration array per CDE solver, by name) or
 * vtkFluidReporter (density, velocity) adds, appended to
 * <prefix>_<time>.vtm with the block in <prefix>_<time>/<prefix>_<time>_<k>.vt?
 * (vtkCellReporter.cpp, vtkForceReporter.cpp, vtkCDEReporter.cpp,
 * vtkFluidReporter.cpp; VTK XML in ASCII mode, as the reference writes it).
 * `coarsening` is the grid reporters' coarsening factor (1 = every node).
 * LBIB_VTK_CELL_PNG (vtkCellPNGReporter) needs a graphics stack and writes
 * nothing.  A geometry file ending in ".vtm" given to lbib_create_from_files
 * is read like Geometry::loadGeometryVTK (Geometry.cpp:162-306). */
#define LBIB_VTK_CELLS 1
#define LBIB_VTK_FORCES 2
#define LBIB_VTK_CDE 3
#define LBIB_VTK_FLUID 4
#define LBIB_VTK_CELL_PNG 5
int lbib_write_vtk(lbib_handle* h, const char* prefix, unsigned time, int kind, int coarsening);

/* Reads a .vtm geometry as Geometry::loadGeometryVTK does, on the host only
 * (no GPU, no handle): counts[0] nodes (ids 0..n-1, positions xy[2n] before
 * GeometryNode's perturbation) and counts[1] connections (id1, id2, domain
 * per connection).  Up to capNodes / capConns entries are written. */
int lbib_read_vtm_geometry(const char* path, unsigned* ids, double* xy, int capNodes, unsigned* conns,
                           int capConns, int* counts);

/* Last error: code; message into buf; index of the node/connection involved. */
int lbib_last_error(lbib_handle* h, char* buf, int len, long long* index);

/* Timing of the last lbib_step / lbib_lattice_step call measured with CUDA
 * events on the handle's stream: out[0] = total ms, out[1] = ms in the
 * stream-collide kernel (summed over steps, when profiling is on), out[2] =
 * stream-collide launches timed, out[3] = kernels launched in total. */
int lbib_last_timing(lbib_handle* h, double* out);

/* Enables or disables per-kernel timing of the stream-collide kernel. */
int lbib_set_profiling(lbib_handle* h, int on);

#ifdef __cplusplus
}
#endif

#endif /* LBIBCELL_H */
