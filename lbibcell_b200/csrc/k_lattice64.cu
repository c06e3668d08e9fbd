// k_lattice64.cu — FP64 (plain) lattice kernels.  Compiled with --fmad=false:
// the results are bit-identical to the reference's double-precision run.
//
//   stream_collide64  fused pull streaming + D2Q9 BGK/Luo collision + S D2Q5
//                     species with reaction.  Replaces FluidSolver::advect/collide
//                     and CDESolver*::advect/collide (SimulationRunner.cpp:244-288).
//                     Pull streaming f_q(x) <- f*_q(x - c_q) on the periodic
//                     lattice (GeometryHandler.cpp:476-589) is the same
//                     permutation as the reference's swap scheme
//                     (FluidSolver.cpp:185-194, 259-264).
//   outlet64          MassSolverBoxOutlet::calculateMass (MassSolverBoxOutlet.cpp:42-72).
//   init64            SimulationRunner::initSolvers (SimulationRunner.cpp:290-306).
#include "lattice_math.cuh"
#include "kernels.cuh"

namespace lbib {

// NS = number of species (a.S), a compile-time constant so that the pulled
// species values stay in registers.  MODE bit 0 (COUPLED): some species'
// reaction reads a partner species or the cell type (the partner's getC() is
// its pre-collide sum while it has not collided at this node, its
// post-collide sum after).  MODE bit 1 (MASSNODE): per-node mass source.
// MODE bit 2 (GUO): GuoZhengShi2002ForceModel in place of Luo1993ForceModel
// (it reads the node's stored velocity before overwriting it).  MODE bit 3
// (BOUNCE): species whose advect keeps the populations of links with a
// boundary node (DiracD2Q5::advect, DiracD2Q5.cpp:166-180): the swap with the
// W (S) neighbour is skipped when the node has a W (S) boundary node, so the
// node's own opposite population stays.
template <int NS, int MODE>
__global__ void __launch_bounds__(256) stream_collide64(LatticeArgs<double> a) {
    constexpr bool COUPLED = (MODE & 1) != 0;   // coupled species reactions
    constexpr bool MASSNODE = (MODE & 2) != 0;  // per-node mass source
    constexpr bool GUO = (MODE & 4) != 0;       // Guo force model
    constexpr bool BOUNCE = (MODE & 8) != 0;    // a DiracD2Q5 species (bounce-back at boundary links)
    pdl_wait();
    if (a.status->halt) return;
    // grid (nx/256, ny): one lattice node per thread
    const int nx = a.nx, ny = a.ny;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nx) return;
    const int y = blockIdx.y;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const size_t L = a.L;
    const unsigned rC = (unsigned)y * nx, rM = (unsigned)ym * nx, rP = (unsigned)yp * nx;
    const unsigned n = rC + x;
    const double* fin = a.fin;
    double f[9];
    f[T] = fin[0 * L + rC + x];
    f[E] = fin[1 * L + rC + xm];
    f[N] = fin[2 * L + rM + x];
    f[W] = fin[3 * L + rC + xp];
    f[S] = fin[4 * L + rP + x];
    f[NE] = fin[5 * L + rM + xm];
    f[NW] = fin[6 * L + rM + xp];
    f[SW] = fin[7 * L + rP + xp];
    f[SE] = fin[8 * L + rP + xm];

    const uint32_t dom = a.dom[n];
    double rta = 0.0;
    if (MASSNODE) rta = a.massNode[n];
    else if (a.massTab != nullptr && dom < (uint32_t)a.nDomains) rta = a.massTab[dom];
    double fx = 0.0, fy = 0.0;
    if (a.tileCount[(y / kTile) * a.tilesX + (x / kTile)] > 0) {
        fx = a.force[n];
        fy = a.force[L + n];
    }
    double ux, uy;
    if (GUO) collide_fluid64_guo(f, rta, fx, fy, a.tauF, a.u[n], a.u[L + n], guo_ne_y(a.forceModel), ux, uy);
    else collide_fluid64(f, rta, fx, fy, a.tauF, ux, uy);
    a.u[n] = ux;
    a.u[L + n] = uy;
    // MassSolverBoxOutlet (MassSolverBoxOutlet.cpp:42-72) on the x=0 column and
    // the y=0 row: fused here because no later stage of the step touches those
    // nodes (membrane nodes keep 2 lu from the edges, GeometryHandler.cpp:618-636).
    // The corner is rescaled twice, as the column pass and then the row pass do.
    const int passes = a.outlet ? (x == 0) + (y == 0) : 0;
    double sc[2] = {1.0, 1.0};
    for (int p = 0; p < passes; ++p) {
        // rho in the reference's slot order after localSwap: T, W, S, E, N, SW, SE, NE, NW
        double rho = 0.0;
        rho += f[T]; rho += f[W]; rho += f[S]; rho += f[E]; rho += f[N];
        rho += f[SW]; rho += f[SE]; rho += f[NE]; rho += f[NW];
        sc[p] = 1.0 / rho;
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] *= sc[p];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) a.fout[q * L + n] = f[q];

    double gAll[NS > 0 ? NS : 1][5];
    uint8_t bW = 0, bWe = 0, bS = 0, bSn = 0;  // W / S boundary nodes here, at the E and N neighbours
    if (BOUNCE) {
        bW = a.bounceW[n];
        bWe = a.bounceW[rC + xp];
        bS = a.bounceS[n];
        bSn = a.bounceS[rP + x];
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const double* gin = a.gin + (size_t)k * 5 * L;
        gAll[k][T] = gin[0 * L + rC + x];
        if (BOUNCE && a.sp[k].bounce) {
            gAll[k][E] = bW ? gin[3 * L + n] : gin[1 * L + rC + xm];
            gAll[k][N] = bS ? gin[4 * L + n] : gin[2 * L + rM + x];
            gAll[k][W] = bWe ? gin[1 * L + n] : gin[3 * L + rC + xp];
            gAll[k][S] = bSn ? gin[2 * L + n] : gin[4 * L + rP + x];
        } else {
            gAll[k][E] = gin[1 * L + rC + xm];
            gAll[k][N] = gin[2 * L + rM + x];
            gAll[k][W] = gin[3 * L + rC + xp];
            gAll[k][S] = gin[4 * L + rP + x];
        }
    }
    // the species' getC() as a coupled reaction reads it, and the node's cell
    // type (copied from the per-domain table after every step's move)
    double Cs[NS > 0 ? NS : 1];
    uint32_t ctype = 0;
    if (COUPLED) {
#pragma unroll
        for (int k = 0; k < NS; ++k) Cs[k] = sum5(gAll[k]);
        if (a.status->cellTypesCopied) ctype = dom < (uint32_t)a.nDomains ? a.ctypeTab[dom] : 1u;
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        double* g = gAll[k];
        double src = 0.0;
        if (a.srcTab != nullptr && dom < (uint32_t)a.nDomains) src = a.srcTab[(size_t)k * a.nDomains + dom];
        double Cp = 0.0;
        if (COUPLED) {
#pragma unroll
            for (int j = 0; j < NS; ++j)
                if (a.sp[k].partner == j) Cp = Cs[j];
        }
        collide_cde64<COUPLED>(g, ux, uy, a.sp[k], src, Cp, dom, ctype, a.status->iteration);
        if (COUPLED) Cs[k] = sum5_swapped(g);
        for (int p = 0; p < passes; ++p)
#pragma unroll
            for (int q = 0; q < 5; ++q) g[q] *= sc[p];
        double* gout = a.gout + (size_t)k * 5 * L;
#pragma unroll
        for (int q = 0; q < 5; ++q) gout[q * L + n] = g[q];
    }
}

// Column x=0 (all y) then row y=0 (all x); the corner (0,0) is rescaled
// twice, first by the column pass.  rho is summed in the reference's slot
// order after FluidSolver::localSwap: T, W, S, E, N, SW, SE, NE, NW.
__device__ __forceinline__ void rescale_node64(double* f, double* g, int nS, size_t L, size_t n) {
    const int order[9] = {Dir::T, Dir::W, Dir::S, Dir::E, Dir::N, Dir::SW, Dir::SE, Dir::NE, Dir::NW};
    double rho = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) rho += f[(size_t)order[i] * L + n];
    const double sc = 1.0 / rho;
#pragma unroll
    for (int q = 0; q < 9; ++q) f[(size_t)q * L + n] *= sc;
    for (int k = 0; k < nS; ++k)
#pragma unroll
        for (int q = 0; q < 5; ++q) g[((size_t)k * 5 + q) * L + n] *= sc;
}

__global__ void outlet64(double* f, double* g, int nS, int nx, int ny, size_t L, const Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    // threads [0, ny): column nodes (0, i); thread 0 also runs the corner's
    // row pass after its column pass.  threads [ny, ny + nx - 1): row nodes (x, 0), x >= 1.
    if (i < ny) {
        rescale_node64(f, g, nS, L, (size_t)i * nx);
        if (i == 0) rescale_node64(f, g, nS, L, 0);
    } else if (i < ny + nx - 1) {
        const int x = i - ny + 1;
        rescale_node64(f, g, nS, L, (size_t)x);
    }
}

// FluidSolver::initSolver (f_T = 1, then collide with zero force and mass)
// and the species' initial conditions.  withVel: FluidSolver::initWithVelocity
// at the uniform velocity (vx, vy) (SimulationRunner::initSolvers(Field<double>),
// SimulationRunner.cpp:308-320): the distributions are the equilibrium at
// rho = 1, the stored velocity is (vx, vy), and the species' initSolver
// collides at that velocity.
__global__ void init64(double* f, double* g, double* u, int nS, size_t L, double tauF, const uint32_t* dom,
                       SpeciesConst sp0, SpeciesConst sp1, SpeciesConst sp2, double init0, double init1, double init2,
                       int withVel, double vx, double vy) {
    pdl_wait();
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L) return;
    double fi[9] = {1.0, 0, 0, 0, 0, 0, 0, 0, 0};
    double ux, uy;
    if (withVel) {
        equilibrium_at_velocity64(vx, vy, fi);
        ux = vx;
        uy = vy;
    } else {
        collide_fluid64(fi, 0.0, 0.0, 0.0, tauF, ux, uy);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) f[(size_t)q * L + n] = fi[q];
    u[n] = ux;
    u[L + n] = uy;
    const SpeciesConst sp[3] = {sp0, sp1, sp2};
    const double init[3] = {init0, init1, init2};
    for (int k = 0; k < nS; ++k) {
        double gi[5];
        if (sp[k].kind == RX_NONE) {
            // CDESolverD2Q5::initSolver — CDESolverD2Q5.cpp:37-40
            gi[0] = 1.0; gi[1] = gi[2] = gi[3] = gi[4] = 0.0;
            collide_cde64(gi, ux, uy, sp[k], 0.0, 0.0, dom[n], 0u, 0u);
        } else if (sp[k].kind == RX_SIGNAL) {
            // tutorial_01_CDESolverD2Q5_SIGNAL::initSolver — :46-57
            const double v = dom[n] == 0 ? 0.0 : 1.0 / 5.0;
            for (int q = 0; q < 5; ++q) gi[q] = v;
        } else {
            for (int q = 0; q < 5; ++q) gi[q] = init[k] / 5.0;
        }
        for (int q = 0; q < 5; ++q) g[((size_t)k * 5 + q) * L + n] = gi[q];
    }
}

// The boundary solvers of the boundary nodes recorded by the previous step's
// crossings: BoundarySolverNoFlux(D2Q5)::preAdvect, then postAdvect
// (BoundarySolverNoFlux.cpp:36-105, BoundarySolverNoFluxD2Q5.cpp:37-106), as
// two passes over the (node, slot) list before the stream-collide kernel.
//
// A boundary node in slot d (E, N, W, S) of lattice node n lies between n and
// its neighbour n + c_d; the population it acts on is direction dir =
// inverse(d), which node n pulls from n + c_d.  preAdvect forms, from node n's
// state before the step and the boundary node's velocity, D = feq_b(dir) +
// (g_dir(n) - feq_n(dir)) for the first CDE solver each boundary solver serves
// (its loop returns after that one).  postAdvect then swaps D into the
// post-advect value of direction dir of each served species in turn, so the
// first gets D and each further one the previous one's value.  Pulling makes
// "post-advect value of dir at n" the stored slot (dir, n + c_d), which no
// other node reads: the swap writes there, and the stream-collide kernel pulls
// the result.  The first pass only reads (every D sees the state before any
// swap, as all preAdvects run before the advection); the second only swaps.
template <typename Real>
__global__ void noflux_pre_kernel(LatticeArgs<Real> a) {
    pdl_wait();
    if (a.status->halt) return;
    const int cnt = min(*a.nfN, a.nfCap);
    const size_t L = a.L;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += gridDim.x * blockDim.x) {
        const uint32_t key = a.nfKeys[e];
        const size_t n = key >> 2;
        const int d = (int)(key & 3u) + 1;                             // E, N, W, S
        const int dir = d == E ? W : (d == N ? S : (d == W ? E : N));  // boundary node -> n
        const NfSpec& sp = a.nfTab[a.nfSpec[key] - 1];
        const double ub = a.nfU[2 * (size_t)key], vb = a.nfU[2 * (size_t)key + 1];
        const double uPrevX = a.u[n], uPrevY = a.u[L + n];  // the fluid velocity of the previous step
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if (j >= sp.nSolvers) break;
            const Real* gk = a.gin + (size_t)sp.s[j].cde[0] * 5 * L;
            // CDESolverD2Q5::getC over the stored slots (T, W, S, E, N directions)
            double C = 0.0;
            C += (double)gk[(size_t)T * L + n];
            C += (double)gk[(size_t)W * L + n];
            C += (double)gk[(size_t)S * L + n];
            C += (double)gk[(size_t)E * L + n];
            C += (double)gk[(size_t)N * L + n];
            const bool d2q5 = sp.s[j].kind == NF_NOFLUX_D2Q5;
            const double Cf = d2q5 ? C / 6.0 : C / 4.0;
            const double c3 = d2q5 ? 3.0 : 2.0;
            double feq;
            if (dir == E) feq = Cf * (1 + c3 * ub);
            else if (dir == N) feq = Cf * (1 + c3 * vb);
            else if (dir == W) feq = Cf * (1 - c3 * ub);
            else feq = Cf * (1 - c3 * vb);
            // CDESolverD2Q5::calculateEquilibrium(dir) (CDESolverD2Q5.cpp:109-135)
            const double w1 = C / 6.0;
            double eq;
            if (dir == E) eq = w1 * (1.0 + uPrevX * 3.0);
            else if (dir == N) eq = w1 * (1.0 + uPrevY * 3.0);
            else if (dir == W) eq = w1 * (1.0 + (-uPrevX) * 3.0);
            else eq = w1 * (1.0 + (-uPrevY) * 3.0);
            const double fneq = (double)gk[(size_t)dir * L + n] - eq;
            a.nfD[2 * (size_t)e + j] = feq + fneq;
        }
    }
}

template <typename Real>
__global__ void noflux_post_kernel(LatticeArgs<Real> a) {
    pdl_wait();
    if (a.status->halt) return;
    const int cnt = min(*a.nfN, a.nfCap);
    const size_t L = a.L;
    const int nx = a.nx, ny = a.ny;
    Real* g = const_cast<Real*>(a.gin);  // the current state, before this step's pull
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += gridDim.x * blockDim.x) {
        const uint32_t key = a.nfKeys[e];
        const size_t n = key >> 2;
        const int d = (int)(key & 3u) + 1;
        const int dir = d == E ? W : (d == N ? S : (d == W ? E : N));
        const NfSpec& sp = a.nfTab[a.nfSpec[key] - 1];
        int x = (int)(n % (size_t)nx), y = (int)(n / (size_t)nx);
        if (d == E) x = x == nx - 1 ? 0 : x + 1;
        else if (d == N) y = y == ny - 1 ? 0 : y + 1;
        else if (d == W) x = x == 0 ? nx - 1 : x - 1;
        else y = y == 0 ? ny - 1 : y - 1;
        const size_t from = (size_t)y * nx + x;  // node n pulls direction dir from here
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if (j >= sp.nSolvers) break;
            double cur = a.nfD[2 * (size_t)e + j];
            for (int c = 0; c < sp.s[j].nCde; ++c) {
                Real* slot = g + ((size_t)sp.s[j].cde[c] * 5 + dir) * L + from;
                const double t = (double)*slot;
                *slot = (Real)cur;
                cur = t;
            }
        }
    }
}

template <typename Real>
void launch_noflux(const LatticeArgs<Real>& a, cudaStream_t s) {
    launch_pdl(noflux_pre_kernel<Real>, 296, 256, 0, s, a);
    launch_pdl(noflux_post_kernel<Real>, 296, 256, 0, s, a);
}
template void launch_noflux<double>(const LatticeArgs<double>&, cudaStream_t);
template void launch_noflux<float>(const LatticeArgs<float>&, cudaStream_t);

void launch_stream_collide64(const LatticeArgs<double>& a, cudaStream_t s) {
    const dim3 grid((unsigned)((a.nx + 255) / 256), (unsigned)a.ny);
    if (a.nfTab != nullptr) launch_noflux<double>(a, s);
    const int mode = (a.coupled ? 1 : 0) | (a.massNode != nullptr ? 2 : 0) | (a.forceModel != FM_LUO ? 4 : 0) |
                     (a.bounceW != nullptr ? 8 : 0);
    switch (mode * 4 + (a.S < 3 ? a.S : 3)) {
#define LBIB_SC_CASE(M, N) \
    case M * 4 + N: launch_pdl(stream_collide64<N, M>, grid, 256, 0, s, a); break;
        LBIB_SC_CASE(0, 0) LBIB_SC_CASE(0, 1) LBIB_SC_CASE(0, 2) LBIB_SC_CASE(0, 3)
        LBIB_SC_CASE(2, 0) LBIB_SC_CASE(2, 1) LBIB_SC_CASE(2, 2) LBIB_SC_CASE(2, 3)
        // coupled reactions need a partner species: two or three species
        LBIB_SC_CASE(1, 2) LBIB_SC_CASE(1, 3) LBIB_SC_CASE(3, 2) LBIB_SC_CASE(3, 3)
        // the same with the Guo force model
        LBIB_SC_CASE(4, 0) LBIB_SC_CASE(4, 1) LBIB_SC_CASE(4, 2) LBIB_SC_CASE(4, 3)
        LBIB_SC_CASE(6, 0) LBIB_SC_CASE(6, 1) LBIB_SC_CASE(6, 2) LBIB_SC_CASE(6, 3)
        LBIB_SC_CASE(5, 2) LBIB_SC_CASE(5, 3) LBIB_SC_CASE(7, 2) LBIB_SC_CASE(7, 3)
        // DiracD2Q5 species with the plain fluid (the combination create accepts)
        LBIB_SC_CASE(8, 1) LBIB_SC_CASE(8, 2) LBIB_SC_CASE(8, 3)
#undef LBIB_SC_CASE
        default: break;
    }
}

void launch_outlet64(double* f, double* g, int nS, int nx, int ny, size_t L, const Status* st, cudaStream_t s) {
    const int n = nx + ny;
    launch_pdl(outlet64, (n + 255) / 256, 256, 0, s, f, g, nS, nx, ny, L, st);
}

void launch_init64(double* f, double* g, double* u, int nS, size_t L, double tauF, const uint32_t* dom,
                   const double* vel, const SpeciesConst* sp, const double* init, cudaStream_t s) {
    launch_pdl(init64, (unsigned)((L + 255) / 256), 256, 0, s, f, g, u, nS, L, tauF, dom, sp[0], sp[1], sp[2], init[0],
               init[1], init[2], vel != nullptr ? 1 : 0, vel != nullptr ? vel[0] : 0.0, vel != nullptr ? vel[1] : 0.0);
}

}  // namespace lbib
