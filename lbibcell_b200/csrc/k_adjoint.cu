// k_adjoint.cu — reverse-mode (adjoint) step of the FP64 lattice.
//
// One launch runs the adjoint of one time step of the differentiated lattice
// run: pull streaming, FluidSolver::collide with the Luo force term
// (FluidSolver.cpp:103-183, Luo1993ForceModel.cpp:29-70), the D2Q5 species
// collide with their reaction source (CDESolverD2Q5.cpp:75-107,
// tutorial_01_CDESolverD2Q5_SIGNAL.cpp:102-135) and the box outlet rescale
// (MassSolverBoxOutlet.cpp:42-72).  The geometry is frozen: the spread force
// field, the domain ids and the per-domain mass table are constants of the run.
//
// Notation (per lattice node x, step t):
//   A_t        stored state after step t (fluid planes, then species planes),
//   f_q(x)   = A_{t-1,q}(x - c_q)     the pulled inputs of step t,
//   P_t(q, x)  dL/d f_q(x) of step t  (the adjoint of the pulled inputs).
// The adjoint of the state stored after step t is then
//   dL/dA_{t,q}(y) = P_{t+1}(q, y + c_q),
// a gather in the direction opposite to the forward pull, so the kernel reads
// P_{t+1} at shifted positions, recomputes step t's collision from A_{t-1},
// runs the chain rule backwards through it node by node and writes P_t.
// At the final step the adjoint of the stored state is the seed dL/dC_k(x)
// (C_k = sum of the species' five values) for every species direction.
//
// Parameter gradients, accumulated without contended atomics:
//   part[b][0], part[b][1 + k]  dL/d(1/tauF), dL/d(1/tau_k) summed by thread
//                               block b (each block owns its slots; the same
//                               blocks cover the same nodes every step),
//   racc[k][x]                  dL/d source_k at node x (RX_LINEAR species),
//   macc[x]                     dL/d rhoToAdd at node x (FluidSolver::addMass's
//                               per-domain mass source, when the run has one),
//   G[x]                        dL/dF(x) of the force field,
// all summed over the steps; launch_adjoint_finish reduces part, racc and macc
// into grad[0..S], grad[1 + S + k*nDomains + domain] and
// grad[1 + S + S*nDomains + domain].  A seed for the fluid (seedF, the
// gradient of the loss with respect to the final stored distributions) joins
// the species' seed at the final step.
#include "kernels.cuh"

namespace lbib {

namespace {

__device__ __constant__ int kCX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
__device__ __constant__ int kCY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};

__device__ __forceinline__ double weight9(int q) { return q == 0 ? 4.0 / 9.0 : (q < 5 ? 1.0 / 9.0 : 1.0 / 36.0); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Adds v into grad[key] once per group of lanes with the same key (lanes with
// key < 0 add nothing).  Every lane of the warp calls it.
__device__ __forceinline__ void warp_keyed_add(double* grad, int key, double v) {
    const int key0 = __shfl_sync(0xffffffffu, key, 0);
    if (__all_sync(0xffffffffu, key == key0)) {  // the usual case: one domain per warp
        const double sum = warp_sum(v);
        if ((threadIdx.x & 31) == 0 && key0 >= 0 && sum != 0.0) atomicAdd(grad + key0, sum);
        return;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    double sum = 0.0;
#pragma unroll 4
    for (int l = 0; l < 32; ++l) {
        const double t = __shfl_sync(0xffffffffu, v, l);
        if ((peers >> l) & 1u) sum += t;
    }
    const int lane = threadIdx.x & 31;
    if (key >= 0 && lane == __ffs(peers) - 1 && sum != 0.0) atomicAdd(grad + key, sum);
}

}  // namespace

// NS = number of species (compile-time, so that the species' inputs are
// loaded together with the fluid state).  Grid (ceil(nx / kAdjBlock), ny).
// The fluid's adjoint inputs are loaded after the species' reverse pass and
// the gradient accumulators where they are updated, so that a node's values
// are not all live at once (one species: 24 B of spills at 128 registers).
// LBIB_ADJOINT_MIN_BLOCKS (blocks per SM the register budget is sized for)
// trades occupancy against spills.
#ifndef LBIB_ADJOINT_MIN_BLOCKS
#define LBIB_ADJOINT_MIN_BLOCKS 4
#endif
// Threads per block (nodes of one row segment); with the blocks per SM above
// it sets the register budget: 128 x 4 -> 128 registers.  Measured on
// adjoint_512 (T = 2000, K = 100): 256 x 2 backward 75.6 ms, 128 x 4 73.1 ms,
// 64 x 8 73.2 ms; 256 x 1 (no spills, 8 warps per SM) and 128 x 5 (96
// registers, 300 B of spills) are slower.
#ifndef LBIB_ADJOINT_BLOCK
#define LBIB_ADJOINT_BLOCK 128
#endif
constexpr int kAdjBlock = LBIB_ADJOINT_BLOCK;
// Real: the precision the states are stored in.  An FP32-shifted run stores
// f_q - w_q in FP32 (and its species as they are); the reverse step reads
// them back as f and runs its arithmetic in FP64 all the same.
// MOT: the motion form of a run with moving membrane nodes: the step's
// velocity output has its own adjoint input a.gu (the nodes interpolate it),
// the post-collision velocity is written to a.uo, and G holds this step's
// dL/dF alone (the force field changes every step).
template <int NS, typename Real, bool MOT = false>
__global__ void __launch_bounds__(kAdjBlock, LBIB_ADJOINT_MIN_BLOCKS) adjoint_step64(AdjointArgs a) {
    const int nx = a.nx, ny = a.ny;
    const size_t L = a.L;
    const int xr = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = xr < nx;
    const int x = valid ? xr : nx - 1, y = blockIdx.y;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const unsigned rC = (unsigned)y * nx, rM = (unsigned)ym * nx, rP = (unsigned)yp * nx;
    const unsigned n = rC + x;
    // forward pull sources x - c_q and adjoint gather sources x + c_q (offsets
    // within a plane), formed where they are used
    auto pull = [&](int q) -> unsigned {
        const unsigned row = kCY[q] > 0 ? rM : (kCY[q] < 0 ? rP : rC);
        return row + (kCX[q] > 0 ? xm : (kCX[q] < 0 ? xp : x));
    };
    auto push = [&](int q) -> unsigned {
        const unsigned row = kCY[q] > 0 ? rP : (kCY[q] < 0 ? rM : rC);
        return row + (kCX[q] > 0 ? xp : (kCX[q] < 0 ? xm : x));
    };

    // ---- the inputs of the forward recomputation and of the species ------
    // The stored state, the domain ids, the force field and the mass table
    // are written by no kernel of the reverse pass, and every kernel before
    // the previous launch has completed (the previous launch, an adjoint step
    // of the same pass with a.chained, let this one start only after its own
    // wait): they are loaded before the wait, during the previous step's last
    // wave.  The adjoint planes and the accumulators are read after it.
    const Real* __restrict__ fprev = (const Real*)a.fprev;
    double f[9], lf[9];
#pragma unroll
    for (int q = 0; q < 9; ++q)
        f[q] = sizeof(Real) == 8 ? (double)fprev[(size_t)q * L + pull(q)]
                                 : (double)fprev[(size_t)q * L + pull(q)] + weight9(q);
    double gA[NS > 0 ? NS : 1][5], muA[NS > 0 ? NS : 1][5];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const Real* gp = (const Real*)a.gprev + (size_t)k * 5 * L;
#pragma unroll
        for (int q = 0; q < 5; ++q) gA[k][q] = gp[(size_t)q * L + pull(q)];
    }
    const uint32_t dom = a.dom[n];
    // The force field of a differentiated run is zero outside the force tiles,
    // so it and G are read and written everywhere: no load waits on another.
    const double fx = a.force[n], fy = a.force[L + n];
    double rta = 0.0;
    if (a.massTab != nullptr && dom < (uint32_t)a.nDomains) rta = a.massTab[dom];
    pdl_wait();
    pdl_launch_dependents();
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        if (a.seed) {
            const double sd = a.seed[(size_t)k * L + n];
#pragma unroll
            for (int q = 0; q < 5; ++q) muA[k][q] = sd;
        } else {
            const float* pg = a.pg + (size_t)k * 5 * L;
#pragma unroll
            for (int q = 0; q < 5; ++q) muA[k][q] = (double)pg[(size_t)q * L + push(q)];
        }
    }
    double gTauK[NS > 0 ? NS : 1];
    const bool hasMass = a.macc != nullptr && a.massTab != nullptr && dom < (uint32_t)a.nDomains && isfinite(rta);
    if (!isfinite(rta)) rta = 0.0;

    // ---- forward recomputation of the fluid collision --------------------
    const double tauI = a.tauIF;
    double rhoF = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) rhoF += f[q];
    const double rho = rhoF + rta;
    double jx = 0.0, jy = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        jx += kCX[q] * f[q];
        jy += kCY[q] * f[q];
    }
    const double rhoI = 1.0 / rho;
    const double ux = jx * rhoI, uy = jy * rhoI;
    const double lastTerm = 1.5 * (ux * ux + uy * uy);
    // equilibrium and post-collision value of direction q
    auto feqw = [&](int q) {
        const double cu = kCX[q] * ux + kCY[q] * uy;
        return weight9(q) * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - lastTerm);
    };
    auto fs = [&](int q) {
        return f[q] - f[q] * tauI + feqw(q) * tauI + 3.0 * weight9(q) * rhoF * (kCX[q] * fx + kCY[q] * fy);
    };
    double jox = 0.0, joy = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double v = fs(q);
        jox += kCX[q] * v;
        joy += kCY[q] * v;
    }
    const double uox = jox * rhoI, uoy = joy * rhoI;  // FluidSolver::velocity_ after collide
    // box outlet: node-local rescale(s) by 1/sum(f) on x = 0 and y = 0 (corner twice)
    const int passes = a.outlet ? (x == 0) + (y == 0) : 0;
    double s1 = 1.0, s2 = 1.0;
    if (passes >= 1) {
        double r = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) r += fs(q);
        s1 = 1.0 / r;
    }
    if (passes == 2) {
        double r = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) r += fs(q) * s1;
        s2 = 1.0 / r;
    }

    // ---- species, backwards (their velocity and outlet terms feed the fluid)
    double D1 = 0.0, D2 = 0.0;      // dL/ds1, dL/ds2 from the species
    double muox = 0.0, muoy = 0.0;  // dL/d(post-collision velocity)
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        double* g = gA[k];
        double* mu = muA[k];
        const SpeciesConst sp = a.sp[k];
        const double tauIk = a.tauI[k];
        const double C = g[0] + g[1] + g[2] + g[3] + g[4];
        const double C3 = C * (1.0 / 3.0), C6 = C * (1.0 / 6.0);
        double temp[5];
        temp[0] = C3;
        temp[1] = C6 * (1.0 + 3.0 * uox);
        temp[2] = C6 * (1.0 + 3.0 * uoy);
        temp[3] = C6 * (1.0 - 3.0 * uox);
        temp[4] = C6 * (1.0 - 3.0 * uoy);
        // dR/dC; the reaction value R itself only enters the outlet terms
        double dRdC = 0.0;
        if (sp.kind == RX_LINEAR) dRdC = -sp.decay;
        else if (sp.kind == RX_SIGNAL && !(dom == 1 && a.iteration < 5000u)) dRdC = -0.00001;
        const bool react = sp.kind != RX_NONE;
        auto reaction = [&]() {
            if (sp.kind == RX_LINEAR) {
                double src = 0.0;
                if (a.srcTab != nullptr && dom < (uint32_t)a.nDomains) src = a.srcTab[(size_t)k * a.nDomains + dom];
                return src - sp.decay * C;
            }
            if (sp.kind == RX_SIGNAL) return (dom == 1 && a.iteration < 5000u) ? 0.0001 : -0.00001 * C;
            return 0.0;
        };
        const double R = passes ? reaction() : 0.0;
        auto gs = [&](int q) {
            return g[q] - g[q] * tauIk + temp[q] * tauIk + (react ? R * (q == 0 ? (1.0 / 3.0) : (1.0 / 6.0)) : 0.0);
        };
        // outlet rescales of the species (same factors as the fluid)
        if (passes == 2) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                D2 += mu[q] * (gs(q) * s1);
                mu[q] *= s2;
            }
        }
        if (passes >= 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                D1 += mu[q] * gs(q);
                mu[q] *= s1;
            }
        }
        // collide, backwards
        double gTau = 0.0;
#pragma unroll
        for (int q = 0; q < 5; ++q) gTau += mu[q] * (temp[q] - g[q]);
        const double mR = react ? (mu[0] * (1.0 / 3.0) + (mu[1] + mu[2] + mu[3] + mu[4]) * (1.0 / 6.0)) : 0.0;
        const double mC = tauIk * (mu[0] * (1.0 / 3.0) +
                                   (mu[1] * (1.0 + 3.0 * uox) + mu[2] * (1.0 + 3.0 * uoy) +
                                    mu[3] * (1.0 - 3.0 * uox) + mu[4] * (1.0 - 3.0 * uoy)) * (1.0 / 6.0)) +
                          dRdC * mR;
        muox += tauIk * C * 0.5 * (mu[1] - mu[3]);
        muoy += tauIk * C * 0.5 * (mu[2] - mu[4]);
        if (valid) {
            float* qg = a.qg + (size_t)k * 5 * L;
#pragma unroll
            for (int q = 0; q < 5; ++q) qg[(size_t)q * L + n] = (float)((1.0 - tauIk) * mu[q] + mC);
        }
        gTauK[k] = valid ? gTau : 0.0;
        if (valid && sp.kind == RX_LINEAR) a.racc[(size_t)k * L + n] += mR;
    }

    // ---- the fluid's adjoint inputs, loaded once the species are done (the
    // node's values are not all held at once: no register spills) ----------
#pragma unroll
    for (int q = 0; q < 9; ++q)
        lf[q] = a.seed ? (a.seedF ? a.seedF[(size_t)q * L + n] : 0.0) : (double)a.pf[(size_t)q * L + push(q)];

    // ---- fluid: outlet, velocity output and collide, backwards -----------
    if (passes == 2) {
        double d = D2;
#pragma unroll
        for (int q = 0; q < 9; ++q) d += lf[q] * (fs(q) * s1);
#pragma unroll
        for (int q = 0; q < 9; ++q) lf[q] = s2 * lf[q] - s2 * s2 * d;
    }
    if (passes >= 1) {
        double d = D1;
#pragma unroll
        for (int q = 0; q < 9; ++q) d += lf[q] * fs(q);
#pragma unroll
        for (int q = 0; q < 9; ++q) lf[q] = s1 * lf[q] - s1 * s1 * d;
    }
    // post-collision velocity uo = (sum c_q fs_q) / rho
    if (MOT) {
        muox += a.gu[n];
        muoy += a.gu[L + n];
        if (valid) {
            a.uo[n] = uox;
            a.uo[L + n] = uoy;
        }
    }
    double mrho = -(uox * muox + uoy * muoy) * rhoI;
    const double mjox = muox * rhoI, mjoy = muoy * rhoI;
#pragma unroll
    for (int q = 0; q < 9; ++q) lf[q] += kCX[q] * mjox + kCY[q] * mjoy;

    double gTauF = 0.0, mrhoF = 0.0, mfx = 0.0, mfy = 0.0, mux = 0.0, muy = 0.0, mlast = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double w = weight9(q);
        gTauF += lf[q] * (feqw(q) - f[q]);
        const double mfeq = lf[q] * tauI;
        mrhoF += lf[q] * 3.0 * w * (kCX[q] * fx + kCY[q] * fy);
        mfx += lf[q] * 3.0 * w * rhoF * kCX[q];
        mfy += lf[q] * 3.0 * w * rhoF * kCY[q];
        const double cu = kCX[q] * ux + kCY[q] * uy;
        mrho += mfeq * w * (1.0 + 3.0 * cu + 4.5 * cu * cu - lastTerm);
        const double mcu = mfeq * w * rho * (3.0 + 9.0 * cu);
        mux += mcu * kCX[q];
        muy += mcu * kCY[q];
        mlast -= mfeq * w * rho;
    }
    mux += mlast * 3.0 * ux;
    muy += mlast * 3.0 * uy;
    const double mjx = mux * rhoI, mjy = muy * rhoI;
    mrho -= (ux * mux + uy * muy) * rhoI;
    mrhoF += mrho;
    // rho = sum f + rhoToAdd: dL/d rhoToAdd = dL/d rho
    if (valid && hasMass) a.macc[n] += mrho;
    if (valid) {
#pragma unroll
        for (int q = 0; q < 9; ++q)
            a.qf[(size_t)q * L + n] = (float)((1.0 - tauI) * lf[q] + mrhoF + kCX[q] * mjx + kCY[q] * mjy);
        if (MOT) {
            a.G[n] = mfx;
            a.G[L + n] = mfy;
        } else {
            a.G[n] += mfx;
            a.G[L + n] += mfy;
        }
    }
    // relaxation-time gradients: block sums into this block's own slots (the
    // same slots every step), reduced over blocks once at the end of the pass
    __shared__ double red[kAdjBlock / 32][1 + kMaxSpecies];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double v0 = warp_sum(valid ? gTauF : 0.0);
    if (lane == 0) red[warp][0] = v0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const double v = warp_sum(gTauK[k]);
        if (lane == 0) red[warp][1 + k] = v;
    }
    __syncthreads();
    if (threadIdx.x <= NS) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
        double* slot = a.part + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * (1 + NS) + threadIdx.x;
        *slot += t;
    }
}

// Sums the per-block relaxation-time partials (nBlocks x width) into grad[0..width).
__global__ void adjoint_part_reduce(const double* part, int nBlocks, int width, double* grad) {
    pdl_wait();
    __shared__ double red[8];
    for (int j = 0; j < width; ++j) {
        double t = 0.0;
        for (int b = threadIdx.x; b < nBlocks; b += blockDim.x) t += part[(size_t)b * width + j];
        t = warp_sum(t);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
            grad[j] = s;
        }
        __syncthreads();
    }
}

// Sums the per-node source-rate partials into grad[1 + S + k*nDomains + dom].
__global__ void adjoint_rate_reduce(const double* racc, const uint32_t* dom, size_t L, int S, int nDomains,
                                    double* grad) {
    pdl_wait();
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = n < L;
    const uint32_t d = valid ? dom[n] : 0u;
    for (int k = 0; k < S; ++k) {
        const int key = (valid && d < (uint32_t)nDomains) ? 1 + S + k * nDomains + (int)d : -1;
        warp_keyed_add(grad, key, valid ? racc[(size_t)k * L + n] : 0.0);
    }
}

__global__ void set_iteration_kernel(Status* st, unsigned it) {
    pdl_wait(); st->iteration = it; }

int adjoint_blocks(int nx, int ny) { return ((nx + kAdjBlock - 1) / kAdjBlock) * ny; }

void launch_adjoint_step64(const AdjointArgs& a, cudaStream_t s) {
    const dim3 grid((unsigned)((a.nx + kAdjBlock - 1) / kAdjBlock), (unsigned)a.ny);
    switch (a.S + (a.fp32 ? 4 : 0)) {
        case 0: launch_ex(a.chained != 0, adjoint_step64<0, double>, grid, kAdjBlock, 0, s, a); break;
        case 1: launch_ex(a.chained != 0, adjoint_step64<1, double>, grid, kAdjBlock, 0, s, a); break;
        case 2: launch_ex(a.chained != 0, adjoint_step64<2, double>, grid, kAdjBlock, 0, s, a); break;
        case 3: launch_ex(a.chained != 0, adjoint_step64<3, double>, grid, kAdjBlock, 0, s, a); break;
        case 4: launch_ex(a.chained != 0, adjoint_step64<0, float>, grid, kAdjBlock, 0, s, a); break;
        case 5: launch_ex(a.chained != 0, adjoint_step64<1, float>, grid, kAdjBlock, 0, s, a); break;
        case 6: launch_ex(a.chained != 0, adjoint_step64<2, float>, grid, kAdjBlock, 0, s, a); break;
        default: launch_ex(a.chained != 0, adjoint_step64<3, float>, grid, kAdjBlock, 0, s, a); break;
    }
}

void launch_adjoint_step64_motion(const AdjointArgs& a, cudaStream_t s) {
    const dim3 grid((unsigned)((a.nx + kAdjBlock - 1) / kAdjBlock), (unsigned)a.ny);
    switch (a.S + (a.fp32 ? 4 : 0)) {
        case 0: adjoint_step64<0, double, true><<<grid, kAdjBlock, 0, s>>>(a); break;
        case 1: adjoint_step64<1, double, true><<<grid, kAdjBlock, 0, s>>>(a); break;
        case 2: adjoint_step64<2, double, true><<<grid, kAdjBlock, 0, s>>>(a); break;
        case 3: adjoint_step64<3, double, true><<<grid, kAdjBlock, 0, s>>>(a); break;
        case 4: adjoint_step64<0, float, true><<<grid, kAdjBlock, 0, s>>>(a); break;
        case 5: adjoint_step64<1, float, true><<<grid, kAdjBlock, 0, s>>>(a); break;
        case 6: adjoint_step64<2, float, true><<<grid, kAdjBlock, 0, s>>>(a); break;
        default: adjoint_step64<3, float, true><<<grid, kAdjBlock, 0, s>>>(a); break;
    }
}

__global__ void to_float_kernel(const double* in, float* out, size_t n) {
    pdl_wait();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}

void launch_to_float(const double* in, float* out, size_t n, cudaStream_t s) {
    launch_pdl(to_float_kernel, (unsigned)((n + 255) / 256), 256, 0, s, in, out, n);
}

// Sums the per-node mass-source partials into grad[base + dom].
__global__ void adjoint_mass_reduce(const double* macc, const uint32_t* dom, size_t L, int nDomains, int base,
                                    double* grad) {
    pdl_wait();
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = n < L;
    const uint32_t d = valid ? dom[n] : 0u;
    const int key = (valid && d < (uint32_t)nDomains) ? base + (int)d : -1;
    warp_keyed_add(grad, key, valid ? macc[n] : 0.0);
}

void launch_adjoint_finish(const AdjointArgs& a, cudaStream_t s) {
    launch_pdl(adjoint_part_reduce, 1, 256, 0, s, a.part, adjoint_blocks(a.nx, a.ny), 1 + a.S, a.grad);
    if (a.S > 0 && a.srcTab != nullptr)
        launch_pdl(adjoint_rate_reduce, (unsigned)((a.L + 255) / 256), 256, 0, s, a.racc, a.dom, a.L, a.S, a.nDomains,
                                                                          a.grad);
    if (a.macc != nullptr && a.massTab != nullptr)
        launch_pdl(adjoint_mass_reduce, (unsigned)((a.L + 255) / 256), 256, 0, s, a.macc, a.dom, a.L, a.nDomains,
                   1 + a.S + a.S * a.nDomains, a.grad);
}

void launch_set_iteration(Status* st, unsigned it, cudaStream_t s) { launch_pdl(set_iteration_kernel, 1, 1, 0, s, st, it); }

}  // namespace lbib
