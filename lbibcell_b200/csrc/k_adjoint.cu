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
// Parameter gradients accumulate in `grad`:
//   grad[0]                     dL/d(1/tauF)
//   grad[1 + k]                 dL/d(1/tau_k)
//   grad[1 + S + k*nDom + d]    dL/d source_k[d]   (RX_LINEAR species)
// and dL/dF(x) of the force field in G (summed over steps, force tiles only).
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

__global__ void __launch_bounds__(256) adjoint_step64(AdjointArgs a) {
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = n < a.L;
    const size_t nn = valid ? n : 0;
    const int nx = a.nx, ny = a.ny;
    const size_t L = a.L;
    const int x = (int)(nn % (size_t)nx), y = (int)(nn / (size_t)nx);
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const size_t rC = (size_t)y * nx, rM = (size_t)ym * nx, rP = (size_t)yp * nx;
    // forward pull sources x - c_q and adjoint gather sources x + c_q
    const size_t pull[9] = {rC + x, rC + xm, rM + x, rC + xp, rP + x, rM + xm, rM + xp, rP + xp, rP + xm};
    const size_t push[9] = {rC + x, rC + xp, rP + x, rC + xm, rM + x, rP + xp, rP + xm, rM + xm, rM + xp};

    // ---- forward recomputation of the fluid collision -------------------
    double f[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = a.fprev[(size_t)q * L + pull[q]];
    const uint32_t dom = a.dom[nn];
    double rta = 0.0;
    if (a.massTab != nullptr && dom < (uint32_t)a.nDomains) rta = a.massTab[dom];
    if (!isfinite(rta)) rta = 0.0;
    const bool tile = a.tileCount[(y / kTile) * a.tilesX + (x / kTile)] > 0;
    double fx = 0.0, fy = 0.0;
    if (tile) {
        fx = a.force[nn];
        fy = a.force[L + nn];
    }
    const double tauI = 1.0 / a.tauF;
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
    const double ux = jx / rho, uy = jy / rho;
    const double lastTerm = 1.5 * (ux * ux + uy * uy);
    double fs[9], feqw[9];
    double jox = 0.0, joy = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double w = weight9(q);
        const double cu = kCX[q] * ux + kCY[q] * uy;
        feqw[q] = w * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - lastTerm);
        fs[q] = f[q] - f[q] * tauI + feqw[q] * tauI + 3.0 * w * rhoF * (kCX[q] * fx + kCY[q] * fy);
        jox += kCX[q] * fs[q];
        joy += kCY[q] * fs[q];
    }
    const double uox = jox / rho, uoy = joy / rho;  // FluidSolver::velocity_ after collide
    // box outlet: node-local rescale(s) by 1/sum(f) on x = 0 and y = 0 (corner twice)
    const int passes = a.outlet ? (x == 0) + (y == 0) : 0;
    double s1 = 1.0, s2 = 1.0;
    if (passes >= 1) {
        double r = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) r += fs[q];
        s1 = 1.0 / r;
    }
    if (passes == 2) {
        double r = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) r += fs[q] * s1;
        s2 = 1.0 / r;
    }

    // ---- adjoint of the stored fluid state ------------------------------
    double lf[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) lf[q] = a.seed ? 0.0 : a.pf[(size_t)q * L + push[q]];

    double D1 = 0.0, D2 = 0.0;    // dL/ds1, dL/ds2 from the species
    double muox = 0.0, muoy = 0.0;  // dL/d(post-collision velocity)
    for (int k = 0; k < a.S; ++k) {
        const double* gp = a.gprev + (size_t)k * 5 * L;
        double g[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) g[q] = gp[(size_t)q * L + pull[q]];
        const SpeciesConst sp = a.sp[k];
        const double tauIk = 1.0 / sp.tau;
        const double C = g[0] + g[1] + g[2] + g[3] + g[4];
        double temp[5];
        temp[0] = C / 3.0;
        temp[1] = C / 6.0 * (1.0 + 3.0 * uox);
        temp[2] = C / 6.0 * (1.0 + 3.0 * uoy);
        temp[3] = C / 6.0 * (1.0 - 3.0 * uox);
        temp[4] = C / 6.0 * (1.0 - 3.0 * uoy);
        double R = 0.0, dRdC = 0.0;
        if (sp.kind == RX_LINEAR) {
            double src = 0.0;
            if (a.srcTab != nullptr && dom < (uint32_t)a.nDomains) src = a.srcTab[(size_t)k * a.nDomains + dom];
            R = src - sp.decay * C;
            dRdC = -sp.decay;
        } else if (sp.kind == RX_SIGNAL) {
            if (dom == 1 && a.iteration < 5000u) {
                R = 0.0001;
            } else {
                R = -0.00001 * C;
                dRdC = -0.00001;
            }
        }
        const bool react = sp.kind != RX_NONE;
        double gs[5];
#pragma unroll
        for (int q = 0; q < 5; ++q)
            gs[q] = g[q] - g[q] * tauIk + temp[q] * tauIk + (react ? R * (q == 0 ? 1.0 / 3.0 : 1.0 / 6.0) : 0.0);

        double mu[5];
        if (a.seed) {
            const double sd = a.seed[(size_t)k * L + nn];
#pragma unroll
            for (int q = 0; q < 5; ++q) mu[q] = sd;
        } else {
            const double* pg = a.pg + (size_t)k * 5 * L;
#pragma unroll
            for (int q = 0; q < 5; ++q) mu[q] = pg[(size_t)q * L + push[q]];
        }
        // outlet rescales of the species (same factors as the fluid)
        if (passes == 2) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                D2 += mu[q] * (gs[q] * s1);
                mu[q] *= s2;
            }
        }
        if (passes >= 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                D1 += mu[q] * gs[q];
                mu[q] *= s1;
            }
        }
        // collide, backwards
        double gTau = 0.0;
#pragma unroll
        for (int q = 0; q < 5; ++q) gTau += mu[q] * (temp[q] - g[q]);
        const double mR = react ? (mu[0] / 3.0 + (mu[1] + mu[2] + mu[3] + mu[4]) / 6.0) : 0.0;
        const double mC = tauIk * (mu[0] / 3.0 + (mu[1] * (1.0 + 3.0 * uox) + mu[2] * (1.0 + 3.0 * uoy) +
                                                  mu[3] * (1.0 - 3.0 * uox) + mu[4] * (1.0 - 3.0 * uoy)) / 6.0) +
                          dRdC * mR;
        muox += tauIk * C * 0.5 * (mu[1] - mu[3]);
        muoy += tauIk * C * 0.5 * (mu[2] - mu[4]);
        if (valid) {
            double* qg = a.qg + (size_t)k * 5 * L;
#pragma unroll
            for (int q = 0; q < 5; ++q) qg[(size_t)q * L + n] = (1.0 - tauIk) * mu[q] + mC;
        }
        const double gt = warp_sum(valid ? gTau : 0.0);
        if ((threadIdx.x & 31) == 0 && gt != 0.0) atomicAdd(a.grad + 1 + k, gt);
        if (sp.kind == RX_LINEAR && a.srcTab != nullptr) {
            const int key = (valid && dom < (uint32_t)a.nDomains) ? 1 + a.S + k * a.nDomains + (int)dom : -1;
            warp_keyed_add(a.grad, key, valid ? mR : 0.0);
        }
    }

    // ---- fluid: outlet, velocity output and collide, backwards -----------
    if (passes == 2) {
        double d = D2;
#pragma unroll
        for (int q = 0; q < 9; ++q) d += lf[q] * (fs[q] * s1);
#pragma unroll
        for (int q = 0; q < 9; ++q) lf[q] = s2 * lf[q] - s2 * s2 * d;
    }
    if (passes >= 1) {
        double d = D1;
#pragma unroll
        for (int q = 0; q < 9; ++q) d += lf[q] * fs[q];
#pragma unroll
        for (int q = 0; q < 9; ++q) lf[q] = s1 * lf[q] - s1 * s1 * d;
    }
    // post-collision velocity uo = (sum c_q fs_q) / rho
    double mrho = -(uox * muox + uoy * muoy) / rho;
#pragma unroll
    for (int q = 0; q < 9; ++q) lf[q] += (kCX[q] * muox + kCY[q] * muoy) / rho;

    double gTauF = 0.0, mrhoF = 0.0, mfx = 0.0, mfy = 0.0, mux = 0.0, muy = 0.0, mlast = 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double w = weight9(q);
        gTauF += lf[q] * (feqw[q] - f[q]);
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
    const double mjx = mux / rho, mjy = muy / rho;
    mrho -= (ux * mux + uy * muy) / rho;
    mrhoF += mrho;
    if (valid) {
#pragma unroll
        for (int q = 0; q < 9; ++q) a.qf[(size_t)q * L + n] = (1.0 - tauI) * lf[q] + mrhoF + kCX[q] * mjx + kCY[q] * mjy;
        if (tile) {
            a.G[n] += mfx;
            a.G[L + n] += mfy;
        }
    }
    const double gt = warp_sum(valid ? gTauF : 0.0);
    if ((threadIdx.x & 31) == 0 && gt != 0.0) atomicAdd(a.grad, gt);
}

__global__ void set_iteration_kernel(Status* st, unsigned it) { st->iteration = it; }

void launch_adjoint_step64(const AdjointArgs& a, cudaStream_t s) {
    const unsigned blocks = (unsigned)((a.L + 255) / 256);
    adjoint_step64<<<blocks, 256, 0, s>>>(a);
}

void launch_set_iteration(Status* st, unsigned it, cudaStream_t s) { set_iteration_kernel<<<1, 1, 0, s>>>(st, it); }

}  // namespace lbib
