// lattice_math.cuh — per-node collision arithmetic of the FP64 (plain) path.
//
// Every expression keeps the reference's evaluation order so that, compiled
// without FMA contraction (nvcc --fmad=false), the results are bit-identical
// to the reference's double-precision build:
//   FluidSolver::collide           libs/LbmLib/src/solver/FluidSolver/FluidSolver.cpp:103-183
//   Luo1993ForceModel              libs/LbmLib/src/solver/FluidSolver/Luo1993ForceModel.cpp:29-70
//   CDESolverD2Q5::collide         libs/LbmLib/src/solver/CDESolver/CDESolverD2Q5.cpp:75-107
//   reaction source dt*R/3, dt*R/6 libs/LbmLib/src/solver/CDESolver/tutorial_01_CDESolverD2Q5_SIGNAL.cpp:102-135
// Inputs are in natural direction order (the reference's order after
// advect); outputs are the post-collision values in natural order.
#pragma once

#include "lbib_internal.cuh"

namespace lbib {

__host__ __device__ __forceinline__ double sum9(const double* f) {
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) r += f[i];
    return r;
}

__host__ __device__ __forceinline__ double sum5(const double* g) {
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < 5; ++i) r += g[i];
    return r;
}

// Luo1993ForceModel::computeVelocity
__host__ __device__ __forceinline__ void luo_velocity(double rho, const double* fi, double& ux, double& uy) {
    const double rhoI = 1.0 / rho;
    ux = (fi[E] + fi[NE] + fi[SE] - (fi[NW] + fi[W] + fi[SW])) * rhoI;
    uy = (fi[NE] + fi[N] + fi[NW] - (fi[SW] + fi[S] + fi[SE])) * rhoI;
}

// FluidSolver::collide in place on fi[9]; returns the post-collision velocity.
__host__ __device__ __forceinline__ void collide_fluid64(double* fi, double rhoToAdd, double fx, double fy,
                                                        double tauF, double& uxo, double& uyo) {
    const double W0 = 4.0 / 9.0, W1 = 1.0 / 9.0, W2 = 1.0 / 36.0;
    double rho = sum9(fi);
    if (isfinite(rhoToAdd)) rho += rhoToAdd;
    double ux, uy;
    luo_velocity(rho, fi, ux, uy);
    const double ux2 = ux * ux;
    const double uy2 = uy * uy;
    const double lastTerm = 3.0 / 2.0 * (ux2 + uy2);
    const double tauI = 1.0 / tauF;
    const double W3 = 9.0 / 2.0;
    const double W1rho = W1 * rho;
    const double W2rho = W2 * rho;
    const double rhoF = sum9(fi);
    const double W1rho3 = rhoF * 3.0 / 9.0;
    const double W2rho3 = rhoF * 3.0 / 36.0;
    double temp[9];
    temp[T] = W0 * rho * (1.0 - lastTerm) * tauI + 0.0;
    temp[E] = W1rho * (1.0 + 3.0 * ux + W3 * ux2 - lastTerm) * tauI + W1rho3 * fx;
    temp[NE] = W2rho * (1.0 + 3.0 * (ux + uy) + W3 * (ux + uy) * (ux + uy) - lastTerm) * tauI + W2rho3 * (fx + fy);
    temp[N] = W1rho * (1.0 + 3.0 * uy + W3 * uy2 - lastTerm) * tauI + W1rho3 * fy;
    temp[NW] = W2rho * (1.0 + 3.0 * (-ux + uy) + W3 * (-ux + uy) * (-ux + uy) - lastTerm) * tauI + W2rho3 * (-fx + fy);
    temp[W] = W1rho * (1.0 + 3.0 * (-ux) + W3 * ux2 - lastTerm) * tauI + -W1rho3 * fx;
    temp[SW] = W2rho * (1.0 + 3.0 * (-ux - uy) + W3 * (-ux - uy) * (-ux - uy) - lastTerm) * tauI + W2rho3 * (-fx - fy);
    temp[S] = W1rho * (1.0 + 3.0 * (-uy) + W3 * uy2 - lastTerm) * tauI + -W1rho3 * fy;
    temp[SE] = W2rho * (1.0 + 3.0 * (ux - uy) + W3 * (ux - uy) * (ux - uy) - lastTerm) * tauI + W2rho3 * (fx - fy);
#pragma unroll
    for (int d = 0; d < 9; ++d) {
        const double tempD = fi[d];
        fi[d] = tempD - tempD * tauI + temp[d];
    }
    luo_velocity(rho, fi, uxo, uyo);
}

// Reaction term R for one species at one node.
//   RX_LINEAR: R = source[domain] - decay*C (the Lbib species plugins)
//   RX_SIGNAL: tutorial_01_CDESolverD2Q5_SIGNAL.cpp:92-100
__host__ __device__ __forceinline__ double reaction64(int kind, double src, double decay, uint32_t dom,
                                                      unsigned iteration, double C) {
    if (kind == RX_LINEAR) return src - decay * C;
    if (dom == 1 && iteration < 5000u) return 0.0001;
    return -0.00001 * C;
}

// CDESolverD2Q5::collide (kind RX_NONE) or the reaction variant, in place on gi[5].
__host__ __device__ __forceinline__ void collide_cde64(double* gi, double ux, double uy, double tau, int kind,
                                                      double src, double decay, uint32_t dom, unsigned iteration) {
    const double C = sum5(gi);
    const double w0 = C / 3.0;
    const double w1 = C / 6.0;
    const double tauI = 1.0 / tau;
    double temp[5];
    temp[T] = w0;
    temp[E] = w1 * (1.0 + ux * 3.0);
    temp[N] = w1 * (1.0 + uy * 3.0);
    temp[W] = w1 * (1.0 + (-ux) * 3.0);
    temp[S] = w1 * (1.0 + (-uy) * 3.0);
    if (kind == RX_NONE) {
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            const double tempD = gi[d];
            gi[d] = tempD - tempD * tauI + temp[d] * tauI;
        }
    } else {
        const double R = reaction64(kind, src, decay, dom, iteration, C);
        const double deltaT = 1.0;
        const double r0 = deltaT * R / 3.0;
        const double r1 = deltaT * R / 6.0;
        gi[T] = gi[T] - gi[T] * tauI + temp[T] * tauI + r0;
#pragma unroll
        for (int d = 1; d < 5; ++d) gi[d] = gi[d] - gi[d] * tauI + temp[d] * tauI + r1;
    }
}

}  // namespace lbib
