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

// FluidSolver::initWithVelocity (FluidSolver.cpp:62-101): the equilibrium at
// rho = 1 and velocity (u, v), natural direction order.
__host__ __device__ __forceinline__ void equilibrium_at_velocity64(double u, double v, double* fi) {
    const double W0 = 4.0 / 9.0, W1 = 1.0 / 9.0, W2 = 1.0 / 36.0;
    const double rho = 1.0;
    const double u2 = u * u;
    const double v2 = v * v;
    const double W1rho = W1 * rho;
    const double W2rho = W2 * rho;
    const double W3 = 9.0 / 2.0;
    const double lastTerm = 3.0 / 2.0 * (u2 + v2);
    fi[T] = W0 * rho * (1.0 - lastTerm);
    fi[E] = W1rho * (1.0 + 3.0 * u + W3 * u2 - lastTerm);
    fi[NE] = W2rho * (1.0 + 3.0 * (u + v) + W3 * (u + v) * (u + v) - lastTerm);
    fi[N] = W1rho * (1.0 + 3.0 * v + W3 * v2 - lastTerm);
    fi[NW] = W2rho * (1.0 + 3.0 * (-u + v) + W3 * (-u + v) * (-u + v) - lastTerm);
    fi[W] = W1rho * (1.0 + 3.0 * (-u) + W3 * u2 - lastTerm);
    fi[SW] = W2rho * (1.0 + 3.0 * (-u - v) + W3 * (-u - v) * (-u - v) - lastTerm);
    fi[S] = W1rho * (1.0 + 3.0 * (-v) + W3 * v2 - lastTerm);
    fi[SE] = W2rho * (1.0 + 3.0 * (u - v) + W3 * (u - v) * (u - v) - lastTerm);
}

// GuoZhengShi2002ForceModel::computeVelocity (GuoZhengShi2002ForceModel.cpp:60-78):
// the momentum includes half the force.
__host__ __device__ __forceinline__ void guo_velocity(double rho, const double* fi, double fx, double fy, double& ux,
                                                      double& uy) {
    const double rhoI = 1.0 / rho;
    ux = (fi[E] + fi[NE] + fi[SE] - (fi[NW] + fi[W] + fi[SW]) + 0.5 * fx) * rhoI;
    uy = (fi[NE] + fi[N] + fi[NW] - (fi[SW] + fi[S] + fi[SE]) + 0.5 * fy) * rhoI;
}

// FluidSolver::collide with GuoZhengShi2002ForceModel as the force model
// (the base class FluidSolver.hpp:41 names in a comment).  The equilibrium
// uses u of guo_velocity; the force term (GuoZhengShi2002ForceModel.cpp:29-58)
// is (1 - 1/2tau) w_i [3 (e_i - v) + 9 (e_i . v) e_i] . F with v the node's
// stored velocity (FluidSolver::getVelocity, the last collide's result: vx,
// vy).  neY is the coefficient of v_y in the NE term's F_y factor: the
// reference writes -3 (`9.0*u.x - 3.0*u.y + 3.0`, :51); the expansion above
// gives +6.  The expressions keep the reference's evaluation order.
__host__ __device__ __forceinline__ void collide_fluid64_guo(double* fi, double rhoToAdd, double fx, double fy,
                                                            double tauF, double vx, double vy, double neY,
                                                            double& uxo, double& uyo) {
    const double W0 = 4.0 / 9.0, W1 = 1.0 / 9.0, W2 = 1.0 / 36.0;
    double rho = sum9(fi);
    if (isfinite(rhoToAdd)) rho += rhoToAdd;
    double ux, uy;
    guo_velocity(rho, fi, fx, fy, ux, uy);
    const double ux2 = ux * ux;
    const double uy2 = uy * uy;
    const double lastTerm = 3.0 / 2.0 * (ux2 + uy2);
    const double tauI = 1.0 / tauF;
    const double W3 = 9.0 / 2.0;
    const double W1rho = W1 * rho;
    const double W2rho = W2 * rho;
    const double G0 = (1.0 - 0.5 / tauF) * 4.0 / 9.0;
    const double G1 = (1.0 - 0.5 / tauF) / 9.0;
    const double G2 = (1.0 - 0.5 / tauF) / 36.0;
    double fc[9];
    fc[T] = G0 * (-3.0 * vx * fx - 3.0 * vy * fy);
    fc[E] = G1 * ((6.0 * vx + 3.0) * fx - 3.0 * vy * fy);
    fc[N] = G1 * (-3.0 * vx * fx + (6.0 * vy + 3.0) * fy);
    fc[W] = G1 * ((6.0 * vx - 3.0) * fx - 3.0 * vy * fy);
    fc[S] = G1 * (-3.0 * vx * fx + (6.0 * vy - 3.0) * fy);
    fc[NE] = G2 * ((6.0 * vx + 9.0 * vy + 3.0) * fx + (9.0 * vx + neY * vy + 3.0) * fy);
    fc[NW] = G2 * ((6.0 * vx - 9.0 * vy - 3.0) * fx + (-9.0 * vx + 6.0 * vy + 3.0) * fy);
    fc[SW] = G2 * ((6.0 * vx + 9.0 * vy - 3.0) * fx + (9.0 * vx + 6.0 * vy - 3.0) * fy);
    fc[SE] = G2 * ((6.0 * vx - 9.0 * vy + 3.0) * fx + (-9.0 * vx + 6.0 * vy - 3.0) * fy);
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
#pragma unroll
    for (int d = 0; d < 9; ++d) {
        const double tempD = fi[d];
        fi[d] = tempD - tempD * tauI + temp[d];
    }
    guo_velocity(rho, fi, fx, fy, uxo, uyo);
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

// x^4 rounded once: x*x and (x*x)^2 split into exact head and tail with fma
// (Dekker's exact product), the tails summed, one final rounding.  The result
// is the correctly rounded x^4 except within about 2^-100 of a rounding
// boundary.
__host__ __device__ __forceinline__ double pow4_rn(double x) {
    const double p = x * x;
    const double pe = fma(x, x, -p);
    const double q = p * p;
    const double qe = fma(p, p, -q);
    return q + (qe + 2.0 * p * pe);
}

// The two reaction terms a species' collide adds to slot T (r0) and to E, N,
// W, S (r1), each in its solver's own expression order.  C is the species'
// concentration, Cp that of the partner species the reaction reads (as the
// partner's getC() returns it at that moment), ctype the node's cell type.
// COUPLED = false compiles only the RX_LINEAR / RX_SIGNAL terms (the
// lattice kernels instantiate it when no species has a coupled kind).
template <bool COUPLED = true>
__host__ __device__ __forceinline__ void reaction_terms64(const SpeciesConst& sp, double src, double C, double Cp,
                                                          uint32_t dom, uint32_t ctype, unsigned iteration,
                                                          double& r0, double& r1) {
    switch (COUPLED ? sp.kind : RX_LINEAR) {
        case RX_T2_R: {  // tutorial_02_CDESolverD2Q5_R.cpp:94-105,130-132 (gamma 100, a 0.1, deltaT 1e-4)
            const double R = dom != 0 ? 100.0 * (0.1 - C + C * C * Cp) : 0.0;
            r0 = 1.0e-4 * R / 3.0;
            r1 = 1.0e-4 * R / 6.0;
            return;
        }
        case RX_T2_L: {  // tutorial_02_CDESolverD2Q5_L.cpp:94-106 (b 0.9; R is the partner)
            const double R = dom != 0 ? 100.0 * (0.9 - Cp * Cp * C) : 0.0;
            r0 = 1.0e-4 * R / 3.0;
            r1 = 1.0e-4 * R / 6.0;
            return;
        }
        case RX_SCHNAK_U:  // SchnakenbergD2Q5u.cpp:114-121 (gamma 800, a 0.1)
            r0 = sp.dt * 800.0 * (0.1 - C + C * C * Cp) / 3.0;
            r1 = sp.dt * 800.0 * (0.1 - C + C * C * Cp) / 6.0;
            if (dom == 0) r0 = r1 = 0.0;
            return;
        case RX_SCHNAK_V:  // SchnakenbergD2Q5v.cpp:110-117 (b 0.9; u is the partner)
            r0 = sp.dt * 800.0 * (0.9 - Cp * Cp * C) / 3.0;
            r1 = sp.dt * 800.0 * (0.9 - Cp * Cp * C) / 6.0;
            if (dom == 0) r0 = r1 = 0.0;
            return;
        case RX_BMP: {  // CDESolverD2Q5BMP.cpp:107-120: decay 0.001, Hill production 1e-5 on cell type 2
            if (ctype == 2) {
                const double h4 = pow4_rn(Cp);
                r0 = sp.dt * 0.00001 / 3.0 * h4 / (sp.hill + h4);
                r1 = sp.dt * 0.00001 / 6.0 * h4 / (sp.hill + h4);
            } else {
                r0 = sp.dt * (-0.001 * C) / 3.0;
                r1 = sp.dt * (-0.001 * C) / 6.0;
            }
            return;
        }
        default: {  // RX_LINEAR, RX_SIGNAL
            const double R = reaction64(sp.kind, src, sp.decay, dom, iteration, C);
            const double deltaT = 1.0;
            r0 = deltaT * R / 3.0;
            r1 = deltaT * R / 6.0;
            return;
        }
    }
}

// CDESolverD2Q5::collide (kind RX_NONE) or the reaction variant, in place on gi[5].
template <bool COUPLED = true>
__host__ __device__ __forceinline__ void collide_cde64(double* gi, double ux, double uy, const SpeciesConst& sp,
                                                      double src, double Cp, uint32_t dom, uint32_t ctype,
                                                      unsigned iteration) {
    const double C = sum5(gi);
    const double w0 = C / 3.0;
    const double w1 = C / 6.0;
    const double tauI = 1.0 / sp.tau;
    double temp[5];
    temp[T] = w0;
    temp[E] = w1 * (1.0 + ux * 3.0);
    temp[N] = w1 * (1.0 + uy * 3.0);
    temp[W] = w1 * (1.0 + (-ux) * 3.0);
    temp[S] = w1 * (1.0 + (-uy) * 3.0);
    if (sp.kind == RX_NONE) {
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            const double tempD = gi[d];
            gi[d] = tempD - tempD * tauI + temp[d] * tauI;
        }
    } else {
        double r0, r1;
        reaction_terms64<COUPLED>(sp, src, C, Cp, dom, ctype, iteration, r0, r1);
        gi[T] = gi[T] - gi[T] * tauI + temp[T] * tauI + r0;
#pragma unroll
        for (int d = 1; d < 5; ++d) gi[d] = gi[d] - gi[d] * tauI + temp[d] * tauI + r1;
    }
}

// getC() of a species whose array is in post-collide order (after
// localSwap): the sum runs T, W, S, E, N over the direction-indexed slots.
__host__ __device__ __forceinline__ double sum5_swapped(const double* gi) {
    double C = 0.0;
    C += gi[T];
    C += gi[W];
    C += gi[S];
    C += gi[E];
    C += gi[N];
    return C;
}

}  // namespace lbib
