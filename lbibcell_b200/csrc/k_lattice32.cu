// k_lattice32.cu — FP32-shifted lattice kernels.
//
// Storage: h_q = f_q - w_q (deviation from the rest state rho0 = 1, u = 0) in
// FP32; collision arithmetic in FP32.  Algebraically the same update as the
// FP64 path (FluidSolver.cpp:103-183 with Luo1993ForceModel.cpp:29-70):
//   rho_F = 1 + sum h                      (force term density, no rhoToAdd)
//   rho   = rho_F + rhoToAdd
//   u     = (sum c_q h_q) / rho
//   h_q' = h_q + (heq_q - h_q)/tau + 3 w_q rho_F (c_q . F)
//   heq_q = w_q (rho - 1) + w_q rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2)
//   u'    = u + (rho_F / rho) F            (= sum c_q f_q' / rho)
// Species (rest state 0) are stored as g_q and updated as in
// CDESolverD2Q5.cpp:75-107 with the dt*R/3, dt*R/6 source.
#include "kernels.cuh"
#include "lattice_math.cuh"

namespace lbib {

// Cache hints of the stream-collide kernel's distribution traffic (a tuning
// knob, chosen by measurement): bit 0 loads the pulled inputs with the
// evict-first policy (each is read once), bit 1 stores the outputs with it.
// Both (3): the kernel itself is as fast as without, and the membrane stages
// of the step keep more of their data in L2 (tissue_1024: 195.2 -> 189.6 us
// per step on one B200).
#ifndef LBIB_COLLIDE_CACHE_HINTS
#define LBIB_COLLIDE_CACHE_HINTS 3
#endif
__device__ __forceinline__ float ld_dist(const float* p) {
    if (LBIB_COLLIDE_CACHE_HINTS & 1) return __ldcs(p);
    return *p;
}
__device__ __forceinline__ void st_dist(float* p, float v) {
    if (LBIB_COLLIDE_CACHE_HINTS & 2) __stcs(p, v);
    else *p = v;
}

__device__ __forceinline__ float reaction32(int kind, float src, float decay, uint32_t dom, unsigned iteration,
                                            float C) {
    if (kind == RX_LINEAR) return src - decay * C;
    if (kind == RX_SIGNAL) return (dom == 1 && iteration < 5000u) ? 0.0001f : -0.00001f * C;
    return 0.0f;
}

// The reaction terms for slot T (r0) and E, N, W, S (r1): the FP64 solvers'
// terms (reaction_terms64) in FP32.  COUPLED = false compiles only the
// RX_LINEAR / RX_SIGNAL terms.
template <bool COUPLED>
__device__ __forceinline__ void reaction_terms32(const SpeciesConst& sp, float src, float C, float Cp, uint32_t dom,
                                                 uint32_t ctype, unsigned iteration, float& r0, float& r1) {
    if (COUPLED && coupled_kind(sp.kind)) {
        float R, dt = sp.dtf;  // the rate the solver multiplies by its deltaT
        switch (sp.kind) {
            case RX_T2_R: R = dom != 0 ? 100.0f * (0.1f - C + C * C * Cp) : 0.0f; dt = 1.0e-4f; break;
            case RX_T2_L: R = dom != 0 ? 100.0f * (0.9f - Cp * Cp * C) : 0.0f; dt = 1.0e-4f; break;
            case RX_SCHNAK_U: R = dom != 0 ? 800.0f * (0.1f - C + C * C * Cp) : 0.0f; break;
            case RX_SCHNAK_V: R = dom != 0 ? 800.0f * (0.9f - Cp * Cp * C) : 0.0f; break;
            default:  // RX_BMP
                if (ctype == 2) {
                    const float h2 = Cp * Cp, h4 = h2 * h2;
                    R = 0.00001f * h4 / (sp.hillf + h4);
                } else {
                    R = -0.001f * C;
                }
                break;
        }
        const float x = dt * R;
        r0 = x * (1.0f / 3.0f);
        r1 = x * (1.0f / 6.0f);
        return;
    }
    const float R = reaction32(sp.kind, src, sp.decayf, dom, iteration, C);
    r0 = R * (1.0f / 3.0f);
    r1 = R * (1.0f / 6.0f);
}

// NS = number of species, a compile-time constant so that every input of a
// node (9 + 5 NS values) is loaded before any arithmetic.  Grid (nx/256, ny).
// MODE bit 0 (COUPLED): a species' reaction reads a partner species (its
// pre-collide sum until it has collided at this node, its post-collide sum
// after) or the node's cell type.  MODE bit 1 (MASSNODE): the mass source is
// per node (massNode) instead of per domain.  MODE bit 2 (GUO): the Guo
// force model (below).  MODE bit 3 (BOUNCE): DiracD2Q5 species keep the
// populations of links with a boundary node (as in stream_collide64).  Each combination is its own instantiation, so that
// the plain case carries no code for the others.
//
// Guo force model (GuoZhengShi2002ForceModel.cpp:29-78) in shifted form:
//   u     = (sum c_q h_q + F/2) / rho
//   h_q' = h_q + (heq_q - h_q)/tau + G_q [3 (c_q - v) . F + 9 (c_q . v)(c_q . F)]
//   G_q   = (1 - 1/2tau) w_q,  v = the node's stored velocity (last collide)
//   u'    = (sum c_q h_q' + F/2) / rho
// with the reference's NE coefficient (-3 v_y in place of +6 v_y in the F_y
// factor) for FM_GUO: G_NE * 9 v_y F_y less on NE.
// Blocks per SM the kernel's register budget is sized for (a tuning knob,
// chosen by measurement).  6 (40 registers, no spills, 48 warps per SM)
// against the compiler's own 48 registers (5 blocks): tissue_1024 step
// 177.0 -> 174.5 us, the kernel 37.4 -> 35.2 us inside the step; 8 (32
// registers) spills and is slower.
#ifndef LBIB_COLLIDE_MIN_BLOCKS
#define LBIB_COLLIDE_MIN_BLOCKS 6
#endif
template <int NS, int MODE>
__global__ void __launch_bounds__(256, LBIB_COLLIDE_MIN_BLOCKS) stream_collide32(LatticeArgs<float> a) {
    constexpr bool COUPLED = (MODE & 1) != 0;   // coupled species reactions
    constexpr bool MASSNODE = (MODE & 2) != 0;  // per-node mass source
    constexpr bool GUO = (MODE & 4) != 0;       // Guo force model
    constexpr bool BOUNCE = (MODE & 8) != 0;    // a DiracD2Q5 species (bounce-back at boundary links)
    pdl_wait();
    if (a.status->halt) return;
    const int nx = a.nx, ny = a.ny;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nx) return;
    const int y = blockIdx.y;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const size_t L = a.L;
    const unsigned rC = (unsigned)y * nx, rM = (unsigned)ym * nx, rP = (unsigned)yp * nx;
    const unsigned n = rC + x;
    const float* __restrict__ fin = a.fin;
    const float hT = ld_dist(&fin[0 * L + rC + x]);
    const float hE = ld_dist(&fin[1 * L + rC + xm]);
    const float hN = ld_dist(&fin[2 * L + rM + x]);
    const float hW = ld_dist(&fin[3 * L + rC + xp]);
    const float hS = ld_dist(&fin[4 * L + rP + x]);
    const float hNE = ld_dist(&fin[5 * L + rM + xm]);
    const float hNW = ld_dist(&fin[6 * L + rM + xp]);
    const float hSW = ld_dist(&fin[7 * L + rP + xp]);
    const float hSE = ld_dist(&fin[8 * L + rP + xm]);
    float gi[NS > 0 ? NS : 1][5];
    uint8_t bW = 0, bWe = 0, bS = 0, bSn = 0;
    if (BOUNCE) {
        bW = a.bounceW[n];
        bWe = a.bounceW[rC + xp];
        bS = a.bounceS[n];
        bSn = a.bounceS[rP + x];
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const float* __restrict__ gin = a.gin + (size_t)k * 5 * L;
        gi[k][0] = ld_dist(&gin[0 * L + rC + x]);
        if (BOUNCE && a.sp[k].bounce) {
            gi[k][1] = bW ? ld_dist(&gin[3 * L + n]) : ld_dist(&gin[1 * L + rC + xm]);
            gi[k][2] = bS ? ld_dist(&gin[4 * L + n]) : ld_dist(&gin[2 * L + rM + x]);
            gi[k][3] = bWe ? ld_dist(&gin[1 * L + n]) : ld_dist(&gin[3 * L + rC + xp]);
            gi[k][4] = bSn ? ld_dist(&gin[2 * L + n]) : ld_dist(&gin[4 * L + rP + x]);
        } else {
            gi[k][1] = ld_dist(&gin[1 * L + rC + xm]);
            gi[k][2] = ld_dist(&gin[2 * L + rM + x]);
            gi[k][3] = ld_dist(&gin[3 * L + rC + xp]);
            gi[k][4] = ld_dist(&gin[4 * L + rP + x]);
        }
    }
    const uint32_t dom = a.dom[n];
    float rta = 0.0f;
    if (MASSNODE) rta = (float)a.massNode[n];
    else if (a.massTab != nullptr && dom < (uint32_t)a.nDomains) rta = (float)a.massTab[dom];
    float Fx = 0.0f, Fy = 0.0f;
    if (a.tileCount[(y / kTile) * a.tilesX + (x / kTile)] > 0) {
        Fx = a.force[n];
        Fy = a.force[L + n];
    }
    const float drho = ((hT + hE) + (hN + hW)) + ((hS + hNE) + (hNW + hSW)) + hSE;
    const float dr = drho + rta;          // rho - 1
    const float rhoF = 1.0f + drho;
    const float rho = rhoF + rta;
    float jx = (hE - hW) + (hNE - hNW) + (hSE - hSW);
    float jy = (hN - hS) + (hNE - hSE) + (hNW - hSW);
    if (GUO) {
        jx += 0.5f * Fx;
        jy += 0.5f * Fy;
    }
    const float rinv = 1.0f / rho;
    const float ux = jx * rinv, uy = jy * rinv;
    const float tauI = a.tauIf;
    const float usq = 1.5f * (ux * ux + uy * uy);
    const float w0 = 4.0f / 9.0f, w1 = 1.0f / 9.0f, w2 = 1.0f / 36.0f;
    float ho[9];
    if (!GUO) {
        const float f3 = 3.0f * rhoF;
        ho[0] = hT + (w0 * dr + w0 * rho * (-usq) - hT) * tauI;
#define LBIB_Q(idx, h, w, cu, cf)                                                 \
    {                                                                             \
        const float c_u = (cu);                                                   \
        const float heq = (w) * dr + (w) * rho * (3.0f * c_u + 4.5f * c_u * c_u - usq); \
        ho[idx] = (h) + (heq - (h)) * tauI + (w) * f3 * (cf);                     \
    }
        LBIB_Q(1, hE, w1, ux, Fx)
        LBIB_Q(2, hN, w1, uy, Fy)
        LBIB_Q(3, hW, w1, -ux, -Fx)
        LBIB_Q(4, hS, w1, -uy, -Fy)
        LBIB_Q(5, hNE, w2, ux + uy, Fx + Fy)
        LBIB_Q(6, hNW, w2, -ux + uy, -Fx + Fy)
        LBIB_Q(7, hSW, w2, -ux - uy, -Fx - Fy)
        LBIB_Q(8, hSE, w2, ux - uy, Fx - Fy)
#undef LBIB_Q
    } else {
        const float vx = a.u[n], vy = a.u[L + n];  // the stored velocity, before it is overwritten
        const float gf = a.gff;
        const float vF = vx * Fx + vy * Fy;
        ho[0] = hT + (w0 * dr + w0 * rho * (-usq) - hT) * tauI + w0 * gf * (-3.0f * vF);
#define LBIB_G(idx, h, w, cu, cv, cF)                                             \
    {                                                                             \
        const float c_u = (cu);                                                   \
        const float heq = (w) * dr + (w) * rho * (3.0f * c_u + 4.5f * c_u * c_u - usq); \
        ho[idx] = (h) + (heq - (h)) * tauI + (w) * gf * (3.0f * ((cF) - vF) + 9.0f * (cv) * (cF)); \
    }
        LBIB_G(1, hE, w1, ux, vx, Fx)
        LBIB_G(2, hN, w1, uy, vy, Fy)
        LBIB_G(3, hW, w1, -ux, -vx, -Fx)
        LBIB_G(4, hS, w1, -uy, -vy, -Fy)
        LBIB_G(5, hNE, w2, ux + uy, vx + vy, Fx + Fy)
        LBIB_G(6, hNW, w2, -ux + uy, -vx + vy, -Fx + Fy)
        LBIB_G(7, hSW, w2, -ux - uy, -vx - vy, -Fx - Fy)
        LBIB_G(8, hSE, w2, ux - uy, vx - vy, Fx - Fy)
#undef LBIB_G
        if (a.forceModel == FM_GUO) ho[5] -= w2 * gf * 9.0f * vy * Fy;
    }
    float uxo, uyo;
    if (!GUO) {
        const float s = rhoF * rinv;
        uxo = ux + s * Fx;
        uyo = uy + s * Fy;
    } else {
        const float jxo = (ho[1] - ho[3]) + (ho[5] - ho[6]) + (ho[8] - ho[7]);
        const float jyo = (ho[2] - ho[4]) + (ho[5] - ho[8]) + (ho[6] - ho[7]);
        uxo = (jxo + 0.5f * Fx) * rinv;
        uyo = (jyo + 0.5f * Fy) * rinv;
    }
    a.u[n] = uxo;
    a.u[L + n] = uyo;
    // MassSolverBoxOutlet on the x=0 column and the y=0 row (the corner twice),
    // fused here as in the FP64 kernel: f' = f / rho, i.e.
    // h' = (h - w * dh) / (1 + dh) with dh = sum h.
    const int passes = a.outlet ? (x == 0) + (y == 0) : 0;
    float rs[2] = {1.0f, 1.0f};
    for (int p = 0; p < passes; ++p) {
        const float wq[9] = {w0, w1, w1, w1, w1, w2, w2, w2, w2};
        float dh = 0.0f;
#pragma unroll
        for (int q = 0; q < 9; ++q) dh += ho[q];
        rs[p] = 1.0f / (1.0f + dh);
#pragma unroll
        for (int q = 0; q < 9; ++q) ho[q] = (ho[q] - wq[q] * dh) * rs[p];
    }
    float* __restrict__ fo = a.fout;
#pragma unroll
    for (int q = 0; q < 9; ++q) st_dist(&fo[q * L + n], ho[q]);

    // Species: e0 = C - 4 e1 rather than C/3, so that the equilibrium sums to C
    // exactly up to one rounding: with C/3 and C/6 each rounded in FP32 the
    // relaxation adds a systematic 3e-8 C / tau per step.
    const unsigned iteration = NS > 0 ? a.status->iteration : 0u;
    float Cs[NS > 0 ? NS : 1];
    uint32_t ctype = 0;
    if (COUPLED) {
#pragma unroll
        for (int k = 0; k < NS; ++k) Cs[k] = ((gi[k][0] + gi[k][1]) + (gi[k][2] + gi[k][3])) + gi[k][4];
        if (a.status->cellTypesCopied) ctype = dom < (uint32_t)a.nDomains ? a.ctypeTab[dom] : 1u;
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const float gT = gi[k][0], gE = gi[k][1], gN = gi[k][2], gW = gi[k][3], gS = gi[k][4];
        const float C = ((gT + gE) + (gN + gW)) + gS;
        const float tI = a.sp[k].tIf;
        float src = 0.0f;
        if (a.srcTab != nullptr && dom < (uint32_t)a.nDomains) src = (float)a.srcTab[(size_t)k * a.nDomains + dom];
        float Cp = 0.0f;
        if (COUPLED) {
#pragma unroll
            for (int j = 0; j < NS; ++j)
                if (a.sp[k].partner == j) Cp = Cs[j];
        }
        float r0, r1;
        reaction_terms32<COUPLED>(a.sp[k], src, C, Cp, dom, ctype, iteration, r0, r1);
        const float e1 = C * (1.0f / 6.0f), e0 = C - 4.0f * e1;
        float go[5];
        go[0] = gT + (e0 - gT) * tI + r0;
        go[1] = gE + (e1 * (1.0f + 3.0f * uxo) - gE) * tI + r1;
        go[2] = gN + (e1 * (1.0f + 3.0f * uyo) - gN) * tI + r1;
        go[3] = gW + (e1 * (1.0f - 3.0f * uxo) - gW) * tI + r1;
        go[4] = gS + (e1 * (1.0f - 3.0f * uyo) - gS) * tI + r1;
        if (COUPLED) Cs[k] = ((go[0] + go[1]) + (go[2] + go[3])) + go[4];
        for (int p = 0; p < passes; ++p)
#pragma unroll
            for (int q = 0; q < 5; ++q) go[q] *= rs[p];
        float* __restrict__ gop = a.gout + (size_t)k * 5 * L;
#pragma unroll
        for (int q = 0; q < 5; ++q) st_dist(&gop[q * L + n], go[q]);
    }
}

// MassSolverBoxOutlet in shifted storage: f' = f / rho, i.e.
// h' = h / rho + w (1/rho - 1) = (h - w * drho) / rho with drho = sum h.
__device__ __forceinline__ void rescale_node32(float* f, float* g, int nS, size_t L, size_t n) {
    const float wq[9] = {4.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f,
                         1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f};
    float drho = 0.0f;
#pragma unroll
    for (int q = 0; q < 9; ++q) drho += f[(size_t)q * L + n];
    const float rinv = 1.0f / (1.0f + drho);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const float h = f[(size_t)q * L + n];
        f[(size_t)q * L + n] = (h - wq[q] * drho) * rinv;
    }
    for (int k = 0; k < nS; ++k)
#pragma unroll
        for (int q = 0; q < 5; ++q) g[((size_t)k * 5 + q) * L + n] *= rinv;
}

__global__ void outlet32(float* f, float* g, int nS, int nx, int ny, size_t L, const Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ny) {
        rescale_node32(f, g, nS, L, (size_t)i * nx);
        if (i == 0) rescale_node32(f, g, nS, L, 0);
    } else if (i < ny + nx - 1) {
        rescale_node32(f, g, nS, L, (size_t)(i - ny + 1));
    }
}

// Initial state: the FP64 initial collision (f_T = 1, zero force and mass)
// converted to deviations, and the species' initial conditions.  withVel:
// FluidSolver::initWithVelocity at the uniform velocity (vx, vy) instead
// (equilibrium at rho = 1, FluidSolver.cpp:62-101), and the species'
// initSolver collides at that velocity.
__global__ void init32(float* f, float* g, float* u, int nS, size_t L, double tauF, const uint32_t* dom,
                       SpeciesConst sp0, SpeciesConst sp1, SpeciesConst sp2, double init0, double init1,
                       double init2, int withVel, double vx, double vy) {
    pdl_wait();
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L) return;
    const double wq[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                          1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
    const double tauI = 1.0 / tauF;
    if (withVel) {
        double fi[9];
        equilibrium_at_velocity64(vx, vy, fi);
        for (int q = 0; q < 9; ++q) f[(size_t)q * L + n] = (float)(fi[q] - wq[q]);
        u[n] = (float)vx;
        u[L + n] = (float)vy;
    } else {
        // f_q' = f_q - f_q/tau + w_q/tau with f = (1, 0, ..., 0), so h_q = (f_q - w_q)(1 - 1/tau).
        for (int q = 0; q < 9; ++q) {
            const double f0 = q == 0 ? 1.0 : 0.0;
            f[(size_t)q * L + n] = (float)((f0 - wq[q]) * (1.0 - tauI));
        }
        u[n] = 0.0f;
        u[L + n] = 0.0f;
    }
    const SpeciesConst sp[3] = {sp0, sp1, sp2};
    const double init[3] = {init0, init1, init2};
    for (int k = 0; k < nS; ++k) {
        double gi[5];
        if (sp[k].kind == RX_NONE && withVel) {
            gi[0] = 1.0; gi[1] = gi[2] = gi[3] = gi[4] = 0.0;
            collide_cde64(gi, vx, vy, sp[k], 0.0, 0.0, dom[n], 0u, 0u);
        } else if (sp[k].kind == RX_NONE) {
            const double tI = 1.0 / sp[k].tau;
            gi[0] = 1.0 - tI + (1.0 / 3.0) * tI;
            for (int q = 1; q < 5; ++q) gi[q] = (1.0 / 6.0) * tI;
        } else if (sp[k].kind == RX_SIGNAL) {
            for (int q = 0; q < 5; ++q) gi[q] = dom[n] == 0 ? 0.0 : 0.2;
        } else {
            for (int q = 0; q < 5; ++q) gi[q] = init[k] / 5.0;
        }
        for (int q = 0; q < 5; ++q) g[((size_t)k * 5 + q) * L + n] = (float)gi[q];
    }
}

void launch_stream_collide32(const LatticeArgs<float>& args, cudaStream_t s) {
    // the per-node constants in FP32, rounded once here (IEEE double
    // division, then round to nearest: the values the kernel formed per node)
    LatticeArgs<float> a = args;
    a.tauIf = (float)(1.0 / a.tauF);
    a.gff = (float)(1.0 - 0.5 / a.tauF);
    for (int k = 0; k < a.S && k < kMaxSpecies; ++k) {
        SpeciesConst& c = a.sp[k];
        c.tIf = (float)(1.0 / c.tau);
        c.decayf = (float)c.decay;
        c.dtf = (float)c.dt;
        c.hillf = (float)c.hill;
    }
    const dim3 grid((unsigned)((a.nx + 255) / 256), (unsigned)a.ny);
    if (a.nfTab != nullptr) launch_noflux<float>(a, s);
    const int mode = (a.coupled ? 1 : 0) | (a.massNode != nullptr ? 2 : 0) | (a.forceModel != FM_LUO ? 4 : 0) |
                     (a.bounceW != nullptr ? 8 : 0);
    switch (mode * 4 + (a.S < 3 ? a.S : 3)) {
#define LBIB_SC_CASE(M, N) \
    case M * 4 + N: launch_pdl(stream_collide32<N, M>, grid, 256, 0, s, a); break;
        LBIB_SC_CASE(0, 0) LBIB_SC_CASE(0, 1) LBIB_SC_CASE(0, 2) LBIB_SC_CASE(0, 3)
        LBIB_SC_CASE(2, 0) LBIB_SC_CASE(2, 1) LBIB_SC_CASE(2, 2) LBIB_SC_CASE(2, 3)
        // coupled reactions need a partner species: two or three species
        LBIB_SC_CASE(1, 2) LBIB_SC_CASE(1, 3) LBIB_SC_CASE(3, 2) LBIB_SC_CASE(3, 3)
        // the same with the Guo force model
        LBIB_SC_CASE(4, 0) LBIB_SC_CASE(4, 1) LBIB_SC_CASE(4, 2) LBIB_SC_CASE(4, 3)
        LBIB_SC_CASE(6, 0) LBIB_SC_CASE(6, 1) LBIB_SC_CASE(6, 2) LBIB_SC_CASE(6, 3)
        LBIB_SC_CASE(5, 2) LBIB_SC_CASE(5, 3) LBIB_SC_CASE(7, 2) LBIB_SC_CASE(7, 3)
        LBIB_SC_CASE(8, 1) LBIB_SC_CASE(8, 2) LBIB_SC_CASE(8, 3)
#undef LBIB_SC_CASE
        default: break;
    }
}

void launch_outlet32(float* f, float* g, int nS, int nx, int ny, size_t L, const Status* st, cudaStream_t s) {
    const int n = nx + ny;
    launch_pdl(outlet32, (n + 255) / 256, 256, 0, s, f, g, nS, nx, ny, L, st);
}

void launch_init32(float* f, float* g, float* u, int nS, size_t L, double tauF, const uint32_t* dom, const double* vel,
                   const SpeciesConst* sp, const double* init, cudaStream_t s) {
    launch_pdl(init32, (unsigned)((L + 255) / 256), 256, 0, s, f, g, u, nS, L, tauF, dom, sp[0], sp[1], sp[2], init[0],
               init[1], init[2], vel != nullptr ? 1 : 0, vel != nullptr ? vel[0] : 0.0, vel != nullptr ? vel[1] : 0.0);
}

}  // namespace lbib
