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
#include <cstdlib>

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

// ---------------------------------------------------------------------------
// The same step, four nodes per thread, for the plain modes (MODE 0 and 2:
// no coupled reactions, the Luo force model, no bounce-back species) and rows
// of a multiple of 256 nodes.  Each plane's row segment is read with aligned
// 128-bit loads; the x-1 / x+1 pull sources come from the neighbouring lane
// by warp shuffle, and lanes 0 and 31 load the one value past their warp's
// 128 nodes (the row wraps).  The outputs go out as 128-bit stores.  The
// per-node arithmetic is the scalar kernel's, expression for expression, and
// the results are the same to the last bit.  Measured on tissue_1024 (one
// B200, inside the step): 40.4 us per launch against 35.3 us for the scalar
// kernel (127 registers, 16 warps per SM against 40 registers, 48 warps),
// although a probe of the bare access pattern (21 planes in, 21 out, a sum
// per node) runs 28.7 us this way against 30.0 us with one node per thread:
// the four nodes' collision arithmetic, run one after another per thread, is
// not hidden.  The scalar kernel is the default; LBIB_COLLIDE_X4=1 selects
// this one.
__device__ __forceinline__ float4 ld_dist4(const float* p) {
    if (LBIB_COLLIDE_CACHE_HINTS & 1) return __ldcs(reinterpret_cast<const float4*>(p));
    return *reinterpret_cast<const float4*>(p);
}
__device__ __forceinline__ void st_dist4(float* p, float4 v) {
    if (LBIB_COLLIDE_CACHE_HINTS & 2) __stcs(reinterpret_cast<float4*>(p), v);
    else *reinterpret_cast<float4*>(p) = v;
}
// The values at x0 + DX .. x0 + 3 + DX of one plane row (DX = -1, 0, +1).
// Every lane of the warp calls it (the shuffles).
template <int DX>
__device__ __forceinline__ float4 ld_row4(const float* row, int x0, int nx, int lane) {
    const float4 v = ld_dist4(row + x0);
    if (DX == 0) return v;
    if (DX < 0) {
        float l = __shfl_up_sync(0xffffffffu, v.w, 1);
        if (lane == 0) l = ld_dist(row + (x0 == 0 ? nx - 1 : x0 - 1));
        return make_float4(l, v.x, v.y, v.z);
    }
    float r = __shfl_down_sync(0xffffffffu, v.x, 1);
    if (lane == 31) r = ld_dist(row + (x0 + 4 == nx ? 0 : x0 + 4));
    return make_float4(v.y, v.z, v.w, r);
}
__device__ __forceinline__ float& comp4(float4& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); }

#ifndef LBIB_COLLIDE4_MIN_BLOCKS
#define LBIB_COLLIDE4_MIN_BLOCKS 6
#endif
template <int NS, int MODE>
__global__ void __launch_bounds__(64, LBIB_COLLIDE4_MIN_BLOCKS) stream_collide32x4(LatticeArgs<float> a) {
    static_assert((MODE & ~2) == 0, "plain modes only");
    constexpr bool MASSNODE = (MODE & 2) != 0;
    pdl_wait();
    if (a.status->halt) return;
    const int nx = a.nx, ny = a.ny;
    const int x0 = blockIdx.x * 256 + threadIdx.x * 4, y = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const size_t L = a.L;
    const size_t rC = (size_t)y * nx, rM = (size_t)ym * nx, rP = (size_t)yp * nx;
    const size_t n0 = rC + x0;
    const float* __restrict__ fin = a.fin;
    float4 H[9];
    H[0] = ld_row4<0>(fin + 0 * L + rC, x0, nx, lane);
    H[1] = ld_row4<-1>(fin + 1 * L + rC, x0, nx, lane);
    H[2] = ld_row4<0>(fin + 2 * L + rM, x0, nx, lane);
    H[3] = ld_row4<1>(fin + 3 * L + rC, x0, nx, lane);
    H[4] = ld_row4<0>(fin + 4 * L + rP, x0, nx, lane);
    H[5] = ld_row4<-1>(fin + 5 * L + rM, x0, nx, lane);
    H[6] = ld_row4<1>(fin + 6 * L + rM, x0, nx, lane);
    H[7] = ld_row4<1>(fin + 7 * L + rP, x0, nx, lane);
    H[8] = ld_row4<-1>(fin + 8 * L + rP, x0, nx, lane);
    float4 G[NS > 0 ? NS : 1][5];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const float* __restrict__ gin = a.gin + (size_t)k * 5 * L;
        G[k][0] = ld_row4<0>(gin + 0 * L + rC, x0, nx, lane);
        G[k][1] = ld_row4<-1>(gin + 1 * L + rC, x0, nx, lane);
        G[k][2] = ld_row4<0>(gin + 2 * L + rM, x0, nx, lane);
        G[k][3] = ld_row4<1>(gin + 3 * L + rC, x0, nx, lane);
        G[k][4] = ld_row4<0>(gin + 4 * L + rP, x0, nx, lane);
    }
    const uint4 dom4 = *reinterpret_cast<const uint4*>(a.dom + n0);
    float4 F = make_float4(0.0f, 0.0f, 0.0f, 0.0f), Fy4 = F;
    if (a.tileCount[(y / kTile) * a.tilesX + (x0 / kTile)] > 0) {  // the four nodes share a tile
        F = *reinterpret_cast<const float4*>(a.force + n0);
        Fy4 = *reinterpret_cast<const float4*>(a.force + L + n0);
    }
    const unsigned iteration = NS > 0 ? a.status->iteration : 0u;
    const float tauI = a.tauIf;
    const float w0 = 4.0f / 9.0f, w1 = 1.0f / 9.0f, w2 = 1.0f / 36.0f;
    float4 U, V;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t dom = j == 0 ? dom4.x : (j == 1 ? dom4.y : (j == 2 ? dom4.z : dom4.w));
        float rta = 0.0f;
        if (MASSNODE) rta = (float)a.massNode[n0 + j];
        else if (a.massTab != nullptr && dom < (uint32_t)a.nDomains) rta = (float)a.massTab[dom];
        const float Fx = comp4(F, j), Fy = comp4(Fy4, j);
        const float hT = comp4(H[0], j), hE = comp4(H[1], j), hN = comp4(H[2], j), hW = comp4(H[3], j),
                    hS = comp4(H[4], j), hNE = comp4(H[5], j), hNW = comp4(H[6], j), hSW = comp4(H[7], j),
                    hSE = comp4(H[8], j);
        const float drho = ((hT + hE) + (hN + hW)) + ((hS + hNE) + (hNW + hSW)) + hSE;
        const float dr = drho + rta;
        const float rhoF = 1.0f + drho;
        const float rho = rhoF + rta;
        const float jx = (hE - hW) + (hNE - hNW) + (hSE - hSW);
        const float jy = (hN - hS) + (hNE - hSE) + (hNW - hSW);
        const float rinv = 1.0f / rho;
        const float ux = jx * rinv, uy = jy * rinv;
        const float usq = 1.5f * (ux * ux + uy * uy);
        float ho[9];
        const float f3 = 3.0f * rhoF;
        ho[0] = hT + (w0 * dr + w0 * rho * (-usq) - hT) * tauI;
#define LBIB_Q4(idx, h, w, cu, cf)                                                \
    {                                                                             \
        const float c_u = (cu);                                                   \
        const float heq = (w) * dr + (w) * rho * (3.0f * c_u + 4.5f * c_u * c_u - usq); \
        ho[idx] = (h) + (heq - (h)) * tauI + (w) * f3 * (cf);                     \
    }
        LBIB_Q4(1, hE, w1, ux, Fx)
        LBIB_Q4(2, hN, w1, uy, Fy)
        LBIB_Q4(3, hW, w1, -ux, -Fx)
        LBIB_Q4(4, hS, w1, -uy, -Fy)
        LBIB_Q4(5, hNE, w2, ux + uy, Fx + Fy)
        LBIB_Q4(6, hNW, w2, -ux + uy, -Fx + Fy)
        LBIB_Q4(7, hSW, w2, -ux - uy, -Fx - Fy)
        LBIB_Q4(8, hSE, w2, ux - uy, Fx - Fy)
#undef LBIB_Q4
        const float sF = rhoF * rinv;
        const float uxo = ux + sF * Fx, uyo = uy + sF * Fy;
        comp4(U, j) = uxo;
        comp4(V, j) = uyo;
        const int passes = a.outlet ? (x0 + j == 0) + (y == 0) : 0;
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
#pragma unroll
        for (int q = 0; q < 9; ++q) comp4(H[q], j) = ho[q];
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            const float gT = comp4(G[k][0], j), gE = comp4(G[k][1], j), gN = comp4(G[k][2], j),
                        gW = comp4(G[k][3], j), gS = comp4(G[k][4], j);
            const float C = ((gT + gE) + (gN + gW)) + gS;
            const float tI = a.sp[k].tIf;
            float src = 0.0f;
            if (a.srcTab != nullptr && dom < (uint32_t)a.nDomains) src = (float)a.srcTab[(size_t)k * a.nDomains + dom];
            float r0, r1;
            reaction_terms32<false>(a.sp[k], src, C, 0.0f, dom, 0u, iteration, r0, r1);
            const float e1 = C * (1.0f / 6.0f), e0 = C - 4.0f * e1;
            float go[5];
            go[0] = gT + (e0 - gT) * tI + r0;
            go[1] = gE + (e1 * (1.0f + 3.0f * uxo) - gE) * tI + r1;
            go[2] = gN + (e1 * (1.0f + 3.0f * uyo) - gN) * tI + r1;
            go[3] = gW + (e1 * (1.0f - 3.0f * uxo) - gW) * tI + r1;
            go[4] = gS + (e1 * (1.0f - 3.0f * uyo) - gS) * tI + r1;
            for (int p = 0; p < passes; ++p)
#pragma unroll
                for (int q = 0; q < 5; ++q) go[q] *= rs[p];
#pragma unroll
            for (int q = 0; q < 5; ++q) comp4(G[k][q], j) = go[q];
        }
    }
    *reinterpret_cast<float4*>(a.u + n0) = U;
    *reinterpret_cast<float4*>(a.u + L + n0) = V;
    float* __restrict__ fo = a.fout;
#pragma unroll
    for (int q = 0; q < 9; ++q) st_dist4(fo + q * L + n0, H[q]);
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        float* __restrict__ gop = a.gout + (size_t)k * 5 * L;
#pragma unroll
        for (int q = 0; q < 5; ++q) st_dist4(gop + q * L + n0, G[k][q]);
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
    // LBIB_COLLIDE_X4=1 (read when the kernel is launched or captured): four
    // nodes per thread for the plain modes on rows of a multiple of 256 nodes.
    // Off by default: slower inside the step (below).
    const char* x4 = std::getenv("LBIB_COLLIDE_X4");
    if ((mode == 0 || mode == 2) && a.nx % 256 == 0 && x4 && x4[0] == '1') {
        const dim3 grid4((unsigned)(a.nx / 256), (unsigned)a.ny);
        switch (mode * 4 + (a.S < 3 ? a.S : 3)) {
            case 0: launch_pdl(stream_collide32x4<0, 0>, grid4, 64, 0, s, a); break;
            case 1: launch_pdl(stream_collide32x4<1, 0>, grid4, 64, 0, s, a); break;
            case 2: launch_pdl(stream_collide32x4<2, 0>, grid4, 64, 0, s, a); break;
            case 3: launch_pdl(stream_collide32x4<3, 0>, grid4, 64, 0, s, a); break;
            case 8: launch_pdl(stream_collide32x4<0, 2>, grid4, 64, 0, s, a); break;
            case 9: launch_pdl(stream_collide32x4<1, 2>, grid4, 64, 0, s, a); break;
            case 10: launch_pdl(stream_collide32x4<2, 2>, grid4, 64, 0, s, a); break;
            default: launch_pdl(stream_collide32x4<3, 2>, grid4, 64, 0, s, a); break;
        }
        return;
    }
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
