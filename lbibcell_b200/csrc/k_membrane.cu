// k_membrane.cu — immersed-boundary and geometry kernels.  Compiled with
// --fmad=false: every FP64 result is bit-identical to the reference.
//
//   force_eval       ForceSolver::calculateForce (ForceSolver.cpp:42-85) over a
//                    per-node CSR of force records in insertion order
//                    (ForceStructs.hpp:49-588).
//   spread           SimulationRunner::distributeForce + GeometryNode::distributeForce
//                    (SimulationRunner.cpp:425-453, GeometryNode.cpp:228-235) as a
//                    deterministic gather: each 16x16 lattice tile collects the
//                    membrane nodes whose 4x4 stencil overlaps it, sorts them by
//                    id and every lattice node sums its contributions in id order
//                    (the reference's serial map order).  No floating-point atomics.
//   interp_move      GeometryNode::collectVelocity (GeometryNode.cpp:216-226, slot
//                    order (4x+y) mod 16 from GeometryHandler.cpp:641), the speed
//                    check (LagrangianPoint.cpp:92-103) and GeometryNode::move
//                    (GeometryNode.cpp:245-254); positions that need the
//                    reference's random perturbation (GeometryNode.cpp:153-214)
//                    are flagged for the host, which owns the generator.
//   crossings        Connection::generateBoundaryNodes / insertBoundaryNode
//                    (Connection.cpp:181-324): every crossing of a connection with
//                    a lattice line is a candidate for one (node, slot); the
//                    closest wins, ties keep the earlier connection.
//   reinit           PhysicalNode::updateDomainIdentifier + CDESolverD2Q5::reinitialise
//                    (PhysicalNode.cpp:109-124, CDESolverD2Q5.cpp:156-228) in
//                    row-major order semantics, processed in dependency rounds.
//   domain_fill      GeometryHandler::updateAllDomainIdentifiers (GeometryHandler.cpp:68-85).
#include <cub/cub.cuh>

#include "kernels.cuh"
#include "lattice_math.cuh"

namespace lbib {

// ---------------------------------------------------------------------------
// fastCos and the Dirac weight: GeometryNode.cpp:55-94.
__device__ __forceinline__ double fast_cos(const double x) {
    const double halfPi = M_PI / 2.0;
    const double doublePi = 2.0 * M_PI;
    double cs;
    double tempx = x + halfPi;
    if (tempx > M_PI) tempx -= doublePi;
    if (tempx < .00) {
        cs = 1.27323954 * tempx + 0.405284735 * tempx * tempx;
    } else {
        cs = 1.27323954 * tempx - 0.405284735 * tempx * tempx;
    }
    if (cs < 0.0) {
        cs = 0.225 * (cs * -cs - cs) + cs;
    } else {
        cs = 0.225 * (cs * cs - cs) + cs;
    }
    return cs;
}

__device__ __forceinline__ double dirac(const double dx, const double dy) {
    const double halfPi = M_PI / 2.0;
    return ((1.0 + fast_cos(halfPi * dx)) * (1.0 + fast_cos(halfPi * dy))) / 16.0;
}

// ---------------------------------------------------------------------------
// Force evaluation
__device__ __forceinline__ int tile_agg_add(int* arr, int tile, bool valid);
__device__ void tile_slot_node(const MembraneDev& m, TileDev& t, int i, bool ok, int nx, int ny, Status* st);

// `begin`: the first kernel of a step (begin_step).
// `slots`: also enter the node in the per-tile lists of the FP32-shifted
// spread (the tile counts were cleared before the launch).
__global__ void force_eval_kernel(MembraneDev m, Status* st, unsigned iteration, int begin, TileDev t, int nx,
                                  int ny, int slots) {
    pdl_wait();
    if (st->halt) return;
    if (begin && blockIdx.x == 0 && threadIdx.x == 0) begin_step(st);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const double x1 = m.x[i], y1 = m.y[i];
    double Fx = 0.0, Fy = 0.0;
    const int r0 = m.foff[i], r1 = m.foff[i + 1];
    for (int r = r0; r < r1; ++r) {
        const int type = m.ftype[r];
        const double* p = m.fpar + 4 * (size_t)r;
        const int j = m.fpartner[r];
        if ((type == 0 || type == 7 || type == 5 || type == 6) && (j < 0 || j >= m.topo->M)) {
            raise_error(st, ERR_FORCE_NODE, i, ST_FORCE);
            return;
        }
        switch (type) {
            case 0: case 7: {  // spring between two nodes: f = k(|d| - l0), along d
                const double x2 = m.x[j], y2 = m.y[j];
                const double dist = sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
                const double f = p[0] * (dist - p[1]);
                Fx += ((x2 - x1) * f) / dist;
                Fy += ((y2 - y1) * f) / dist;
                break;
            }
            case 1: {  // anchor spring to (x, y)
                const double tx = p[0], ty = p[1];
                const double dist = sqrt((tx - x1) * (tx - x1) + (ty - y1) * (ty - y1));
                const double f = p[2] * (dist - p[3]);
                if (dist != 0.0) {
                    Fx += ((tx - x1) * f) / dist;
                    Fy += ((ty - y1) * f) / dist;
                }
                break;
            }
            case 2:  // constant force
                Fx += p[0];
                Fy += p[1];
                break;
            case 3: {  // horizontal slider at y
                const double dist = sqrt((x1 - x1) * (x1 - x1) + (p[0] - y1) * (p[0] - y1));
                const double f = p[1] * (dist - p[2]);
                Fx += 0.0;
                Fy += (y1 < p[0]) ? f : -f;
                break;
            }
            case 4: {  // vertical slider at x
                const double dist = sqrt((p[0] - x1) * (p[0] - x1) + (y1 - y1) * (y1 - y1));
                const double f = p[1] * (dist - p[2]);
                Fx += (x1 < p[0]) ? f : -f;
                Fy += 0.0;
                break;
            }
            default: {  // 5, 6: constant-magnitude pull toward the partner
                const double x2 = m.x[j], y2 = m.y[j];
                const double dist = sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
                Fx += ((x2 - x1) * p[0]) / dist;
                Fy += ((y2 - y1) * p[0]) / dist;
                break;
            }
        }
    }
    m.fx[i] = Fx;
    m.fy[i] = Fy;
    if (slots) tile_slot_node(m, t, i, true, nx, ny, st);
}

// dL/d of every force record's parameters from dL/dF of the node forces
// (the membrane-force gradient of a differentiated run), through the
// record's force as force_eval_kernel forms it (ForceStructs.hpp:49-588):
// each record of node i adds to F_i only, so
// dL/dp = (dL/dF_i) . dF_i/dp, with the positions fixed.  Parameters a type
// does not read get 0.  gpar: 4 per record, in record order.
__global__ void force_param_grad_kernel(MembraneDev m, const double* gfx, const double* gfy, double* gpar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const double x1 = m.x[i], y1 = m.y[i], gx = gfx[i], gy = gfy[i];
    for (int r = m.foff[i]; r < m.foff[i + 1]; ++r) {
        const int type = m.ftype[r];
        const double* p = m.fpar + 4 * (size_t)r;
        const int j = m.fpartner[r];
        double g[4] = {0.0, 0.0, 0.0, 0.0};
        switch (type) {
            case 0: case 7: case 5: case 6: {
                if (j < 0 || j >= m.topo->M) break;
                const double dx = m.x[j] - x1, dy = m.y[j] - y1;
                const double dist = sqrt(dx * dx + dy * dy);
                const double gd = (gx * dx + gy * dy) / dist;  // (dL/dF) . d / |d|
                if (type == 5 || type == 6) {
                    g[0] = gd;                      // F = f d/|d|
                } else {
                    g[0] = (dist - p[1]) * gd;      // F = k (|d| - l0) d/|d|
                    g[1] = -p[0] * gd;
                }
                break;
            }
            case 1: {  // F = k (|d| - l0) d/|d|, d = (tx, ty) - x; none at |d| = 0
                const double dx = p[0] - x1, dy = p[1] - y1;
                const double dist = sqrt(dx * dx + dy * dy);
                if (dist == 0.0) break;
                const double gdd = gx * dx + gy * dy;
                const double a = 1.0 - p[3] / dist, b = p[3] * gdd / (dist * dist * dist);
                g[0] = p[2] * (a * gx + b * dx);  // dF/dtx: k [(1 - l0/|d|) I + l0 d d^T / |d|^3]
                g[1] = p[2] * (a * gy + b * dy);
                g[2] = (dist - p[3]) * gdd / dist;
                g[3] = -p[2] * gdd / dist;
                break;
            }
            case 2:  // F = (fx, fy)
                g[0] = gx;
                g[1] = gy;
                break;
            case 3: case 4: {  // sliders: F_y (3) or F_x (4) = +-k (|c - y| - l0), + below c
                const double pos = type == 3 ? y1 : x1, gc = type == 3 ? gy : gx;
                const double dist = fabs(p[0] - pos);
                const double sgn = pos < p[0] ? 1.0 : -1.0;
                const double dd = p[0] > pos ? 1.0 : (p[0] < pos ? -1.0 : 0.0);  // d|c - pos| / dc
                g[0] = gc * sgn * p[1] * dd;
                g[1] = gc * sgn * (dist - p[2]);
                g[2] = -gc * sgn * p[1];
                break;
            }
            default:
                break;
        }
        for (int q = 0; q < 4; ++q) gpar[4 * (size_t)r + q] = g[q];
    }
}

void launch_force_param_grad(const MembraneDev& m, const double* gfx, const double* gfy, double* gpar,
                             cudaStream_t s) {
    if (m.Mcap == 0) return;
    force_param_grad_kernel<<<(m.Mcap + 127) / 128, 128, 0, s>>>(m, gfx, gfy, gpar);
}

template <typename Real>
void launch_force_eval(const MembraneDev& m, Status* st, unsigned iteration, cudaStream_t s, bool begin,
                       TileDev* tiles, int nx, int ny) {
    if (m.Mcap == 0) return;
    TileDev t{};
    if (tiles) {
        t = *tiles;
        cudaMemsetAsync(t.count, 0, sizeof(int) * (t.nTiles + 1), s);
    }
    launch_pdl(force_eval_kernel, (m.Mcap + 127) / 128, 128, 0, s, m, st, iteration, begin ? 1 : 0, t, nx, ny,
               tiles ? 1 : 0);
}
template void launch_force_eval<double>(const MembraneDev&, Status*, unsigned, cudaStream_t, bool, TileDev*, int,
                                        int);
template void launch_force_eval<float>(const MembraneDev&, Status*, unsigned, cudaStream_t, bool, TileDev*, int,
                                       int);

// ---------------------------------------------------------------------------
// Spreading

// Stencil of a membrane node (GeometryHandler.cpp:613-643): the loop
//   for x in [ceil(X-2), floor(X+2)], for y in [ceil(Y-2), floor(Y+2)]:
//       slot[(4x + y) % 16] = node(x, y)
// binds 16 slots.  The ranges are 4 wide, except when rounding of X+2 or X-2
// makes them 5 wide (e.g. X = 32 - 1 ulp); then later writes replace earlier
// ones with the same slot, and the bound set is what the last writers leave.
struct Stencil {
    int x0, x1, y0, y1;
};

__device__ __forceinline__ bool stencil_range(double X, double Y, int nx, int ny, Stencil& s) {
    s.x0 = (int)ceil(X - 2.0);
    s.y0 = (int)ceil(Y - 2.0);
    s.x1 = (int)floor(X + 2.0);
    s.y1 = (int)floor(Y + 2.0);
    const int wx = s.x1 - s.x0, wy = s.y1 - s.y0;
    return wx >= 3 && wx <= 4 && wy >= 3 && wy <= 4 && s.x0 >= 0 && s.y0 >= 0 && s.x1 < nx && s.y1 < ny;
}

// Is lattice node (x, y) bound by the stencil (the last writer of its slot)?
__device__ __forceinline__ bool in_stencil(const Stencil& s, int x, int y) {
    if (x < s.x0 || x > s.x1 || y < s.y0 || y > s.y1) return false;
    if (s.x1 - s.x0 == 3 && s.y1 - s.y0 == 3) return true;
    const int slot = (4 * x + y) & 15;
    for (int xp = x; xp <= s.x1; ++xp)
        for (int yp = (xp == x ? y + 1 : s.y0); yp <= s.y1; ++yp)
            if (((4 * xp + yp) & 15) == slot) return false;
    return true;
}

// The lattice node bound to slot k (k = 0..15).
__device__ __forceinline__ void stencil_slot(const Stencil& s, int k, int& xk, int& yk) {
    if (s.x1 - s.x0 == 3 && s.y1 - s.y0 == 3) {
        const int base = ((4 * s.x0 + s.y0) % 16 + 16) % 16;
        const int r = (k - base + 16) & 15;
        xk = s.x0 + (r >> 2);
        yk = s.y0 + (r & 3);
        return;
    }
    xk = -1; yk = -1;
    for (int x = s.x0; x <= s.x1; ++x)
        for (int y = s.y0; y <= s.y1; ++y)
            if (((4 * x + y) & 15) == k) { xk = x; yk = y; }
}

// Lanes with the same tile share one atomic.
__device__ __forceinline__ int tile_agg_add(int* arr, int tile, bool valid) {
    const unsigned act = __activemask();
    const unsigned grp = __match_any_sync(act, valid ? tile : -1);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(grp) - 1;
    int base = 0;
    if (valid && lane == leader) base = atomicAdd(&arr[tile], __popc(grp));
    base = __shfl_sync(grp, base, leader);
    return base + __popc(grp & ((1u << lane) - 1u));
}

// FP32-shifted runs: node i into the fixed-size slot lists of the (up to 2 x 2)
// tiles its stencil covers.
__device__ void tile_slot_node(const MembraneDev& m, TileDev& t, int i, bool ok, int nx, int ny, Status* st) {
    Stencil sc{0, 0, 0, 0};
    if (ok && !stencil_range(m.bx[i], m.by[i], nx, ny, sc)) {
        raise_error(st, ERR_STENCIL, i, ST_SPREAD);
        ok = false;
    }
    const int tx0 = sc.x0 / kTile, tx1 = sc.x1 / kTile, ty0 = sc.y0 / kTile, ty1 = sc.y1 / kTile;
    for (int j = 0; j < 4; ++j) {
        const int tx = tx0 + (j & 1), ty = ty0 + (j >> 1);
        const bool v = ok && tx <= tx1 && ty <= ty1;
        const int tile = v ? ty * t.tilesX + tx : -1;
        const int slot = tile_agg_add(t.count, tile, v);
        if (v) {
            if (slot < kTileSlots) t.slots[(size_t)tile * kTileSlots + slot] = i;
            else raise_error(st, ERR_CAPACITY, tile, ST_SPREAD);
        }
    }
}

__global__ void tile_slot_kernel(MembraneDev m, TileDev t, int nx, int ny, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    tile_slot_node(m, t, i, i < m.topo->M, nx, ny, st);
}

__global__ void tile_count_kernel(MembraneDev m, TileDev t, int nx, int ny, Status* st, int pass) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool ok = i < m.topo->M;
    Stencil sc{0, 0, 0, 0};
    if (ok && !stencil_range(m.bx[i], m.by[i], nx, ny, sc)) {
        raise_error(st, ERR_STENCIL, i, ST_SPREAD);
        ok = false;
    }
    const int tx0 = sc.x0 / kTile, tx1 = sc.x1 / kTile, ty0 = sc.y0 / kTile, ty1 = sc.y1 / kTile;
    // up to 2 x 2 tiles per stencil; all lanes run the four rounds together
    for (int j = 0; j < 4; ++j) {
        const int tx = tx0 + (j & 1), ty = ty0 + (j >> 1);
        const bool v = ok && tx <= tx1 && ty <= ty1;
        const int tile = v ? ty * t.tilesX + tx : -1;
        if (pass == 0) {
            tile_agg_add(t.count, tile, v);
        } else {
            const int slot = tile_agg_add(t.fill, tile, v);
            if (v) {
                const int pos = t.start[tile] + slot;
                if (pos < t.cap) t.list[pos] = i;
            }
        }
    }
}

// Membrane stencils per tile held in shared memory: most tiles hold fewer than
// kSpreadSmall; the others go to the kSpreadLarge variant.
constexpr int kSpreadSmall = 256;
constexpr int kSpreadLarge = 768;
constexpr size_t spread_smem(int cap) {
    return (size_t)cap * (12 * sizeof(double) + 2 * sizeof(int) + 8 * sizeof(unsigned short));
}

// Per-tile entry: the stencil origin relative to the tile (+4) and the stencil
// widths, packed in one word: ox | oy << 8 | (x1-x0) << 16 | (y1-y0) << 20.
__device__ __forceinline__ int pack_stencil(const Stencil& s, int tileX0, int tileY0) {
    return (s.x0 - tileX0 + 4) | ((s.y0 - tileY0 + 4) << 8) | ((s.x1 - s.x0) << 16) | ((s.y1 - s.y0) << 20);
}

// Sorts the tile's membrane indices ascending (= id order) into `out`.
template <int ITEMS>
__device__ __forceinline__ void sort_tile_list(const int* list, int cnt, int sortBits, int* out, void* tmp) {
    typedef cub::BlockRadixSort<int, 256, ITEMS> Sort;
    int keys[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int k = threadIdx.x * ITEMS + j;
        keys[j] = k < cnt ? list[k] : 0x7fffffff;
    }
    Sort(*(typename Sort::TempStorage*)tmp).Sort(keys, 0, sortBits);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int k = threadIdx.x * ITEMS + j;
        if (k < cnt) out[k] = keys[j];
    }
}

// Each 16x16 tile: its membrane nodes sorted by id; per node the Dirac factors
// A_i = 1 + fastCos(pi/2 (x0 + i - X)) and B_j = 1 + fastCos(pi/2 (y0 + j - Y)),
// so that the weight of lattice node (x0+i, y0+j) is (A_i * B_j) / 16, the same
// expression as calculateDiscreteDeltaDirac (GeometryNode.cpp:89-94).  Each warp
// covers two rows of the tile and first collects, in id order, the entries
// whose stencil rows meet its rows; every lattice node then adds its
// contributions in id order.
// Used by FP64 runs, whose summation order must be the reference's.
template <typename Real, int kSpreadMax, int kMinCount>
__global__ void __launch_bounds__(256) spread_kernel(MembraneDev m, TileDev t, Real* force, int nx, int ny, size_t L,
                                                     Status* st, int sortBits) {
    pdl_wait();
    if (st->halt) return;
    const int tile = blockIdx.x;
    const int cnt = t.count[tile];
    // each size class handles the tiles whose count it fits best
    if (cnt == 0 || cnt < kMinCount || (kMinCount == 0 && cnt > kSpreadMax)) return;
    if (cnt > kSpreadMax || t.start[tile] + cnt > t.cap) {
        if (threadIdx.x == 0) raise_error(st, ERR_CAPACITY, tile, ST_SPREAD);
        return;
    }
    extern __shared__ __align__(16) unsigned char smem[];
    double* fac = (double*)smem;                          // kSpreadMax x 10: A[5], B[5]
    double* sfx = fac + 10 * kSpreadMax;
    double* sfy = sfx + kSpreadMax;
    int* code = (int*)(sfy + kSpreadMax);
    int* order = code + kSpreadMax;                      // sorted membrane indices
    unsigned short* wlist = (unsigned short*)(order + kSpreadMax);  // 8 warps x kSpreadMax
    __shared__ __align__(16) unsigned char sortTmp[sizeof(typename cub::BlockRadixSort<int, 256, (kSpreadMax + 255) / 256>::TempStorage)];
    const int* list = t.list + t.start[tile];
    if (kSpreadMax <= 256 || cnt <= 256) sort_tile_list<1>(list, cnt, sortBits, order, sortTmp);
    else if (kSpreadMax <= 512 || cnt <= 512) sort_tile_list<2>(list, cnt, sortBits, order, sortTmp);
    else sort_tile_list<(kSpreadMax + 255) / 256>(list, cnt, sortBits, order, sortTmp);
    __syncthreads();
    const int tx = tile % t.tilesX, ty = tile / t.tilesX;
    const int tileX0 = tx * kTile, tileY0 = ty * kTile;
    const double halfPi = M_PI / 2.0;
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
        const int i = order[k];
        const double X = m.x[i], Y = m.y[i];
        sfx[k] = m.fx[i];
        sfy[k] = m.fy[i];
        Stencil sc;
        stencil_range(m.bx[i], m.by[i], nx, ny, sc);
        code[k] = pack_stencil(sc, tileX0, tileY0);
        double* f = fac + 10 * k;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            f[q] = 1.0 + fast_cos(halfPi * ((double)(sc.x0 + q) - X));
            f[5 + q] = 1.0 + fast_cos(halfPi * ((double)(sc.y0 + q) - Y));
        }
    }
    __syncthreads();
    // per-warp list of the entries whose stencil rows meet the warp's rows
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wy0 = (warp << 1) + 4;  // local rows + 4
    unsigned short* wl = wlist + warp * kSpreadMax;
    int wn = 0;
    for (int k0 = 0; k0 < cnt; k0 += 32) {
        const int k = k0 + lane;
        bool rel = false;
        if (k < cnt) {
            const int c = code[k];
            const int oy = (c >> 8) & 0xff, hy = (c >> 20) & 0xf;
            rel = !(oy + hy < wy0 || oy > wy0 + 1);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, rel);
        if (rel) wl[wn + __popc(bal & ((1u << lane) - 1u))] = (unsigned short)k;
        wn += __popc(bal);
    }
    __syncwarp();
    const int lx = lane & 15, ly = threadIdx.x >> 4;
    const int x = tileX0 + lx, y = tileY0 + ly;
    double ax = 0.0, ay = 0.0;
    for (int e = 0; e < wn; ++e) {
        const int k = wl[e];
        const int c = code[k];
        const int ox = c & 0xff, oy = (c >> 8) & 0xff, hx = (c >> 16) & 0xf, hy = (c >> 20) & 0xf;
        const int dx = lx + 4 - ox, dy = ly + 4 - oy;
        bool hit;
        if (hx == 3 && hy == 3) {
            hit = (unsigned)dx < 4u && (unsigned)dy < 4u;
        } else {
            Stencil sc{ox - 4 + tileX0, ox - 4 + tileX0 + hx, oy - 4 + tileY0, oy - 4 + tileY0 + hy};
            hit = in_stencil(sc, x, y);
        }
        if (hit) {
            const double* f = fac + 10 * k;
            const double dl = (f[dx] * f[5 + dy]) / 16.0;
            ax += sfx[k] * dl;
            ay += sfy[k] * dl;
        }
    }
    if (x >= nx || y >= ny) return;
    const size_t n = (size_t)y * nx + x;
    force[n] = (Real)ax;
    force[L + n] = (Real)ay;
}

// FP32-shifted runs: each 16x16 tile scatters the contributions of the
// membrane nodes listed for it into 64-bit fixed-point accumulators (2^-44) in
// shared memory.  Each contribution dirac * F_i is formed in FP64 exactly as in
// the ordered gather and rounded once; the integer sums are exact, so the
// field does not depend on the order of the list (it is deterministic) and no
// sort is needed.  The rounding is far below FP32 resolution.
constexpr double kForceFix = 17592186044416.0;  // 2^44
constexpr int kScatterChunk = 256;
__global__ void __launch_bounds__(256) spread_fixed_kernel(MembraneDev m, TileDev t, float* force, int nx, int ny,
                                                           size_t L, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int tile = blockIdx.x;
    const int cnt = min(t.count[tile], kTileSlots);
    if (cnt == 0) return;
    // each 64-bit fixed-point sum is kept as a signed high part (bits 22..63)
    // and an unsigned low part (bits 0..21), each summed with 32-bit integer
    // atomics: the low parts of up to 1024 contributions cannot overflow
    __shared__ int accHi[2][kTile * kTile];
    __shared__ unsigned accLo[2][kTile * kTile];
    __shared__ double fa[kScatterChunk][5], fb[kScatterChunk][5], sF[2][kScatterChunk];
    __shared__ int org[kScatterChunk];
    for (int j = threadIdx.x; j < kTile * kTile; j += blockDim.x) {
        accHi[0][j] = accHi[1][j] = 0;
        accLo[0][j] = accLo[1][j] = 0u;
    }

    const int tx = tile % t.tilesX, ty = tile / t.tilesX;
    const int tileX0 = tx * kTile, tileY0 = ty * kTile;
    const int* list = t.slots + (size_t)tile * kTileSlots;
    const double halfPi = M_PI / 2.0;
    for (int c0 = 0; c0 < cnt; c0 += kScatterChunk) {
        const int nc = min(kScatterChunk, cnt - c0);
        __syncthreads();
        for (int e = threadIdx.x; e < nc; e += blockDim.x) {
            const int i = list[c0 + e];
            const double X = m.x[i], Y = m.y[i];
            Stencil sc;
            stencil_range(m.bx[i], m.by[i], nx, ny, sc);
            org[e] = pack_stencil(sc, tileX0, tileY0);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                fa[e][q] = 1.0 + fast_cos(halfPi * ((double)(sc.x0 + q) - X));
                fb[e][q] = 1.0 + fast_cos(halfPi * ((double)(sc.y0 + q) - Y));
            }
            sF[0][e] = m.fx[i];
            sF[1][e] = m.fy[i];
        }
        __syncthreads();
        // one item per (node, slot row r): slots k = 4 r .. 4 r + 3 of the
        // node's 16 (in a 4 x 4 stencil, column dx = r, rows dy = 0..3)
        for (int j = threadIdx.x; j < 4 * nc; j += blockDim.x) {
            const int e = j >> 2, r = j & 3;
            const int c = org[e];
            const int ox = (c & 0xff) - 4, oy = ((c >> 8) & 0xff) - 4, hx = (c >> 16) & 0xf, hy = (c >> 20) & 0xf;
            const bool plain = hx == 3 && hy == 3;
            if (plain && (unsigned)(ox + r) >= (unsigned)kTile) continue;  // the column lies outside the tile
            const Stencil sc{ox + tileX0, ox + tileX0 + hx, oy + tileY0, oy + tileY0 + hy};
            const double Fx = sF[0][e], Fy = sF[1][e];
#pragma unroll
            for (int t4 = 0; t4 < 4; ++t4) {
                int dx, dy;  // node of slot k relative to the stencil origin
                if (plain) {
                    dx = r;
                    dy = t4;
                } else {
                    // wider stencil: the node bound to slot k (last writer of the slot)
                    int xk, yk;
                    stencil_slot(sc, 4 * r + t4, xk, yk);
                    if (xk < 0) continue;
                    dx = xk - sc.x0;
                    dy = yk - sc.y0;
                }
                const int lx = ox + dx, ly = oy + dy;
                if ((unsigned)lx >= (unsigned)kTile || (unsigned)ly >= (unsigned)kTile) continue;
                const double dl = (fa[e][dx] * fb[e][dy]) / 16.0;
                const long long vx = __double2ll_rn(Fx * dl * kForceFix);
                const long long vy = __double2ll_rn(Fy * dl * kForceFix);
                const int node = ly * kTile + lx;
                atomicAdd(&accHi[0][node], (int)(vx >> 22));
                atomicAdd(&accLo[0][node], (unsigned)(vx & 0x3fffff));
                atomicAdd(&accHi[1][node], (int)(vy >> 22));
                atomicAdd(&accLo[1][node], (unsigned)(vy & 0x3fffff));
            }
        }
    }
    __syncthreads();
    const int lx = threadIdx.x & 15, ly = threadIdx.x >> 4;
    const int x = tileX0 + lx, y = tileY0 + ly;
    if (x >= nx || y >= ny) return;
    const size_t n = (size_t)y * nx + x;
    const long long sx = (long long)accHi[0][threadIdx.x] * (1ll << 22) + (long long)accLo[0][threadIdx.x];
    const long long sy = (long long)accHi[1][threadIdx.x] * (1ll << 22) + (long long)accLo[1][threadIdx.x];
    force[n] = (float)((double)sx * (1.0 / kForceFix));
    force[L + n] = (float)((double)sy * (1.0 / kForceFix));
}

template <typename Real>
void launch_spread(const MembraneDev& m, TileDev& t, Real* force, int nx, int ny, size_t L, Status* st,
                   unsigned iteration, cudaStream_t s, bool slotsFilled) {
    if (!slotsFilled) cudaMemsetAsync(t.count, 0, sizeof(int) * (t.nTiles + 1), s);
    if (m.Mcap == 0) return;
    const int blocks = (m.Mcap + 127) / 128;
    if constexpr (sizeof(Real) == 4) {
        // one pass into fixed per-tile slots (done by the force kernel when
        // slotsFilled), then the fixed-point scatter
        if (!slotsFilled) launch_pdl(tile_slot_kernel, blocks, 128, 0, s, m, t, nx, ny, st);
        launch_pdl(spread_fixed_kernel, t.nTiles, 256, 0, s, m, t, (float*)force, nx, ny, L, st);
    } else {
        // exact lists (count, scan, fill), then the ordered gather
        cudaMemsetAsync(t.fill, 0, sizeof(int) * t.nTiles, s);
        launch_pdl(tile_count_kernel, blocks, 128, 0, s, m, t, nx, ny, st, 0);
        cub::DeviceScan::ExclusiveSum(t.scanTmp, t.scanTmpBytes, t.count, t.start, t.nTiles + 1, s);
        launch_pdl(tile_count_kernel, blocks, 128, 0, s, m, t, nx, ny, st, 1);
        int bits = 1;
        while ((1 << bits) < m.Mcap + 1 && bits < 31) ++bits;
        launch_pdl(spread_kernel<Real, kSpreadSmall, 0>, t.nTiles, 256, spread_smem(kSpreadSmall), s, m, t, force, nx,
                   ny, L, st, bits);
        launch_pdl(spread_kernel<Real, kSpreadLarge, kSpreadSmall + 1>, t.nTiles, 256, spread_smem(kSpreadLarge), s, m,
                   t, force, nx, ny, L, st, bits);
    }
}
template void launch_spread<double>(const MembraneDev&, TileDev&, double*, int, int, size_t, Status*, unsigned,
                                    cudaStream_t, bool);
template void launch_spread<float>(const MembraneDev&, TileDev&, float*, int, int, size_t, Status*, unsigned,
                                   cudaStream_t, bool);

// ---------------------------------------------------------------------------
// Interpolation and motion

__device__ __forceinline__ bool needs_perturbation(double X, double Y) {
    // The four tests of GeometryNode::perturbatePosition (GeometryNode.cpp:160, 174, 189, 202).
    if (fabs((double)(int)X - X) <= kEPSILON) return true;
    if (fabs((double)(int)Y - Y) <= kEPSILON) return true;
    if (fabs(Y - floor(Y) - (X - floor(X))) <= kEPSILON) return true;
    if (fabs(ceil(Y) - Y - (X - floor(X))) <= kEPSILON) return true;
    return false;
}

template <typename Real>
__global__ void interp_move_kernel(MembraneDev m, const Real* u, int nx, int ny, size_t L, CrossDev c, Status* st,
                                   unsigned iteration) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const double X = m.x[i], Y = m.y[i];
    Stencil sc;
    if (!stencil_range(m.bx[i], m.by[i], nx, ny, sc)) {
        raise_error(st, ERR_STENCIL, i, ST_INTERP_MOVE);
        return;
    }
    // the Dirac factors of the stencil's columns and rows, each formed once:
    // (fa * fb) / 16 is calculateDiscreteDeltaDirac's expression
    const double halfPi = M_PI / 2.0;
    double fa[5], fb[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        fa[q] = 1.0 + fast_cos(halfPi * ((double)(sc.x0 + q) - X));
        fb[q] = 1.0 + fast_cos(halfPi * ((double)(sc.y0 + q) - Y));
    }
    auto pick = [](const double* v, int i) {
        return i == 0 ? v[0] : i == 1 ? v[1] : i == 2 ? v[2] : i == 3 ? v[3] : v[4];
    };
    double vx = 0.0, vy = 0.0;
    for (int k = 0; k < 16; ++k) {
        int xk, yk;
        stencil_slot(sc, k, xk, yk);
        const size_t n = (size_t)yk * nx + xk;
        const double dl = (pick(fa, xk - sc.x0) * pick(fb, yk - sc.y0)) / 16.0;
        vx += (double)u[n] * dl;
        vy += (double)u[L + n] * dl;
    }
    m.vx[i] = vx;
    m.vy[i] = vy;
    const double CS = 1 / sqrt(3.0);
    if (((vx * vx) + (vy * vy)) > CS) {
        raise_error(st, ERR_SPEED, i, ST_INTERP_MOVE);
        return;
    }
    m.ox[i] = X;
    m.oy[i] = Y;
    const double Xn = X + vx, Yn = Y + vy;
    m.x[i] = Xn;
    m.y[i] = Yn;
    if (needs_perturbation(Xn, Yn)) {
        const int k = atomicAdd(&st->nPerturbNode, 1);
        if (k < c.perturbCap) c.perturbList[k] = i;
        raise_halt(st, ST_INTERP_MOVE);
    }
}

template <typename Real>
void launch_interp_move(const MembraneDev& m, const Real* u, int nx, int ny, size_t L, CrossDev& c, Status* st,
                        unsigned iteration, cudaStream_t s) {
    if (m.Mcap == 0) return;
    launch_pdl(interp_move_kernel<Real>, (m.Mcap + 127) / 128, 128, 0, s, m, u, nx, ny, L, c, st, iteration);
}
template void launch_interp_move<double>(const MembraneDev&, const double*, int, int, size_t, CrossDev&, Status*,
                                         unsigned, cudaStream_t);
template void launch_interp_move<float>(const MembraneDev&, const float*, int, int, size_t, CrossDev&, Status*,
                                        unsigned, cudaStream_t);

// Adjoint of the spread for a differentiated run with frozen positions.  The
// spread adds dirac(x - X_i) * F_i to every lattice node x of node i's stencil
// (GeometryNode::distributeForce, GeometryNode.cpp:228-235), so
// dL/dF_i = sum over the same 16 slots of dirac * dL/dF(x): the interpolation
// of collectVelocity (GeometryNode.cpp:216-226) applied to G = dL/dF.
__global__ void force_adjoint_kernel(MembraneDev m, const double* G, int nx, int ny, size_t L, double* gfx,
                                     double* gfy) {
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const double X = m.x[i], Y = m.y[i];
    Stencil sc;
    double gx = 0.0, gy = 0.0;
    if (stencil_range(m.bx[i], m.by[i], nx, ny, sc)) {
        for (int k = 0; k < 16; ++k) {
            int xk, yk;
            stencil_slot(sc, k, xk, yk);
            const size_t n = (size_t)yk * nx + xk;
            const double dl = dirac((double)xk - X, (double)yk - Y);
            gx += G[n] * dl;
            gy += G[L + n] * dl;
        }
    }
    gfx[i] = gx;
    gfy[i] = gy;
}

void launch_force_adjoint(const MembraneDev& m, const double* G, int nx, int ny, size_t L, double* gfx,
                          double* gfy, cudaStream_t s) {
    if (m.Mcap == 0) return;
    launch_pdl(force_adjoint_kernel, (m.Mcap + 127) / 128, 128, 0, s, m, G, nx, ny, L, gfx, gfy);
}

// Connection::perturbConnection's tests (Connection.cpp:339, 363).
// Connections whose end points share an x or a y to within EPSILON
// (Connection::perturbConnection's tests, Connection.cpp:339-340, 363-364) are
// counted and listed (up to cap); the crossing kernel, the next, raises the
// halt, so that every block here sees the same halt word and the list is
// complete.
__global__ void perturb_conn_kernel(MembraneDev m, Status* st, int* list, int cap) {
    pdl_wait();
    if (st->halt) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.topo->C) return;
    const int a = m.ca[c], b = m.cb[c];
    if (fabs(m.x[a] - m.x[b]) < kEPSILON || fabs(m.y[a] - m.y[b]) < kEPSILON) {
        const int k = atomicAdd(&st->nPerturbConn, 1);
        if (k < cap) list[k] = c;
    }
}

void launch_perturb_conn_check(const MembraneDev& m, Status* st, unsigned iteration, cudaStream_t s, int* list,
                               int cap) {
    if (m.Ccap == 0) return;
    launch_pdl(perturb_conn_kernel, (m.Ccap + 127) / 128, 128, 0, s, m, st, list, cap);
}

// ---------------------------------------------------------------------------
// Crossings: three passes over the connections.
//   pass 0: closest distance per (node, slot) by atomicMin on the distance bits
//           (non-negative doubles order like their bit patterns);
//   pass 1: among records at that distance, the earliest connection;
//   pass 2: the winner writes its domain; the winner of a node's last present
//           slot (order E,N,W,S = the reference's boundaryNodes_ scan order)
//           decides the node's tentative domain (PhysicalNode.cpp:111-115).
constexpr unsigned long long kEmpty = ~0ull;

__device__ __forceinline__ int slot_code(int d) {  // E,N,W,S -> 0..3
    return d - 1;
}

// Pass 0: every crossing of a connection with a lattice line is a candidate
// boundary node for one (node, slot) key.  The closest distance per key is
// found by atomicMin on the distance's bits; each candidate is recorded for
// passes 1 and 2 and for the reset of its key at the end of the step.  A warp
// reserves its records with one atomic.  A connection may be long (the
// cut across a cell that a division adds, until remeshing splits it): the
// loops run over the lattice lines between its end points, which the bounds
// test below keeps on the lattice.

struct CrossRec {
    uint32_t key;
    uint32_t dom;
    unsigned long long bits;
};

__device__ __forceinline__ bool make_record(int nx, int ny, int px, int py, int dirSlot, double bx, double by,
                                            uint32_t bdom, CrossRec& r) {
    if (px < 0 || py < 0 || px >= nx || py >= ny) return false;
    const size_t node = (size_t)py * nx + px;
    const double d2 = ((double)px - bx) * ((double)px - bx) + ((double)py - by) * ((double)py - by);
    r.bits = (unsigned long long)__double_as_longlong(d2);
    r.key = (uint32_t)(node * 4 + slot_code(dirSlot));
    r.dom = bdom;
    return true;
}

// Exclusive prefix of `count` over the active lanes plus one atomicAdd per warp.
__device__ __forceinline__ int warp_reserve(int* counter, int count) {
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;
    int incl = count;
    for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(act, incl, off);
        if (lane >= off && ((act >> (lane - off)) & 1u)) incl += v;
    }
    const int last = 31 - __clz(act);
    const int total = __shfl_sync(act, incl, last);
    const int leader = __ffs(act) - 1;
    int base = 0;
    if (lane == leader && total > 0) base = atomicAdd(counter, total);
    base = __shfl_sync(act, base, leader);
    return base + incl - count;
}

// Calls fn(k, record) for the candidate records of connection cn in a fixed
// order (k = 0, 1, ...); returns the number of records, or -1 after raising
// the error of a connection that cannot be processed.  The kernel enumerates
// three times (count, emit, list first writers) so that no per-thread record
// array is needed.
template <class Fn>
__device__ __forceinline__ int for_each_record(const MembraneDev& m, int cn, int nx, int ny, Status* st, bool report,
                                               Fn fn) {
    const int a = m.ca[cn], b = m.cb[cn];
    const double x1 = m.x[a], y1 = m.y[a], x2 = m.x[b], y2 = m.y[b];
    const uint32_t D = m.cdom[cn];
    const double maxX = x1 < x2 ? x2 : x1, maxY = y1 < y2 ? y2 : y1;
    const double minX = x2 < x1 ? x2 : x1, minY = y2 < y1 ? y2 : y1;
    const double mm = (y2 - y1) / (x2 - x1);
    const double nn = y1 - (y2 - y1) / (x2 - x1) * x1;
    if (!isfinite(mm)) {
        if (report) raise_error(st, ERR_VERTICAL, cn, ST_CROSSINGS);
        return -1;
    }
    if (!(minX >= -1.0 && maxX <= nx + 1.0 && minY >= -1.0 && maxY <= ny + 1.0)) {
        // keeps the line loops bounded for positions off the lattice
        if (report) raise_error(st, ERR_EDGE_W, cn, ST_CROSSINGS);
        return -1;
    }
    const bool eastward = x1 < x2, southward = y1 > y2;
    int k = 0;
    CrossRec r;
    for (int i = (int)ceil(minX); i <= (int)floor(maxX); i++) {
        const double yc = mm * i + nn;
        // fluidS gets its N slot, fluidN its S slot (Connection.cpp:273-279)
        if (!make_record(nx, ny, i, (int)floor(yc), N, (double)i, yc, eastward ? 0u : D, r)) break;
        fn(k++, r);
        if (!make_record(nx, ny, i, (int)ceil(yc), S, (double)i, yc, eastward ? D : 0u, r)) break;
        fn(k++, r);
    }
    for (int i = (int)ceil(minY); i <= (int)floor(maxY); i++) {
        const double xc = (i - nn) / mm;
        // fluidW gets its E slot, fluidE its W slot (Connection.cpp:307-313)
        if (!make_record(nx, ny, (int)floor(xc), i, E, xc, (double)i, southward ? 0u : D, r)) break;
        fn(k++, r);
        if (!make_record(nx, ny, (int)ceil(xc), i, W, xc, (double)i, southward ? D : 0u, r)) break;
        fn(k++, r);
    }
    const int want = 2 * (max(0, (int)floor(maxX) - (int)ceil(minX) + 1) + max(0, (int)floor(maxY) - (int)ceil(minY) + 1));
    if (k != want) {
        if (report) raise_error(st, ERR_EDGE_W, cn, ST_CROSSINGS);
        return -1;
    }
    return k;
}

__global__ void crossings_kernel(MembraneDev m, CrossDev c, int nx, int ny, Status* st) {
    pdl_wait();
    if (st->halt) return;
    if (st->nPerturbConn > 0) {
        // connections to perturb first (perturb_conn_kernel): the host does it
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_halt(st, ST_PERTURB_CONN);
        return;
    }
    const int cn = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = cn < m.topo->C;
    int nrec = 0;
    if (live) {
        nrec = for_each_record(m, cn, nx, ny, st, true, [](int, const CrossRec&) {});
        if (nrec < 0) nrec = 0;
    }
    // records of this step (they also list the keys to reset at the end of
    // the step) and the closest distance per key
    const int rb = warp_reserve(&st->pad[2], nrec);
    if (nrec > 0) {
        for_each_record(m, cn, nx, ny, st, false, [&](int k, const CrossRec& r) {
            const int idx = rb + k;
            if (idx < c.recCap) {
                c.recKey[idx] = r.key; c.recConn[idx] = (uint32_t)cn; c.recDom[idx] = r.dom; c.recDist[idx] = r.bits;
            } else {
                raise_error(st, ERR_CAPACITY, cn, ST_CROSSINGS);
            }
            atomicMin(&c.bnDist[r.key], r.bits);
        });
    }
}

// Pass 1: among records at the closest distance, the earliest connection.
__global__ void cross_tie_kernel(CrossDev c, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int n = min(st->pad[2], c.recCap);
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t key = c.recKey[r];
        if (c.bnDist[key] == c.recDist[r]) atomicMin(&c.bnConn[key], c.recConn[r]);
    }
}

// Pass 2: the winner writes its domain; the winner of a node's last present
// slot (order E,N,W,S = the reference's boundaryNodes_ scan order) decides the
// node's tentative domain (PhysicalNode.cpp:111-115).
// The boundary node of a winning record whose connection carries boundary
// solvers: its position on the lattice line (BoundaryNode(i, getYPos(m, i, n))
// or BoundaryNode(getXPos(m, i, n), i), Connection.cpp:243-312) and its
// velocity, interpolated along the connection (Connection::calculateVelocity,
// Connection.cpp:146-168), kept for the next step's no-flux solvers.
__device__ __forceinline__ void record_noflux(const MembraneDev& m, CrossDev& c, int conn, uint32_t key, int nx) {
    const int desc = m.cdesc[conn];
    if (desc < 0 || c.nfTab[desc].nSolvers == 0) return;
    const int a = m.ca[conn], b = m.cb[conn];
    const double x1 = m.x[a], y1 = m.y[a], x2 = m.x[b], y2 = m.y[b];
    const double mm = (y2 - y1) / (x2 - x1);
    const double nn = y1 - (y2 - y1) / (x2 - x1) * x1;
    const size_t node = key >> 2;
    const int s = (int)(key & 3u);  // E, N, W, S
    const int px = (int)(node % (size_t)nx), py = (int)(node / (size_t)nx);
    double bx, by;
    if (s == 1 || s == 3) {  // N / S slot: a crossing with the vertical line x = px
        bx = (double)px;
        by = mm * px + nn;
    } else {                 // E / W slot: a crossing with the horizontal line y = py
        bx = (py - nn) / mm;
        by = (double)py;
    }
    const double l = sqrt((x1 - bx) * (x1 - bx) + (y1 - by) * (y1 - by));
    const double Lc = sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    const double vx1 = m.vx[a], vy1 = m.vy[a], vx2 = m.vx[b], vy2 = m.vy[b];
    c.nfU[2 * (size_t)key] = (vx2 - vx1) * l / Lc + vx1;
    c.nfU[2 * (size_t)key + 1] = (vy2 - vy1) * l / Lc + vy1;
    c.nfSpec[key] = (uint8_t)(desc + 1);
    const int k = atomicAdd(c.nfN, 1);
    if (k < c.nfCap) c.nfKeys[k] = key;
}

// GeometryHandler::connectGeometryNodesToPhysicalNodes for one node
// (GeometryHandler.cpp:608-644): a node that left its previous unit cell
// (GeometryNode::isUpdateNeeded, GeometryNode.cpp:256-261, Rectangle.cpp
// pointWithinBounds) is bound again from its current position, after the
// edge test; the others keep their binding.
__device__ __forceinline__ void edge_check_node(const MembraneDev& m, int i, int nx, int ny, Status* st, int stage) {
    const double X = m.x[i], Y = m.y[i], ox = m.ox[i], oy = m.oy[i];
    const bool within = (X >= floor(ox)) && (X < ceil(ox)) && (Y <= ceil(oy)) && (Y > floor(oy));
    if (within) return;
    m.bx[i] = X;
    m.by[i] = Y;
    if (X - 2.0 < 0) raise_error(st, ERR_EDGE_W, i, stage);
    else if (Y - 2.0 < 0) raise_error(st, ERR_EDGE_S, i, stage);
    else if (X + 2.0 > nx) raise_error(st, ERR_EDGE_E, i, stage);
    else if (Y + 2.0 > ny) raise_error(st, ERR_EDGE_N, i, stage);
}

__global__ void cross_win_kernel(CrossDev c, MembraneDev m, const uint32_t* dom, int nx, int ny, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int n = min(st->pad[2], c.recCap);
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t key = c.recKey[r];
        if (c.bnDist[key] != c.recDist[r] || c.bnConn[key] != c.recConn[r]) continue;
        const uint32_t bdom = c.recDom[r];
        const size_t node = key >> 2;
        const int s = (int)(key & 3u);
        c.bnDom[key] = bdom;
        if (c.nfTab != nullptr) record_noflux(m, c, (int)c.recConn[r], key, nx);
        if (c.bounceW != nullptr && s >= 2) {
            // DiracD2Q5's advect skips the swap with the W / S neighbour when
            // this node has a boundary node there (DiracD2Q5.cpp:166-180)
            (s == 2 ? c.bounceW : c.bounceS)[node] = 1;
            const int k = atomicAdd(c.bounceN, 1);
            if (k < c.bounceCap) c.bounceKeys[k] = key;
            else raise_error(st, ERR_CAPACITY, (int)node, ST_CROSSINGS);
        }
        if (s == 2) c.wDom[node] = bdom + 1;
        bool last = true;
        for (int s2 = s + 1; s2 < 4; ++s2)
            if (c.bnDist[node * 4 + s2] != kEmpty) last = false;
        if (last && bdom != dom[node]) {
            const int k = atomicAdd(&st->nChanged, 1);
            if (k < c.changedCap) {
                c.changedNode[k] = (uint32_t)node;
                c.changedDom[k] = bdom;
                c.mark[node] = k + 1;  // the node's position in the list, for the re-initialisation
            } else {
                raise_error(st, ERR_CAPACITY, (int)node, ST_CROSSINGS);
            }
        }
    }
    // GeometryHandler::connectGeometryNodesToPhysicalNodes' edge test of the
    // moved nodes, over the same grid
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.topo->M; i += gridDim.x * blockDim.x)
        edge_check_node(m, i, nx, ny, st, ST_CROSSINGS);
}

// Clears the previous step's no-flux boundary nodes (after the stream-collide
// that used them, before this step's crossings set the new ones).
__global__ void noflux_reset_kernel(CrossDev c) {
    pdl_wait();
    const int n = min(*c.nfN, c.nfCap);
    for (int k = threadIdx.x; k < n; k += blockDim.x) c.nfSpec[c.nfKeys[k]] = 0;
    __syncthreads();
    if (threadIdx.x == 0) *c.nfN = 0;
}

// Clears the previous step's W / S boundary-node marks (after the
// stream-collide that used them, before this step's crossings set new ones).
__global__ void bounce_reset_kernel(CrossDev c) {
    pdl_wait();
    const int n = min(*c.bounceN, c.bounceCap);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const uint32_t key = c.bounceKeys[k];
        ((key & 3u) == 2u ? c.bounceW : c.bounceS)[key >> 2] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) *c.bounceN = 0;
}

// GeometryHandler::connectGeometryNodesToPhysicalNodes' edge test for nodes
// that left their previous unit cell (GeometryHandler.cpp:610-636,
// GeometryNode.cpp:256-261, Rectangle.cpp pointWithinBounds).
__global__ void edge_check_kernel(MembraneDev m, int nx, int ny, Status* st, int stage) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    edge_check_node(m, i, nx, ny, st, stage);
}

template <typename Real>
void launch_crossings(const MembraneDev& m, CrossDev& c, const uint32_t* dom, int nx, int ny, size_t L, Status* st,
                      unsigned iteration, cudaStream_t s) {
    if (m.Ccap == 0) return;
    const int blocks = (m.Ccap + 127) / 128;
    if (c.nfTab != nullptr) launch_pdl(noflux_reset_kernel, 1, 1024, 0, s, c);
    if (c.bounceW != nullptr) launch_pdl(bounce_reset_kernel, 1, 1024, 0, s, c);
    // the record count (st->pad[2]) is zero here: cleared with the status
    // word before a run and by the first kernel of each step
    launch_pdl(crossings_kernel, blocks, 128, 0, s, m, c, nx, ny, st);
    // grid-stride over the step's records (their count is known on the device
    // only): 8 blocks per SM, so that each thread's chain of dependent loads
    // overlaps many others
    launch_pdl(cross_tie_kernel, 148 * 8, 256, 0, s, c, st);
    launch_pdl(cross_win_kernel, 148 * 8, 256, 0, s, c, m, dom, nx, ny, st);
}
template void launch_crossings<double>(const MembraneDev&, CrossDev&, const uint32_t*, int, int, size_t, Status*,
                                       unsigned, cudaStream_t);
template void launch_crossings<float>(const MembraneDev&, CrossDev&, const uint32_t*, int, int, size_t, Status*,
                                      unsigned, cudaStream_t);

void launch_edge_check(const MembraneDev& m, int nx, int ny, Status* st, unsigned iteration, cudaStream_t s) {
    if (m.Mcap == 0) return;
    launch_pdl(edge_check_kernel, (m.Mcap + 127) / 128, 128, 0, s, m, nx, ny, st, ST_REMESH);
}

// ---------------------------------------------------------------------------
// Reinitialisation of the species at nodes whose domain changed.
//
// The reference visits all lattice nodes in row-major order; a changed node
// takes its new domain and re-initialises from its E,N,W,S neighbours of the
// same domain that have no boundary node on the link, reading neighbours that
// come earlier in the order with their new state and later ones with their old
// state.  Here one block sorts the changed nodes, records for each the earlier
// changed nodes among its E,N,W,S,NE (read after write) and SW (write after
// read) neighbours, and processes nodes in rounds once those are done.
constexpr int kReinitMax = 4096;  // changed nodes per step (dynamic shared memory)
constexpr size_t kReinitSmem = (size_t)kReinitMax * (sizeof(unsigned long long) + 8 * sizeof(int) + 1) + 16;

template <typename Real>
__device__ void reinit_node(size_t n, uint32_t newDom, uint32_t* dom, Real* g, const Real* u, int nS,
                            const SpeciesConst* sp, const double* srcTab, int nDomains, const uint32_t* ctypeTab,
                            int cellTypesCopied, const CrossDev& c, int nx, int ny, size_t L, Status* st,
                            unsigned iteration) {
    // Every value the update may read is loaded before any is used (the
    // neighbours' domains and distributions, the node's boundary slots and
    // velocity), so that the loads overlap instead of forming a chain; the
    // arithmetic below is the reference's, in its order.
    const uint32_t oldDom = dom[n];
    const int x = (int)(n % nx), y = (int)(n / nx);
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const size_t nb[5] = {(size_t)y * nx + xp, (size_t)yp * nx + x, (size_t)y * nx + xm, (size_t)ym * nx + x,
                          (size_t)yp * nx + xp};  // E, N, W, S, then NE
    uint32_t dnb[5];
#pragma unroll
    for (int s = 0; s < 5; ++s) dnb[s] = dom[nb[s]];
    bool hasBN[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) hasBN[s] = c.bnDist[n * 4 + s] != kEmpty;
    const double ux = (double)u[n], uy = (double)u[L + n];
    dom[n] = newDom;
    // boundaryNodes_[NE] aliases (domainIdentifier_, cellType_): null only if both are 0.
    const uint32_t ctype = cellTypesCopied ? (oldDom < (uint32_t)nDomains ? ctypeTab[oldDom] : 1u) : 0u;
    const bool neNull = newDom == 0 && ctype == 0;
    double Cnew[kMaxSpecies] = {0.0, 0.0, 0.0};  // getC() of the species already re-initialised here
    bool coupled = false;
    for (int k = 0; k < nS; ++k) coupled |= sp[k].partner >= 0;
    for (int k = 0; k < nS; ++k) {
        const Real* gk = g + (size_t)k * 5 * L;
        // the five slots of the four neighbours and NE, read unconditionally
        Real gv[5][5];
#pragma unroll
        for (int s = 0; s < 5; ++s)
#pragma unroll
            for (int q = 0; q < 5; ++q) gv[s][q] = gk[(size_t)q * L + nb[s]];
        // getC() in slot order after localSwap: T, W, S, E, N
        auto cOf = [](const Real* v) {
            double C = 0.0;
            C += (double)v[0];
            C += (double)v[3];
            C += (double)v[4];
            C += (double)v[1];
            C += (double)v[2];
            return C;
        };
        const int style = sp[k].reinit;
        double sumC = 0.0;
        int counter = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (!hasBN[s] && newDom == dnb[s]) {
                sumC += cOf(gv[s]);
                counter++;
            }
        }
        if (counter == 0 && style != RI_DIAG && neNull && newDom == dnb[4]) {
            sumC += cOf(gv[4]);
            counter++;
            atomicAdd(&st->nDiagReinit, 1);
        }
        if (counter == 0 && style == RI_DIAG) {
            // NE, NW, SW, SE of the same domain, no boundary-node test
            const size_t dg[4] = {nb[4], (size_t)yp * nx + xm, (size_t)ym * nx + xm, (size_t)ym * nx + xp};
            for (int s = 0; s < 4; ++s) {
                if (dom[dg[s]] != newDom) continue;
                Real v[5];
                for (int q = 0; q < 5; ++q) v[q] = gk[(size_t)q * L + dg[s]];
                sumC += cOf(v);
                counter++;
            }
            if (counter != 0) atomicAdd(&st->nDiagReinit, 1);
        }
        if (counter == 0 && style == RI_ALL4) {
            // all of E, N, W, S whatever their domain
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                sumC += cOf(gv[s]);
                counter++;
            }
        }
        if (counter == 0) atomicAdd(&st->nFailedReinit, 1);
        sumC /= static_cast<double>(counter);
        double gi[5];
        for (int q = 0; q < 5; ++q) gi[q] = style == RI_DIAG ? sumC / 4.0 : sumC / 5.0;
        const double src = (srcTab != nullptr && newDom < (uint32_t)nDomains) ? srcTab[(size_t)k * nDomains + newDom]
                                                                            : 0.0;
        // a coupled reaction reads the partner's getC(): re-initialised
        // already (an earlier species), else its state from this step's collide
        double Cp = 0.0;
        const int pj = sp[k].partner;
        if (pj >= 0 && pj < nS) {
            if (pj < k) {
                Cp = Cnew[pj];
            } else {
                Real v[5];
                for (int q = 0; q < 5; ++q) v[q] = g[((size_t)pj * 5 + q) * L + n];
                Cp = cOf(v);
            }
        }
        collide_cde64(gi, ux, uy, sp[k], src, Cp, newDom, ctype, iteration);
        if (coupled) Cnew[k] = sum5_swapped(gi);
        Real* go = g + (size_t)k * 5 * L;
        for (int q = 0; q < 5; ++q) go[(size_t)q * L + n] = (Real)gi[q];
    }
}

// The earlier changed nodes a changed node n waits for: its E,N,W,S (read
// after write: n reads their new state) and NE / SW neighbours (SW reads n's
// old state through its NE fallback) with a smaller row-major index; with a
// species that falls back on all four diagonals (RI_DIAG) also NW / SE; -1 none.
constexpr int kReinitDeps = 8;
__device__ __forceinline__ void reinit_deps(const CrossDev& c, size_t n, int nx, int ny, int* deps) {
    const int x = (int)(n % nx), y = (int)(n / nx);
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const size_t nbs[8] = {(size_t)y * nx + xp,  (size_t)yp * nx + x,  (size_t)y * nx + xm,  (size_t)ym * nx + x,
                           (size_t)yp * nx + xp, (size_t)ym * nx + xm, (size_t)yp * nx + xm, (size_t)ym * nx + xp};
#pragma unroll
    for (int d = 0; d < 8; ++d) deps[d] = (d < 6 || c.diag8) && nbs[d] < n ? c.mark[nbs[d]] - 1 : -1;
}

// (Each changed node's position in the list is marked where the crossings
// append it, in cross_win_kernel; the block kernel clears the marks.)
// Step 1, across the whole GPU: the nodes that wait for no other changed node
// (almost all of them) are re-initialised at once.  No two such nodes read
// each other (a changed neighbour in any of the six directions makes one of
// the two wait for the other), so the order among them does not matter.
template <typename Real>
__global__ void reinit_free_kernel(CrossDev c, uint32_t* dom, Real* g, const Real* u, int nS, SpeciesConst sp0,
                                   SpeciesConst sp1, SpeciesConst sp2, const double* srcTab, int nDomains,
                                   const uint32_t* ctypeTab, int nx, int ny, size_t L, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int cnt = st->nChanged;
    if (cnt > kReinitMax || cnt > c.changedCap) return;  // reported by the block kernel
    const SpeciesConst sp[3] = {sp0, sp1, sp2};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
        const size_t n = c.changedNode[k];
        int deps[kReinitDeps];
        reinit_deps(c, n, nx, ny, deps);
        bool free = true;
#pragma unroll
        for (int d = 0; d < kReinitDeps; ++d) free &= deps[d] < 0;
        if (!free) {
            // listed for the one-block pass; the mark says where
            const int w = atomicAdd(c.nWait, 1);
            c.waitList[w] = k;
            c.reinitDone[k] = 2 + w;
        } else {
            c.reinitDone[k] = 1;
        }
        if (free)
            reinit_node<Real>(n, c.changedDom[k], dom, g, u, nS, sp, srcTab, nDomains, ctypeTab, st->cellTypesCopied,
                              c, nx, ny, L, st, st->iteration);
    }
}

template <typename Real>
__global__ void __launch_bounds__(1024) reinit_kernel(CrossDev c, uint32_t* dom, Real* g, const Real* u, int nS,
                                                      SpeciesConst sp0, SpeciesConst sp1, SpeciesConst sp2,
                                                      const double* srcTab, int nDomains, const uint32_t* ctypeTab,
                                                      int cellTypesCopied, int nx, int ny, size_t L, Status* st,
                                                      unsigned iteration) {
    pdl_wait();
    const int cnt = st->nChanged;
    if (st->halt || cnt == 0) {
        if (threadIdx.x == 0) *c.nWait = 0;
        return;
    }
    if (cnt > kReinitMax || cnt > c.changedCap) {
        if (threadIdx.x == 0) {
            raise_error(st, ERR_CAPACITY, cnt, ST_REINIT);
            *c.nWait = 0;
        }
        return;
    }
    const SpeciesConst sp[3] = {sp0, sp1, sp2};
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long* key = (unsigned long long*)smem;  // node << 32 | newDom
    int(*deps)[kReinitDeps] = (int(*)[kReinitDeps])(key + kReinitMax);
    unsigned char* done = (unsigned char*)(deps + kReinitMax);
    __shared__ int remaining;
    // Step 2, one block: only the nodes that wait for others (listed by the
    // wide pass, usually few or none), in dependency rounds.  A dependency is
    // done when the wide pass re-initialised it (reinitDone 1) or when this
    // pass did (done[w] of its place w in the wait list, reinitDone 2 + w).
    const int nw = min(*c.nWait, cnt);
    if (threadIdx.x == 0) remaining = nw;
    for (int w = threadIdx.x; w < nw; w += blockDim.x) {
        const int k = c.waitList[w];
        key[w] = (((unsigned long long)c.changedNode[k]) << 32) | c.changedDom[k];
        reinit_deps(c, (size_t)c.changedNode[k], nx, ny, deps[w]);
        done[w] = 0;
    }
    __syncthreads();
    int rounds = 0;
    while (remaining > 0 && rounds < kReinitMax + 1) {
        __shared__ int nowDone;
        if (threadIdx.x == 0) nowDone = 0;
        __syncthreads();
        for (int w = threadIdx.x; w < nw; w += blockDim.x) {
            if (done[w]) continue;
            bool ready = true;
            for (int d = 0; d < kReinitDeps; ++d) {
                const int p = deps[w][d];
                if (p < 0) continue;
                const int v = c.reinitDone[p];
                if (v != 1 && done[v - 2] != 1) ready = false;
            }
            if (ready) done[w] = 2;  // processing this round
        }
        __syncthreads();
        for (int w = threadIdx.x; w < nw; w += blockDim.x) {
            if (done[w] == 2) {
                reinit_node<Real>((size_t)(key[w] >> 32), (uint32_t)(key[w] & 0xffffffffu), dom, g, u, nS, sp, srcTab,
                                  nDomains, ctypeTab, st->cellTypesCopied, c, nx, ny, L, st, st->iteration);
                atomicAdd(&nowDone, 1);
            }
        }
        __syncthreads();
        for (int w = threadIdx.x; w < nw; w += blockDim.x)
            if (done[w] == 2) done[w] = 1;
        if (threadIdx.x == 0) remaining -= nowDone;
        __syncthreads();
        ++rounds;
    }
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) c.mark[(size_t)c.changedNode[k]] = 0;
    if (threadIdx.x == 0) *c.nWait = 0;
}

template <typename Real>
void launch_reinit(CrossDev& c, uint32_t* dom, Real* g, const Real* u, int nS, const SpeciesConst* sp,
                   const double* srcTab, int nDomains, const uint32_t* ctypeTab, int cellTypesCopied, int nx, int ny,
                   size_t L, Status* st, unsigned iteration, cudaStream_t s) {
    if (c.changedCap <= 0) return;
    constexpr size_t smemBytes = kReinitSmem;
    launch_pdl(reinit_free_kernel<Real>, 148, 256, 0, s, c, dom, g, u, nS, sp[0], sp[1], sp[2], srcTab, nDomains,
               ctypeTab, nx, ny, L, st);
    launch_pdl(reinit_kernel<Real>, 1, 1024, smemBytes, s, c, dom, g, u, nS, sp[0], sp[1], sp[2], srcTab, nDomains, ctypeTab,
                                           cellTypesCopied, nx, ny, L, st, iteration);
}
template void launch_reinit<double>(CrossDev&, uint32_t*, double*, const double*, int, const SpeciesConst*,
                                    const double*, int, const uint32_t*, int, int, int, size_t, Status*, unsigned,
                                    cudaStream_t);
template void launch_reinit<float>(CrossDev&, uint32_t*, float*, const float*, int, const SpeciesConst*,
                                   const double*, int, const uint32_t*, int, int, int, size_t, Status*, unsigned,
                                   cudaStream_t);

// ---------------------------------------------------------------------------
// Domain fill: one block per row; the row's domain id at x >= 1 is the domain
// of the last W-slot boundary node at x' in [1, x], else dom(0, y), which must
// be 0 (GeometryHandler.cpp:68-85).  Reads and clears the W-slot plane.
// The kernel also resets the (node, slot) entries the step's crossings wrote
// (every written key has a record), after the re-initialisation that read
// them; that part runs on a halted step too.
__global__ void __launch_bounds__(256) domain_fill_kernel(CrossDev c, uint32_t* dom, int nx, int ny, Status* st) {
    pdl_wait();
    const int nrec = min(st->pad[2], c.recCap);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nrec; k += gridDim.x * blockDim.x) {
        const uint32_t key = c.recKey[k];
        c.bnDist[key] = kEmpty;
        c.bnConn[key] = ~0u;
    }
    if (st->halt) return;
    const int y = blockIdx.x;
    const size_t row = (size_t)y * nx;
    const uint32_t left = dom[row];
    if (left != 0) {
        if (threadIdx.x == 0) raise_error(st, ERR_LEFT_DOMAIN, y, ST_DOMAIN);
        return;
    }
    const int chunk = (nx + blockDim.x - 1) / blockDim.x;
    const int xb = threadIdx.x * chunk;
    const int xe = min(nx, xb + chunk);
    // last W mark in this thread's chunk (x >= 1): (x << 32 | value)
    unsigned long long last = 0;
    for (int x = max(xb, 1); x < xe; ++x) {
        const uint32_t w = c.wDom[row + x];
        if (w) last = ((unsigned long long)(x + 1) << 32) | (w - 1);
    }
    typedef cub::BlockScan<unsigned long long, 256> Scan;
    __shared__ typename Scan::TempStorage tmp;
    unsigned long long carry;
    Scan(tmp).ExclusiveScan(last, carry, 0ull, cub::Max());
    uint32_t cur = carry ? (uint32_t)(carry & 0xffffffffu) : left;
    for (int x = max(xb, 1); x < xe; ++x) {
        const uint32_t w = c.wDom[row + x];
        if (w) {
            cur = w - 1;
            c.wDom[row + x] = 0;
        }
        dom[row + x] = cur;
    }
}


void launch_domain_fill(CrossDev& c, uint32_t* dom, int nx, int ny, size_t L, Status* st, unsigned iteration,
                        cudaStream_t s) {
    launch_pdl(domain_fill_kernel, ny, 256, 0, s, c, dom, nx, ny, st);
}


// ---------------------------------------------------------------------------
// Topology checks

__global__ void remesh_check_kernel(Status* st) {
    pdl_wait();
    if (st->halt) return;
    if (st->remesh) raise_halt(st, ST_REMESH);
}

void launch_remesh_check(Status* st, unsigned iteration, cudaStream_t s) { launch_pdl(remesh_check_kernel, 1, 1, 0, s, st); }

// GeometryHandler::coarsenBoundary's test (GeometryHandler.cpp:444-449): the
// span from the previous node to the next node is below MAXLENGTH.
__global__ void coarsen_check_kernel(MembraneDev m, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const int p = m.prev[i], q = m.next[i];
    const double dx = m.x[q] - m.x[p], dy = m.y[q] - m.y[p];
    const double length = sqrt(dx * dx + dy * dy);
    if (length < kMAXLENGTH) {
        st->coarsen = 1;
        raise_halt(st, ST_COARSEN);
    }
}

void launch_coarsen_check(const MembraneDev& m, Status* st, unsigned iteration, cudaStream_t s) {
    if (m.Mcap == 0) return;
    launch_pdl(coarsen_check_kernel, (m.Mcap + 127) / 128, 128, 0, s, m, st);
}

__global__ void clear_forces_kernel(MembraneDev m) {
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= m.topo->M) m.foff[i] = 0;
}

void launch_clear_forces(MembraneDev& m, cudaStream_t s) {
    launch_pdl(clear_forces_kernel, (m.Mcap + 1 + 255) / 256, 256, 0, s, m);
}

// Tension renewal when the force list holds only tension pairs: node i gets
// one type-6 record toward each ring neighbour, ordered by the position of the
// contributing connection in the connection vector
// (tutorial_01_BioSolverMembraneTension.cpp:52-73 adds them in that order).
__global__ void tension_pos_kernel(MembraneDev m, int* outPos, int* inPos) {
    pdl_wait();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.topo->C) return;
    outPos[m.ca[c]] = c;
    inPos[m.cb[c]] = c;
}

__global__ void tension_fill_kernel(MembraneDev m, const int* outPos, const int* inPos, double force) {
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m.topo->M) return;
    m.foff[i] = 2 * i;
    if (i == m.topo->M) return;
    const int nextNode = m.cb[outPos[i]], prevNode = m.ca[inPos[i]];
    const int first = outPos[i] < inPos[i] ? 0 : 1;
    m.ftype[2 * i + first] = 6;
    m.fpartner[2 * i + first] = nextNode;
    m.ftype[2 * i + 1 - first] = 6;
    m.fpartner[2 * i + 1 - first] = prevNode;
    for (int q = 0; q < 4; ++q) {
        m.fpar[4 * (2 * i) + q] = q == 0 ? force : 0.0;
        m.fpar[4 * (2 * i + 1) + q] = q == 0 ? force : 0.0;
    }
}

void launch_tension_renewal(MembraneDev& m, int* outPos, int* inPos, double force, cudaStream_t s) {
    if (m.Mcap == 0) return;
    launch_pdl(tension_pos_kernel, (m.Ccap + 127) / 128, 128, 0, s, m, outPos, inPos);
    launch_pdl(tension_fill_kernel, (m.Mcap + 1 + 127) / 128, 128, 0, s, m, outPos, inPos, force);
}

// ---------------------------------------------------------------------------
// Areas (GeometryHandler::computeAreas, shoelace in ring order) and the
// LbibAreaRegulator mass source per domain.
// One block per cell: the terms x_i y_j - x_j y_i are formed in parallel;
// one thread adds them in ring order (the summation order of the shoelace
// sum is part of the result).
constexpr int kAreaMax = 4096;

__global__ void __launch_bounds__(256) areas_kernel(MembraneDev m, double* area, Status* st) {
    pdl_wait();
    const int cell = blockIdx.x;
    const int b = m.ringStart[cell], e = m.ringStart[cell + 1];
    const int np = e - b;
    __shared__ double terms[kAreaMax];
    if (np > kAreaMax) {
        if (threadIdx.x == 0 && st) raise_error(st, ERR_CAPACITY, cell, ST_BIO);
        return;
    }
    for (int k = threadIdx.x; k < np; k += blockDim.x) {
        const int i = m.ringNode[b + k];
        const int j = m.ringNode[b + (k + 1 == np ? 0 : k + 1)];
        terms[k] = m.x[i] * m.y[j] - m.x[j] * m.y[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int k = 0; k < np; ++k) sum += terms[k];
        area[cell] = sum / 2.0;
    }
}

// ctypeTab == nullptr: LbibAreaRegulator, target = factor x the first area,
// rate strength (target - A) / target.  Otherwise
// tutorial_01_BioSolverAreaRegulator (tutorial_01_BioSolverAreaRegulator.cpp:
// 44-97): target = factor (TARGETAREA), rate strength (target - A) (KP), and
// cells of type 1 get maxsource whatever their area.
// acc != nullptr (FP32-shifted runs): the cell's area is first formed from
// its fixed-point sum, which is reset for the next step (on a halted step too).
constexpr double kAreaFix = 16777216.0;  // 2^24: the fixed-point scale of the shoelace terms
__global__ void area_regulator_kernel(MembraneDev m, double* area, double* target, double* massTab,
                                      int nDomains, double factor, double strength, double maxsource,
                                      const uint32_t* ctypeTab, unsigned long long* acc, const Status* st) {
    pdl_wait();
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= m.nCells) return;
    if (acc != nullptr) {
        area[cell] = (double)(long long)acc[cell] * (1.0 / kAreaFix) / 2.0;
        acc[cell] = 0ull;
    }
    if (st->halt) return;
    const double A = area[cell];
    double r;
    if (ctypeTab == nullptr) {
        if (isnan(target[cell])) target[cell] = factor * A;
        const double tgt = target[cell];
        r = strength * (tgt - A) / tgt;
    } else {
        if (isnan(target[cell])) target[cell] = factor;
        r = strength * (target[cell] - A);
    }
    if (r > maxsource) r = maxsource;
    else if (r < -maxsource) r = -maxsource;
    const uint32_t d = m.ringDom[cell];
    if (d < (uint32_t)nDomains && d != 0) {
        if (ctypeTab != nullptr && ctypeTab[d] == 1) r = maxsource;
        massTab[d] = r;
    }
}

// tutorial_02_BioSolverGrowth::applyBioProcess (tutorial_02_BioSolverGrowth.cpp:
// 44-80): every node inside a cell gets the mass source MAXSOURCE = 0.001 where
// R^2 L > 1 (THRESHOLD) and MAXSOURCE / 10 elsewhere; R and L are the species'
// getC() after the step (post-collide slot order T, W, S, E, N).  The source is
// per node: FluidSolver::addMass sets the next collide's rhoToAdd.  iR < 0:
// BioSolverGrowth (BioSolverGrowth.cpp:41-62), 0.0025 at every node inside a cell.
template <typename Real>
__global__ void growth_kernel(const Real* g, const uint32_t* dom, size_t L, int iR, int iL, double* massNode,
                              const Status* st) {
    pdl_wait();
    if (st->halt) return;
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L) return;
    const uint32_t d = dom[n];
    double src = 0.0;
    if (d != 0) {
        auto cOf = [&](int k) {
            const Real* gk = g + (size_t)k * 5 * L;
            double C = 0.0;
            C += (double)gk[0 * L + n];
            C += (double)gk[3 * L + n];
            C += (double)gk[4 * L + n];
            C += (double)gk[1 * L + n];
            C += (double)gk[2 * L + n];
            return C;
        };
        if (iR < 0) {
            src = 0.0025;  // BioSolverGrowth: the same source everywhere inside cells
        } else {
            const double R = cOf(iR), Lc = cOf(iL);
            const double maxsource = 0.001;
            src = R * R * Lc > 1.0 ? maxsource : maxsource / 10.0;
        }
    }
    massNode[n] = src;
}

// The per-domain rates of an area regulator as per-node sources, for runs
// whose host bio solvers change domains after the bio step (a division's
// cureLattice): FluidSolver::addMass gave each node its rate by the domain it
// had at bio time, which the next collide applies whatever the node's domain
// is by then.
__global__ void mass_expand_kernel(const uint32_t* dom, size_t L, const double* massTab, int nDomains,
                                   double* massNode, const Status* st) {
    pdl_wait();
    if (st->halt) return;
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L) return;
    const uint32_t d = dom[n];
    massNode[n] = (d != 0 && d < (uint32_t)nDomains) ? massTab[d] : 0.0;
}

void launch_mass_expand(const uint32_t* dom, size_t L, const double* massTab, int nDomains, double* massNode,
                        const Status* st, cudaStream_t s) {
    launch_pdl(mass_expand_kernel, (unsigned)((L + 255) / 256), 256, 0, s, dom, L, massTab, nDomains, massNode, st);
}

template <typename Real>
void launch_growth(const Real* g, const uint32_t* dom, size_t L, int iR, int iL, double* massNode, const Status* st,
                   cudaStream_t s) {
    launch_pdl(growth_kernel<Real>, (unsigned)((L + 255) / 256), 256, 0, s, g, dom, L, iR, iL, massNode, st);
}
template void launch_growth<double>(const double*, const uint32_t*, size_t, int, int, double*, const Status*,
                                    cudaStream_t);
template void launch_growth<float>(const float*, const uint32_t*, size_t, int, int, double*, const Status*,
                                   cudaStream_t);

// FP32-shifted runs: the per-cell shoelace sums over the connections in any
// order, each term x_a y_b - x_b y_a (a -> b along the ring) rounded to 64-bit
// fixed point (2^-24), so that the integer sums are exact and independent of
// the order; no ring ranking is needed.  FP64 runs keep the ring-ordered sum.
__global__ void areas_fixed_kernel(MembraneDev m, const int* cellOfDom, int nDomains, unsigned long long* acc) {
    pdl_wait();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    int cell = -1;
    long long v = 0;
    if (c < m.topo->C) {
        const int a = m.ca[c], b = m.cb[c];
        const uint32_t d = m.cdom[c];
        if (d < (uint32_t)nDomains) cell = cellOfDom[d];
        v = __double2ll_rn((m.x[a] * m.y[b] - m.x[b] * m.y[a]) * kAreaFix);
    }
    // one atomic per run of equal cells in the warp (connections of a cell are mostly contiguous)
    const unsigned peers = __match_any_sync(0xffffffffu, cell);
    long long sum = 0;
    for (int l = 0; l < 32; ++l) {
        const long long t = __shfl_sync(0xffffffffu, v, l);
        if ((peers >> l) & 1u) sum += t;
    }
    if (cell >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1)
        atomicAdd(acc + cell, (unsigned long long)sum);
}

void launch_areas(const MembraneDev& m, double* area, Status* st, cudaStream_t s) {
    if (m.nCells == 0) return;
    launch_pdl(areas_kernel, m.nCells, 256, 0, s, m, area, st);
}

// The fixed-point sums as areas (the conversion of area_regulator_kernel),
// the sums cleared for their next use.
__global__ void areas_fixed_finish_kernel(int nCells, unsigned long long* acc, double* area) {
    pdl_wait();
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= nCells) return;
    area[cell] = (double)(long long)acc[cell] * (1.0 / kAreaFix) / 2.0;
    acc[cell] = 0ull;
}

void launch_areas_fixed(const MembraneDev& m, const int* cellOfDom, int nDomains, unsigned long long* acc,
                        double* area, cudaStream_t s) {
    if (m.nCells == 0) return;
    if (m.Ccap > 0) launch_pdl(areas_fixed_kernel, (m.Ccap + 255) / 256, 256, 0, s, m, cellOfDom, nDomains, acc);
    launch_pdl(areas_fixed_finish_kernel, (m.nCells + 127) / 128, 128, 0, s, m.nCells, acc, area);
}

// The fixed device array of lbib_areas_static: the per-cell sums of one call.
// Every call on a device writes and reads this same array.
static __device__ __align__(256) double g_areaScratch[kStaticAreaCells];

cudaError_t static_area_scratch(double** ptr) {
    return cudaGetSymbolAddress((void**)ptr, g_areaScratch);
}

void launch_area_regulator(const MembraneDev& m, double* area, double* target, double* massTab, int nDomains,
                           double factor, double strength, double maxsource, const uint32_t* ctypeTab,
                           const Status* st, cudaStream_t s) {
    if (m.nCells == 0) return;
    launch_pdl(areas_kernel, m.nCells, 256, 0, s, m, area, (Status*)st);
    launch_pdl(area_regulator_kernel, (m.nCells + 127) / 128, 128, 0, s, m, area, target, massTab, nDomains, factor,
               strength, maxsource, ctypeTab, (unsigned long long*)nullptr, st);
}

void launch_area_regulator_fixed(const MembraneDev& m, const int* cellOfDom, unsigned long long* acc, double* area,
                                 double* target, double* massTab, int nDomains, double factor, double strength,
                                 double maxsource, const uint32_t* ctypeTab, const Status* st, cudaStream_t s) {
    if (m.nCells == 0 || m.Ccap == 0) return;
    launch_pdl(areas_fixed_kernel, (m.Ccap + 255) / 256, 256, 0, s, m, cellOfDom, nDomains, acc);
    launch_pdl(area_regulator_kernel, (m.nCells + 127) / 128, 128, 0, s, m, area, target, massTab, nDomains, factor,
               strength, maxsource, ctypeTab, acc, st);
}

// ---------------------------------------------------------------------------
// Differentiated runs with moving membrane nodes.  The forward of one step is
// the spread of the node forces from the step-start positions X, the lattice
// step, then X' = X + (the post-collision velocity interpolated at X): the
// reference's distributeForce, collide and collectVelocity + move
// (GeometryNode.cpp:216-254) without the perturbation, whose random jumps
// have no derivative.  The stencil follows from X (stencil_range of the
// position itself: the 4x4 lattice nodes within 2 lu, the set the reference's
// binding holds while the node stays in its unit cell).

// d fast_cos / dx: the derivative of the approximation itself (its two
// parabolas and the 0.225 correction), so that the gradients are those of
// the forward as it is computed.
__device__ __forceinline__ double fast_cos_deriv(const double x) {
    const double halfPi = M_PI / 2.0;
    const double doublePi = 2.0 * M_PI;
    double tempx = x + halfPi;
    if (tempx > M_PI) tempx -= doublePi;
    double c, dc;
    if (tempx < .00) {
        c = 1.27323954 * tempx + 0.405284735 * tempx * tempx;
        dc = 1.27323954 + 2.0 * 0.405284735 * tempx;
    } else {
        c = 1.27323954 * tempx - 0.405284735 * tempx * tempx;
        dc = 1.27323954 - 2.0 * 0.405284735 * tempx;
    }
    // cs = 0.225 (c |c| - c) + c
    return c < 0.0 ? dc * (1.0 + 0.225 * (-2.0 * c - 1.0)) : dc * (1.0 + 0.225 * (2.0 * c - 1.0));
}

// Sixteen lanes per membrane node, one per stencil slot (two nodes per warp):
// a node's 16 scattered lattice reads are issued at once instead of one
// after another, and the sums over the slots are shuffles within the lanes'
// group of 16 (every lane of the warp takes part, in range or not).
constexpr int kMotionBlock = 128;

__device__ __forceinline__ double group16_sum(double v) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void motion_spread_kernel(const double* X, const double* Y, const double* ax, const double* ay, int M,
                                     int nx, int ny, size_t L, double* out, Status* st) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t >> 4), k = (int)(t & 15);
    if (i >= M) return;
    const double xi = X[i], yi = Y[i];
    Stencil sc;
    if (!stencil_range(xi, yi, nx, ny, sc)) {
        if (k == 0) raise_error(st, ERR_STENCIL, i, ST_SPREAD);
        return;
    }
    int xk, yk;
    stencil_slot(sc, k, xk, yk);
    const size_t n = (size_t)yk * nx + xk;
    const double dl = dirac((double)xk - xi, (double)yk - yi);
    atomicAdd(out + n, dl * ax[i]);
    atomicAdd(out + L + n, dl * ay[i]);
}

void launch_motion_spread(const double* X, const double* Y, const double* ax, const double* ay, int M, int nx,
                          int ny, size_t L, double* out, Status* st, cudaStream_t s) {
    if (M <= 0) return;
    const unsigned blocks = (unsigned)(((long long)M * 16 + kMotionBlock - 1) / kMotionBlock);
    motion_spread_kernel<<<blocks, kMotionBlock, 0, s>>>(X, Y, ax, ay, M, nx, ny, L, out, st);
}

template <typename Real>
__global__ void motion_move_kernel(const double* X0, const double* Y0, double* X1, double* Y1, int M, const Real* u,
                                   int nx, int ny, size_t L, Status* st) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t >> 4), k = (int)(t & 15);
    double xi = 0.0, yi = 0.0, vx = 0.0, vy = 0.0;
    bool ok = false;
    if (i < M) {
        xi = X0[i];
        yi = Y0[i];
        Stencil sc;
        ok = stencil_range(xi, yi, nx, ny, sc);
        if (ok) {
            int xk, yk;
            stencil_slot(sc, k, xk, yk);
            const size_t n = (size_t)yk * nx + xk;
            const double dl = dirac((double)xk - xi, (double)yk - yi);
            vx = (double)u[n] * dl;
            vy = (double)u[L + n] * dl;
        }
    }
    vx = group16_sum(vx);
    vy = group16_sum(vy);
    if (i >= M || k != 0) return;
    if (!ok) {
        raise_error(st, ERR_STENCIL, i, ST_INTERP_MOVE);
        X1[i] = xi;
        Y1[i] = yi;
        return;
    }
    const double CS = 1 / sqrt(3.0);
    if (!(((vx * vx) + (vy * vy)) <= CS)) raise_error(st, ERR_SPEED, i, ST_INTERP_MOVE);  // NaN too
    X1[i] = xi + vx;
    Y1[i] = yi + vy;
}

template <typename Real>
void launch_motion_move(const double* X0, const double* Y0, double* X1, double* Y1, int M, const Real* u, int nx,
                        int ny, size_t L, Status* st, cudaStream_t s) {
    if (M <= 0) return;
    const unsigned blocks = (unsigned)(((long long)M * 16 + kMotionBlock - 1) / kMotionBlock);
    motion_move_kernel<Real><<<blocks, kMotionBlock, 0, s>>>(X0, Y0, X1, Y1, M, u, nx, ny, L, st);
}
template void launch_motion_move<double>(const double*, const double*, double*, double*, int, const double*, int,
                                         int, size_t, Status*, cudaStream_t);
template void launch_motion_move<float>(const double*, const double*, double*, double*, int, const float*, int, int,
                                        size_t, Status*, cudaStream_t);

// With w(a) = 1 + fast_cos(pi/2 (a - X)) the weight of lattice node (a, b)
// is w(a) w(b) / 16, and d/dX of it is -pi/2 fast_cos'(pi/2 (a - X)) w(b) / 16
// (likewise in Y).  A node whose stencil leaves the lattice was refused by
// the forward (ERR_STENCIL) and contributes nothing here.
__global__ void motion_adjoint_kernel(const double* X, const double* Y, const double* fx, const double* fy,
                                      double* lx, double* ly, const double* uo, const double* G, double* gfx,
                                      double* gfy, int M, int nx, int ny, size_t L) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t >> 4), k = (int)(t & 15);
    double gX = 0.0, gY = 0.0, gx = 0.0, gy = 0.0, lamx = 0.0, lamy = 0.0;
    bool ok = false;
    if (i < M) {
        const double xi = X[i], yi = Y[i];
        Stencil sc;
        ok = stencil_range(xi, yi, nx, ny, sc);
        if (ok) {
            const double halfPi = M_PI / 2.0;
            lamx = lx[i];
            lamy = ly[i];
            int xk, yk;
            stencil_slot(sc, k, xk, yk);
            const size_t n = (size_t)yk * nx + xk;
            const double ax = halfPi * ((double)xk - xi), ay = halfPi * ((double)yk - yi);
            const double wa = 1.0 + fast_cos(ax), wb = 1.0 + fast_cos(ay);
            const double dl = (wa * wb) / 16.0;
            const double dX = -halfPi * fast_cos_deriv(ax) * wb / 16.0;
            const double dY = -halfPi * wa * fast_cos_deriv(ay) / 16.0;
            const double Gx = G[n], Gy = G[L + n];
            const double c = lamx * uo[n] + lamy * uo[L + n] + fx[i] * Gx + fy[i] * Gy;
            gX = dX * c;
            gY = dY * c;
            gx = dl * Gx;
            gy = dl * Gy;
        }
    }
    gX = group16_sum(gX);
    gY = group16_sum(gY);
    gx = group16_sum(gx);
    gy = group16_sum(gy);
    if (!ok || k != 0) return;
    lx[i] = lamx + gX;
    ly[i] = lamy + gY;
    gfx[i] += gx;
    gfy[i] += gy;
}

void launch_motion_adjoint(const double* X, const double* Y, const double* fx, const double* fy, double* lx,
                           double* ly, const double* uo, const double* G, double* gfx, double* gfy, int M, int nx,
                           int ny, size_t L, cudaStream_t s) {
    if (M <= 0) return;
    const unsigned blocks = (unsigned)(((long long)M * 16 + kMotionBlock - 1) / kMotionBlock);
    motion_adjoint_kernel<<<blocks, kMotionBlock, 0, s>>>(X, Y, fx, fy, lx, ly, uo, G, gfx, gfy, M, nx, ny, L);
}

}  // namespace lbib

namespace lbib {

void init_kernel_attributes() {
    cudaFuncSetAttribute(spread_kernel<double, kSpreadSmall, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)spread_smem(kSpreadSmall));
    cudaFuncSetAttribute(spread_kernel<double, kSpreadLarge, kSpreadSmall + 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)spread_smem(kSpreadLarge));
    cudaFuncSetAttribute(reinit_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kReinitSmem);
    cudaFuncSetAttribute(reinit_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kReinitSmem);
    init_kernel_attributes_topology();
}

}  // namespace lbib
