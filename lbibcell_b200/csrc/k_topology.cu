// k_topology.cu — membrane topology edits on the device.
//
//   remesh    GeometryHandler::remeshBoundary (GeometryHandler.cpp:385-431) as
//             count + scatter (block counts and their prefix in one kernel): every connection longer than MAXLENGTH gets a new
//             node at its midpoint; the new node ids continue from the largest
//             id in connection order (Geometry::addGeometryNode,
//             Geometry.cpp:382-400); the split connection leaves the vector and
//             its two halves are appended (Geometry::eraseConnection /
//             addConnection, Geometry.cpp:433-452).  Up to two passes run on
//             the device (SimulationRunner.cpp:190-199 repeats until nothing is
//             split); a third pass that would still split, a new node that
//             needs the random perturbation, or a full buffer hands the step to
//             the host.
//   coarsen   GeometryHandler::coarsenBoundary (GeometryHandler.cpp:433-461):
//             nodes are visited in id order and removed when their neighbours
//             are closer than MAXLENGTH; a removal erases the node's two
//             connections and appends one from its predecessor to its successor
//             (Geometry::removeGeometryNode, Geometry.cpp:402-431).  Removals
//             only interact along a ring, so one thread per cell runs the
//             id-ordered visit over that cell's candidates (a node is a
//             candidate if it is one at the start or a smaller-id neighbour
//             was removed); the new connections are appended in removal order.
//   rings     the node order of GeometryHandler::computeAreas (first connection
//             of each domain in vector order, then the second node's outgoing
//             connection) by pointer jumping, one block per cell.
#include <cub/cub.cuh>

#include "kernels.cuh"

namespace lbib {

size_t topo_scan_bytes(int n) {
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (int*)nullptr, (int*)nullptr, n, (cudaStream_t)0);
    return b;
}

// |d| < MAXLENGTH and |d| > MAXLENGTH for a squared length d2, as the
// reference tests them (the correctly rounded sqrt, Connection::getLength,
// Connection.cpp:389-394), with the root taken only within a few ulps of
// MAXLENGTH^2: the rounded root is monotonic, so well below it is below
// MAXLENGTH and at or above it is not (and the other way round).
// Position of the n-th (from 0) set bit of w; w has more than n set bits.
__device__ __forceinline__ int nth_set_bit(unsigned w, int n) {
    int base = 0;
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) {
        const unsigned low = (1u << sh) - 1u;
        const int c = __popc(w & low);
        if (n >= c) {
            n -= c;
            w >>= sh;
            base += sh;
        } else {
            w &= low;
        }
    }
    return base;
}

__device__ __forceinline__ bool shorter_than_max(double d2) {
    constexpr double m2 = kMAXLENGTH * kMAXLENGTH;
    if (d2 < m2 * (1.0 - 1e-12)) return true;
    if (d2 >= m2) return false;
    return sqrt(d2) < kMAXLENGTH;
}
__device__ __forceinline__ bool longer_than_max(double d2) {
    constexpr double m2 = kMAXLENGTH * kMAXLENGTH;
    if (d2 > m2 * (1.0 + 1e-12)) return true;
    if (d2 <= m2) return false;
    return sqrt(d2) > kMAXLENGTH;
}

// Perturbation tests of a new node (GeometryNode.cpp:160, 174, 189, 202).
__device__ __forceinline__ bool new_node_needs_rng(double X, double Y) {
    if (fabs((double)(int)X - X) <= kEPSILON) return true;
    if (fabs((double)(int)Y - Y) <= kEPSILON) return true;
    if (fabs(Y - floor(Y) - (X - floor(X))) <= kEPSILON) return true;
    if (fabs(ceil(Y) - Y - (X - floor(X))) <= kEPSILON) return true;
    return false;
}

// Warp-aggregated atomics: lanes with the same key share one atomic.
__device__ __forceinline__ int agg_add(int* addr, int key) {
    const unsigned act = __activemask();
    const unsigned grp = __match_any_sync(act, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(grp) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(addr, __popc(grp));
    base = __shfl_sync(grp, base, leader);
    return base + __popc(grp & ((1u << lane) - 1u));
}

// Minimum of v per key, where v increases with the lane (a warp's
// connection indices): the group's lowest lane holds the group's minimum.
__device__ __forceinline__ void agg_min(int* addr, int key, int v) {
    const unsigned act = __activemask();
    const unsigned grp = __match_any_sync(act, key);
    if ((int)(threadIdx.x & 31) == __ffs(grp) - 1) atomicMin(addr, v);
}

// ---------------------------------------------------------------------------
// Remesh

constexpr int kRemeshBlock = 256;  // connections per block of the count and apply kernels

// Connection c is split: longer than MAXLENGTH (Connection::getLength,
// Connection.cpp:389-394).  `rng`: its new node needs the random perturbation.
__device__ __forceinline__ bool remesh_split(const MembraneDev& m, int c, bool& rng) {
    const int a = m.ca[c], b = m.cb[c];
    const double x1 = m.x[a], y1 = m.y[a], x2 = m.x[b], y2 = m.y[b];
    const bool split = longer_than_max((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2));
    rng = split && new_node_needs_rng((x1 + x2) / 2, (y1 + y2) / 2);
    return split;
}

// Pass decision.  Each block counts its connections to split (t.flag[block])
// and the new nodes that need the random generator (T->nRng); the last block
// to finish forms the exclusive prefix of the block counts (t.rank[block]),
// and decides: K = the total, or 0 with a halt when the pass would overflow a
// buffer (the host runs it then; so it does a third pass,
// remesh_commit_kernel).  New nodes that need the random perturbation are
// made on the device all the same and listed for the host, which perturbs
// them before the pass is committed (remesh_commit_kernel).
__global__ void __launch_bounds__(kRemeshBlock) remesh_count_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    // a halted step leaves the counts alone (a pass may wait for the host's
    // perturbation of its new nodes); no block of this kernel raises a halt
    // before every block has read it, so all blocks return together
    if (st->halt) return;
    Topo* T = m.topo;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool f = false, rng = false;
    if (c < T->C) f = remesh_split(m, c, rng);
    const int cnt = __syncthreads_count(f);
    const int nr = __syncthreads_count(rng);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        t.flag[blockIdx.x] = cnt;
        if (nr) atomicAdd(&T->nRng, nr);
        __threadfence();
        last = atomicAdd(&T->done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // each thread sums a run of consecutive block counts, one block-wide scan
    // of the runs, then each thread writes its run's prefixes
    typedef cub::BlockScan<int, kRemeshBlock> Scan;
    __shared__ typename Scan::TempStorage tmp;
    const int nb = (int)gridDim.x;
    const int per = (nb + kRemeshBlock - 1) / kRemeshBlock;
    const int beg = threadIdx.x * per, end = min(beg + per, nb);
    int local = 0;
    for (int b = beg; b < end; ++b) local += __ldcg(&t.flag[b]);
    int ex, carry;
    Scan(tmp).ExclusiveSum(local, ex, carry);
    for (int b = beg; b < end; ++b) {
        t.rank[b] = ex;
        ex += __ldcg(&t.flag[b]);
    }
    if (threadIdx.x == 0) {
        const int K = carry, C = T->C, M = T->M;
        const bool run = K > 0 && M + K <= m.Mcap && C + K <= m.Ccap;
        T->K = run ? K : 0;
        if (!run) T->nRng = 0;  // kept for the apply and commit kernels of a pass that runs
        T->rngFill = 0;
        T->done = 0;
        if (K > 0 && !run) raise_halt(st, ST_REMESH);
    }
}

// Applies the pass: connection c's rank among the split ones is its block's
// prefix plus the split connections before it in the block (the same test
// on the same positions as the count).
__global__ void __launch_bounds__(kRemeshBlock) remesh_apply_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (st->halt) return;
    Topo* T = m.topo;
    const int K = T->K;
    if (K == 0) return;
    const int C = T->C, M = T->M;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool rng = false;
    const bool f = c < C && remesh_split(m, c, rng);
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __shared__ int wsum[kRemeshBlock / 32];
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    if (c >= C) return;
    int r = t.rank[blockIdx.x] + __popc(bal & ((1u << lane) - 1u));
    for (int i = 0; i < w; ++i) r += wsum[i];
    if (!f) {
        const int dst = c - r;
        t.ca2[dst] = m.ca[c]; t.cb2[dst] = m.cb[c]; t.cdom2[dst] = m.cdom[c]; t.cdesc2[dst] = m.cdesc[c];
        return;
    }
    const int a = m.ca[c], b = m.cb[c];
    const int j = M + r;
    const double x = (m.x[a] + m.x[b]) / 2, y = (m.y[a] + m.y[b]) / 2;
    m.x[j] = x; m.y[j] = y;
    m.ox[j] = x - 5.0; m.oy[j] = y - 5.0;   // GeometryNode.cpp:98-103
    m.bx[j] = x; m.by[j] = y;               // bound at once (remesh_commit_kernel tests the edges)
    m.vx[j] = 0.0; m.vy[j] = 0.0; m.fx[j] = 0.0; m.fy[j] = 0.0;
    m.id[j] = T->maxId + 1 + (unsigned)r;
    m.next[a] = j; m.prev[j] = a; m.next[j] = b; m.prev[b] = j;
    m.foff[j + 1] = m.foff[M];              // new nodes carry no forces
    // GeometryNode's constructor perturbs a node made on a lattice line or
    // diagonal (GeometryNode.cpp:98-117): the host draws it, in id order
    if (rng) t.rngList[atomicAdd(&T->rngFill, 1)] = j;
    const int base = C - K + 2 * r;
    t.ca2[base] = a; t.cb2[base] = j; t.cdom2[base] = m.cdom[c]; t.cdesc2[base] = m.cdesc[c];
    t.ca2[base + 1] = j; t.cb2[base + 1] = b; t.cdom2[base + 1] = m.cdom[c]; t.cdesc2[base + 1] = m.cdesc[c];
}

// Commits the pass: copies the new connection list back (the last block to
// finish updates the counts; every block has read K, C and M before any block
// counts itself done), and checks what comes next in the reference:
//  - a connection of the new list still longer than MAXLENGTH (a split half
//    of one longer than 2 * MAXLENGTH) needs another pass
//    (SimulationRunner.cpp:190-199 repeats the remeshing); that rare case goes
//    to the host;
//  - the new nodes are bound to the lattice at once (GeometryHandler.cpp:
//    427-428): their old position is 5 lu away, so they are never in their
//    old unit cell, take their binding from the current position (perturbed
//    by the host where needed) and the edge test of connectGeometryNodesToPhysicalNodes
//    (GeometryHandler.cpp:618-644).  The nodes that existed before the pass
//    were bound, and tested, by the crossing stage from the same positions.
__global__ void remesh_commit_kernel(MembraneDev m, TopoDev t, int nx, int ny, Status* st) {
    pdl_wait();
    Topo* T = m.topo;
    const int K = T->K;
    if (K == 0) return;
    if (T->nRng > 0) {
        // new nodes wait for the host's perturbation; the step resumes here
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_halt(st, ST_REMESH_RNG);
        return;
    }
    const int C = T->C, M = T->M;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < C + K) {
        const int a = t.ca2[c], b = t.cb2[c];
        m.ca[c] = a; m.cb[c] = b; m.cdom[c] = t.cdom2[c]; m.cdesc[c] = t.cdesc2[c];
        const double x1 = m.x[a], y1 = m.y[a], x2 = m.x[b], y2 = m.y[b];
        if (longer_than_max((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2))) raise_halt(st, ST_REMESH);
    }
    if (c < K) {
        const int i = M + c;
        const double X = m.x[i], Y = m.y[i];
        m.bx[i] = X;  // bound at its (perturbed) position
        m.by[i] = Y;
        if (X - 2.0 < 0) raise_error(st, ERR_EDGE_W, i, ST_REMESH);
        else if (Y - 2.0 < 0) raise_error(st, ERR_EDGE_S, i, ST_REMESH);
        else if (X + 2.0 > nx) raise_error(st, ERR_EDGE_E, i, ST_REMESH);
        else if (Y + 2.0 > ny) raise_error(st, ERR_EDGE_N, i, ST_REMESH);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&T->done, 1u) == gridDim.x - 1) {
            T->M += K;
            T->C += K;
            T->maxId += K;
            T->changed = 1;
            T->K = 0;
            T->done = 0;
        }
    }
}

int launch_remesh(MembraneDev& m, TopoDev& t, int nx, int ny, Status* st, cudaStream_t s, bool commitOnly) {
    if (m.Ccap == 0) return 0;
    int n = 0;
    if (!commitOnly) {
        // the count and the apply kernel partition the connections alike
        const int cb = (m.Ccap + kRemeshBlock - 1) / kRemeshBlock;
        launch_pdl(remesh_count_kernel, cb, kRemeshBlock, 0, s, m, t, st);
        launch_pdl(remesh_apply_kernel, cb, kRemeshBlock, 0, s, m, t, st);
        n = 2;
    }
    // a pass runs only when C + K <= Ccap: this grid covers the new list
    launch_pdl(remesh_commit_kernel, (m.Ccap + 255) / 256, 256, 0, s, m, t, nx, ny, st);
    return n + 1;
}

// ---------------------------------------------------------------------------
// Coarsen

// Node -> its incoming / outgoing connection; node -> cell; candidates.
__global__ void conn_links_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.topo->C) return;
    t.outConn[m.ca[c]] = c;
    t.inConn[m.cb[c]] = c;
    t.connAlive[c] = 1;
}

__global__ void coarsen_cand_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    t.removed[i] = 0;
    t.ncAlive[i] = 0;
    const int p = m.prev[i], q = m.next[i];
    const double dx = m.x[q] - m.x[p], dy = m.y[q] - m.y[p];
    const bool cand = shorter_than_max(dx * dx + dy * dy);
    const unsigned bal = __ballot_sync(__activemask(), cand);
    if (cand && (threadIdx.x & 31) == __ffs(bal) - 1) atomicAdd(&m.topo->nCand, __popc(bal));
}

constexpr int kCoarsenMax = 2048;  // nodes of one ring held in shared memory
constexpr size_t kCoarsenSmem = (size_t)kCoarsenMax * (2 * sizeof(double) + sizeof(unsigned long long) +
                                                       7 * sizeof(int) + 2) +
                                 (size_t)kCoarsenMax / 32 * sizeof(unsigned);

// One block per cell.  The ring (in ring order, rebuilt just before) is
// loaded into shared memory as a circular list; thread 0 then visits the
// ring's nodes in id order like GeometryHandler::coarsenBoundary, testing
// only nodes whose span is short at the start or whose neighbour was removed
// (every other node keeps a span >= MAXLENGTH and stays).
// Handles: h < Ccap is connection index h; h >= Ccap is the connection made by
// removing node h - Ccap.
__global__ void __launch_bounds__(256) coarsen_cell_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (st->halt || m.topo->nCand == 0) return;
    const int cell = blockIdx.x;
    const int b = m.ringStart[cell], len = m.ringStart[cell + 1] - b;
    if (len > kCoarsenMax) {
        if (threadIdx.x == 0) raise_error(st, ERR_CAPACITY, cell, ST_COARSEN);
        return;
    }
    extern __shared__ __align__(16) unsigned char smem[];
    double* sx = (double*)smem;
    double* sy = sx + kCoarsenMax;
    unsigned long long* ord = (unsigned long long*)(sy + kCoarsenMax);
    int* node = (int*)(ord + kCoarsenMax);
    int* pl = node + kCoarsenMax;
    int* nl = pl + kCoarsenMax;
    int* hin = nl + kCoarsenMax;
    int* hout = hin + kCoarsenMax;
    // boundary descriptor of each position's incoming connection, and the
    // ring's domain (one per cell), so that the serial visit below reads no
    // global memory (it does where a ring mixes domains)
    int* inDesc = hout + kCoarsenMax;
    __shared__ uint32_t ringDomS;
    __shared__ int mixedDom;
    int* rankOf = inDesc + kCoarsenMax;                 // ring position -> place in id order
    unsigned* visit = (unsigned*)(rankOf + kCoarsenMax); // bit j: the node at place j is a candidate
    unsigned char* dirty = (unsigned char*)(visit + kCoarsenMax / 32);
    unsigned char* gone = dirty + kCoarsenMax;
    __shared__ int anyDirty;
    if (threadIdx.x == 0) {
        anyDirty = 0;
        mixedDom = 0;
        ringDomS = len > 0 ? m.cdom[t.inConn[m.ringNode[b]]] : 0u;
    }
    int p2 = 1;
    while (p2 < len) p2 <<= 1;
    __syncthreads();
    for (int k = threadIdx.x; k < p2; k += blockDim.x) {
        if (k < len) {
            const int i = m.ringNode[b + k];
            node[k] = i;
            sx[k] = m.x[i];
            sy[k] = m.y[i];
            pl[k] = k == 0 ? len - 1 : k - 1;
            nl[k] = k == len - 1 ? 0 : k + 1;
            hin[k] = t.inConn[i];
            if (m.cdom[hin[k]] != ringDomS) mixedDom = 1;
            inDesc[k] = m.cdesc[hin[k]];
            hout[k] = t.outConn[i];
            ord[k] = ((unsigned long long)i << 32) | (unsigned)k;
            gone[k] = 0;
        } else {
            ord[k] = ~0ull;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < len; k += blockDim.x) {
        const int p = pl[k], q = nl[k];
        const double dx = sx[q] - sx[p], dy = sy[q] - sy[p];
        dirty[k] = shorter_than_max(dx * dx + dy * dy);
        if (dirty[k]) anyDirty = 1;
    }
    __syncthreads();
    if (!anyDirty) {
        for (int k = threadIdx.x; k < len; k += blockDim.x) t.removed[node[k]] = 0;
        return;
    }
    // id order of the ring's nodes
    for (int size = 2; size <= p2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int k = threadIdx.x; k < p2; k += blockDim.x) {
                const int j = k ^ stride;
                if (j > k) {
                    const bool up = (k & size) == 0;
                    const unsigned long long x = ord[k], y = ord[j];
                    if ((x > y) == up) { ord[k] = y; ord[j] = x; }
                }
            }
            __syncthreads();
        }
    }
    // the candidates as bits in id order, so that the visit below jumps from
    // one to the next instead of stepping over every node
    const int nw = (len + 31) >> 5;
    for (int j = threadIdx.x; j < nw * 32; j += blockDim.x) {
        const bool cand = j < len && dirty[(int)(ord[j] & 0xffffffffu)];
        if (j < len) rankOf[(int)(ord[j] & 0xffffffffu)] = j;
        const unsigned bits = __ballot_sync(0xffffffffu, cand);
        if ((threadIdx.x & 31) == 0) visit[j >> 5] = bits;
    }
    __shared__ unsigned wantBits[kCoarsenMax / 32];
    for (int w = threadIdx.x; w < kCoarsenMax / 32; w += blockDim.x) wantBits[w] = 0u;
    __syncthreads();
    if (threadIdx.x < 32) {
        // The visit in id order, 32 candidates per round.  Each lane takes the
        // next candidate place and tests it against the state at the start of
        // the round.  The round keeps the places before T, where T is the
        // first place whose outcome an earlier removal of the round changes:
        // a candidate next to a removed node (its neighbour link changes), or
        // a node that a removal makes a candidate at a later place (the id
        // order visits it there).  The kept removals touch disjoint links, so
        // they are applied together, and the next round starts at T.  The
        // result is the one of the one-by-one visit.
        const int lane = threadIdx.x;
        const int Ccap = m.Ccap;
        int removedHere = 0;
        int j0 = 0;
        while (j0 < len) {
            // the places of the next (up to) 32 candidates at or after j0
            const int w0 = j0 >> 5;
            unsigned word = w0 + lane < nw ? visit[w0 + lane] : 0u;
            if (lane == 0) word &= ~0u << (j0 & 31);
            const int cnt = __popc(word);
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            if (total == 0) {
                j0 = (w0 + 32) << 5;
                continue;
            }
            // lane l takes candidate l: the word holding it, then its bit
            int src = 0;
#pragma unroll
            for (int st2 = 16; st2 > 0; st2 >>= 1)
                if (__shfl_sync(0xffffffffu, incl, src + st2 - 1) <= lane) src += st2;
            const bool valid = lane < total;
            const int srcS = valid ? src : 31;
            const unsigned srcWord = __shfl_sync(0xffffffffu, word, srcS);
            const int before = __shfl_sync(0xffffffffu, incl - cnt, srcS);
            const int P = valid ? ((w0 + srcS) << 5) + nth_set_bit(srcWord, lane - before) : 0x7fffffff;
            int k = 0, p = 0, q = 0;
            bool want = false;
            if (valid) {
                k = (int)(ord[P] & 0xffffffffu);
                p = pl[k];
                q = nl[k];
                if (dirty[k]) {
                    const double dx = sx[q] - sx[p], dy = sy[q] - sy[p];
                    want = shorter_than_max(dx * dx + dy * dy);
                }
            }
            const int rp = valid ? rankOf[p] : 0, rq = valid ? rankOf[q] : 0;
            if (want) atomicOr(&wantBits[P >> 5], 1u << (P & 31));
            __syncwarp();
            // a removal before this place takes away this node's neighbour
            const bool conflict = valid && ((rp < P && ((wantBits[rp >> 5] >> (rp & 31)) & 1u)) ||
                                            (rq < P && ((wantBits[rq >> 5] >> (rq & 31)) & 1u)));
            int T = 0x7fffffff;
            if (conflict) T = P;
            if (want) {  // the neighbours become candidates at their places
                if (rp > P) T = min(T, rp);
                if (rq > P) T = min(T, rq);
            }
            T = (int)__reduce_min_sync(0xffffffffu, (unsigned)T);
            const int lastP = __shfl_sync(0xffffffffu, P, min(total, 32) - 1);
            if (T > lastP) T = lastP + 1;
            __syncwarp();
            if (want) atomicAnd(&wantBits[P >> 5], ~(1u << (P & 31)));
            if (want && P < T) {
                gone[k] = 1;
                ++removedHere;
                const int i = node[k];
                const int h1 = hin[k], h2 = hout[k];
                uint32_t dom = ringDomS;
                const int desc = inDesc[k];
                if (h1 < Ccap) {
                    t.connAlive[h1] = 0;
                    if (mixedDom) dom = m.cdom[h1];
                } else {
                    t.ncAlive[h1 - Ccap] = 0;
                    if (mixedDom) dom = t.ncDom[h1 - Ccap];
                }
                if (h2 < Ccap) t.connAlive[h2] = 0;
                else t.ncAlive[h2 - Ccap] = 0;
                t.ncA[i] = node[p]; t.ncB[i] = node[q]; t.ncDom[i] = dom; t.ncDesc[i] = desc; t.ncAlive[i] = 1;
                nl[p] = q; pl[q] = p;
                hout[p] = Ccap + i; hin[q] = Ccap + i;
                inDesc[q] = desc;
                dirty[p] = 1; dirty[q] = 1;
                atomicOr(&visit[rp >> 5], 1u << (rp & 31));
                atomicOr(&visit[rq >> 5], 1u << (rq & 31));
            }
            __syncwarp();
            j0 = T;
        }
        removedHere = __reduce_add_sync(0xffffffffu, removedHere);
        if (lane == 0 && removedHere) atomicAdd(&m.topo->removed, removedHere);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < len; k += blockDim.x) {
        const int i = node[k];
        t.removed[i] = gone[k];
        if (!gone[k]) {
            m.prev[i] = node[pl[k]];
            m.next[i] = node[nl[k]];
        }
    }
}

// Compaction flags: kept nodes; alive original connections; alive new ones.
__global__ void coarsen_flags_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const Topo* T = m.topo;
    if (i <= m.Mcap) t.nflag[i] = (!st->halt && T->removed && i < T->M && !t.removed[i]) ? 1 : 0;
    if (i <= m.Ccap) t.flag[i] = (!st->halt && T->removed && i < T->C && t.connAlive[i]) ? 1 : 0;
}

// Gathers the kept nodes and the alive connections into the scratch copies.
__global__ void coarsen_gather_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (st->halt || m.topo->removed == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int M = m.topo->M, C = m.topo->C;
    if (i < M && !t.removed[i]) {
        const int d = t.nrank[i];
        double* a = t.dalt;
        const size_t cap = (size_t)m.Mcap;
        a[0 * cap + d] = m.x[i]; a[1 * cap + d] = m.y[i]; a[2 * cap + d] = m.ox[i]; a[3 * cap + d] = m.oy[i];
        a[4 * cap + d] = m.vx[i]; a[5 * cap + d] = m.vy[i]; a[6 * cap + d] = m.fx[i]; a[7 * cap + d] = m.fy[i];
        a[8 * cap + d] = m.bx[i]; a[9 * cap + d] = m.by[i];
        t.id2[d] = m.id[i];
        t.prev2[d] = t.nrank[m.prev[i]];
        t.next2[d] = t.nrank[m.next[i]];
    }
    const int Calive = t.rank[m.Ccap];
    if (i < C && t.connAlive[i]) {
        const int d = t.rank[i];
        t.ca2[d] = t.nrank[m.ca[i]]; t.cb2[d] = t.nrank[m.cb[i]]; t.cdom2[d] = m.cdom[i]; t.cdesc2[d] = m.cdesc[i];
    }
    if (i < M && t.ncAlive[i]) {
        // new connections follow the alive originals, in removal (= id) order
        const int d = Calive + t.succ[i];
        t.ca2[d] = t.nrank[t.ncA[i]]; t.cb2[d] = t.nrank[t.ncB[i]]; t.cdom2[d] = t.ncDom[i]; t.cdesc2[d] = t.ncDesc[i];
    }
}

__global__ void coarsen_scatter_back_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (st->halt || m.topo->removed == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int Mn = t.nrank[m.Mcap];
    const int Cn = t.rank[m.Ccap] + t.succ[m.Mcap];
    if (i < Mn) {
        const double* a = t.dalt;
        const size_t cap = (size_t)m.Mcap;
        m.x[i] = a[0 * cap + i]; m.y[i] = a[1 * cap + i]; m.ox[i] = a[2 * cap + i]; m.oy[i] = a[3 * cap + i];
        m.vx[i] = a[4 * cap + i]; m.vy[i] = a[5 * cap + i]; m.fx[i] = a[6 * cap + i]; m.fy[i] = a[7 * cap + i];
        m.bx[i] = a[8 * cap + i]; m.by[i] = a[9 * cap + i];
        m.id[i] = t.id2[i]; m.prev[i] = t.prev2[i]; m.next[i] = t.next2[i];
    }
    if (i <= Mn) m.foff[i] = 0;  // the force list is empty at a coarsening step
    if (i < Cn) { m.ca[i] = t.ca2[i]; m.cb[i] = t.cb2[i]; m.cdom[i] = t.cdom2[i]; m.cdesc[i] = t.cdesc2[i]; }
}

__global__ void coarsen_commit_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (st->halt) return;
    Topo* T = m.topo;
    if (T->removed == 0) { T->nCand = 0; return; }
    const int Mn = t.nrank[m.Mcap];
    T->M = Mn;
    T->C = t.rank[m.Ccap] + t.succ[m.Mcap];
    if (Mn > 0) T->maxId = m.id[Mn - 1];
    T->changed = 1;
    T->removed = 0;
    T->nCand = 0;
}

// ncAlive as an int flag array for the scan of new connections
__global__ void coarsen_ncflag_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m.Mcap) return;
    t.dist[i] = (!st->halt && m.topo->removed && i < m.topo->M && t.ncAlive[i]) ? 1 : 0;
}

int launch_coarsen(MembraneDev& m, TopoDev& t, Status* st, cudaStream_t s) {
    const int nCells = t.nCellsCap;
    if (m.Mcap == 0 || nCells == 0) return 0;
    const int mb = (m.Mcap + 1 + 255) / 256, cbk = (m.Ccap + 1 + 255) / 256;
    const int gb = ((m.Mcap > m.Ccap ? m.Mcap : m.Ccap) + 1 + 255) / 256;
    int n = launch_rings(m, t, st, s);  // ring order after this step's remeshing
    launch_pdl(conn_links_kernel, cbk, 256, 0, s, m, t, st);
    launch_pdl(coarsen_cand_kernel, mb, 256, 0, s, m, t, st);
    constexpr size_t smemBytes = kCoarsenSmem;
    launch_pdl(coarsen_cell_kernel, nCells, 256, smemBytes, s, m, t, st);
    launch_pdl(coarsen_flags_kernel, gb, 256, 0, s, m, t, st);
    launch_pdl(coarsen_ncflag_kernel, mb, 256, 0, s, m, t, st);
    cub::DeviceScan::ExclusiveSum(t.scanTmp, t.scanTmpBytes, t.nflag, t.nrank, m.Mcap + 1, s);
    cub::DeviceScan::ExclusiveSum(t.scanTmp, t.scanTmpBytes, t.flag, t.rank, m.Ccap + 1, s);
    cub::DeviceScan::ExclusiveSum(t.scanTmp, t.scanTmpBytes, t.dist, t.succ, m.Mcap + 1, s);
    launch_pdl(coarsen_gather_kernel, gb, 256, 0, s, m, t, st);
    launch_pdl(coarsen_scatter_back_kernel, gb, 256, 0, s, m, t, st);
    launch_pdl(coarsen_commit_kernel, 1, 1, 0, s, m, t, st);
    return n + 15;
}

// ---------------------------------------------------------------------------
// Rings

__global__ void ring_first_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (!m.topo->changed) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.topo->C) return;
    t.outConn[m.ca[c]] = c;
    agg_min(&t.firstConn[m.cdom[c]], (int)m.cdom[c], c);
}

__global__ void ring_count_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (!m.topo->changed) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const int cell = t.cellOfDom[m.cdom[t.outConn[i]]];
    agg_add(&t.cellCount[cell], cell);
}

__global__ void ring_fill_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (!m.topo->changed) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const uint32_t d = m.cdom[t.outConn[i]];
    const int cell = t.cellOfDom[d];
    const int k = agg_add(&t.cellFill[cell], cell);
    t.members[t.cellStart[cell] + k] = i;
    const int start = m.cb[t.firstConn[d]];
    // break the ring before its start node: the node whose successor is the start is last
    t.succ[i] = m.next[i] == start ? -1 : m.next[i];
    t.dist[i] = m.next[i] == start ? 0 : 1;
}

constexpr int kRingPerThread = 16;  // 256 threads x 16 = 4096 nodes per ring

__global__ void __launch_bounds__(256) ring_rank_kernel(MembraneDev m, TopoDev t, Status* st) {
    pdl_wait();
    if (!m.topo->changed) return;
    const int cell = blockIdx.x;
    const int b = t.cellStart[cell], len = t.cellCount[cell];
    if (len > 256 * kRingPerThread) {
        if (threadIdx.x == 0) raise_error(st, ERR_CAPACITY, cell, ST_BIO);
        return;
    }
    int ns[kRingPerThread], nd[kRingPerThread];
    for (int round = 0; (1 << round) < len; ++round) {
        for (int k = 0; k < kRingPerThread; ++k) {
            const int idx = threadIdx.x + k * 256;
            if (idx >= len) break;
            const int i = t.members[b + idx];
            const int sc = t.succ[i];
            if (sc >= 0) { nd[k] = t.dist[i] + t.dist[sc]; ns[k] = t.succ[sc]; }
            else { nd[k] = t.dist[i]; ns[k] = -1; }
        }
        __syncthreads();
        for (int k = 0; k < kRingPerThread; ++k) {
            const int idx = threadIdx.x + k * 256;
            if (idx >= len) break;
            const int i = t.members[b + idx];
            t.succ[i] = ns[k];
            t.dist[i] = nd[k];
        }
        __syncthreads();
    }
    for (int k = 0; k < kRingPerThread; ++k) {
        const int idx = threadIdx.x + k * 256;
        if (idx >= len) break;
        const int i = t.members[b + idx];
        const int d = t.dist[i];
        if (d >= 0 && d < len) m.ringNode[b + (len - 1 - d)] = i;
        else raise_error(st, ERR_STATE, i, ST_BIO);
    }
    if (threadIdx.x == 0) m.ringStart[cell] = b;
    if (threadIdx.x == 0 && cell == gridDim.x - 1) m.ringStart[cell + 1] = b + len;
}

__global__ void ring_done_kernel(MembraneDev m, TopoDev t) {
    pdl_wait();
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < t.nDomains) t.firstConn[d] = 0x7fffffff;
    if (d == 0) m.topo->changed = 0;
}

// The listed connections to perturb (perturb_conn_kernel, t.rngList), each
// with its place in its cell's ring walk (the rings are current: the host
// rebuilds them first when the topology changed).  The walk visits the
// connection leaving the ring's last node first (the domain's first
// connection), then those leaving ranks 0, 1, ..., len - 2.
__global__ void conn_perturb_gather_kernel(MembraneDev m, TopoDev t, int n, ConnPerturbRec* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int c = t.rngList[k];
    ConnPerturbRec r{};
    r.a = m.ca[c];
    r.b = m.cb[c];
    r.dom = (int)m.cdom[c];
    r.xa = m.x[r.a]; r.ya = m.y[r.a]; r.xb = m.x[r.b]; r.yb = m.y[r.b];
    r.walk = -1;
    r.z = -1;
    const int cell = (uint32_t)r.dom < (uint32_t)t.nDomains ? t.cellOfDom[r.dom] : -1;
    if (cell >= 0 && cell < m.nCells) {
        const int s0 = m.ringStart[cell], len = m.ringStart[cell + 1] - s0;
        int rank = -1;
        for (int j = 0; j < len; ++j)
            if (m.ringNode[s0 + j] == r.a) { rank = j; break; }
        if (rank >= 0 && len >= 2) {
            r.len = len;
            r.walk = rank == len - 1 ? 0 : rank + 1;
            r.z = m.ringNode[s0 + len - 2];
            r.xz = m.x[r.z];
            r.yz = m.y[r.z];
        }
    }
    out[k] = r;
}

void launch_conn_perturb_gather(const MembraneDev& m, const TopoDev& t, int n, ConnPerturbRec* out, cudaStream_t s) {
    if (n <= 0) return;
    conn_perturb_gather_kernel<<<(n + 127) / 128, 128, 0, s>>>(m, t, n, out);
}

int launch_rings(MembraneDev& m, TopoDev& t, Status* st, cudaStream_t s) {
    const int nCells = t.nCellsCap;
    if (m.Mcap == 0 || nCells == 0) return 0;
    const int mb = (m.Mcap + 255) / 256, cbk = (m.Ccap + 255) / 256;
    cudaMemsetAsync(t.cellCount, 0, sizeof(int) * (nCells + 1), s);
    cudaMemsetAsync(t.cellFill, 0, sizeof(int) * nCells, s);
    launch_pdl(ring_first_kernel, cbk, 256, 0, s, m, t, st);
    launch_pdl(ring_count_kernel, mb, 256, 0, s, m, t, st);
    cub::DeviceScan::ExclusiveSum(t.scanTmp, t.scanTmpBytes, t.cellCount, t.cellStart, nCells + 1, s);
    launch_pdl(ring_fill_kernel, mb, 256, 0, s, m, t, st);
    launch_pdl(ring_rank_kernel, nCells, 256, 0, s, m, t, st);
    launch_pdl(ring_done_kernel, (t.nDomains + 255) / 256, 256, 0, s, m, t);
    return 7;
}

}  // namespace lbib

namespace lbib {

void init_kernel_attributes_topology() {
    cudaFuncSetAttribute(coarsen_cell_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarsenSmem);
    // loaded now rather than at a host event's first use (modules load lazily)
    cudaFuncAttributes fa;
    cudaFuncGetAttributes(&fa, conn_perturb_gather_kernel);
}

}  // namespace lbib
