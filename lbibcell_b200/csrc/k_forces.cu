// k_forces.cu — edits of the membrane force list on the device, and the
// cell-junction bio solver.  Compiled with --fmad=false: the junction search
// compares distances that must round as the reference's do.
//
//   force list edit   ForceSolver::deleteForceType(T) followed by addForce of
//                     new records (ForceSolver.cpp:107-139, 183-215).  The list
//                     is a CSR by node in insertion order; an edit keeps each
//                     node's records of other types in their order and appends
//                     the new records of that node in the order the reference
//                     adds them.
//   cell junctions    tutorial_01_BioSolverCellJunction::applyBioProcess
//                     (tutorial_01_BioSolverCellJunction.cpp:47-99; the
//                     tutorial_02 and plain BioSolverCellJunction are the same
//                     solver): every FREQUENCY-th iteration, drop all type-7
//                     forces; then, for each node in id order, find the closest
//                     node of another cell within RADIUS
//                     (Geometry::getGeometryNodesWithinRadiusWithAvoidanceClosest,
//                     Geometry.cpp:350-374; fastneighborlist,
//                     FastNeighborList.hpp:400-468) and add a type-7 spring
//                     each way between the two.
#include <cub/cub.cuh>

#include "kernels.cuh"

namespace lbib {

// ---------------------------------------------------------------------------
// Force list edit

// Copies the current list (offsets and records) to the scratch buffers that
// the fill kernel reads from.
__global__ void force_snapshot_kernel(MembraneDev m, ForceScratch fs, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int M = m.topo->M;
    const int R = m.foff[M];
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= M; i += stride) fs.foffS[i] = m.foff[i];
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += stride) {
        fs.ftypeS[r] = m.ftype[r];
        fs.fpartnerS[r] = m.fpartner[r];
#pragma unroll
        for (int q = 0; q < 4; ++q) fs.fparS[4 * (size_t)r + q] = m.fpar[4 * (size_t)r + q];
    }
}

// Records of node i after the edit: the kept ones plus the generated ones.
__device__ __forceinline__ int gen_count(const ForceScratch& fs, int gen, int i) {
    if (gen == GEN_NONE) return 0;
    if (gen == GEN_TENSION) return 2;
    if (gen == GEN_LIST) return fs.listOff[i + 1] - fs.listOff[i];
    return (fs.closest[i] >= 0 ? 1 : 0) + fs.inCnt[i];
}

__global__ void force_count_kernel(MembraneDev m, ForceScratch fs, int delType, int gen, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m.Mcap) return;
    const int M = m.topo->M;
    if (i >= M) {
        fs.cnt[i] = 0;
        return;
    }
    int keep = 0;
    for (int r = fs.foffS[i]; r < fs.foffS[i + 1]; ++r) keep += fs.ftypeS[r] != delType;
    fs.cnt[i] = keep + gen_count(fs, gen, i);
}

__device__ __forceinline__ void put_record(MembraneDev& m, int r, int type, int partner, double p0, double p1) {
    m.ftype[r] = type;
    m.fpartner[r] = partner;
    m.fpar[4 * (size_t)r + 0] = p0;
    m.fpar[4 * (size_t)r + 1] = p1;
    m.fpar[4 * (size_t)r + 2] = 0.0;
    m.fpar[4 * (size_t)r + 3] = 0.0;
}

// m.foff holds the exclusive scan of fs.cnt.  Generated records:
//   GEN_TENSION   one type-6 record toward each ring neighbour, ordered by the
//                 position of the contributing connection in the connection
//                 vector (the membrane-tension plugin adds them connection by
//                 connection);
//   GEN_JUNCTION  type-7 springs (K, L0) in the order of the node j whose search
//                 added them: node j's own record toward its closest node, and
//                 the record toward j of the node j found.
__global__ void force_fill_kernel(MembraneDev m, ForceScratch fs, int delType, int gen, double tensionForce,
                                  double K, double L0, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int M = m.topo->M;
    if (i >= M) return;
    if (m.foff[M] > fs.Fcap) {
        raise_error(st, ERR_CAPACITY, m.foff[M], ST_BIO);
        return;
    }
    int o = m.foff[i];
    for (int r = fs.foffS[i]; r < fs.foffS[i + 1]; ++r) {
        if (fs.ftypeS[r] == delType) continue;
        m.ftype[o] = fs.ftypeS[r];
        m.fpartner[o] = fs.fpartnerS[r];
#pragma unroll
        for (int q = 0; q < 4; ++q) m.fpar[4 * (size_t)o + q] = fs.fparS[4 * (size_t)r + q];
        ++o;
    }
    if (gen == GEN_NONE) return;
    if (gen == GEN_LIST) {
        for (int r = fs.listOff[i]; r < fs.listOff[i + 1]; ++r, ++o) {
            m.ftype[o] = fs.listType[r];
            m.fpartner[o] = fs.listPartner[r];
#pragma unroll
            for (int q = 0; q < 4; ++q) m.fpar[4 * (size_t)o + q] = fs.listPar[4 * (size_t)r + q];
        }
        return;
    }
    if (gen == GEN_TENSION) {
        const int out = fs.outPos[i], in = fs.inPos[i];
        const int nextNode = m.cb[out], prevNode = m.ca[in];
        put_record(m, o + (out < in ? 0 : 1), 6, nextNode, tensionForce, 0.0);
        put_record(m, o + (out < in ? 1 : 0), 6, prevNode, tensionForce, 0.0);
        return;
    }
    // junctions: the finders of node i in ascending order (insertion sort of
    // this node's own segment; segments hold a few entries)
    int* seg = fs.inList + fs.inOff[i];
    const int n = fs.inCnt[i];
    for (int a = 1; a < n; ++a) {
        const int v = seg[a];
        int b = a - 1;
        while (b >= 0 && seg[b] > v) {
            seg[b + 1] = seg[b];
            --b;
        }
        seg[b + 1] = v;
    }
    const int own = fs.closest[i];
    bool ownDone = own < 0;
    for (int a = 0; a < n; ++a) {
        const int j = seg[a];
        if (!ownDone && i < j) {
            put_record(m, o++, 7, own, K, L0);
            ownDone = true;
        }
        put_record(m, o++, 7, j, K, L0);
    }
    if (!ownDone) put_record(m, o++, 7, own, K, L0);
}

size_t force_scan_bytes(int n) {
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (int*)nullptr, (int*)nullptr, n, (cudaStream_t)0);
    return b;
}

size_t junction_sort_bytes(int n, int bits) {
    size_t b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b, (const unsigned*)nullptr, (unsigned*)nullptr, (const int*)nullptr,
                                    (int*)nullptr, n, 0, bits, (cudaStream_t)0);
    return b;
}

// Connection position of each node's outgoing (ca == i) and incoming (cb == i)
// connection; the incoming one is GeometryNode::getConnection<0>
// (Geometry.cpp:147-149), whose domain is the node's
// getDomainIdOfAdjacentConnections (GeometryNode.cpp:267-283).
__global__ void conn_pos_kernel(MembraneDev m, ForceScratch fs) {
    pdl_wait();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.topo->C) return;
    fs.outPos[m.ca[c]] = c;
    fs.inPos[m.cb[c]] = c;
}

int launch_force_edit(MembraneDev& m, ForceScratch& fs, int delType, int gen, double tensionForce, double K,
                      double L0, Status* st, cudaStream_t s) {
    if (m.Mcap == 0) return 0;
    launch_pdl(force_snapshot_kernel, 296, 256, 0, s, m, fs, st);
    launch_pdl(force_count_kernel, (m.Mcap + 1 + 255) / 256, 256, 0, s, m, fs, delType, gen, st);
    cub::DeviceScan::ExclusiveSum(fs.scanTmp, fs.scanTmpBytes, fs.cnt, m.foff, m.Mcap + 1, s);
    launch_pdl(force_fill_kernel, (m.Mcap + 127) / 128, 128, 0, s, m, fs, delType, gen, tensionForce, K, L0, st);
    return 4;
}

// ---------------------------------------------------------------------------
// Cell junctions

// fastneighborlist::getIndex (FastNeighborList.hpp:508-520) with the bins of
// Geometry (Geometry.cpp:56-59): NX = ceil(LX / MAXBINSIZE) bins of LX / NX =
// 1 lu (MAXBINSIZE = 1, Constants.hpp:62-64), clamped to the lattice.
__device__ __forceinline__ int bin_index(double pos, int n) {
    if (pos < 0.0) pos = 0.0;
    int b = (int)floor(pos / 1.0);
    if (b >= n) b = n - 1;
    return b;
}

__global__ void junction_bin_kernel(MembraneDev m, ForceScratch fs, int nx, int ny) {
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.Mcap) return;
    unsigned key = (unsigned)nx * (unsigned)ny;  // unused slots sort last
    if (i < m.topo->M) key = (unsigned)bin_index(m.y[i], ny) * (unsigned)nx + (unsigned)bin_index(m.x[i], nx);
    fs.binKey[i] = key;
    fs.binIdx[i] = i;
}

// binStart[key] = first sorted position of each bin present.  Entries of
// bins absent now keep old values; a lookup checks the key found there.
__global__ void bin_start_kernel(MembraneDev m, ForceScratch fs) {
    pdl_wait();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m.Mcap) return;
    const unsigned key = fs.binKeySorted[p];
    if (key >= fs.binCap) return;
    if (p == 0 || fs.binKeySorted[p - 1] != key) fs.binStart[key] = p;
}

// First sorted position of bin `key`, or Mcap when the bin is empty.
__device__ __forceinline__ int bin_first(const ForceScratch& fs, int mcap, unsigned key) {
    const int p = fs.binStart[key];
    return (p >= 0 && p < mcap && fs.binKeySorted[p] == key) ? p : mcap;
}


// The junction step's cell list: every node linked into its bin's list (in
// no particular order), the previous call's heads cleared first.  No sort: the
// query below breaks ties by (bin, node index) itself.
__global__ void junction_unlink_kernel(ForceScratch fs) {
    pdl_wait();
    const int n = *fs.linkPrevM;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        fs.binHead[fs.linkKey[i]] = -1;
}

__global__ void junction_link_kernel(MembraneDev m, ForceScratch fs, int nx, int ny, Status* st) {
    pdl_wait();
    const int M = m.topo->M;
    const bool halt = st->halt != 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) *fs.linkPrevM = halt ? 0 : M;
    if (halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const unsigned key = (unsigned)bin_index(m.y[i], ny) * (unsigned)nx + (unsigned)bin_index(m.x[i], nx);
    fs.linkKey[i] = key;
    fs.binNext[i] = atomicExch(&fs.binHead[key], i);
}

// The query of node i: the reference visits the candidates in the order its
// cell list returns them (bins by row, then column, within a bin in id order:
// the list is rebuilt from the id-ordered node map after every move,
// Geometry.cpp:531-535), drops those farther than the radius (distance >
// radius) or with i's domain, and keeps the first of the smallest distance
// (std::min_element with <).  Here the bins are visited in that order and a
// candidate of the same distance replaces the best one only within its bin
// and with a smaller node index: the same node wins.
__global__ void junction_query_kernel(MembraneDev m, ForceScratch fs, int nx, int ny, double radius, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int M = m.topo->M;
    if (i >= M) return;
    const double xi = m.x[i], yi = m.y[i];
    const uint32_t avoid = m.cdom[fs.inPos[i]];
    const int bx0 = bin_index(xi - radius, nx), bx1 = bin_index(xi + radius, nx);
    const int by0 = bin_index(yi - radius, ny), by1 = bin_index(yi + radius, ny);
    int best = -1;
    unsigned bestKey = 0;
    double bestD = 0.0;
    int steps = 0;  // a well-formed list holds each node once
    for (int by = by0; by <= by1; ++by)
        for (int bx = bx0; bx <= bx1; ++bx) {
            const unsigned key = (unsigned)by * (unsigned)nx + (unsigned)bx;
            for (int j = fs.binHead[key]; j >= 0; j = fs.binNext[j]) {
                if (++steps > M) {
                    raise_error(st, ERR_STATE, i, ST_BIO);
                    fs.closest[i] = -1;
                    return;
                }
                const double xj = m.x[j], yj = m.y[j];
                const double d = sqrt((xj - xi) * (xj - xi) + (yj - yi) * (yj - yi));
                if (d > radius) continue;
                if (m.cdom[fs.inPos[j]] == avoid) continue;
                if (best < 0 || d < bestD || (d == bestD && key == bestKey && j < best)) {
                    best = j;
                    bestD = d;
                    bestKey = key;
                }
            }
        }
    fs.closest[i] = best;
}

__global__ void junction_incount_kernel(MembraneDev m, ForceScratch fs, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const int c = fs.closest[i];
    if (c >= 0) atomicAdd(&fs.inCnt[c], 1);
}

__global__ void junction_infill_kernel(MembraneDev m, ForceScratch fs, Status* st) {
    pdl_wait();
    if (st->halt) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.topo->M) return;
    const int c = fs.closest[i];
    if (c >= 0) fs.inList[fs.inOff[c] + atomicAdd(&fs.inFill[c], 1)] = i;
}

int launch_cell_list(MembraneDev& m, ForceScratch& fs, int nx, int ny, cudaStream_t s) {
    if (m.Mcap == 0) return 0;
    const int n = m.Mcap;
    launch_pdl(conn_pos_kernel, (m.Ccap + 127) / 128, 128, 0, s, m, fs);
    launch_pdl(junction_bin_kernel, (n + 255) / 256, 256, 0, s, m, fs, nx, ny);
    cub::DeviceRadixSort::SortPairs(fs.sortTmp, fs.sortTmpBytes, fs.binKey, fs.binKeySorted, fs.binIdx,
                                    fs.binIdxSorted, n, 0, fs.sortBits, s);
    launch_pdl(bin_start_kernel, (n + 255) / 256, 256, 0, s, m, fs);
    return 3;
}

// Range queries for host plugins, on the cell list of launch_cell_list: hits in
// the cell list's order (bins by row, then column, id order within a bin);
// distance > radius drops a node (FastNeighborList.hpp:400-421), and with
// avoid >= 0 so does a node whose getDomainIdOfAdjacentConnections equals it
// (:425-444); the closest is the first hit of the smallest distance (:447-465).
// One thread per query point.
__global__ void range_query_kernel(MembraneDev m, ForceScratch fs, int nx, int ny, const double* qx,
                                   const double* qy, const long long* avoid, int nq, double radius, int mode,
                                   unsigned* ids, int cap, int* count, long long* closest) {
    pdl_wait();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const double x = qx[q], y = qy[q];
    const long long av = avoid != nullptr ? avoid[q] : -1;
    const int bx0 = bin_index(x - radius, nx), bx1 = bin_index(x + radius, nx);
    const int by0 = bin_index(y - radius, ny), by1 = bin_index(y + radius, ny);
    int n = 0, best = -1;
    double bestD = 0.0;
    for (int by = by0; by <= by1; ++by)
        for (int bx = bx0; bx <= bx1; ++bx) {
            const unsigned key = (unsigned)by * (unsigned)nx + (unsigned)bx;
            for (int p = bin_first(fs, m.Mcap, key); p < m.Mcap && fs.binKeySorted[p] == key;
                 ++p) {
                const int j = fs.binIdxSorted[p];
                const double xj = m.x[j], yj = m.y[j];
                const double d = sqrt((xj - x) * (xj - x) + (yj - y) * (yj - y));
                if (d > radius) continue;
                if (av >= 0 && (long long)m.cdom[fs.inPos[j]] == av) continue;
                if (mode == 0) {
                    if (n < cap) ids[n] = m.id[j];
                    ++n;
                } else if (best < 0 || d < bestD) {
                    best = j;
                    bestD = d;
                }
            }
        }
    if (mode == 0) *count = n;
    else closest[q] = best < 0 ? -1 : (long long)m.id[best];
}

void launch_range_query(MembraneDev& m, ForceScratch& fs, int nx, int ny, const double* qx, const double* qy,
                        const long long* avoid, int nq, double radius, int mode, unsigned* ids, int cap, int* count,
                        long long* closest, cudaStream_t s) {
    if (nq <= 0) return;
    launch_pdl(range_query_kernel, (nq + 127) / 128, 128, 0, s, m, fs, nx, ny, qx, qy, avoid, nq, radius, mode, ids,
               cap, count, closest);
}

int launch_junctions(MembraneDev& m, ForceScratch& fs, int nx, int ny, double radius, double K, double L0,
                     Status* st, cudaStream_t s) {
    if (m.Mcap == 0) return 0;
    const int n = m.Mcap;
    launch_pdl(conn_pos_kernel, (m.Ccap + 127) / 128, 128, 0, s, m, fs);
    launch_pdl(junction_unlink_kernel, 148 * 4, 256, 0, s, fs);
    launch_pdl(junction_link_kernel, (n + 255) / 256, 256, 0, s, m, fs, nx, ny, st);
    launch_pdl(junction_query_kernel, (n + 127) / 128, 128, 0, s, m, fs, nx, ny, radius, st);
    cudaMemsetAsync(fs.inCnt, 0, sizeof(int) * (n + 1), s);
    cudaMemsetAsync(fs.inFill, 0, sizeof(int) * n, s);
    launch_pdl(junction_incount_kernel, (n + 255) / 256, 256, 0, s, m, fs, st);
    cub::DeviceScan::ExclusiveSum(fs.scanTmp, fs.scanTmpBytes, fs.inCnt, fs.inOff, n + 1, s);
    launch_pdl(junction_infill_kernel, (n + 255) / 256, 256, 0, s, m, fs, st);
    // ForceSolver::deleteForceType(7), then the new springs
    return 8 + launch_force_edit(m, fs, 7, GEN_JUNCTION, 0.0, K, L0, st, s);
}

int launch_tension_edit(MembraneDev& m, ForceScratch& fs, double force, Status* st, cudaStream_t s) {
    if (m.Mcap == 0) return 0;
    launch_pdl(conn_pos_kernel, (m.Ccap + 127) / 128, 128, 0, s, m, fs);
    return 1 + launch_force_edit(m, fs, 6, GEN_TENSION, force, 0.0, 0.0, st, s);
}

}  // namespace lbib
