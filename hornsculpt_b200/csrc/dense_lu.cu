// Batched dense complex LU with partial pivoting, triangular solves and the
// FP64 refinement residual (cuda_solver.cu:1485-1581). The plain form
// factors in FP64; the mixed form factors an FP32 copy and refines in FP64
// (the reference factors in FP32 with cuSOLVER getrf/getrs).
//
// Matrices are column-major N x N complex (interleaved reals), one per
// frequency of the batch (blockIdx.y / blockIdx.z). Right-looking blocked LU
// with panel width 32: a single-CTA panel factorisation per matrix, row
// interchanges outside the panel, a unit-lower triangular solve for the U
// block row and a shared-memory tiled complex GEMM for the trailing update.
#include "device_once.hpp"
#include "device_types.cuh"
#include "kernel_timer.hpp"

#include <cooperative_groups.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

namespace hsb {
namespace {

constexpr int kPanel = 32;

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// complex element type of a real type
template <class R> struct Cx;
template <> struct Cx<double> {
    using type = double2;
};
template <> struct Cx<float> {
    using type = float2;
};
template <class R> using C2 = typename Cx<R>::type;
template <class R> __device__ __forceinline__ C2<R> mk(R x, R y) {
    C2<R> v;
    v.x = x;
    v.y = y;
    return v;
}
template <class R> __device__ __forceinline__ C2<R> ld2(const R *p) { return *reinterpret_cast<const C2<R> *>(p); }
template <class R> __device__ __forceinline__ void st2(R *p, C2<R> v) { *reinterpret_cast<C2<R> *>(p) = v; }
template <class R> __device__ __forceinline__ C2<R> cmul(C2<R> a, C2<R> b) {
    return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// v -= a * b
template <class R> __device__ __forceinline__ void csub(C2<R> &v, C2<R> a, C2<R> b) {
    v.x -= a.x * b.x - a.y * b.y;
    v.y -= a.x * b.y + a.y * b.x;
}

// Panel factorisation of columns [k0, k0+jb) over rows [k0, N) of one matrix.
template <class R>
__global__ void __launch_bounds__(512) panelKernel(R *LU, uint32_t N, uint32_t k0, uint32_t jb, int *pivots,
                                                   int *info) {
    R *M = LU + size_t(blockIdx.x) * N * N * 2;
    int *piv = pivots + size_t(blockIdx.x) * N;
    __shared__ R sVal[16];
    __shared__ int sIdx[16];
    __shared__ C2<R> sRow[kPanel];
    __shared__ int sPivot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (uint32_t j = 0; j < jb; ++j) {
        const uint32_t c = k0 + j;
        // argmax |re|+|im| over rows [c, N), first index on ties
        R best = -1;
        int bestRow = int(c);
        for (uint32_t i = c + threadIdx.x; i < N; i += blockDim.x) {
            const C2<R> v = ld2(M + 2 * (size_t(c) * N + i));
            const R a = fabs(v.x) + fabs(v.y);
            if (a > best) {
                best = a;
                bestRow = int(i);
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const R ob = __shfl_down_sync(0xffffffffu, best, off);
            const int oi = __shfl_down_sync(0xffffffffu, bestRow, off);
            if (ob > best || (ob == best && oi < bestRow)) {
                best = ob;
                bestRow = oi;
            }
        }
        if (lane == 0) {
            sVal[warp] = best;
            sIdx[warp] = bestRow;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            R b = sVal[0];
            int bi = sIdx[0];
            for (int w = 1; w < warps; ++w)
                if (sVal[w] > b || (sVal[w] == b && sIdx[w] < bi)) {
                    b = sVal[w];
                    bi = sIdx[w];
                }
            sPivot = bi;
            piv[c] = bi;
            if (!(b > 0) && *info == 0)
                atomicCAS(info, 0, int(c) + 1);
        }
        __syncthreads();
        const int p = sPivot;
        if (threadIdx.x < jb && p != int(c)) {
            R *a = M + 2 * (size_t(k0 + threadIdx.x) * N + c);
            R *b = M + 2 * (size_t(k0 + threadIdx.x) * N + p);
            const C2<R> va = ld2(a), vb = ld2(b);
            st2(a, vb);
            st2(b, va);
        }
        __syncthreads();
        if (threadIdx.x < jb)
            sRow[threadIdx.x] = ld2(M + 2 * (size_t(k0 + threadIdx.x) * N + c));
        __syncthreads();
        const C2<R> d = sRow[j];
        const R den = d.x * d.x + d.y * d.y;
        const C2<R> inv = den > 0 ? mk<R>(d.x / den, -d.y / den) : mk<R>(0, 0);
        for (uint32_t i = c + 1 + threadIdx.x; i < N; i += blockDim.x) {
            R *col = M + 2 * (size_t(c) * N + i);
            const C2<R> l = cmul<R>(ld2(col), inv);
            st2(col, l);
            for (uint32_t q = j + 1; q < jb; ++q) {
                R *e = M + 2 * (size_t(k0 + q) * N + i);
                C2<R> v = ld2(e);
                csub<R>(v, l, sRow[q]);
                st2(e, v);
            }
        }
        __syncthreads();
    }
}

// Panel factorisation with the panel resident in shared memory (rows
// [k0, N) x jb columns). Rows stay in place: step j selects the pivot among
// the rows not yet selected (largest |re|+|im|, lowest row on ties), every
// thread eliminates column j from its own rows and takes its candidate for
// column j+1 in the same pass, so a column costs one barrier. The selection
// order is turned into the LAPACK interchange sequence at the end and the
// panel is written back in interchanged order.
template <class R>
__global__ void __launch_bounds__(1024) panelSmemKernel(R *LU, uint32_t N, uint32_t k0, uint32_t jb, int *pivots,
                                                        int *info) {
    extern __shared__ __align__(16) unsigned char rawSmem[];
    const uint32_t rows = N - k0;
    C2<R> *P = reinterpret_cast<C2<R> *>(rawSmem);                 // [jb][rows]
    int *arrangement = reinterpret_cast<int *>(P + size_t(jb) * rows);  // position -> local row
    int *where = arrangement + rows;                                 // local row -> position
    uint32_t taken = 0;  // bit r: this thread's r-th row (threadIdx.x + r * blockDim.x) is a pivot row
    __shared__ R sBest[2][32];
    __shared__ int sRow[2][32];
    __shared__ int sSel[kPanel];
    R *M = LU + size_t(blockIdx.x) * N * N * 2;
    int *piv = pivots + size_t(blockIdx.x) * N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    // stage the panel: a batch of independent column loads in flight per thread
    constexpr int kLoad = sizeof(R) == 8 ? 4 : 8;
    for (uint32_t i = threadIdx.x; i < rows; i += blockDim.x) {
        for (uint32_t q0 = 0; q0 < jb; q0 += kLoad) {
            C2<R> v[kLoad];
#pragma unroll
            for (int t = 0; t < kLoad; ++t)
                if (q0 + t < jb)
                    v[t] = ld2(M + 2 * (size_t(k0 + q0 + t) * N + k0 + i));
#pragma unroll
            for (int t = 0; t < kLoad; ++t)
                if (q0 + t < jb)
                    P[size_t(q0 + t) * rows + i] = v[t];
        }
        arrangement[i] = int(i);
        where[i] = int(i);
    }
    __syncthreads();
    // candidates for column 0
    R best = -1;
    int bestRow = int(rows);
    for (uint32_t i = threadIdx.x; i < rows; i += blockDim.x) {
        const C2<R> v = P[i];
        R a = fabs(v.x) + fabs(v.y);
        if (!(a >= R(0)))
            a = 0;  // a NaN row competes as zero, so a pivot row always exists
        if (a > best) {
            best = a;
            bestRow = int(i);
        }
    }
    for (uint32_t j = 0; j < jb; ++j) {
        const int buf = j & 1;
        for (int off = 16; off > 0; off >>= 1) {
            const R ob = __shfl_down_sync(0xffffffffu, best, off);
            const int oi = __shfl_down_sync(0xffffffffu, bestRow, off);
            if (ob > best || (ob == best && oi < bestRow)) {
                best = ob;
                bestRow = oi;
            }
        }
        if (lane == 0) {
            sBest[buf][warp] = best;
            sRow[buf][warp] = bestRow;
        }
        __syncthreads();
        // every warp reduces the warp candidates by shuffles (same result in every warp)
        R pb = lane < warps ? sBest[buf][lane] : R(-1);
        int p = lane < warps ? sRow[buf][lane] : int(rows);
        for (int off = 16; off > 0; off >>= 1) {
            const R ob = __shfl_xor_sync(0xffffffffu, pb, off);
            const int oi = __shfl_xor_sync(0xffffffffu, p, off);
            if (ob > pb || (ob == pb && oi < p)) {
                pb = ob;
                p = oi;
            }
        }
        if (threadIdx.x == 0) {
            sSel[j] = p;
            if (!(pb > 0) && *info == 0)
                atomicCAS(info, 0, int(k0 + j) + 1);
        }
        const C2<R> d = P[size_t(j) * rows + p];
        const R den = d.x * d.x + d.y * d.y;
        const R rden = den > 0 ? R(1) / den : R(0);
        const C2<R> inv = mk<R>(d.x * rden, -d.y * rden);
        best = -1;
        bestRow = int(rows);
        uint32_t r = 0;
        for (uint32_t i = threadIdx.x; i < rows; i += blockDim.x, ++r) {
            if (int(i) == p)
                taken |= 1u << r;
            if (taken >> r & 1u)
                continue;
            const C2<R> l = cmul<R>(P[size_t(j) * rows + i], inv);
            P[size_t(j) * rows + i] = l;
            // eliminate in chunks of columns: loads first, then updates and stores
            constexpr int kChunk = sizeof(R) == 8 ? 4 : 8;
            C2<R> next = mk<R>(0, 0);
            for (uint32_t q0 = j + 1; q0 < jb; q0 += kChunk) {
                C2<R> v[kChunk], pv[kChunk];
#pragma unroll
                for (int t = 0; t < kChunk; ++t)
                    if (q0 + t < jb) {
                        v[t] = P[size_t(q0 + t) * rows + i];
                        pv[t] = P[size_t(q0 + t) * rows + p];
                    }
#pragma unroll
                for (int t = 0; t < kChunk; ++t)
                    if (q0 + t < jb) {
                        csub<R>(v[t], l, pv[t]);
                        P[size_t(q0 + t) * rows + i] = v[t];
                    }
                if (q0 == j + 1)
                    next = v[0];
            }
            if (j + 1 < jb) {
                R a = fabs(next.x) + fabs(next.y);
                if (!(a >= R(0)))
                    a = 0;
                if (a > best) {
                    best = a;
                    bestRow = int(i);
                }
            }
        }
    }
    __syncthreads();
    // selection order -> interchange sequence (row k0+j swapped with row piv[k0+j])
    if (threadIdx.x == 0)
        for (uint32_t j = 0; j < jb; ++j) {
            const int r = sSel[j], pj = where[r], rj = arrangement[j];
            piv[k0 + j] = int(k0) + pj;
            arrangement[j] = r;
            arrangement[pj] = rj;
            where[r] = int(j);
            where[rj] = pj;
        }
    __syncthreads();
    for (uint32_t q = 0; q < jb; ++q)
        for (uint32_t i = threadIdx.x; i < rows; i += blockDim.x)
            st2(M + 2 * (size_t(k0 + q) * N + k0 + i), P[size_t(q) * rows + arrangement[i]]);
}

// Panel factorisation for tall panels, spread over a thread-block cluster:
// CTA r of the cluster owns panel rows [r * rowsPerBlock, ...). The first
// `cap` of them live in shared memory, one per thread; the rest (at most
// kGlobalSlots per thread) stay in place in global memory and are eliminated
// there by their thread. Pivot choice, tie rule and interchange sequence are
// those of panelSmemKernel. Per column: each warp's best candidate goes to its
// CTA's shared memory (double-buffered by column parity); one cluster barrier;
// every warp reduces the candidates of all CTAs through distributed shared
// memory; one warp per CTA copies the pivot row from the CTA that holds it
// (distributed shared memory, or global memory for a row kept there); each
// CTA eliminates its own rows. Rows that are pivots never change again, so
// reading them remotely needs no further barrier. Write-back: a row kept in
// global memory moves only when it is a pivot, to one of the first jb
// positions, whose own rows are in CTA 0's shared memory; such rows are copied
// first, and after a cluster barrier the shared-memory rows are written to
// their final positions. A final cluster barrier keeps every CTA's shared
// memory alive until all remote reads are done.
template <class R> constexpr uint32_t kClusterRows = sizeof(R) == 8 ? 384 : 768;
constexpr uint32_t kMaxCluster = 16;
constexpr int kGlobalSlots = 4;

template <class R> struct ClusterPanelShared {
    R best[32];
    int idx[32];
    R ctaBest[2];  // this CTA's candidate per column parity
    int ctaIdx[2];
    C2<R> pivot[kPanel];
    int sel[kPanel];
    int mapRow[2 * kPanel], mapPos[2 * kPanel];
    int mapCount;
};

template <class R, int Slots>
__global__ void __launch_bounds__(1024) panelClusterKernel(R *LU, uint32_t N, uint32_t k0, uint32_t jb,
                                                           uint32_t rowsPerBlock, uint32_t cap, int *pivots,
                                                           int *info) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char rawSmem[];
    __shared__ ClusterPanelShared<R> sh;
    C2<R> *P = reinterpret_cast<C2<R> *>(rawSmem);  // [jb][cap]
    const uint32_t rank = cluster.block_rank(), C = cluster.num_blocks();
    const uint32_t rows = N - k0, rowBegin = rank * rowsPerBlock;
    const uint32_t myRows = rowBegin < rows ? min(rowsPerBlock, rows - rowBegin) : 0u;
    R *M = LU + size_t(blockIdx.y) * N * N * 2;
    int *piv = pivots + size_t(blockIdx.y) * N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = int(blockDim.x >> 5);
    const uint32_t i = threadIdx.x;
    // slot 0: shared-memory row i; slot s >= 1: global row cap + (s - 1) * blockDim + i
    const auto local = [&](int s) { return s == 0 ? i : cap + uint32_t(s - 1) * blockDim.x + i; };
    const auto owns = [&](int s) { return s == 0 ? (i < cap && i < myRows) : local(s) < myRows; };
    const auto column = [&](uint32_t q) { return M + 2 * (size_t(k0 + q) * N + k0); };  // panel column q
    constexpr int kLoad = sizeof(R) == 8 ? 4 : 8;
    if (owns(0))
        for (uint32_t q0 = 0; q0 < jb; q0 += kLoad) {
            C2<R> v[kLoad];
#pragma unroll
            for (int t = 0; t < kLoad; ++t)
                if (q0 + t < jb)
                    v[t] = ld2(column(q0 + t) + 2 * (rowBegin + i));
#pragma unroll
            for (int t = 0; t < kLoad; ++t)
                if (q0 + t < jb)
                    P[size_t(q0 + t) * cap + i] = v[t];
        }
    const auto magnitude = [](C2<R> z) {
        const R a = fabs(z.x) + fabs(z.y);
        return a >= R(0) ? a : R(0);  // a NaN row competes as zero, so a pivot row always exists
    };
    bool taken[1 + Slots];
    R best = R(-1);
    int bestRow = int(rows);
#pragma unroll
    for (int s = 0; s <= Slots; ++s) {
        taken[s] = !owns(s);
        if (!taken[s]) {
            const uint32_t g = rowBegin + local(s);
            const R m = magnitude(s == 0 ? P[i] : ld2(column(0) + 2 * g));
            if (m > best || (m == best && int(g) < bestRow)) {
                best = m;
                bestRow = int(g);
            }
        }
    }
    for (uint32_t j = 0; j < jb; ++j) {
        const int buf = j & 1;
        for (int off = 16; off > 0; off >>= 1) {
            const R ob = __shfl_xor_sync(0xffffffffu, best, off);
            const int oi = __shfl_xor_sync(0xffffffffu, bestRow, off);
            if (ob > best || (ob == best && oi < bestRow)) {
                best = ob;
                bestRow = oi;
            }
        }
        if (lane == 0) {
            sh.best[warp] = best;
            sh.idx[warp] = bestRow;
        }
        __syncthreads();
        if (warp == 0) {  // this CTA's candidate
            R b = lane < W ? sh.best[lane] : R(-1);
            int r = lane < W ? sh.idx[lane] : int(rows);
            for (int off = 16; off > 0; off >>= 1) {
                const R ob = __shfl_xor_sync(0xffffffffu, b, off);
                const int oi = __shfl_xor_sync(0xffffffffu, r, off);
                if (ob > b || (ob == b && oi < r)) {
                    b = ob;
                    r = oi;
                }
            }
            if (lane == 0) {
                sh.ctaBest[buf] = b;
                sh.ctaIdx[buf] = r;
            }
        }
        cluster.sync();
        // the candidates of all CTAs, one per lane, read through distributed shared memory
        R pb = R(-1);
        int p = int(rows);
        if (uint32_t(lane) < C) {
            const ClusterPanelShared<R> *other = cluster.map_shared_rank(&sh, lane);
            pb = other->ctaBest[buf];
            p = other->ctaIdx[buf];
        }
        for (int off = 16; off > 0; off >>= 1) {
            const R ob = __shfl_xor_sync(0xffffffffu, pb, off);
            const int oi = __shfl_xor_sync(0xffffffffu, p, off);
            if (ob > pb || (ob == pb && oi < p)) {
                pb = ob;
                p = oi;
            }
        }
        if (warp == 0) {
            // copy the pivot row (columns j.. of panel row p) from the CTA that holds it
            const uint32_t owner = uint32_t(p) / rowsPerBlock, at = uint32_t(p) % rowsPerBlock;
            if (uint32_t(lane) >= j && uint32_t(lane) < jb) {
                if (at < cap)
                    sh.pivot[lane] = cluster.map_shared_rank(P, int(owner))[size_t(lane) * cap + at];
                else
                    sh.pivot[lane] = ld2(column(lane) + 2 * uint32_t(p));
            }
            if (rank == 0 && lane == 0) {
                sh.sel[j] = p;
                if (!(pb > 0) && *info == 0)
                    atomicCAS(info, 0, int(k0 + j) + 1);
            }
        }
        __syncthreads();
        const C2<R> d = sh.pivot[j];
        const R den = d.x * d.x + d.y * d.y;
        const R rden = den > 0 ? R(1) / den : R(0);
        const C2<R> inv = mk<R>(d.x * rden, -d.y * rden);
        best = -1;
        bestRow = int(rows);
#pragma unroll
        for (int s = 0; s <= Slots; ++s) {
            if (taken[s])
                continue;
            const uint32_t g = rowBegin + local(s);
            if (int(g) == p) {
                taken[s] = true;
                continue;
            }
            C2<R> next = mk<R>(0, 0);
            if (s == 0) {
                const C2<R> l = cmul<R>(P[size_t(j) * cap + i], inv);
                P[size_t(j) * cap + i] = l;
                for (uint32_t q0 = j + 1; q0 < jb; q0 += kLoad) {
                    C2<R> v[kLoad];
#pragma unroll
                    for (int t = 0; t < kLoad; ++t)
                        if (q0 + t < jb)
                            v[t] = P[size_t(q0 + t) * cap + i];
#pragma unroll
                    for (int t = 0; t < kLoad; ++t)
                        if (q0 + t < jb) {
                            csub<R>(v[t], l, sh.pivot[q0 + t]);
                            P[size_t(q0 + t) * cap + i] = v[t];
                        }
                    if (q0 == j + 1)
                        next = v[0];
                }
            } else {
                const C2<R> l = cmul<R>(ld2(column(j) + 2 * g), inv);
                st2(column(j) + 2 * g, l);
                for (uint32_t q0 = j + 1; q0 < jb; q0 += kLoad) {
                    C2<R> v[kLoad];
#pragma unroll
                    for (int t = 0; t < kLoad; ++t)
                        if (q0 + t < jb)
                            v[t] = ld2(column(q0 + t) + 2 * g);
#pragma unroll
                    for (int t = 0; t < kLoad; ++t)
                        if (q0 + t < jb) {
                            csub<R>(v[t], l, sh.pivot[q0 + t]);
                            st2(column(q0 + t) + 2 * g, v[t]);
                        }
                    if (q0 == j + 1)
                        next = v[0];
                }
            }
            if (j + 1 < jb) {
                const R m = magnitude(next);
                if (m > best || (m == best && int(g) < bestRow)) {
                    best = m;
                    bestRow = int(g);
                }
            }
        }
    }
    cluster.sync();
    // Interchange sequence and the final position of every row that moved, by warp 0 of
    // rank 0: the (row, position) pairs of the moved rows live in lane registers, two per
    // lane (at most 2 * jb), and each lookup is one ballot.
    if (rank == 0 && warp == 0) {
        int rowA = -1, posA = 0, rowB = -1, posB = 0;  // slots lane and lane + 32
        int n = 0;
        const auto whereOf = [&](int row) {  // current position of a row
            const unsigned a = __ballot_sync(0xffffffffu, rowA == row), b = __ballot_sync(0xffffffffu, rowB == row);
            if (a)
                return __shfl_sync(0xffffffffu, posA, __ffs(a) - 1);
            if (b)
                return __shfl_sync(0xffffffffu, posB, __ffs(b) - 1);
            return row;
        };
        const auto rowAt = [&](int pos) {  // row currently at a position
            const unsigned a = __ballot_sync(0xffffffffu, rowA >= 0 && posA == pos);
            const unsigned b = __ballot_sync(0xffffffffu, rowB >= 0 && posB == pos);
            if (a)
                return __shfl_sync(0xffffffffu, rowA, __ffs(a) - 1);
            if (b)
                return __shfl_sync(0xffffffffu, rowB, __ffs(b) - 1);
            return pos;
        };
        const auto setWhere = [&](int row, int pos) {
            const unsigned a = __ballot_sync(0xffffffffu, rowA == row), b = __ballot_sync(0xffffffffu, rowB == row);
            if (a) {
                if (lane == __ffs(a) - 1)
                    posA = pos;
            } else if (b) {
                if (lane == __ffs(b) - 1)
                    posB = pos;
            } else {
                if (n < 32 && lane == n) {
                    rowA = row;
                    posA = pos;
                } else if (n >= 32 && lane == n - 32) {
                    rowB = row;
                    posB = pos;
                }
                ++n;
            }
        };
        for (uint32_t j = 0; j < jb; ++j) {
            const int r = sh.sel[j], pj = whereOf(r), rj = rowAt(int(j));
            if (lane == 0)
                piv[k0 + j] = int(k0) + pj;
            setWhere(r, int(j));
            setWhere(rj, pj);
        }
        const unsigned a = __ballot_sync(0xffffffffu, rowA >= 0 && rowA != posA);
        const unsigned b = __ballot_sync(0xffffffffu, rowB >= 0 && rowB != posB);
        const unsigned below = (1u << lane) - 1u;
        if (a >> lane & 1u) {
            sh.mapRow[__popc(a & below)] = rowA;
            sh.mapPos[__popc(a & below)] = posA;
        }
        if (b >> lane & 1u) {
            sh.mapRow[__popc(a) + __popc(b & below)] = rowB;
            sh.mapPos[__popc(a) + __popc(b & below)] = posB;
        }
        if (lane == 0)
            sh.mapCount = __popc(a) + __popc(b);
    }
    cluster.sync();
    if (rank != 0) {  // a local copy of rank 0's map
        const ClusterPanelShared<R> *root = cluster.map_shared_rank(&sh, 0);
        for (uint32_t q = threadIdx.x; q < 2 * kPanel; q += blockDim.x) {
            sh.mapRow[q] = root->mapRow[q];
            sh.mapPos[q] = root->mapPos[q];
        }
        if (threadIdx.x == 0)
            sh.mapCount = root->mapCount;
    }
    __syncthreads();
    const int moved = sh.mapCount;
    const auto finalPosition = [&](uint32_t g) {
        uint32_t pos = g;
        for (int q = 0; q < moved; ++q)
            if (sh.mapRow[q] == int(g))
                pos = uint32_t(sh.mapPos[q]);
        return pos;
    };
    // pivots kept in global memory move to their positions (< jb; those rows are in CTA 0's shared memory)
#pragma unroll
    for (int s = 1; s <= Slots; ++s)
        if (owns(s)) {
            const uint32_t g = rowBegin + local(s), pos = finalPosition(g);
            if (pos != g)
                for (uint32_t q = 0; q < jb; ++q)
                    st2(column(q) + 2 * pos, ld2(column(q) + 2 * g));
        }
    cluster.sync();
    if (owns(0)) {
        const uint32_t g = rowBegin + i, pos = finalPosition(g);
        for (uint32_t q = 0; q < jb; ++q)
            st2(column(q) + 2 * pos, P[size_t(q) * cap + i]);
    }
    cluster.sync();  // keep rank 0's map alive until every CTA has read it
}

template <class R> size_t panelSmemBytes(uint32_t rows, uint32_t jb) {
    return size_t(rows) * jb * sizeof(C2<R>) + size_t(rows) * 8;
}
constexpr size_t kPanelSmemLimit = 220 * 1024;

// FP32 panel factorisation with the panel in registers, for full 32-column
// panels of at most kRegPanelRows rows: thread t owns panel rows
// t + r * blockDim.x (r < kRegRowsPerThread), 32 complex values each, so the
// elimination reads nothing but the pivot row. Pivot rule, tie rule and
// interchange sequence are those of panelSmemKernel, and every entry of a
// row that is not yet a pivot row is updated by the same operations in the
// same order (a pivot row's multiplier is zero, which leaves finite values
// unchanged).
//
// Per column, each warp reduces its candidates by shuffles and the lane that
// holds the warp's best row writes that row's remaining columns to the
// warp's slot in shared memory; after the column's one barrier every warp
// reduces the warp candidates, reads the pivot row from the winning warp's
// slot and eliminates its own rows. Slots and candidates alternate with the
// column's parity: a warp writes the slot of column j + 2 only after the
// barrier of column j + 1, which every reader of column j has passed.
//
// Register indices must be constants, and a fully unrolled 32-column body is
// too long for the instruction cache (an earlier build stalled on
// instruction fetch for most of its cycles). So each row is rotated instead:
// at column j, a[r][c] holds column j + c for c < 32 - j and the finished
// columns j + c - 32 after them. The loop body handles kRegUnroll columns
// with constant indices (updates of the entries c >= 32 - j are predicated
// off) and rotates the rows by kRegUnroll at its end; after the 32 columns
// every row is back in column order.
// Eight warps, so that each SM sub-partition holds two and a thread may use
// 255 registers: 64 per row.
constexpr int kRegRowsPerThread = 3;
constexpr int kRegUnroll = 2;
constexpr uint32_t kRegPanelThreads = 256;
constexpr uint32_t kRegPanelRows = kRegRowsPerThread * kRegPanelThreads;
constexpr int kRegPanelWarps = int(kRegPanelThreads / 32);

__global__ void __launch_bounds__(kRegPanelThreads, 1) panelRegKernel(float *LU, uint32_t N, uint32_t k0, int *pivots,
                                                                      int *info) {
    constexpr int RT = kRegRowsPerThread, U = kRegUnroll;
    static_assert(kPanel % U == 0, "the column groups must tile the panel");
    __shared__ __align__(16) float2 sCand[2][kRegPanelWarps][kPanel];
    __shared__ float sBest[2][kRegPanelWarps];
    __shared__ int sRow[2][kRegPanelWarps];
    __shared__ int sSel[kPanel];
    __shared__ int arrangement[kRegPanelRows], where[kRegPanelRows];
    const uint32_t rows = N - k0, T = blockDim.x;
    float *M = LU + size_t(blockIdx.x) * N * N * 2;
    int *piv = pivots + size_t(blockIdx.x) * N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = int(T >> 5);
    int row[RT];
    bool have[RT], taken[RT];
    float2 a[RT][kPanel];
#pragma unroll
    for (int r = 0; r < RT; ++r) {
        row[r] = int(threadIdx.x + r * T);
        have[r] = uint32_t(row[r]) < rows;
        taken[r] = !have[r];
    }
#pragma unroll
    for (int q = 0; q < kPanel; ++q) {
        const float *col = M + 2 * (size_t(k0 + q) * N + k0);
#pragma unroll
        for (int r = 0; r < RT; ++r)
            a[r][q] = have[r] ? ld2<float>(col + 2 * row[r]) : make_float2(0.f, 0.f);
    }
    for (uint32_t i = threadIdx.x; i < rows; i += T) {
        arrangement[i] = int(i);
        where[i] = int(i);
    }
    const auto magnitude = [](float2 z) {
        const float m = fabsf(z.x) + fabsf(z.y);
        return m >= 0.f ? m : 0.f;  // a NaN row competes as zero, so a pivot row always exists
    };
#pragma unroll 1
    for (int j0 = 0; j0 < kPanel; j0 += U) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            // column j = j0 + u sits at index u of the rotated rows; its remaining
            // columns at indices u .. u + left - 1
            const int j = j0 + u, buf = j & 1, left = kPanel - j;
            float best = -1.f;
            int bestRow = int(rows), bestSlot = -1;
#pragma unroll
            for (int r = 0; r < RT; ++r)
                if (!taken[r]) {
                    const float m = magnitude(a[r][u]);
                    if (m > best) {  // rows ascend with r: ties keep the lower row
                        best = m;
                        bestRow = row[r];
                        bestSlot = r;
                    }
                }
            const int myRow = bestRow;
            for (int off = 16; off > 0; off >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, best, off);
                const int oi = __shfl_xor_sync(0xffffffffu, bestRow, off);
                if (ob > best || (ob == best && oi < bestRow)) {
                    best = ob;
                    bestRow = oi;
                }
            }
            // the warp's candidate row (slot entry c = column j + c; entries past the
            // panel's end are never read)
            if (bestSlot >= 0 && myRow == bestRow) {
                float4 *dst = reinterpret_cast<float4 *>(&sCand[buf][warp][0]);
#pragma unroll
                for (int c = 0; c < kPanel; c += 2) {
                    float2 x0 = a[0][(u + c) % kPanel], x1 = a[0][(u + c + 1) % kPanel];
#pragma unroll
                    for (int r = 1; r < RT; ++r)
                        if (bestSlot == r) {
                            x0 = a[r][(u + c) % kPanel];
                            x1 = a[r][(u + c + 1) % kPanel];
                        }
                    dst[c / 2] = make_float4(x0.x, x0.y, x1.x, x1.y);
                }
            }
            if (lane == 0) {
                sBest[buf][warp] = best;
                sRow[buf][warp] = bestRow;
            }
            __syncthreads();
            // every warp reduces the warp candidates by shuffles (same result in every warp)
            float pb = lane < warps ? sBest[buf][lane] : -1.f;
            int p = lane < warps ? sRow[buf][lane] : int(rows), pw = lane;
            for (int off = 16; off > 0; off >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, pb, off);
                const int oi = __shfl_xor_sync(0xffffffffu, p, off), ow = __shfl_xor_sync(0xffffffffu, pw, off);
                if (ob > pb || (ob == pb && oi < p)) {
                    pb = ob;
                    p = oi;
                    pw = ow;
                }
            }
            if (threadIdx.x == 0) {
                sSel[j] = p;
                if (!(pb > 0.f) && *info == 0)
                    atomicCAS(info, 0, int(k0) + j + 1);
            }
            const float2 *prow = sCand[buf][pw];
            const float2 d = prow[0];
            const float den = d.x * d.x + d.y * d.y;
            const float rden = den > 0.f ? 1.f / den : 0.f;
            const float2 inv = make_float2(d.x * rden, -d.y * rden);
            // a row already chosen as a pivot row keeps its values: its multiplier is zero
            float2 l[RT];
#pragma unroll
            for (int r = 0; r < RT; ++r) {
                taken[r] |= p == row[r];
                const float2 m = cmul<float>(a[r][u], inv);
                l[r] = taken[r] ? make_float2(0.f, 0.f) : m;
                a[r][u] = taken[r] ? a[r][u] : m;
            }
#pragma unroll
            for (int c = 1; c < kPanel; ++c) {
                if (c >= left)  // finished columns
                    break;
                const float2 pv = prow[c];
#pragma unroll
                for (int r = 0; r < RT; ++r)
                    csub<float>(a[r][(u + c) % kPanel], l[r], pv);
            }
        }
        // rotate every row left by U: index c takes column j0 + U + c
        float2 t[RT][U];
#pragma unroll
        for (int r = 0; r < RT; ++r) {
#pragma unroll
            for (int c = 0; c < U; ++c)
                t[r][c] = a[r][c];
#pragma unroll
            for (int c = 0; c + U < kPanel; ++c)
                a[r][c] = a[r][c + U];
#pragma unroll
            for (int c = 0; c < U; ++c)
                a[r][kPanel - U + c] = t[r][c];
        }
    }
    __syncthreads();
    // selection order -> interchange sequence (row k0+j swapped with row piv[k0+j])
    if (threadIdx.x == 0)
        for (int j = 0; j < kPanel; ++j) {
            const int r = sSel[j], pj = where[r], rj = arrangement[j];
            piv[k0 + j] = int(k0) + pj;
            arrangement[j] = r;
            arrangement[pj] = rj;
            where[r] = j;
            where[rj] = pj;
        }
    __syncthreads();
    // row r of this thread goes to position where[row]; one running pointer per row
    float *out[RT];
#pragma unroll
    for (int r = 0; r < RT; ++r)
        out[r] = M + 2 * (size_t(k0) * N + k0 + (have[r] ? where[row[r]] : 0));
    const size_t stride = size_t(N) * 2;
#pragma unroll
    for (int q = 0; q < kPanel; ++q)
#pragma unroll
        for (int r = 0; r < RT; ++r) {
            if (have[r])
                st2<float>(out[r], a[r][q]);
            out[r] += stride;
        }
}

// Row interchanges of the panel applied to columns outside it.
template <class R> __global__ void swapKernel(R *LU, uint32_t N, uint32_t k0, uint32_t jb, const int *pivots) {
    const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= N || (col >= k0 && col < k0 + jb))
        return;
    R *M = LU + size_t(blockIdx.y) * N * N * 2 + 2 * size_t(col) * N;
    const int *piv = pivots + size_t(blockIdx.y) * N;
    for (uint32_t c = k0; c < k0 + jb; ++c) {
        const int p = piv[c];
        if (p != int(c)) {
            const C2<R> a = ld2(M + 2 * c), b = ld2(M + 2 * p);
            st2(M + 2 * c, b);
            st2(M + 2 * p, a);
        }
    }
}

// U12 = L11^{-1} A12 (unit lower L11 of the panel) for columns
// [k0 + jb, cEnd), 32 per CTA: L11 and the 32x32 tile of A12 are staged in
// shared memory with coalesced column reads; a warp solves one column at a
// time (lane = row, L11 row in registers, the solved unknown broadcast by
// shuffle).
template <class R>
__global__ void __launch_bounds__(256) trsmKernel(R *LU, uint32_t N, uint32_t k0, uint32_t jb, uint32_t cEnd) {
    __shared__ C2<R> L[kPanel][kPanel + 1];
    __shared__ C2<R> X[kPanel][kPanel + 1];  // [column][row]
    R *M = LU + size_t(blockIdx.y) * N * N * 2;
    const uint32_t c0 = k0 + jb + blockIdx.x * kPanel;
    const uint32_t cols = min(uint32_t(kPanel), cEnd - c0);
    for (uint32_t e = threadIdx.x; e < jb * jb; e += blockDim.x) {
        const uint32_t r = e % jb, c = e / jb;
        L[r][c] = ld2(M + 2 * (size_t(k0 + c) * N + k0 + r));
    }
    for (uint32_t e = threadIdx.x; e < cols * jb; e += blockDim.x) {
        const uint32_t r = e % jb, c = e / jb;
        X[c][r] = ld2(M + 2 * (size_t(c0 + c) * N + k0 + r));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    C2<R> row[kPanel];
#pragma unroll
    for (int m = 0; m < kPanel; ++m)
        row[m] = (lane < int(jb) && m < int(jb)) ? L[lane][m] : mk<R>(0, 0);
    for (uint32_t c = warp; c < cols; c += blockDim.x >> 5) {
        C2<R> v = lane < int(jb) ? X[c][lane] : mk<R>(0, 0);
#pragma unroll
        for (int m = 0; m < kPanel; ++m) {
            const C2<R> xm = mk<R>(__shfl_sync(0xffffffffu, v.x, m), __shfl_sync(0xffffffffu, v.y, m));
            if (lane > m)
                csub<R>(v, row[m], xm);
        }
        if (lane < int(jb))
            X[c][lane] = v;
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < cols * jb; e += blockDim.x) {
        const uint32_t r = e % jb, c = e / jb;
        st2(M + 2 * (size_t(c0 + c) * N + k0 + r), X[c][r]);
    }
}

// A22 -= L21 * U12 with 64x64 output tiles, K = jb <= 32, over rows
// [k0 + jb, N) and columns [k0 + jb, cEnd).
template <class R>
__global__ void __launch_bounds__(256) gemmKernel(R *LU, uint32_t N, uint32_t k0, uint32_t jb, uint32_t cEnd) {
    extern __shared__ __align__(16) unsigned char rawSmem[];
    C2<R> *sA = reinterpret_cast<C2<R> *>(rawSmem);  // [kPanel][64]  L21 tile, k-major
    C2<R> *sB = sA + kPanel * 64;                      // [kPanel][64]  U12 tile, k-major
    R *M = LU + size_t(blockIdx.z) * N * N * 2;
    const uint32_t r0 = k0 + jb + blockIdx.x * 64, c0 = k0 + jb + blockIdx.y * 64;
    for (uint32_t e = threadIdx.x; e < jb * 64; e += blockDim.x) {
        const uint32_t kk = e / 64, x = e % 64;
        const uint32_t r = r0 + x, c = c0 + x;
        sA[kk * 64 + x] = r < N ? ld2(M + 2 * (size_t(k0 + kk) * N + r)) : mk<R>(0, 0);
        sB[kk * 64 + x] = c < cEnd ? ld2(M + 2 * (size_t(c) * N + k0 + kk)) : mk<R>(0, 0);
    }
    __syncthreads();
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    C2<R> acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
            acc[i][j] = mk<R>(0, 0);
    for (uint32_t kk = 0; kk < jb; ++kk) {
        C2<R> a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            a[i] = sA[kk * 64 + tx + 16 * i];
            b[i] = sB[kk * 64 + ty + 16 * i];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                acc[i][j].x += a[i].x * b[j].x - a[i].y * b[j].y;
                acc[i][j].y += a[i].x * b[j].y + a[i].y * b[j].x;
            }
    }
    // the 16 outputs are read first (independent loads in flight), then written
    C2<R> old[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t r = r0 + tx + 16 * i, c = c0 + ty + 16 * j;
            old[i][j] = (r < N && c < cEnd) ? ld2(M + 2 * (size_t(c) * N + r)) : mk<R>(0, 0);
        }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t r = r0 + tx + 16 * i, c = c0 + ty + 16 * j;
            if (r < N && c < cEnd)
                st2(M + 2 * (size_t(c) * N + r), mk<R>(old[i][j].x - acc[i][j].x, old[i][j].y - acc[i][j].y));
        }
}

// ---------------------------------------------------------------------------
// FP32 trailing update of the two-level factorisation on the tensor cores
// (tcgen05): A22 -= L21 * U12 with K = kOuter = 128 complex columns, as a real
// GEMM of the split complex operands, output real parts and imaginary parts
// side by side:
//   [C_re, C_im] = [L_re, L_im] * [[U_re, U_im]; [-U_im, U_re]].
// Operands are multiplied as hi*hi + hi*lo + lo*hi (3xTF32: TF32 hi part plus
// TF32 remainder) with FP32 accumulation, which keeps FP32 accuracy.
//
// packKernel converts L21 and U12 once per outer block into operand tiles
// that are already in the tensor cores' shared-memory layout (K-major,
// unswizzled canonical layout: 8-row x 16-byte core matrices, row groups 128 B
// apart (SBO), 16-byte K chunks (rows/8)*128 B apart (LBO)), hi then lo, one
// tile per 128 rows (A) or 64 complex columns (B, 128 operand rows) and per
// stage of 16 complex K columns. trailingTensorKernel then owns 128 complex
// rows x 64 complex columns of A22 (an M = 128, N = 128 real accumulator in
// tensor memory) and runs three roles:
//   * warp 0 copies the stage tiles into a ring of kTcStages shared-memory
//     buffers with bulk asynchronous copies that complete on the buffer's
//     `full` mbarrier;
//   * warp 1 issues the stage's MMAs from one thread and commits them to the
//     buffer's `empty` mbarrier, which lets warp 0 refill it; after the last
//     stage it commits to `done`;
//   * every thread loads its 32 outputs of A22 at the start (the loads overlap
//     the main loop), waits for `done`, reads its accumulator row (32 lanes x
//     32 columns, real and imaginary parts) from tensor memory and writes the
//     updated outputs (a warp writes 32 consecutive rows of a column).
// Every wait is bounded by a clock budget; a timeout leaves kTensorTimeout in
// the LU status word and skips the update.
// ---------------------------------------------------------------------------
constexpr int kOuter = 128;                            // outer block width of the two-level factorisation
constexpr int kTcRows = 128, kTcCols = 64, kTcK = 16;  // complex rows, complex columns, complex K per stage
constexpr int kTcStages = 3, kTcThreads = 256;
constexpr int kTcSteps = kOuter / kTcK;                // stages per update
constexpr int kTcTile = 2 * kTcRows * (2 * kTcK);      // floats of one operand tile, hi + lo (A and B alike)
constexpr size_t kTcSmem = size_t(kTcStages) * 2 * kTcTile * sizeof(float);  // 192 KB: one CTA per SM
constexpr int kTensorTimeout = -1;
constexpr long long kWaitCycles = 4000000000ll;  // about two seconds

static_assert(2 * kTcCols == kTcRows, "A and B operand tiles have the same shape");
static_assert(kOuter % kTcK == 0 && kOuter % kPanel == 0, "outer block must hold whole stages and panels");
static_assert(kTcSmem > 114 * 1024 && kTcSmem <= 227 * 1024, "one CTA per SM keeps tensor-memory allocation uncontended");

// floats of the packed operand tiles of one matrix (the first outer block has the most)
size_t packFloats(uint32_t N) {
    if (N <= uint32_t(kOuter))
        return 0;
    const size_t rest = N - kOuter;
    return ((rest + kTcRows - 1) / kTcRows + (rest + kTcCols - 1) / kTcCols) * kTcSteps * size_t(kTcTile);
}

__device__ __forceinline__ uint32_t smemAddr(const void *p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ float tf32Round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// offset (floats) of element (row r, k) in a K-major core-matrix tile of `rows` rows
__device__ __forceinline__ int coreOffset(int r, int k, int rows) {
    return ((k >> 2) * (rows >> 3) + (r >> 3)) * 32 + (r & 7) * 4 + (k & 3);
}

// UMMA shared-memory matrix descriptor: start, LBO, SBO (16-byte units), version 1, no swizzle
__device__ __forceinline__ uint64_t matrixDescriptor(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}

// Bounded wait for the phase of `parity` on an mbarrier; false on timeout.
__device__ __forceinline__ bool waitPhase(uint32_t bar, uint32_t parity) {
    const long long start = clock64();
    uint32_t done = 0;
    while (!done) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity));
        if (!done && clock64() - start > kWaitCycles)
            return false;
    }
    return true;
}

// Operand tiles of one outer block: per matrix the A tiles of L21 [row tile][stage], then the B tiles
// of U12 [column tile][stage]. Grid: (row tiles + column tiles, stages, matrices).
__global__ void __launch_bounds__(256) packKernel(const float *LU, uint32_t N, uint32_t K0, float *pack,
                                                  size_t packStride) {
    const uint32_t begin = K0 + kOuter, rest = N - begin;
    const uint32_t rowTiles = (rest + kTcRows - 1) / kTcRows, t = blockIdx.x, c = blockIdx.y;
    const float *M = LU + size_t(blockIdx.z) * N * N * 2;
    float *hi = pack + blockIdx.z * packStride + (size_t(t) * kTcSteps + c) * kTcTile, *lo = hi + kTcTile / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t kc = K0 + c * kTcK;
    // a warp fills whole core matrices: lane = (row & 7) * 4 + (k & 3), 32 stores to 128 contiguous bytes
    if (t < rowTiles) {  // A: row i takes (L_re, L_im) at k and k + 16
        const uint32_t r0 = begin + t * kTcRows;
        float2 v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int cm = warp + 8 * q, i = (cm % 16) * 8 + (lane >> 2), k = (cm / 16) * 4 + (lane & 3);
            v[q] = r0 + i < N ? *reinterpret_cast<const float2 *>(M + 2 * (size_t(kc + k) * N + r0 + i))
                              : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int cm = warp + 8 * q, i = (cm % 16) * 8 + (lane >> 2), k = (cm / 16) * 4 + (lane & 3);
            const float hr = tf32Round(v[q].x), hm = tf32Round(v[q].y);
            hi[coreOffset(i, k, kTcRows)] = hr;
            lo[coreOffset(i, k, kTcRows)] = tf32Round(v[q].x - hr);
            hi[coreOffset(i, k + kTcK, kTcRows)] = hm;
            lo[coreOffset(i, k + kTcK, kTcRows)] = tf32Round(v[q].y - hm);
        }
    } else {  // B: operand row j takes (U_re, -U_im), row j + 64 takes (U_im, U_re)
        const uint32_t c0 = begin + (t - rowTiles) * kTcCols;
        float2 v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int cm = warp + 8 * q, j = (cm % 8) * 8 + (lane >> 2), k = (cm / 8) * 4 + (lane & 3);
            v[q] = c0 + j < N ? *reinterpret_cast<const float2 *>(M + 2 * (size_t(c0 + j) * N + kc + k))
                              : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int cm = warp + 8 * q, j = (cm % 8) * 8 + (lane >> 2), k = (cm / 8) * 4 + (lane & 3);
            const float parts[4] = {v[q].x, -v[q].y, v[q].y, v[q].x};  // (j, k), (j, k+16), (j+64, k), (j+64, k+16)
            const int rows[4] = {j, j, j + kTcCols, j + kTcCols}, ks[4] = {k, k + kTcK, k, k + kTcK};
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const float h = tf32Round(parts[p]);
                hi[coreOffset(rows[p], ks[p], kTcRows)] = h;
                lo[coreOffset(rows[p], ks[p], kTcRows)] = tf32Round(parts[p] - h);
            }
        }
    }
}

__global__ void __launch_bounds__(kTcThreads, 1) trailingTensorKernel(float *LU, uint32_t N, uint32_t K0,
                                                                      const float *pack, size_t packStride,
                                                                      int *info) {
    extern __shared__ __align__(1024) float ring[];  // kTcStages x {A hi, A lo, B hi, B lo}
    __shared__ __align__(8) uint64_t full[kTcStages], empty[kTcStages], done;
    __shared__ uint32_t tmemBase;
    constexpr int NB = 2 * kTcCols;  // real accumulator columns
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t begin = K0 + kOuter, rest = N - begin;
    const uint32_t rowTiles = (rest + kTcRows - 1) / kTcRows;
    const uint32_t r0 = begin + blockIdx.x * kTcRows, c0 = begin + blockIdx.y * kTcCols;
    float *M = LU + size_t(blockIdx.z) * N * N * 2;
    const float *tilesA = pack + blockIdx.z * packStride + size_t(blockIdx.x) * kTcSteps * kTcTile;
    const float *tilesB = pack + blockIdx.z * packStride + (size_t(rowTiles) + blockIdx.y) * kTcSteps * kTcTile;
    // this thread's outputs: row 32 (warp % 4) + lane, columns 32 (warp / 4) .. + 31
    const int quarter = warp & 3, half = warp >> 2;
    const uint32_t row = r0 + quarter * 32 + lane, col0 = c0 + half * 32;
    float2 old[32];
#pragma unroll
    for (int j = 0; j < 32; ++j)
        old[j] = (row < N && col0 + j < N) ? *reinterpret_cast<const float2 *>(M + 2 * (size_t(col0 + j) * N + row))
                                           : make_float2(0.f, 0.f);
    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(&empty[s])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(&done)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(&tmemBase)),
                     "r"(NB));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        asm volatile("tcgen05.fence::before_thread_sync;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmemBase;
    bool ok = true;
    int issued = 0;
    if (warp == 0) {  // producer
        for (int c = 0; c < kTcSteps; ++c) {
            const int s = c % kTcStages;
            if (c >= kTcStages) {  // the MMAs of stage c - kTcStages have read this buffer
                ok = __all_sync(0xffffffffu, waitPhase(smemAddr(&empty[s]), uint32_t((c - kTcStages) / kTcStages) & 1u));
                if (!ok)
                    break;
            }
            if (lane == 0) {
                const uint32_t dst = smemAddr(ring + size_t(s) * 2 * kTcTile), bar = smemAddr(&full[s]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                             "r"(uint32_t(2 * kTcTile * sizeof(float))));
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                    "l"(tilesA + size_t(c) * kTcTile), "r"(uint32_t(kTcTile * sizeof(float))), "r"(bar)
                    : "memory");
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        dst + uint32_t(kTcTile * sizeof(float))),
                    "l"(tilesB + size_t(c) * kTcTile), "r"(uint32_t(kTcTile * sizeof(float))), "r"(bar)
                    : "memory");
            }
            issued = c + 1;
        }
    } else if (warp == 1) {  // MMA issue
        // D: F32; A, B: TF32, K-major; N = NB (>> 3), M = 128 (>> 4)
        constexpr uint32_t idesc =
            (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(NB >> 3) << 17) | (uint32_t(kTcRows >> 4) << 24);
        constexpr uint32_t lbo = (kTcRows / 8) * 128, sbo = 128;
        for (int c = 0; c < kTcSteps; ++c) {
            const int s = c % kTcStages;
            ok = __all_sync(0xffffffffu, waitPhase(smemAddr(&full[s]), uint32_t(c / kTcStages) & 1u));
            if (!ok)
                break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (lane == 0) {
                const uint32_t aHi = smemAddr(ring + size_t(s) * 2 * kTcTile), aLo = aHi + kTcTile * 2;
                const uint32_t bHi = aHi + kTcTile * 4, bLo = bHi + kTcTile * 2;
                const uint32_t As[3] = {aHi, aHi, aLo}, Bs[3] = {bHi, bLo, bHi};
#pragma unroll
                for (int pass = 0; pass < 3; ++pass)
#pragma unroll
                    for (int step = 0; step < 2 * kTcK / 8; ++step) {
                        const uint64_t da = matrixDescriptor(As[pass] + uint32_t(2 * step) * lbo, lbo, sbo);
                        const uint64_t db = matrixDescriptor(Bs[pass] + uint32_t(2 * step) * lbo, lbo, sbo);
                        const uint32_t accumulate = (c | pass | step) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                            "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
                    }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smemAddr(&empty[s])));
                if (c == kTcSteps - 1)  // completes when every MMA of the CTA has
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                        smemAddr(&done)));
            }
            __syncwarp();
        }
    }
    const bool accumulated = __syncthreads_and(ok && waitPhase(smemAddr(&done), 0));
    if (!accumulated) {
        if (tid == 0)
            atomicCAS(info, 0, kTensorTimeout);
        if (warp == 0)  // let the last copies into each buffer land before the CTA exits
            for (int c = issued > kTcStages ? issued - kTcStages : 0; c < issued; ++c)
                waitPhase(smemAddr(&full[c % kTcStages]), uint32_t(c / kTcStages) & 1u);
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (accumulated) {
        uint32_t re[32], im[32];
        const uint32_t lanes = uint32_t(quarter * 32) << 16;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(re[0]), "=r"(re[1]), "=r"(re[2]), "=r"(re[3]), "=r"(re[4]), "=r"(re[5]), "=r"(re[6]), "=r"(re[7]),
              "=r"(re[8]), "=r"(re[9]), "=r"(re[10]), "=r"(re[11]), "=r"(re[12]), "=r"(re[13]), "=r"(re[14]),
              "=r"(re[15]), "=r"(re[16]), "=r"(re[17]), "=r"(re[18]), "=r"(re[19]), "=r"(re[20]), "=r"(re[21]),
              "=r"(re[22]), "=r"(re[23]), "=r"(re[24]), "=r"(re[25]), "=r"(re[26]), "=r"(re[27]), "=r"(re[28]),
              "=r"(re[29]), "=r"(re[30]), "=r"(re[31])
            : "r"(tmem + lanes + uint32_t(half * 32)));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(im[0]), "=r"(im[1]), "=r"(im[2]), "=r"(im[3]), "=r"(im[4]), "=r"(im[5]), "=r"(im[6]), "=r"(im[7]),
              "=r"(im[8]), "=r"(im[9]), "=r"(im[10]), "=r"(im[11]), "=r"(im[12]), "=r"(im[13]), "=r"(im[14]),
              "=r"(im[15]), "=r"(im[16]), "=r"(im[17]), "=r"(im[18]), "=r"(im[19]), "=r"(im[20]), "=r"(im[21]),
              "=r"(im[22]), "=r"(im[23]), "=r"(im[24]), "=r"(im[25]), "=r"(im[26]), "=r"(im[27]), "=r"(im[28]),
              "=r"(im[29]), "=r"(im[30]), "=r"(im[31])
            : "r"(tmem + lanes + uint32_t(kTcCols + half * 32)));
        asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (row < N && col0 + j < N)
                *reinterpret_cast<float2 *>(M + 2 * (size_t(col0 + j) * N + row)) =
                    make_float2(old[j].x - __uint_as_float(re[j]), old[j].y - __uint_as_float(im[j]));
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 2)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NB));
}

// U12 = L11^{-1} A12 for the outer block (L11: the kOuter x kOuter unit lower
// triangle at (K0, K0)), over the trailing columns [K0 + kOuter, N). L11 is
// staged in shared memory column by column (coalesced); a warp solves one
// column at a time with lane l holding rows l, l + 32, l + 64, l + 96 in
// registers and the solved unknown broadcast by shuffle.
constexpr int kTrsmColumns = 64, kTrsmThreads = 512;
constexpr size_t kTrsmSmem = size_t(kOuter) * kOuter * sizeof(float2);  // 128 KB

__global__ void __launch_bounds__(kTrsmThreads, 1) trsmBlockKernel(float *LU, uint32_t N, uint32_t K0) {
    extern __shared__ __align__(16) float2 Lc[];  // [column m][row]
    float *M = LU + size_t(blockIdx.y) * N * N * 2;
    for (uint32_t e = threadIdx.x; e < uint32_t(kOuter * kOuter); e += blockDim.x) {
        const uint32_t r = e % kOuter, m = e / kOuter;
        Lc[e] = *reinterpret_cast<const float2 *>(M + 2 * (size_t(K0 + m) * N + K0 + r));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t c0 = K0 + kOuter + blockIdx.x * kTrsmColumns;
    for (uint32_t c = c0 + warp; c < min(N, c0 + kTrsmColumns); c += kTrsmThreads / 32) {
        float2 *col = reinterpret_cast<float2 *>(M + 2 * (size_t(c) * N + K0));
        float2 v[4];
#pragma unroll
        for (int s = 0; s < 4; ++s)
            v[s] = col[lane + 32 * s];
#pragma unroll
        for (int sb = 0; sb < 4; ++sb)
#pragma unroll 8
            for (int mm = 0; mm < 32; ++mm) {
                const int m = 32 * sb + mm;
                const float2 x =
                    make_float2(__shfl_sync(0xffffffffu, v[sb].x, mm), __shfl_sync(0xffffffffu, v[sb].y, mm));
#pragma unroll
                for (int s = sb; s < 4; ++s)
                    if (lane + 32 * s > m) {
                        const float2 a = Lc[m * kOuter + lane + 32 * s];
                        v[s].x -= a.x * x.x - a.y * x.y;
                        v[s].y -= a.x * x.y + a.y * x.x;
                    }
            }
#pragma unroll
        for (int s = 0; s < 4; ++s)
            col[lane + 32 * s] = v[s];
    }
}

// Forward / back substitution of one right-hand side per CTA, with the
// vector staged in shared memory. Blocks of 32 unknowns: warp 0 loads the
// 32x32 diagonal block into registers (independent coalesced loads, lane =
// row) and solves it with shuffles; then every thread updates its rows with
// the block's 32 columns.
template <class R>
__global__ void __launch_bounds__(sizeof(R) == 8 ? 256 : 512) solveKernel(const R *LU, const int *pivots, uint32_t N, uint32_t E, R *X) {
    extern __shared__ __align__(16) unsigned char rawSmem[];
    C2<R> *x = reinterpret_cast<C2<R> *>(rawSmem);
    const uint32_t e = blockIdx.x, f = blockIdx.y;
    const R *M = LU + size_t(f) * N * N * 2;
    // the factorisation's row interchanges, composed into one permutation
    // (stored after the batch's interchange sequences): a parallel gather
    const int *perm = pivots + (size_t(gridDim.y) + f) * N;
    R *out = X + (size_t(f) * E + e) * N * 2;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
        x[i] = ld2(out + 2 * perm[i]);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const C2<R> zero = mk<R>(0, 0);
    // forward: unit lower triangle
    for (uint32_t k = 0; k < N; k += 32) {
        const uint32_t kb = min(32u, N - k);
        if (warp == 0) {
            C2<R> L[32];
#pragma unroll
            for (int m = 0; m < 32; ++m)
                L[m] = (m < int(kb) && lane < int(kb)) ? ld2(M + 2 * (size_t(k + m) * N + k + lane)) : zero;
            C2<R> mine = lane < int(kb) ? x[k + lane] : zero;
#pragma unroll
            for (int m = 0; m < 32; ++m) {
                const C2<R> xm = mk<R>(__shfl_sync(0xffffffffu, mine.x, m), __shfl_sync(0xffffffffu, mine.y, m));
                if (lane > m)
                    csub<R>(mine, L[m], xm);
            }
            if (lane < int(kb))
                x[k + lane] = mine;
        }
        __syncthreads();
        if (kb == 32) {
            for (uint32_t i = k + 32 + threadIdx.x; i < N; i += blockDim.x) {
                C2<R> v = x[i];
#pragma unroll
                for (int m = 0; m < 32; ++m)
                    csub<R>(v, ld2(M + 2 * (size_t(k + m) * N + i)), x[k + m]);
                x[i] = v;
            }
        }
        __syncthreads();
    }
    // backward: upper triangle with its diagonal
    const uint32_t blocks = (N + 31) / 32;
    for (uint32_t bi = blocks; bi-- > 0;) {
        const uint32_t k = bi * 32, kb = min(32u, N - k);
        if (warp == 0) {
            C2<R> U[32];
#pragma unroll
            for (int m = 0; m < 32; ++m)
                U[m] = (m < int(kb) && lane < int(kb)) ? ld2(M + 2 * (size_t(k + m) * N + k + lane)) : zero;
            C2<R> mine = lane < int(kb) ? x[k + lane] : zero;
#pragma unroll
            for (int m = 31; m >= 0; --m) {
                if (m < int(kb)) {
                    if (lane == m) {
                        const C2<R> d = U[m];
                        const R den = d.x * d.x + d.y * d.y;
                        mine = mk<R>((mine.x * d.x + mine.y * d.y) / den, (mine.y * d.x - mine.x * d.y) / den);
                    }
                    const C2<R> xm = mk<R>(__shfl_sync(0xffffffffu, mine.x, m), __shfl_sync(0xffffffffu, mine.y, m));
                    if (lane < m)
                        csub<R>(mine, U[m], xm);
                }
            }
            if (lane < int(kb))
                x[k + lane] = mine;
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) {
            C2<R> v = x[i];
            if (kb == 32) {
#pragma unroll
                for (int m = 0; m < 32; ++m)
                    csub<R>(v, ld2(M + 2 * (size_t(k + m) * N + i)), x[k + m]);
            } else {
                for (uint32_t m = 0; m < kb; ++m)
                    csub<R>(v, ld2(M + 2 * (size_t(k + m) * N + i)), x[k + m]);
            }
            x[i] = v;
        }
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
        st2(out + 2 * i, x[i]);
}

// Blocked triangular solves for many CTAs. The row interchanges of a
// factorisation are composed once into a permutation (permutationKernel,
// stored after the interchanges), so a solve starts with a parallel gather of
// the right-hand side into a work vector. Forward and backward substitution
// then run in blocks of kTriBlock unknowns, one launch per block: CTA 0 brings
// the next block's rows up to date with the block solved last and solves the
// next diagonal block (32 x 32 sub-blocks in warp 0's registers, as in
// solveKernel); the other CTAs apply the block solved last to every remaining
// row (64 rows x 4 column groups of 32 per CTA, coalesced column reads, the four
// partial sums added in a fixed order). The backward sweep writes each solved
// block to the output vector.
constexpr uint32_t kTriBlock = 128, kTriRows = 64;
constexpr uint32_t kSmallSolve = 1024;  // up to this N the one-CTA-per-system kernel is faster

__global__ void permutationKernel(const int *pivots, uint32_t N, int *perm) {
    extern __shared__ int p[];  // [N] the permutation, [N] the interchange sequence
    int *piv = p + N;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
        p[i] = int(i);
        piv[i] = pivots[size_t(blockIdx.x) * N + i];
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (uint32_t c = 0; c < N; ++c) {
            const int q = piv[c];
            if (q != int(c)) {
                const int t = p[c];
                p[c] = p[q];
                p[q] = t;
            }
        }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
        perm[size_t(blockIdx.x) * N + i] = p[i];
}

// work[f][e][i] = x[f][e][perm[f][i]]
template <class R> __global__ void gatherRhsKernel(const R *x, const int *perm, uint32_t N, uint32_t E, R *work) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, e = blockIdx.y, f = blockIdx.z;
    if (i >= N)
        return;
    const size_t v = (size_t(f) * E + e) * N;
    st2(work + 2 * (v + i), ld2(x + 2 * (v + perm[size_t(f) * N + i])));
}

// One step of a sweep. Known block: unknowns [c0, c0 + cw) (cw = 0 on the first step); next block
// [n0, n0 + nw). Forward (Lower): unit lower triangle, updated rows [n0 + nw, N). Backward: upper
// triangle with its diagonal, updated rows [0, n0).
template <class R, bool Lower>
__global__ void __launch_bounds__(256) triStepKernel(const R *LU, uint32_t N, uint32_t E, R *work, R *out, uint32_t c0,
                                                     uint32_t cw, uint32_t n0, uint32_t nw) {
    __shared__ C2<R> y[kTriBlock];
    __shared__ C2<R> part[4][kTriBlock];
    __shared__ C2<R> v[kTriBlock];
    const uint32_t e = blockIdx.y, f = blockIdx.z, tid = threadIdx.x;
    const R *M = LU + size_t(f) * N * N * 2;
    R *w = work + (size_t(f) * E + e) * N * 2;
    const C2<R> zero = mk<R>(0, 0);
    for (uint32_t i = tid; i < cw; i += blockDim.x)
        y[i] = ld2(w + 2 * (c0 + i));
    __syncthreads();
    if (blockIdx.x > 0) {  // rows outside the next block
        const uint32_t i = tid % kTriRows, g = tid / kTriRows;
        const uint32_t r = (Lower ? n0 + nw : 0) + (blockIdx.x - 1) * kTriRows + i;
        const uint32_t rEnd = Lower ? N : n0;
        C2<R> acc = zero;
        if (r < rEnd) {
            if (cw == kTriBlock) {  // full block: the 32 column loads in flight together
                C2<R> a[32];
#pragma unroll
                for (int c = 0; c < 32; ++c)
                    a[c] = ld2(M + 2 * (size_t(c0 + 32 * g + c) * N + r));
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const C2<R> b = y[32 * g + c];
                    acc.x += a[c].x * b.x - a[c].y * b.y;
                    acc.y += a[c].x * b.y + a[c].y * b.x;
                }
            } else {
                const uint32_t cEnd = min(cw, 32 * g + 32);
                for (uint32_t c = 32 * g; c < cEnd; ++c) {
                    const C2<R> a = ld2(M + 2 * (size_t(c0 + c) * N + r)), b = y[c];
                    acc.x += a.x * b.x - a.y * b.y;
                    acc.y += a.x * b.y + a.y * b.x;
                }
            }
        }
        part[g][i] = acc;
        __syncthreads();
        if (g == 0 && r < rEnd) {
            C2<R> t = ld2(w + 2 * r);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                t.x -= part[q][i].x;
                t.y -= part[q][i].y;
            }
            st2(w + 2 * r, t);
        }
        return;
    }
    // CTA 0: the next block's rows, then its diagonal block
    {
        const uint32_t i = tid % kTriBlock, g = tid / kTriBlock;  // 2 groups of 64 columns
        C2<R> acc = zero;
        if (i < nw) {
            const uint32_t cEnd = min(cw, 64 * g + 64);
            for (uint32_t c = 64 * g; c < cEnd; c += 16) {  // 16 column loads in flight together
                C2<R> a[16];
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    a[q] = c + q < cEnd ? ld2(M + 2 * (size_t(c0 + c + q) * N + n0 + i)) : zero;
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const C2<R> b = c + q < cEnd ? y[c + q] : zero;
                    acc.x += a[q].x * b.x - a[q].y * b.y;
                    acc.y += a[q].x * b.y + a[q].y * b.x;
                }
            }
        }
        part[g][i] = acc;
        __syncthreads();
        if (tid < nw) {
            C2<R> t = ld2(w + 2 * (n0 + tid));
            t.x -= part[0][tid].x + part[1][tid].x;
            t.y -= part[0][tid].y + part[1][tid].y;
            v[tid] = t;
        }
        __syncthreads();
    }
    const int lane = tid & 31, warp = tid >> 5;
    const uint32_t subs = (nw + 31) / 32;
    for (uint32_t q = 0; q < subs; ++q) {
        const uint32_t sb = Lower ? q : subs - 1 - q;  // sub-block order
        const uint32_t k = 32 * sb, kb = min(32u, nw - k);
        if (warp == 0) {
            C2<R> L[32];
#pragma unroll
            for (int m = 0; m < 32; ++m)
                L[m] = (m < int(kb) && lane < int(kb)) ? ld2(M + 2 * (size_t(n0 + k + m) * N + n0 + k + lane)) : zero;
            C2<R> mine = lane < int(kb) ? v[k + lane] : zero;
            if (Lower) {
#pragma unroll
                for (int m = 0; m < 32; ++m) {
                    const C2<R> xm = mk<R>(__shfl_sync(0xffffffffu, mine.x, m), __shfl_sync(0xffffffffu, mine.y, m));
                    if (lane > m)
                        csub<R>(mine, L[m], xm);
                }
            } else {
#pragma unroll
                for (int m = 31; m >= 0; --m) {
                    if (m < int(kb)) {
                        if (lane == m) {
                            const C2<R> d = L[m];
                            const R den = d.x * d.x + d.y * d.y;
                            mine = mk<R>((mine.x * d.x + mine.y * d.y) / den, (mine.y * d.x - mine.x * d.y) / den);
                        }
                        const C2<R> xm =
                            mk<R>(__shfl_sync(0xffffffffu, mine.x, m), __shfl_sync(0xffffffffu, mine.y, m));
                        if (lane < m)
                            csub<R>(mine, L[m], xm);
                    }
                }
            }
            if (lane < int(kb))
                v[k + lane] = mine;
        }
        __syncthreads();
        // the rest of the block: rows after (forward) or before (backward) the sub-block
        const uint32_t rBegin = Lower ? k + kb : 0, rEnd = Lower ? nw : k;
        for (uint32_t r = rBegin + tid; r < rEnd; r += blockDim.x) {
            C2<R> t = v[r];
#pragma unroll 8
            for (uint32_t m = 0; m < kb; ++m)
                csub<R>(t, ld2(M + 2 * (size_t(n0 + k + m) * N + n0 + r)), v[k + m]);
            v[r] = t;
        }
        __syncthreads();
    }
    if (tid < nw) {
        st2(w + 2 * (n0 + tid), v[tid]);
        if (!Lower)
            st2(out + 2 * ((size_t(f) * E + e) * N + n0 + tid), v[tid]);
    }
}

// r = b - A x per row (FP64 accumulation), plus mass-scaled squares for the
// norms. A CTA takes 32 rows; its 8 warps take every 8th column, and the 8
// partial sums are added in a fixed order (deterministic).
__global__ void __launch_bounds__(256) residualKernel(const double *A, const double *b, const double *x,
                                                      const double *mass, uint32_t N, uint32_t E, double *correction,
                                                      double *squares) {
    __shared__ double2 part[8][32];
    const uint32_t lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const uint32_t a = blockIdx.x * 32 + lane;
    const uint32_t e = blockIdx.y, f = blockIdx.z;
    const double *M = A + size_t(f) * N * N * 2;
    const double *xv = x + (size_t(f) * E + e) * N * 2;
    double re = 0, im = 0;
    if (a < N)
        for (uint32_t c = g; c < N; c += 8) {
            const double2 m = ld2(M + 2 * (size_t(c) * N + a));
            const double2 v = ld2(xv + 2 * c);
            re += m.x * v.x - m.y * v.y;
            im += m.x * v.y + m.y * v.x;
        }
    part[g][lane] = mk<double>(re, im);
    __syncthreads();
    if (g != 0 || a >= N)
        return;
    re = 0;
    im = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        re += part[w][lane].x;
        im += part[w][lane].y;
    }
    const size_t idx = (size_t(f) * E + e) * N + a;
    const double2 bb = ld2(b + 2 * idx);
    re = bb.x - re;
    im = bb.y - im;
    st2(correction + 2 * idx, mk<double>(re, im));
    const double s = mass[a];
    squares[2 * idx] = (re * s) * (re * s) + (im * s) * (im * s);
    squares[2 * idx + 1] = (bb.x * s) * (bb.x * s) + (bb.y * s) * (bb.y * s);
}

// Deterministic per-vector sums of the squares -> norms[2] per (f, e).
__global__ void normKernel(const double *squares, uint32_t N, double *norms) {
    __shared__ double red[2][256];
    const size_t v = blockIdx.x;
    double r = 0, b = 0;
    for (uint32_t a = threadIdx.x; a < N; a += blockDim.x) {
        r += squares[2 * (v * N + a)];
        b += squares[2 * (v * N + a) + 1];
    }
    red[0][threadIdx.x] = r;
    red[1][threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < unsigned(s)) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        norms[2 * v] = sqrt(red[0][0]);
        norms[2 * v + 1] = sqrt(red[1][0]);
    }
}

__global__ void addKernel(double *x, const double *c, size_t count) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count)
        x[i] += c[i];
}
__global__ void addFromFloatKernel(double *x, const float *c, size_t count) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count)
        x[i] += double(c[i]);
}
__global__ void toFloatKernel(const double *in, float *out, size_t count) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count)
        out[i] = float(in[i]);
}

// Largest cluster the panel kernel may use on this device: 16 CTAs (opt-in)
// when the device can schedule such a cluster with full panel shared memory,
// else the portable 8, else none.
template <class R> uint32_t clusterLimitNow() {
    const size_t smem = size_t(kPanel) * kClusterRows<R> * sizeof(C2<R>);
    int limit = 0;
    for (const void *kernel : {reinterpret_cast<const void *>(panelClusterKernel<R, 0>),
                               reinterpret_cast<const void *>(panelClusterKernel<R, kGlobalSlots>)})
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
    for (uint32_t c : {kMaxCluster, 8u}) {
        if (c > 8 && (cudaFuncSetAttribute(panelClusterKernel<R, 0>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                          cudaSuccess ||
                      cudaFuncSetAttribute(panelClusterKernel<R, kGlobalSlots>,
                                           cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
            cudaGetLastError();
            continue;
        }
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(c, 1);
        cfg.blockDim = dim3(1024);  // the largest launch: rows kept in global memory as well
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, panelClusterKernel<R, kGlobalSlots>, &cfg) == cudaSuccess &&
            clusters > 0) {
            limit = int(c);
            break;
        }
        cudaGetLastError();
    }
    return uint32_t(limit);
}
template <class R> uint32_t clusterLimit() {
    static PerDeviceValue<uint32_t> limit;
    return limit.get([]() { return clusterLimitNow<R>(); });
}

// Right-looking LU with partial pivoting, 32-wide panels. FP64 runs one
// level: every panel updates the whole trailing matrix (K = 32). FP32 runs two
// levels: panels update only the rest of their kOuter-wide outer block, then
// the outer block's U12 is solved (trsmBlockKernel) and the trailing matrix is
// updated once with K = kOuter on the tensor cores (trailingTensorKernel).
// Pivot choices follow the same rule in both; only the order of the update
// sums differs.
template <class R> void factor(R *LU, uint32_t N, uint32_t B, int *pivots, int *info, cudaStream_t stream,
                               KernelTimer *timer, float *pack) {
    check(cudaMemsetAsync(info, 0, sizeof(int), stream), "LU info reset");
    const size_t gemmSmem = 2 * kPanel * 64 * sizeof(C2<R>);
    static PerDeviceOnce attributes;
    attributes.run([&]() {
        check(cudaFuncSetAttribute(gemmKernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(gemmSmem)),
              "gemm smem attribute");
        check(cudaFuncSetAttribute(panelSmemKernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(kPanelSmemLimit)),
              "panel smem attribute");
        if constexpr (sizeof(R) == 4) {
            check(cudaFuncSetAttribute(trailingTensorKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTcSmem)),
                  "tensor update smem attribute");
            check(cudaFuncSetAttribute(trsmBlockKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTrsmSmem)),
                  "block trsm smem attribute");
        }
    });
    const uint32_t outer = sizeof(R) == 4 ? uint32_t(kOuter) : N;
    for (uint32_t K0 = 0; K0 < N; K0 += outer) {
        const uint32_t end = std::min(N, K0 + outer);
        for (uint32_t k0 = K0; k0 < end; k0 += kPanel) {
            const uint32_t jb = std::min(uint32_t(kPanel), end - k0);
            {
                TimedScope s(timer, "lu_panel", stream);
                const size_t bytes = panelSmemBytes<R>(N - k0, jb);
                const uint32_t rows = N - k0;
                const uint32_t limit = clusterLimit<R>();
                if (sizeof(R) == 4 && jb == uint32_t(kPanel) && rows <= kRegPanelRows) {
                    const uint32_t threads =
                        std::max(32u, ((rows + kRegRowsPerThread - 1) / kRegRowsPerThread + 31) / 32 * 32);
                    panelRegKernel<<<B, threads, 0, stream>>>(reinterpret_cast<float *>(LU), N, k0, pivots, info);
                } else if (bytes > kPanelSmemLimit && rows <= limit * (kClusterRows<R> + kGlobalSlots * 1024u)) {
                    // as few CTAs as hold the panel in shared memory, else the whole cluster with the
                    // rows beyond kClusterRows per CTA kept in global memory
                    const uint32_t C = std::min(limit, (rows + kClusterRows<R> - 1) / kClusterRows<R>);
                    const uint32_t perBlock = (rows + C - 1) / C;
                    const uint32_t cap = std::min(perBlock, kClusterRows<R>);
                    cudaLaunchConfig_t cfg{};
                    cfg.gridDim = dim3(C, B);
                    cfg.blockDim = dim3(perBlock <= cap ? (perBlock + 31) / 32 * 32 : 1024u);
                    cfg.dynamicSmemBytes = size_t(jb) * cap * sizeof(C2<R>);
                    cfg.stream = stream;
                    cudaLaunchAttribute attr[1];
                    attr[0].id = cudaLaunchAttributeClusterDimension;
                    attr[0].val.clusterDim.x = C;
                    attr[0].val.clusterDim.y = 1;
                    attr[0].val.clusterDim.z = 1;
                    cfg.attrs = attr;
                    cfg.numAttrs = 1;
                    if (perBlock <= cap)
                        check(cudaLaunchKernelEx(&cfg, panelClusterKernel<R, 0>, LU, N, k0, jb, perBlock, cap, pivots,
                                                 info),
                              "cluster panel launch");
                    else
                        check(cudaLaunchKernelEx(&cfg, panelClusterKernel<R, kGlobalSlots>, LU, N, k0, jb, perBlock, cap,
                                                 pivots, info),
                              "cluster panel launch");
                } else if (bytes <= kPanelSmemLimit)
                    panelSmemKernel<R><<<B, std::min(1024u, (N - k0 + 31) / 32 * 32), bytes, stream>>>(
                        LU, N, k0, jb, pivots, info);
                else
                    panelKernel<R><<<B, 512, 0, stream>>>(LU, N, k0, jb, pivots, info);
            }
            {
                TimedScope s(timer, "lu_swap", stream);
                swapKernel<R><<<dim3((N + 127) / 128, B), 128, 0, stream>>>(LU, N, k0, jb, pivots);
            }
            const uint32_t cols = end - k0 - jb;  // columns of the outer block right of the panel
            if (cols) {
                {
                    TimedScope s(timer, "lu_trsm", stream);
                    trsmKernel<R><<<dim3((cols + kPanel - 1) / kPanel, B), 256, 0, stream>>>(LU, N, k0, jb, end);
                }
                TimedScope s(timer, "lu_gemm", stream);
                const uint32_t rows = N - k0 - jb;
                gemmKernel<R><<<dim3((rows + 63) / 64, (cols + 63) / 64, B), 256, gemmSmem, stream>>>(LU, N, k0, jb,
                                                                                                      end);
            }
            check(cudaGetLastError(), "LU launch");
        }
        if constexpr (sizeof(R) == 4) {
            if (end < N) {
                const uint32_t rest = N - end;
                {
                    TimedScope s(timer, "lu_trsm_outer", stream);
                    trsmBlockKernel<<<dim3((rest + kTrsmColumns - 1) / kTrsmColumns, B), kTrsmThreads, kTrsmSmem,
                                      stream>>>(LU, N, K0);
                }
                const uint32_t rowTiles = (rest + kTcRows - 1) / kTcRows, colTiles = (rest + kTcCols - 1) / kTcCols;
                const size_t packStride = packFloats(N);
                {
                    TimedScope s(timer, "lu_pack", stream);
                    packKernel<<<dim3(rowTiles + colTiles, kTcSteps, B), 256, 0, stream>>>(LU, N, K0, pack, packStride);
                }
                TimedScope s(timer, "lu_gemm_tensor", stream);
                trailingTensorKernel<<<dim3(rowTiles, colTiles, B), kTcThreads, kTcSmem, stream>>>(LU, N, K0, pack,
                                                                                                    packStride, info);
                check(cudaGetLastError(), "LU outer update launch");
            }
        }
    }
}

template <class R> void solve(const R *LU, const int *pivots, uint32_t N, uint32_t B, uint32_t E, R *x,
                              void *scratch, cudaStream_t stream, KernelTimer *timer) {
    TimedScope s(timer, "lu_solve", stream);
    const size_t smem = size_t(N) * sizeof(C2<R>);
    if (N <= kSmallSolve) {  // one CTA per system: the vector in shared memory, no launch per block
        static PerDeviceHighWater attr;
        if (smem > 48 * 1024 && attr.raise(smem))
            check(cudaFuncSetAttribute(solveKernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                  "solve smem attribute");
        solveKernel<R><<<dim3(E, B), sizeof(R) == 8 ? 256 : 512, smem, stream>>>(LU, pivots, N, E, x);
        check(cudaGetLastError(), "triangular solve launch");
        return;
    }
    const int *perm = pivots + size_t(B) * N;
    R *work = static_cast<R *>(scratch);
    gatherRhsKernel<R><<<dim3((N + 255) / 256, E, B), 256, 0, stream>>>(x, perm, N, E, work);
    const uint32_t blocks = (N + kTriBlock - 1) / kTriBlock;
    // forward: block b is solved in step b with the rows updated by block b - 1
    for (uint32_t b = 0; b < blocks; ++b) {
        const uint32_t n0 = b * kTriBlock, nw = std::min(kTriBlock, N - n0);
        const uint32_t c0 = b ? n0 - kTriBlock : 0, cw = b ? kTriBlock : 0;
        const uint32_t rows = N - n0 - nw;
        triStepKernel<R, true><<<dim3(1 + (rows + kTriRows - 1) / kTriRows, E, B), 256, 0, stream>>>(
            LU, N, E, work, x, c0, cw, n0, nw);
    }
    // backward: from the last block up
    for (uint32_t q = 0; q < blocks; ++q) {
        const uint32_t b = blocks - 1 - q;
        const uint32_t n0 = b * kTriBlock, nw = std::min(kTriBlock, N - n0);
        const uint32_t c0 = q ? n0 + kTriBlock : 0, cw = q ? std::min(kTriBlock, N - c0) : 0;
        triStepKernel<R, false><<<dim3(1 + (n0 + kTriRows - 1) / kTriRows, E, B), 256, 0, stream>>>(
            LU, N, E, work, x, c0, cw, n0, nw);
    }
    check(cudaGetLastError(), "triangular solve launch");
}

template <class R> void permutation(const int *pivots, uint32_t N, uint32_t B, cudaStream_t stream) {
    const size_t smem = 2 * size_t(N) * sizeof(int);
    static PerDeviceHighWater attr;
    if (smem > 48 * 1024 && attr.raise(smem))
        check(cudaFuncSetAttribute(permutationKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
              "permutation smem attribute");
    permutationKernel<<<B, 256, smem, stream>>>(pivots, N, const_cast<int *>(pivots) + size_t(B) * N);
    check(cudaGetLastError(), "permutation launch");
}

}  // namespace

void luFactorBatch(double *LU, uint32_t N, uint32_t B, int *pivots, int *info, cudaStream_t stream,
                   KernelTimer *timer) {
    factor<double>(LU, N, B, pivots, info, stream, timer, nullptr);
    permutation<double>(pivots, N, B, stream);
}
void luFactorBatch(float *LU, uint32_t N, uint32_t B, int *pivots, int *info, cudaStream_t stream,
                   KernelTimer *timer, float *pack) {
    factor<float>(LU, N, B, pivots, info, stream, timer, pack);
    permutation<float>(pivots, N, B, stream);
}
void luSolveBatch(const double *LU, const int *pivots, uint32_t N, uint32_t B, uint32_t E, double *x,
                  void *scratch, cudaStream_t stream, KernelTimer *timer) {
    solve<double>(LU, pivots, N, B, E, x, scratch, stream, timer);
}
void luSolveBatch(const float *LU, const int *pivots, uint32_t N, uint32_t B, uint32_t E, float *x,
                  void *scratch, cudaStream_t stream, KernelTimer *timer) {
    solve<float>(LU, pivots, N, B, E, x, scratch, stream, timer);
}

void residualBatch(const double *A, const double *b, const double *x, const double *mass, uint32_t N, uint32_t B,
                   uint32_t E, double *correction, double *norms, cudaStream_t stream, KernelTimer *timer) {
    double *squares = norms + 2 * size_t(B) * E;  // scratch after the norms
    {
        TimedScope s(timer, "residual", stream);
        residualKernel<<<dim3((N + 31) / 32, E, B), 256, 0, stream>>>(A, b, x, mass, N, E, correction, squares);
    }
    {
        TimedScope s(timer, "residual_norm", stream);
        normKernel<<<unsigned(B * E), 256, 0, stream>>>(squares, N, norms);
    }
    check(cudaGetLastError(), "residual launch");
}

void addCorrectionBatch(double *x, const double *correction, size_t count, cudaStream_t stream) {
    addKernel<<<unsigned((count + 255) / 256), 256, 0, stream>>>(x, correction, count);
    check(cudaGetLastError(), "refinement update launch");
}
void addCorrectionBatch(double *x, const float *correction, size_t count, cudaStream_t stream) {
    addFromFloatKernel<<<unsigned((count + 255) / 256), 256, 0, stream>>>(x, correction, count);
    check(cudaGetLastError(), "refinement update launch");
}
void roundToFloat(const double *in, float *out, size_t count, cudaStream_t stream) {
    toFloatKernel<<<unsigned((count + 255) / 256), 256, 0, stream>>>(in, out, count);
    check(cudaGetLastError(), "FP32 rounding launch");
}

namespace {
// Device memory of the LU test hook, freed on every exit path.
struct HookBuffer {
    void *p = nullptr;
    explicit HookBuffer(size_t bytes) { check(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "LU hook allocation"); }
    ~HookBuffer() { cudaFree(p); }
    HookBuffer(const HookBuffer &) = delete;
    HookBuffer &operator=(const HookBuffer &) = delete;
};
}  // namespace

void debugLuFactor(bool fp32, uint32_t N, uint32_t B, const double *matrices, double *factors, int *pivots,
                   int *info) {
    const size_t reals = size_t(B) * N * N * 2;
    cudaStream_t stream = nullptr;
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "LU hook stream");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{stream};
    HookBuffer lu(reals * (fp32 ? sizeof(float) : sizeof(double))), piv(luWorkspaceBytes(N, B)), status(sizeof(int));
    if (fp32) {
        HookBuffer pack(luPackBytes(N, B));
        std::vector<float> host(matrices, matrices + reals);
        check(cudaMemcpyAsync(lu.p, host.data(), reals * sizeof(float), cudaMemcpyHostToDevice, stream), "LU hook upload");
        luFactorBatch(static_cast<float *>(lu.p), N, B, static_cast<int *>(piv.p), static_cast<int *>(status.p), stream,
                      nullptr, static_cast<float *>(pack.p));
        check(cudaMemcpyAsync(host.data(), lu.p, reals * sizeof(float), cudaMemcpyDeviceToHost, stream), "LU hook download");
        check(cudaMemcpyAsync(pivots, piv.p, size_t(B) * N * sizeof(int), cudaMemcpyDeviceToHost, stream), "LU hook pivots");
        check(cudaMemcpyAsync(info, status.p, sizeof(int), cudaMemcpyDeviceToHost, stream), "LU hook status");
        check(cudaStreamSynchronize(stream), "LU hook");
        std::copy(host.begin(), host.end(), factors);
        return;
    }
    check(cudaMemcpyAsync(lu.p, matrices, reals * sizeof(double), cudaMemcpyHostToDevice, stream), "LU hook upload");
    luFactorBatch(static_cast<double *>(lu.p), N, B, static_cast<int *>(piv.p), static_cast<int *>(status.p), stream,
                  nullptr);
    check(cudaMemcpyAsync(factors, lu.p, reals * sizeof(double), cudaMemcpyDeviceToHost, stream), "LU hook download");
    check(cudaMemcpyAsync(pivots, piv.p, size_t(B) * N * sizeof(int), cudaMemcpyDeviceToHost, stream), "LU hook pivots");
    check(cudaMemcpyAsync(info, status.p, sizeof(int), cudaMemcpyDeviceToHost, stream), "LU hook status");
    check(cudaStreamSynchronize(stream), "LU hook");
}

size_t luWorkspaceBytes(uint32_t N, uint32_t B) { return 2 * size_t(B) * N * sizeof(int); }
size_t luPackBytes(uint32_t N, uint32_t B) { return size_t(B) * packFloats(N) * sizeof(float); }

}  // namespace hsb
