// FP64 Burton-Miller Galerkin assembly for sm_100a (the plain form).
//
// Method: modules/bem/cuda/cuda_solver.cu:266-540 with the FP64 sample of
// panel_integrals.cuh:166-198 — regular disjoint pairs with the qualified
// Dunavant 4/6/8 rule (or an accepted whole-panel 8/14 rule), touching pairs
// with Sauter-Schwab sectors, near pairs with their plan patches, plus half
// the P1 mass, rows equilibrated by the reciprocal lumped mass.
//
// B200 layout: a batch of frequencies runs in one launch (blockIdx.y). Each
// unordered regular or near pair is integrated once and yields both ordered
// blocks, because the reverse direction's double-layer kernel is the forward
// adjoint kernel at the same points. Pair blocks are written to per-pair
// records (no atomics) and reduced to the matrix by two deterministic
// gathers (trial vertex, then test vertex), so results are bit-reproducible.
#include "autotune.hpp"
#include "device_once.hpp"
#include "device_types.cuh"
#include "host_mesh.hpp"
#include "kernel_timer.hpp"

#include <algorithm>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace hsb {
namespace {

constexpr double kInvFourPi = 0.07957747154594766788;
constexpr size_t kGatherColumnSmem = 200 * 1024;  // fused column gather: 3T complex FP64 entries

// Rule points (b0, b1, b2, w) of the four regular bins, in bin order
// (offsets 0, 6, 18, 34).
constexpr int kRulePoints = 98;
__constant__ double cRule[kRulePoints * 4];
__constant__ double cGauss20[40];

template <int NP> __device__ constexpr int ruleOffset() {
    return NP == 6 ? 0 : NP == 12 ? 6 : NP == 16 ? 18 : 34;
}

void cudaCheck(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

__device__ __forceinline__ void flagError(int *error, int code) { atomicExch(error, code); }

// First entry of bin `bin` of frequency f (exactly packed bins when offsets are given).
__device__ __forceinline__ size_t binStart(const uint64_t *offsets, size_t capacity, int f, int bin) {
    return offsets ? size_t(offsets[f * kBins + bin]) : (size_t(f) * kBins + bin) * capacity;
}

// Moment accumulators of one ordered pair: MG = sum g bt bs, MP = sum P bt bs,
// MQ = sum Q bt bs (3x3 complex each) where, for delta = x_test - y_trial,
// g = w exp(-ikr)/(4 pi r), P = g (1+ikr) (delta.n_trial)/r^2 (double layer),
// Q = -g (1+ikr) (delta.n_test)/r^2 (adjoint double layer).
struct PairMoments {
    double g[18], p[18], q[18];
};

// Record entry o (0..11 forward block (test t, trial s); 12..23 reverse
// block (test s, trial t)) of an unordered pair from its moments. Forward:
// A_ij = -MP_ij + i k (n_t.n_s) MG_ij + alpha G (curl_ti . curl_sj),
// b_i = sum_j (-MG_ij + (i/k) MQ_ij); reverse swaps P and Q and transposes.
template <class Real>
__device__ __forceinline__ void pairRecordValue(int o, const Real *MG, const Real *MP, const Real *MQ,
                                                const DPanel &t, const DPanel &s, double k, double invk,
                                                double &re, double &im) {
    const double nn = t.n[0] * s.n[0] + t.n[1] * s.n[1] + t.n[2] * s.n[2];
    const bool reverse = o >= 12;
    const int e = reverse ? o - 12 : o;
    const Real *X = reverse ? MQ : MP;  // double-layer moments of this direction
    const Real *Y = reverse ? MP : MQ;  // adjoint moments of this direction
    if (e < 9) {
        // forward element (i, j); reverse element (row j of s, col i of t) = moments (i, j)
        const int row = e / 3, col = e % 3;
        const int i = reverse ? col : row, j = reverse ? row : col;
        const int m = 2 * (3 * i + j);
        double gre = 0, gim = 0;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            gre += MG[2 * c];
            gim += MG[2 * c + 1];
        }
        const double curl = t.curl[3 * i] * s.curl[3 * j] + t.curl[3 * i + 1] * s.curl[3 * j + 1] +
                            t.curl[3 * i + 2] * s.curl[3 * j + 2];
        re = -X[m] - k * nn * MG[m + 1] + gim * curl * invk;
        im = -X[m + 1] + k * nn * MG[m] - gre * curl * invk;
    } else {
        const int a = e - 9;  // local row of this direction's test panel
        double sg_re = 0, sg_im = 0, sy_re = 0, sy_im = 0;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int m = reverse ? 2 * (3 * b + a) : 2 * (3 * a + b);
            sg_re += MG[m];
            sg_im += MG[m + 1];
            sy_re += Y[m];
            sy_im += Y[m + 1];
        }
        re = -sg_re - sy_im * invk;
        im = -sg_im + sy_re * invk;
    }
}

// ---------------------------------------------------------------------------
// Regular pairs: one unordered pair per NP threads, thread x owns test point x
// and sweeps the NP trial points, contracting trial bases on the fly.
// ---------------------------------------------------------------------------
// 128 threads: four CTAs (16 warps) per SM within the 128 registers a thread
// may use at that occupancy (the register file is split between the four SM
// sub-partitions, so 192-thread CTAs would stop at two per SM).
constexpr int kPlainThreads = 128;

template <int NP>
__global__ void __launch_bounds__(kPlainThreads, 4) regularPairsKernel(const DPanel *__restrict__ panels, uint32_t T,
                                                          const double *__restrict__ ks,
                                                          const uint2 *__restrict__ bins,
                                                          const uint32_t *__restrict__ binCounts, size_t binCapacity,
                                                          const uint64_t *__restrict__ binOffsets, int bin,
                                                          double *__restrict__ records, SlotMap map, int *error) {
    constexpr int PPC = kPlainThreads / NP;  // pairs per CTA; the last NP-group of threads may idle
    constexpr int RO = ruleOffset<NP>();
    __shared__ double sS[kPlainThreads][18];
    __shared__ double sM[PPC][54];
    // per trial point of each pair: its offset from the trial panel's first
    // vertex and that offset against the trial and test normals
    __shared__ double sY[kPlainThreads][5];
    const int f = blockIdx.y;
    const double k = ks[f], invk = 1.0 / k;
    const uint32_t count = binCounts[f * kBins + bin];
    const uint2 *list = bins + binStart(binOffsets, binCapacity, f, bin);
    double *rec = records + size_t(f) * map.planeSlots * kRecordDoubles;
    const int l = threadIdx.x / NP, x = threadIdx.x % NP;
    const double *yRow = &sY[l * NP][0];
    for (uint32_t base = blockIdx.x * PPC; base < count; base += gridDim.x * PPC) {
        const uint32_t p = base + l;
        const bool mine = l < PPC && p < count;
        uint2 pr = make_uint2(0, 0);
        if (mine) {
            // thread x places the pair's trial point x
            pr = list[p];
            const DPanel &S = panels[pr.y], &A = panels[pr.x];
            const double b1 = cRule[4 * (RO + x) + 1], b2 = cRule[4 * (RO + x) + 2];
            double e[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                e[c] = S.e1[c] * b1 + S.e2[c] * b2;
            sY[threadIdx.x][0] = e[0];
            sY[threadIdx.x][1] = e[1];
            sY[threadIdx.x][2] = e[2];
            sY[threadIdx.x][3] = e[0] * S.n[0] + e[1] * S.n[1] + e[2] * S.n[2];
            sY[threadIdx.x][4] = e[0] * A.n[0] + e[1] * A.n[1] + e[2] * A.n[2];
        }
        __syncthreads();
        if (mine) {
            const DPanel &A = panels[pr.x];
            const DPanel &S = panels[pr.y];
            const double bx1 = cRule[4 * (RO + x) + 1], bx2 = cRule[4 * (RO + x) + 2];
            // test point x relative to the trial panel's first vertex
            const double P0 = (A.v0[0] - S.v0[0]) + (A.e1[0] * bx1 + A.e2[0] * bx2);
            const double P1 = (A.v0[1] - S.v0[1]) + (A.e1[1] * bx1 + A.e2[1] * bx2);
            const double P2 = (A.v0[2] - S.v0[2]) + (A.e1[2] * bx1 + A.e2[2] * bx2);
            const double w0 = cRule[4 * (RO + x) + 3] * 4.0 * A.area * S.area * kInvFourPi;
            // (x - y).n_s = P.n_s - e(y).n_s, (x - y).n_t = P.n_t - e(y).n_t
            const double psP = P0 * S.n[0] + P1 * S.n[1] + P2 * S.n[2];
            const double qtP = P0 * A.n[0] + P1 * A.n[1] + P2 * A.n[2];
            double sp[6] = {0, 0, 0, 0, 0, 0}, sq[6] = {0, 0, 0, 0, 0, 0}, sg[6] = {0, 0, 0, 0, 0, 0};
            bool bad = false;
#pragma unroll(NP == 6 ? 6 : 4)
            for (int y = 0; y < NP; ++y) {
                const double b0 = cRule[4 * (RO + y)], b1 = cRule[4 * (RO + y) + 1], b2 = cRule[4 * (RO + y) + 2];
                const double wy = cRule[4 * (RO + y) + 3];
                const double *Y = yRow + 5 * y;
                const double dx = P0 - Y[0], dy = P1 - Y[1], dz = P2 - Y[2];
                const double r2 = dx * dx + dy * dy + dz * dz;
                bad |= !(r2 > 0) || !isfinite(r2);
                const double rinv = rsqrt(r2);
                const double r = r2 * rinv, kr = k * r;
                double sn, cs;
                sincos(kr, &sn, &cs);
                const double sc = w0 * wy * rinv;
                const double gr = cs * sc, gi = -sn * sc;
                const double rr = gr - gi * kr, ri = gi + gr * kr;
                const double rinv2 = rinv * rinv;
                const double ps = (psP - Y[3]) * rinv2;
                const double qt = (Y[4] - qtP) * rinv2;
                const double Pr = rr * ps, Pi = ri * ps, Qr = rr * qt, Qi = ri * qt;
                const double bb[3] = {b0, b1, b2};
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    sp[2 * j] += Pr * bb[j];
                    sp[2 * j + 1] += Pi * bb[j];
                    sq[2 * j] += Qr * bb[j];
                    sq[2 * j + 1] += Qi * bb[j];
                    sg[2 * j] += gr * bb[j];
                    sg[2 * j + 1] += gi * bb[j];
                }
            }
            if (bad)
                flagError(error, kErrDistance);
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                sS[threadIdx.x][c] = sg[c];
                sS[threadIdx.x][6 + c] = sp[c];
                sS[threadIdx.x][12 + c] = sq[c];
            }
        }
        __syncthreads();
        // Test-side contraction: M[kind][i][j] = sum_x bt_i(x) S_kind,j(x).
        for (int item = threadIdx.x; item < PPC * 27; item += kPlainThreads) {
            const int pl = item / 27, e = item % 27, kind = e / 9, i = (e % 9) / 3, j = e % 3;
            if (base + pl >= count)
                continue;
            double re = 0, im = 0;
            for (int xx = 0; xx < NP; ++xx) {
                const int th = pl * NP + xx;
                const double bt = cRule[4 * (RO + xx) + i];
                re += bt * sS[th][kind * 6 + 2 * j];
                im += bt * sS[th][kind * 6 + 2 * j + 1];
            }
            sM[pl][kind * 18 + 2 * (3 * i + j)] = re;
            sM[pl][kind * 18 + 2 * (3 * i + j) + 1] = im;
        }
        __syncthreads();
        for (int item = threadIdx.x; item < PPC * 24; item += kPlainThreads) {
            const int pl = item / 24, o = item % 24;
            if (base + pl >= count)
                continue;
            const uint2 pr = list[base + pl];
            double re, im;
            pairRecordValue(o, &sM[pl][0], &sM[pl][18], &sM[pl][36], panels[pr.x], panels[pr.y], k, invk, re, im);
            const size_t slot = o < 12 ? mapSlot(map, T, pr.x, pr.y) : mapSlot(map, T, pr.y, pr.x);
            const int e = o < 12 ? o : o - 12;
            if (!isfinite(re) || !isfinite(im))
                flagError(error, kErrNonFinite);
            if (slot == kNoSlot) {
                flagError(error, kErrEscapedPlan);
                continue;
            }
            double *dst = rec + mapOffset(map.planeSlots, slot, e);
            dst[0] = re;
            dst[1] = im;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Mixed form: the Green-kernel sample with FP32 arithmetic. The displacement
// and the phase k*r stay in FP64 (the phase reduced modulo 2 pi before the
// FP32 sine/cosine), because rounding r or k*r to FP32 leaves an
// O(eps_fp32 * k*r) phase error that no quadrature refinement removes
// (panel_integrals.cuh:91-142 keeps FP64 for k*r > 1 for the same reason).
// Returns g, P and Q (see PairMoments) as (re, im) pairs.
// ---------------------------------------------------------------------------
constexpr double kTwoPiHi = 6.283185307179586, kTwoPiLo = 2.4492935982947064e-16, kInvTwoPi = 0.15915494309189535;

__device__ __forceinline__ void mixedValues(double dx, double dy, double dz, float w, double k, const float *ns,
                                            const float *nt, float (&val)[6], bool &bad) {
    const float fx = float(dx), fy = float(dy), fz = float(dz);
    const float r2 = fx * fx + fy * fy + fz * fz;
    bad |= !(r2 > 0.f) || !isfinite(r2);
    const float rinv = rsqrtf(r2);
    // r in FP64 from one Newton step on the FP32 reciprocal root
    const double r2d = dx * dx + dy * dy + dz * dz;
    double y = double(rinv);
    y = y * (1.5 - 0.5 * r2d * y * y);
    const double ph = k * (r2d * y);
    const double turns = (ph * kInvTwoPi + 6755399441055744.0) - 6755399441055744.0;  // round to nearest
    const double th = fma(-turns, kTwoPiLo, fma(-turns, kTwoPiHi, ph));
    float sn, cs;
    __sincosf(float(th), &sn, &cs);  // th in [-pi, pi]: hardware sin/cos, absolute error about 4e-7
    const float kr = float(ph);
    const float sc = w * rinv;
    const float gr = cs * sc, gi = -sn * sc;
    const float rr = gr - gi * kr, ri = gi + gr * kr;
    const float rinv2 = rinv * rinv;
    const float ps = (fx * ns[0] + fy * ns[1] + fz * ns[2]) * rinv2;
    const float qt = -(fx * nt[0] + fy * nt[1] + fz * nt[2]) * rinv2;
    val[0] = gr;
    val[1] = gi;
    val[2] = rr * ps;
    val[3] = ri * ps;
    val[4] = rr * qt;
    val[5] = ri * qt;
}

// Regular pairs in the mixed form: one unordered pair per thread, NP x NP
// samples, trial bases contracted per test point, no FP64 per sample.
//
// Phase. Rounding r or k*r to FP32 leaves an O(eps_fp32 * k*r) phase error
// that no quadrature refinement removes (panel_integrals.cuh:91-142 keeps
// FP64 for k*r > 1 for that reason). Here the pair's centre distance r0 and
// its phase k*r0 are FP64 (reduced modulo 2 pi once per pair) and each sample
// adds k*(r - r0) = k*Delta/(r + r0) with Delta = r^2 - r0^2. With c the
// centre displacement, p the test point's offset and e(y) = E1 b1 + E2 b2 the
// trial point's offset (trial edges E1, E2), Delta = (2c + p).p
// - 2 (c + p).e(y) + |e(y)|^2, a quadratic in the trial barycentrics whose
// coefficients are formed once per pair and test point; its terms are
// O(r0 * h), so the FP32 phase error is O(eps * k * h), independent of k*r0.
// r^2 = r0^2 + Delta. sin/cos of the phase reduced to [-pi, pi] use the
// hardware approximation (absolute error about 4e-7).
// Amplitude. FP32 throughout (relative error ~eps_fp32, as for the
// reference's mixed sample); the double-layer projection (x - y).n_trial is
// constant over the trial panel and the adjoint one affine in b1, b2.
// Rule table per point: b0, b1, b2, w, b1^2, 2 b1 b2, b2^2, 0.
__constant__ float cRuleF[kRulePoints * 8];

// Both records of an unordered regular pair (forward: test A, trial S;
// reverse: test S, trial A) from its FP32 moments (the layout and formulas of
// pairRecordValue), stored straight into the record planes. ps = plane stride.
__device__ __forceinline__ void storePairRecords(const float (&M)[54], const MixedPanel *__restrict__ pa,
                                                 const MixedPanel *__restrict__ pb, float k, float invk, float *fwd,
                                                 float *rev, size_t ps, bool &nonFinite) {
    const float *MG = M, *MP = M + 18, *MQ = M + 36;
    const float4 na = pa->n, nb = pb->n;
    const float knn = k * (na.x * nb.x + na.y * nb.y + na.z * nb.z);
    float gre = 0.f, gim = 0.f;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        gre += MG[2 * c];
        gim += MG[2 * c + 1];
    }
    gre *= invk;
    gim *= invk;
    const float4 ca[3] = {pa->curl[0], pa->curl[1], pa->curl[2]}, cs[3] = {pb->curl[0], pb->curl[1], pb->curl[2]};
    float check = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i)      // A's local vertex
#pragma unroll
        for (int j = 0; j < 3; ++j) {  // S's local vertex
            const float curl = ca[i].x * cs[j].x + ca[i].y * cs[j].y + ca[i].z * cs[j].z;
            const int m = 2 * (3 * i + j);
            // forward element (row i, col j); reverse element (row j, col i)
            const float fr = fmaf(gim, curl, fmaf(-knn, MG[m + 1], -MP[m]));
            const float fi = fmaf(-gre, curl, fmaf(knn, MG[m], -MP[m + 1]));
            const float rr = fmaf(gim, curl, fmaf(-knn, MG[m + 1], -MQ[m]));
            const float ri = fmaf(-gre, curl, fmaf(knn, MG[m], -MQ[m + 1]));
            *reinterpret_cast<float2 *>(fwd + j * ps + 2 * i) = make_float2(fr, fi);
            *reinterpret_cast<float2 *>(rev + i * ps + 2 * j) = make_float2(rr, ri);
            check += fabsf(fr) + fabsf(fi) + fabsf(rr) + fabsf(ri);
        }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // forward rhs row a (A's vertex): sum over S's vertices; reverse rhs row a (S's vertex): over A's
        float fgr = 0.f, fgi = 0.f, fyr = 0.f, fyi = 0.f, rgr = 0.f, rgi = 0.f, ryr = 0.f, ryi = 0.f;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int mf = 2 * (3 * a + b), mr = 2 * (3 * b + a);
            fgr += MG[mf];
            fgi += MG[mf + 1];
            fyr += MQ[mf];
            fyi += MQ[mf + 1];
            rgr += MG[mr];
            rgi += MG[mr + 1];
            ryr += MP[mr];
            ryi += MP[mr + 1];
        }
        const float2 fv = make_float2(fmaf(-fyi, invk, -fgr), fmaf(fyr, invk, -fgi));
        const float2 rv = make_float2(fmaf(-ryi, invk, -rgr), fmaf(ryr, invk, -rgi));
        *reinterpret_cast<float2 *>(fwd + 3 * ps + 2 * a) = fv;
        *reinterpret_cast<float2 *>(rev + 3 * ps + 2 * a) = rv;
        check += fabsf(fv.x) + fabsf(fv.y) + fabsf(rv.x) + fabsf(rv.y);
    }
    nonFinite |= !isfinite(check);
}

template <int NP>
__global__ void __launch_bounds__(128, 4) regularMixedKernel(const MixedPanel *__restrict__ mpanels,
                                                             const Bounds *__restrict__ bounds, uint32_t T,
                                                             const double *__restrict__ ks,
                                                             const uint2 *__restrict__ bins,
                                                             const uint32_t *__restrict__ binCounts, size_t binCapacity,
                                                             const uint64_t *__restrict__ binOffsets, int bin,
                                                             float *__restrict__ records, int *error) {
    constexpr int RO = ruleOffset<NP>();
    constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52: adding and subtracting rounds to an integer
    constexpr double kTwoPi = 6.283185307179586, kTwoPiLo = 2.4492935982947064e-16, kInvTwoPi = 0.15915494309189535;
    constexpr float kRoundF = 12582912.f;  // 1.5 * 2^23, the same for FP32
    constexpr float kTwoPiHiF = 6.28318548f, kTwoPiLoF = -1.74845553e-7f, kInvTwoPiF = 0.159154943f;
    const int f = blockIdx.y;
    const double k = ks[f];
    const float kf = float(k), invkf = float(1.0 / k);
    const uint32_t count = binCounts[f * kBins + bin];
    const uint2 *list = bins + binStart(binOffsets, binCapacity, f, bin);
    float *rec = records + size_t(f) * T * T * kRecordDoubles;
    const size_t planeStride = size_t(T) * T * 6;
    bool bad = false, nonFinite = false;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
        const uint2 pr = list[p];
        const MixedPanel &A = mpanels[pr.x], &S = mpanels[pr.y];
        const V3 ca = bounds[pr.x].center, cb = bounds[pr.y].center;
        // centre displacement, distance and phase (reduced to [-pi, pi]) in FP64
        const double cx = ca.x - cb.x, cy = ca.y - cb.y, cz = ca.z - cb.z;
        const double r0sqd = cx * cx + cy * cy + cz * cz, r0 = sqrt(r0sqd);
        const double ph0 = k * r0;
        const double turns = (ph0 * kInvTwoPi + kRound) - kRound;
        const float theta0 = float(fma(-turns, kTwoPiLo, fma(-turns, kTwoPi, ph0)));
        const float c[3] = {float(cx), float(cy), float(cz)};
        const float r0f = float(r0), r0sq = float(r0sqd);
        // test first vertex minus trial first vertex, about the centres
        const float4 aOff = A.offset, sOff = S.offset, aE1 = A.e1, aE2 = A.e2, sE1 = S.e1, sE2 = S.e2, aN = A.n,
                     sN = S.n;
        const float o0[3] = {aOff.x - sOff.x, aOff.y - sOff.y, aOff.z - sOff.z};
        const float ae1[3] = {aE1.x, aE1.y, aE1.z}, ae2[3] = {aE2.x, aE2.y, aE2.z};
        const float se1[3] = {sE1.x, sE1.y, sE1.z}, se2[3] = {sE2.x, sE2.y, sE2.z};
        const float ns[3] = {sN.x, sN.y, sN.z}, nt[3] = {aN.x, aN.y, aN.z};
        // |e(y)|^2 coefficients and trial edges against the test normal
        const float E11 = sE1.w, E12 = sN.w, E22 = sE2.w;
        const float t1 = se1[0] * nt[0] + se1[1] * nt[1] + se1[2] * nt[2];
        const float t2 = se2[0] * nt[0] + se2[1] * nt[1] + se2[2] * nt[2];
        const float w4 = 4.f * aOff.w * sOff.w * float(kInvFourPi);
        float M[54];
#pragma unroll
        for (int i = 0; i < 54; ++i)
            M[i] = 0.f;
        float r2min = 3.4e38f;
#pragma unroll 1
        for (int x = 0; x < NP; ++x) {
            const float bx1 = cRuleF[8 * (RO + x) + 1], bx2 = cRuleF[8 * (RO + x) + 2];
            // P: test point minus the trial panel's first vertex, about the centres; CP = c + P
            float P[3], CP[3], C2P[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                P[i] = fmaf(ae1[i], bx1, fmaf(ae2[i], bx2, o0[i]));
                CP[i] = c[i] + P[i];
                C2P[i] = c[i] + CP[i];
            }
            const float psx = CP[0] * ns[0] + CP[1] * ns[1] + CP[2] * ns[2];
            const float qtx = -(CP[0] * nt[0] + CP[1] * nt[1] + CP[2] * nt[2]);
            // Delta = Ax + a1 b1 + a2 b2 + E11 b1^2 + 2 E12 b1 b2 + E22 b2^2
            const float Ax = C2P[0] * P[0] + C2P[1] * P[1] + C2P[2] * P[2];
            const float a1 = -2.f * (CP[0] * se1[0] + CP[1] * se1[1] + CP[2] * se1[2]);
            const float a2 = -2.f * (CP[0] * se2[0] + CP[1] * se2[1] + CP[2] * se2[2]);
            const float wx = cRuleF[8 * (RO + x) + 3] * w4;
            float G[6], U[6], Q[6];
#pragma unroll
            for (int i = 0; i < 6; ++i)
                G[i] = U[i] = Q[i] = 0.f;
#pragma unroll(NP <= 16 ? NP : 4)
            for (int y = 0; y < NP; ++y) {
                const float *ry = cRuleF + 8 * (RO + y);
                const float b0 = ry[0], b1 = ry[1], b2 = ry[2];
                const float delta = fmaf(E22, ry[6], fmaf(E12, ry[5], fmaf(E11, ry[4], fmaf(a2, b2, fmaf(a1, b1, Ax)))));
                const float r2 = r0sq + delta;
                r2min = fminf(r2min, r2);
                const float rinv = rsqrtf(r2);
                const float r = r2 * rinv;
                const float theta = fmaf(kf, __fdividef(delta, r + r0f), theta0);
                const float qn = fmaf(theta, kInvTwoPiF, kRoundF) - kRoundF;
                float sn, cs;
                __sincosf(fmaf(-qn, kTwoPiLoF, fmaf(-qn, kTwoPiHiF, theta)), &sn, &cs);
                const float kr = kf * r;
                const float sc = (wx * ry[3]) * rinv;
                const float gr = cs * sc, gi = -sn * sc;
                const float rr = fmaf(-gi, kr, gr), ri = fmaf(gr, kr, gi);
                const float rinv2 = rinv * rinv;
                const float ur = rr * rinv2, ui = ri * rinv2;
                const float qt = fmaf(t1, b1, fmaf(t2, b2, qtx));
                const float qr = ur * qt, qi = ui * qt;
                const float bs[3] = {b0, b1, b2};
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    G[2 * j] = fmaf(gr, bs[j], G[2 * j]);
                    G[2 * j + 1] = fmaf(gi, bs[j], G[2 * j + 1]);
                    U[2 * j] = fmaf(ur, bs[j], U[2 * j]);
                    U[2 * j + 1] = fmaf(ui, bs[j], U[2 * j + 1]);
                    Q[2 * j] = fmaf(qr, bs[j], Q[2 * j]);
                    Q[2 * j + 1] = fmaf(qi, bs[j], Q[2 * j + 1]);
                }
            }
            const float bt[3] = {cRuleF[8 * (RO + x)], bx1, bx2};
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float bp = bt[i] * psx;
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    M[6 * i + j] = fmaf(bt[i], G[j], M[6 * i + j]);
                    M[18 + 6 * i + j] = fmaf(bp, U[j], M[18 + 6 * i + j]);
                    M[36 + 6 * i + j] = fmaf(bt[i], Q[j], M[36 + 6 * i + j]);
                }
            }
        }
        bad |= !(r2min > 0.f);
        storePairRecords(M, &A, &S, kf, invkf, rec + (size_t(pr.y) * T + pr.x) * 6,
                         rec + (size_t(pr.x) * T + pr.y) * 6, planeStride, nonFinite);
    }
    if (bad)
        flagError(error, kErrDistance);
    if (nonFinite)
        flagError(error, kErrNonFinite);
}

// Number of 8 x 4 pair tiles before block q of trial panels j = 4q .. 4q + 3
// (block q holds q / 2 + 1 tiles of 8 test panels i = 8p .. 8p + 7, i < j).
__host__ __device__ inline uint64_t tilesBefore(uint64_t q) {
    const uint64_t m = q / 2;
    return q % 2 ? (m + 1) * (m + 1) : m * (m + 1);
}

// Sorts unordered regular pairs of each frequency into rule bins. Pairs are
// enumerated in tiles of 8 test x 4 trial panels, one tile per warp, so a
// warp's pairs (kept in lane order by the warp-aggregated appends) write both
// orientations of their records in runs of whole sectors: 8 consecutive slots
// per trial panel forward, 4 per test panel in reverse. A thread decodes its
// pair, reads the pair code and both panels' bounds once, then classifies it
// at every frequency of the batch.
__global__ void classifyPairsKernel(const uint8_t *__restrict__ pairCode, const Bounds *__restrict__ bounds,
                                    uint32_t T, const double *__restrict__ ks, uint32_t B, double tol,
                                    uint32_t minDegree, uint2 *bins, uint32_t *binCounts, size_t binCapacity,
                                    const uint64_t *binOffsets, bool countOnly, int *error) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t threads = 32 * tilesBefore((uint64_t(T) + 3) / 4);
    for (uint64_t base = uint64_t(blockIdx.x) * blockDim.x; base < threads; base += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t tile = (base + threadIdx.x) / 32;  // the same for the whole warp
        uint32_t i = 0, j = 0;
        uint8_t code = kPairTouching;  // no bin
        Bounds bi{}, bj{};
        if (tile < threads / 32) {
            uint64_t m = uint64_t((sqrt(4.0 * double(tile) + 1.0) - 1.0) * 0.5);
            while (m * (m + 1) > tile)
                --m;
            while ((m + 1) * (m + 2) <= tile)
                ++m;
            const uint64_t q = tile >= (m + 1) * (m + 1) ? 2 * m + 1 : 2 * m;
            const uint64_t p = tile - tilesBefore(q);
            i = uint32_t(8 * p + (lane & 7));
            j = uint32_t(4 * q + (lane >> 3));
        }
        if (j < T && i < j) {
            code = pairCode[uint64_t(j) * (j - 1) / 2 + i];
            if (code == kPairRegular) {
                bi = bounds[i];
                bj = bounds[j];
            }
        }
        for (uint32_t f = 0; f < B; ++f) {
            int bin = -1;
            if (code == kPairWhole8)
                bin = 2;
            else if (code == kPairWhole14)
                bin = 3;
            else if (code == kPairRegular) {
                const unsigned d = qualifiedDegree(bi, bj, ks[f], tol, minDegree);
                if (d == 4)
                    bin = 0;
                else if (d == 6)
                    bin = 1;
                else if (d == 8)
                    bin = 2;
                else
                    flagError(error, kErrEscapedPlan);
            }
#pragma unroll
            for (int b = 0; b < kBins; ++b) {
                const unsigned mask = __ballot_sync(0xffffffffu, bin == b);
                if (!mask)
                    continue;
                uint32_t start = 0;
                if (lane == unsigned(__ffs(mask) - 1))
                    start = atomicAdd(&binCounts[f * kBins + b], uint32_t(__popc(mask)));
                start = __shfl_sync(0xffffffffu, start, __ffs(mask) - 1);
                if (bin == b && !countOnly)
                    bins[binStart(binOffsets, binCapacity, int(f), b) + start + __popc(mask & ((1u << lane) - 1))] =
                        make_uint2(i, j);
            }
        }
    }
}

// Exclusive scan of the bin counts of all frequencies into bin offsets (a few
// dozen entries, one thread); the counts start again from zero for the fill pass.
__global__ void binOffsetsKernel(uint32_t *binCounts, uint64_t *binOffsets, uint32_t n) {
    uint64_t sum = 0;
    for (uint32_t q = 0; q < n; ++q) {
        binOffsets[q] = sum;
        sum += binCounts[q];
        binCounts[q] = 0;
    }
}

// The classification of classifyPairsKernel for a list of unordered pairs
// (i < j): the fast-multipole near field, whose records are only those of the
// near support pairs. Appends warp-aggregated like the full enumeration.
__global__ void classifyListKernel(const uint2 *__restrict__ list, uint64_t count, const uint8_t *__restrict__ pairCode,
                                   const Bounds *__restrict__ bounds, const double *__restrict__ ks, uint32_t B,
                                   double tol, uint32_t minDegree, uint2 *bins, uint32_t *binCounts,
                                   size_t binCapacity, int *error) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t padded = (count + 31) / 32 * 32;
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < padded; q += uint64_t(gridDim.x) * blockDim.x) {
        uint8_t code = kPairTouching;
        uint2 pr = make_uint2(0, 0);
        Bounds bi{}, bj{};
        if (q < count) {
            pr = list[q];
            code = pairCode[uint64_t(pr.y) * (pr.y - 1) / 2 + pr.x];
            if (code == kPairRegular) {
                bi = bounds[pr.x];
                bj = bounds[pr.y];
            }
        }
        for (uint32_t f = 0; f < B; ++f) {
            int bin = -1;
            if (code == kPairWhole8)
                bin = 2;
            else if (code == kPairWhole14)
                bin = 3;
            else if (code == kPairRegular) {
                const unsigned d = qualifiedDegree(bi, bj, ks[f], tol, minDegree);
                bin = d == 4 ? 0 : d == 6 ? 1 : d == 8 ? 2 : -1;
                if (bin < 0)
                    flagError(error, kErrEscapedPlan);
            }
#pragma unroll
            for (int b = 0; b < kBins; ++b) {
                const unsigned mask = __ballot_sync(0xffffffffu, bin == b);
                if (!mask)
                    continue;
                uint32_t start = 0;
                if (lane == unsigned(__ffs(mask) - 1))
                    start = atomicAdd(&binCounts[f * kBins + b], uint32_t(__popc(mask)));
                start = __shfl_sync(0xffffffffu, start, __ffs(mask) - 1);
                if (bin == b)
                    bins[(size_t(f) * kBins + b) * binCapacity + start + __popc(mask & ((1u << lane) - 1))] = pr;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Touching pairs (cuda_solver.cu:382-429): one CTA per ordered job, threads
// over (sector, u, v, w), the radial Gauss variable factored out because
// every sector map is linear in r about the shared vertex.
// ---------------------------------------------------------------------------
struct Moments13 {
    double m[18], b[6], g[2];
};

__device__ __forceinline__ void sampleFp64(Moments13 &acc, const DPanel &t, const DPanel &s, double dx, double dy,
                                           double dz, const double *bt, const double *bs, double w, double k,
                                           double invk, bool coincident, bool &bad) {
    const double r2 = dx * dx + dy * dy + dz * dz;
    bad |= !(r2 > 0) || !isfinite(r2);
    const double rinv = rsqrt(r2);
    const double r = r2 * rinv, kr = k * r;
    double sn, cs;
    sincos(kr, &sn, &cs);
    const double sc = w * rinv;
    const double gr = cs * sc, gi = -sn * sc;
    acc.g[0] += gr;
    acc.g[1] += gi;
    const double rr = gr - gi * kr, ri = gi + gr * kr;
    const double rinv2 = rinv * rinv;
    const double ps = coincident ? 0.0 : (dx * s.n[0] + dy * s.n[1] + dz * s.n[2]) * rinv2;
    const double qt = coincident ? 0.0 : -(dx * t.n[0] + dy * t.n[1] + dz * t.n[2]) * rinv2;
    const double nn = t.n[0] * s.n[0] + t.n[1] * s.n[1] + t.n[2] * s.n[2];
    const double ar = -rr * ps - k * nn * gi, ai = -ri * ps + k * nn * gr;
    const double br = -gr - ri * qt * invk, bi = -gi + rr * qt * invk;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        acc.b[2 * i] += br * bt[i];
        acc.b[2 * i + 1] += bi * bt[i];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double bij = bt[i] * bs[j];
            acc.m[2 * (3 * i + j)] += ar * bij;
            acc.m[2 * (3 * i + j) + 1] += ai * bij;
        }
    }
}

// Block sums of N values, left in smem[0][0..N). Within a warp a
// reduce-scatter per group of 32 values: after the pass at distance h a lane
// keeps the h partial sums of the half its lane bit h selects, so after five
// passes (31 shuffles per group instead of 32 x 5) lane l holds the sum of
// value l of the group. The warps' sums are then added in warp order by the
// thread that owns each value.
template <int N>
__device__ __forceinline__ void blockReduce(double (&v)[N], double (*smem)[N]) {
    constexpr int G = (N + 31) / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int gi = 0; gi < G; ++gi) {
        double x[32];
#pragma unroll
        for (int c = 0; c < 32; ++c)
            x[c] = 32 * gi + c < N ? v[32 * gi + c] : 0.0;
#pragma unroll
        for (int h = 16; h >= 1; h >>= 1) {
            const bool upper = (lane & h) != 0;
#pragma unroll
            for (int c = 0; c < h; ++c) {
                const double send = upper ? x[c] : x[c + h], keep = upper ? x[c + h] : x[c];
                x[c] = keep + __shfl_xor_sync(0xffffffffu, send, h);
            }
        }
        if (32 * gi + lane < N)
            smem[warp][32 * gi + lane] = x[0];
    }
    __syncthreads();
    const int warps = blockDim.x >> 5;
    for (int c = threadIdx.x; c < N; c += blockDim.x) {
        double sum = smem[0][c];
        for (int w = 1; w < warps; ++w)
            sum += smem[w][c];
        smem[0][c] = sum;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(128) singularKernel(const DPanel *__restrict__ panels, uint32_t T,
                                                      const TouchingJob *__restrict__ jobs,
                                                      const double *__restrict__ ks,
                                                      const double *__restrict__ gauss, uint32_t order,
                                                      double *__restrict__ records, SlotMap map, int *error) {
    __shared__ double red[4][26];
    const TouchingJob job = jobs[blockIdx.x];
    const int f = blockIdx.y;
    const double k = ks[f], invk = 1.0 / k;
    const DPanel &t = panels[job.test];
    const DPanel &s = panels[job.trial];
    const bool coincident = job.topology == kCoincident;
    Permutation perm;
    perm.topology = job.topology;
    for (int i = 0; i < 3; ++i) {
        perm.test[i] = job.permTest[i];
        perm.trial[i] = job.permTrial[i];
    }
    const double w4 = 4.0 * t.area * s.area * kInvFourPi;
    const uint32_t per = order * order * order;
    const uint32_t count = sectorCount(job.topology) * per;
    Moments13 acc;
#pragma unroll
    for (int c = 0; c < 18; ++c)
        acc.m[c] = 0;
#pragma unroll
    for (int c = 0; c < 6; ++c)
        acc.b[c] = 0;
    acc.g[0] = acc.g[1] = 0;
    bool bad = false;
    for (uint32_t idx = threadIdx.x; idx < count; idx += blockDim.x) {
        uint32_t tuple = idx % per;
        const uint32_t w = tuple % order;
        tuple /= order;
        const uint32_t v = tuple % order;
        const uint32_t u = tuple / order;
        PairPoint p = sauterSchwab(job.topology, idx / per, 1.0, gauss[2 * u], gauss[2 * v], gauss[2 * w]);
        p.w *= gauss[2 * u + 1] * gauss[2 * v + 1] * gauss[2 * w + 1];
        p = permutePoint(p, perm);
        const double lx = (t.v0[0] - s.v0[0]) + ((t.e1[0] * p.t[1] + t.e2[0] * p.t[2]) - (s.e1[0] * p.s[1] + s.e2[0] * p.s[2]));
        const double ly = (t.v0[1] - s.v0[1]) + ((t.e1[1] * p.t[1] + t.e2[1] * p.t[2]) - (s.e1[1] * p.s[1] + s.e2[1] * p.s[2]));
        const double lz = (t.v0[2] - s.v0[2]) + ((t.e1[2] * p.t[1] + t.e2[2] * p.t[2]) - (s.e1[2] * p.s[1] + s.e2[2] * p.s[2]));
        for (uint32_t ri = 0; ri < order; ++ri) {
            const double r = gauss[2 * ri];
            double bt[3], bs[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                bt[i] = r * p.t[i];
                bs[i] = r * p.s[i];
            }
            bt[perm.test[0]] += 1 - r;
            bs[perm.trial[0]] += 1 - r;
            sampleFp64(acc, t, s, lx * r, ly * r, lz * r, bt, bs, p.w * r * r * r * gauss[2 * ri + 1] * w4, k, invk,
                       coincident, bad);
        }
    }
    if (bad)
        flagError(error, kErrDistance);
    double v[26];
#pragma unroll
    for (int c = 0; c < 18; ++c)
        v[c] = acc.m[c];
#pragma unroll
    for (int c = 0; c < 6; ++c)
        v[18 + c] = acc.b[c];
    v[24] = acc.g[0];
    v[25] = acc.g[1];
    blockReduce<26>(v, red);
    if (threadIdx.x < 12) {
        const int o = threadIdx.x;
        double re, im;
        if (o < 9) {
            const int i = o / 3, j = o % 3;
            const double curl = t.curl[3 * i] * s.curl[3 * j] + t.curl[3 * i + 1] * s.curl[3 * j + 1] +
                                t.curl[3 * i + 2] * s.curl[3 * j + 2];
            re = red[0][2 * o] + red[0][25] * curl * invk;
            im = red[0][2 * o + 1] - red[0][24] * curl * invk;
        } else {
            re = red[0][18 + 2 * (o - 9)];
            im = red[0][18 + 2 * (o - 9) + 1] + (coincident ? t.area / (6.0 * k) : 0.0);
        }
        if (!isfinite(re) || !isfinite(im))
            flagError(error, kErrNonFinite);
        const size_t slot = mapSlot(map, T, job.test, job.trial);
        if (slot == kNoSlot)
            flagError(error, kErrEscapedPlan);
        else {
            double *dst = records + size_t(f) * map.planeSlots * kRecordDoubles + mapOffset(map.planeSlots, slot, o);
            dst[0] = re;
            dst[1] = im;
        }
    }
}

// Mixed form of the touching pairs: one warp per ordered job, FP32 samples.
// The sector maps do not depend on the job, so the (sector, u, v, w) tuples
// come from a table built once per singular order in FP64
// (buildSingularTable): canonical-order barycentrics at radius 1, the
// weight, and coefficients (a1, a2, b1, b2) of the displacement
// l = A1 a1 + A2 a2 - B1 b1 - B2 b2 over the canonical edges A (test) and B
// (trial) from the first shared vertex. For shared edges and coincident
// panels the shared edges are merged and their coefficients are differences
// formed in FP64, so l keeps FP32 relative accuracy where the two points
// nearly meet. Touching pairs have k*r <= 2 k h, so the FP32 phase needs no
// FP64 help; it is reduced to [-pi, pi] for the hardware sin/cos (absolute
// error about 4e-7). Moments accumulate in canonical order and are permuted
// back to local order once per job.
__global__ void __launch_bounds__(128, 6) singularMixedKernel(const DPanel *__restrict__ panels, uint32_t T,
                                                           const TouchingJob *__restrict__ jobs, uint32_t jobCount,
                                                           const double *__restrict__ ks,
                                                           const float4 *__restrict__ table, uint32_t order,
                                                           float *__restrict__ records, int *error) {
    constexpr float kRoundF = 12582912.f, kTwoPiHiF = 6.28318548f, kTwoPiLoF = -1.74845553e-7f,
                    kInvTwoPiF = 0.159154943f;
    const uint32_t jobIndex = blockIdx.x * 4 + (threadIdx.x >> 5);
    const unsigned lane = threadIdx.x & 31;
    if (jobIndex >= jobCount)
        return;  // warp-uniform
    const TouchingJob job = jobs[jobIndex];
    const int f = blockIdx.y;
    const double k = ks[f], invk = 1.0 / k;
    const float kf = float(k), invkf = float(invk);
    const DPanel &t = panels[job.test];
    const DPanel &s = panels[job.trial];
    const bool coincident = job.topology == kCoincident;
    // canonical edges from the first shared vertex, in FP64 then rounded
    float A1[3], A2[3], B1[3], B2[3];
    {
        const int ta = job.permTest[0], tb = job.permTest[1], tc = job.permTest[2];
        const int sa = job.permTrial[0], sb = job.permTrial[1], sc = job.permTrial[2];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double te[3] = {0.0, t.e1[i], t.e2[i]}, se[3] = {0.0, s.e1[i], s.e2[i]};
            A1[i] = float(te[tb] - te[ta]);
            A2[i] = float(te[tc] - te[ta]);
            B1[i] = float(se[sb] - se[sa]);
            B2[i] = float(se[sc] - se[sa]);
        }
    }
    const float w4 = float(4.0 * t.area * s.area * kInvFourPi);
    const float tn[3] = {float(t.n[0]), float(t.n[1]), float(t.n[2])};
    const float sn3[3] = {float(s.n[0]), float(s.n[1]), float(s.n[2])};
    const float knn = kf * float(t.n[0] * s.n[0] + t.n[1] * s.n[1] + t.n[2] * s.n[2]);
    const uint32_t per = order * order * order;
    const uint32_t count = sectorCount(job.topology) * per;
    const uint32_t base = job.topology == kSharedVertex ? 0u : job.topology == kSharedEdge ? 2u * per : 7u * per;
    const float4 *tuples = table + 3 * size_t(base);
    const float4 *radial = table + 3 * size_t(13 * per);
    float m[18], b[6], g[2] = {0.f, 0.f};
#pragma unroll
    for (int c = 0; c < 18; ++c)
        m[c] = 0.f;
#pragma unroll
    for (int c = 0; c < 6; ++c)
        b[c] = 0.f;
    bool bad = false;
    for (uint32_t idx = lane; idx < count; idx += 32) {
        const float4 q0 = tuples[3 * idx], q1 = tuples[3 * idx + 1], q2 = tuples[3 * idx + 2];
        const float pt[3] = {q0.x, q0.y, q0.z}, pq[3] = {q0.w, q1.x, q1.y};
        float l[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
            l[i] = fmaf(A1[i], q1.z, fmaf(A2[i], q1.w, fmaf(-B1[i], q2.x, -B2[i] * q2.y)));
        const float ps1 = coincident ? 0.f : l[0] * sn3[0] + l[1] * sn3[1] + l[2] * sn3[2];
        const float qt1 = coincident ? 0.f : -(l[0] * tn[0] + l[1] * tn[1] + l[2] * tn[2]);
        const float lr2 = l[0] * l[0] + l[1] * l[1] + l[2] * l[2];
        bad |= !(lr2 > 0.f) || !isfinite(lr2);
        const float linv = rsqrtf(lr2), llen = lr2 * linv;
        const float pw = q2.z * w4;
#pragma unroll 4
        for (uint32_t ri = 0; ri < order; ++ri) {
            const float4 rad = radial[ri];  // (r, r^3 w_r, 1/r, 1 - r)
            const float r = rad.x;
            // sample at radial fraction r: displacement r*l, distance r*|l|
            const float rinv = linv * rad.z, kr = kf * (llen * r);
            // phase reduced to [-pi, pi], hardware sin/cos (absolute error about 4e-7)
            const float qn = fmaf(kr, kInvTwoPiF, kRoundF) - kRoundF;
            float sn, cs;
            __sincosf(fmaf(-qn, kTwoPiLoF, fmaf(-qn, kTwoPiHiF, kr)), &sn, &cs);
            const float sc = pw * rad.y * rinv;
            const float gr = cs * sc, gi = -sn * sc;
            g[0] += gr;
            g[1] += gi;
            const float rr = fmaf(-gi, kr, gr), ri2 = fmaf(gr, kr, gi);
            // (r l).n / (r |l|)^2 = (l.n) / (r |l|^2)
            const float inv = rinv * linv;
            const float ps = ps1 * inv, qt = qt1 * inv;
            const float ar = fmaf(-rr, ps, -knn * gi), ai = fmaf(-ri2, ps, knn * gr);
            const float br = fmaf(-ri2 * qt, invkf, -gr), bi = fmaf(rr * qt, invkf, -gi);
            const float bt[3] = {fmaf(r, pt[0], rad.w), r * pt[1], r * pt[2]};
            const float bs[3] = {fmaf(r, pq[0], rad.w), r * pq[1], r * pq[2]};
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                b[2 * i] = fmaf(br, bt[i], b[2 * i]);
                b[2 * i + 1] = fmaf(bi, bt[i], b[2 * i + 1]);
                const float ari = ar * bt[i], aii = ai * bt[i];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    m[2 * (3 * i + j)] = fmaf(ari, bs[j], m[2 * (3 * i + j)]);
                    m[2 * (3 * i + j) + 1] = fmaf(aii, bs[j], m[2 * (3 * i + j) + 1]);
                }
            }
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0)
        flagError(error, kErrDistance);
    // Warp sums of the 26 moment values as a reduce-scatter: after the pass at
    // distance h a lane keeps the h partial sums of the half its lane bit h
    // selects, so after five passes (31 shuffles instead of 26 x 5) lane l holds
    // the sum of value l.
    float v[32];
#pragma unroll
    for (int c = 0; c < 18; ++c)
        v[c] = m[c];
#pragma unroll
    for (int c = 0; c < 6; ++c)
        v[18 + c] = b[c];
    v[24] = g[0];
    v[25] = g[1];
#pragma unroll
    for (int c = 26; c < 32; ++c)
        v[c] = 0.f;
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool upper = (lane & unsigned(h)) != 0;
#pragma unroll
        for (int c = 0; c < h; ++c) {
            const float send = upper ? v[c] : v[c + h], keep = upper ? v[c + h] : v[c];
            v[c] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
    }
    const float sum = v[0];  // value `lane`
    // lanes 0..11 write record entry `lane`: canonical index of each local vertex
    int invT[3], invS[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        invT[job.permTest[c]] = c;
        invS[job.permTrial[c]] = c;
    }
    const int o = lane < 12 ? int(lane) : 0;
    const int i = o < 9 ? o / 3 : o - 9, j = o % 3;
    const int src = o < 9 ? 2 * (3 * invT[i] + invS[j]) : 18 + 2 * invT[i];
    const float vre = __shfl_sync(0xffffffffu, sum, src), vim = __shfl_sync(0xffffffffu, sum, src + 1);
    const float g0 = __shfl_sync(0xffffffffu, sum, 24), g1 = __shfl_sync(0xffffffffu, sum, 25);
    if (lane < 12) {
        double re, im;
        if (o < 9) {
            const double curl = t.curl[3 * i] * s.curl[3 * j] + t.curl[3 * i + 1] * s.curl[3 * j + 1] +
                                t.curl[3 * i + 2] * s.curl[3 * j + 2];
            re = double(vre) + double(g1) * curl * invk;
            im = double(vim) - double(g0) * curl * invk;
        } else {
            re = vre;
            im = double(vim) + (coincident ? t.area / (6.0 * k) : 0.0);
        }
        if (!isfinite(re) || !isfinite(im))
            flagError(error, kErrNonFinite);
        float *dst = records + size_t(f) * T * T * kRecordDoubles + recordOffset(T, size_t(job.trial) * T + job.test, o);
        *reinterpret_cast<float2 *>(dst) = make_float2(float(re), float(im));
    }
}

// ---------------------------------------------------------------------------
// Near pairs (cuda_solver.cu:430-518, near_projection.hpp:228-254): one CTA
// per unordered pair, both directions from the shared patch samples.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void nearSample(double (&acc)[54], const DPanel &t, const DPanel &s, const double *bt,
                                           const double *bs, double w, double k, bool &bad) {
    const double dx = (t.v0[0] - s.v0[0]) + ((t.e1[0] * bt[1] + t.e2[0] * bt[2]) - (s.e1[0] * bs[1] + s.e2[0] * bs[2]));
    const double dy = (t.v0[1] - s.v0[1]) + ((t.e1[1] * bt[1] + t.e2[1] * bt[2]) - (s.e1[1] * bs[1] + s.e2[1] * bs[2]));
    const double dz = (t.v0[2] - s.v0[2]) + ((t.e1[2] * bt[1] + t.e2[2] * bt[2]) - (s.e1[2] * bs[1] + s.e2[2] * bs[2]));
    const double r2 = dx * dx + dy * dy + dz * dz;
    bad |= !(r2 > 0) || !isfinite(r2);
    const double rinv = rsqrt(r2);
    const double r = r2 * rinv, kr = k * r;
    double sn, cs;
    sincos(kr, &sn, &cs);
    const double sc = w * rinv;
    const double gr = cs * sc, gi = -sn * sc;
    const double rr = gr - gi * kr, ri = gi + gr * kr;
    const double rinv2 = rinv * rinv;
    const double ps = (dx * s.n[0] + dy * s.n[1] + dz * s.n[2]) * rinv2;
    const double qt = -(dx * t.n[0] + dy * t.n[1] + dz * t.n[2]) * rinv2;
    const double val[6] = {gr, gi, rr * ps, ri * ps, rr * qt, ri * qt};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double bij = bt[i] * bs[j];
#pragma unroll
            for (int kind = 0; kind < 3; ++kind) {
                acc[kind * 18 + 2 * (3 * i + j)] += val[2 * kind] * bij;
                acc[kind * 18 + 2 * (3 * i + j) + 1] += val[2 * kind + 1] * bij;
            }
        }
}

// Mixed-form near sample: FP64 displacement and phase, FP32 kernel values
// and accumulation.
__device__ __forceinline__ void nearSample(float (&acc)[54], const DPanel &t, const DPanel &s, const double *bt,
                                           const double *bs, double w, double k, bool &bad) {
    const double dx = (t.v0[0] - s.v0[0]) + ((t.e1[0] * bt[1] + t.e2[0] * bt[2]) - (s.e1[0] * bs[1] + s.e2[0] * bs[2]));
    const double dy = (t.v0[1] - s.v0[1]) + ((t.e1[1] * bt[1] + t.e2[1] * bt[2]) - (s.e1[1] * bs[1] + s.e2[1] * bs[2]));
    const double dz = (t.v0[2] - s.v0[2]) + ((t.e1[2] * bt[1] + t.e2[2] * bt[2]) - (s.e1[2] * bs[1] + s.e2[2] * bs[2]));
    const float ns[3] = {float(s.n[0]), float(s.n[1]), float(s.n[2])};
    const float nt[3] = {float(t.n[0]), float(t.n[1]), float(t.n[2])};
    float val[6];
    mixedValues(dx, dy, dz, float(w), k, ns, nt, val, bad);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float bij = float(bt[i] * bs[j]);
#pragma unroll
            for (int kind = 0; kind < 3; ++kind) {
                acc[kind * 18 + 2 * (3 * i + j)] += val[2 * kind] * bij;
                acc[kind * 18 + 2 * (3 * i + j) + 1] += val[2 * kind + 1] * bij;
            }
        }
}

// Green values (g, P, Q as re/im pairs) of one sample of a near pair in the
// plain form, FP64.
__device__ __forceinline__ void plainValues(double dx, double dy, double dz, double w, double k, const DPanel &t,
                                            const DPanel &s, double (&val)[6], bool &bad) {
    const double r2 = dx * dx + dy * dy + dz * dz;
    bad |= !(r2 > 0) || !isfinite(r2);
    const double rinv = rsqrt(r2);
    const double r = r2 * rinv, kr = k * r;
    double sn, cs;
    sincos(kr, &sn, &cs);
    const double sc = w * rinv;
    const double gr = cs * sc, gi = -sn * sc;
    const double rr = gr - gi * kr, ri = gi + gr * kr;
    const double rinv2 = rinv * rinv;
    const double ps = (dx * s.n[0] + dy * s.n[1] + dz * s.n[2]) * rinv2;
    const double qt = -(dx * t.n[0] + dy * t.n[1] + dz * t.n[2]) * rinv2;
    val[0] = gr;
    val[1] = gi;
    val[2] = rr * ps;
    val[3] = ri * ps;
    val[4] = rr * qt;
    val[5] = ri * qt;
}

// Near pairs whose patches are all tensor patches: one warp per unordered
// pair. Lane (x, half) owns test point x of the patch rule and half of the
// trial points; trial bases are contracted in registers, test bases through
// shared memory by the 27 lanes that own a (kind, i, j) moment. Pairs with
// projected patches go to nearKernel.
template <bool Mixed>
__global__ void __launch_bounds__(64, Mixed ? 10 : 1) nearWarpKernel(const DPanel *__restrict__ panels, uint32_t T,
                                                      const NearPairJob *__restrict__ jobs, uint32_t jobCount,
                                                      const Patch *__restrict__ patches, const double *__restrict__ ks,
                                                      std::conditional_t<Mixed, float, double> *__restrict__ records,
                                                      SlotMap map, int *error) {
    using Acc = std::conditional_t<Mixed, float, double>;
    __shared__ Acc sS[2][64][18];     // per warp: trial-contracted values S(x)
    __shared__ double sB[2][64][3];   // per warp: mapped test barycentrics
    __shared__ double sY[2][64][3];   // per warp: mapped trial barycentrics
    __shared__ double sE[2][64][3];   // per warp: trial points' offsets from the trial panel's first vertex
    __shared__ double sM[2][54];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t pairIndex = blockIdx.x * 2 + warp;
    if (pairIndex >= jobCount)
        return;
    const NearPairJob job = jobs[pairIndex];
    const int f = blockIdx.y;
    const double k = ks[f], invk = 1.0 / k;
    const DPanel &t = panels[job.first];
    const DPanel &s = panels[job.second];
    const double w4 = 4.0 * t.area * s.area * kInvFourPi;
    bool bad = false;
    double own[2] = {0, 0};  // lanes 0..26: accumulated moment (kind, i, j) of this pair
    const double d0[3] = {t.v0[0] - s.v0[0], t.v0[1] - s.v0[1], t.v0[2] - s.v0[2]};
    for (uint32_t q = 0; q < job.patchCount; ++q) {
        const Patch &patch = patches[job.firstPatch + q];
        const int n = patch.degree == 14 ? 64 : 16;
        const int ro = patch.degree == 14 ? 34 : 18;  // rule offsets of the 16- and 64-point bins
        // mapped rule points of this patch (test from patch.test, trial from patch.trial)
        for (int idx = lane; idx < n; idx += 32) {
            double by[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                sB[warp][idx][i] = cRule[4 * (ro + idx)] * patch.test[i] + cRule[4 * (ro + idx) + 1] * patch.test[3 + i] +
                                   cRule[4 * (ro + idx) + 2] * patch.test[6 + i];
                by[i] = cRule[4 * (ro + idx)] * patch.trial[i] + cRule[4 * (ro + idx) + 1] * patch.trial[3 + i] +
                        cRule[4 * (ro + idx) + 2] * patch.trial[6 + i];
                sY[warp][idx][i] = by[i];
            }
            // the trial point's offset from the trial panel's first vertex, once per patch point
#pragma unroll
            for (int c = 0; c < 3; ++c)
                sE[warp][idx][c] = s.e1[c] * by[1] + s.e2[c] * by[2];
        }
        __syncwarp();
        const double wpatch = patch.areaFraction * w4;
        // lane -> test points x = lane (+32) ; for n = 16, lanes 16..31 take the second half of the trial points
        const int xCount = n == 16 ? 1 : 2;
        for (int xi = 0; xi < xCount; ++xi) {
            const int x = n == 16 ? (lane & 15) : lane + 32 * xi;
            const int y0 = n == 16 ? (lane >> 4) * 8 : 0, y1 = n == 16 ? y0 + 8 : n;
            const double *bt = sB[warp][x];
            const double Dx = d0[0] + (t.e1[0] * bt[1] + t.e2[0] * bt[2]);
            const double Dy = d0[1] + (t.e1[1] * bt[1] + t.e2[1] * bt[2]);
            const double Dz = d0[2] + (t.e1[2] * bt[1] + t.e2[2] * bt[2]);
            const double wx = cRule[4 * (ro + x) + 3] * wpatch;
            Acc S[18];
#pragma unroll
            for (int c = 0; c < 18; ++c)
                S[c] = 0;
            for (int y = y0; y < y1; ++y) {
                const double *bs = sY[warp][y], *ey = sE[warp][y];
                const double dx = Dx - ey[0];
                const double dy = Dy - ey[1];
                const double dz = Dz - ey[2];
                const double w = wx * cRule[4 * (ro + y) + 3];
                Acc val[6];
                if constexpr (Mixed) {
                    const float ns[3] = {float(s.n[0]), float(s.n[1]), float(s.n[2])};
                    const float nt[3] = {float(t.n[0]), float(t.n[1]), float(t.n[2])};
                    mixedValues(dx, dy, dz, float(w), k, ns, nt, val, bad);
                } else {
                    plainValues(dx, dy, dz, w, k, t, s, val, bad);
                }
#pragma unroll
                for (int kind = 0; kind < 3; ++kind)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        S[kind * 6 + 2 * j] += val[2 * kind] * Acc(bs[j]);
                        S[kind * 6 + 2 * j + 1] += val[2 * kind + 1] * Acc(bs[j]);
                    }
            }
            if (n == 16) {
#pragma unroll
                for (int c = 0; c < 18; ++c)
                    S[c] += __shfl_xor_sync(0xffffffffu, S[c], 16);
                if (lane < 16)
#pragma unroll
                    for (int c = 0; c < 18; ++c)
                        sS[warp][x][c] = S[c];
            } else {
#pragma unroll
                for (int c = 0; c < 18; ++c)
                    sS[warp][x][c] = S[c];
            }
        }
        __syncwarp();
        if (lane < 27) {
            const int kind = lane / 9, i = (lane % 9) / 3, j = lane % 3;
            double re = 0, im = 0;
            for (int x = 0; x < n; ++x) {
                re += sB[warp][x][i] * sS[warp][x][kind * 6 + 2 * j];
                im += sB[warp][x][i] * sS[warp][x][kind * 6 + 2 * j + 1];
            }
            own[0] += re;
            own[1] += im;
        }
        __syncwarp();
    }
    if (lane < 27) {
        const int kind = lane / 9, e = lane % 9;
        sM[warp][kind * 18 + 2 * e] = own[0];
        sM[warp][kind * 18 + 2 * e + 1] = own[1];
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0)
        flagError(error, kErrDistance);
    __syncwarp();
    if (lane < 24) {
        const int o = lane;
        double re, im;
        pairRecordValue(o, &sM[warp][0], &sM[warp][18], &sM[warp][36], t, s, k, invk, re, im);
        if (!isfinite(re) || !isfinite(im))
            flagError(error, kErrNonFinite);
        const size_t slot = o < 12 ? mapSlot(map, T, job.first, job.second) : mapSlot(map, T, job.second, job.first);
        const int e = o < 12 ? o : o - 12;
        if (slot != kNoSlot) {
            Acc *dst = records + size_t(f) * map.planeSlots * kRecordDoubles + mapOffset(map.planeSlots, slot, e);
            dst[0] = Acc(re);
            dst[1] = Acc(im);
        } else
            flagError(error, kErrEscapedPlan);
    }
}

template <bool Mixed>
__global__ void __launch_bounds__(128) nearKernel(const DPanel *__restrict__ panels, uint32_t T,
                                                  const NearPairJob *__restrict__ jobs,
                                                  const Patch *__restrict__ patches, const double *__restrict__ ks,
                                                  std::conditional_t<Mixed, float, double> *__restrict__ records,
                                                  SlotMap map, int *error) {
    using Acc = std::conditional_t<Mixed, float, double>;
    __shared__ double red[4][54];
    __shared__ double pts[2][64][3];
    const NearPairJob job = jobs[blockIdx.x];
    const int f = blockIdx.y;
    const double k = ks[f], invk = 1.0 / k;
    const DPanel &t = panels[job.first];
    const DPanel &s = panels[job.second];
    const double w4 = 4.0 * t.area * s.area * kInvFourPi;
    Acc acc[54];
#pragma unroll
    for (int c = 0; c < 54; ++c)
        acc[c] = 0;
    bool bad = false;
    FanPanel ft, fs;
    for (int i = 0; i < 3; ++i) {
        ft.v[i] = V3{t.v0[0] + (i == 1 ? t.e1[0] : i == 2 ? t.e2[0] : 0.0), t.v0[1] + (i == 1 ? t.e1[1] : i == 2 ? t.e2[1] : 0.0),
                     t.v0[2] + (i == 1 ? t.e1[2] : i == 2 ? t.e2[2] : 0.0)};
        fs.v[i] = V3{s.v0[0] + (i == 1 ? s.e1[0] : i == 2 ? s.e2[0] : 0.0), s.v0[1] + (i == 1 ? s.e1[1] : i == 2 ? s.e2[1] : 0.0),
                     s.v0[2] + (i == 1 ? s.e1[2] : i == 2 ? s.e2[2] : 0.0)};
    }
    ft.n = V3{t.n[0], t.n[1], t.n[2]};
    fs.n = V3{s.n[0], s.n[1], s.n[2]};
    ft.area = t.area;
    fs.area = s.area;
    for (uint32_t q = 0; q < job.patchCount; ++q) {
        const Patch &patch = patches[job.firstPatch + q];
        const int n = patch.degree == 14 ? 64 : 16;
        const int ro = patch.degree == 14 ? 34 : 18;  // rule offsets of the 16- and 64-point bins
        if (!patch.projection) {
            __syncthreads();
            for (int idx = threadIdx.x; idx < 2 * n; idx += blockDim.x) {
                const int side = idx / n, x = idx % n;
                const double *pv = side ? patch.trial : patch.test;
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    pts[side][x][i] = cRule[4 * (ro + x)] * pv[i] + cRule[4 * (ro + x) + 1] * pv[3 + i] +
                                      cRule[4 * (ro + x) + 2] * pv[6 + i];
            }
            __syncthreads();
            for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
                const int x = idx / n, y = idx % n;
                const double w = cRule[4 * (ro + x) + 3] * cRule[4 * (ro + y) + 3] * patch.areaFraction * w4;
                nearSample(acc, t, s, pts[0][x], pts[1][y], w, k, bad);
            }
            continue;
        }
        const uint32_t order = 20 * patch.intervals;
        const uint32_t points = uint32_t(n) * 3 * order * order;
        for (uint32_t idx = threadIdx.x; idx < points; idx += blockDim.x) {
            uint32_t rest = idx;
            const uint32_t radial = rest % order;
            rest /= order;
            const uint32_t angular = rest % order;
            rest /= order;
            const uint32_t edge = rest % 3, outer = rest / 3;
            GaussPoint u{cGauss20[2 * (angular % 20)], cGauss20[2 * (angular % 20) + 1]};
            GaussPoint v{cGauss20[2 * (radial % 20)], cGauss20[2 * (radial % 20) + 1]};
            u.x = (angular / 20 + u.x) / patch.intervals;
            v.x = (radial / 20 + v.x) / patch.intervals;
            u.w /= patch.intervals;
            v.w /= patch.intervals;
            const double ob[3] = {cRule[4 * (ro + outer)], cRule[4 * (ro + outer) + 1], cRule[4 * (ro + outer) + 2]};
            const ProjOuter po = projOuter(ob, cRule[4 * (ro + outer) + 3], patch, ft, fs);
            const PairPoint pp = projPoint(po, projRay(po, projEdge(po, edge, fs), u), v);
            nearSample(acc, t, s, pp.t, pp.s, pp.w * w4, k, bad);
        }
    }
    if (bad)
        flagError(error, kErrDistance);
    __syncthreads();
    double accd[54];
#pragma unroll
    for (int c = 0; c < 54; ++c)
        accd[c] = acc[c];
    blockReduce<54>(accd, red);
    if (threadIdx.x < 24) {
        const int o = threadIdx.x;
        double re, im;
        pairRecordValue(o, &red[0][0], &red[0][18], &red[0][36], t, s, k, invk, re, im);
        if (!isfinite(re) || !isfinite(im))
            flagError(error, kErrNonFinite);
        const size_t slot = o < 12 ? mapSlot(map, T, job.first, job.second) : mapSlot(map, T, job.second, job.first);
        const int e = o < 12 ? o : o - 12;
        if (slot != kNoSlot) {
            Acc *dst = records + size_t(f) * map.planeSlots * kRecordDoubles + mapOffset(map.planeSlots, slot, e);
            dst[0] = Acc(re);
            dst[1] = Acc(im);
        } else
            flagError(error, kErrEscapedPlan);
    }
}

// ---------------------------------------------------------------------------
// Deterministic gathers: records -> per-(test panel, trial vertex) columns ->
// matrix entries, and records x flux -> right-hand side.
// ---------------------------------------------------------------------------
// Both gathers in one CTA per matrix column (trial vertex b, frequency f),
// for meshes whose 3T column entries fit in shared memory: first the
// per-(test panel, local row) sums over the trial panels at b (coalesced
// plane reads), then each row's sum over its incident panels plus the half
// mass, written as a contiguous column. Same summation order as
// gatherTrialKernel followed by gatherTestKernel.
// Three complex values of a record plane entry as three vector loads (entries
// are 6 values: 24 B in FP32, 48 B in FP64, so 8- and 16-byte aligned).
__device__ __forceinline__ void load6(const float *r, float (&v)[6]) {
    const float2 *q = reinterpret_cast<const float2 *>(r);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float2 x = q[c];
        v[2 * c] = x.x;
        v[2 * c + 1] = x.y;
    }
}
__device__ __forceinline__ void load6(const double *r, double (&v)[6]) {
    const double2 *q = reinterpret_cast<const double2 *>(r);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double2 x = q[c];
        v[2 * c] = x.x;
        v[2 * c + 1] = x.y;
    }
}

template <class Rec>
__global__ void __launch_bounds__(512, 2) gatherColumnKernel(const Rec *__restrict__ records,
                                                          const uint32_t *__restrict__ incOffsets,
                                                          const uint32_t *__restrict__ incPanel,
                                                          const uint8_t *__restrict__ incLocal,
                                                          const DPanel *__restrict__ panels,
                                                          const double *__restrict__ rowScale, uint32_t T, uint32_t N,
                                                          double *__restrict__ A) {
    extern __shared__ double2 column[];  // [3T]: entry (test panel t, local row la) of column b
    const uint32_t b = blockIdx.x;
    const int f = blockIdx.y;
    const Rec *rec = records + size_t(f) * T * T * kRecordDoubles;
    const uint32_t o0 = incOffsets[b], o1 = incOffsets[b + 1];
    for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) {
        double acc[6] = {0, 0, 0, 0, 0, 0};
        // trial panels at b in chunks of 4: the record loads of a chunk are in flight together
        for (uint32_t o = o0; o < o1; o += 4) {
            Rec v[4][6];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (o + u < o1)
                    load6(rec + recordOffset(T, size_t(incPanel[o + u]) * T + t, incLocal[o + u]), v[u]);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (o + u < o1)
#pragma unroll
                    for (int c = 0; c < 6; ++c)
                        acc[c] += double(v[u][c]);
        }
#pragma unroll
        for (int la = 0; la < 3; ++la)
            column[3 * t + la] = make_double2(acc[2 * la], acc[2 * la + 1]);
    }
    __syncthreads();
    for (uint32_t a = threadIdx.x; a < N; a += blockDim.x) {
        double re = 0, im = 0;
        const uint32_t a0 = incOffsets[a], a1 = incOffsets[a + 1];
        for (uint32_t o = a0; o < a1; o += 4) {
            uint32_t t[4], n[4][3];
            int la[4];
            double area[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (o + u < a1) {
                    t[u] = incPanel[o + u];
                    la[u] = incLocal[o + u];
                    const DPanel &p = panels[t[u]];
                    n[u][0] = p.nodes[0];
                    n[u][1] = p.nodes[1];
                    n[u][2] = p.nodes[2];
                    area[u] = p.area;
                }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (o + u < a1) {
                    const double2 v = column[3 * t[u] + la[u]];
                    re += v.x;
                    im += v.y;
                    if (n[u][0] == b || n[u][1] == b || n[u][2] == b)
                        re += area[u] * (a == b ? 2.0 : 1.0) / 24.0;
                }
        }
        const double sc = rowScale[a];
        double *dst = A + (size_t(f) * N * N + size_t(b) * N + a) * 2;
        dst[0] = re * sc;
        dst[1] = im * sc;
    }
}

template <class Rec>
__global__ void gatherTrialKernel(const Rec *__restrict__ records, const uint32_t *__restrict__ incOffsets,
                                  const uint32_t *__restrict__ incPanel, const uint8_t *__restrict__ incLocal,
                                  uint32_t T, uint32_t N, Rec *__restrict__ columns) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t b = blockIdx.y;
    const int f = blockIdx.z;
    if (t >= T)
        return;
    const Rec *rec = records + size_t(f) * T * T * kRecordDoubles;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t o = incOffsets[b]; o < incOffsets[b + 1]; ++o) {
        const uint32_t s = incPanel[o];
        const int lb = incLocal[o];
        // column lb of the (trial s, test t) block: 3 contiguous complex values
        Rec v[6];
        load6(rec + recordOffset(T, size_t(s) * T + t, lb), v);
#pragma unroll
        for (int c = 0; c < 6; ++c)
            acc[c] += double(v[c]);
    }
    Rec *dst = columns + (size_t(f) * N + b) * 6 * T + 6 * size_t(t);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        dst[c] = Rec(acc[c]);
}

template <class Rec>
__global__ void gatherTestKernel(const Rec *__restrict__ columns, const DPanel *__restrict__ panels,
                                 const uint32_t *__restrict__ incOffsets, const uint32_t *__restrict__ incPanel,
                                 const uint8_t *__restrict__ incLocal, const double *__restrict__ rowScale, uint32_t T,
                                 uint32_t N, double *__restrict__ A) {
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t b = blockIdx.y;
    const int f = blockIdx.z;
    if (a >= N)
        return;
    const Rec *col = columns + (size_t(f) * N + b) * 6 * T;
    double re = 0, im = 0;
    for (uint32_t o = incOffsets[a]; o < incOffsets[a + 1]; ++o) {
        const uint32_t t = incPanel[o];
        const int la = incLocal[o];
        re += double(col[6 * size_t(t) + 2 * la]);
        im += double(col[6 * size_t(t) + 2 * la + 1]);
        const DPanel &p = panels[t];
        if (p.nodes[0] == b || p.nodes[1] == b || p.nodes[2] == b)
            re += p.area * (a == b ? 2.0 : 1.0) / 24.0;
    }
    const double sc = rowScale[a];
    double *dst = A + (size_t(f) * N * N + size_t(b) * N + a) * 2;
    dst[0] = re * sc;
    dst[1] = im * sc;
}

// Per-panel right-hand-side partials: sum over trial panels s of the
// (s, t) moments times the flux of s. A CTA takes 32 test panels; its 8
// warps take every 8th trial panel, and the partial sums are added in a
// fixed order (deterministic).
template <class Rec>
__global__ void __launch_bounds__(256) rhsPanelKernel(const Rec *__restrict__ records, const double *__restrict__ flux,
                                                      uint32_t T, uint32_t E, double *__restrict__ panelRhs) {
    __shared__ double part[8][32][6];
    const uint32_t lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const uint32_t t = blockIdx.x * 32 + lane;
    const uint32_t e = blockIdx.y;
    const int f = blockIdx.z;
    const Rec *rec = records + size_t(f) * T * T * kRecordDoubles;
    const double *q = flux + (size_t(f) * E + e) * 2 * T;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (t < T)
        for (uint32_t s = g; s < T; s += 8) {
            const double qr = q[2 * s], qi = q[2 * s + 1];
            if (qr == 0 && qi == 0)
                continue;
            Rec r[6];
            load6(rec + recordOffset(T, size_t(s) * T + t, 9), r);
#pragma unroll
            for (int la = 0; la < 3; ++la) {
                const double rr = r[2 * la], ri = r[2 * la + 1];
                acc[2 * la] += rr * qr - ri * qi;
                acc[2 * la + 1] += rr * qi + ri * qr;
            }
        }
#pragma unroll
    for (int c = 0; c < 6; ++c)
        part[g][lane][c] = acc[c];
    __syncthreads();
    if (g != 0 || t >= T)
        return;
    double *dst = panelRhs + (size_t(f) * E + e) * 6 * T + 6 * size_t(t);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        double v = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w)
            v += part[w][lane][c];
        dst[c] = v;
    }
}

__global__ void rhsVertexKernel(const double *__restrict__ panelRhs, const uint32_t *__restrict__ incOffsets,
                                const uint32_t *__restrict__ incPanel, const uint8_t *__restrict__ incLocal,
                                const double *__restrict__ rowScale, uint32_t T, uint32_t N, uint32_t E,
                                double *__restrict__ rhs) {
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t e = blockIdx.y;
    const int f = blockIdx.z;
    if (a >= N)
        return;
    const double *src = panelRhs + (size_t(f) * E + e) * 6 * T;
    double re = 0, im = 0;
    for (uint32_t o = incOffsets[a]; o < incOffsets[a + 1]; ++o) {
        re += src[6 * size_t(incPanel[o]) + 2 * incLocal[o]];
        im += src[6 * size_t(incPanel[o]) + 2 * incLocal[o] + 1];
    }
    double *dst = rhs + ((size_t(f) * E + e) * N + a) * 2;
    dst[0] = re * rowScale[a];
    dst[1] = im * rowScale[a];
}

int smCount() {
    static PerDeviceValue<int> count;
    return count.get([]() {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, currentDevice()) != cudaSuccess || n <= 0)
            n = 148;
        return n;
    });
}

template <int NP>
void launchRegular(const AssemblyGeometry &g, const double *ks, uint32_t B, const AssemblyWorkspace &ws, int bin,
                   int *error, cudaStream_t stream, KernelTimer *timer, bool mixed, const SlotMap &map) {
    const char *names[kBins] = {"regular_q6", "regular_q12", "regular_q16", "regular_q64"};
    const char *mixedNames[kBins] = {"regular_mixed_q6", "regular_mixed_q12", "regular_mixed_q16",
                                     "regular_mixed_q64"};
    TimedScope scope(timer, mixed ? mixedNames[bin] : names[bin], stream);
    // Grid of the grid-stride pair loop in CTAs per SM: each pair is one
    // independent item, so the choice moves only the load balance and occupancy.
    static constexpr int kMixedCtas[] = {16, 8, 24, 32};
    static constexpr int kPlainCtas[] = {8, 4, 16};
    const int candidates = mixed ? 4 : 3;
    const auto launch = [&](int c) {
        if (mixed) {
            const dim3 grid(unsigned(smCount() * kMixedCtas[c]), B);
            regularMixedKernel<NP><<<grid, 128, 0, stream>>>(g.mixedPanels, g.bounds, g.T, ks, ws.bins, ws.binCounts,
                                                             ws.binCapacity, ws.binOffsets, bin,
                                                             static_cast<float *>(ws.records), error);
        } else {
            const dim3 grid(unsigned(smCount() * kPlainCtas[c]), B);
            regularPairsKernel<NP><<<grid, kPlainThreads, 0, stream>>>(g.panels, g.T, ks, ws.bins, ws.binCounts,
                                                             ws.binCapacity, ws.binOffsets, bin,
                                                             static_cast<double *>(ws.records), map, error);
        }
        cudaCheck(cudaGetLastError(), "regular pair assembly launch");
    };
    // size class: the form, the rule, the batch and the mesh size to a power of two
    const std::string key = std::string(mixed ? "regular_mixed" : "regular_fp64") + "_q" + std::to_string(NP) +
                            "_B" + std::to_string(B) + "_T2^" + std::to_string(31 - __builtin_clz(g.T | 1u)) +
                            (map.row ? "_near" : "");
    Autotuner &tuner = Autotuner::instance();
    int c = tuner.choice(key);
    // tuned on first use, outside a capture and outside a profiled solve (whose
    // per-family times would count the candidates' launches)
    if (c < 0 && tuner.enabled() && !(timer && timer->enabled()) && !capturing(stream)) {
        tuner.tune(key, candidates, stream, launch);
        return;
    }
    launch(c < 0 ? 0 : c);
}

}  // namespace

std::vector<float> buildSingularTable(unsigned order) {
    const auto gauss = gaussLegendre01(order);
    const size_t per = size_t(order) * order * order;
    std::vector<float> out((13 * per) * 12 + order * 4, 0.f);
    const uint32_t topologies[3] = {kSharedVertex, kSharedEdge, kCoincident};
    size_t row = 0;
    for (uint32_t topo : topologies)
        for (unsigned sector = 0; sector < sectorCount(topo); ++sector)
            for (size_t tuple = 0; tuple < per; ++tuple, ++row) {
                const size_t wi = tuple % order, vi = (tuple / order) % order, ui = tuple / (size_t(order) * order);
                const PairPoint p = sauterSchwab(topo, sector, 1.0, gauss[ui].x, gauss[vi].x, gauss[wi].x);
                // displacement coefficients over the canonical edges (shared ones merged)
                double a1 = p.t[1], a2 = p.t[2], b1 = p.s[1], b2 = p.s[2];
                if (topo == kSharedEdge || topo == kCoincident) {
                    a1 -= b1;
                    b1 = 0;
                }
                if (topo == kCoincident) {
                    a2 -= b2;
                    b2 = 0;
                }
                float *q = &out[12 * row];
                const double v[11] = {p.t[0], p.t[1], p.t[2], p.s[0], p.s[1], p.s[2], a1, a2, b1, b2,
                                      p.w * gauss[ui].w * gauss[vi].w * gauss[wi].w};
                for (int c = 0; c < 11; ++c)
                    q[c] = float(v[c]);
            }
    for (unsigned ri = 0; ri < order; ++ri) {
        const double r = gauss[ri].x;
        out[12 * 13 * per + 4 * ri] = float(r);
        out[12 * 13 * per + 4 * ri + 1] = float(r * r * r * gauss[ri].w);
        out[12 * 13 * per + 4 * ri + 2] = float(1.0 / r);
        out[12 * 13 * per + 4 * ri + 3] = float(1.0 - r);
    }
    return out;
}

namespace {
void uploadRuleTablesNow(cudaStream_t stream) {
    double table[kRulePoints * 4];
    const unsigned degrees[kBins] = {4, 6, 8, 14};
    int o = 0;
    for (int b = 0; b < kBins; ++b) {
        const auto r = triangleRule(degrees[b]);
        for (const auto &p : r) {
            table[4 * o] = p.b[0];
            table[4 * o + 1] = p.b[1];
            table[4 * o + 2] = p.b[2];
            table[4 * o + 3] = p.w;
            ++o;
        }
    }
    cudaCheck(cudaMemcpyToSymbolAsync(cRule, table, sizeof(table), 0, cudaMemcpyHostToDevice, stream), "rule upload");
    static float tableF[kRulePoints * 8];
    for (int i = 0; i < kRulePoints; ++i) {
        const double b1 = table[4 * i + 1], b2 = table[4 * i + 2];
        const double v[8] = {table[4 * i], b1, b2, table[4 * i + 3], b1 * b1, 2 * b1 * b2, b2 * b2, 0.0};
        for (int c = 0; c < 8; ++c)
            tableF[8 * i + c] = float(v[c]);
    }
    cudaCheck(cudaMemcpyToSymbolAsync(cRuleF, tableF, sizeof(tableF), 0, cudaMemcpyHostToDevice, stream),
              "rule upload");
    double g20[40];
    const auto g = gaussLegendre01(20);
    for (int i = 0; i < 20; ++i) {
        g20[2 * i] = g[i].x;
        g20[2 * i + 1] = g[i].w;
    }
    cudaCheck(cudaMemcpyToSymbolAsync(cGauss20, g20, sizeof(g20), 0, cudaMemcpyHostToDevice, stream), "gauss upload");
    cudaCheck(cudaStreamSynchronize(stream), "rule upload sync");
}
}  // namespace

// The rule tables in constant memory, once per device (each device has its own
// copy of the __constant__ arrays).
void uploadRuleTables(cudaStream_t stream) {
    static PerDeviceOnce once;
    once.run([&]() { uploadRuleTablesNow(stream); });
}

bool gatherUsesColumns(uint32_t T) { return size_t(3) * T * sizeof(double2) > kGatherColumnSmem; }

size_t recordBytes(uint32_t T, bool mixed) { return size_t(T) * T * kRecordDoubles * (mixed ? 4 : 8); }

size_t assemblyWorkspaceBytes(uint32_t T, uint32_t N, uint32_t E, uint32_t B, bool mixed) {
    const size_t pairs = size_t(T) * (T - 1) / 2;
    const size_t columns = gatherUsesColumns(T) ? size_t(N) * 6 * T * (mixed ? 4 : 8) : 0;
    const size_t bins = (T > kExactBinsT ? 1 : kBins) * pairs * sizeof(uint2);
    return size_t(B) * (recordBytes(T, mixed) + columns + size_t(E) * 6 * T * 8 + bins + kBins * (4 + 8));
}

namespace {
// Pair records of B frequencies: classification into rule bins (all
// unordered pairs, or the listed ones), then the regular, touching and near
// kernels, every record stored at its slot of `map`.
void computeRecords(const AssemblyGeometry &g, const double *ks, const double *gaussSingular, uint32_t B,
                    const AssemblyWorkspace &ws, const SlotMap &map, const uint2 *pairList, uint64_t listCount,
                    int *error, cudaStream_t stream, KernelTimer *timer, bool mixed) {
    const uint64_t pairs = uint64_t(g.T) * (g.T - 1) / 2;
    double *recD = static_cast<double *>(ws.records);
    float *recF = static_cast<float *>(ws.records);
    cudaCheck(cudaMemsetAsync(ws.binCounts, 0, sizeof(uint32_t) * kBins * B, stream), "bin reset");
    if (pairList) {
        TimedScope scope(timer, "classify_pairs", stream);
        if (listCount) {
            const unsigned blocks = unsigned(std::min<uint64_t>((listCount + 255) / 256, uint64_t(smCount()) * 16));
            classifyListKernel<<<blocks, 256, 0, stream>>>(pairList, listCount, g.pairCode, g.bounds, ks, B,
                                                           g.nearTolerance, g.minimumDegree, ws.bins, ws.binCounts,
                                                           ws.binCapacity, error);
            cudaCheck(cudaGetLastError(), "pair list classification launch");
        }
    } else if (pairs) {
        TimedScope scope(timer, "classify_pairs", stream);
        const unsigned blocks = unsigned(std::min<uint64_t>((pairs + 255) / 256, uint64_t(smCount()) * 16));
        if (ws.binOffsets) {  // count, scan, fill
            classifyPairsKernel<<<blocks, 256, 0, stream>>>(g.pairCode, g.bounds, g.T, ks, B, g.nearTolerance,
                                                            g.minimumDegree, ws.bins, ws.binCounts, ws.binCapacity,
                                                            ws.binOffsets, true, error);
            binOffsetsKernel<<<1, 1, 0, stream>>>(ws.binCounts, ws.binOffsets, B * kBins);
        }
        classifyPairsKernel<<<blocks, 256, 0, stream>>>(g.pairCode, g.bounds, g.T, ks, B, g.nearTolerance,
                                                        g.minimumDegree, ws.bins, ws.binCounts, ws.binCapacity,
                                                        ws.binOffsets, false, error);
        cudaCheck(cudaGetLastError(), "pair classification launch");
    }
    launchRegular<6>(g, ks, B, ws, 0, error, stream, timer, mixed, map);
    launchRegular<12>(g, ks, B, ws, 1, error, stream, timer, mixed, map);
    launchRegular<16>(g, ks, B, ws, 2, error, stream, timer, mixed, map);
    launchRegular<64>(g, ks, B, ws, 3, error, stream, timer, mixed, map);
    if (g.touchingCount) {
        TimedScope scope(timer, mixed ? "singular_mixed" : "singular", stream);
        if (mixed)
            singularMixedKernel<<<dim3((g.touchingCount + 3) / 4, B), 128, 0, stream>>>(
                g.panels, g.T, g.touching, g.touchingCount, ks, g.singularTable, g.singularOrder, recF, error);
        else
            singularKernel<<<dim3(g.touchingCount, B), 128, 0, stream>>>(g.panels, g.T, g.touching, ks,
                                                                         gaussSingular, g.singularOrder, recD, map,
                                                                         error);
        cudaCheck(cudaGetLastError(), "singular assembly launch");
    }
    if (g.nearPairCount - g.projectedPairCount) {
        TimedScope scope(timer, "near", stream);
        const uint32_t tensorPairs = g.nearPairCount - g.projectedPairCount;
        const dim3 grid((tensorPairs + 1) / 2, B);
        if (mixed)
            nearWarpKernel<true><<<grid, 64, 0, stream>>>(g.panels, g.T, g.nearPairs, tensorPairs, g.patches, ks,
                                                          recF, map, error);
        else
            nearWarpKernel<false><<<grid, 64, 0, stream>>>(g.panels, g.T, g.nearPairs, tensorPairs, g.patches, ks,
                                                           recD, map, error);
        cudaCheck(cudaGetLastError(), "near assembly launch");
    }
    if (g.projectedPairCount) {
        TimedScope scope(timer, "near_projected", stream);
        const NearPairJob *projected = g.nearPairs + (g.nearPairCount - g.projectedPairCount);
        if (mixed)
            nearKernel<true><<<dim3(g.projectedPairCount, B), 128, 0, stream>>>(g.panels, g.T, projected, g.patches,
                                                                                ks, recF, map, error);
        else
            nearKernel<false><<<dim3(g.projectedPairCount, B), 128, 0, stream>>>(g.panels, g.T, projected, g.patches,
                                                                                 ks, recD, map, error);
        cudaCheck(cudaGetLastError(), "projected near assembly launch");
    }
}
}  // namespace

void assembleBatch(const AssemblyGeometry &g, const double *ks, const double *gaussSingular, const double *flux,
                   uint32_t E, uint32_t B, const AssemblyWorkspace &ws, double *A, double *rhs, int *error,
                   cudaStream_t stream, KernelTimer *timer, bool mixed) {
    if (g.N > 65535 || B > 65535 || E > 65535)
        throw std::runtime_error("Dense assembly grid limits exceeded (more than 65535 vertices, frequencies or excitations).");
    SlotMap dense;
    dense.planeSlots = size_t(g.T) * g.T;
    computeRecords(g, ks, gaussSingular, B, ws, dense, nullptr, 0, error, stream, timer, mixed);
    double *recD = static_cast<double *>(ws.records);
    float *recF = static_cast<float *>(ws.records);
    const size_t columnBytes = size_t(3) * g.T * sizeof(double2);
    if (!gatherUsesColumns(g.T)) {
        TimedScope scope(timer, "gather_column", stream);
        static PerDeviceOnce attributes;
        attributes.run([]() {
            cudaCheck(cudaFuncSetAttribute(gatherColumnKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(kGatherColumnSmem)),
                      "gather smem attribute");
            cudaCheck(cudaFuncSetAttribute(gatherColumnKernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(kGatherColumnSmem)),
                      "gather smem attribute");
        });
        const dim3 grid(g.N, B);
        if (mixed)
            gatherColumnKernel<<<grid, 512, columnBytes, stream>>>(recF, g.incOffsets, g.incPanel, g.incLocal,
                                                                   g.panels, g.rowScale, g.T, g.N, A);
        else
            gatherColumnKernel<<<grid, 512, columnBytes, stream>>>(recD, g.incOffsets, g.incPanel, g.incLocal,
                                                                   g.panels, g.rowScale, g.T, g.N, A);
        cudaCheck(cudaGetLastError(), "column gather launch");
    } else {
        {
            TimedScope scope(timer, "gather_trial", stream);
            const dim3 grid((g.T + 127) / 128, g.N, B);
            if (mixed)
                gatherTrialKernel<<<grid, 128, 0, stream>>>(recF, g.incOffsets, g.incPanel, g.incLocal, g.T, g.N,
                                                            static_cast<float *>(ws.columns));
            else
                gatherTrialKernel<<<grid, 128, 0, stream>>>(recD, g.incOffsets, g.incPanel, g.incLocal, g.T, g.N,
                                                            static_cast<double *>(ws.columns));
            cudaCheck(cudaGetLastError(), "trial gather launch");
        }
        {
            TimedScope scope(timer, "gather_test", stream);
            const dim3 grid((g.N + 127) / 128, g.N, B);
            if (mixed)
                gatherTestKernel<<<grid, 128, 0, stream>>>(static_cast<const float *>(ws.columns), g.panels,
                                                           g.incOffsets, g.incPanel, g.incLocal, g.rowScale, g.T, g.N,
                                                           A);
            else
                gatherTestKernel<<<grid, 128, 0, stream>>>(static_cast<const double *>(ws.columns), g.panels,
                                                           g.incOffsets, g.incPanel, g.incLocal, g.rowScale, g.T, g.N,
                                                           A);
            cudaCheck(cudaGetLastError(), "test gather launch");
        }
    }
    {
        TimedScope scope(timer, "rhs_panel", stream);
        const dim3 grid((g.T + 31) / 32, E, B);
        if (mixed)
            rhsPanelKernel<<<grid, 256, 0, stream>>>(recF, flux, g.T, E, ws.panelRhs);
        else
            rhsPanelKernel<<<grid, 256, 0, stream>>>(recD, flux, g.T, E, ws.panelRhs);
    }
    {
        TimedScope scope(timer, "rhs_vertex", stream);
        rhsVertexKernel<<<dim3((g.N + 127) / 128, E, B), 128, 0, stream>>>(ws.panelRhs, g.incOffsets, g.incPanel,
                                                                           g.incLocal, g.rowScale, g.T, g.N, E, rhs);
    }
    cudaCheck(cudaGetLastError(), "rhs gather launch");
}

// ---------------------------------------------------------------------------
// Fast-multipole near field: records of the near panel pairs only (SlotMap
// over a panel-pair CSR), reduced into the near support-pair CSR values and
// the near part of the right-hand side.
// ---------------------------------------------------------------------------
namespace {

// vals[e] for entry e = (i, j) of the near CSR: rowScale_i (sum over the
// panels a of star i and s of star j of block entry (la, lb) of record (a, s)
// plus the P1 mass term of the panels holding both i and j). One warp per row.
__global__ void nearValuesKernel(const double *__restrict__ records, SlotMap map, const uint32_t *__restrict__ nearRow,
                                 const uint32_t *__restrict__ nearCol, const uint32_t *__restrict__ incOffsets,
                                 const uint32_t *__restrict__ incPanel, const uint8_t *__restrict__ incLocal,
                                 const DPanel *__restrict__ panels, const double *__restrict__ rowScale, uint32_t T,
                                 uint32_t N, double2 *vals, int *error) {
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= N)
        return;
    const double sc = rowScale[i];
    for (uint32_t e = nearRow[i] + lane; e < nearRow[i + 1]; e += 32) {
        const uint32_t j = nearCol[e];
        double re = 0, im = 0;
        for (uint32_t oa = incOffsets[i]; oa < incOffsets[i + 1]; ++oa) {
            const uint32_t a = incPanel[oa];
            const int la = incLocal[oa];
            for (uint32_t os = incOffsets[j]; os < incOffsets[j + 1]; ++os) {
                const size_t slot = mapSlot(map, T, a, incPanel[os]);
                if (slot == kNoSlot) {
                    flagError(error, kErrEscapedPlan);
                    continue;
                }
                const double *r = records + mapOffset(map.planeSlots, slot, 3 * la + incLocal[os]);
                re += r[0];
                im += r[1];
            }
            const DPanel &p = panels[a];
            if (p.nodes[0] == j || p.nodes[1] == j || p.nodes[2] == j)
                re += p.area * (i == j ? 2.0 : 1.0) / 24.0;
        }
        vals[e] = make_double2(re * sc, im * sc);
    }
}

// Near right-hand side: rhs_i = rowScale_i sum over near j, panels s of star j
// (weight 1/3: a panel's flux is emitted through its three vertex supports)
// and panels a of star i of rhs moment la of record (a, s) times q_s.
__global__ void nearRhsKernel(const double *__restrict__ records, SlotMap map, const uint32_t *__restrict__ nearRow,
                              const uint32_t *__restrict__ nearCol, const uint32_t *__restrict__ incOffsets,
                              const uint32_t *__restrict__ incPanel, const uint8_t *__restrict__ incLocal,
                              const double2 *__restrict__ flux, const double *__restrict__ rowScale, uint32_t T,
                              uint32_t N, uint32_t E, double2 *rhs, int *error) {
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const uint32_t ex = blockIdx.y;
    if (i >= N)
        return;
    const double2 *q = flux + size_t(ex) * T;
    double re = 0, im = 0;
    for (uint32_t e = nearRow[i] + lane; e < nearRow[i + 1]; e += 32) {
        const uint32_t j = nearCol[e];
        for (uint32_t os = incOffsets[j]; os < incOffsets[j + 1]; ++os) {
            const uint32_t sp = incPanel[os];
            const double2 qs = q[sp];
            if (qs.x == 0 && qs.y == 0)
                continue;
            double mr = 0, mi = 0;
            for (uint32_t oa = incOffsets[i]; oa < incOffsets[i + 1]; ++oa) {
                const size_t slot = mapSlot(map, T, incPanel[oa], sp);
                if (slot == kNoSlot) {
                    flagError(error, kErrEscapedPlan);
                    continue;
                }
                const double *r = records + mapOffset(map.planeSlots, slot, 9 + incLocal[oa]);
                mr += r[0];
                mi += r[1];
            }
            re += (mr * qs.x - mi * qs.y) / 3.0;
            im += (mr * qs.y + mi * qs.x) / 3.0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0)
        rhs[size_t(ex) * N + i] = make_double2(re * rowScale[i], im * rowScale[i]);
}

}  // namespace

size_t nearFieldWorkspaceBytes(size_t pairSlots, uint64_t pairCount) {
    return pairSlots * kRecordDoubles * 8 + kBins * pairCount * sizeof(uint2) + kBins * 16;
}

void assembleNearField(const AssemblyGeometry &g, const double *k, const double *gaussSingular, const double *flux,
                       uint32_t E, const NearFieldLayout &nf, void *workspace, double *vals, double *rhsNear,
                       int *error, cudaStream_t stream, KernelTimer *timer) {
    char *w = static_cast<char *>(workspace);
    AssemblyWorkspace ws{};
    ws.records = w;
    ws.bins = reinterpret_cast<uint2 *>(w + nf.pairSlots * kRecordDoubles * 8);
    ws.binCounts = reinterpret_cast<uint32_t *>(w + nf.pairSlots * kRecordDoubles * 8 + kBins * nf.pairCount * sizeof(uint2));
    ws.binCapacity = nf.pairCount;
    ws.binOffsets = nullptr;
    SlotMap map;
    map.row = nf.pairRow;
    map.col = nf.pairCol;
    map.planeSlots = nf.pairSlots;
    cudaCheck(cudaMemsetAsync(ws.records, 0, nf.pairSlots * kRecordDoubles * 8, stream), "near record reset");
    computeRecords(g, k, gaussSingular, 1, ws, map, nf.pairList, nf.pairCount, error, stream, timer, false);
    {
        TimedScope scope(timer, "fmm_near_values", stream);
        nearValuesKernel<<<(g.N * 32 + 255) / 256, 256, 0, stream>>>(
            static_cast<const double *>(ws.records), map, nf.nearRow, nf.nearCol, g.incOffsets, g.incPanel,
            g.incLocal, g.panels, g.rowScale, g.T, g.N, reinterpret_cast<double2 *>(vals), error);
        cudaCheck(cudaGetLastError(), "near values launch");
    }
    {
        TimedScope scope(timer, "fmm_near_rhs", stream);
        nearRhsKernel<<<dim3((g.N * 32 + 255) / 256, E), 256, 0, stream>>>(
            static_cast<const double *>(ws.records), map, nf.nearRow, nf.nearCol, g.incOffsets, g.incPanel,
            g.incLocal, reinterpret_cast<const double2 *>(flux), g.rowScale, g.T, g.N, E,
            reinterpret_cast<double2 *>(rhsNear), error);
        cudaCheck(cudaGetLastError(), "near rhs launch");
    }
}

}  // namespace hsb
