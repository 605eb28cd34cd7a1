// Interaction planning on the GPU: pair classification and the adaptive
// largest-error refinement of tensor-rule near pairs, one warp per pair
// (interaction_plan.cpp:156-504, pair_quadrature.cpp:143-226, 329-575,
// 644-683). See plan_device.hpp for how the plan stays bit-identical to the
// host planner's.
//
// This file is compiled with -fmad=false: the geometric decisions
// (qualification, near and projection tests, diameters, halving) and the
// sample points repeat the host planner's IEEE operations exactly. Only the
// moment sums use explicit fma(), and their rounding is covered by the bounds
// below.
#include "plan_device.hpp"
#include "device_once.hpp"
#include "planner_geom.cuh"

#include <math.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace hsb {
namespace {

// The pair code is large; letting the compiler decide what to inline keeps the
// kernel's instruction footprint small (a force-inlined build stalled on
// instruction fetch).
#if defined(__CUDACC__)
#define PD_HD __host__ __device__
#define PD_NOINLINE __noinline__
#else
#define PD_HD
#define PD_NOINLINE
#endif

constexpr uint32_t kLeafCap = 2048;  // leaves held per warp (pending + at the depth limit + requested)
constexpr int kRulePoints = 64;      // largest rule (collapsed tensor Gauss degree 14)
constexpr int kPts = 7;              // per point: barycentrics (3), local point (3), weight
constexpr double kUnit = 0x1p-53;    // unit roundoff
// Margin factor on every rounding bound: the bounds below are first-order
// worst cases; a decision is trusted only when its gap is four times larger.
constexpr double kSafety = 4;

enum : uint8_t { kSkip = 0, kOnDevice = 1, kProjected = 2 };
enum : int { kPairRule = 0, kPairWhole = 1, kPairHost = 2 };

// A leaf: its sub-triangles, also as quadtree paths from the whole panels
// (2 bits per halving, child order of quarter()), and its estimate.
struct LeafHdr {
    Sub a, b;
    double error, errB, intB, da, db;
    uint32_t depth, degree, pathA, pathB, depthA, depthB, joins, pad;
};

// A patch as the device writes it: the two quadtree paths, the degree and
// whether its order against the patch before it is left to the host. The host
// rebuilds the barycentric vertices by replaying quarter() along the paths,
// the operations the refinement performed.
struct PatchCode {
    uint32_t pathA, pathB;
    uint8_t depthA, depthB, degree, joins;
};

struct PairRecord {
    uint32_t first, second, patchFirst, count, maxDepth, uncertain;  // uncertain: runs of unknown order
    double relError;
};

struct RuleTables {
    const double *pts[4];  // (b0, b1, b2, w) rows of the degree 6, 8, 12 and 14 rules
    int n[4];
};

struct ClassifyParams {
    const HostPanel *panels;
    const Bounds *bounds;
    double k, tol, nearRatio;
    uint32_t regularOrder;
};

struct AdaptiveParams {
    const HostPanel *panels;
    RuleTables rules;
    double k, tol;
    uint32_t maxDepth;
    int allPairs;
};

// One warp's memory: leaf arena, pending and depth-limit lists, point tables.
struct WarpMem {
    LeafHdr *hdr;
    double *integ;  // kLeafCap x 72: each leaf's moments (36 complex)
    uint32_t *pend;
    double *pendErr;
    uint32_t *atl;
    double *pts;   // test and trial point tables, 2 x kRulePoints x kPts
    double *rows;  // one chunk of row items of a moment computation, W x kRowValues
};

struct PairOutput {
    PatchCode *pool;
    unsigned long long poolCap, *poolUsed;
    PairRecord *records;
    unsigned long long *recordCount;
    uint8_t *whole;  // all-pairs mode: unordered pair index -> whole-panel degree
    unsigned long long *samples;  // kernel samples evaluated (both rules of every estimate)
};

// ---- warp policies: the same pair code runs with 32 lanes on the device and
// with one lane on the host (test emulation) ----
struct LaneWarp {
    static constexpr int W = 1;
    HS_HD int lane() const { return 0; }
    HS_HD double max(double x) const { return x; }
    HS_HD bool any(bool x) const { return x; }
    HS_HD double bcast(double x, int) const { return x; }
    HS_HD void sync() const {}
    HS_HD bool leader() const { return true; }
};

#if defined(__CUDACC__)
struct DeviceWarp {
    static constexpr int W = 32;
    __device__ int lane() const { return threadIdx.x & 31; }
    __device__ double max(double x) const {
        for (int o = 16; o; o >>= 1)
            x = fmax(x, __shfl_xor_sync(~0u, x, o));
        return x;
    }
    __device__ bool any(bool x) const { return __any_sync(~0u, x); }
    __device__ double bcast(double x, int src) const { return __shfl_sync(~0u, x, src); }
    __device__ void sync() const { __syncwarp(); }
    __device__ bool leader() const { return lane() == 0; }
};
#endif

// Moment values: 72 (36 complex, index 2 (9c + 3i + j) + re/im, channel c,
// test function i, trial function j) and 4 magnitude sums (values 72..75).
// After a moment computation lane l holds values [128/W l, 128/W (l+1)).
constexpr int kValues = 128;
constexpr int kRowValues = 32;  // per row item: 12 complex inner sums, 4 magnitude sums, its test barycentrics, pad

// Tensor moments of one rule over sub-triangles a (test) and b (trial)
// (the host's tensorMoments). The test barycentrics depend on the test point
// only, so each lane sums one row of trial points (a test point, or a share
// of its trial points when rows are short) into 12 complex inner sums
// In[c][j] = sum_q ker_c w bs_j, kept in `rows`; then the owners of the
// moment values add bt_i In[c][j] over the rows. `own` receives the lane's
// values; `bad` is set for a coincident point.
template <class Wp>
PD_HD PD_NOINLINE void tensorMoments(const Wp &w, const HostPanel &t, const HostPanel &s, const Sub &a, const Sub &b,
                         const double *rule, int n, double k, double scale, double *pts, double *rows, double *own,
                         bool &bad) {
    constexpr int W = Wp::W;
    for (int q = w.lane(); q < n; q += W) {
        const double *x = rule + 4 * q;
        double bt[3] = {0, 0, 0}, bs[3] = {0, 0, 0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                bt[i] += x[j] * a.v[j][i];
                bs[i] += x[j] * b.v[j][i];
            }
        const V3 lt = localPoint(t, bt), ls = localPoint(s, bs);
        double *T = pts + kPts * q, *S = pts + kPts * (kRulePoints + q);
        T[0] = bt[0], T[1] = bt[1], T[2] = bt[2], T[3] = lt.x, T[4] = lt.y, T[5] = lt.z, T[6] = x[3];
        S[0] = bs[0], S[1] = bs[1], S[2] = bs[2], S[3] = ls.x, S[4] = ls.y, S[5] = ls.z, S[6] = x[3];
    }
    w.sync();
    const V3 origin = t.v[0] - s.v[0];
    const double fab = a.fraction * b.fraction;
    const int split = n < W ? W / n : 1, items = n * split;  // lanes per test point
    // Row items in chunks of W (one per lane), so `rows` holds W records; the
    // owners of the moment values add each chunk's records in item order.
    constexpr int own_n = kValues / W;
    const int base = own_n * w.lane();
    double acc[own_n];
    for (int o = 0; o < own_n; ++o)
        acc[o] = 0;
    for (int c0 = 0; c0 < items; c0 += W) {
        const int it = c0 + w.lane();
        if (it < items) {
            const int xi = it / split, h = it - xi * split;
            const double *T = pts + kPts * xi;
            const double tx = T[3], ty = T[4], tz = T[5], tw = T[6] * fab;
            double in[24], m[4] = {0, 0, 0, 0};
#pragma unroll
            for (int v = 0; v < 24; ++v)
                in[v] = 0;
            for (int qi = h; qi < n; qi += split) {
                const double *S = pts + kPts * (kRulePoints + qi);
                const V3 d{origin.x + (tx - S[3]), origin.y + (ty - S[4]), origin.z + (tz - S[5])};
                const double r = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
                if (!(r > 0)) {
                    bad = true;
                    continue;
                }
                double sn, cs;
                sincos(-k * r, &sn, &cs);  // exp(-i k r)
                const double ir = 1 / r, gr = cs * ir, gi = sn * ir, kr = k * r, f = scale * ir * ir;
                const double dr = (-gr + gi * kr) * f, di = (-gr * kr - gi) * f;
                const double wgt = tw * S[6];
                const double kre[4] = {gr, dr * d.x, dr * d.y, dr * d.z};
                const double kim[4] = {gi, di * d.x, di * d.y, di * d.z};
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double wb = wgt * S[j];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        in[2 * (3 * c + j)] = fma(kre[c], wb, in[2 * (3 * c + j)]);
                        in[2 * (3 * c + j) + 1] = fma(kim[c], wb, in[2 * (3 * c + j) + 1]);
                    }
                }
                // magnitude of each channel's terms: |G| = 1/r, |grad G| <= (1 + kr)/r^2
                const double md = wgt * (1 + kr) * f * ir;
                m[0] += wgt * ir;
                m[1] += md * fabs(d.x);
                m[2] += md * fabs(d.y);
                m[3] += md * fabs(d.z);
            }
            double *R = rows + kRowValues * (it - c0);
#pragma unroll
            for (int v = 0; v < 24; ++v)
                R[v] = in[v];
            R[24] = m[0], R[25] = m[1], R[26] = m[2], R[27] = m[3];
            R[28] = T[0], R[29] = T[1], R[30] = T[2];
        }
        w.sync();
        const int chunk = items - c0 < W ? items - c0 : W;
        for (int o = 0; o < own_n; ++o) {
            const int v = base + o;
            if (v < 72) {
                const int comp = v >> 1, ri = v & 1, c = comp / 9, i = (comp % 9) / 3, j = comp % 3;
                const int col = 2 * (3 * c + j) + ri;
                for (int q = 0; q < chunk; ++q)
                    acc[o] = fma(rows[kRowValues * q + 28 + i], rows[kRowValues * q + col], acc[o]);
            } else if (v < 76) {
                for (int q = 0; q < chunk; ++q)
                    acc[o] += rows[kRowValues * q + 24 + (v - 72)];
            }
        }
        w.sync();
    }
    for (int o = 0; o < own_n; ++o)
        own[o] = acc[o];
    w.sync();  // the point tables and rows are rewritten by the next call
}

// Embedded-rule estimate of one leaf (the host's estimate(), tensor form):
// moments of the lower and higher rule, error = max |hi - lo|. Also the
// bounds on how far the device values can lie from the host's:
//   per moment value, |device - host| <= (2 m + 64) u A_c for a rule of m
//   samples, A_c the sum of |terms| of channel c (both sides' summation
//   errors, at most m u A_c each, and kernel values within 32 u);
//   errB bounds |error_device - error_host|, intB a moment value.
template <class Wp>
PD_HD void estimateLeaf(const Wp &w, const HostPanel &t, const HostPanel &s, const LeafHdr &L, const RuleTables &R,
                        double k, double scale, double *pts, double *rows, double *hiOwn, double &error,
                        double &errB,
                        double &intB, double &mnL, bool &bad) {
    constexpr int own_n = kValues / Wp::W;
    const int lo = L.degree == 8 ? 0 : 2, hi = lo + 1;
    double loOwn[own_n];
    // L lives in the warp's arena: its sub-triangles are read where the point
    // tables are built and hold no registers during the sample loops
    tensorMoments(w, t, s, L.a, L.b, R.pts[lo], R.n[lo], k, scale, pts, rows, loOwn, bad);
    tensorMoments(w, t, s, L.a, L.b, R.pts[hi], R.n[hi], k, scale, pts, rows, hiOwn, bad);
    // magnitude sums live in values 72..75
    const int magLane = 72 / own_n, magOff = 72 - magLane * own_n;
    double Elo = 0, Ehi = 0;
    for (int c = 0; c < 4; ++c) {
        const double al = w.bcast(loOwn[(magOff + c) % own_n], magLane);
        const double ah = w.bcast(hiOwn[(magOff + c) % own_n], magLane);
        const double ml = double(R.n[lo]) * R.n[lo], mh = double(R.n[hi]) * R.n[hi];
        Elo = fmax(Elo, (2 * ml + 64) * kUnit * al);
        Ehi = fmax(Ehi, (2 * mh + 64) * kUnit * ah);
    }
    double dmax = 0, hmax = 0;
    bool nonFinite = false;
    const int base = own_n * w.lane();
    for (int v = 0; v < own_n; v += 2) {
        if (base + v >= 72)
            break;
        const double dr = hiOwn[v] - loOwn[v], di = hiOwn[v + 1] - loOwn[v + 1];
        const double dab = hypot(dr, di), hab = hypot(hiOwn[v], hiOwn[v + 1]);
        nonFinite = nonFinite || !isfinite(dab) || !isfinite(hab);
        dmax = fmax(dmax, dab);
        hmax = fmax(hmax, hab);
    }
    bad = w.any(bad || nonFinite);
    error = w.max(dmax);
    mnL = w.max(hmax);
    errB = 1.4142135623730951 * (Ehi + Elo) + 8 * kUnit * error;
    intB = Ehi;
}

HS_HD bool separated(double x, double y, double bound) { return fabs(x - y) > kSafety * bound; }

// Top two pending errors: (largest, its list position, second largest, its position).
struct Top2 {
    double e1, e2;
    uint32_t p1, p2;
};
template <class Wp> PD_HD Top2 topTwo(const Wp &w, const double *err, uint32_t n) {
    Top2 t{-1, -1, 0xffffffffu, 0xffffffffu};
    for (uint32_t i = w.lane(); i < n; i += Wp::W) {
        const double e = err[i];
        if (e > t.e1) {
            t.e2 = t.e1, t.p2 = t.p1;
            t.e1 = e, t.p1 = i;
        } else if (e > t.e2) {
            t.e2 = e, t.p2 = i;
        }
    }
    if (Wp::W > 1)
        for (int o = 1; o < Wp::W; o <<= 1) {
            Top2 u;
#if defined(__CUDA_ARCH__)
            u.e1 = __shfl_xor_sync(~0u, t.e1, o);
            u.e2 = __shfl_xor_sync(~0u, t.e2, o);
            u.p1 = __shfl_xor_sync(~0u, t.p1, o);
            u.p2 = __shfl_xor_sync(~0u, t.p2, o);
#else
            u = t;
#endif
            // merge, ties to the lower position so every lane agrees
            const bool firstMine = t.e1 > u.e1 || (t.e1 == u.e1 && t.p1 < u.p1);
            Top2 m;
            if (firstMine) {
                m.e1 = t.e1, m.p1 = t.p1;
                const bool sMine = t.e2 > u.e1 || (t.e2 == u.e1 && t.p2 < u.p1);
                m.e2 = sMine ? t.e2 : u.e1;
                m.p2 = sMine ? t.p2 : u.p1;
            } else {
                m.e1 = u.e1, m.p1 = u.p1;
                const bool sMine = t.e1 > u.e2 || (t.e1 == u.e2 && t.p1 < u.p2);
                m.e2 = sMine ? t.e1 : u.e2;
                m.p2 = sMine ? t.p1 : u.p2;
            }
            t = m;
        }
    return t;
}

PD_HD PD_NOINLINE void writeLeaf(LeafHdr &h, const Sub &a, const Sub &b, const HostPanel &t, const HostPanel &s, uint32_t depth,
                     uint32_t degree, uint32_t pathA, uint32_t depthA, uint32_t pathB, uint32_t depthB) {
    h.a = a;
    h.b = b;
    h.da = subDiameter(t, a, t.v[0]);
    h.db = subDiameter(s, b, t.v[0]);
    h.depth = depth;
    h.degree = degree;
    h.pathA = pathA;
    h.pathB = pathB;
    h.depthA = depthA;
    h.depthB = depthB;
    h.error = h.errB = h.intB = 0;
    h.joins = h.pad = 0;
}

// The four children of leaf slots[0] (halving its test side when splitTest,
// else its trial side), written to slots[3], slots[2], slots[1] and last
// slots[0], the parent's own slot. One lane.
PD_HD PD_NOINLINE void spawnChildren(LeafHdr *hdr, const uint32_t *slots, const HostPanel &t, const HostPanel &s,
                                     bool splitTest) {
    const LeafHdr &v = hdr[slots[0]];
    const Sub parent = splitTest ? v.a : v.b;
    const uint32_t depth = v.depth, pathA = v.pathA, pathB = v.pathB, depthA = v.depthA, depthB = v.depthB;
    for (int c = 3; c >= 0; --c) {
        Sub child;
        quarterChild(parent, c, child);
        LeafHdr &h = hdr[slots[c]];
        if (splitTest)
            writeLeaf(h, child, v.b, t, s, depth + 1, 8, pathA | (uint32_t(c) << (2 * depthA)), depthA + 1, pathB,
                      depthB);
        else
            writeLeaf(h, v.a, child, t, s, depth + 1, 8, pathA, depthA, pathB | (uint32_t(c) << (2 * depthB)),
                      depthB + 1);
    }
}

// The largest-error refinement of one tensor pair (the host's adaptivePair
// without projection), with every decision checked against the rounding
// bounds. Returns kPairRule (patches written to the pool, record appended),
// kPairWhole (all-pairs mode single whole-panel rule, degree in `whole`) or
// kPairHost (the host planner must refine this pair).
template <class Wp>
PD_HD int refinePair(const Wp &w, uint32_t ti, uint32_t si, const AdaptiveParams &P, const WarpMem &M,
                     const PairOutput &O, unsigned long long &samples) {
    constexpr int own_n = kValues / Wp::W;
    const HostPanel &t = P.panels[ti], &s = P.panels[si];
    const double scale = maxD(t.maxEdge, s.maxEdge);
    const bool promoteRoot = !isNearPair(t, s, 1.0);
    const int base = own_n * w.lane();
    double integral[own_n];
    for (int v = 0; v < own_n; ++v)
        integral[v] = 0;
    double absError = 0, absB = 0, intB = 0;
    uint32_t nLeaf = 0, nPend = 0, nAtl = 0;
    uint32_t req[4];
    int nReq = 0;
    if (w.leader())
        writeLeaf(M.hdr[0], wholeSub(), wholeSub(), t, s, 0, 8, 0, 0, 0, 0);
    w.sync();
    req[nReq++] = nLeaf++;
    for (;;) {
        for (int r = 0; r < nReq; ++r) {
            const LeafHdr &L = M.hdr[req[r]];
            {
                const int lo = L.degree == 8 ? 0 : 2;
                samples += (unsigned long long)(P.rules.n[lo]) * P.rules.n[lo] +
                           (unsigned long long)(P.rules.n[lo + 1]) * P.rules.n[lo + 1];
            }
            double hiOwn[own_n], error = 0, errB = 0, leafIntB = 0, mnL = 0;
            bool bad = false;
            estimateLeaf(w, t, s, L, P.rules, P.k, scale, M.pts, M.rows, hiOwn, error, errB, leafIntB, mnL, bad);
            if (bad)
                return kPairHost;
            for (int v = 0; v < own_n && base + v < 72; ++v)
                M.integ[size_t(req[r]) * 72 + base + v] = hiOwn[v];
            w.sync();
            if (w.leader()) {
                M.hdr[req[r]].error = error;
                M.hdr[req[r]].errB = errB;
                M.hdr[req[r]].intB = leafIntB;
            }
            // running sums, in the host's order
            absError += error;
            absB += errB + 2 * kUnit * absError;
            double mnI = 0;
            for (int v = 0; v < own_n && base + v < 72; v += 2) {
                integral[v] += hiOwn[v];
                integral[v + 1] += hiOwn[v + 1];
                mnI = fmax(mnI, hypot(integral[v], integral[v + 1]));
            }
            mnI = w.max(mnI);
            intB += leafIntB + 2 * kUnit * (mnI + mnL);
            w.sync();
            const bool outerLimit = L.depth == P.maxDepth && L.degree == 14;
            if (outerLimit) {
                if (w.leader())
                    M.atl[nAtl] = req[r];
                ++nAtl;
            } else {
                if (w.leader()) {
                    M.pend[nPend] = req[r];
                    M.pendErr[nPend] = error;
                }
                ++nPend;
            }
            w.sync();
        }
        nReq = 0;
        double mn = 0;
        bool nonFinite = false;
        for (int v = 0; v < own_n && base + v < 72; v += 2) {
            const double m = hypot(integral[v], integral[v + 1]);
            nonFinite = nonFinite || !isfinite(m);
            mn = fmax(mn, m);
        }
        if (w.any(nonFinite))
            return kPairHost;
        mn = w.max(mn);
        const double thr = P.tol * .2 * mn;
        const double mnB = 1.4142135623730951 * intB + 3 * kUnit * mn;
        const double thrB = P.tol * .2 * mnB + 2 * kUnit * thr;
        if (!separated(absError, thr, absB + thrB))
            return kPairHost;
        if (absError <= thr) {
            // patches at the depth limit in insertion order, then the pending
            // leaves by decreasing error (distinct beyond their bounds)
            if (!(mn > 0))
                return kPairHost;
            const double relError = absError / mn;
            if (!isfinite(relError) || relError > P.tol)
                return kPairHost;
            const uint32_t count = nAtl + nPend;
            // Descending device errors. Each host error lies within kSafety
            // errB of the device's; where those intervals overlap (a run of
            // leaves whose order the device cannot know), the leaves after the
            // first are marked and the host orders the run by its own
            // estimates. Runs never overlap one another, so the order between
            // runs is the host's.
            double runLow = INFINITY;
            for (uint32_t k = 0; k < nPend; ++k) {
                const Top2 top = topTwo(w, M.pendErr, nPend);
                const double B = kSafety * M.hdr[M.pend[top.p1]].errB;
                const bool joins = top.e1 + B >= runLow;
                runLow = joins ? fmin(runLow, top.e1 - B) : top.e1 - B;
                w.sync();
                if (w.leader()) {
                    M.atl[nAtl + k] = M.pend[top.p1];
                    M.pendErr[top.p1] = -1;  // removed
                    M.hdr[M.pend[top.p1]].joins = joins ? 1 : 0;
                }
                w.sync();
            }
            uint32_t maxDepth = 0, degree0 = 0;
            for (uint32_t k = 0; k < count; ++k) {
                const LeafHdr &h = M.hdr[M.atl[k]];
                maxDepth = h.depth > maxDepth ? h.depth : maxDepth;
                degree0 = k == 0 ? h.degree : degree0;
            }
            uint32_t uncertain = 0;
            for (uint32_t k = nAtl; k < count; ++k)
                uncertain |= M.hdr[M.atl[k]].joins;
            if (P.allPairs && maxDepth == 0 && count == 1) {
                if (w.leader())
                    O.whole[unorderedPairIndex(ti, si)] = uint8_t(degree0);
                return kPairWhole;
            }
            unsigned long long first = 0;
#if defined(__CUDA_ARCH__)
            if (w.leader())
                first = atomicAdd(O.poolUsed, (unsigned long long)count);
            first = __shfl_sync(~0u, first, 0);
#else
            first = __atomic_fetch_add(O.poolUsed, (unsigned long long)count, __ATOMIC_RELAXED);
#endif
            if (first + count > O.poolCap)
                return kPairHost;
            for (uint32_t k = w.lane(); k < count; k += Wp::W) {
                const LeafHdr &h = M.hdr[M.atl[k]];
                // joins: the order against the patch before it is the host's to settle
                O.pool[first + k] = PatchCode{h.pathA, h.pathB, uint8_t(h.depthA), uint8_t(h.depthB),
                                              uint8_t(h.degree), uint8_t(k >= nAtl && h.joins ? 1 : 0)};
            }
            if (w.leader()) {
                unsigned long long slot;
#if defined(__CUDA_ARCH__)
                slot = atomicAdd(O.recordCount, 1ull);
#else
                slot = __atomic_fetch_add(O.recordCount, 1ull, __ATOMIC_RELAXED);
#endif
                O.records[slot] = PairRecord{ti, si, uint32_t(first), count, maxDepth, uncertain, relError};
            }
            return kPairRule;
        }
        if (nPend == 0)
            return kPairHost;
        const Top2 top = topTwo(w, M.pendErr, nPend);
        const uint32_t vSlot = M.pend[top.p1];
        const LeafHdr &vh = M.hdr[vSlot];  // v stays in the arena; its slot goes to its first child
        const double vError = vh.error, vErrB = vh.errB, vIntB = vh.intB;
        const uint32_t vDepth = vh.depth, vDegree = vh.degree;
        const bool splitTest = vh.da >= vh.db;
        if (top.p2 != 0xffffffffu && !separated(top.e1, top.e2, vErrB + M.hdr[M.pend[top.p2]].errB))
            return kPairHost;
        w.sync();
        if (w.leader()) {  // remove v: the last pending entry takes its place
            M.pend[top.p1] = M.pend[nPend - 1];
            M.pendErr[top.p1] = M.pendErr[nPend - 1];
        }
        --nPend;
        absError = maxD(0.0, absError - vError);
        absB += vErrB + 2 * kUnit * (absError + vError);
        double mnI = 0;
        for (int v2 = 0; v2 < own_n && base + v2 < 72; v2 += 2) {
            integral[v2] -= M.integ[size_t(vSlot) * 72 + base + v2];
            integral[v2 + 1] -= M.integ[size_t(vSlot) * 72 + base + v2 + 1];
            mnI = fmax(mnI, hypot(integral[v2], integral[v2 + 1]));
        }
        mnI = w.max(mnI);
        intB += vIntB + 2 * kUnit * mnI * 2;
        w.sync();
        if (vDegree == 8 && (vDepth == P.maxDepth || (promoteRoot && vDepth == 0))) {
            if (w.leader())
                M.hdr[vSlot].degree = 14;  // same patch, the degree 12/14 pair of rules
            req[nReq++] = vSlot;
        } else {
            if (nPend + nAtl + 4 > 50000 || nLeaf + 3 > kLeafCap)
                return kPairHost;
            const uint32_t slots[4] = {vSlot, nLeaf, nLeaf + 1, nLeaf + 2};
            nLeaf += 3;
            if (w.leader())
                spawnChildren(M.hdr, slots, t, s, splitTest);
            for (int c = 0; c < 4; ++c)
                req[nReq++] = slots[c];
        }
        w.sync();
    }
}

// ---- root pre-pass (all-pairs mode) ----
// Most pairs of the all-pairs table end at their root estimate (the whole-panel
// degree-8 rule). Four lanes take one pair, lane c summing kernel channel c of
// both rules in registers; the first decision of the refinement, with the same
// bounds as refinePair, settles the pair when it clearly converges at the root.
// Every other pair goes on to refineKernel.
struct RootChannel {
    double dmax, hmax, Elo, Ehi;
    bool bad;
};

// Channel c (0: G, 1..3: the gradient components) of the root leaf's two rules.
PD_HD RootChannel rootChannel(const HostPanel &t, const HostPanel &s, int c, const RuleTables &R, double k,
                              double scale) {
    const V3 origin = t.v[0] - s.v[0];
    double hi[18], lo[18], A[2] = {0, 0};
    bool bad = false;
    for (int rr = 1; rr >= 0; --rr) {  // the degree 8 rule, then the degree 6 rule
        const double *rule = R.pts[rr];
        const int n = R.n[rr];
        double *m = rr == 1 ? hi : lo;
        for (int v = 0; v < 18; ++v)
            m[v] = 0;
        for (int x = 0; x < n; ++x) {
            // whole test panel: the rule's barycentrics are the point's
            const double bt[3] = {rule[4 * x], rule[4 * x + 1], rule[4 * x + 2]}, wx = rule[4 * x + 3];
            const V3 lt = localPoint(t, bt);
            double in[6] = {0, 0, 0, 0, 0, 0};
            for (int q = 0; q < n; ++q) {
                const double bs[3] = {rule[4 * q], rule[4 * q + 1], rule[4 * q + 2]};
                const V3 ls = localPoint(s, bs);
                const V3 d{origin.x + (lt.x - ls.x), origin.y + (lt.y - ls.y), origin.z + (lt.z - ls.z)};
                const double r = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
                if (!(r > 0)) {
                    bad = true;
                    continue;
                }
                double sn, cs;
                sincos(-k * r, &sn, &cs);
                const double ir = 1 / r, gr = cs * ir, gi = sn * ir, kr = k * r, f = scale * ir * ir;
                const double wgt = wx * rule[4 * q + 3];
                double vr, vi, mag;
                if (c == 0) {
                    vr = gr, vi = gi, mag = ir;
                } else {
                    const double dc = c == 1 ? d.x : c == 2 ? d.y : d.z;
                    vr = (-gr + gi * kr) * f * dc;
                    vi = (-gr * kr - gi) * f * dc;
                    mag = (1 + kr) * f * ir * fabs(dc);
                }
                A[rr] += wgt * mag;
                for (int j = 0; j < 3; ++j) {
                    in[2 * j] = fma(vr * wgt, bs[j], in[2 * j]);
                    in[2 * j + 1] = fma(vi * wgt, bs[j], in[2 * j + 1]);
                }
            }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    m[2 * (3 * i + j)] = fma(bt[i], in[2 * j], m[2 * (3 * i + j)]);
                    m[2 * (3 * i + j) + 1] = fma(bt[i], in[2 * j + 1], m[2 * (3 * i + j) + 1]);
                }
        }
    }
    RootChannel out{0, 0, 0, 0, bad};
    for (int v = 0; v < 18; v += 2) {
        const double dab = hypot(hi[v] - lo[v], hi[v + 1] - lo[v + 1]), hab = hypot(hi[v], hi[v + 1]);
        out.bad = out.bad || !isfinite(dab) || !isfinite(hab);
        out.dmax = fmax(out.dmax, dab);
        out.hmax = fmax(out.hmax, hab);
    }
    const double ml = double(R.n[0]) * R.n[0], mh = double(R.n[1]) * R.n[1];
    out.Elo = (2 * ml + 64) * kUnit * A[0];
    out.Ehi = (2 * mh + 64) * kUnit * A[1];
    return out;
}

#if defined(__CUDACC__)
// rootChannel with the kernel evaluations shared by the pair's four lanes:
// lane c evaluates every fourth trial point for all four channels, and a 4 x 4
// shuffle transpose hands each lane its own channel of the four points.
__device__ RootChannel rootChannelQuad(const HostPanel &t, const HostPanel &s, int c, bool active,
                                       const RuleTables &R, double k, double scale) {
    const V3 origin = t.v[0] - s.v[0];
    double hi[18], lo[18], A[2] = {0, 0};
    bool bad = false;
    for (int rr = 1; rr >= 0; --rr) {
        const double *rule = R.pts[rr];
        const int n = R.n[rr];
        double *m = rr == 1 ? hi : lo;
        for (int v = 0; v < 18; ++v)
            m[v] = 0;
        for (int x = 0; x < n; ++x) {
            const double bt[3] = {rule[4 * x], rule[4 * x + 1], rule[4 * x + 2]}, wx = rule[4 * x + 3];
            const V3 lt = localPoint(t, bt);
            double in[6] = {0, 0, 0, 0, 0, 0};
            for (int q0 = 0; q0 < n; q0 += 4) {
                // this lane's point: all four channels (value times weight, magnitude times weight)
                const int q = q0 + c;
                double vr[4] = {0, 0, 0, 0}, vi[4] = {0, 0, 0, 0}, mg[4] = {0, 0, 0, 0};
                if (active && q < n) {
                    const double bs[3] = {rule[4 * q], rule[4 * q + 1], rule[4 * q + 2]};
                    const V3 ls = localPoint(s, bs);
                    const V3 d{origin.x + (lt.x - ls.x), origin.y + (lt.y - ls.y), origin.z + (lt.z - ls.z)};
                    const double r = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
                    if (!(r > 0)) {
                        bad = true;
                    } else {
                        double sn, cs;
                        sincos(-k * r, &sn, &cs);
                        const double ir = 1 / r, gr = cs * ir, gi = sn * ir, kr = k * r, f = scale * ir * ir;
                        const double wgt = wx * rule[4 * q + 3];
                        const double dr = (-gr + gi * kr) * f, di = (-gr * kr - gi) * f, md = (1 + kr) * f * ir;
                        vr[0] = gr * wgt, vi[0] = gi * wgt, mg[0] = ir * wgt;
                        const double dd[3] = {d.x, d.y, d.z};
#pragma unroll
                        for (int ch = 1; ch < 4; ++ch) {
                            vr[ch] = dr * dd[ch - 1] * wgt;
                            vi[ch] = di * dd[ch - 1] * wgt;
                            mg[ch] = md * fabs(dd[ch - 1]) * wgt;
                        }
                    }
                }
                // transpose: in round o, lane c receives point q0 + (c ^ o)'s channel c
#pragma unroll
                for (int o = 0; o < 4; ++o) {
                    const int send = c ^ o;  // the channel the partner lane needs
                    const double sr = send == 0 ? vr[0] : send == 1 ? vr[1] : send == 2 ? vr[2] : vr[3];
                    const double si = send == 0 ? vi[0] : send == 1 ? vi[1] : send == 2 ? vi[2] : vi[3];
                    const double sm = send == 0 ? mg[0] : send == 1 ? mg[1] : send == 2 ? mg[2] : mg[3];
                    const double gotr = __shfl_xor_sync(~0u, sr, o), goti = __shfl_xor_sync(~0u, si, o),
                                 gotm = __shfl_xor_sync(~0u, sm, o);
                    const int qq = q0 + (c ^ o);
                    if (qq < n) {
                        const double bs[3] = {rule[4 * qq], rule[4 * qq + 1], rule[4 * qq + 2]};
                        A[rr] += gotm;
                        for (int j = 0; j < 3; ++j) {
                            in[2 * j] = fma(gotr, bs[j], in[2 * j]);
                            in[2 * j + 1] = fma(goti, bs[j], in[2 * j + 1]);
                        }
                    }
                }
            }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    m[2 * (3 * i + j)] = fma(bt[i], in[2 * j], m[2 * (3 * i + j)]);
                    m[2 * (3 * i + j) + 1] = fma(bt[i], in[2 * j + 1], m[2 * (3 * i + j) + 1]);
                }
        }
    }
    RootChannel out{0, 0, 0, 0, bad};
    for (int v = 0; v < 18; v += 2) {
        const double dab = hypot(hi[v] - lo[v], hi[v + 1] - lo[v + 1]), hab = hypot(hi[v], hi[v + 1]);
        out.bad = out.bad || !isfinite(dab) || !isfinite(hab);
        out.dmax = fmax(out.dmax, dab);
        out.hmax = fmax(out.hmax, hab);
    }
    const double ml = double(R.n[0]) * R.n[0], mh = double(R.n[1]) * R.n[1];
    out.Elo = (2 * ml + 64) * kUnit * A[0];
    out.Ehi = (2 * mh + 64) * kUnit * A[1];
    return out;
}
#endif

// The refinement's first decision from the channels' maxima (refinePair's
// formulas for a single root leaf): 8 when the root clearly converges (the
// pair's rule is the whole-panel degree-8 patch), 0 when the pair must be
// refined further or its decision is too close to call.
PD_HD uint8_t rootDecision(double error, double mn, double Elo, double Ehi, bool bad, double tol) {
    if (bad)
        return 0;
    const double errB = 1.4142135623730951 * (Ehi + Elo) + 8 * kUnit * error;
    const double absError = error, absB = errB + 2 * kUnit * absError;
    const double intB = Ehi + 2 * kUnit * (mn + mn);
    const double thr = tol * .2 * mn;
    const double mnB = 1.4142135623730951 * intB + 3 * kUnit * mn;
    const double thrB = tol * .2 * mnB + 2 * kUnit * thr;
    if (!separated(absError, thr, absB + thrB) || !(absError <= thr) || !(mn > 0))
        return 0;
    const double relError = absError / mn;
    return isfinite(relError) && relError <= tol ? 8 : 0;
}

// Pair classification (the host's processPair test): 0 no adaptive rule,
// kOnDevice a tensor pair, kProjected a pair on projected patches.
HS_HD uint8_t classifyPair(const ClassifyParams &P, uint32_t i, uint32_t j) {
    const HostPanel &a = P.panels[i], &b = P.panels[j];
    if (!panelsDisjoint(a, b))
        return kSkip;
    const unsigned degree = qualifiedDegree(P.bounds[i], P.bounds[j], P.k, P.tol, P.regularOrder);
    const double h = maxD(a.maxEdge, b.maxEdge);
    const double limit = P.bounds[i].radius + P.bounds[j].radius + P.nearRatio * h;
    const double dx = a.centroid.x - b.centroid.x, dy = a.centroid.y - b.centroid.y, dz = a.centroid.z - b.centroid.z;
    const bool geometricNear =
        degree && P.nearRatio > 0 && dx * dx + dy * dy + dz * dz < limit * limit && isNearPair(a, b, P.nearRatio);
    if (degree && !geometricNear)
        return kSkip;
    return useProjection(a, b, maxD(a.maxEdge, b.maxEdge)) ? kProjected : kOnDevice;
}

// Unordered pair index u = j (j - 1) / 2 + i, i < j (interaction_plan.hpp:19-22), inverted.
HS_HD void pairOfIndex(unsigned long long u, uint32_t &i, uint32_t &j) {
    unsigned long long jj = (unsigned long long)((1 + sqrt(1 + 8.0 * double(u))) / 2);
    while (jj * (jj - 1) / 2 > u)
        --jj;
    while ((jj + 1) * jj / 2 <= u)
        ++jj;
    j = uint32_t(jj);
    i = uint32_t(u - jj * (jj - 1) / 2);
}

#if defined(__CUDACC__)
// Two passes: with null lists only the counts are taken, then the lists are
// filled (their order is irrelevant: results are keyed by pair). Appends are
// aggregated per warp.
__global__ void classifyKernel(ClassifyParams P, const uint2 *candidates, unsigned long long count, int allPairs,
                               uint2 *deviceList, unsigned long long *deviceCount, uint2 *hostList,
                               unsigned long long *hostCount) {
    const int lane = threadIdx.x & 31;
    const unsigned long long warp = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
    const unsigned long long warps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long b = warp * 32; b < count; b += warps * 32) {
        const unsigned long long p = b + lane;
        uint8_t c = kSkip;
        uint32_t i = 0, j = 0;
        if (p < count) {
            if (allPairs) {
                pairOfIndex(p, i, j);
            } else {
                i = candidates[p].x;
                j = candidates[p].y;
            }
            c = classifyPair(P, i, j);
        }
        const unsigned md = __ballot_sync(~0u, c == kOnDevice), mh = __ballot_sync(~0u, c == kProjected);
        unsigned long long bd = 0, bh = 0;
        if (lane == 0) {
            if (md)
                bd = atomicAdd(deviceCount, (unsigned long long)__popc(md));
            if (mh)
                bh = atomicAdd(hostCount, (unsigned long long)__popc(mh));
        }
        bd = __shfl_sync(~0u, bd, 0);
        bh = __shfl_sync(~0u, bh, 0);
        const unsigned below = (1u << lane) - 1;
        if (c == kOnDevice && deviceList)
            deviceList[bd + __popc(md & below)] = make_uint2(i, j);
        if (c == kProjected && hostList)
            hostList[bh + __popc(mh & below)] = make_uint2(i, j);
    }
}

constexpr int kRootThreads = 128;

// Four lanes per pair; lane c sums channel c. A settled pair writes its
// whole-panel degree, the others are appended to `rest` for refineKernel.
__global__ void __launch_bounds__(kRootThreads) rootKernel(AdaptiveParams P, const uint2 *list,
                                                           unsigned long long count, uint8_t *whole, uint2 *rest,
                                                           unsigned long long *restCount) {
    const unsigned long long g = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    const unsigned long long p = g >> 2;
    const int c = int(g & 3);
    const bool active = p < count;
    // pairs beyond the list run pair 0's geometry inactive, so every lane joins the shuffles
    const uint2 pr = list[active ? p : 0];
    const HostPanel &t = P.panels[pr.x], &s = P.panels[pr.y];
    RootChannel ch = rootChannelQuad(t, s, c, active, P.rules, P.k, maxD(t.maxEdge, s.maxEdge));
    if (!active)
        ch = RootChannel{0, 0, 0, 0, false};
    for (int o = 1; o <= 2; o <<= 1) {  // maxima over the pair's four lanes
        ch.dmax = fmax(ch.dmax, __shfl_xor_sync(~0u, ch.dmax, o));
        ch.hmax = fmax(ch.hmax, __shfl_xor_sync(~0u, ch.hmax, o));
        ch.Elo = fmax(ch.Elo, __shfl_xor_sync(~0u, ch.Elo, o));
        ch.Ehi = fmax(ch.Ehi, __shfl_xor_sync(~0u, ch.Ehi, o));
        ch.bad = ch.bad || __shfl_xor_sync(~0u, int(ch.bad), o) != 0;
    }
    if (!active || c != 0)
        return;
    const uint8_t degree = rootDecision(ch.dmax, ch.hmax, ch.Elo, ch.Ehi, ch.bad, P.tol);
    if (degree)
        whole[unorderedPairIndex(pr.x, pr.y)] = degree;
    else
        rest[atomicAdd(restCount, 1ull)] = pr;
}

constexpr int kWarpsPerBlock = 4;

constexpr int kWarpSmemDoubles = 2 * kRulePoints * kPts + 32 * kRowValues;
constexpr size_t kRefineSmem = sizeof(double) * kWarpSmemDoubles * kWarpsPerBlock;

__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3) refineKernel(AdaptiveParams P, const uint2 *list,
                                                                     unsigned long long count,
                                                                     unsigned long long *next, WarpMem arena,
                                                                     PairOutput O, uint2 *flagged,
                                                                     unsigned long long *flagCount) {
    extern __shared__ double smem[];
    const DeviceWarp w;
    const int wInBlock = threadIdx.x >> 5;
    const size_t warpId = size_t(blockIdx.x) * kWarpsPerBlock + wInBlock;
    WarpMem M;
    M.hdr = arena.hdr + warpId * kLeafCap;
    M.integ = arena.integ + warpId * kLeafCap * 72;
    M.pend = arena.pend + warpId * kLeafCap;
    M.pendErr = arena.pendErr + warpId * kLeafCap;
    M.atl = arena.atl + warpId * kLeafCap;
    M.pts = smem + size_t(kWarpSmemDoubles) * wInBlock;
    M.rows = M.pts + 2 * kRulePoints * kPts;
    unsigned long long samples = 0;
    for (;;) {
        unsigned long long p = 0;
        if (w.leader())
            p = atomicAdd(next, 1ull);
        p = __shfl_sync(~0u, p, 0);
        if (p >= count)
            break;
        const uint2 pr = list[p];
        const int r = refinePair(w, pr.x, pr.y, P, M, O, samples);
        if (r == kPairHost && w.leader())
            flagged[atomicAdd(flagCount, 1ull)] = pr;
        __syncwarp();
    }
    if (w.leader())
        atomicAdd(O.samples, samples);
}
#endif

void check(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        throw OutOfMemory(std::string(what) + ": " + cudaGetErrorString(e));
    if (e != cudaSuccess)
        throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// The sub-triangle at the end of a quadtree path (2 bits per level, child
// order of quarter()), by the halvings the refinement performed.
Sub subOfPath(uint32_t path, uint32_t depth) {
    Sub cur = wholeSub(), next;
    for (uint32_t l = 0; l < depth; ++l) {
        quarterChild(cur, int((path >> (2 * l)) & 3), next);
        cur = next;
    }
    return cur;
}

struct DevMem {
    void *p = nullptr;
    DevMem() = default;
    explicit DevMem(size_t bytes) { alloc(bytes); }
    void alloc(size_t bytes) { check(cudaMalloc(&p, bytes ? bytes : 16), "planner allocation"); }
    DevMem(const DevMem &) = delete;
    DevMem &operator=(const DevMem &) = delete;
    ~DevMem() {
        if (p)
            cudaFree(p);
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

std::vector<double> ruleRows(unsigned degree) {
    const auto rule = triangleRule(degree);
    std::vector<double> rows;
    for (const auto &p : rule) {
        rows.push_back(p.b[0]);
        rows.push_back(p.b[1]);
        rows.push_back(p.b[2]);
        rows.push_back(p.w);
    }
    if (rule.size() > size_t(kRulePoints))
        throw std::logic_error("triangle rule larger than the device planner's point table");
    return rows;
}

using Clock = std::chrono::steady_clock;
double msSince(Clock::time_point t0) { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

}  // namespace

Plan makePlanOnDevice(const Space &sp, const PlanSettings &st, double maxK, cudaStream_t stream,
                      const volatile int32_t *cancel, DevicePlanStats *stats, bool emulate) {
    const auto t0 = Clock::now();
    PlanFrame f = beginPlan(sp, st, maxK);
    double phase[5] = {msSince(t0), 0, 0, 0, 0};  // frame, classification, refinement, readback, flattening
    const uint32_t T = uint32_t(sp.panels.size());
    const unsigned long long units =
        f.allPairs ? (unsigned long long)T * (T - 1) / 2 : (unsigned long long)f.candidates.size();
    const std::vector<double> rules[4] = {ruleRows(6), ruleRows(8), ruleRows(12), ruleRows(14)};
    std::vector<uint2> deviceList, hostList;
    std::vector<PairRecord> records;
    std::vector<PatchCode> pool;
    std::vector<uint8_t> whole;
    std::vector<uint2> flagged;
    size_t devicePairs = 0;
    unsigned long long sampleTotal = 0, rootSamples = 0;
    size_t rootSettled = 0;
    double refineKernelMs = 0;
    if (cancel && *cancel)
        throw Cancelled();
    if (emulate) {
        // The device algorithm on host threads with one-lane warps.
        ClassifyParams C{sp.panels.data(), f.bounds.data(), maxK, st.tol, st.nearRatio, st.regularOrder};
        for (unsigned long long p = 0; p < units; ++p) {
            uint32_t i, j;
            if (f.allPairs)
                pairOfIndex(p, i, j);
            else
                i = f.candidates[p].first, j = f.candidates[p].second;
            const uint8_t c = classifyPair(C, i, j);
            if (c == kOnDevice)
                deviceList.push_back(make_uint2(i, j));
            else if (c == kProjected)
                hostList.push_back(make_uint2(i, j));
        }
        phase[1] = msSince(t0);
        AdaptiveParams A{sp.panels.data(), {}, maxK, st.tol, st.maxDepth, f.allPairs ? 1 : 0};
        for (int r = 0; r < 4; ++r)
            A.rules.pts[r] = rules[r].data(), A.rules.n[r] = int(rules[r].size() / 4);
        if (f.allPairs)
            whole.assign(units, 0);
        pool.resize(size_t(64) * deviceList.size() + 65536);
        records.resize(deviceList.size());
        unsigned long long poolUsed = 0, recordCount = 0;
        PairOutput O{pool.data(), pool.size(), &poolUsed, records.data(), &recordCount, whole.data(), &sampleTotal};
        const unsigned workers = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<uint2> refineList;  // all-pairs mode: the pairs the root pre-pass leaves
        if (f.allPairs) {
            std::vector<uint8_t> settled(deviceList.size(), 0);
            std::atomic<size_t> nextRoot{0};
            std::vector<std::thread> rootThreads;
            for (unsigned wkr = 0; wkr < workers; ++wkr)
                rootThreads.emplace_back([&]() {
                    for (;;) {
                        const size_t p = nextRoot.fetch_add(1);
                        if (p >= deviceList.size())
                            return;
                        const HostPanel &t = sp.panels[deviceList[p].x], &s = sp.panels[deviceList[p].y];
                        RootChannel m{0, 0, 0, 0, false};
                        for (int c = 0; c < 4; ++c) {
                            const RootChannel ch = rootChannel(t, s, c, A.rules, maxK, maxD(t.maxEdge, s.maxEdge));
                            m.dmax = fmax(m.dmax, ch.dmax);
                            m.hmax = fmax(m.hmax, ch.hmax);
                            m.Elo = fmax(m.Elo, ch.Elo);
                            m.Ehi = fmax(m.Ehi, ch.Ehi);
                            m.bad = m.bad || ch.bad;
                        }
                        const uint8_t degree = rootDecision(m.dmax, m.hmax, m.Elo, m.Ehi, m.bad, A.tol);
                        if (degree) {
                            whole[unorderedPairIndex(deviceList[p].x, deviceList[p].y)] = degree;
                            settled[p] = 1;
                        }
                    }
                });
            for (auto &th : rootThreads)
                th.join();
            for (size_t p = 0; p < deviceList.size(); ++p)
                if (!settled[p])
                    refineList.push_back(deviceList[p]);
            rootSettled = deviceList.size() - refineList.size();
            rootSamples = deviceList.size() * (unsigned long long)(A.rules.n[0] * A.rules.n[0] + A.rules.n[1] * A.rules.n[1]);
        } else {
            refineList = deviceList;
        }
        std::atomic<size_t> next{0};
        std::mutex flagMutex;
        std::vector<std::thread> threads;
        for (unsigned wkr = 0; wkr < workers; ++wkr)
            threads.emplace_back([&]() {
                std::vector<LeafHdr> hdr(kLeafCap);
                std::vector<double> integ(size_t(kLeafCap) * 72), pendErr(kLeafCap), pts(2 * kRulePoints * kPts),
                    rows(size_t(kRulePoints) * kRowValues);
                std::vector<uint32_t> pend(kLeafCap), atl(kLeafCap);
                WarpMem M{hdr.data(), integ.data(), pend.data(), pendErr.data(), atl.data(), pts.data(), rows.data()};
                unsigned long long samples = 0;
                for (;;) {
                    const size_t p = next.fetch_add(1);
                    if (p >= refineList.size())
                        break;
                    if (refinePair(LaneWarp{}, refineList[p].x, refineList[p].y, A, M, O, samples) == kPairHost) {
                        std::lock_guard<std::mutex> lock(flagMutex);
                        flagged.push_back(refineList[p]);
                    }
                }
                __atomic_fetch_add(&sampleTotal, samples, __ATOMIC_RELAXED);
            });
        for (auto &th : threads)
            th.join();
        phase[2] = msSince(t0);
        sampleTotal += rootSamples;
        records.resize(recordCount);
        pool.resize(std::min<size_t>(poolUsed, pool.size()));
        devicePairs = deviceList.size();
    } else {
#if defined(__CUDACC__)
        // geometry and rules
        DevMem dPanels(sizeof(HostPanel) * T), dBounds(sizeof(Bounds) * T);
        check(cudaMemcpyAsync(dPanels.p, sp.panels.data(), sizeof(HostPanel) * T, cudaMemcpyHostToDevice, stream),
              "planner upload");
        check(cudaMemcpyAsync(dBounds.p, f.bounds.data(), sizeof(Bounds) * T, cudaMemcpyHostToDevice, stream),
              "planner upload");
        DevMem dRules[4];
        AdaptiveParams A{dPanels.as<HostPanel>(), {}, maxK, st.tol, st.maxDepth, f.allPairs ? 1 : 0};
        for (int r = 0; r < 4; ++r) {
            dRules[r].alloc(rules[r].size() * sizeof(double));
            check(cudaMemcpyAsync(dRules[r].p, rules[r].data(), rules[r].size() * sizeof(double),
                                  cudaMemcpyHostToDevice, stream),
                  "planner upload");
            A.rules.pts[r] = dRules[r].as<double>();
            A.rules.n[r] = int(rules[r].size() / 4);
        }
        DevMem dCand(f.allPairs ? 16 : sizeof(uint2) * f.candidates.size());
        if (!f.allPairs && !f.candidates.empty()) {
            std::vector<uint2> c(f.candidates.size());
            for (size_t i = 0; i < c.size(); ++i)
                c[i] = make_uint2(f.candidates[i].first, f.candidates[i].second);
            check(cudaMemcpyAsync(dCand.p, c.data(), sizeof(uint2) * c.size(), cudaMemcpyHostToDevice, stream),
                  "planner upload");
            check(cudaStreamSynchronize(stream), "planner upload");
        }
        // classification: counts first, then the lists
        DevMem dCounters(8 * sizeof(unsigned long long));
        unsigned long long *counters = dCounters.as<unsigned long long>();
        check(cudaMemsetAsync(counters, 0, 8 * sizeof(unsigned long long), stream), "planner reset");
        int device = 0, sms = 0;
        check(cudaGetDevice(&device), "device query");
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query");
        ClassifyParams C{dPanels.as<HostPanel>(), dBounds.as<Bounds>(), maxK, st.tol, st.nearRatio, st.regularOrder};
        const unsigned blocks = unsigned(std::max<unsigned long long>(
            1, std::min<unsigned long long>((units + 255) / 256, 16ull * sms)));
        unsigned long long n2[2] = {0, 0};
        if (units) {
            classifyKernel<<<blocks, 256, 0, stream>>>(C, dCand.as<uint2>(), units, f.allPairs ? 1 : 0, nullptr,
                                                       counters, nullptr, counters + 1);
            check(cudaGetLastError(), "planner classification");
            check(cudaMemcpyAsync(n2, counters, sizeof(n2), cudaMemcpyDeviceToHost, stream), "planner readback");
            check(cudaStreamSynchronize(stream), "planner classification");
        }
        const unsigned long long nDevice = n2[0], nHost = n2[1];
        phase[1] = msSince(t0);
        DevMem dDeviceList(sizeof(uint2) * nDevice), dHostList(sizeof(uint2) * nHost);
        if (units) {
            check(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), stream), "planner reset");
            classifyKernel<<<blocks, 256, 0, stream>>>(C, dCand.as<uint2>(), units, f.allPairs ? 1 : 0,
                                                       dDeviceList.as<uint2>(), counters, dHostList.as<uint2>(),
                                                       counters + 1);
            check(cudaGetLastError(), "planner classification");
            check(cudaStreamSynchronize(stream), "planner classification");
        }
        hostList.resize(nHost);
        if (nHost)
            check(cudaMemcpyAsync(hostList.data(), dHostList.p, sizeof(uint2) * nHost, cudaMemcpyDeviceToHost, stream),
                  "planner readback");
        devicePairs = nDevice;
        // refinement: arenas for the resident warps, the patch pool sized by
        // the free memory
        static PerDeviceOnce attributes;
        attributes.run([] {
            check(cudaFuncSetAttribute(refineKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kRefineSmem)),
                  "planner kernel attribute");
        });
        int blocksPerSm = 0;
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocksPerSm, refineKernel, 32 * kWarpsPerBlock,
                                                            kRefineSmem),
              "planner occupancy");
        blocksPerSm = std::max(1, blocksPerSm);
        size_t freeBytes = 0, totalBytes = 0;
        check(cudaMemGetInfo(&freeBytes, &totalBytes), "device memory query");
        const size_t warpBytes = (sizeof(LeafHdr) + 72 * sizeof(double) + 2 * sizeof(uint32_t) + sizeof(double)) *
                                 size_t(kLeafCap);
        size_t grid = size_t(sms) * blocksPerSm;  // resident blocks, fewer when memory is short
        grid = std::max<size_t>(1, std::min(grid, freeBytes / 4 / (warpBytes * kWarpsPerBlock)));
        const size_t warps = grid * kWarpsPerBlock;
        DevMem dHdr(sizeof(LeafHdr) * kLeafCap * warps), dInteg(sizeof(double) * 72 * kLeafCap * warps),
            dPend(sizeof(uint32_t) * kLeafCap * warps), dPendErr(sizeof(double) * kLeafCap * warps),
            dAtl(sizeof(uint32_t) * kLeafCap * warps);
        // Patch codes and records of one launch chunk; read back after each
        // chunk, so the pool is bounded by the chunk's pairs.
        const unsigned long long chunk = std::min<unsigned long long>(1ull << 18, std::max(nDevice, 1ull));
        check(cudaMemGetInfo(&freeBytes, &totalBytes), "device memory query");
        const size_t poolCap =
            std::max<size_t>(4096, std::min<size_t>(64 * chunk + 4096, freeBytes / 4 / sizeof(PatchCode)));
        DevMem dPool(sizeof(PatchCode) * poolCap), dRecords(sizeof(PairRecord) * chunk),
            dFlagged(sizeof(uint2) * std::max<unsigned long long>(nDevice, 1));
        DevMem dWhole(f.allPairs ? units : 16);
        if (f.allPairs)
            check(cudaMemsetAsync(dWhole.p, 0, units, stream), "planner reset");
        WarpMem arena{dHdr.as<LeafHdr>(), dInteg.as<double>(), dPend.as<uint32_t>(), dPendErr.as<double>(),
                      dAtl.as<uint32_t>(), nullptr, nullptr};
        PairOutput O{dPool.as<PatchCode>(), poolCap, counters + 2, dRecords.as<PairRecord>(), counters + 3,
                     dWhole.as<uint8_t>(), counters + 6};
        struct Events {  // kernel time of the refinement launches
            cudaEvent_t a = nullptr, b = nullptr;
            ~Events() {
                if (a)
                    cudaEventDestroy(a);
                if (b)
                    cudaEventDestroy(b);
            }
        } events;
        check(cudaEventCreate(&events.a), "planner event");
        check(cudaEventCreate(&events.b), "planner event");
        const cudaEvent_t evStart = events.a, evStop = events.b;
        // all-pairs mode: the root pre-pass settles the pairs that end at their
        // root estimate; the rest go to the refinement
        const uint2 *refineList = dDeviceList.as<uint2>();
        unsigned long long nRefine = nDevice;
        DevMem dRest(f.allPairs ? sizeof(uint2) * std::max(nDevice, 1ull) : 16);
        if (f.allPairs && nDevice) {
            check(cudaMemsetAsync(counters + 7, 0, sizeof(unsigned long long), stream), "planner reset");
            check(cudaEventRecord(evStart, stream), "planner event");
            rootKernel<<<unsigned((nDevice * 4 + kRootThreads - 1) / kRootThreads), kRootThreads, 0, stream>>>(
                A, dDeviceList.as<uint2>(), nDevice, dWhole.as<uint8_t>(), dRest.as<uint2>(), counters + 7);
            check(cudaGetLastError(), "planner root pre-pass");
            check(cudaEventRecord(evStop, stream), "planner event");
            unsigned long long nRest = 0;
            check(cudaMemcpyAsync(&nRest, counters + 7, sizeof(nRest), cudaMemcpyDeviceToHost, stream),
                  "planner readback");
            check(cudaStreamSynchronize(stream), "planner root pre-pass");
            float rootMs = 0;
            check(cudaEventElapsedTime(&rootMs, evStart, evStop), "planner event");
            refineKernelMs += rootMs;
            rootSamples = nDevice * (unsigned long long)(A.rules.n[0] * A.rules.n[0] + A.rules.n[1] * A.rules.n[1]);
            rootSettled = nDevice - nRest;
            refineList = dRest.as<uint2>();
            nRefine = nRest;
        }
        for (unsigned long long begin = 0; begin < nRefine; begin += chunk) {
            if (cancel && *cancel)
                throw Cancelled();
            const unsigned long long n = std::min(chunk, nRefine - begin);
            check(cudaMemsetAsync(counters + 2, 0, 2 * sizeof(unsigned long long), stream), "planner reset");
            check(cudaMemsetAsync(counters + 5, 0, sizeof(unsigned long long), stream), "planner reset");
            check(cudaEventRecord(evStart, stream), "planner event");
            refineKernel<<<unsigned(grid), 32 * kWarpsPerBlock, kRefineSmem, stream>>>(
                A, refineList + begin, n, counters + 5, arena, O, dFlagged.as<uint2>(), counters + 4);
            check(cudaGetLastError(), "planner refinement");
            check(cudaEventRecord(evStop, stream), "planner event");
            unsigned long long n2c[2] = {};
            check(cudaMemcpyAsync(n2c, counters + 2, sizeof(n2c), cudaMemcpyDeviceToHost, stream), "planner readback");
            check(cudaStreamSynchronize(stream), "planner refinement");
            float chunkMs = 0;
            check(cudaEventElapsedTime(&chunkMs, evStart, evStop), "planner event");
            refineKernelMs += chunkMs;
            const unsigned long long used = std::min<unsigned long long>(n2c[0], poolCap), nRec = n2c[1];
            const size_t r0 = records.size(), p0 = pool.size();
            records.resize(r0 + nRec);
            pool.resize(p0 + used);
            if (nRec)
                check(cudaMemcpyAsync(records.data() + r0, dRecords.p, sizeof(PairRecord) * nRec,
                                      cudaMemcpyDeviceToHost, stream),
                      "planner readback");
            if (used)
                check(cudaMemcpyAsync(pool.data() + p0, dPool.p, sizeof(PatchCode) * used, cudaMemcpyDeviceToHost,
                                      stream),
                      "planner readback");
            check(cudaStreamSynchronize(stream), "planner readback");
            if (pool.size() > 0xffffffffull)
                throw OutOfMemory("Interaction plan exceeds 2^32 quadrature patches.");
            for (size_t r = r0; r < records.size(); ++r)
                records[r].patchFirst += uint32_t(p0);
        }
        unsigned long long n5[7] = {};
        phase[2] = msSince(t0);
        check(cudaMemcpyAsync(n5, counters, sizeof(n5), cudaMemcpyDeviceToHost, stream), "planner readback");
        check(cudaStreamSynchronize(stream), "planner readback");
        sampleTotal = n5[6] + rootSamples;
        const unsigned long long nFlag = n5[4];
        flagged.resize(nFlag);
        if (nFlag)
            check(cudaMemcpyAsync(flagged.data(), dFlagged.p, sizeof(uint2) * nFlag, cudaMemcpyDeviceToHost, stream),
                  "planner readback");
        if (f.allPairs) {
            whole.resize(units);
            check(cudaMemcpyAsync(whole.data(), dWhole.p, units, cudaMemcpyDeviceToHost, stream), "planner readback");
        }
        check(cudaStreamSynchronize(stream), "planner readback");
#else
        throw Unsupported("device planner unavailable in this build");
#endif
    }
    const double deviceMs = msSince(t0);
    phase[3] = deviceMs;
    const auto t1 = Clock::now();
    const unsigned workers = std::max(1u, std::min<unsigned>(64, std::thread::hardware_concurrency()));
    const auto parallel = [&](size_t count, size_t grain, auto &&body) {
        std::atomic<size_t> next{0};
        std::vector<std::thread> threads;
        for (unsigned wkr = 0; wkr < std::min<size_t>(workers, (count + grain - 1) / grain); ++wkr)
            threads.emplace_back([&]() {
                for (;;) {
                    const size_t begin = next.fetch_add(grain);
                    if (begin >= count)
                        return;
                    for (size_t q = begin; q < std::min(count, begin + grain); ++q)
                        body(q);
                }
            });
        for (auto &th : threads)
            th.join();
    };
    const auto decode = [&](const PatchCode &c, Patch &p) {
        const Sub a = subOfPath(c.pathA, c.depthA), b = subOfPath(c.pathB, c.depthB);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                p.test[3 * i + j] = a.v[i][j];
                p.trial[3 * i + j] = b.v[i][j];
            }
        p.areaFraction = a.fraction * b.fraction;
        p.degree = c.degree;
        p.projection = 0;
        p.intervals = 1;
        p.pad = 0;
    };
    // Runs of leaves whose order the device could not decide: the host
    // orders each by its own error estimates (pair_quadrature.cpp:644-683 as
    // the host planner evaluates them); a tie among them leaves the order to
    // the host planner's heap, so such a pair is refined on the host.
    size_t resolved = 0;
    std::vector<int32_t> settled(records.size(), -1);  // record -> its resolved patches
    std::vector<std::vector<Patch>> settledPatches;
    {
        std::vector<size_t> uncertain;
        for (size_t r = 0; r < records.size(); ++r)
            if (records[r].uncertain)
                uncertain.push_back(r);
        std::vector<uint8_t> tie(uncertain.size(), 0);
        settledPatches.resize(uncertain.size());
        parallel(uncertain.size(), 1, [&](size_t u) {
            const PairRecord &rec = records[uncertain[u]];
            const PatchCode *codes = pool.data() + rec.patchFirst;
            std::vector<Patch> &pp = settledPatches[u];
            pp.resize(rec.count);
            for (uint32_t q = 0; q < rec.count; ++q)
                decode(codes[q], pp[q]);
            const HostPanel &t = sp.panels[rec.first], &s = sp.panels[rec.second];
            std::vector<std::pair<double, Patch>> run;
            for (uint32_t k = 0; k < rec.count;) {
                uint32_t e = k + 1;
                while (e < rec.count && codes[e].joins)
                    ++e;
                if (e - k > 1) {
                    run.clear();
                    for (uint32_t q = k; q < e; ++q)
                        run.emplace_back(hostPatchError(t, s, pp[q], maxK), pp[q]);
                    std::stable_sort(run.begin(), run.end(),
                                     [](const auto &x, const auto &y) { return x.first > y.first; });
                    for (size_t q = 1; q < run.size(); ++q)
                        tie[u] |= run[q].first == run[q - 1].first ? 1 : 0;
                    for (size_t q = 0; q < run.size(); ++q)
                        pp[k + q] = run[q].second;
                }
                k = e;
            }
        });
        std::vector<uint8_t> drop(records.size(), 0);
        for (size_t u = 0; u < uncertain.size(); ++u) {
            if (tie[u]) {
                drop[uncertain[u]] = 1;
                flagged.push_back(make_uint2(records[uncertain[u]].first, records[uncertain[u]].second));
            } else {
                settled[uncertain[u]] = int32_t(u);
                ++resolved;
            }
        }
        size_t kept = 0;
        for (size_t r = 0; r < records.size(); ++r)
            if (!drop[r]) {
                settled[kept] = settled[r];
                records[kept++] = records[r];
            }
        records.resize(kept);
        settled.resize(kept);
    }
    const double hostT0 = msSince(t0);
    // the host refines projected and flagged pairs
    std::vector<std::pair<uint32_t, uint32_t>> hostPairs;
    hostPairs.reserve(hostList.size() + flagged.size());
    for (const auto &p : hostList)
        hostPairs.emplace_back(p.x, p.y);
    for (const auto &p : flagged)
        hostPairs.emplace_back(p.x, p.y);
    std::sort(hostPairs.begin(), hostPairs.end());
    const std::vector<PairRule> hostRules = planPairsOnHost(sp, st, maxK, hostPairs, 0, cancel);
    const double hostT1 = msSince(t0);
    // Flatten in (first, second) order, the host planner's order
    // (appendPairRule's rules): offsets first, then every pair's patches are
    // decoded or copied straight to their place.
    struct Item {
        uint64_t key;
        int32_t host;  // index into hostRules, or -1 - record index
        uint64_t offset;
    };
    std::vector<Item> items;
    items.reserve(records.size() + hostRules.size());
    for (size_t r = 0; r < records.size(); ++r)
        items.push_back({(uint64_t(records[r].first) << 32) | records[r].second, -1 - int32_t(r), 0});
    for (size_t h = 0; h < hostPairs.size(); ++h)
        items.push_back({(uint64_t(hostPairs[h].first) << 32) | hostPairs[h].second, int32_t(h), 0});
    std::sort(items.begin(), items.end(), [](const Item &x, const Item &y) { return x.key < y.key; });
    if (f.allPairs)
        for (unsigned long long u = 0; u < units; ++u)
            if (whole[u])
                f.plan.wholePanelDegrees[u] = whole[u];
    Plan &plan = f.plan;
    uint64_t total = 0;
    plan.near.reserve(2 * items.size());
    for (auto &it : items) {
        const uint32_t i = uint32_t(it.key >> 32), j = uint32_t(it.key & 0xffffffffu);
        uint32_t count, maxDepth;
        double relError;
        if (it.host >= 0) {
            const PairRule &r = hostRules[size_t(it.host)];
            count = uint32_t(r.patches.size()), maxDepth = r.maxDepth, relError = r.relError;
            if (f.allPairs && maxDepth == 0 && count == 1 && !r.patches[0].projection) {
                plan.wholePanelDegrees[unorderedPairIndex(i, j)] = uint8_t(r.patches[0].degree);
                plan.maxRelError = std::max(plan.maxRelError, relError);
                it.offset = ~0ull;
                continue;
            }
        } else {
            const PairRecord &r = records[size_t(-1 - it.host)];
            count = r.count, maxDepth = r.maxDepth, relError = r.relError;
        }
        it.offset = total;
        plan.near.push_back({i, j, uint32_t(total), count, 0});
        plan.near.push_back({j, i, uint32_t(total), count, 1});
        plan.maxDepth = std::max(plan.maxDepth, maxDepth);
        plan.maxRelError = std::max(plan.maxRelError, relError);
        total += count;
    }
    if (total > 0xffffffffull)
        throw OutOfMemory("Interaction plan exceeds 2^32 quadrature patches.");
    const double hostT2 = msSince(t0);
    plan.patches.resize(total);
    parallel(items.size(), 256, [&](size_t q) {
        const Item &it = items[q];
        if (it.offset == ~0ull)
            return;
        Patch *out = plan.patches.data() + it.offset;
        if (it.host >= 0) {
            const PairRule &r = hostRules[size_t(it.host)];
            std::copy(r.patches.begin(), r.patches.end(), out);
            return;
        }
        const size_t rec = size_t(-1 - it.host);
        const PairRecord &r = records[rec];
        if (settled[rec] >= 0) {
            const auto &pp = settledPatches[size_t(settled[rec])];
            std::copy(pp.begin(), pp.end(), out);
        } else {
            for (uint32_t k = 0; k < r.count; ++k)
                decode(pool[r.patchFirst + k], out[k]);
        }
    });
    const double hostT3 = msSince(t0);
    finishPlan(f.plan, T);
    phase[4] = msSince(t0);
    if (stats) {
        stats->devicePairs = devicePairs;
        stats->projectedPairs = hostList.size();
        stats->flaggedPairs = flagged.size();
        stats->resolvedPairs = resolved;
        stats->samples = sampleTotal;
        stats->rootSettledPairs = rootSettled;
        stats->refineKernelMs = refineKernelMs;
        size_t wholeCount = 0;
        for (const auto b : whole)
            wholeCount += b != 0;
        stats->wholePanelPairs = wholeCount;
        stats->deviceMs = deviceMs;
        for (int i = 0; i < 5; ++i)  // phase durations
            stats->phaseMs[i] = phase[i] - (i ? phase[i - 1] : 0.0);
        const double hostMarks[5] = {phase[3], hostT0, hostT1, hostT2, hostT3};
        for (int i = 0; i < 4; ++i)
            stats->hostPhaseMs[i] = hostMarks[i + 1] - hostMarks[i];
        stats->hostPhaseMs[4] = phase[4] - hostT3;
        stats->hostMs = msSince(t1);
    }
    return std::move(f.plan);
}

}  // namespace hsb
