// Far-field operator of the fast-multipole form: leaf emission (P2M),
// rotation-coaxial-rotation translations (M2M, M2L, L2L) and leaf testing
// (L2P) of the six expansion channels V (3) and W (3), FP64.
//
// Reference stages (support_fmm_operator.cu:1220-1296): P2M
// emitSpherical (wideband_leaf.cu:64-150), LF transfers rotate -> axial ->
// rotate (wideband_rotation.cu:19-99, wideband_axial.cu:10-90), L2P
// testSpherical. Work layout here: one CTA per output node for every
// translation (its links in a fixed order, so sums are deterministic), one
// warp per quadrature point for expansion tables, the local expansion's
// divergence formed once per leaf in coefficient space.
#include "fmm.hpp"
#include "fmm_math.cuh"
#include "kernel_timer.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>

namespace hsb {
namespace {

void fmmCheck(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw CudaError(std::string("CUDA fast multipole ") + what + ": " + cudaGetErrorString(e));
}

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    ~DevBuf() {
        if (p)
            cudaFree(p);
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
    void upload(const void *src, size_t n, cudaStream_t s) {
        ensure(n);
        if (n)
            fmmCheck(cudaMemcpyAsync(p, src, n, cudaMemcpyHostToDevice, s), "upload");
    }
    void ensure(size_t n) {
        if (n <= bytes)
            return;
        if (p)
            fmmCheck(cudaFree(p), "free");
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, n) != cudaSuccess) {
            p = nullptr;
            throw OutOfMemory("CUDA fast multipole workspace allocation failed.");
        }
        bytes = n;
    }
};
template <class T> void uploadVec(DevBuf &b, const std::vector<T> &v, cudaStream_t s) {
    b.upload(v.data(), v.size() * sizeof(T), s);
}

struct FmmPanel {
    double v0[3], e1[3], e2[3], n[3], curl[9], area;
    uint32_t nodes[3], pad;
};
// A panel touching a leaf's pressure supports: bit a of mask set when vertex
// a belongs to the leaf; inc[a] the vertex-incidence index of (vertex, panel).
struct FmmItem {
    uint32_t panel, mask, inc[3];
};
// One translation input: source node, Wigner class, coaxial class, azimuth.
struct TransLink {
    uint32_t source, wclass, cclass, pad;
    double phi;
};

// Panel rule of the far field: per point b0, b1, b2 and the physical weight
// fraction (sum 1), in device memory per operator (its degree can be promoted).
constexpr int kWarps = 8;
constexpr size_t kMaxShared = 227 * 1024;  // dynamic shared memory per CTA (opt-in)

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulConj(double2 a, double2 b) {  // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// Complex arithmetic of either precision (the translations run in FP64, or in
// FP32 on scaled coefficients in the mixed form).
template <class R> struct CxOf;
template <> struct CxOf<double> {
    using T = double2;
};
template <> struct CxOf<float> {
    using T = float2;
};
template <class R> using C2R = typename CxOf<R>::T;
template <class R, class A, class B> __device__ __forceinline__ C2R<R> mkc(A x, B y) {
    C2R<R> v;
    v.x = R(x);
    v.y = R(y);
    return v;
}
template <class R> __device__ __forceinline__ C2R<R> cmulT(C2R<R> a, C2R<R> b) {
    return mkc<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class R> __device__ __forceinline__ C2R<R> caddT(C2R<R> a, C2R<R> b) { return mkc<R>(a.x + b.x, a.y + b.y); }

// Warp table of the regular solid harmonics at d: j_n(k|d|) (n <= P),
// Theta_n^m(cos t) (triIndex) and exp(i m phi) (m <= P).
struct PointTable {
    double *j, *th;
    double2 *eph;
};
// Doubles of one table, even so that every table starts 16-byte aligned.
HS_HD size_t tableDoubles(int P) {
    const size_t d = size_t(P + 1) + size_t(P + 1) * (P + 2) / 2 + 2 * size_t(P + 1);
    return (d + 1) & ~size_t(1);
}
__device__ PointTable tableAt(double *base, int P) {
    PointTable t;
    t.eph = reinterpret_cast<double2 *>(base);
    t.j = base + 2 * (P + 1);
    t.th = t.j + (P + 1);
    return t;
}
__device__ void fillTable(const PointTable &t, int P, double dx, double dy, double dz, double k, int lane) {
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double ct = r > 0 ? dz / r : 1.0;
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    const double ph = atan2(dy, dx);
    if (lane == 0)
        besselJ(P, k * r, t.j);
    for (int m = lane; m <= P; m += 32) {
        thetaColumn(m, P, ct, st, t.th);
        double s, c;
        sincos(m * ph, &s, &c);
        t.eph[m] = make_double2(c, s);
    }
    __syncwarp();
}
// R_n^m = j_n Y_n^m from a table.
__device__ __forceinline__ double2 solidR(const PointTable &t, int n, int m) {
    const int am = m < 0 ? -m : m;
    const double a = t.j[n] * t.th[triIndex(n, am)];
    const double2 e = t.eph[am];
    if (m >= 0)
        return make_double2(a * e.x, a * e.y);
    const double sg = (am & 1) ? -1.0 : 1.0;  // Theta_n^-m = (-1)^m Theta_n^m, exp(-i m phi)
    return make_double2(sg * a * e.x, -sg * a * e.y);
}
__device__ __forceinline__ void decode(int k, int &n, int &m) {
    n = int(sqrtf(float(k)));  // corrected below (k < 2^24)
    while (n * n > k)
        --n;
    while ((n + 1) * (n + 1) <= k)
        ++n;
    m = k - n * n - n;
}

// Quadrature point q of an item's panel: position and the six channel strengths.
__device__ void pointStrengths(const FmmPanel &P, uint32_t mask, const double *rule, int q, const double2 *p,
                               double *x, double2 (&s)[6]) {
    const double b0 = rule[4 * q], b1 = rule[4 * q + 1], b2 = rule[4 * q + 2];
    const double w = rule[4 * q + 3] * P.area;
    for (int d = 0; d < 3; ++d)
        x[d] = P.v0[d] + b1 * P.e1[d] + b2 * P.e2[d];
    const double b[3] = {b0, b1, b2};
    double2 phiP = make_double2(0, 0);  // sum_a phi_a p_a
    double2 curl[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (int a = 0; a < 3; ++a) {
        if (!((mask >> a) & 1))
            continue;
        const double2 pa = p[P.nodes[a]];
        phiP = cadd(phiP, make_double2(b[a] * pa.x, b[a] * pa.y));
        for (int d = 0; d < 3; ++d)
            curl[d] = cadd(curl[d], make_double2(P.curl[3 * a + d] * pa.x, P.curl[3 * a + d] * pa.y));
    }
    for (int d = 0; d < 3; ++d) {
        s[d] = make_double2(w * P.n[d] * phiP.x, w * P.n[d] * phiP.y);
        s[3 + d] = make_double2(w * curl[d].x, w * curl[d].y);
    }
}

// Right-hand-side source: panel s's flux q_s emitted through the leaf's
// vertex supports of s, 1/3 per support (channel 0).
__device__ void fluxStrength(const FmmPanel &P, uint32_t panel, uint32_t mask, const double *rule, int q,
                             const double2 *flux, double *x, double2 (&s)[6]) {
    const double b1 = rule[4 * q + 1], b2 = rule[4 * q + 2];
    const double w = rule[4 * q + 3] * P.area * double(__popc(mask)) / 3.0;
    for (int d = 0; d < 3; ++d)
        x[d] = P.v0[d] + b1 * P.e1[d] + b2 * P.e2[d];
    const double2 qs = flux[panel];
    s[0] = make_double2(w * qs.x, w * qs.y);
    for (int c = 1; c < 6; ++c)
        s[c] = make_double2(0, 0);
}

// P2M of the leaves of one level: M[c][n,m] = sum over points s_c conj(R_n^m(y - centre)).
__global__ void __launch_bounds__(256) p2mKernel(const FmmPanel *__restrict__ panels,
                                                 const uint32_t *__restrict__ leaves, const uint32_t *__restrict__ itemStart,
                                                 const FmmItem *__restrict__ items, const double *__restrict__ centers,
                                                 const uint64_t *__restrict__ coefOffset, int p, double k,
                                                 const double2 *__restrict__ pvec, double2 *M, int rhsMode,
                                                 float2 *M32, const double *__restrict__ sigma,
                                                 const double *__restrict__ rule, int rulePts) {
    extern __shared__ double smem[];
    const int P = p;
    const int nch = rhsMode ? 1 : 6;
    const size_t td = tableDoubles(P);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *tables = smem;
    double2 *str = reinterpret_cast<double2 *>(smem + kWarps * td);  // [warp][6]
    const uint32_t leaf = leaves[blockIdx.x];
    const double *c = centers + 3 * size_t(leaf);
    const uint32_t i0 = itemStart[blockIdx.x], i1 = itemStart[blockIdx.x + 1];
    const uint32_t points = (i1 - i0) * rulePts;
    const int nc = (P + 1) * (P + 1);
    double2 *out = M + coefOffset[leaf];
    float2 *out32 = M32 ? M32 + coefOffset[leaf] : nullptr;
    const PointTable mine = tableAt(tables + warp * td, P);
    for (int chunk = 0; chunk * 256 < nc; ++chunk) {
        const int kk = chunk * 256 + threadIdx.x;
        int n = 0, m = 0;
        if (kk < nc)
            decode(kk, n, m);
        double2 acc[6];
        for (int ch = 0; ch < 6; ++ch)
            acc[ch] = make_double2(0, 0);
        for (uint32_t base = 0; base < points; base += kWarps) {
            const uint32_t idx = base + warp;
            if (idx < points) {
                const FmmItem it = items[i0 + idx / rulePts];
                double x[3];
                double2 s[6];
                if (rhsMode)
                    fluxStrength(panels[it.panel], it.panel, it.mask, rule, idx % rulePts, pvec, x, s);
                else
                    pointStrengths(panels[it.panel], it.mask, rule, idx % rulePts, pvec, x, s);
                fillTable(mine, P, x[0] - c[0], x[1] - c[1], x[2] - c[2], k, lane);
                if (lane < 6)
                    str[warp * 6 + lane] = s[lane];
            }
            __syncthreads();
            if (kk < nc)
                for (int w = 0; w < kWarps && base + w < points; ++w) {
                    const PointTable t = tableAt(tables + w * td, P);
                    const double2 R = solidR(t, n, m);
                    for (int ch = 0; ch < nch; ++ch)
                        acc[ch] = cadd(acc[ch], cmulConj(R, str[w * 6 + ch]));
                }
            __syncthreads();
        }
        if (kk < nc) {
            if (out32)  // scaled FP32 moments: M sigma_n, sigma_n = (2n+1)!! / (k a)^n of the level
                for (int ch = 0; ch < nch; ++ch)
                    out32[size_t(ch) * nc + kk] = make_float2(float(acc[ch].x * sigma[n]), float(acc[ch].y * sigma[n]));
            else
                for (int ch = 0; ch < nch; ++ch)
                    out[size_t(ch) * nc + kk] = acc[ch];
        }
    }
}

// One translation per link into the CTA's output node, channels in chunks:
// rotate the input to the link axis, coaxial translation, rotate back. A
// thread owns one coefficient for every channel of the chunk, so each Wigner
// and coaxial entry is read once per chunk; the azimuth phases are applied
// when the input is staged and when the output is accumulated.
// The channels [blockIdx.y * CPC, +CPC) of the output node go to one CTA:
// channels are independent outputs, so spreading them over CTAs multiplies
// the grid (few output nodes on the coarse levels) with no reduction.
template <int CPC, class R>
__global__ void __launch_bounds__(256) translateKernel(const uint32_t *__restrict__ outNodes,
                                                       const uint32_t *__restrict__ linkStart,
                                                       const TransLink *__restrict__ links, int pin, int pout,
                                                       const C2R<R> *__restrict__ inCoef, C2R<R> *outCoef,
                                                       const uint64_t *__restrict__ coefOffset,
                                                       const R *__restrict__ wigner,
                                                       const uint64_t *__restrict__ wignerStart,
                                                       const C2R<R> *__restrict__ coax,
                                                       const uint64_t *__restrict__ coaxStart, int zeroFirst,
                                                       int nch, int K, C2R<R> *partial) {
    constexpr int chunkCh = CPC;
    extern __shared__ double smem[];
    const int nin = (pin + 1) * (pin + 1), nout = (pout + 1) * (pout + 1);
    const int pmax = pin > pout ? pin : pout;
    const int nmax = nin > nout ? nin : nout;
    C2R<R> *eph = reinterpret_cast<C2R<R> *>(smem);
    C2R<R> *a = eph + (pmax + 1);
    C2R<R> *b = a + size_t(chunkCh) * nmax;
    C2R<R> *cbuf = b + size_t(chunkCh) * nmax;
    // K CTAs share an output node's links (contiguous parts); with K > 1 each
    // writes its own partial sum, added in a fixed order by reduceKernel
    const uint32_t oi = blockIdx.x / K, part = blockIdx.x % K;
    const uint32_t node = outNodes[oi];
    const int cFirst = blockIdx.y * CPC, cEnd = min(nch, cFirst + CPC);
    if (cFirst >= nch)
        return;
    C2R<R> *out = K > 1 ? partial + size_t(blockIdx.x) * 6 * nout : outCoef + coefOffset[node];
    if (zeroFirst || K > 1)
        for (int i = cFirst * nout + threadIdx.x; i < cEnd * nout; i += blockDim.x)
            out[i] = mkc<R>(0, 0);
    __syncthreads();
    const uint32_t l0 = linkStart[oi], len = linkStart[oi + 1] - l0;
    const uint32_t lBegin = l0 + uint32_t(uint64_t(len) * part / K), lEnd = l0 + uint32_t(uint64_t(len) * (part + 1) / K);
    for (uint32_t li = lBegin; li < lEnd; ++li) {
        const TransLink L = links[li];
        const C2R<R> *in = inCoef + coefOffset[L.source];
        const R *dtab = wigner + wignerStart[L.wclass];
        const C2R<R> *ctab = coax + coaxStart[L.cclass];
        for (int m = threadIdx.x; m <= pmax; m += blockDim.x) {
            double sn, cs;
            sincos(m * L.phi, &sn, &cs);
            eph[m] = mkc<R>(cs, sn);
        }
        __syncthreads();
        for (int c0 = cFirst; c0 < cEnd; c0 += chunkCh) {
            const int cc = min(chunkCh, cEnd - c0);
            // staged input with the azimuth phase: a[n, m] = in[n, m] exp(i m phi)
            for (int i = threadIdx.x; i < cc * nin; i += blockDim.x) {
                const int ch = i / nin, kk = i - ch * nin;
                int n, m;
                decode(kk, n, m);
                const C2R<R> e = m >= 0 ? eph[m] : mkc<R>(eph[-m].x, -eph[-m].y);
                a[ch * nin + kk] = cmulT<R>(in[size_t(c0 + ch) * nin + kk], e);
            }
            __syncthreads();
            // forward rotation: b[n, m'] = sum_m a[n, m] d^n[m, m']
            for (int kk = threadIdx.x; kk < nin; kk += blockDim.x) {
                int n, mp;
                decode(kk, n, mp);
                const int w = 2 * n + 1, base = n * n;
                const R *d = dtab + wignerOffset(n) + (mp + n);
                C2R<R> acc[CPC];
#pragma unroll
                for (int ch = 0; ch < CPC; ++ch)
                    acc[ch] = mkc<R>(0, 0);
                for (int j = 0; j < w; ++j) {
                    const R dv = d[size_t(j) * w];
#pragma unroll
                    for (int ch = 0; ch < CPC; ++ch)
                        if (ch < cc) {
                            const C2R<R> v = a[ch * nin + base + j];
                            acc[ch].x += v.x * dv;
                            acc[ch].y += v.y * dv;
                        }
                }
#pragma unroll
                for (int ch = 0; ch < CPC; ++ch)
                    if (ch < cc)
                        b[ch * nin + kk] = acc[ch];
            }
            __syncthreads();
            // coaxial translation per |m|: c[n', m] = sum_n C_|m|[n][n'] b[n, m]
            for (int kk = threadIdx.x; kk < nout; kk += blockDim.x) {
                int np, m;
                decode(kk, np, m);
                const int am = m < 0 ? -m : m;
                C2R<R> acc[CPC];
#pragma unroll
                for (int ch = 0; ch < CPC; ++ch)
                    acc[ch] = mkc<R>(0, 0);
                if (am <= pin) {
                    size_t off = 0;
                    for (int j = 0; j < am; ++j)
                        off += size_t(pin + 1 - j) * (pout + 1 - j);
                    const int wo = pout + 1 - am;
                    const C2R<R> *C = ctab + off + (np - am);
                    for (int n = am; n <= pin; ++n) {
                        const C2R<R> cv = C[size_t(n - am) * wo];
                        const int src = n * n + n + m;
#pragma unroll
                        for (int ch = 0; ch < CPC; ++ch)
                            if (ch < cc)
                                acc[ch] = caddT<R>(acc[ch], cmulT<R>(cv, b[ch * nin + src]));
                    }
                }
#pragma unroll
                for (int ch = 0; ch < CPC; ++ch)
                    if (ch < cc)
                        cbuf[ch * nout + kk] = acc[ch];
            }
            __syncthreads();
            // back rotation: out[n, m1] += exp(-i m1 phi) sum_m d^n[m1, m] c[n, m]
            for (int kk = threadIdx.x; kk < nout; kk += blockDim.x) {
                int n, m1;
                decode(kk, n, m1);
                const int w = 2 * n + 1, base = n * n;
                const R *d = dtab + wignerOffset(n) + size_t(m1 + n) * w;
                C2R<R> acc[CPC];
#pragma unroll
                for (int ch = 0; ch < CPC; ++ch)
                    acc[ch] = mkc<R>(0, 0);
                for (int j = 0; j < w; ++j) {
                    const R dv = d[j];
#pragma unroll
                    for (int ch = 0; ch < CPC; ++ch)
                        if (ch < cc) {
                            const C2R<R> v = cbuf[ch * nout + base + j];
                            acc[ch].x += v.x * dv;
                            acc[ch].y += v.y * dv;
                        }
                }
                const C2R<R> e = m1 >= 0 ? mkc<R>(eph[m1].x, -eph[m1].y) : eph[-m1];
#pragma unroll
                for (int ch = 0; ch < CPC; ++ch)
                    if (ch < cc) {
                        const size_t o = size_t(c0 + ch) * nout + kk;
                        out[o] = caddT<R>(out[o], cmulT<R>(acc[ch], e));
                    }
            }
            __syncthreads();
        }
    }
}

// out[node] (+)= sum over k of the K partial sums of the node, in order of k.
template <class R>
__global__ void reduceKernel(const uint32_t *__restrict__ outNodes, const uint64_t *__restrict__ coefOffset,
                             const C2R<R> *__restrict__ partial, int K, int nout, int nch, int assign,
                             C2R<R> *outCoef) {
    const uint32_t oi = blockIdx.x;
    C2R<R> *out = outCoef + coefOffset[outNodes[oi]];
    for (int e = threadIdx.x; e < nch * nout; e += blockDim.x) {
        C2R<R> acc = assign ? mkc<R>(0, 0) : out[e];
        for (int k = 0; k < K; ++k)
            acc = caddT<R>(acc, partial[(size_t(oi) * K + k) * 6 * nout + e]);
        out[e] = acc;
    }
}

// Grouped M2L. The links of a level whose translation vectors share the polar
// class and the distance (one Wigner block, one coaxial table) are cut into
// chunks of G links; one CTA takes a chunk with all channels, so every table
// entry it reads serves 6 G columns, and writes each link's local contribution
// u (phases applied) to its own slot. m2lSumKernel then adds the slots of each
// target in link order: the result is independent of the chunking and of the
// scheduling. Shared memory: two coefficient buffers [nc][cpad] (cpad odd:
// conflict-free column-strided staging), the links' azimuth phases and the
// m-major order of the coaxial outputs.
constexpr int kGroupTile = 6;  // columns per thread item

__host__ __device__ inline size_t groupSmemBytes(int p, int cpad, int g, size_t complexBytes) {
    const size_t nc = size_t(p + 1) * (p + 1);
    return 2 * nc * cpad * complexBytes + size_t(g) * (p + 1) * complexBytes + nc * 4 + size_t(p + 2) * 4;
}

template <class R>
__global__ void __launch_bounds__(256) m2lGroupKernel(const uint2 *__restrict__ chunks,
                                                      const uint32_t *__restrict__ sorted,
                                                      const TransLink *__restrict__ links, int p, int nch, int cpad,
                                                      int gmax, const C2R<R> *__restrict__ inCoef,
                                                      const uint64_t *__restrict__ coefOffset,
                                                      const R *__restrict__ wigner,
                                                      const uint64_t *__restrict__ wignerStart,
                                                      const C2R<R> *__restrict__ coax,
                                                      const uint64_t *__restrict__ coaxStart, C2R<R> *__restrict__ u) {
    using CT = C2R<R>;
    extern __shared__ double smem[];
    const int nc = (p + 1) * (p + 1);
    CT *bufA = reinterpret_cast<CT *>(smem);
    CT *bufB = bufA + size_t(nc) * cpad;
    CT *eph = bufB + size_t(nc) * cpad;                        // [gmax][p + 1]
    int *qmap = reinterpret_cast<int *>(eph + size_t(gmax) * (p + 1));  // m-major position -> kk
    int *coaxOff = qmap + nc;                                  // [p + 2]: offset of |m| in a coaxial table
    const uint2 chunk = chunks[blockIdx.x];
    const int count = int(chunk.y), C = count * nch;
    const TransLink L0 = links[sorted[chunk.x]];
    const R *dtab = wigner + wignerStart[L0.wclass];
    const CT *ctab = coax + coaxStart[L0.cclass];
    // phases, m-major order and coaxial block offsets
    for (int e = threadIdx.x; e < count * (p + 1); e += blockDim.x) {
        const int i = e / (p + 1), m = e - i * (p + 1);
        double sn, cs;
        sincos(m * links[sorted[chunk.x + i]].phi, &sn, &cs);
        eph[e] = mkc<R>(cs, sn);
    }
    for (int kk = threadIdx.x; kk < nc; kk += blockDim.x) {
        int n, m;
        decode(kk, n, m);
        const int a = m < 0 ? -m : m;
        // order m = 0, 1, -1, 2, -2, ...; block |m| = a holds n = a .. p
        const int before = a == 0 ? 0 : (p + 1) + 2 * ((a - 1) * (p + 1) - a * (a - 1) / 2);
        const int q = before + (m < 0 ? p + 1 - a : 0) + (n - a);
        qmap[q] = kk;
    }
    if (threadIdx.x == 0) {
        int off = 0;
        for (int a = 0; a <= p + 1; ++a) {
            coaxOff[a] = off;
            off += (p + 1 - a) * (p + 1 - a);
        }
    }
    __syncthreads();
    // staged inputs with the azimuth phase: A[kk][col] = M_src[ch][kk] exp(i m phi)
    for (int e = threadIdx.x; e < C * nc; e += blockDim.x) {
        const int col = e / nc, kk = e - col * nc;
        const int i = col / nch, ch = col - i * nch;
        int n, m;
        decode(kk, n, m);
        const uint32_t src = links[sorted[chunk.x + i]].source;
        const CT ph = eph[i * (p + 1) + (m < 0 ? -m : m)];
        const CT v = inCoef[coefOffset[src] + size_t(ch) * nc + kk];
        bufA[size_t(kk) * cpad + col] = cmulT<R>(v, m < 0 ? mkc<R>(ph.x, -ph.y) : ph);
    }
    __syncthreads();
    const int tiles = (C + kGroupTile - 1) / kGroupTile;
    // Rotations in items of two rows of one degree n (rows n^2 + 2q and + 1; the
    // odd last row of a degree alone) by kGroupTile columns: each staged value
    // read serves both rows. Pair q of degree n is item n (n + 1) / 2 + q.
    const int pairs = (p + 1) * (p + 2) / 2;
    // forward rotation: B[n, m'] = sum_m A[n, m] d^n[m, m']
    for (int e = threadIdx.x; e < tiles * pairs; e += blockDim.x) {
        const int tile = e / pairs, pq = e - tile * pairs, c0 = tile * kGroupTile;
        int n = int((sqrtf(8.f * pq + 1.f) - 1.f) * .5f);
        while (n * (n + 1) / 2 > pq)
            --n;
        while ((n + 1) * (n + 2) / 2 <= pq)
            ++n;
        const int r0 = 2 * (pq - n * (n + 1) / 2);  // row m' + n of the first row
        const bool two = r0 + 1 < 2 * n + 1;
        const int w = 2 * n + 1;
        const R *d = dtab + wignerOffset(n) + r0;
        const CT *x = bufA + size_t(n) * n * cpad + c0;
        CT a0[kGroupTile], a1[kGroupTile];
#pragma unroll
        for (int c = 0; c < kGroupTile; ++c)
            a0[c] = a1[c] = mkc<R>(0, 0);
#pragma unroll 2
        for (int j = 0; j < w; ++j) {
            const R d0 = d[size_t(j) * w], d1 = two ? d[size_t(j) * w + 1] : R(0);
#pragma unroll
            for (int c = 0; c < kGroupTile; ++c) {
                const CT v = x[size_t(j) * cpad + c];
                a0[c].x += v.x * d0;
                a0[c].y += v.y * d0;
                a1[c].x += v.x * d1;
                a1[c].y += v.y * d1;
            }
        }
        CT *o = bufB + size_t(n * n + r0) * cpad + c0;
#pragma unroll
        for (int c = 0; c < kGroupTile; ++c)
            if (c0 + c < C) {
                o[c] = a0[c];
                if (two)
                    o[cpad + c] = a1[c];
            }
    }
    __syncthreads();
    // coaxial translation per |m| (outputs in m-major order, so a warp reads
    // consecutive entries of one table block): A[n', m] = sum_n C_|m|[n][n'] B[n, m]
    for (int e = threadIdx.x; e < tiles * nc; e += blockDim.x) {
        const int tile = e / nc, q = e - tile * nc, c0 = tile * kGroupTile;
        const int kk = qmap[q];
        int np, m;
        decode(kk, np, m);
        const int a = m < 0 ? -m : m, wo = p + 1 - a;
        const CT *Ct = ctab + coaxOff[a] + (np - a);
        CT acc[kGroupTile];
#pragma unroll
        for (int c = 0; c < kGroupTile; ++c)
            acc[c] = mkc<R>(0, 0);
        for (int n = a; n <= p; ++n) {
            const CT cv = Ct[size_t(n - a) * wo];
            const CT *x = bufB + size_t(n * n + n + m) * cpad + c0;
#pragma unroll
            for (int c = 0; c < kGroupTile; ++c)
                acc[c] = caddT<R>(acc[c], cmulT<R>(cv, x[c]));
        }
#pragma unroll
        for (int c = 0; c < kGroupTile; ++c)
            if (c0 + c < C)
                bufA[size_t(kk) * cpad + c0 + c] = acc[c];
    }
    __syncthreads();
    // back rotation: B[n, m1] = sum_m d^n[m1, m] A[n, m]
    for (int e = threadIdx.x; e < tiles * pairs; e += blockDim.x) {
        const int tile = e / pairs, pq = e - tile * pairs, c0 = tile * kGroupTile;
        int n = int((sqrtf(8.f * pq + 1.f) - 1.f) * .5f);
        while (n * (n + 1) / 2 > pq)
            --n;
        while ((n + 1) * (n + 2) / 2 <= pq)
            ++n;
        const int r0 = 2 * (pq - n * (n + 1) / 2);  // row m1 + n of the first row
        const bool two = r0 + 1 < 2 * n + 1;
        const int w = 2 * n + 1;
        const R *d0p = dtab + wignerOffset(n) + size_t(r0) * w;
        const R *d1p = two ? d0p + w : d0p;
        const CT *x = bufA + size_t(n) * n * cpad + c0;
        CT a0[kGroupTile], a1[kGroupTile];
#pragma unroll
        for (int c = 0; c < kGroupTile; ++c)
            a0[c] = a1[c] = mkc<R>(0, 0);
#pragma unroll 2
        for (int j = 0; j < w; ++j) {
            const R d0 = d0p[j], d1 = d1p[j];
#pragma unroll
            for (int c = 0; c < kGroupTile; ++c) {
                const CT v = x[size_t(j) * cpad + c];
                a0[c].x += v.x * d0;
                a0[c].y += v.y * d0;
                a1[c].x += v.x * d1;
                a1[c].y += v.y * d1;
            }
        }
        CT *o = bufB + size_t(n * n + r0) * cpad + c0;
#pragma unroll
        for (int c = 0; c < kGroupTile; ++c)
            if (c0 + c < C) {
                o[c] = a0[c];
                if (two)
                    o[cpad + c] = a1[c];
            }
    }
    __syncthreads();
    // each link's contribution with the conjugate phase, into its own slot
    for (int e = threadIdx.x; e < C * nc; e += blockDim.x) {
        const int col = e / nc, kk = e - col * nc;
        const int i = col / nch, ch = col - i * nch;
        int n, m;
        decode(kk, n, m);
        const CT ph = eph[i * (p + 1) + (m < 0 ? -m : m)];
        const CT v = bufB[size_t(kk) * cpad + col];
        u[(size_t(sorted[chunk.x + i]) * nch + ch) * nc + kk] = cmulT<R>(v, m < 0 ? ph : mkc<R>(ph.x, -ph.y));
    }
}

// out[target] += sum over the target's links, in link order, of their slots.
template <class R>
__global__ void __launch_bounds__(256) m2lSumKernel(const uint32_t *__restrict__ outNodes,
                                                    const uint32_t *__restrict__ linkStart,
                                                    const uint64_t *__restrict__ coefOffset, int nc, int nch,
                                                    const C2R<R> *__restrict__ u, C2R<R> *outCoef) {
    const uint32_t oi = blockIdx.x;
    const uint32_t l0 = linkStart[oi], l1 = linkStart[oi + 1];
    C2R<R> *out = outCoef + coefOffset[outNodes[oi]];
    for (int e = blockIdx.y * blockDim.x + threadIdx.x; e < nch * nc; e += gridDim.y * blockDim.x) {
        C2R<R> acc = out[e];
        for (uint32_t l = l0; l < l1; ++l)
            acc = caddT<R>(acc, u[size_t(l) * nch * nc + e]);
        out[e] = acc;
    }
}

// Coefficient-space derivatives of a regular expansion (k = 1 scaling):
// dz R_n^m = A(n,m) R_{n-1}^m - A(n+1,m) R_{n+1}^m, d+ = dx + i dy and d- = dx - i dy
// raise / lower m with the coefficients below.
__device__ __forceinline__ double coefA(int n, int m) {
    return n <= 0 ? 0.0 : sqrt(fmax(0.0, double(n * n - m * m) / ((2.0 * n - 1) * (2.0 * n + 1))));
}
__device__ __forceinline__ double coefBm(int n, int m) {
    return n <= 0 ? 0.0 : sqrt(fmax(0.0, double((n - m - 1) * (n - m)) / ((2.0 * n - 1) * (2.0 * n + 1))));
}
__device__ __forceinline__ double coefBp(int n, int m) {
    return n < 0 ? 0.0 : sqrt(fmax(0.0, double((n + m + 1) * (n + m + 2)) / ((2.0 * n + 1) * (2.0 * n + 3))));
}
__device__ __forceinline__ double coefCm(int n, int m) {
    return n <= 0 ? 0.0 : sqrt(fmax(0.0, double((n + m - 1) * (n + m)) / ((2.0 * n - 1) * (2.0 * n + 1))));
}
__device__ __forceinline__ double coefCp(int n, int m) {
    return n < 0 ? 0.0 : sqrt(fmax(0.0, double((n - m + 1) * (n - m + 2)) / ((2.0 * n + 1) * (2.0 * n + 3))));
}
__device__ __forceinline__ double2 coefAt(const double2 *L, int p, int n, int m) {
    if (n < 0 || n > p || m < -n || m > n)
        return make_double2(0, 0);
    return L[coefIndex(n, m)];
}

// A leaf's local coefficients (channels x nc) into shared memory: FP64 as
// stored, or the mixed form's scaled FP32 locals L^ = L tau_n unscaled to
// L = L^ sigma_n (tau_n = 1 / sigma_n).
__device__ void loadLocals(const double2 *L64, const float2 *L32, const double *sigma, uint64_t offset, int channels,
                           int nc, double2 *Ls) {
    if (L32) {
        for (int i = threadIdx.x; i < channels * nc; i += blockDim.x) {
            int n, m;
            decode(i % nc, n, m);
            const float2 v = L32[offset + i];
            Ls[i] = make_double2(double(v.x) * sigma[n], double(v.y) * sigma[n]);
        }
    } else {
        for (int i = threadIdx.x; i < channels * nc; i += blockDim.x)
            Ls[i] = L64[offset + i];
    }
    __syncthreads();
}

// L2P of the leaves of one level: forms D = div V (degree p + 1) in shared
// memory, then one warp per item evaluates V, W, D at its quadrature points
// and writes the item's incidence contributions
//   far[inc_a] = sum_q w phi_a (D + i k n.V) - (i / k) w curl_a . W.
__global__ void __launch_bounds__(256) l2pKernel(const FmmPanel *__restrict__ panels,
                                                 const uint32_t *__restrict__ leaves, const uint32_t *__restrict__ itemStart,
                                                 const FmmItem *__restrict__ items, const double *__restrict__ centers,
                                                 const uint64_t *__restrict__ coefOffset, int p, double k,
                                                 const double2 *__restrict__ Lcoef, double2 *far,
                                                 const float2 *__restrict__ L32, const double *__restrict__ sigma,
                                                 const double *__restrict__ rule, int rulePts, double2 *scratch) {
    extern __shared__ double smem[];
    const int P = p + 1, nc = (p + 1) * (p + 1), nd = (P + 1) * (P + 1);
    const size_t td = tableDoubles(P);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // coefficients in shared memory, or for high orders in the block's slice of a
    // global scratch (L1/L2-resident), leaving shared memory to the point tables
    double2 *Ls = scratch ? scratch + size_t(blockIdx.x) * (6 * nc + nd) : reinterpret_cast<double2 *>(smem);  // [6][nc]
    double2 *Ld = Ls + 6 * nc;                                                                               // [nd]
    double *tables = scratch ? smem : reinterpret_cast<double *>(Ld + nd);
    const uint32_t leaf = leaves[blockIdx.x];
    loadLocals(Lcoef, L32, sigma, coefOffset[leaf], 6, nc, Ls);
    __syncthreads();
    // D = dx Vx + dy Vy + dz Vz = (d+ U- + d- U+) / 2 + dz Vz, U-+ = Vx -+ i Vy (times k)
    for (int kk = threadIdx.x; kk < nd; kk += blockDim.x) {
        int n, m;
        decode(kk, n, m);
        const double2 *Vx = Ls, *Vy = Ls + nc, *Vz = Ls + 2 * nc;
        const auto U = [&](int nn, int mm, double sign) {  // Vx + sign i Vy
            const double2 x = coefAt(Vx, p, nn, mm), y = coefAt(Vy, p, nn, mm);
            return make_double2(x.x - sign * y.y, x.y + sign * y.x);
        };
        // dz: L_{n+1,m} A(n+1,m) - L_{n-1,m} A(n,m)
        const double2 z1 = coefAt(Vz, p, n + 1, m), z0 = coefAt(Vz, p, n - 1, m);
        const double a1 = coefA(n + 1, m), a0 = coefA(n, m);
        double2 d = make_double2(z1.x * a1 - z0.x * a0, z1.y * a1 - z0.y * a0);
        // d+ U-: U-_{n+1,m-1} Bm(n+1,m-1) + U-_{n-1,m-1} Bp(n-1,m-1)
        const double2 u1 = U(n + 1, m - 1, -1), u0 = U(n - 1, m - 1, -1);
        const double bm = coefBm(n + 1, m - 1), bp = coefBp(n - 1, m - 1);
        d.x += 0.5 * (u1.x * bm + u0.x * bp);
        d.y += 0.5 * (u1.y * bm + u0.y * bp);
        // d- U+: -(U+_{n+1,m+1} Cm(n+1,m+1) + U+_{n-1,m+1} Cp(n-1,m+1))
        const double2 v1 = U(n + 1, m + 1, 1), v0 = U(n - 1, m + 1, 1);
        const double cm = coefCm(n + 1, m + 1), cp = coefCp(n - 1, m + 1);
        d.x -= 0.5 * (v1.x * cm + v0.x * cp);
        d.y -= 0.5 * (v1.y * cm + v0.y * cp);
        Ld[kk] = make_double2(k * d.x, k * d.y);
    }
    __syncthreads();
    const uint32_t i0 = itemStart[blockIdx.x], i1 = itemStart[blockIdx.x + 1];
    const double *c = centers + 3 * size_t(leaf);
    const PointTable t = tableAt(tables + warp * td, P);
    for (uint32_t it = i0 + warp; it < i1; it += kWarps) {
        const FmmItem item = items[it];
        const FmmPanel &Pn = panels[item.panel];
        double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
        for (int q = 0; q < rulePts; ++q) {
            const double b1 = rule[4 * q + 1], b2 = rule[4 * q + 2];
            double x[3];
            for (int d = 0; d < 3; ++d)
                x[d] = Pn.v0[d] + b1 * Pn.e1[d] + b2 * Pn.e2[d];
            fillTable(t, P, x[0] - c[0], x[1] - c[1], x[2] - c[2], k, lane);
            double2 f[7];
            for (int ch = 0; ch < 7; ++ch)
                f[ch] = make_double2(0, 0);
            for (int kk = lane; kk < nd; kk += 32) {
                int n, m;
                decode(kk, n, m);
                const double2 R = solidR(t, n, m);
                if (kk < nc)
                    for (int ch = 0; ch < 6; ++ch)
                        f[ch] = cadd(f[ch], cmul(Ls[ch * nc + kk], R));
                f[6] = cadd(f[6], cmul(Ld[kk], R));
            }
            for (int ch = 0; ch < 7; ++ch)
                for (int o = 16; o > 0; o >>= 1) {
                    f[ch].x += __shfl_xor_sync(0xffffffffu, f[ch].x, o);
                    f[ch].y += __shfl_xor_sync(0xffffffffu, f[ch].y, o);
                }
            __syncwarp();
            // fields = -i k * sums
            double2 F[7];
            for (int ch = 0; ch < 7; ++ch)
                F[ch] = make_double2(k * f[ch].y, -k * f[ch].x);
            const double w = rule[4 * q + 3] * Pn.area;
            const double bq[3] = {rule[4 * q], b1, b2};
            // D + i k n.V
            double2 nv = make_double2(0, 0);
            for (int d = 0; d < 3; ++d) {
                nv.x += Pn.n[d] * F[d].x;
                nv.y += Pn.n[d] * F[d].y;
            }
            const double2 s0 = make_double2(F[6].x - k * nv.y, F[6].y + k * nv.x);
            for (int a = 0; a < 3; ++a) {
                if (!((item.mask >> a) & 1))
                    continue;
                double2 cw = make_double2(0, 0);
                for (int d = 0; d < 3; ++d) {
                    cw.x += Pn.curl[3 * a + d] * F[3 + d].x;
                    cw.y += Pn.curl[3 * a + d] * F[3 + d].y;
                }
                // - (i / k) w curl . W
                acc[a].x += w * bq[a] * s0.x + w * cw.y / k;
                acc[a].y += w * bq[a] * s0.y - w * cw.x / k;
            }
        }
        if (lane == 0)
            for (int a = 0; a < 3; ++a)
                if ((item.mask >> a) & 1)
                    far[item.inc[a]] = acc[a];
    }
}

// L2P of the right-hand-side field S (channel 0): forms grad S (degree p + 1)
// in shared memory, then one warp per item writes
//   far[inc_a] = sum_q w phi_a (-S + (i / k) n . grad S)
// (the far part of -S q - alpha K' q with alpha = -i / k).
__global__ void __launch_bounds__(256) l2pRhsKernel(const FmmPanel *__restrict__ panels,
                                                    const uint32_t *__restrict__ leaves,
                                                    const uint32_t *__restrict__ itemStart,
                                                    const FmmItem *__restrict__ items, const double *__restrict__ centers,
                                                    const uint64_t *__restrict__ coefOffset, int p, double k,
                                                    const double2 *__restrict__ Lcoef, double2 *far,
                                                    const float2 *__restrict__ L32, const double *__restrict__ sigma,
                                                    const double *__restrict__ rule, int rulePts, double2 *scratch) {
    extern __shared__ double smem[];
    const int P = p + 1, nc = (p + 1) * (p + 1), nd = (P + 1) * (P + 1);
    const size_t td = tableDoubles(P);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double2 *Ls = scratch ? scratch + size_t(blockIdx.x) * (nc + 3 * nd) : reinterpret_cast<double2 *>(smem);  // [nc]
    double2 *Lg = Ls + nc;  // [3][nd]: d/dx, d/dy, d/dz
    double *tables = scratch ? smem : reinterpret_cast<double *>(Lg + 3 * nd);
    const uint32_t leaf = leaves[blockIdx.x];
    loadLocals(Lcoef, L32, sigma, coefOffset[leaf], 1, nc, Ls);
    __syncthreads();
    for (int kk = threadIdx.x; kk < nd; kk += blockDim.x) {
        int n, m;
        decode(kk, n, m);
        const double2 z1 = coefAt(Ls, p, n + 1, m), z0 = coefAt(Ls, p, n - 1, m);
        const double a1 = coefA(n + 1, m), a0 = coefA(n, m);
        const double2 dz = make_double2(z1.x * a1 - z0.x * a0, z1.y * a1 - z0.y * a0);
        const double2 u1 = coefAt(Ls, p, n + 1, m - 1), u0 = coefAt(Ls, p, n - 1, m - 1);
        const double bm = coefBm(n + 1, m - 1), bp = coefBp(n - 1, m - 1);
        const double2 dp = make_double2(u1.x * bm + u0.x * bp, u1.y * bm + u0.y * bp);
        const double2 v1 = coefAt(Ls, p, n + 1, m + 1), v0 = coefAt(Ls, p, n - 1, m + 1);
        const double cm = coefCm(n + 1, m + 1), cp = coefCp(n - 1, m + 1);
        const double2 dm = make_double2(-(v1.x * cm + v0.x * cp), -(v1.y * cm + v0.y * cp));
        // dx = (d+ + d-) / 2, dy = -i (d+ - d-) / 2
        Lg[kk] = make_double2(0.5 * k * (dp.x + dm.x), 0.5 * k * (dp.y + dm.y));
        Lg[nd + kk] = make_double2(0.5 * k * (dp.y - dm.y), -0.5 * k * (dp.x - dm.x));
        Lg[2 * nd + kk] = make_double2(k * dz.x, k * dz.y);
    }
    __syncthreads();
    const uint32_t i0 = itemStart[blockIdx.x], i1 = itemStart[blockIdx.x + 1];
    const double *c = centers + 3 * size_t(leaf);
    const PointTable t = tableAt(tables + warp * td, P);
    for (uint32_t it = i0 + warp; it < i1; it += kWarps) {
        const FmmItem item = items[it];
        const FmmPanel &Pn = panels[item.panel];
        double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
        for (int q = 0; q < rulePts; ++q) {
            const double b1 = rule[4 * q + 1], b2 = rule[4 * q + 2];
            double x[3];
            for (int d = 0; d < 3; ++d)
                x[d] = Pn.v0[d] + b1 * Pn.e1[d] + b2 * Pn.e2[d];
            fillTable(t, P, x[0] - c[0], x[1] - c[1], x[2] - c[2], k, lane);
            double2 f[4];
            for (int ch = 0; ch < 4; ++ch)
                f[ch] = make_double2(0, 0);
            for (int kk = lane; kk < nd; kk += 32) {
                int n, m;
                decode(kk, n, m);
                const double2 R = solidR(t, n, m);
                if (kk < nc)
                    f[0] = cadd(f[0], cmul(Ls[kk], R));
                for (int d = 0; d < 3; ++d)
                    f[1 + d] = cadd(f[1 + d], cmul(Lg[d * nd + kk], R));
            }
            for (int ch = 0; ch < 4; ++ch)
                for (int o = 16; o > 0; o >>= 1) {
                    f[ch].x += __shfl_xor_sync(0xffffffffu, f[ch].x, o);
                    f[ch].y += __shfl_xor_sync(0xffffffffu, f[ch].y, o);
                }
            __syncwarp();
            double2 F[4];
            for (int ch = 0; ch < 4; ++ch)
                F[ch] = make_double2(k * f[ch].y, -k * f[ch].x);  // -i k * sums
            double2 dn = make_double2(0, 0);
            for (int d = 0; d < 3; ++d) {
                dn.x += Pn.n[d] * F[1 + d].x;
                dn.y += Pn.n[d] * F[1 + d].y;
            }
            // -S + (i / k) n.grad S
            const double2 v = make_double2(-F[0].x - dn.y / k, -F[0].y + dn.x / k);
            const double w = rule[4 * q + 3] * Pn.area;
            const double bq[3] = {rule[4 * q], b1, b2};
            for (int a = 0; a < 3; ++a)
                if ((item.mask >> a) & 1) {
                    acc[a].x += w * bq[a] * v.x;
                    acc[a].y += w * bq[a] * v.y;
                }
        }
        if (lane == 0)
            for (int a = 0; a < 3; ++a)
                if ((item.mask >> a) & 1)
                    far[item.inc[a]] = acc[a];
    }
}

// y_i = sum of the incidence contributions of vertex i (fixed order).
__global__ void starSumKernel(const double2 *__restrict__ far, const uint32_t *__restrict__ incOffsets, uint32_t N,
                              double2 *y) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N)
        return;
    double2 s = make_double2(0, 0);
    for (uint32_t j = incOffsets[i]; j < incOffsets[i + 1]; ++j)
        s = cadd(s, far[j]);
    y[i] = s;
}

// Coaxial translation tables: one thread per (class, |m|, n, n'). fl holds
// per class 4 pi i^? f_l(k t) Y_l^0(z) premultiplied: fl[class][l].
__global__ void coaxKernel(uint32_t classes, const int *__restrict__ pin, const int *__restrict__ pout,
                           const uint64_t *__restrict__ start, const double2 *__restrict__ fl, int lmax,
                           const double *__restrict__ gaunt, const uint32_t *__restrict__ gauntOff, int gP,
                           double2 *coax) {
    const uint32_t cls = blockIdx.y;
    if (cls >= classes)
        return;
    const int a = pin[cls], b = pout[cls];
    size_t total = 0;
    for (int j = 0; j <= min(a, b); ++j)
        total += size_t(a + 1 - j) * (b + 1 - j);
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        size_t off = 0;
        int mm = 0;
        while (off + size_t(a + 1 - mm) * (b + 1 - mm) <= e) {
            off += size_t(a + 1 - mm) * (b + 1 - mm);
            ++mm;
        }
        const size_t r = e - off;
        const int wo = b + 1 - mm;
        const int n = mm + int(r / wo), np = mm + int(r % wo);
        const double *g = gaunt + gauntOff[(size_t(mm) * (gP + 1) + n) * (gP + 1) + np];
        const double2 *f = fl + size_t(cls) * (lmax + 1);
        double2 acc = make_double2(0, 0);
        int idx = 0;
        for (int l = abs(n - np); l <= n + np; l += 2, ++idx) {
            const int e4 = ((n - np - l) / 2) & 1;  // i^(n - n' - l) = (-1)^((n - n' - l) / 2)
            const double sg = e4 ? -1.0 : 1.0;
            acc.x += sg * g[idx] * f[l].x;
            acc.y += sg * g[idx] * f[l].y;
        }
        coax[start[cls] + e] = acc;
    }
}

// ------------------------------------------------ plane-wave (diagonal) M2L
// Electrically large levels translate in the plane-wave form instead of
// rotate-coaxial-rotate (the reference's LF/HF switch,
// fmm/wideband_transfer.cpp:266-310, and its diagonal product,
// cuda/support_fmm_operator.cu:36-76). With s on the unit sphere,
//   sigma(s) = sum_nm i^n M_nm Y_n^m(s)                 (source signature),
//   psi(s)   = sum over links T_t(s) sigma_source(s),
//   T_t(s)   = sum_{l<=p} (2l+1) (-i)^l h_l(k|t|) P_l(s.t/|t|),
//   L_nm    += (-i)^n  int conj(Y_n^m(s)) psi(s) dOmega,
// for t = target centre - source centre; the sphere rule (Gauss-Legendre in
// cos(theta) x uniform azimuth) is exact for the degree 3p of the integrand.
// Conversions are separable: a Legendre stage per (m, theta row) and a Fourier
// stage per (theta row, azimuth), O(p^3) per node; a link costs O(p^2).
constexpr int kHfRows = 8;  // theta rows per chunk of the conversion kernels

// sigma of the nodes `ids` (one CTA per node and channel).
__global__ void __launch_bounds__(256) signatureKernel(const double2 *__restrict__ Mc,
                                                       const uint64_t *__restrict__ coefOffset,
                                                       const uint32_t *__restrict__ ids, int p,
                                                       const double *__restrict__ theta, int nth, int nph, int nch,
                                                       double2 *sigma) {
    extern __shared__ double smem[];
    const int nc = (p + 1) * (p + 1), tri = (p + 1) * (p + 2) / 2, mw = 2 * p + 1;
    double2 *Mi = reinterpret_cast<double2 *>(smem);  // i^n M_nm
    double2 *A = Mi + nc;                             // [mw][kHfRows]
    double2 *root = A + size_t(mw) * kHfRows;         // exp(2 pi i q / nph)
    const uint32_t node = blockIdx.x, ch = blockIdx.y;
    const double2 *M = Mc + coefOffset[ids[node]] + size_t(ch) * nc;
    for (int i = threadIdx.x; i < nc; i += blockDim.x) {
        int n, m;
        decode(i, n, m);
        const double2 v = M[i];
        // i^n: 1, i, -1, -i
        const int r = n & 3;
        Mi[i] = r == 0 ? v : r == 1 ? make_double2(-v.y, v.x) : r == 2 ? make_double2(-v.x, -v.y) : make_double2(v.y, -v.x);
    }
    for (int q = threadIdx.x; q < nph; q += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * q / nph, &sn, &cs);
        root[q] = make_double2(cs, sn);
    }
    __syncthreads();
    const size_t Q = size_t(nth) * nph;
    double2 *out = sigma + (size_t(node) * nch + ch) * Q;
    for (int i0 = 0; i0 < nth; i0 += kHfRows) {
        for (int e = threadIdx.x; e < mw * kHfRows; e += blockDim.x) {
            const int m = e % mw - p, ii = e / mw, i = i0 + ii;
            double2 acc = make_double2(0, 0);
            if (i < nth) {
                const int am = m < 0 ? -m : m;
                const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;  // Theta_n^-m = (-1)^m Theta_n^m
                const double *th = theta + size_t(i) * tri;
                for (int n = am; n <= p; ++n) {
                    const double t = sg * th[triIndex(n, am)];
                    const double2 v = Mi[coefIndex(n, m)];
                    acc.x += t * v.x;
                    acc.y += t * v.y;
                }
            }
            A[size_t(m + p) * kHfRows + ii] = acc;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < kHfRows * nph; e += blockDim.x) {
            const int ii = e / nph, j = e % nph, i = i0 + ii;
            if (i >= nth)
                continue;
            double2 acc = make_double2(0, 0);
            for (int m = -p; m <= p; ++m) {
                const int q = int(((long long)(m + nph) * j) % nph);
                acc = cadd(acc, cmul(A[size_t(m + p) * kHfRows + ii], root[q]));
            }
            out[size_t(i) * nph + j] = acc;
        }
        __syncthreads();
    }
}

// psi of every target node with links at the level (CTA: target x sample chunk):
// psi_o(s) = sum over its links T_class(s) sigma_source(s), in link order.
__global__ void __launch_bounds__(256) diagonalKernel(const uint32_t *__restrict__ linkStart,
                                                      const uint32_t *__restrict__ linkSource,
                                                      const uint32_t *__restrict__ linkClass,
                                                      const double2 *__restrict__ T, const double2 *__restrict__ sigma,
                                                      size_t Q, int nch, double2 *psi) {
    const uint32_t o = blockIdx.x;
    const size_t q = size_t(blockIdx.y) * blockDim.x + threadIdx.x;
    if (q >= Q)
        return;
    double2 acc[6];
#pragma unroll
    for (int c = 0; c < 6; ++c)
        acc[c] = make_double2(0, 0);
    for (uint32_t li = linkStart[o]; li < linkStart[o + 1]; ++li) {
        const double2 t = T[size_t(linkClass[li]) * Q + q];
        const double2 *src = sigma + size_t(linkSource[li]) * nch * Q + q;
#pragma unroll
        for (int c = 0; c < 6; ++c)
            if (c < nch)
                acc[c] = cadd(acc[c], cmul(t, src[size_t(c) * Q]));
    }
#pragma unroll
    for (int c = 0; c < 6; ++c)
        if (c < nch)
            psi[(size_t(o) * nch + c) * Q + q] = acc[c];
}

// L_nm += (-i)^n sum_i w_i Theta_n^m(x_i) (2 pi / nph) sum_j exp(-i m phi_j) psi(i, j)
// for each target node (CTA: target x channel).
__global__ void __launch_bounds__(256) projectKernel(const double2 *__restrict__ psi,
                                                     const uint32_t *__restrict__ outNodes,
                                                     const uint64_t *__restrict__ coefOffset, int p,
                                                     const double *__restrict__ theta,
                                                     const double *__restrict__ weights, int nth, int nph, int nch,
                                                     double2 *Lc) {
    extern __shared__ double smem[];
    const int nc = (p + 1) * (p + 1), tri = (p + 1) * (p + 2) / 2, mw = 2 * p + 1;
    double2 *acc = reinterpret_cast<double2 *>(smem);  // [nc]
    double2 *B = acc + nc;                             // [mw][kHfRows]
    double2 *root = B + size_t(mw) * kHfRows;
    const uint32_t o = blockIdx.x, ch = blockIdx.y;
    for (int i = threadIdx.x; i < nc; i += blockDim.x)
        acc[i] = make_double2(0, 0);
    for (int q = threadIdx.x; q < nph; q += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * q / nph, &sn, &cs);
        root[q] = make_double2(cs, sn);
    }
    __syncthreads();
    const size_t Q = size_t(nth) * nph;
    const double2 *in = psi + (size_t(o) * nch + ch) * Q;
    for (int i0 = 0; i0 < nth; i0 += kHfRows) {
        for (int e = threadIdx.x; e < mw * kHfRows; e += blockDim.x) {
            const int m = e % mw - p, ii = e / mw, i = i0 + ii;
            double2 b = make_double2(0, 0);
            if (i < nth) {
                const double2 *row = in + size_t(i) * nph;
                for (int j = 0; j < nph; ++j) {
                    const double2 r = root[int(((long long)(m + nph) * j) % nph)];
                    const double2 v = row[j];
                    b.x += v.x * r.x + v.y * r.y;  // v conj(r)
                    b.y += v.y * r.x - v.x * r.y;
                }
                b.x *= weights[i];
                b.y *= weights[i];
            }
            B[size_t(m + p) * kHfRows + ii] = b;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < nc; k += blockDim.x) {
            int n, m;
            decode(k, n, m);
            const int am = m < 0 ? -m : m;
            const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
            double2 a = acc[k];
            for (int ii = 0; ii < kHfRows && i0 + ii < nth; ++ii) {
                const double t = sg * theta[size_t(i0 + ii) * tri + triIndex(n, am)];
                const double2 b = B[size_t(m + p) * kHfRows + ii];
                a.x += t * b.x;
                a.y += t * b.y;
            }
            acc[k] = a;
        }
        __syncthreads();
    }
    double2 *L = Lc + coefOffset[outNodes[o]] + size_t(ch) * nc;
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
        int n, m;
        decode(k, n, m);
        const double2 v = acc[k];
        // (-i)^n: 1, -i, -1, i
        const int r = n & 3;
        const double2 w = r == 0 ? v : r == 1 ? make_double2(v.y, -v.x) : r == 2 ? make_double2(-v.x, -v.y)
                                                                        : make_double2(-v.y, v.x);
        L[k] = cadd(L[k], w);
    }
}

// T_class(s_q) = sum_{l<=p} coef[class][l] P_l(s_q . u_class), coef = (2l+1) (-i)^l h_l(k|t|)
// (one thread per class and sample).
__global__ void hfTransferKernel(uint32_t classes, const double *__restrict__ dirs, const double2 *__restrict__ coef,
                                 int p, const double *__restrict__ x, int nth, int nph, double2 *T) {
    const size_t Q = size_t(nth) * nph;
    const size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (e >= Q * classes)
        return;
    const uint32_t c = uint32_t(e / Q);
    const size_t q = e % Q;
    const int i = int(q / nph), j = int(q % nph);
    const double ct = x[i], st = sqrt(fmax(0.0, 1.0 - ct * ct));
    double sp, cp;
    sincospi(2.0 * j / nph, &sp, &cp);
    const double u = st * cp * dirs[3 * c] + st * sp * dirs[3 * c + 1] + ct * dirs[3 * c + 2];
    const double2 *cf = coef + size_t(c) * (p + 1);
    double p0 = 1.0, p1 = u;
    double2 acc = make_double2(cf[0].x, cf[0].y);
    if (p >= 1)
        acc = make_double2(acc.x + cf[1].x * u, acc.y + cf[1].y * u);
    for (int l = 2; l <= p; ++l) {
        const double p2 = ((2 * l - 1) * u * p1 - (l - 1) * p0) / l;
        acc.x += cf[l].x * p2;
        acc.y += cf[l].y * p2;
        p0 = p1;
        p1 = p2;
    }
    T[e] = acc;
}

// FP32 coaxial tables of the mixed form: each entry (class, |m|, n, n') of the
// FP64 table times exp(logRow[class][n'] + logCol[class][n]), the sigma factors
// that take the scaled input coefficient to its unscaled value and the
// unscaled output to its scaled value (the exponent split in two so that no
// FP64 intermediate overflows).
__global__ void coaxScaleKernel(uint32_t classes, const int *__restrict__ pin, const int *__restrict__ pout,
                                const uint64_t *__restrict__ start, const double2 *__restrict__ coax,
                                const double *__restrict__ logRow, const double *__restrict__ logCol, int stride,
                                float2 *coax32) {
    const uint32_t cls = blockIdx.y;
    if (cls >= classes)
        return;
    const int a = pin[cls], b = pout[cls];
    size_t total = 0;
    for (int j = 0; j <= min(a, b); ++j)
        total += size_t(a + 1 - j) * (b + 1 - j);
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        size_t off = 0;
        int mm = 0;
        while (off + size_t(a + 1 - mm) * (b + 1 - mm) <= e) {
            off += size_t(a + 1 - mm) * (b + 1 - mm);
            ++mm;
        }
        const size_t r = e - off;
        const int wo = b + 1 - mm;
        const int n = mm + int(r / wo), np = mm + int(r % wo);
        const double ex = logRow[size_t(cls) * stride + np] + logCol[size_t(cls) * stride + n];
        const double half = exp(0.5 * ex);
        const double2 v = coax[start[cls] + e];
        coax32[start[cls] + e] = make_float2(float(v.x * half * half), float(v.y * half * half));
    }
}

// ---------------------------------------------------------------- host math

// Gauss-Legendre nodes and weights on [-1, 1] by Newton iteration.
void gaussLegendre(int n, std::vector<double> &x, std::vector<double> &w) {
    x.resize(n);
    w.resize(n);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(kFmmPi * (i + 0.75) / (n + 0.5)), dp = 0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1, p1 = z;
            for (int j = 2; j <= n; ++j) {
                const double p2 = ((2.0 * j - 1) * z * p1 - (j - 1.0) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) {
                p1 = z;
                p0 = 1;
            }
            dp = n * (z * p1 - p0) / (z * z - 1);
            const double dz = p1 / dp;
            z -= dz;
            if (std::abs(dz) < 1e-16)
                break;
        }
        x[i] = z;
        w[i] = 2 / ((1 - z * z) * dp * dp);
    }
}

// Gaunt coefficients 2 pi int Theta_n^m Theta_l^0 Theta_n'^m, per (m, n, n') the
// values for l = |n - n'|, |n - n'| + 2, ..., n + n' (others vanish).
struct GauntTable {
    int P = -1;
    std::vector<double> values;
    std::vector<uint32_t> offsets;  // (m * (P + 1) + n) * (P + 1) + n'
};
const GauntTable &gauntTable(int P) {
    static std::mutex mu;
    static std::map<int, GauntTable> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto found = cache.find(P);
    if (found != cache.end())
        return found->second;
    GauntTable g;
    g.P = P;
    const int L = 2 * P;
    std::vector<double> xq, wq;
    gaussLegendre((3 * P) / 2 + 2, xq, wq);
    const size_t tri = size_t(L + 1) * (L + 2) / 2;
    std::vector<double> th(xq.size() * tri);
    for (size_t q = 0; q < xq.size(); ++q)
        for (int m = 0; m <= L; ++m)
            thetaColumn(m, L, xq[q], std::sqrt(std::max(0.0, 1 - xq[q] * xq[q])), th.data() + q * tri);
    g.offsets.assign(size_t(P + 1) * (P + 1) * (P + 1), 0);
    for (int m = 0; m <= P; ++m)
        for (int n = m; n <= P; ++n)
            for (int np = m; np <= P; ++np) {
                g.offsets[(size_t(m) * (P + 1) + n) * (P + 1) + np] = uint32_t(g.values.size());
                for (int l = std::abs(n - np); l <= n + np; l += 2) {
                    double s = 0;
                    for (size_t q = 0; q < xq.size(); ++q) {
                        const double *t = th.data() + q * tri;
                        s += wq[q] * t[triIndex(n, m)] * t[triIndex(l, 0)] * t[triIndex(np, m)];
                    }
                    g.values.push_back(2 * kFmmPi * s);
                }
            }
    return cache.emplace(P, std::move(g)).first->second;
}

// Wigner small-d blocks d^n[m, m'] (n <= P) for one polar angle.
void wignerBlocks(int P, double cosb, std::vector<double> &out) {
    const double sh = std::sqrt(std::max(0.0, (1 - cosb) / 2)), chh = std::sqrt(std::max(0.0, (1 + cosb) / 2));
    const size_t base = out.size();
    out.resize(base + wignerOffset(P + 1));
    for (int n = 0; n <= P; ++n) {
        const int w = 2 * n + 1;
        double *d = out.data() + base + wignerOffset(n);
        for (int m = -n; m <= n; ++m)
            for (int mp = -n; mp <= n; ++mp)
                d[size_t(m + n) * w + (mp + n)] = wignerSmallD(n, m, mp, cosb, sh, chh);
    }
}

// Per-class radial factors 4 pi f_l(k t) Y_l^0(z), l <= lmax (f = h or j).
void radialFactors(double kt, bool hankel, int lmax, std::complex<double> *f) {
    std::vector<double> j(lmax + 1), y(lmax + 1);
    besselJ(lmax, kt, j.data());
    if (hankel)
        besselY(lmax, kt, y.data());
    for (int l = 0; l <= lmax; ++l) {
        const double ylm0 = std::sqrt((2.0 * l + 1) / (4 * kFmmPi));
        f[l] = 4 * kFmmPi * ylm0 * std::complex<double>(j[l], hankel ? -y[l] : 0.0);
    }
}

int64_t gcd64(int64_t a, int64_t b) {
    a = std::llabs(a);
    b = std::llabs(b);
    while (b) {
        const int64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace

// -------------------------------------------------------------- the operator

struct FmmOperator::Impl {
    uint32_t N = 0, T = 0;
    std::vector<uint32_t> incOffsets;
    // per level (index = tree level): order, nodes with pressure supports
    int lmin = 0, lmax = -1;
    std::vector<int> order;
    std::vector<std::vector<uint32_t>> levelNodes;
    std::vector<std::vector<uint32_t>> leafNodes;  // leaves with pressure supports, per level
    std::vector<std::vector<uint32_t>> leafItemStart;
    std::vector<FmmItem> items;
    std::vector<uint32_t> itemBase;  // per level: first item of the level's leaf list
    // translations (host plans, per level)
    struct Plan {
        std::vector<uint32_t> outNodes, linkStart;
        std::vector<TransLink> links;
        std::vector<std::tuple<int, double, bool>> coaxUse;  // (level, distance, hankel) per coax class of the plan
    };
    std::vector<Plan> m2m, m2l, l2l;  // m2m[l]: parents at l; m2l[l]; l2l[l]: children at l
    std::vector<double> wclassCos;    // polar class -> cos(theta)
    std::vector<int> wclassP;         // polar class -> order needed (set in prepare)
    // device
    DevBuf panels, centers, coefOffset, incOff, far, y;
    DevBuf Mc, Lc, partial;
    DevBuf wigner, wignerStart, coax, coaxStart, coaxPin, coaxPout, fl, gaunt, gauntOff;
    DevBuf dItems;
    std::vector<uint64_t> hostCoefOffset;
    size_t coefTotal = 0;
    int wignerP = -1;
    int gauntP = -1;
    // plan buffers per (kind, level)
    struct DevPlan {
        DevBuf out, start, links;
        uint32_t count = 0;
    };
    std::vector<DevPlan> dm2m, dm2l, dl2l;
    // Grouped M2L per level: links in (polar class, coaxial class) order, the
    // groups as (first, count) in that order, and per mode (0: six channels,
    // 1: right-hand side) the chunks of the prepared order and whether the
    // level uses the grouped kernel (shared memory and slot buffer permitting).
    struct GroupPlan {
        DevBuf sorted;
        std::vector<std::pair<uint32_t, uint32_t>> groups;
        DevBuf chunks[2];
        uint32_t chunkCount[2] = {0, 0};
        int g[2] = {0, 0}, cpad[2] = {0, 0}, p = -1;
        bool active[2] = {false, false};
    };
    std::vector<GroupPlan> gm2l;
    DevBuf slots;  // per-link M2L contributions (largest grouped level)
    bool groupedM2l = true;
    std::vector<DevBuf> dLeaves, dLeafStart;
    std::vector<std::vector<uint32_t>> coaxClassOf;  // per kind*levels: local coax class index -> global
    // The far-field apply as a CUDA graph per mode (0: operator, 1: right-hand
    // side). After each prepare() the first apply of a mode runs its launches
    // directly (and sizes every buffer they use); the second is captured and
    // every later one replays the graph, the source and the result passing
    // through fixed staging buffers (the reference captures its M2L chunks the
    // same way on second contact, support_m2l_graph.hpp:52-78).
    // Mixed form (setFp32): scaled FP32 expansions. With a_l the level's node
    // radius and sigma_n = (2n+1)!! / (k a_l)^n, moments are stored as
    // M sigma_n and locals as L / sigma_n, both O(1) where the unscaled
    // coefficients span many decades (h_n(k t) reaches 1e75 at low k t); the
    // coaxial tables carry the matching factors, rotations act within a degree
    // and commute with them. P2M and L2P stay FP64 and convert at the boundary.
    bool fp32 = false;
    DevBuf Mc32, Lc32, partial32, coax32, wigner32, sigma, logRow, logCol;
    std::vector<double> hostWigner;
    bool wigner32Valid = false;
    int sigmaStride = 0;
    const double *levelSigma(int l) const { return fp32 ? sigma.as<double>() + size_t(l) * sigmaStride : nullptr; }
    // Plane-wave M2L per level: the offset class of every M2L link (offsets in
    // units of the level's cell width, so a handful of classes per level), the
    // link sources as indices into the level's node list, and the tables of the
    // prepared wavenumber. prepare() turns a level plane-wave when k times its
    // shortest M2L distance reaches hfThreshold and the diagonal form's roundoff
    // stays inside the expansion tolerance (FP64 operator only).
    struct HfLevel {
        bool active = false;
        int p = 0, nth = 0, nph = 0;
        std::vector<std::array<int64_t, 3>> offsets;
        DevBuf ids, linkSource, linkClass, theta, x, weights, coef, dirs, T, sigma, psi;
    };
    std::vector<HfLevel> hf;
    double hfThreshold = 8.0;
    double tolerance = 1e-8;  // expansion tolerance of the last prepare()
    DevBuf rule, l2pScratch;
    int rulePts = 0;
    unsigned panelDegree = 4;
    bool useGraphs = true;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint32_t applies[2] = {0, 0};
    DevBuf stageIn, stageOut;
    void dropGraphs() {
        for (auto &g : graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        applies[0] = applies[1] = 0;
    }
    ~Impl() { dropGraphs(); }
};

namespace {
uint64_t polarKey(int64_t x, int64_t y, int64_t z) {
    const int64_t n2 = x * x + y * y + z * z;
    if (z == 0)
        return 0;
    const int64_t z2 = z * z, g = gcd64(z2, n2);
    return (uint64_t(z > 0 ? 2 : 1) << 60) | (uint64_t(z2 / g) << 30) | uint64_t(n2 / g);
}
}  // namespace

FmmOperator::FmmOperator(const Space &space, const FmmTreeSettings &settings) : impl_(std::make_unique<Impl>()) {
    Impl &I = *impl_;
    I.N = uint32_t(space.vertices.size());
    I.T = uint32_t(space.panels.size());
    std::vector<double> V(3 * size_t(I.N));
    for (uint32_t v = 0; v < I.N; ++v) {
        V[3 * v] = space.vertices[v].x;
        V[3 * v + 1] = space.vertices[v].y;
        V[3 * v + 2] = space.vertices[v].z;
    }
    std::vector<uint32_t> tri(3 * size_t(I.T));
    for (uint32_t t = 0; t < I.T; ++t)
        for (int a = 0; a < 3; ++a)
            tri[3 * t + a] = space.panels[t].nodes[a];
    tree_ = buildSupportTree(V.data(), I.N, tri.data(), I.T, settings);
    I.incOffsets = space.incOffsets;
    const auto &nodes = tree_.nodes;
    const int levels = int(tree_.levels.size());
    // near CSR (rows i, columns of the near leaves' supports)
    {
        std::vector<std::vector<uint32_t>> nearSources(nodes.size());
        for (const auto &lk : tree_.ppNear)
            nearSources[lk.target].push_back(lk.source);
        nearRow_.assign(I.N + 1, 0);
        std::vector<std::vector<uint32_t>> rows(I.N);
        for (uint32_t ln = 0; ln < nodes.size(); ++ln) {
            if (nearSources[ln].empty())
                continue;
            std::vector<uint32_t> cols;
            for (uint32_t s : nearSources[ln])
                for (uint32_t q = nodes[s].firstP; q < nodes[s].firstP + nodes[s].countP; ++q)
                    cols.push_back(tree_.pressureOrder[q]);
            std::sort(cols.begin(), cols.end());
            for (uint32_t q = nodes[ln].firstP; q < nodes[ln].firstP + nodes[ln].countP; ++q)
                rows[tree_.pressureOrder[q]] = cols;
        }
        for (uint32_t i = 0; i < I.N; ++i)
            nearRow_[i + 1] = nearRow_[i] + uint32_t(rows[i].size());
        nearCol_.reserve(nearRow_[I.N]);
        for (uint32_t i = 0; i < I.N; ++i)
            nearCol_.insert(nearCol_.end(), rows[i].begin(), rows[i].end());
    }
    // near panel pairs: the panels of the stars of every near leaf pair, both orientations
    {
        std::vector<std::vector<uint32_t>> leafPanels(nodes.size());
        for (uint32_t ln = 0; ln < nodes.size(); ++ln) {
            if (!nodes[ln].leaf() || !nodes[ln].countP)
                continue;
            auto &ps = leafPanels[ln];
            for (uint32_t q = nodes[ln].firstP; q < nodes[ln].firstP + nodes[ln].countP; ++q) {
                const uint32_t v = tree_.pressureOrder[q];
                for (uint32_t j = space.incOffsets[v]; j < space.incOffsets[v + 1]; ++j)
                    ps.push_back(space.incPanel[j]);
            }
            std::sort(ps.begin(), ps.end());
            ps.erase(std::unique(ps.begin(), ps.end()), ps.end());
        }
        std::vector<std::vector<uint32_t>> rows(I.T);
        for (const auto &lk : tree_.ppNear)
            for (uint32_t a : leafPanels[lk.target]) {
                auto &r = rows[a];
                r.insert(r.end(), leafPanels[lk.source].begin(), leafPanels[lk.source].end());
                for (uint32_t b : leafPanels[lk.source])
                    rows[b].push_back(a);
            }
        panelRow_.assign(I.T + 1, 0);
        for (uint32_t a = 0; a < I.T; ++a) {
            auto &r = rows[a];
            std::sort(r.begin(), r.end());
            r.erase(std::unique(r.begin(), r.end()), r.end());
            panelRow_[a + 1] = panelRow_[a] + uint32_t(r.size());
        }
        panelCol_.reserve(panelRow_[I.T]);
        for (uint32_t a = 0; a < I.T; ++a) {
            for (uint32_t b : rows[a])
                if (a < b)
                    panelPairs_.emplace_back(a, b);
            panelCol_.insert(panelCol_.end(), rows[a].begin(), rows[a].end());
            std::vector<uint32_t>().swap(rows[a]);
        }
    }
    // levels taking part in the far field
    I.lmin = levels;
    I.lmax = -1;
    for (const auto &lk : tree_.ppFar) {
        I.lmin = std::min<int>(I.lmin, nodes[lk.target].level);
        I.lmax = std::max<int>(I.lmax, nodes[lk.target].level);
    }
    if (tree_.ppFar.empty())
        return;
    I.lmax = levels - 1;  // expansions reach every leaf below the coarsest far level
    I.levelNodes.assign(levels, {});
    I.leafNodes.assign(levels, {});
    I.leafItemStart.assign(levels, {});
    std::vector<uint64_t> coefSlot(nodes.size(), UINT64_MAX);
    for (int l = I.lmin; l < levels; ++l)
        for (uint32_t id : tree_.levels[l])
            if (nodes[id].countP)
                I.levelNodes[l].push_back(id);
    // items of the leaves (panels of the leaf's vertex stars, by panel id)
    I.dLeaves.resize(levels);
    I.dLeafStart.resize(levels);
    I.itemBase.assign(levels + 1, 0);
    for (int l = I.lmin; l < levels; ++l) {
        I.itemBase[l] = uint32_t(I.items.size());
        for (uint32_t id : I.levelNodes[l]) {
            if (!nodes[id].leaf())
                continue;
            I.leafNodes[l].push_back(id);
            I.leafItemStart[l].push_back(uint32_t(I.items.size()) - I.itemBase[l]);
            std::map<uint32_t, FmmItem> touched;
            for (uint32_t q = nodes[id].firstP; q < nodes[id].firstP + nodes[id].countP; ++q) {
                const uint32_t v = tree_.pressureOrder[q];
                for (uint32_t j = space.incOffsets[v]; j < space.incOffsets[v + 1]; ++j) {
                    const uint32_t t = space.incPanel[j];
                    const int a = space.incLocal[j];
                    auto &it = touched[t];
                    it.panel = t;
                    it.mask |= 1u << a;
                    it.inc[a] = j;
                }
            }
            for (auto &kv : touched)
                I.items.push_back(kv.second);
        }
        I.leafItemStart[l].push_back(uint32_t(I.items.size()) - I.itemBase[l]);
    }
    // translation plans with their polar and coaxial classes
    std::map<uint64_t, int> polar;
    const auto polarClass = [&](int64_t x, int64_t y, int64_t z) {
        const uint64_t key = polarKey(x, y, z);
        auto f = polar.find(key);
        if (f != polar.end())
            return f->second;
        const double c = z == 0 ? 0.0 : double(z) / std::sqrt(double(x * x + y * y + z * z));
        I.wclassCos.push_back(c);
        I.wclassP.push_back(0);
        return polar[key] = int(I.wclassCos.size()) - 1;
    };
    I.m2m.assign(levels, {});
    I.m2l.assign(levels, {});
    I.l2l.assign(levels, {});
    const auto widthOf = [&](int l) { return 2 * nodes[tree_.levels[l][0]].half; };
    // M2L: targets at level l with their far sources (sorted), coax class per distance
    {
        std::vector<std::vector<uint32_t>> farSources(nodes.size());
        for (const auto &lk : tree_.ppFar)
            farSources[lk.target].push_back(lk.source);
        for (int l = I.lmin; l < levels; ++l) {
            Impl::Plan &pl = I.m2l[l];
            std::map<int64_t, int> dist;
            const double w = widthOf(l);
            for (uint32_t id : I.levelNodes[l]) {
                auto &src = farSources[id];
                if (src.empty())
                    continue;
                std::sort(src.begin(), src.end());
                pl.outNodes.push_back(id);
                pl.linkStart.push_back(uint32_t(pl.links.size()));
                for (uint32_t s : src) {
                    const double d[3] = {nodes[id].center[0] - nodes[s].center[0],
                                         nodes[id].center[1] - nodes[s].center[1],
                                         nodes[id].center[2] - nodes[s].center[2]};
                    const int64_t ix = std::llround(d[0] / w), iy = std::llround(d[1] / w), iz = std::llround(d[2] / w);
                    const int64_t n2 = ix * ix + iy * iy + iz * iz;
                    auto f = dist.find(n2);
                    int cc;
                    if (f == dist.end()) {
                        cc = int(pl.coaxUse.size());
                        pl.coaxUse.emplace_back(l, std::sqrt(double(n2)) * w, true);
                        dist[n2] = cc;
                    } else
                        cc = f->second;
                    TransLink lk{s, uint32_t(polarClass(ix, iy, iz)), uint32_t(cc), 0, std::atan2(d[1], d[0])};
                    pl.links.push_back(lk);
                }
            }
            pl.linkStart.push_back(uint32_t(pl.links.size()));
        }
    }
    // M2M (parents at level l from children at l + 1) and L2L (children at l + 1 from parents at l)
    for (int l = I.lmin; l + 1 < levels; ++l) {
        Impl::Plan &up = I.m2m[l], &down = I.l2l[l + 1];
        const double h = 0.5 * widthOf(l + 1);  // child half width
        up.coaxUse.emplace_back(l, std::sqrt(3.0) * h, false);
        down.coaxUse.emplace_back(l + 1, std::sqrt(3.0) * h, false);
        for (uint32_t id : I.levelNodes[l]) {
            if (nodes[id].leaf())
                continue;
            up.outNodes.push_back(id);
            up.linkStart.push_back(uint32_t(up.links.size()));
            for (uint32_t c : nodes[id].child) {
                if (c == kNoNode || !nodes[c].countP)
                    continue;
                const double d[3] = {nodes[id].center[0] - nodes[c].center[0], nodes[id].center[1] - nodes[c].center[1],
                                     nodes[id].center[2] - nodes[c].center[2]};
                const int64_t ix = d[0] > 0 ? 1 : -1, iy = d[1] > 0 ? 1 : -1, iz = d[2] > 0 ? 1 : -1;
                up.links.push_back({c, uint32_t(polarClass(ix, iy, iz)), 0, 0, std::atan2(d[1], d[0])});
                down.outNodes.push_back(c);
                down.linkStart.push_back(uint32_t(down.links.size()));
                down.links.push_back({id, uint32_t(polarClass(-ix, -iy, -iz)), 0, 0, std::atan2(-d[1], -d[0])});
            }
        }
        up.linkStart.push_back(uint32_t(up.links.size()));
        down.linkStart.push_back(uint32_t(down.links.size()));
    }
    // geometry upload
    std::vector<FmmPanel> fp(I.T);
    for (uint32_t t = 0; t < I.T; ++t) {
        const HostPanel &hp = space.panels[t];
        FmmPanel &q = fp[t];
        const double v0[3] = {hp.v[0].x, hp.v[0].y, hp.v[0].z};
        const double v1[3] = {hp.v[1].x, hp.v[1].y, hp.v[1].z};
        const double v2[3] = {hp.v[2].x, hp.v[2].y, hp.v[2].z};
        for (int d = 0; d < 3; ++d) {
            q.v0[d] = v0[d];
            q.e1[d] = v1[d] - v0[d];
            q.e2[d] = v2[d] - v0[d];
        }
        q.n[0] = hp.n.x;
        q.n[1] = hp.n.y;
        q.n[2] = hp.n.z;
        for (int a = 0; a < 3; ++a) {
            q.curl[3 * a] = hp.curl[a].x;
            q.curl[3 * a + 1] = hp.curl[a].y;
            q.curl[3 * a + 2] = hp.curl[a].z;
            q.nodes[a] = hp.nodes[a];
        }
        q.area = hp.area;
    }
    cudaStream_t s = nullptr;
    uploadVec(I.panels, fp, s);
    std::vector<double> cen(3 * nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i)
        for (int d = 0; d < 3; ++d)
            cen[3 * i + d] = nodes[i].center[d];
    uploadVec(I.centers, cen, s);
    uploadVec(I.incOff, I.incOffsets, s);
    uploadVec(I.dItems, I.items, s);
    I.dm2m.resize(levels);
    I.dm2l.resize(levels);
    I.dl2l.resize(levels);
    for (int l = I.lmin; l < levels; ++l) {
        uploadVec(I.dLeaves[l], I.leafNodes[l], s);
        uploadVec(I.dLeafStart[l], I.leafItemStart[l], s);
        const auto put = [&](Impl::DevPlan &d, const Impl::Plan &p) {
            d.count = uint32_t(p.outNodes.size());
            uploadVec(d.out, p.outNodes, s);
            uploadVec(d.start, p.linkStart, s);
            uploadVec(d.links, p.links, s);
        };
        put(I.dm2m[l], I.m2m[l]);
        put(I.dm2l[l], I.m2l[l]);
        put(I.dl2l[l], I.l2l[l]);
    }
    // grouped M2L: links sorted by (polar class, coaxial class, link index)
    I.gm2l.resize(levels);
    for (int l = I.lmin; l < levels; ++l) {
        const auto &lk = I.m2l[l].links;
        if (lk.empty())
            continue;
        std::vector<uint32_t> order(lk.size());
        for (uint32_t i = 0; i < order.size(); ++i)
            order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            return lk[a].wclass != lk[b].wclass ? lk[a].wclass < lk[b].wclass : lk[a].cclass < lk[b].cclass;
        });
        Impl::GroupPlan &gp = I.gm2l[l];
        for (uint32_t i = 0; i < order.size();) {
            uint32_t j = i + 1;
            while (j < order.size() && lk[order[j]].wclass == lk[order[i]].wclass &&
                   lk[order[j]].cclass == lk[order[i]].cclass)
                ++j;
            gp.groups.emplace_back(i, j - i);
            i = j;
        }
        uploadVec(gp.sorted, order, s);
    }
    // plane-wave link classes (offset vectors of the M2L links, per level)
    I.hf.resize(levels);
    for (int l = I.lmin; l < levels; ++l) {
        const Impl::Plan &pl = I.m2l[l];
        if (pl.links.empty())
            continue;
        Impl::HfLevel &h = I.hf[l];
        std::map<uint32_t, uint32_t> index;
        for (uint32_t i = 0; i < I.levelNodes[l].size(); ++i)
            index[I.levelNodes[l][i]] = i;
        std::map<std::array<int64_t, 3>, uint32_t> cls;
        std::vector<uint32_t> src, cl;
        const double w = widthOf(l);
        for (size_t o = 0; o + 1 < pl.linkStart.size(); ++o)
            for (uint32_t li = pl.linkStart[o]; li < pl.linkStart[o + 1]; ++li) {
                const uint32_t sid = pl.links[li].source, tid = pl.outNodes[o];
                std::array<int64_t, 3> off;
                for (int d = 0; d < 3; ++d)
                    off[d] = std::llround((nodes[tid].center[d] - nodes[sid].center[d]) / w);
                const auto f = cls.emplace(off, uint32_t(h.offsets.size()));
                if (f.second)
                    h.offsets.push_back(off);
                cl.push_back(f.first->second);
                src.push_back(index.at(sid));
            }
        uploadVec(h.ids, I.levelNodes[l], s);
        uploadVec(h.linkSource, src, s);
        uploadVec(h.linkClass, cl, s);
    }
    setPanelDegree(4, nullptr);
    fmmCheck(cudaDeviceSynchronize(), "setup");
    I.far.ensure(3 * size_t(I.T) * 16);
}

FmmOperator::~FmmOperator() = default;

void FmmOperator::setPanelDegree(unsigned degree, cudaStream_t stream) {
    Impl &I = *impl_;
    const std::vector<TriPoint> rule = triangleRule(degree);
    double ws = 0;
    for (const auto &r : rule)
        ws += r.w;
    std::vector<double> hr(4 * rule.size());
    for (size_t q = 0; q < rule.size(); ++q) {
        hr[4 * q] = rule[q].b[0];
        hr[4 * q + 1] = rule[q].b[1];
        hr[4 * q + 2] = rule[q].b[2];
        hr[4 * q + 3] = rule[q].w / ws;
    }
    // ordered after the work already queued on `stream` that reads the old rule
    uploadVec(I.rule, hr, stream);
    fmmCheck(cudaStreamSynchronize(stream), "rule upload");
    I.rulePts = int(rule.size());
    I.panelDegree = degree;
    I.dropGraphs();
}

unsigned FmmOperator::panelDegree() const { return impl_->panelDegree; }

void FmmOperator::setFp32(bool enabled) {
    impl_->fp32 = enabled;
    impl_->dropGraphs();
}

void FmmOperator::setHfThreshold(double threshold) {
    impl_->hfThreshold = threshold;
    impl_->dropGraphs();
}

void FmmOperator::setGroupedM2l(bool enabled) {
    impl_->groupedM2l = enabled;
    impl_->dropGraphs();
}

// Plane-wave levels of the prepared wavenumber and their tables: the sphere
// rule (Gauss-Legendre in cos(theta) with ceil((3p+2)/2) nodes, 3p+2 uniform
// azimuths: exact for the degree 3p of sigma T conj(Y)), Theta_n^m at the rule's
// rows, and T of every offset class.
void FmmOperator::prepareHf(cudaStream_t stream) {
    Impl &I = *impl_;
    const int levels = int(tree_.levels.size());
    for (int l = I.lmin; l < levels; ++l) {
        Impl::HfLevel &h = I.hf[l];
        h.active = false;
        if (I.fp32 || h.offsets.empty() || I.order[l] < 8)
            continue;
        const double w = 2 * tree_.nodes[tree_.levels[l][0]].half;
        double tmin = 1e300;
        for (const auto &o : h.offsets)
            tmin = std::min(tmin, w * std::sqrt(double(o[0] * o[0] + o[1] * o[1] + o[2] * o[2])));
        if (k_ * tmin < I.hfThreshold)
            continue;
        const int p = I.order[l];
        // Diagonal-stability guard: the transfer sum carries terms up to
        // (2p+1)|h_p(k t)|, which for p > k t grow far beyond the result (about
        // |h_0(k t)| = 1 / (k t)); their FP64 roundoff, eps (2p+1) |h_p(k t_min)| k t_min
        // relative, must stay within the expansion tolerance, or the level keeps the
        // rotational form (measured plane-wave errors sit at or below this estimate).
        {
            std::vector<double> yb(p + 1);
            besselY(p, k_ * tmin, yb.data());
            const double amplification = double(2 * p + 1) * std::fabs(yb[p]) * k_ * tmin;
            if (!(std::numeric_limits<double>::epsilon() * amplification <= I.tolerance))
                continue;
        }
        h.active = true;
        h.p = p;
        h.nth = (3 * p + 3) / 2;
        h.nph = 3 * p + 2;
        std::vector<double> gx, gw;
        gaussLegendre(h.nth, gx, gw);
        const size_t tri = size_t(p + 1) * (p + 2) / 2;
        std::vector<double> theta(size_t(h.nth) * tri), weights(h.nth);
        for (int i = 0; i < h.nth; ++i) {
            const double st = std::sqrt(std::max(0.0, 1 - gx[i] * gx[i]));
            for (int m = 0; m <= p; ++m)
                thetaColumn(m, p, gx[i], st, theta.data() + size_t(i) * tri);
            weights[i] = gw[i] * 2 * kFmmPi / h.nph;
        }
        uploadVec(h.theta, theta, stream);
        uploadVec(h.x, gx, stream);
        uploadVec(h.weights, weights, stream);
        // T coefficients per class: (2l+1) (-i)^l h_l(k |t|), h_l = j_l - i y_l
        const size_t classes = h.offsets.size();
        std::vector<double> dirs(3 * classes);
        std::vector<std::complex<double>> coef(classes * (p + 1));
        std::vector<double> jb(p + 1), yb(p + 1);
        for (size_t c = 0; c < classes; ++c) {
            const auto &o = h.offsets[c];
            const double len = std::sqrt(double(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]));
            for (int d = 0; d < 3; ++d)
                dirs[3 * c + d] = double(o[d]) / len;
            const double kt = k_ * len * w;
            besselJ(p, kt, jb.data());
            besselY(p, kt, yb.data());
            for (int n = 0; n <= p; ++n) {
                const std::complex<double> hn(jb[n], -yb[n]);
                const std::complex<double> mi[4] = {{1, 0}, {0, -1}, {-1, 0}, {0, 1}};
                coef[c * (p + 1) + n] = double(2 * n + 1) * mi[n & 3] * hn;
            }
        }
        uploadVec(h.dirs, dirs, stream);
        uploadVec(h.coef, coef, stream);
        const size_t Q = size_t(h.nth) * h.nph;
        h.T.ensure(classes * Q * 16);
        hfTransferKernel<<<unsigned((classes * Q + 255) / 256), 256, 0, stream>>>(
            uint32_t(classes), h.dirs.as<double>(), h.coef.as<double2>(), p, h.x.as<double>(), h.nth, h.nph,
            h.T.as<double2>());
        fmmCheck(cudaGetLastError(), "plane-wave transfer launch");
        h.sigma.ensure(I.levelNodes[l].size() * 6 * Q * 16);
        h.psi.ensure(I.m2l[l].outNodes.size() * 6 * Q * 16);
    }
}

void FmmOperator::setGraphs(bool enabled) {
    impl_->useGraphs = enabled;
    impl_->dropGraphs();
}

void FmmOperator::prepare(double k, double tolerance, cudaStream_t stream) {
    Impl &I = *impl_;
    I.dropGraphs();  // the tables and orders below change what a graph would replay
    k_ = k;
    levelInfo_.clear();
    if (tree_.ppFar.empty())
        return;
    const auto &nodes = tree_.nodes;
    const int levels = int(tree_.levels.size());
    const double d0 = -std::log10(std::clamp(tolerance, 1e-15, 1e-2));
    I.tolerance = tolerance;
    I.order.assign(levels, 0);
    for (int l = I.lmin; l < levels; ++l) {
        double r = 0;
        for (uint32_t id : I.levelNodes[l])
            r = std::max(r, nodes[id].radiusP);
        const double kd = 2 * k * r;
        const int hf = int(std::ceil(kd + 1.8 * std::pow(d0, 2.0 / 3.0) * std::cbrt(kd)));
        const int lf = int(std::ceil(1.3 * d0)) + 1;
        I.order[l] = std::min(kFmmMaxOrder, std::max(hf, lf));
        levelInfo_.push_back({uint32_t(l), uint32_t(I.order[l]), uint32_t(I.levelNodes[l].size()),
                              uint32_t(I.m2l[l].links.size()), r, 0});
    }
    // coefficient storage: 6 channels per node of every taking part level
    I.hostCoefOffset.assign(nodes.size(), 0);
    size_t at = 0;
    for (int l = I.lmin; l < levels; ++l) {
        const size_t nc = size_t(I.order[l] + 1) * (I.order[l] + 1);
        for (uint32_t id : I.levelNodes[l]) {
            I.hostCoefOffset[id] = at;
            at += 6 * nc;
        }
    }
    I.coefTotal = at;
    I.Mc.ensure(at * 16);
    I.Lc.ensure(at * 16);
    uploadVec(I.coefOffset, I.hostCoefOffset, stream);
    // Wigner tables (per polar class, to the largest order it meets)
    std::vector<int> need(I.wclassCos.size(), 0);
    for (int l = I.lmin; l < levels; ++l) {
        for (const auto &lk : I.m2l[l].links)
            need[lk.wclass] = std::max(need[lk.wclass], I.order[l]);
        for (const auto &lk : I.m2m[l].links)
            need[lk.wclass] = std::max({need[lk.wclass], I.order[l], I.order[l + 1]});
        for (const auto &lk : I.l2l[l].links)
            need[lk.wclass] = std::max({need[lk.wclass], I.order[l], I.order[l - 1]});
    }
    bool grow = false;
    for (size_t c = 0; c < need.size(); ++c)
        grow |= need[c] > I.wclassP[c];
    if (grow) {
        std::vector<double> tab;
        std::vector<uint64_t> start;
        for (size_t c = 0; c < need.size(); ++c) {
            I.wclassP[c] = std::max(I.wclassP[c], need[c]);
            start.push_back(tab.size());
            wignerBlocks(I.wclassP[c], I.wclassCos[c], tab);
        }
        uploadVec(I.wigner, tab, stream);
        uploadVec(I.wignerStart, start, stream);
        I.hostWigner = std::move(tab);
        I.wigner32Valid = false;
    }
    // coaxial classes of this wavenumber
    int P = 0;
    for (int l = I.lmin; l < levels; ++l)
        P = std::max(P, I.order[l]);
    const GauntTable &g = gauntTable(P);
    if (I.gauntP != P) {
        uploadVec(I.gaunt, g.values, stream);
        uploadVec(I.gauntOff, g.offsets, stream);
        I.gauntP = P;
    }
    std::vector<int> pin, pout;
    std::vector<uint64_t> start;
    std::vector<std::complex<double>> fl;
    const int lmaxF = 2 * P;
    uint64_t total = 0;
    const auto addClass = [&](int a, int b, double t, bool hankel) {
        pin.push_back(a);
        pout.push_back(b);
        start.push_back(total);
        for (int j = 0; j <= std::min(a, b); ++j)
            total += uint64_t(a + 1 - j) * (b + 1 - j);
        const size_t at0 = fl.size();
        fl.resize(at0 + lmaxF + 1);
        radialFactors(k * t, hankel, lmaxF, fl.data() + at0);
        return uint32_t(pin.size() - 1);
    };
    I.coaxClassOf.assign(3 * levels, {});
    // per class: (level, sign) of the log-sigma factor of its output degree and of its input degree
    std::vector<std::pair<int, int>> rowScale, colScale;
    for (int l = I.lmin; l < levels; ++l) {
        for (const auto &u : I.m2l[l].coaxUse) {  // M = M^ / sigma_l in, L^ = L / sigma_l out
            I.coaxClassOf[l].push_back(addClass(I.order[l], I.order[l], std::get<1>(u), true));
            rowScale.push_back({l, -1});
            colScale.push_back({l, -1});
        }
        for (const auto &u : I.m2m[l].coaxUse) {  // child moments M^ / sigma_(l+1) in, M sigma_l out
            I.coaxClassOf[levels + l].push_back(addClass(I.order[l + 1], I.order[l], std::get<1>(u), false));
            rowScale.push_back({l, 1});
            colScale.push_back({l + 1, -1});
        }
        for (const auto &u : I.l2l[l].coaxUse) {  // parent locals L^ sigma_(l-1) in, L / sigma_l out
            I.coaxClassOf[2 * levels + l].push_back(addClass(I.order[l - 1], I.order[l], std::get<1>(u), false));
            rowScale.push_back({l, -1});
            colScale.push_back({l - 1, 1});
        }
    }
    uploadVec(I.coaxPin, pin, stream);
    uploadVec(I.coaxPout, pout, stream);
    uploadVec(I.coaxStart, start, stream);
    uploadVec(I.fl, fl, stream);
    I.coax.ensure(total * 16);
    coaxKernel<<<dim3(64, uint32_t(pin.size())), 256, 0, stream>>>(
        uint32_t(pin.size()), I.coaxPin.as<int>(), I.coaxPout.as<int>(), I.coaxStart.as<uint64_t>(),
        I.fl.as<double2>(), lmaxF, I.gaunt.as<double>(), I.gauntOff.as<uint32_t>(), P, I.coax.as<double2>());
    fmmCheck(cudaGetLastError(), "coaxial table launch");
    prepareHf(stream);
    for (auto &info : levelInfo_)
        info.planeWave = I.hf[info.level].active ? 1 : 0;
    if (I.fp32) {
        // log sigma_n per level, sigma_n = (2n+1)!! / (k a_l)^n with a_l the level's node radius
        const int stride = P + 1;
        std::vector<double> logSigma(size_t(levels) * stride, 0.0), sigma(size_t(levels) * stride, 1.0);
        for (const auto &info : levelInfo_) {
            const double lka = std::log(std::max(k * info.radius, 1e-300));
            double lf = 0;  // log (2n+1)!!
            for (int n = 0; n <= P; ++n) {
                if (n)
                    lf += std::log(2.0 * n + 1);
                const double v = std::clamp(lf - n * lka, -600.0, 600.0);
                logSigma[size_t(info.level) * stride + n] = v;
                sigma[size_t(info.level) * stride + n] = std::exp(v);
            }
        }
        I.sigmaStride = stride;
        uploadVec(I.sigma, sigma, stream);
        std::vector<double> lr(pin.size() * stride), lc(pin.size() * stride);
        for (size_t c = 0; c < pin.size(); ++c)
            for (int n = 0; n <= P; ++n) {
                lr[c * stride + n] = rowScale[c].second * logSigma[size_t(rowScale[c].first) * stride + n];
                lc[c * stride + n] = colScale[c].second * logSigma[size_t(colScale[c].first) * stride + n];
            }
        uploadVec(I.logRow, lr, stream);
        uploadVec(I.logCol, lc, stream);
        I.coax32.ensure(std::max<uint64_t>(total, 1) * 8);
        coaxScaleKernel<<<dim3(64, uint32_t(pin.size())), 256, 0, stream>>>(
            uint32_t(pin.size()), I.coaxPin.as<int>(), I.coaxPout.as<int>(), I.coaxStart.as<uint64_t>(),
            I.coax.as<double2>(), I.logRow.as<double>(), I.logCol.as<double>(), stride, I.coax32.as<float2>());
        fmmCheck(cudaGetLastError(), "scaled coaxial table launch");
        if (!I.wigner32Valid) {
            std::vector<float> w32(I.hostWigner.begin(), I.hostWigner.end());
            uploadVec(I.wigner32, w32, stream);
            I.wigner32Valid = true;
        }
        I.Mc32.ensure(std::max<size_t>(at, 1) * 8);
        I.Lc32.ensure(std::max<size_t>(at, 1) * 8);
    }
    // local coax class ids -> global ids in the link lists
    for (int l = I.lmin; l < levels; ++l) {
        const auto remap = [&](const Impl::Plan &pl, Impl::DevPlan &d, const std::vector<uint32_t> &cls) {
            if (pl.links.empty())
                return;
            std::vector<TransLink> links = pl.links;
            for (auto &lk : links)
                lk.cclass = cls[lk.cclass];
            uploadVec(d.links, links, stream);
        };
        remap(I.m2l[l], I.dm2l[l], I.coaxClassOf[l]);
        remap(I.m2m[l], I.dm2m[l], I.coaxClassOf[levels + l]);
        remap(I.l2l[l], I.dl2l[l], I.coaxClassOf[2 * levels + l]);
    }
    // Grouped M2L of the rotational levels, per mode: the largest chunk whose
    // buffers fit 110 KB of shared memory (two CTAs per SM), else single links
    // up to the opt-in limit; the slot buffer of the largest level must stay
    // within a quarter of the free memory (24 GB at most), else the level runs
    // the per-target translation kernel.
    {
        const size_t cb = I.fp32 ? 8 : 16;
        size_t freeBytes = 0, totalBytes = 0;
        if (cudaMemGetInfo(&freeBytes, &totalBytes) != cudaSuccess)
            freeBytes = 0;
        const size_t cap = std::min<size_t>(size_t(24) << 30, freeBytes / 4 + I.slots.bytes);
        size_t slotBytes = 0;
        for (int l = I.lmin; l < levels; ++l) {
            Impl::GroupPlan &gp = I.gm2l[l];
            gp.active[0] = gp.active[1] = false;
            if (gp.groups.empty() || !I.groupedM2l || I.hf[l].active)
                continue;
            const int p = I.order[l];
            const size_t nc = size_t(p + 1) * (p + 1), links = I.m2l[l].links.size();
            for (int mode = 0; mode < 2; ++mode) {
                const int nch = mode == 0 ? 6 : 1;
                int g = 0, cpad = 0;
                for (int cand = 16; cand >= 1 && !g; --cand)
                    if (groupSmemBytes(p, (cand * nch) | 1, cand, cb) <= 110 * 1024) {
                        g = cand;
                        cpad = (cand * nch) | 1;
                    }
                if (!g && groupSmemBytes(p, nch | 1, 1, cb) <= kMaxShared) {
                    g = 1;
                    cpad = nch | 1;
                }
                const size_t need = links * nch * nc * cb;
                if (!g || need > cap)
                    continue;
                slotBytes = std::max(slotBytes, need);
                if (gp.g[mode] != g) {
                    std::vector<uint2> chunks;
                    for (const auto &[first, count] : gp.groups)
                        for (uint32_t o = 0; o < count; o += uint32_t(g))
                            chunks.push_back(make_uint2(first + o, std::min<uint32_t>(uint32_t(g), count - o)));
                    uploadVec(gp.chunks[mode], chunks, stream);
                    gp.chunkCount[mode] = uint32_t(chunks.size());
                    gp.g[mode] = g;
                }
                gp.cpad[mode] = cpad;
                gp.active[mode] = true;
            }
        }
        I.slots.ensure(slotBytes);
    }
    fmmCheck(cudaStreamSynchronize(stream), "prepare");
}

void FmmOperator::applyFar(const double *p, size_t stride, uint32_t S, double *y, cudaStream_t stream,
                           KernelTimer *timer) {
    for (uint32_t sys = 0; sys < S; ++sys)
        run(p + sys * stride, false, y + size_t(sys) * impl_->N * 2, stream, timer);
}

void FmmOperator::applyFarRhs(const double *q, uint32_t S, double *y, cudaStream_t stream, KernelTimer *timer) {
    for (uint32_t sys = 0; sys < S; ++sys)
        run(q + size_t(sys) * impl_->T * 2, true, y + size_t(sys) * impl_->N * 2, stream, timer);
}

void FmmOperator::run(const double *src, bool rhs, double *y, cudaStream_t stream, KernelTimer *timer) {
    Impl &I = *impl_;
    const int mode = rhs ? 1 : 0;
    const bool capturable = stream != nullptr && stream != cudaStreamLegacy && stream != cudaStreamPerThread;
    // with kernel profiling on, plain launches keep every family's time
    const bool profiling = timer && timer->enabled();
    if (!I.useGraphs || !capturable || profiling || tree_.ppFar.empty() ||
        (!I.graph[mode] && I.applies[mode]++ == 0)) {
        launchApply(src, rhs, y, stream, timer);
        return;
    }
    const size_t inBytes = size_t(rhs ? I.T : I.N) * 16, outBytes = size_t(I.N) * 16;
    if (!I.graph[mode]) {
        I.stageIn.ensure(size_t(std::max(I.T, I.N)) * 16);  // allocated before the capture
        I.stageOut.ensure(outBytes);
        cudaGraph_t g = nullptr;
        fmmCheck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed), "far-field graph capture");
        try {
            launchApply(I.stageIn.as<double>(), rhs, I.stageOut.as<double>(), stream, nullptr);
        } catch (...) {
            cudaStreamEndCapture(stream, &g);
            if (g)
                cudaGraphDestroy(g);
            throw;
        }
        fmmCheck(cudaStreamEndCapture(stream, &g), "far-field graph capture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        fmmCheck(e, "far-field graph instantiation");
        I.graph[mode] = exec;
    }
    TimedScope scope(timer, "fmm_far_graph", stream);
    fmmCheck(cudaMemcpyAsync(I.stageIn.p, src, inBytes, cudaMemcpyDeviceToDevice, stream), "far-field graph input");
    fmmCheck(cudaGraphLaunch(I.graph[mode], stream), "far-field graph launch");
    fmmCheck(cudaMemcpyAsync(y, I.stageOut.p, outBytes, cudaMemcpyDeviceToDevice, stream), "far-field graph output");
}

// M2L of one plane-wave level: signatures of the level's nodes, the diagonal
// products along the links, projection of each target's field onto its locals.
void FmmOperator::planeWaveM2L(int l, int nch, cudaStream_t stream) {
    Impl &I = *impl_;
    Impl::HfLevel &h = I.hf[l];
    const int p = h.p, nc = (p + 1) * (p + 1), mw = 2 * p + 1;
    const size_t Q = size_t(h.nth) * h.nph;
    const size_t sm = (size_t(nc) + size_t(mw) * kHfRows + h.nph) * 16;
    if (sm > kMaxShared)
        throw Unsupported("Fast-multipole plane-wave order exceeds the shared-memory tables; refine the tree.");
    fmmCheck(cudaFuncSetAttribute(signatureKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)), "signature smem");
    fmmCheck(cudaFuncSetAttribute(projectKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)), "project smem");
    const uint32_t nodes = uint32_t(I.levelNodes[l].size()), outs = I.dm2l[l].count;
    signatureKernel<<<dim3(nodes, nch), 256, sm, stream>>>(I.Mc.as<double2>(), I.coefOffset.as<uint64_t>(),
                                                           h.ids.as<uint32_t>(), p, h.theta.as<double>(), h.nth, h.nph,
                                                           nch, h.sigma.as<double2>());
    diagonalKernel<<<dim3(outs, unsigned((Q + 255) / 256)), 256, 0, stream>>>(
        I.dm2l[l].start.as<uint32_t>(), h.linkSource.as<uint32_t>(), h.linkClass.as<uint32_t>(), h.T.as<double2>(),
        h.sigma.as<double2>(), Q, nch, h.psi.as<double2>());
    projectKernel<<<dim3(outs, nch), 256, sm, stream>>>(h.psi.as<double2>(), I.dm2l[l].out.as<uint32_t>(),
                                                        I.coefOffset.as<uint64_t>(), p, h.theta.as<double>(),
                                                        h.weights.as<double>(), h.nth, h.nph, nch, I.Lc.as<double2>());
    fmmCheck(cudaGetLastError(), "plane-wave M2L launch");
}

void FmmOperator::launchApply(const double *src, bool rhs, double *y, cudaStream_t stream, KernelTimer *timer) {
    Impl &I = *impl_;
    const uint32_t N = I.N;
    const double2 *pv = reinterpret_cast<const double2 *>(src);
    double2 *yv = reinterpret_cast<double2 *>(y);
    if (tree_.ppFar.empty()) {
        fmmCheck(cudaMemsetAsync(yv, 0, size_t(N) * 16, stream), "zero far");
        return;
    }
    const int nch = rhs ? 1 : 6;
    const int levels = int(tree_.levels.size());
    fmmCheck(cudaMemsetAsync(I.far.p, 0, 3 * size_t(I.T) * 16, stream), "zero contributions");
    if (I.fp32)
        fmmCheck(cudaMemsetAsync(I.Lc32.p, 0, I.coefTotal * 8, stream), "zero locals");
    else
        fmmCheck(cudaMemsetAsync(I.Lc.p, 0, I.coefTotal * 16, stream), "zero locals");
    // channels per CTA: enough CTAs for about four waves of 148 SMs, fewer
    // (more reuse of each Wigner and coaxial entry) when the level has many nodes
    const auto translate = [&](Impl::DevPlan &d, int pin, int pout, auto *in, auto *out, bool zero) {
        using CT = std::remove_cv_t<std::remove_pointer_t<decltype(out)>>;
        using RT = decltype(CT{}.x);
        constexpr bool f32 = std::is_same_v<RT, float>;
        if (!d.count)
            return;
        const int nmax = std::max((pin + 1) * (pin + 1), (pout + 1) * (pout + 1)), nout = (pout + 1) * (pout + 1);
        // all channels in one CTA where shared memory allows two CTAs per SM (each
        // Wigner and coaxial entry then serves every channel), links split over K
        // CTAs per output node for about eight CTAs per SM
        const auto bytes = [&](int c) { return (size_t(3) * c * nmax + std::max(pin, pout) + 1) * sizeof(CT); };
        int cpc = nch == 1 ? 1 : 6;
        while (cpc > 1 && bytes(cpc) > 110 * 1024)
            cpc = cpc == 6 ? 3 : cpc == 3 ? 2 : 1;
        const size_t sm = bytes(cpc);
        const unsigned groups = unsigned((nch + cpc - 1) / cpc);
        const int K = int(std::clamp<size_t>((size_t(148) * 8 + d.count * groups - 1) / (d.count * groups), 1, 8));
        DevBuf &partial = f32 ? I.partial32 : I.partial;
        if (K > 1)
            partial.ensure(size_t(d.count) * K * 6 * nout * sizeof(CT));
        const RT *wig;
        const CT *cx;
        if constexpr (f32) {
            wig = I.wigner32.as<float>();
            cx = I.coax32.as<float2>();
        } else {
            wig = I.wigner.as<double>();
            cx = I.coax.as<double2>();
        }
        const dim3 grid(d.count * K, groups);
        const auto launch = [&](auto kernel) {
            fmmCheck(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)),
                     "translate smem");
            kernel<<<grid, 256, sm, stream>>>(d.out.as<uint32_t>(), d.start.as<uint32_t>(), d.links.as<TransLink>(),
                                              pin, pout, in, out, I.coefOffset.as<uint64_t>(), wig,
                                              I.wignerStart.as<uint64_t>(), cx, I.coaxStart.as<uint64_t>(),
                                              zero ? 1 : 0, nch, K, partial.as<CT>());
        };
        if (cpc == 6)
            launch(translateKernel<6, RT>);
        else if (cpc == 3)
            launch(translateKernel<3, RT>);
        else if (cpc == 2)
            launch(translateKernel<2, RT>);
        else
            launch(translateKernel<1, RT>);
        fmmCheck(cudaGetLastError(), "translate launch");
        if (K > 1) {
            reduceKernel<RT><<<d.count, 256, 0, stream>>>(d.out.as<uint32_t>(), I.coefOffset.as<uint64_t>(),
                                                          partial.as<CT>(), K, nout, nch, zero ? 1 : 0, out);
            fmmCheck(cudaGetLastError(), "translate reduce launch");
        }
    };
    {
        TimedScope scope(timer, "fmm_p2m", stream);
        for (int l = I.lmin; l < levels; ++l) {
            const uint32_t leaves = uint32_t(I.leafNodes[l].size());
            if (!leaves)
                continue;
            const int P = I.order[l];
            const size_t td = tableDoubles(P);
            const size_t sm = (kWarps * td) * 8 + kWarps * 6 * 16;
            if (sm > kMaxShared)
                throw Unsupported("Fast-multipole leaf order exceeds the shared-memory tables; refine the tree.");
            fmmCheck(cudaFuncSetAttribute(p2mKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)),
                     "p2m smem");
            p2mKernel<<<leaves, 256, sm, stream>>>(I.panels.as<FmmPanel>(), I.dLeaves[l].as<uint32_t>(),
                                                   I.dLeafStart[l].as<uint32_t>(), I.dItems.as<FmmItem>() + I.itemBase[l],
                                                   I.centers.as<double>(), I.coefOffset.as<uint64_t>(), P, k_, pv,
                                                   I.Mc.as<double2>(), rhs ? 1 : 0,
                                                   I.fp32 ? I.Mc32.as<float2>() : nullptr, I.levelSigma(l),
                                                   I.rule.as<double>(), I.rulePts);
            fmmCheck(cudaGetLastError(), "p2m launch");
        }
    }
    {
        TimedScope scope(timer, "fmm_m2m", stream);
        for (int l = levels - 2; l >= I.lmin; --l)
            if (I.fp32)
                translate(I.dm2m[l], I.order[l + 1], I.order[l], I.Mc32.as<float2>(), I.Mc32.as<float2>(), true);
            else
                translate(I.dm2m[l], I.order[l + 1], I.order[l], I.Mc.as<double2>(), I.Mc.as<double2>(), true);
    }
    // grouped M2L of level l (chunks into per-link slots, then the link-order sums)
    const auto grouped = [&](int l, auto *in, auto *out) {
        using CT = std::remove_cv_t<std::remove_pointer_t<decltype(out)>>;
        using RT = decltype(CT{}.x);
        constexpr bool f32 = std::is_same_v<RT, float>;
        const Impl::GroupPlan &gp = I.gm2l[l];
        const int mode = rhs ? 1 : 0, p = I.order[l], nc = (p + 1) * (p + 1);
        const size_t sm = groupSmemBytes(p, gp.cpad[mode], gp.g[mode], sizeof(CT));
        const RT *wig;
        const CT *cx;
        if constexpr (f32) {
            wig = I.wigner32.as<float>();
            cx = I.coax32.as<float2>();
        } else {
            wig = I.wigner.as<double>();
            cx = I.coax.as<double2>();
        }
        fmmCheck(cudaFuncSetAttribute(m2lGroupKernel<RT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)),
                 "grouped m2l smem");
        m2lGroupKernel<RT><<<gp.chunkCount[mode], 256, sm, stream>>>(
            gp.chunks[mode].as<uint2>(), gp.sorted.as<uint32_t>(), I.dm2l[l].links.as<TransLink>(), p, nch,
            gp.cpad[mode], gp.g[mode], in, I.coefOffset.as<uint64_t>(), wig, I.wignerStart.as<uint64_t>(), cx,
            I.coaxStart.as<uint64_t>(), I.slots.as<CT>());
        fmmCheck(cudaGetLastError(), "grouped m2l launch");
        const dim3 grid(I.dm2l[l].count, unsigned((nch * nc + 255) / 256));
        TimedScope sums(timer, "fmm_m2l_sum", stream);  // nested in fmm_m2l
        m2lSumKernel<RT><<<grid, 256, 0, stream>>>(I.dm2l[l].out.as<uint32_t>(), I.dm2l[l].start.as<uint32_t>(),
                                                   I.coefOffset.as<uint64_t>(), nc, nch, I.slots.as<CT>(), out);
        fmmCheck(cudaGetLastError(), "m2l sum launch");
    };
    {
        TimedScope scope(timer, "fmm_m2l", stream);
        const int mode = rhs ? 1 : 0;
        for (int l = I.lmin; l < levels; ++l)
            if (I.fp32) {
                if (I.gm2l[l].active[mode])
                    grouped(l, I.Mc32.as<float2>(), I.Lc32.as<float2>());
                else
                    translate(I.dm2l[l], I.order[l], I.order[l], I.Mc32.as<float2>(), I.Lc32.as<float2>(), false);
            } else if (I.hf[l].active)
                planeWaveM2L(l, nch, stream);
            else if (I.gm2l[l].active[mode])
                grouped(l, I.Mc.as<double2>(), I.Lc.as<double2>());
            else
                translate(I.dm2l[l], I.order[l], I.order[l], I.Mc.as<double2>(), I.Lc.as<double2>(), false);
    }
    {
        TimedScope scope(timer, "fmm_l2l", stream);
        for (int l = I.lmin + 1; l < levels; ++l)
            if (I.fp32)
                translate(I.dl2l[l], I.order[l - 1], I.order[l], I.Lc32.as<float2>(), I.Lc32.as<float2>(), false);
            else
                translate(I.dl2l[l], I.order[l - 1], I.order[l], I.Lc.as<double2>(), I.Lc.as<double2>(), false);
    }
    {
        TimedScope scope(timer, "fmm_l2p", stream);
        for (int l = I.lmin; l < levels; ++l) {
            const uint32_t leaves = uint32_t(I.leafNodes[l].size());
            if (!leaves)
                continue;
            const int p = I.order[l], P = p + 1;
            const size_t td = tableDoubles(P);
            const size_t nc = size_t(p + 1) * (p + 1), nd = size_t(P + 1) * (P + 1);
            const size_t coefBytes = (rhs ? nc + 3 * nd : 6 * nc + nd) * 16, tableBytes = kWarps * td * 8;
            // high orders keep the coefficients in global scratch, the point tables in shared memory
            const bool spill = coefBytes + tableBytes > kMaxShared;
            const size_t sm = spill ? tableBytes : coefBytes + tableBytes;
            if (sm > kMaxShared)
                throw Unsupported("Fast-multipole leaf order exceeds the shared-memory tables; refine the tree.");
            if (spill)
                I.l2pScratch.ensure(size_t(leaves) * coefBytes);
            double2 *scratch = spill ? I.l2pScratch.as<double2>() : nullptr;
            if (rhs) {
                fmmCheck(cudaFuncSetAttribute(l2pRhsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)),
                         "l2p smem");
                l2pRhsKernel<<<leaves, 256, sm, stream>>>(
                    I.panels.as<FmmPanel>(), I.dLeaves[l].as<uint32_t>(), I.dLeafStart[l].as<uint32_t>(),
                    I.dItems.as<FmmItem>() + I.itemBase[l], I.centers.as<double>(), I.coefOffset.as<uint64_t>(), p, k_,
                    I.Lc.as<double2>(), I.far.as<double2>(), I.fp32 ? I.Lc32.as<float2>() : nullptr,
                    I.levelSigma(l), I.rule.as<double>(), I.rulePts, scratch);
            } else {
                fmmCheck(cudaFuncSetAttribute(l2pKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)),
                         "l2p smem");
                l2pKernel<<<leaves, 256, sm, stream>>>(I.panels.as<FmmPanel>(), I.dLeaves[l].as<uint32_t>(),
                                                       I.dLeafStart[l].as<uint32_t>(),
                                                       I.dItems.as<FmmItem>() + I.itemBase[l], I.centers.as<double>(),
                                                       I.coefOffset.as<uint64_t>(), p, k_, I.Lc.as<double2>(),
                                                       I.far.as<double2>(), I.fp32 ? I.Lc32.as<float2>() : nullptr,
                                                       I.levelSigma(l), I.rule.as<double>(), I.rulePts, scratch);
            }
            fmmCheck(cudaGetLastError(), "l2p launch");
        }
        starSumKernel<<<(N + 255) / 256, 256, 0, stream>>>(I.far.as<double2>(), I.incOff.as<uint32_t>(), N, yv);
        fmmCheck(cudaGetLastError(), "star sum launch");
    }
}

// ------------------------------------------------------------- self-test

double fmmSelfTest() {
    using cd = std::complex<double>;
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(-0.5, 0.5);
    const double k = 3.0;
    const int p = 16;
    const int nc = (p + 1) * (p + 1);
    // direct field of random sources near the origin at targets near t
    const int ns = 12, nt = 6;
    std::vector<std::array<double, 3>> ys(ns), xs(nt);
    std::vector<cd> s(ns);
    for (auto &y : ys)
        y = {U(rng), U(rng), U(rng)};
    for (auto &v : s)
        v = cd(U(rng), U(rng));
    const double t[3] = {2.1, -1.3, 1.7};
    for (auto &x : xs)
        x = {t[0] + U(rng), t[1] + U(rng), t[2] + U(rng)};
    const auto R = [&](int P, const double *d, std::vector<cd> &out) {
        const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const double ct = r > 0 ? d[2] / r : 1, st = std::sqrt(std::max(0.0, 1 - ct * ct)), ph = std::atan2(d[1], d[0]);
        std::vector<double> j(P + 1), th(size_t(P + 1) * (P + 2) / 2);
        besselJ(P, k * r, j.data());
        for (int m = 0; m <= P; ++m)
            thetaColumn(m, P, ct, st, th.data());
        out.assign(size_t(P + 1) * (P + 1), 0);
        for (int n = 0; n <= P; ++n)
            for (int m = -n; m <= n; ++m) {
                const int am = std::abs(m);
                const double sg = (m < 0 && (am & 1)) ? -1 : 1;
                out[coefIndex(n, m)] = j[n] * sg * th[triIndex(n, am)] * std::polar(1.0, m * ph);
            }
    };
    std::vector<cd> M(nc, 0), Rv;
    for (int i = 0; i < ns; ++i) {
        R(p, ys[i].data(), Rv);
        for (int q = 0; q < nc; ++q)
            M[q] += s[i] * std::conj(Rv[q]);
    }
    // rotate -> coaxial (S|R) -> rotate back
    const double tl = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    const double cb = t[2] / tl, ph = std::atan2(t[1], t[0]);
    std::vector<double> dtab;
    wignerBlocks(p, cb, dtab);
    std::vector<cd> a(nc), b(nc, 0), c(nc, 0), L(nc, 0);
    for (int n = 0; n <= p; ++n)
        for (int mp = -n; mp <= n; ++mp) {
            cd acc = 0;
            for (int m = -n; m <= n; ++m)
                acc += M[coefIndex(n, m)] * std::polar(1.0, m * ph) *
                       dtab[wignerOffset(n) + size_t(m + n) * (2 * n + 1) + (mp + n)];
            b[coefIndex(n, mp)] = acc;
        }
    const GauntTable &g = gauntTable(p);
    std::vector<cd> fl(2 * p + 1);
    radialFactors(k * tl, true, 2 * p, fl.data());
    for (int np = 0; np <= p; ++np)
        for (int m = -np; m <= np; ++m) {
            const int am = std::abs(m);
            cd acc = 0;
            for (int n = am; n <= p; ++n) {
                const double *gv = g.values.data() + g.offsets[(size_t(am) * (p + 1) + n) * (p + 1) + np];
                cd cv = 0;
                int idx = 0;
                for (int l = std::abs(n - np); l <= n + np; l += 2, ++idx)
                    cv += (((n - np - l) / 2) & 1 ? -1.0 : 1.0) * gv[idx] * fl[l];
                acc += cv * b[coefIndex(n, m)];
            }
            c[coefIndex(np, m)] = acc;
        }
    for (int n = 0; n <= p; ++n)
        for (int m1 = -n; m1 <= n; ++m1) {
            cd acc = 0;
            for (int m = -n; m <= n; ++m)
                acc += dtab[wignerOffset(n) + size_t(m1 + n) * (2 * n + 1) + (m + n)] * c[coefIndex(n, m)];
            L[coefIndex(n, m1)] = acc * std::polar(1.0, -m1 * ph);
        }
    double err = 0, ref = 0;
    for (int i = 0; i < nt; ++i) {
        cd direct = 0;
        for (int q = 0; q < ns; ++q) {
            const double dx = xs[i][0] - ys[q][0], dy = xs[i][1] - ys[q][1], dz = xs[i][2] - ys[q][2];
            const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
            direct += s[q] * std::polar(1.0 / (4 * kFmmPi * r), -k * r);
        }
        const double d[3] = {xs[i][0] - t[0], xs[i][1] - t[1], xs[i][2] - t[2]};
        R(p, d, Rv);
        cd f = 0;
        for (int q = 0; q < nc; ++q)
            f += L[q] * Rv[q];
        f *= cd(0, -k);
        err = std::max(err, std::abs(f - direct));
        ref = std::max(ref, std::abs(direct));
    }
    return err / ref;
}

}  // namespace hsb
