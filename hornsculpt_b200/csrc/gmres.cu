// Batched left-preconditioned GMRES in FP64, the refinement solver of the
// mixed dense form (GMRES-IR): each outer step solves A d = r for the FP64
// residual r = b - A x with the FP32 LU as preconditioner M, and adds d to x.
//
// Method: DeviceGmresSolver (cuda/device_gmres.cu:171-287) — left-preconditioned
// GMRES(m) with classical Gram-Schmidt applied twice (:144-165) and Givens
// rotations (:226-245). Here the rotations run on the device (one thread per
// system) and the host reads only the residual estimates after each Arnoldi
// step. All reductions add fixed partial sums in a fixed order, so results are
// bitwise repeatable. Systems are s = f * E + e (frequency f of the batch,
// excitation e); vectors are [S][N] complex, interleaved.
#include "device_types.cuh"
#include "kernel_timer.hpp"

#include <algorithm>
#include <functional>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace hsb {
namespace {

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

__device__ __forceinline__ double2 cmulD(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 conjMulD(double2 a, double2 b) {  // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// Fixed-order block sum of a double2 over 256 threads.
__device__ __forceinline__ double2 blockSum256(double2 v, double2 *red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < unsigned(s)) {
            red[threadIdx.x].x += red[threadIdx.x + s].x;
            red[threadIdx.x].y += red[threadIdx.x + s].y;
        }
        __syncthreads();
    }
    const double2 r = red[0];
    __syncthreads();
    return r;
}

// w_s = A_f v_s for every active system; 32 rows x 8 column groups per CTA.
__global__ void __launch_bounds__(256) gemvKernel(const double *A, uint32_t N, uint32_t E, const double *v,
                                                  size_t vStride, double *w, const int *active) {
    __shared__ double2 part[8][32];
    const uint32_t lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const uint32_t a = blockIdx.x * 32 + lane;
    const uint32_t s = blockIdx.y;
    if (!active[s])
        return;
    const uint32_t f = s / E;
    const double *M = A + size_t(f) * N * N * 2;
    const double2 *x = reinterpret_cast<const double2 *>(v + s * vStride);
    double re = 0, im = 0;
    if (a < N)
        for (uint32_t c = g; c < N; c += 8) {
            const double2 m = *reinterpret_cast<const double2 *>(M + 2 * (size_t(c) * N + a));
            const double2 xv = x[c];
            re += m.x * xv.x - m.y * xv.y;
            im += m.x * xv.y + m.y * xv.x;
        }
    part[g][lane] = make_double2(re, im);
    __syncthreads();
    if (g != 0 || a >= N)
        return;
    re = 0;
    im = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        re += part[q][lane].x;
        im += part[q][lane].y;
    }
    reinterpret_cast<double2 *>(w + size_t(s) * N * 2)[a] = make_double2(re, im);
}

__global__ void toDoubleKernel(const float *in, double *out, size_t count) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count)
        out[i] = double(in[i]);
}

// Start of a cycle: beta = |z0|, V_0 = z0 / beta, g = beta e_1. Systems with
// z0 = 0 are inactive from the start.
__global__ void __launch_bounds__(256) startKernel(const double *z, uint32_t N, uint32_t m, double *basis,
                                                   double *g, double *beta, double *estimate, int *active,
                                                   uint32_t *steps) {
    __shared__ double2 red[256];
    const uint32_t s = blockIdx.x;
    const double2 *zs = reinterpret_cast<const double2 *>(z + size_t(s) * N * 2);
    double sq = 0;
    for (uint32_t n = threadIdx.x; n < N; n += blockDim.x)
        sq += zs[n].x * zs[n].x + zs[n].y * zs[n].y;
    const double b = sqrt(blockSum256(make_double2(sq, 0), red).x);
    double2 *v0 = reinterpret_cast<double2 *>(basis + size_t(s) * (m + 1) * N * 2);
    const double inv = b > 0 ? 1.0 / b : 0.0;
    for (uint32_t n = threadIdx.x; n < N; n += blockDim.x)
        v0[n] = make_double2(zs[n].x * inv, zs[n].y * inv);
    if (threadIdx.x == 0) {
        double2 *gs = reinterpret_cast<double2 *>(g + size_t(s) * (m + 1) * 2);
        for (uint32_t i = 0; i <= m; ++i)
            gs[i] = make_double2(i == 0 ? b : 0.0, 0.0);
        beta[s] = b;
        const bool go = b > 0 && isfinite(b);
        active[s] = go ? 1 : 0;
        estimate[s] = go ? 1.0 : 0.0;
        steps[s] = 0;
    }
}

// h_i = <V_i, z> for i <= j (one CTA per (i, system)); added to column j of H.
__global__ void __launch_bounds__(256) dotKernel(const double *basis, const double *z, uint32_t N, uint32_t m,
                                                 uint32_t j, double *hess, double *dots, bool accumulate,
                                                 const int *active) {
    __shared__ double2 red[256];
    const uint32_t i = blockIdx.x, s = blockIdx.y;
    if (!active[s])
        return;
    const double2 *vi = reinterpret_cast<const double2 *>(basis + (size_t(s) * (m + 1) + i) * N * 2);
    const double2 *zs = reinterpret_cast<const double2 *>(z + size_t(s) * N * 2);
    double2 acc = make_double2(0, 0);
    for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) {
        const double2 p = conjMulD(vi[n], zs[n]);
        acc.x += p.x;
        acc.y += p.y;
    }
    const double2 h = blockSum256(acc, red);
    if (threadIdx.x == 0) {
        double2 *col = reinterpret_cast<double2 *>(hess + (size_t(s) * m + j) * (m + 1) * 2);
        col[i] = accumulate ? make_double2(col[i].x + h.x, col[i].y + h.y) : h;
        reinterpret_cast<double2 *>(dots + size_t(s) * (m + 1) * 2)[i] = h;
    }
}

// z -= sum_{i <= j} h_i V_i (h of the latest pass), fixed order in i.
__global__ void subtractKernel(const double *basis, const double *dots, uint32_t N, uint32_t m, uint32_t j,
                               double *z, const int *active) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x, s = blockIdx.y;
    if (n >= N || !active[s])
        return;
    const double2 *h = reinterpret_cast<const double2 *>(dots + size_t(s) * (m + 1) * 2);
    double2 *zs = reinterpret_cast<double2 *>(z + size_t(s) * N * 2);
    double2 v = zs[n];
    for (uint32_t i = 0; i <= j; ++i) {
        const double2 b = reinterpret_cast<const double2 *>(basis + (size_t(s) * (m + 1) + i) * N * 2)[n];
        const double2 p = cmulD(h[i], b);
        v.x -= p.x;
        v.y -= p.y;
    }
    zs[n] = v;
}

// H[j+1][j] = |z|, V_{j+1} = z / |z|.
__global__ void __launch_bounds__(256) normalizeKernel(const double *z, uint32_t N, uint32_t m, uint32_t j,
                                                       double *basis, double *hess, const int *active) {
    __shared__ double2 red[256];
    const uint32_t s = blockIdx.x;
    if (!active[s])
        return;
    const double2 *zs = reinterpret_cast<const double2 *>(z + size_t(s) * N * 2);
    double sq = 0;
    for (uint32_t n = threadIdx.x; n < N; n += blockDim.x)
        sq += zs[n].x * zs[n].x + zs[n].y * zs[n].y;
    const double nrm = sqrt(blockSum256(make_double2(sq, 0), red).x);
    const double inv = nrm > 0 ? 1.0 / nrm : 0.0;
    double2 *vn = reinterpret_cast<double2 *>(basis + (size_t(s) * (m + 1) + j + 1) * N * 2);
    for (uint32_t n = threadIdx.x; n < N; n += blockDim.x)
        vn[n] = make_double2(zs[n].x * inv, zs[n].y * inv);
    if (threadIdx.x == 0)
        reinterpret_cast<double2 *>(hess + (size_t(s) * m + j) * (m + 1) * 2)[j + 1] = make_double2(nrm, 0);
}

// Column j of H: previous rotations, a new rotation that zeroes H[j+1][j],
// the rotated right-hand side g and the residual estimate |g_{j+1}| / beta.
// Rotation k is (c_k real, s_k complex): [x; y] -> [c x + s y; -conj(s) x + c y].
__global__ void givensKernel(uint32_t S, uint32_t m, uint32_t j, double *hess, double *rot, double *g,
                             const double *beta, const double *tol, double *estimate, int *active, uint32_t *steps) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S || !active[s])
        return;
    double2 *col = reinterpret_cast<double2 *>(hess + (size_t(s) * m + j) * (m + 1) * 2);
    double *rs = rot + size_t(s) * m * 3;
    for (uint32_t k = 0; k < j; ++k) {
        const double c = rs[3 * k];
        const double2 sn = make_double2(rs[3 * k + 1], rs[3 * k + 2]);
        const double2 x = col[k], y = col[k + 1];
        const double2 sy = cmulD(sn, y), sx = conjMulD(sn, x);
        col[k] = make_double2(c * x.x + sy.x, c * x.y + sy.y);
        col[k + 1] = make_double2(c * y.x - sx.x, c * y.y - sx.y);
    }
    const double2 a = col[j], b = col[j + 1];
    const double na = hypot(a.x, a.y), nb = hypot(b.x, b.y), r = hypot(na, nb);
    double c = 1, snr = 0, sni = 0;
    double2 top = a;
    if (nb > 0) {
        if (na == 0) {
            c = 0;
            snr = b.x / nb;  // s = conj(b) / |b| gives s b = |b|
            sni = -b.y / nb;
            top = make_double2(nb, 0);
        } else {
            c = na / r;
            const double2 ua = make_double2(a.x / na, a.y / na);  // a / |a|
            // s = (a / |a|) conj(b) / r
            snr = (ua.x * b.x + ua.y * b.y) / r;
            sni = (ua.y * b.x - ua.x * b.y) / r;
            top = make_double2(ua.x * r, ua.y * r);
        }
    }
    rs[3 * j] = c;
    rs[3 * j + 1] = snr;
    rs[3 * j + 2] = sni;
    col[j] = top;
    col[j + 1] = make_double2(0, 0);
    double2 *gs = reinterpret_cast<double2 *>(g + size_t(s) * (m + 1) * 2);
    const double2 gj = gs[j];
    // g_{j+1} = -conj(s) g_j, g_j = c g_j
    gs[j + 1] = make_double2(-(snr * gj.x + sni * gj.y), -(snr * gj.y - sni * gj.x));
    gs[j] = make_double2(c * gj.x, c * gj.y);
    const double est = hypot(gs[j + 1].x, gs[j + 1].y) / beta[s];
    estimate[s] = est;
    steps[s] = j + 1;
    if (!(est > tol[s]) || j + 1 == m)
        active[s] = 0;
}

// y = H^{-1} g over the system's steps, then x += sum_i y_i V_i.
__global__ void __launch_bounds__(256) updateKernel(const double *basis, const double *hess, const double *g,
                                                    const uint32_t *steps, uint32_t N, uint32_t m, double *x) {
    extern __shared__ double2 y[];
    const uint32_t s = blockIdx.x;
    const uint32_t k = steps[s];
    if (k == 0)
        return;
    if (threadIdx.x == 0) {
        const double2 *gs = reinterpret_cast<const double2 *>(g + size_t(s) * (m + 1) * 2);
        for (int i = int(k) - 1; i >= 0; --i) {
            double2 v = gs[i];
            for (uint32_t q = i + 1; q < k; ++q) {
                const double2 h = reinterpret_cast<const double2 *>(hess + (size_t(s) * m + q) * (m + 1) * 2)[i];
                const double2 p = cmulD(h, y[q]);
                v.x -= p.x;
                v.y -= p.y;
            }
            const double2 d = reinterpret_cast<const double2 *>(hess + (size_t(s) * m + i) * (m + 1) * 2)[i];
            const double den = d.x * d.x + d.y * d.y;
            y[i] = den > 0 ? make_double2((v.x * d.x + v.y * d.y) / den, (v.y * d.x - v.x * d.y) / den)
                           : make_double2(0, 0);
        }
    }
    __syncthreads();
    double2 *xs = reinterpret_cast<double2 *>(x + size_t(s) * N * 2);
    for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) {
        double2 v = xs[n];
        for (uint32_t i = 0; i < k; ++i) {
            const double2 b = reinterpret_cast<const double2 *>(basis + (size_t(s) * (m + 1) + i) * N * 2)[n];
            const double2 p = cmulD(y[i], b);
            v.x += p.x;
            v.y += p.y;
        }
        xs[n] = v;
    }
}

}  // namespace

// Workspace pieces, each 256-byte aligned, in carve order.
struct GmresLayout {
    size_t basis, hess, g, dots, rot, beta, estimate, tol, active, steps, z, z32, solve, total;
};

GmresLayout gmresLayout(uint32_t N, uint32_t S, uint32_t m) {
    GmresLayout l{};
    size_t at = 0;
    const auto take = [&at](size_t bytes) {
        const size_t here = at;
        at += (bytes + 255) / 256 * 256;
        return here;
    };
    l.basis = take(size_t(S) * (m + 1) * N * 16);
    l.hess = take(size_t(S) * m * (m + 1) * 16);
    l.g = take(size_t(S) * (m + 1) * 16);
    l.dots = take(size_t(S) * (m + 1) * 16);
    l.rot = take(size_t(S) * m * 24);
    l.beta = take(size_t(S) * 8);
    l.estimate = take(size_t(S) * 8);
    l.tol = take(size_t(S) * 8);
    l.active = take(size_t(S) * 4);
    l.steps = take(size_t(S) * 4);
    l.z = take(size_t(S) * N * 16);
    l.z32 = take(size_t(S) * N * 8);
    l.solve = take(size_t(S) * N * 8);  // triangular-solve scratch
    l.total = at;
    return l;
}

size_t gmresWorkspaceBytes(uint32_t N, uint32_t S, uint32_t m) { return gmresLayout(N, S, m).total; }

uint32_t gmresCycleBatch(const double *A, const float *LU32, const int *pivots, uint32_t N, uint32_t B, uint32_t E,
                         const double *r, double *x, uint32_t m, const std::vector<double> &tolerances,
                         void *workspace, cudaStream_t stream, KernelTimer *timer, std::vector<uint32_t> &stepsOut) {
    const uint32_t S = B * E;
    const GmresLayout l = gmresLayout(N, S, m);
    char *w = static_cast<char *>(workspace);
    double *basis = reinterpret_cast<double *>(w + l.basis);
    double *hess = reinterpret_cast<double *>(w + l.hess);
    double *g = reinterpret_cast<double *>(w + l.g);
    double *dots = reinterpret_cast<double *>(w + l.dots);
    double *rot = reinterpret_cast<double *>(w + l.rot);
    double *beta = reinterpret_cast<double *>(w + l.beta);
    double *estimate = reinterpret_cast<double *>(w + l.estimate);
    double *tol = reinterpret_cast<double *>(w + l.tol);
    if (tolerances.size() != S)
        throw std::runtime_error("GMRES needs one tolerance per system.");
    check(cudaMemcpyAsync(tol, tolerances.data(), S * sizeof(double), cudaMemcpyHostToDevice, stream),
          "GMRES tolerances");
    int *active = reinterpret_cast<int *>(w + l.active);
    uint32_t *steps = reinterpret_cast<uint32_t *>(w + l.steps);
    double *z = reinterpret_cast<double *>(w + l.z);
    float *z32 = reinterpret_cast<float *>(w + l.z32);
    const size_t reals = size_t(S) * N * 2;
    const auto precondition = [&](const double *in) {  // z = M^{-1} in
        TimedScope scope(timer, "gmres_precondition", stream);
        roundToFloat(in, z32, reals, stream);
        luSolveBatch(LU32, pivots, N, B, E, z32, w + l.solve, stream, nullptr);
        toDoubleKernel<<<unsigned((reals + 255) / 256), 256, 0, stream>>>(z32, z, reals);
    };
    precondition(r);
    startKernel<<<S, 256, 0, stream>>>(z, N, m, basis, g, beta, estimate, active, steps);
    check(cudaGetLastError(), "GMRES start launch");
    std::vector<int> hostActive(S);
    uint32_t j = 0;
    for (; j < m; ++j) {
        {
            TimedScope scope(timer, "gmres_matvec", stream);
            gemvKernel<<<dim3((N + 31) / 32, S), 256, 0, stream>>>(
                A, N, E, basis + size_t(j) * N * 2, size_t(m + 1) * N * 2, z, active);
        }
        precondition(z);  // z = M^{-1} A V_j
        {
            TimedScope scope(timer, "gmres_orthogonalize", stream);
            for (int pass = 0; pass < 2; ++pass) {
                dotKernel<<<dim3(j + 1, S), 256, 0, stream>>>(basis, z, N, m, j, hess, dots, pass == 1, active);
                subtractKernel<<<dim3((N + 255) / 256, S), 256, 0, stream>>>(basis, dots, N, m, j, z, active);
            }
            normalizeKernel<<<S, 256, 0, stream>>>(z, N, m, j, basis, hess, active);
            givensKernel<<<(S + 127) / 128, 128, 0, stream>>>(S, m, j, hess, rot, g, beta, tol, estimate, active,
                                                              steps);
        }
        check(cudaGetLastError(), "GMRES step launch");
        check(cudaMemcpyAsync(hostActive.data(), active, S * sizeof(int), cudaMemcpyDeviceToHost, stream),
              "GMRES state");
        check(cudaStreamSynchronize(stream), "GMRES step");
        if (std::none_of(hostActive.begin(), hostActive.end(), [](int a) { return a != 0; })) {
            ++j;
            break;
        }
    }
    {
        TimedScope scope(timer, "gmres_update", stream);
        updateKernel<<<S, 256, m * sizeof(double2), stream>>>(basis, hess, g, steps, N, m, x);
        check(cudaGetLastError(), "GMRES update launch");
    }
    stepsOut.resize(S);
    check(cudaMemcpyAsync(stepsOut.data(), steps, S * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream),
          "GMRES steps");
    check(cudaStreamSynchronize(stream), "GMRES update");
    return j;
}

// The same cycle with the operator and the preconditioner supplied by the
// caller: apply(v, stride, z) writes z_s = A v_s for every system (v_s at
// v + s * stride reals), precondition(in, out) writes out_s = M^{-1} in_s
// (out may equal in). Used by the fast-multipole form, whose A is the near
// matrix plus the far-field expansion operator.
uint32_t gmresCycleOperator(uint32_t N, uint32_t S, const double *r, double *x, uint32_t m,
                            const std::vector<double> &tolerances, void *workspace, cudaStream_t stream,
                            KernelTimer *timer, std::vector<uint32_t> &stepsOut,
                            const std::function<void(const double *, size_t, double *)> &apply,
                            const std::function<void(const double *, double *)> &precondition) {
    const GmresLayout l = gmresLayout(N, S, m);
    char *w = static_cast<char *>(workspace);
    double *basis = reinterpret_cast<double *>(w + l.basis);
    double *hess = reinterpret_cast<double *>(w + l.hess);
    double *g = reinterpret_cast<double *>(w + l.g);
    double *dots = reinterpret_cast<double *>(w + l.dots);
    double *rot = reinterpret_cast<double *>(w + l.rot);
    double *beta = reinterpret_cast<double *>(w + l.beta);
    double *estimate = reinterpret_cast<double *>(w + l.estimate);
    double *tol = reinterpret_cast<double *>(w + l.tol);
    if (tolerances.size() != S)
        throw std::runtime_error("GMRES needs one tolerance per system.");
    check(cudaMemcpyAsync(tol, tolerances.data(), S * sizeof(double), cudaMemcpyHostToDevice, stream),
          "GMRES tolerances");
    int *active = reinterpret_cast<int *>(w + l.active);
    uint32_t *steps = reinterpret_cast<uint32_t *>(w + l.steps);
    double *z = reinterpret_cast<double *>(w + l.z);
    {
        TimedScope scope(timer, "gmres_precondition", stream);
        precondition(r, z);
    }
    startKernel<<<S, 256, 0, stream>>>(z, N, m, basis, g, beta, estimate, active, steps);
    check(cudaGetLastError(), "GMRES start launch");
    std::vector<int> hostActive(S);
    uint32_t j = 0;
    for (; j < m; ++j) {
        apply(basis + size_t(j) * N * 2, size_t(m + 1) * N * 2, z);
        {
            TimedScope scope(timer, "gmres_precondition", stream);
            precondition(z, z);
        }
        {
            TimedScope scope(timer, "gmres_orthogonalize", stream);
            for (int pass = 0; pass < 2; ++pass) {
                dotKernel<<<dim3(j + 1, S), 256, 0, stream>>>(basis, z, N, m, j, hess, dots, pass == 1, active);
                subtractKernel<<<dim3((N + 255) / 256, S), 256, 0, stream>>>(basis, dots, N, m, j, z, active);
            }
            normalizeKernel<<<S, 256, 0, stream>>>(z, N, m, j, basis, hess, active);
            givensKernel<<<(S + 127) / 128, 128, 0, stream>>>(S, m, j, hess, rot, g, beta, tol, estimate, active,
                                                              steps);
        }
        check(cudaGetLastError(), "GMRES step launch");
        check(cudaMemcpyAsync(hostActive.data(), active, S * sizeof(int), cudaMemcpyDeviceToHost, stream),
              "GMRES state");
        check(cudaStreamSynchronize(stream), "GMRES step");
        if (std::none_of(hostActive.begin(), hostActive.end(), [](int a) { return a != 0; })) {
            ++j;
            break;
        }
    }
    {
        TimedScope scope(timer, "gmres_update", stream);
        updateKernel<<<S, 256, m * sizeof(double2), stream>>>(basis, hess, g, steps, N, m, x);
        check(cudaGetLastError(), "GMRES update launch");
    }
    stepsOut.resize(S);
    check(cudaMemcpyAsync(stepsOut.data(), steps, S * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream),
          "GMRES steps");
    check(cudaStreamSynchronize(stream), "GMRES update");
    return j;
}

}  // namespace hsb
