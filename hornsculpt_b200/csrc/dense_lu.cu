// Batched dense complex FP64 LU with partial pivoting, triangular solves and
// the FP64 refinement residual (cuda_solver.cu:1485-1581, plain form: the
// factor is FP64 instead of the reference's FP32 cuSOLVER getrf/getrs).
//
// Matrices are column-major N x N complex (interleaved doubles), one per
// frequency of the batch (blockIdx.y / blockIdx.z). Right-looking blocked
// LU with panel width 32: a single-CTA panel factorisation per matrix, row
// interchanges outside the panel, a unit-lower triangular solve for the U
// block row and a shared-memory tiled complex GEMM for the trailing update.
#include "device_types.cuh"
#include "kernel_timer.hpp"

#include <stdexcept>
#include <string>

namespace hsb {
namespace {

constexpr int kPanel = 32;

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

__device__ __forceinline__ double2 ld2(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ void st2(double *p, double2 v) { *reinterpret_cast<double2 *>(p) = v; }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Panel factorisation of columns [k0, k0+jb) over rows [k0, N) of one matrix.
__global__ void __launch_bounds__(512) panelKernel(double *LU, uint32_t N, uint32_t k0, uint32_t jb, int *pivots,
                                                   int *info) {
    double *M = LU + size_t(blockIdx.x) * N * N * 2;
    int *piv = pivots + size_t(blockIdx.x) * N;
    __shared__ double sVal[16];
    __shared__ int sIdx[16];
    __shared__ double2 sRow[kPanel];
    __shared__ int sPivot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (uint32_t j = 0; j < jb; ++j) {
        const uint32_t c = k0 + j;
        // argmax |re|+|im| over rows [c, N), first index on ties
        double best = -1;
        int bestRow = int(c);
        for (uint32_t i = c + threadIdx.x; i < N; i += blockDim.x) {
            const double2 v = ld2(M + 2 * (size_t(c) * N + i));
            const double a = fabs(v.x) + fabs(v.y);
            if (a > best) {
                best = a;
                bestRow = int(i);
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double ob = __shfl_down_sync(0xffffffffu, best, off);
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
            double b = sVal[0];
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
            double *a = M + 2 * (size_t(k0 + threadIdx.x) * N + c);
            double *b = M + 2 * (size_t(k0 + threadIdx.x) * N + p);
            const double2 va = ld2(a), vb = ld2(b);
            st2(a, vb);
            st2(b, va);
        }
        __syncthreads();
        if (threadIdx.x < jb)
            sRow[threadIdx.x] = ld2(M + 2 * (size_t(k0 + threadIdx.x) * N + c));
        __syncthreads();
        const double2 d = sRow[j];
        const double den = d.x * d.x + d.y * d.y;
        const double2 inv = den > 0 ? make_double2(d.x / den, -d.y / den) : make_double2(0, 0);
        for (uint32_t i = c + 1 + threadIdx.x; i < N; i += blockDim.x) {
            double *col = M + 2 * (size_t(c) * N + i);
            const double2 l = cmul(ld2(col), inv);
            st2(col, l);
            for (uint32_t q = j + 1; q < jb; ++q) {
                double *e = M + 2 * (size_t(k0 + q) * N + i);
                const double2 u = sRow[q];
                double2 v = ld2(e);
                v.x -= l.x * u.x - l.y * u.y;
                v.y -= l.x * u.y + l.y * u.x;
                st2(e, v);
            }
        }
        __syncthreads();
    }
}

// Row interchanges of the panel applied to columns outside it.
__global__ void swapKernel(double *LU, uint32_t N, uint32_t k0, uint32_t jb, const int *pivots) {
    const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= N || (col >= k0 && col < k0 + jb))
        return;
    double *M = LU + size_t(blockIdx.y) * N * N * 2 + 2 * size_t(col) * N;
    const int *piv = pivots + size_t(blockIdx.y) * N;
    for (uint32_t c = k0; c < k0 + jb; ++c) {
        const int p = piv[c];
        if (p != int(c)) {
            const double2 a = ld2(M + 2 * c), b = ld2(M + 2 * p);
            st2(M + 2 * c, b);
            st2(M + 2 * p, a);
        }
    }
}

// U12 = L11^{-1} A12 (unit lower L11 of the panel), one thread per column.
__global__ void trsmKernel(double *LU, uint32_t N, uint32_t k0, uint32_t jb) {
    __shared__ double2 L[kPanel][kPanel];
    double *M = LU + size_t(blockIdx.y) * N * N * 2;
    for (uint32_t e = threadIdx.x; e < jb * jb; e += blockDim.x) {
        const uint32_t r = e % jb, c = e / jb;
        L[r][c] = ld2(M + 2 * (size_t(k0 + c) * N + k0 + r));
    }
    __syncthreads();
    const uint32_t col = k0 + jb + blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= N)
        return;
    double *C = M + 2 * size_t(col) * N;
    double2 x[kPanel];
    for (uint32_t i = 0; i < jb; ++i) {
        double2 v = ld2(C + 2 * (k0 + i));
        for (uint32_t m = 0; m < i; ++m) {
            const double2 l = L[i][m];
            v.x -= l.x * x[m].x - l.y * x[m].y;
            v.y -= l.x * x[m].y + l.y * x[m].x;
        }
        x[i] = v;
        st2(C + 2 * (k0 + i), v);
    }
}

// A22 -= L21 * U12 with 64x64 output tiles, K = jb <= 32.
__global__ void __launch_bounds__(256) gemmKernel(double *LU, uint32_t N, uint32_t k0, uint32_t jb) {
    extern __shared__ double2 smem[];
    double2 *sA = smem;                 // [kPanel][64]  L21 tile, k-major
    double2 *sB = smem + kPanel * 64;   // [kPanel][64]  U12 tile, k-major
    double *M = LU + size_t(blockIdx.z) * N * N * 2;
    const uint32_t r0 = k0 + jb + blockIdx.x * 64, c0 = k0 + jb + blockIdx.y * 64;
    for (uint32_t e = threadIdx.x; e < jb * 64; e += blockDim.x) {
        const uint32_t kk = e / 64, x = e % 64;
        const uint32_t r = r0 + x, c = c0 + x;
        sA[kk * 64 + x] = r < N ? ld2(M + 2 * (size_t(k0 + kk) * N + r)) : make_double2(0, 0);
        sB[kk * 64 + x] = c < N ? ld2(M + 2 * (size_t(c) * N + k0 + kk)) : make_double2(0, 0);
    }
    __syncthreads();
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
            acc[i][j] = make_double2(0, 0);
    for (uint32_t kk = 0; kk < jb; ++kk) {
        double2 a[4], b[4];
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
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t c = c0 + ty + 16 * j;
        if (c >= N)
            continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t r = r0 + tx + 16 * i;
            if (r >= N)
                continue;
            double *e = M + 2 * (size_t(c) * N + r);
            double2 v = ld2(e);
            v.x -= acc[i][j].x;
            v.y -= acc[i][j].y;
            st2(e, v);
        }
    }
}

// Forward / back substitution of one right-hand side per CTA, with the
// vector staged in shared memory (N <= 13000).
__global__ void __launch_bounds__(256) solveKernel(const double *LU, const int *pivots, uint32_t N, uint32_t E,
                                                   double *X) {
    extern __shared__ double2 x[];
    const uint32_t e = blockIdx.x, f = blockIdx.y;
    const double *M = LU + size_t(f) * N * N * 2;
    const int *piv = pivots + size_t(f) * N;
    double *out = X + (size_t(f) * E + e) * N * 2;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
        x[i] = ld2(out + 2 * i);
    __syncthreads();
    if (threadIdx.x == 0)
        for (uint32_t c = 0; c < N; ++c) {
            const int p = piv[c];
            if (p != int(c)) {
                const double2 t = x[c];
                x[c] = x[p];
                x[p] = t;
            }
        }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t k = 0; k < N; k += 32) {
        const uint32_t kb = min(32u, N - k);
        if (warp == 0) {
            double2 mine = lane < int(kb) ? x[k + lane] : make_double2(0, 0);
            for (uint32_t m = 0; m < kb; ++m) {
                const double2 xm = make_double2(__shfl_sync(0xffffffffu, mine.x, m), __shfl_sync(0xffffffffu, mine.y, m));
                if (lane > int(m) && lane < int(kb)) {
                    const double2 l = ld2(M + 2 * (size_t(k + m) * N + k + lane));
                    mine.x -= l.x * xm.x - l.y * xm.y;
                    mine.y -= l.x * xm.y + l.y * xm.x;
                }
            }
            if (lane < int(kb))
                x[k + lane] = mine;
        }
        __syncthreads();
        for (uint32_t i = k + kb + threadIdx.x; i < N; i += blockDim.x) {
            double2 v = x[i];
            for (uint32_t m = 0; m < kb; ++m) {
                const double2 l = ld2(M + 2 * (size_t(k + m) * N + i));
                const double2 xm = x[k + m];
                v.x -= l.x * xm.x - l.y * xm.y;
                v.y -= l.x * xm.y + l.y * xm.x;
            }
            x[i] = v;
        }
        __syncthreads();
    }
    const uint32_t blocks = (N + 31) / 32;
    for (uint32_t bi = blocks; bi-- > 0;) {
        const uint32_t k = bi * 32, kb = min(32u, N - k);
        if (warp == 0) {
            double2 mine = lane < int(kb) ? x[k + lane] : make_double2(0, 0);
            for (int m = int(kb) - 1; m >= 0; --m) {
                if (lane == m) {
                    const double2 d = ld2(M + 2 * (size_t(k + m) * N + k + m));
                    const double den = d.x * d.x + d.y * d.y;
                    mine = make_double2((mine.x * d.x + mine.y * d.y) / den, (mine.y * d.x - mine.x * d.y) / den);
                }
                const double2 xm = make_double2(__shfl_sync(0xffffffffu, mine.x, m), __shfl_sync(0xffffffffu, mine.y, m));
                if (lane < m) {
                    const double2 u = ld2(M + 2 * (size_t(k + m) * N + k + lane));
                    mine.x -= u.x * xm.x - u.y * xm.y;
                    mine.y -= u.x * xm.y + u.y * xm.x;
                }
            }
            if (lane < int(kb))
                x[k + lane] = mine;
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) {
            double2 v = x[i];
            for (uint32_t m = 0; m < kb; ++m) {
                const double2 u = ld2(M + 2 * (size_t(k + m) * N + i));
                const double2 xm = x[k + m];
                v.x -= u.x * xm.x - u.y * xm.y;
                v.y -= u.x * xm.y + u.y * xm.x;
            }
            x[i] = v;
        }
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
        st2(out + 2 * i, x[i]);
}

// r = b - A x per row (FP64), plus mass-scaled squares for the norms.
__global__ void residualKernel(const double *A, const double *b, const double *x, const double *mass, uint32_t N,
                               uint32_t E, double *correction, double *squares) {
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t e = blockIdx.y, f = blockIdx.z;
    if (a >= N)
        return;
    const double *M = A + size_t(f) * N * N * 2;
    const double *xv = x + (size_t(f) * E + e) * N * 2;
    double re = 0, im = 0;
    for (uint32_t c = 0; c < N; ++c) {
        const double2 m = ld2(M + 2 * (size_t(c) * N + a));
        const double2 v = ld2(xv + 2 * c);
        re += m.x * v.x - m.y * v.y;
        im += m.x * v.y + m.y * v.x;
    }
    const size_t idx = (size_t(f) * E + e) * N + a;
    const double2 bb = ld2(b + 2 * idx);
    re = bb.x - re;
    im = bb.y - im;
    st2(correction + 2 * idx, make_double2(re, im));
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

}  // namespace

void luFactorBatch(double *LU, uint32_t N, uint32_t B, int *pivots, int *info, cudaStream_t stream,
                   KernelTimer *timer) {
    check(cudaMemsetAsync(info, 0, sizeof(int), stream), "LU info reset");
    const size_t gemmSmem = 2 * kPanel * 64 * sizeof(double2);
    static bool attr = false;
    if (!attr) {
        check(cudaFuncSetAttribute(gemmKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(gemmSmem)),
              "gemm smem attribute");
        attr = true;
    }
    for (uint32_t k0 = 0; k0 < N; k0 += kPanel) {
        const uint32_t jb = min(uint32_t(kPanel), N - k0);
        {
            TimedScope s(timer, "lu_panel", stream);
            panelKernel<<<B, 512, 0, stream>>>(LU, N, k0, jb, pivots, info);
        }
        {
            TimedScope s(timer, "lu_swap", stream);
            swapKernel<<<dim3((N + 127) / 128, B), 128, 0, stream>>>(LU, N, k0, jb, pivots);
        }
        const uint32_t rest = N - k0 - jb;
        if (rest) {
            {
                TimedScope s(timer, "lu_trsm", stream);
                trsmKernel<<<dim3((rest + 127) / 128, B), 128, 0, stream>>>(LU, N, k0, jb);
            }
            TimedScope s(timer, "lu_gemm", stream);
            gemmKernel<<<dim3((rest + 63) / 64, (rest + 63) / 64, B), 256, gemmSmem, stream>>>(LU, N, k0, jb);
        }
        check(cudaGetLastError(), "LU launch");
    }
}

void luSolveBatch(const double *LU, const int *pivots, uint32_t N, uint32_t B, uint32_t E, double *x,
                  cudaStream_t stream, KernelTimer *timer) {
    const size_t smem = size_t(N) * sizeof(double2);
    if (smem > 227 * 1024)
        throw std::runtime_error("Dense solve vector exceeds shared memory (N too large for the dense form).");
    static size_t attr = 0;
    if (smem > 48 * 1024 && smem > attr) {
        check(cudaFuncSetAttribute(solveKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
              "solve smem attribute");
        attr = smem;
    }
    TimedScope s(timer, "lu_solve", stream);
    solveKernel<<<dim3(E, B), 256, smem, stream>>>(LU, pivots, N, E, x);
    check(cudaGetLastError(), "triangular solve launch");
}

void residualBatch(const double *A, const double *b, const double *x, const double *mass, uint32_t N, uint32_t B,
                   uint32_t E, double *correction, double *norms, cudaStream_t stream, KernelTimer *timer) {
    TimedScope s(timer, "residual", stream);
    double *squares = norms + 2 * size_t(B) * E;  // scratch after the norms
    residualKernel<<<dim3((N + 127) / 128, E, B), 128, 0, stream>>>(A, b, x, mass, N, E, correction, squares);
    normKernel<<<unsigned(B * E), 256, 0, stream>>>(squares, N, norms);
    check(cudaGetLastError(), "residual launch");
}

void addCorrectionBatch(double *x, const double *correction, size_t count, cudaStream_t stream) {
    addKernel<<<unsigned((count + 255) / 256), 256, 0, stream>>>(x, correction, count);
    check(cudaGetLastError(), "refinement update launch");
}

size_t luWorkspaceBytes(uint32_t N, uint32_t B) { return size_t(B) * N * sizeof(int); }

}  // namespace hsb
