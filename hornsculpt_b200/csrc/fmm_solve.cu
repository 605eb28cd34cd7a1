// Fast-multipole linear system: near CSR matrix, block-Jacobi preconditioner
// and the restarted GMRES driver (SupportFmmLinearSolver::solveSeed,
// cuda/support_fmm_solve.cu:401-525, without the finer-seed audit).
#include "device_types.cuh"
#include "fmm.hpp"
#include "kernel_timer.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

namespace hsb {
namespace {

void sysCheck(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw CudaError(std::string("CUDA fast multipole system ") + what + ": " + cudaGetErrorString(e));
}

struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
    Buf() = default;
    Buf(const Buf &) = delete;
    Buf &operator=(const Buf &) = delete;
    ~Buf() {
        if (p)
            cudaFree(p);
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
    void ensure(size_t n) {
        if (n <= bytes)
            return;
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, n) != cudaSuccess) {
            p = nullptr;
            throw OutOfMemory("CUDA fast multipole system allocation failed.");
        }
        bytes = n;
    }
    template <class T> void upload(const std::vector<T> &v, cudaStream_t s) {
        ensure(std::max<size_t>(v.size() * sizeof(T), 16));
        if (!v.empty())
            sysCheck(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
    }
};

constexpr uint32_t kMaxBlock = 64;

// y_i = sum_e vals[e] x[col e] + rowScale_i far_i, one warp per row (fixed order).
__global__ void spmvKernel(const uint32_t *__restrict__ rowStart, const uint32_t *__restrict__ cols,
                           const double2 *__restrict__ vals, const double2 *__restrict__ x, const double2 *__restrict__ far,
                           const double *__restrict__ rowScale, uint32_t N, double2 *y) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= N)
        return;
    double re = 0, im = 0;
    for (uint32_t e = rowStart[row] + lane; e < rowStart[row + 1]; e += 32) {
        const double2 a = vals[e], v = x[cols[e]];
        re += a.x * v.x - a.y * v.y;
        im += a.x * v.y + a.y * v.x;
    }
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) {
        const double2 f = far[row];
        const double s = rowScale[row];
        y[row] = make_double2(re + s * f.x, im + s * f.y);
    }
}

// The mixed form's near product in FP32: FP32 values and products of the
// rounded input, FP32 accumulation; the FP64 far part added with the row scale.
__global__ void spmv32Kernel(const uint32_t *__restrict__ rowStart, const uint32_t *__restrict__ cols,
                             const float2 *__restrict__ vals, const double2 *__restrict__ x,
                             const double2 *__restrict__ far, const double *__restrict__ rowScale, uint32_t N,
                             double2 *y) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= N)
        return;
    float re = 0, im = 0;
    for (uint32_t e = rowStart[row] + lane; e < rowStart[row + 1]; e += 32) {
        const float2 a = vals[e];
        const double2 xd = x[cols[e]];
        const float vx = float(xd.x), vy = float(xd.y);
        re += a.x * vx - a.y * vy;
        im += a.x * vy + a.y * vx;
    }
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) {
        const double2 f = far[row];
        const double s = rowScale[row];
        y[row] = make_double2(double(re) + s * f.x, double(im) + s * f.y);
    }
}

__global__ void roundValuesKernel(const double2 *in, float2 *out, size_t count) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i < count)
        out[i] = make_float2(float(in[i].x), float(in[i].y));
}

// Inverse of each diagonal block by Gauss-Jordan with partial pivoting in
// shared memory ([M | I], nb <= 64). A zero pivot leaves the identity for the
// block and raises the flag.
__global__ void __launch_bounds__(256) blockInverseKernel(const uint32_t *__restrict__ blockStart,
                                                          const uint32_t *__restrict__ blockVerts,
                                                          const uint32_t *__restrict__ rowStart,
                                                          const uint32_t *__restrict__ cols,
                                                          const double2 *__restrict__ vals,
                                                          const uint64_t *__restrict__ invStart, double2 *inv,
                                                          int *flag) {
    extern __shared__ double2 aug[];  // nb x 2nb, row-major
    __shared__ double2 factor[kMaxBlock];
    __shared__ int pivotRow;
    __shared__ int singular;
    const uint32_t b0 = blockStart[blockIdx.x], nb = blockStart[blockIdx.x + 1] - b0;
    const uint32_t w = 2 * nb;
    for (uint32_t e = threadIdx.x; e < nb * w; e += blockDim.x) {
        const uint32_t r = e / w, c = e % w;
        double2 v = make_double2(0, 0);
        if (c < nb) {
            const uint32_t vi = blockVerts[b0 + r], vj = blockVerts[b0 + c];
            uint32_t lo = rowStart[vi], hi = rowStart[vi + 1];
            while (lo < hi) {  // cols sorted per row
                const uint32_t mid = (lo + hi) / 2;
                if (cols[mid] < vj)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            if (lo < rowStart[vi + 1] && cols[lo] == vj)
                v = vals[lo];
        } else if (c - nb == r)
            v = make_double2(1, 0);
        aug[e] = v;
    }
    if (threadIdx.x == 0)
        singular = 0;
    __syncthreads();
    for (uint32_t c = 0; c < nb; ++c) {
        if (threadIdx.x == 0) {
            uint32_t best = c;
            double mag = -1;
            for (uint32_t r = c; r < nb; ++r) {
                const double2 v = aug[r * w + c];
                const double m = v.x * v.x + v.y * v.y;
                if (m > mag) {
                    mag = m;
                    best = r;
                }
            }
            pivotRow = int(best);
            if (!(mag > 0))
                singular = 1;
        }
        __syncthreads();
        if (singular)
            break;
        const uint32_t pr = uint32_t(pivotRow);
        if (pr != c)
            for (uint32_t k = threadIdx.x; k < w; k += blockDim.x) {
                const double2 t = aug[c * w + k];
                aug[c * w + k] = aug[pr * w + k];
                aug[pr * w + k] = t;
            }
        __syncthreads();
        const double2 p = aug[c * w + c];
        const double den = p.x * p.x + p.y * p.y;
        const double2 ip = make_double2(p.x / den, -p.y / den);
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < w; k += blockDim.x) {
            const double2 v = aug[c * w + k];
            aug[c * w + k] = make_double2(v.x * ip.x - v.y * ip.y, v.x * ip.y + v.y * ip.x);
        }
        // column c of every row is read before any row is updated: the thread that
        // updates (r, c) would otherwise overwrite the factor other threads of row r
        // still have to read
        for (uint32_t r = threadIdx.x; r < nb; r += blockDim.x)
            factor[r] = aug[r * w + c];
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < nb * w; e += blockDim.x) {
            const uint32_t r = e / w, k = e % w;
            if (r == c)
                continue;
            const double2 f = factor[r], v = aug[c * w + k];
            aug[e] = make_double2(aug[e].x - (f.x * v.x - f.y * v.y), aug[e].y - (f.x * v.y + f.y * v.x));
        }
        __syncthreads();
    }
    double2 *out = inv + invStart[blockIdx.x];
    for (uint32_t e = threadIdx.x; e < nb * nb; e += blockDim.x) {
        const uint32_t r = e / nb, c = e % nb;
        out[e] = singular ? make_double2(r == c ? 1.0 : 0.0, 0.0) : aug[r * w + nb + c];
    }
    if (singular && threadIdx.x == 0)
        atomicExch(flag, 1);
}

// out[v] = sum_b inv[a][b] in[v_b] per block and system (in-place safe).
__global__ void blockApplyKernel(const uint32_t *__restrict__ blockStart, const uint32_t *__restrict__ blockVerts,
                                 const uint64_t *__restrict__ invStart, const double2 *__restrict__ inv,
                                 const double2 *in, double2 *out, uint32_t N) {
    __shared__ double2 v[kMaxBlock];
    const uint32_t b0 = blockStart[blockIdx.x], nb = blockStart[blockIdx.x + 1] - b0;
    const size_t so = size_t(blockIdx.y) * N;
    for (uint32_t a = threadIdx.x; a < nb; a += blockDim.x)
        v[a] = in[so + blockVerts[b0 + a]];
    __syncthreads();
    const double2 *B = inv + invStart[blockIdx.x];
    for (uint32_t a = threadIdx.x; a < nb; a += blockDim.x) {
        double re = 0, im = 0;
        for (uint32_t c = 0; c < nb; ++c) {
            const double2 m = B[a * nb + c], x = v[c];
            re += m.x * x.x - m.y * x.y;
            im += m.x * x.y + m.y * x.x;
        }
        out[so + blockVerts[b0 + a]] = make_double2(re, im);
    }
}

// r = b - y and the mass-weighted norms |r|_M, |b|_M per system (fixed-order block sums).
__global__ void __launch_bounds__(256) residualNormKernel(const double2 *__restrict__ b, const double2 *__restrict__ y,
                                                          const double *__restrict__ mass, uint32_t N, double2 *r,
                                                          double *norms) {
    __shared__ double sr[256], sb[256];
    const size_t so = size_t(blockIdx.x) * N;
    double ar = 0, ab = 0;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
        const double2 bb = b[so + i], yy = y[so + i];
        const double2 d = make_double2(bb.x - yy.x, bb.y - yy.y);
        r[so + i] = d;
        ar += mass[i] * (d.x * d.x + d.y * d.y);
        ab += mass[i] * (bb.x * bb.x + bb.y * bb.y);
    }
    sr[threadIdx.x] = ar;
    sb[threadIdx.x] = ab;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < unsigned(s)) {
            sr[threadIdx.x] += sr[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        norms[2 * blockIdx.x] = sqrt(sr[0]);
        norms[2 * blockIdx.x + 1] = sqrt(sb[0]);
    }
}

__global__ void addKernel(double *x, const double *d, size_t count) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i < count)
        x[i] += d[i];
}

}  // namespace

struct FmmSystem::Impl {
    uint32_t N = 0, blocks = 0;
    const double *rowScale = nullptr, *mass = nullptr;
    Buf rowStart, cols, vals, blockStart, blockVerts, invStart, inv, flag;
    Buf far, tmp, r, d, norms, gmres, vals32;
    size_t gmresBytes = 0;
    uint32_t gmresS = 0, gmresM = 0;
};

FmmSystem::FmmSystem(FmmOperator &op, const double *rowScale, const double *mass, uint32_t blockWidth)
    : impl_(std::make_unique<Impl>()), op_(op) {
    Impl &I = *impl_;
    const auto &row = op.nearRowStart();
    I.N = uint32_t(row.size() - 1);
    I.rowScale = rowScale;
    I.mass = mass;
    cudaStream_t s = nullptr;
    I.rowStart.upload(row, s);
    I.cols.upload(op.nearCols(), s);
    I.vals.ensure(std::max<size_t>(op.nearCols().size(), 1) * 16);
    // diagonal blocks: consecutive leaves in tree order (spatially adjacent)
    // merged up to the block width, a leaf above it split
    const FmmTree &t = op.tree();
    const uint32_t width = std::clamp<uint32_t>(blockWidth, 1, kMaxBlock);
    std::vector<uint32_t> bs{0}, bv;
    std::vector<uint64_t> is{0};
    std::vector<uint32_t> cur;
    const auto flush = [&]() {
        if (cur.empty())
            return;
        std::sort(cur.begin(), cur.end());
        bv.insert(bv.end(), cur.begin(), cur.end());
        bs.push_back(uint32_t(bv.size()));
        is.push_back(is.back() + uint64_t(cur.size()) * cur.size());
        cur.clear();
    };
    for (const auto &n : t.nodes) {
        if (!n.leaf() || !n.countP)
            continue;
        if (cur.size() + n.countP > width)
            flush();
        for (uint32_t q = 0; q < n.countP; ++q) {
            cur.push_back(t.pressureOrder[n.firstP + q]);
            if (cur.size() == width)
                flush();
        }
    }
    flush();
    if (bv.size() != I.N)
        throw std::logic_error("fast multipole: leaf blocks do not cover the vertices");
    I.blocks = uint32_t(bs.size() - 1);
    I.blockStart.upload(bs, s);
    I.blockVerts.upload(bv, s);
    I.invStart.upload(is, s);
    I.inv.ensure(is.back() * 16);
    I.flag.ensure(16);
    sysCheck(cudaStreamSynchronize(s), "setup");
}

FmmSystem::~FmmSystem() = default;

static __global__ void addScaledKernel(double2 *b, const double2 *far, const double *rowScale, uint32_t N, size_t count) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= count)
        return;
    const double s = rowScale[i % N];
    b[i] = make_double2(b[i].x + s * far[i].x, b[i].y + s * far[i].y);
}

double *FmmSystem::nearValues() { return impl_->vals.as<double>(); }
const uint32_t *FmmSystem::nearRowDevice() const { return impl_->rowStart.as<uint32_t>(); }
const uint32_t *FmmSystem::nearColDevice() const { return impl_->cols.as<uint32_t>(); }

void FmmSystem::addScaled(double *b, const double *far, uint32_t S, cudaStream_t stream) {
    const size_t count = size_t(S) * impl_->N;
    addScaledKernel<<<unsigned((count + 255) / 256), 256, 0, stream>>>(reinterpret_cast<double2 *>(b),
                                                                       reinterpret_cast<const double2 *>(far),
                                                                       impl_->rowScale, impl_->N, count);
    sysCheck(cudaGetLastError(), "rhs far launch");
}

void FmmSystem::residual(const double *b, const double *x, uint32_t S, double *r, std::vector<double> &relative,
                         cudaStream_t stream, KernelTimer *timer) {
    Impl &I = *impl_;
    I.tmp.ensure(size_t(S) * I.N * 16);
    I.norms.ensure(size_t(S) * 16);
    apply(x, size_t(I.N) * 2, S, I.tmp.as<double>(), stream, timer);
    residualNormKernel<<<S, 256, 0, stream>>>(reinterpret_cast<const double2 *>(b), I.tmp.as<double2>(), I.mass, I.N,
                                              reinterpret_cast<double2 *>(r), I.norms.as<double>());
    sysCheck(cudaGetLastError(), "residual launch");
    std::vector<double> norms(2 * S);
    sysCheck(cudaMemcpyAsync(norms.data(), I.norms.p, norms.size() * 8, cudaMemcpyDeviceToHost, stream), "norms");
    sysCheck(cudaStreamSynchronize(stream), "residual");
    relative.resize(S);
    for (uint32_t s = 0; s < S; ++s)
        relative[s] = norms[2 * s + 1] > 0 ? norms[2 * s] / norms[2 * s + 1] : 0.0;
}

void FmmSystem::add(double *x, const double *d, size_t reals, cudaStream_t stream) {
    addKernel<<<unsigned((reals + 255) / 256), 256, 0, stream>>>(x, d, reals);
    sysCheck(cudaGetLastError(), "add launch");
}

void FmmSystem::factorBlocks(cudaStream_t stream, KernelTimer *timer) {
    Impl &I = *impl_;
    TimedScope scope(timer, "fmm_block_jacobi", stream);
    sysCheck(cudaMemsetAsync(I.flag.p, 0, sizeof(int), stream), "flag reset");
    const size_t sm = size_t(kMaxBlock) * 2 * kMaxBlock * 16;
    sysCheck(cudaFuncSetAttribute(blockInverseKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)),
             "block smem");
    blockInverseKernel<<<I.blocks, 256, sm, stream>>>(I.blockStart.as<uint32_t>(), I.blockVerts.as<uint32_t>(),
                                                     I.rowStart.as<uint32_t>(), I.cols.as<uint32_t>(),
                                                     I.vals.as<double2>(), I.invStart.as<uint64_t>(),
                                                     I.inv.as<double2>(), I.flag.as<int>());
    sysCheck(cudaGetLastError(), "block inverse launch");
}

void FmmSystem::apply(const double *x, size_t stride, uint32_t S, double *y, cudaStream_t stream, KernelTimer *timer) {
    Impl &I = *impl_;
    I.far.ensure(size_t(S) * I.N * 16);
    op_.applyFar(x, stride, S, I.far.as<double>(), stream, timer);
    TimedScope scope(timer, "fmm_near", stream);
    for (uint32_t s = 0; s < S; ++s)
        spmvKernel<<<(I.N * 32 + 255) / 256, 256, 0, stream>>>(
            I.rowStart.as<uint32_t>(), I.cols.as<uint32_t>(), I.vals.as<double2>(),
            reinterpret_cast<const double2 *>(x + s * stride), I.far.as<double2>() + size_t(s) * I.N, I.rowScale, I.N,
            reinterpret_cast<double2 *>(y) + size_t(s) * I.N);
    sysCheck(cudaGetLastError(), "near product launch");
}

void FmmSystem::roundNearValues(cudaStream_t stream) {
    Impl &I = *impl_;
    const size_t nnz = std::max<size_t>(op_.nearCols().size(), 1);
    I.vals32.ensure(nnz * 8);
    roundValuesKernel<<<unsigned((nnz + 255) / 256), 256, 0, stream>>>(I.vals.as<double2>(), I.vals32.as<float2>(),
                                                                      op_.nearCols().size());
    sysCheck(cudaGetLastError(), "near value rounding launch");
}

void FmmSystem::applyInner(FmmOperator &inner, const double *x, size_t stride, uint32_t S, double *y,
                           cudaStream_t stream, KernelTimer *timer) {
    Impl &I = *impl_;
    I.far.ensure(size_t(S) * I.N * 16);
    inner.applyFar(x, stride, S, I.far.as<double>(), stream, timer);
    TimedScope scope(timer, "fmm_near_fp32", stream);
    for (uint32_t s = 0; s < S; ++s)
        spmv32Kernel<<<(I.N * 32 + 255) / 256, 256, 0, stream>>>(
            I.rowStart.as<uint32_t>(), I.cols.as<uint32_t>(), I.vals32.as<float2>(),
            reinterpret_cast<const double2 *>(x + s * stride), I.far.as<double2>() + size_t(s) * I.N, I.rowScale, I.N,
            reinterpret_cast<double2 *>(y) + size_t(s) * I.N);
    sysCheck(cudaGetLastError(), "FP32 near product launch");
}

void FmmSystem::precondition(const double *in, double *out, uint32_t S, cudaStream_t stream) {
    Impl &I = *impl_;
    blockApplyKernel<<<dim3(I.blocks, S), 64, 0, stream>>>(I.blockStart.as<uint32_t>(), I.blockVerts.as<uint32_t>(),
                                                          I.invStart.as<uint64_t>(), I.inv.as<double2>(),
                                                          reinterpret_cast<const double2 *>(in),
                                                          reinterpret_cast<double2 *>(out), I.N);
    sysCheck(cudaGetLastError(), "block apply launch");
}

void FmmSystem::solve(const double *b, double *x, uint32_t S, double target, uint32_t restart, uint32_t maxIterations,
                      cudaStream_t stream, KernelTimer *timer, std::vector<double> &relative,
                      std::vector<uint32_t> &iterations, FmmOperator *inner) {
    Impl &I = *impl_;
    const uint32_t N = I.N;
    const size_t reals = size_t(S) * N * 2;
    I.tmp.ensure(reals * 8);
    I.r.ensure(reals * 8);
    I.norms.ensure(size_t(S) * 16);
    if (I.gmresS != S || I.gmresM != restart) {
        I.gmres.ensure(gmresWorkspaceBytes(N, S, restart));
        I.gmresS = S;
        I.gmresM = restart;
    }
    sysCheck(cudaMemsetAsync(x, 0, reals * 8, stream), "solution reset");
    relative.assign(S, 1.0);
    iterations.assign(S, 0);
    std::vector<double> norms(2 * S);
    int singular = 0;
    sysCheck(cudaMemcpyAsync(&singular, I.flag.p, sizeof(int), cudaMemcpyDeviceToHost, stream), "flag");
    // GMRES-IR with an inner operator (the mixed form): the Krylov cycles apply the
    // FP32 operator (scaled FP32 translations, FP32 near values) and each cycle
    // only needs to win a few digits (the FP32 operator holds about six); the
    // residual every cycle starts from is the FP64 operator's.
    const auto applyA = [&](const double *in, size_t stride, double *out) {
        if (inner)
            applyInner(*inner, in, stride, S, out, stream, timer);
        else
            apply(in, stride, S, out, stream, timer);
    };
    const double innerFloor = inner ? 1e-4 : 1e-13;
    const auto pre = [&](const double *in, double *out) { precondition(in, out, S, stream); };
    for (uint32_t total = 0;;) {
        // true residual of the operator
        apply(x, size_t(N) * 2, S, I.tmp.as<double>(), stream, timer);
        residualNormKernel<<<S, 256, 0, stream>>>(reinterpret_cast<const double2 *>(b),
                                                  I.tmp.as<double2>(), I.mass, N, I.r.as<double2>(),
                                                  I.norms.as<double>());
        sysCheck(cudaGetLastError(), "residual launch");
        sysCheck(cudaMemcpyAsync(norms.data(), I.norms.p, norms.size() * 8, cudaMemcpyDeviceToHost, stream),
                 "norms");
        sysCheck(cudaStreamSynchronize(stream), "residual");
        if (singular)
            throw NumericError("Fast-multipole block-Jacobi preconditioner met a singular diagonal block.");
        bool done = true;
        std::vector<double> tol(S);
        for (uint32_t s = 0; s < S; ++s) {
            const double rel = norms[2 * s + 1] > 0 ? norms[2 * s] / norms[2 * s + 1] : 0.0;
            if (!std::isfinite(rel))
                throw NumericError("Fast-multipole residual is not finite.");
            relative[s] = rel;
            tol[s] = rel > target ? std::clamp(0.1 * target / rel, innerFloor, 0.5) : 1.0;
            done = done && rel <= target;
        }
        if (done)
            return;
        if (total >= maxIterations)
            throw NoConvergence("Fast-multipole GMRES did not reach the residual tolerance within the iteration limit.");
        // correction d: A d = r, added to x
        I.d.ensure(reals * 8);
        sysCheck(cudaMemsetAsync(I.d.p, 0, reals * 8, stream), "correction reset");
        std::vector<uint32_t> steps;
        const uint32_t m = std::min(restart, maxIterations - total);
        const uint32_t j = gmresCycleOperator(N, S, I.r.as<double>(), I.d.as<double>(), m, tol, I.gmres.p, stream,
                                              timer, steps, applyA, pre);
        for (uint32_t s = 0; s < S; ++s)
            iterations[s] += steps[s];
        total += std::max(j, 1u);
        addKernel<<<unsigned((reals + 255) / 256), 256, 0, stream>>>(x, I.d.as<double>(), reals);
        sysCheck(cudaGetLastError(), "correction launch");
    }
}

}  // namespace hsb
