// Observer pressure from the boundary traces (cuda_solver.cu:609-673,
// panel_integrals.cuh:298-443): finite points p(x) = sum_T (D p - S q) with
// adaptive quartering of panels within two edge lengths of the observer,
// or the asymptotic far field F(d) exp(-ikR)/R. FP64 throughout; one CTA
// per (frequency, excitation, observer, 256-panel tile), reduced over tiles
// in a fixed order.
#include "device_types.cuh"
#include "host_mesh.hpp"
#include "kernel_timer.hpp"

#include <stdexcept>
#include <string>

namespace hsb {
namespace {

constexpr double kInvFourPi = 0.07957747154594766788;
constexpr int kTile = 256;
// Field rules of degree 4, 6, 8, 12, 14: 6 + 12 + 16 + 49 + 64 points.
constexpr int kFieldPoints = 147;
__constant__ double cField[kFieldPoints * 4];

__device__ __forceinline__ void ruleOf(uint32_t degree, int &offset, int &count) {
    switch (degree) {
    case 4: offset = 0; count = 6; break;
    case 6: offset = 6; count = 12; break;
    case 8: offset = 18; count = 16; break;
    case 12: offset = 34; count = 49; break;
    default: offset = 83; count = 64; break;
    }
}

struct FieldPatch {
    double b[9];
    double fraction;
    uint32_t depth;
};

__device__ FieldPatch child(const FieldPatch &p, int c) {
    double ab[3], ac[3], bc[3];
    for (int i = 0; i < 3; ++i) {
        ab[i] = (p.b[i] + p.b[3 + i]) * .5;
        ac[i] = (p.b[i] + p.b[6 + i]) * .5;
        bc[i] = (p.b[3 + i] + p.b[6 + i]) * .5;
    }
    FieldPatch r;
    r.fraction = p.fraction * .25;
    r.depth = p.depth + 1;
    const double *v0, *v1, *v2;
    if (c == 0) { v0 = p.b; v1 = ab; v2 = ac; }
    else if (c == 1) { v0 = ab; v1 = p.b + 3; v2 = bc; }
    else if (c == 2) { v0 = ac; v1 = bc; v2 = p.b + 6; }
    else { v0 = ab; v1 = bc; v2 = ac; }
    for (int i = 0; i < 3; ++i) {
        r.b[i] = v0[i];
        r.b[3 + i] = v1[i];
        r.b[6 + i] = v2[i];
    }
    return r;
}

// One patch of D p - S q at observer x with its absolute scale.
__device__ void patchField(const double *x, const DPanel &pn, const FieldPatch &fp, int ro, int rc,
                           const double *pressure, double qr, double qi, double k, double &vr, double &vi,
                           double &scale, bool &bad) {
    vr = vi = scale = 0;
    double p[6];
    for (int i = 0; i < 3; ++i) {
        p[2 * i] = pressure[2 * pn.nodes[i]];
        p[2 * i + 1] = pressure[2 * pn.nodes[i] + 1];
    }
    for (int s = 0; s < rc; ++s) {
        const double *q = cField + 4 * (ro + s);
        double bary[3];
        for (int i = 0; i < 3; ++i)
            bary[i] = fp.b[i] * q[0] + fp.b[3 + i] * q[1] + fp.b[6 + i] * q[2];
        const double dx = (x[0] - pn.v0[0]) - (pn.e1[0] * bary[1] + pn.e2[0] * bary[2]);
        const double dy = (x[1] - pn.v0[1]) - (pn.e1[1] * bary[1] + pn.e2[1] * bary[2]);
        const double dz = (x[2] - pn.v0[2]) - (pn.e1[2] * bary[1] + pn.e2[2] * bary[2]);
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        bad |= !(r > 0);
        double sn, cs;
        sincos(k * r, &sn, &cs);
        const double sc = 2.0 * pn.area * fp.fraction * q[3] * kInvFourPi / r;
        const double gr = cs * sc, gi = -sn * sc;
        const double nf = (dx * pn.n[0] + dy * pn.n[1] + dz * pn.n[2]) / (r * r);
        const double dr = (gr - gi * k * r) * nf, di = (gi + gr * k * r) * nf;
        const double pr = p[0] * bary[0] + p[2] * bary[1] + p[4] * bary[2];
        const double pi = p[1] * bary[0] + p[3] * bary[1] + p[5] * bary[2];
        const double dpr = dr * pr - di * pi, dpi = dr * pi + di * pr;
        const double sqr = gr * qr - gi * qi, sqi = gr * qi + gi * qr;
        vr += dpr - sqr;
        vi += dpi - sqi;
        scale += hypot(dpr, dpi) + hypot(sqr, sqi);
    }
}

__device__ void nearField(const double *x, const DPanel &pn, int ro, int rc, const double *pressure, double qr,
                          double qi, double k, double tol, uint32_t maxDepth, double &outr, double &outi,
                          int *error, bool &bad) {
    FieldPatch stack[34];
    int pending = 1;
    stack[0] = FieldPatch{{1, 0, 0, 0, 1, 0, 0, 0, 1}, 1.0, 0};
    outr = outi = 0;
    while (pending) {
        const FieldPatch fp = stack[--pending];
        double cr, ci, cs;
        patchField(x, pn, fp, ro, rc, pressure, qr, qi, k, cr, ci, cs, bad);
        double fr = 0, fi = 0, fs = 0;
        for (int c = 0; c < 4; ++c) {
            double vr, vi, vs;
            patchField(x, pn, child(fp, c), ro, rc, pressure, qr, qi, k, vr, vi, vs, bad);
            fr += vr;
            fi += vi;
            fs += vs;
        }
        if (hypot(fr - cr, fi - ci) <= tol * fmax(fs, 1e-300)) {
            outr += fr;
            outi += fi;
        } else {
            if (fp.depth >= maxDepth || pending + 4 > 34) {
                atomicExch(error, kErrFieldDepth);
                outr = outi = 0;
                return;
            }
            for (int c = 0; c < 4; ++c)
                stack[pending++] = child(fp, c);
        }
    }
}

__global__ void __launch_bounds__(128) fieldKernel(FieldRequest req, const double *ks, const double *pressure,
                                                   const double *flux, const uint32_t *batchDegree, double *partials,
                                                   int *error) {
    __shared__ double red[2][4];
    const uint32_t tiles = (req.T + kTile - 1) / kTile;
    const uint32_t tile = blockIdx.x % tiles;
    uint32_t rest = blockIdx.x / tiles;
    const uint32_t o = rest % req.O;
    rest /= req.O;
    const uint32_t e = rest % req.E;
    const uint32_t f = rest / req.E;
    const double k = ks[f];
    int ro, rc;
    ruleOf(batchDegree[f], ro, rc);
    const double *p = pressure + (size_t(f) * req.E + e) * req.N * 2;
    const double *q = flux + (size_t(f) * req.E + e) * req.T * 2;
    const double *x = req.observers + 3 * o;
    double vr = 0, vi = 0;
    bool bad = false;
    const uint32_t end = min((tile + 1) * kTile, req.T);
    for (uint32_t t = tile * kTile + threadIdx.x; t < end; t += blockDim.x) {
        const DPanel &pn = req.panels[t];
        const double qr = q[2 * t], qi = q[2 * t + 1];
        if (req.farField) {
            const double nf = k * (x[0] * pn.n[0] + x[1] * pn.n[1] + x[2] * pn.n[2]);
            const double ox = pn.v0[0] - req.farOrigin[0], oy = pn.v0[1] - req.farOrigin[1], oz = pn.v0[2] - req.farOrigin[2];
            double pv[6];
            for (int i = 0; i < 3; ++i) {
                pv[2 * i] = p[2 * pn.nodes[i]];
                pv[2 * i + 1] = p[2 * pn.nodes[i] + 1];
            }
            for (int s = 0; s < rc; ++s) {
                const double *w = cField + 4 * (ro + s);
                const double px = ox + pn.e1[0] * w[1] + pn.e2[0] * w[2];
                const double py = oy + pn.e1[1] * w[1] + pn.e2[1] * w[2];
                const double pz = oz + pn.e1[2] * w[1] + pn.e2[2] * w[2];
                const double phase = k * (x[0] * px + x[1] * py + x[2] * pz);
                bad |= !isfinite(phase);
                double sn, cs;
                sincos(phase, &sn, &cs);
                const double sc = 2 * pn.area * w[3] * kInvFourPi;
                const double pr = pv[0] * w[0] + pv[2] * w[1] + pv[4] * w[2];
                const double pi = pv[1] * w[0] + pv[3] * w[1] + pv[5] * w[2];
                const double ir = -nf * pi - qr, ii = nf * pr - qi;
                vr += (cs * ir - sn * ii) * sc;
                vi += (cs * ii + sn * ir) * sc;
            }
        } else {
            const double cx = x[0] - (pn.v0[0] + (pn.e1[0] + pn.e2[0]) / 3.0);
            const double cy = x[1] - (pn.v0[1] + (pn.e1[1] + pn.e2[1]) / 3.0);
            const double cz = x[2] - (pn.v0[2] + (pn.e1[2] + pn.e2[2]) / 3.0);
            double ar, ai, as;
            if (cx * cx + cy * cy + cz * cz > 4 * pn.maxEdge * pn.maxEdge) {
                const FieldPatch whole{{1, 0, 0, 0, 1, 0, 0, 0, 1}, 1.0, 0};
                patchField(x, pn, whole, ro, rc, p, qr, qi, k, ar, ai, as, bad);
            } else
                nearField(x, pn, ro, rc, p, qr, qi, k, req.tolerance, req.maximumDepth, ar, ai, error, bad);
            vr += ar;
            vi += ai;
        }
    }
    if (bad)
        atomicExch(error, kErrDistance);
    if (req.farField) {
        double sn, cs;
        sincos(k * req.farDistance, &sn, &cs);
        const double r = (vr * cs + vi * sn) / req.farDistance, i = (vi * cs - vr * sn) / req.farDistance;
        vr = r;
        vi = i;
    }
    for (int off = 16; off > 0; off >>= 1) {
        vr += __shfl_down_sync(0xffffffffu, vr, off);
        vi += __shfl_down_sync(0xffffffffu, vi, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = vr;
        red[1][threadIdx.x >> 5] = vi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = red[0][0] + red[0][1] + red[0][2] + red[0][3];
        partials[2 * blockIdx.x + 1] = red[1][0] + red[1][1] + red[1][2] + red[1][3];
    }
}

__global__ void finishKernel(const double *partials, uint32_t tiles, size_t outputs, double *out, int *error) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= outputs)
        return;
    double r = 0, im = 0;
    for (uint32_t t = 0; t < tiles; ++t) {
        r += partials[2 * (i * tiles + t)];
        im += partials[2 * (i * tiles + t) + 1];
    }
    if (!isfinite(r) || !isfinite(im))
        atomicExch(error, kErrNonFinite);
    out[2 * i] = r;
    out[2 * i + 1] = im;
}

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

size_t fieldPartialsBytes(uint32_t T, uint32_t E, uint32_t O, uint32_t B) {
    return size_t(B) * E * O * ((T + kTile - 1) / kTile) * 2 * sizeof(double);
}

void evaluateFieldBatch(const FieldRequest &req, const double *ks, const double *pressure, const double *flux,
                        const uint32_t *batchDegree, double *partials, double *out, int *error, cudaStream_t stream,
                        KernelTimer *timer) {
    static bool uploaded = false;
    if (!uploaded) {
        double table[kFieldPoints * 4];
        int o = 0;
        for (unsigned d : {4u, 6u, 8u, 12u, 14u})
            for (const auto &p : triangleRule(d)) {
                table[4 * o] = p.b[0];
                table[4 * o + 1] = p.b[1];
                table[4 * o + 2] = p.b[2];
                table[4 * o + 3] = p.w;
                ++o;
            }
        check(cudaMemcpyToSymbolAsync(cField, table, sizeof(table), 0, cudaMemcpyHostToDevice, stream),
              "field rule upload");
        check(cudaStreamSynchronize(stream), "field rule upload");
        uploaded = true;
    }
    const uint32_t tiles = (req.T + kTile - 1) / kTile;
    const size_t outputs = size_t(req.B) * req.E * req.O;
    if (!outputs)
        return;
    TimedScope s(timer, "field", stream);
    fieldKernel<<<unsigned(outputs * tiles), 128, 0, stream>>>(req, ks, pressure, flux, batchDegree, partials, error);
    finishKernel<<<unsigned((outputs + 127) / 128), 128, 0, stream>>>(partials, tiles, outputs, out, error);
    check(cudaGetLastError(), "field launch");
}

}  // namespace hsb
