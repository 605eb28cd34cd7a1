// Observer pressure from the boundary traces (cuda_solver.cu:609-673,
// panel_integrals.cuh:298-443): finite points p(x) = sum_T (D p - S q) with
// adaptive quartering of panels within two edge lengths of the observer,
// or the asymptotic far field F(d) exp(-ikR)/R. FP64 throughout; one CTA
// per (frequency, excitation, observer, 256-panel tile), reduced over tiles
// in a fixed order.
#include "device_once.hpp"
#include "device_types.cuh"
#include "host_mesh.hpp"
#include "kernel_timer.hpp"

#include <algorithm>
#include <cmath>
#include <mutex>
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

constexpr int32_t kFieldAir = 0, kFieldBoundary = 1, kFieldExcluded = 2, kFieldNotConverged = 3;

// ---------------------------------------------------------------------------
// Post-solve pressure samples at arbitrary points (the exterior form of
// evaluatePressureField, field_evaluation.cpp:330-463): a point within
// minDistance of a panel is "boundary"; otherwise the summed solid angle of
// the panels (field_evaluation.cpp:70-75) decides inside ("excluded") or air;
// air points get p(x) = sum over panels of (D p - S q), each panel integrated
// adaptively (field_evaluation.cpp:85-142): a patch is accepted when its phase
// span k h sqrt(fraction) <= pi and the degree-4 and degree-8 rules agree to
// tolerance times the fine magnitude, else it is quartered, up to maxDepth
// (beyond it the point is "not converged"). One CTA per point, threads over
// panels with an explicit depth-first patch stack in the reference's child
// order; the per-thread sums are added in a fixed order.
// ---------------------------------------------------------------------------
constexpr int kFieldThreads = 256;
constexpr int kFieldStack = 3 * 12 + 1;  // depth-first stack for maxDepth <= 12

// closest-point distance from p to a panel (Ericson, Real-Time Collision
// Detection, 5.1.5, as field_evaluation.cpp:44-69)
__device__ double pointPanelDistance(V3 p, const DPanel &t) {
    const V3 a = v3(t.v0[0], t.v0[1], t.v0[2]), ab = v3(t.e1[0], t.e1[1], t.e1[2]), ac = v3(t.e2[0], t.e2[1], t.e2[2]);
    const V3 b = a + ab, c = a + ac;
    const V3 ap = p - a;
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0)
        return sqrt(norm2(ap));
    const V3 bp = p - b;
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3)
        return sqrt(norm2(bp));
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0)
        return sqrt(norm2(ap - ab * (d1 / (d1 - d3))));
    const V3 cp = p - c;
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6)
        return sqrt(norm2(cp));
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0)
        return sqrt(norm2(ap - ac * (d2 / (d2 - d6))));
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && d4 >= d3 && d5 >= d6) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return sqrt(norm2(bp - (c - b) * w));
    }
    return fabs(dot(ap, v3(t.n[0], t.n[1], t.n[2])));
}

// solid angle of a panel seen from p (Van Oosterom and Strackee)
__device__ double panelSolidAngle(V3 p, const DPanel &t) {
    const V3 a = v3(t.v0[0], t.v0[1], t.v0[2]) - p;
    const V3 b = a + v3(t.e1[0], t.e1[1], t.e1[2]), c = a + v3(t.e2[0], t.e2[1], t.e2[2]);
    const double la = sqrt(norm2(a)), lb = sqrt(norm2(b)), lc = sqrt(norm2(c));
    return 2 * atan2(dot(a, cross(b, c)), la * lb * lc + dot(a, b) * lc + dot(b, c) * la + dot(c, a) * lb);
}

struct SamplePatch {
    double b[9];  // barycentrics of the patch corners in the panel
    double fraction;
    uint32_t depth;
};

// D p - S q over one patch with one rule, and the magnitude sum |D p| + |S q|
__device__ void patchIntegral(const DPanel &t, const SamplePatch &patch, V3 x, double k, const double (&p)[6],
                              double qr, double qi, int offset, int count, double &re, double &im, double &mag) {
    re = im = mag = 0;
    const V3 n = v3(t.n[0], t.n[1], t.n[2]);
    for (int r = 0; r < count; ++r) {
        const double *rule = cField + 4 * (offset + r);
        double b[3];
        for (int i = 0; i < 3; ++i)
            b[i] = patch.b[i] * rule[0] + patch.b[3 + i] * rule[1] + patch.b[6 + i] * rule[2];
        // y = v0 b0 + v1 b1 + v2 b2 with v1 = v0 + e1, v2 = v0 + e2
        V3 y;
        y.x = t.v0[0] * b[0] + (t.v0[0] + t.e1[0]) * b[1] + (t.v0[0] + t.e2[0]) * b[2];
        y.y = t.v0[1] * b[0] + (t.v0[1] + t.e1[1]) * b[1] + (t.v0[1] + t.e2[1]) * b[2];
        y.z = t.v0[2] * b[0] + (t.v0[2] + t.e1[2]) * b[1] + (t.v0[2] + t.e2[2]) * b[2];
        const V3 d = x - y;
        const double rr = sqrt(norm2(d));
        double sn, cs;
        sincos(k * rr, &sn, &cs);
        const double gm = kInvFourPi / rr, gr = gm * cs, gi = -gm * sn;  // exp(-ikr) / (4 pi r)
        const double bq = b[0] + b[1] + b[2];
        const double sr = gr * qr * bq - gi * qi * bq, si = gr * qi * bq + gi * qr * bq;  // g (b . q)
        const double pr = b[0] * p[0] + b[1] * p[2] + b[2] * p[4], pi = b[0] * p[1] + b[1] * p[3] + b[2] * p[5];
        const double proj = dot(d, n) / rr;
        // g (1/r + i k) proj (b . p)
        const double hr = (gr / rr - gi * k) * proj, hi = (gi / rr + gr * k) * proj;
        const double dr = hr * pr - hi * pi, di = hr * pi + hi * pr;
        const double w = 2 * t.area * patch.fraction * rule[3];
        re += w * (dr - sr);
        im += w * (di - si);
        mag += w * (sqrt(dr * dr + di * di) + sqrt(sr * sr + si * si));
    }
}

__global__ void __launch_bounds__(kFieldThreads) pressureFieldKernel(const DPanel *__restrict__ panels, uint32_t T,
                                                                     const double *__restrict__ trace,
                                                                     const double *__restrict__ flux,
                                                                     const double *__restrict__ points, double k,
                                                                     double minDistance, double tolerance,
                                                                     uint32_t maxDepth, double *__restrict__ out,
                                                                     int32_t *__restrict__ status) {
    __shared__ double sA[kFieldThreads], sB[kFieldThreads];
    __shared__ int sFlag[kFieldThreads];
    const uint32_t pt = blockIdx.x, tid = threadIdx.x;
    const V3 x = v3(points[3 * pt], points[3 * pt + 1], points[3 * pt + 2]);
    // classification: boundary distance and solid angle
    int near = 0;
    double angle = 0;
    for (uint32_t t = tid; t < T; t += kFieldThreads) {
        near |= pointPanelDistance(x, panels[t]) <= minDistance;
        angle += panelSolidAngle(x, panels[t]);
    }
    sA[tid] = angle;
    sFlag[tid] = near;
    __syncthreads();
    for (int s = kFieldThreads / 2; s > 0; s >>= 1) {
        if (tid < unsigned(s)) {
            sA[tid] += sA[tid + s];
            sFlag[tid] |= sFlag[tid + s];
        }
        __syncthreads();
    }
    const bool boundary = sFlag[0] != 0;
    const bool inside = fabs(sA[0]) > 2 * 3.14159265358979323846;
    __syncthreads();
    if (boundary || inside) {
        if (tid == 0) {
            status[pt] = boundary ? kFieldBoundary : kFieldExcluded;
            out[2 * pt] = out[2 * pt + 1] = 0;
        }
        return;
    }
    // air: adaptive D p - S q per panel
    double re = 0, im = 0;
    int failed = 0;
    SamplePatch stack[kFieldStack];
    for (uint32_t t = tid; t < T && !failed; t += kFieldThreads) {
        const DPanel &panel = panels[t];
        double p[6];
        for (int i = 0; i < 3; ++i) {
            p[2 * i] = trace[2 * panel.nodes[i]];
            p[2 * i + 1] = trace[2 * panel.nodes[i] + 1];
        }
        const double qr = flux[2 * t], qi = flux[2 * t + 1];
        if (qr == 0 && qi == 0 && p[0] == 0 && p[1] == 0 && p[2] == 0 && p[3] == 0 && p[4] == 0 && p[5] == 0)
            continue;
        int top = 0;
        stack[top++] = SamplePatch{{1, 0, 0, 0, 1, 0, 0, 0, 1}, 1.0, 0};
        while (top > 0) {
            const SamplePatch patch = stack[--top];
            double cr, ci, cm, fr, fi, fm;
            patchIntegral(panel, patch, x, k, p, qr, qi, 0, 6, cr, ci, cm);    // degree 4
            patchIntegral(panel, patch, x, k, p, qr, qi, 18, 16, fr, fi, fm);  // degree 8
            const double span = k * panel.maxEdge * sqrt(patch.fraction);
            const double diff = sqrt((fr - cr) * (fr - cr) + (fi - ci) * (fi - ci));
            if (span <= 3.14159265358979323846 && diff <= tolerance * fmax(fm, 1e-300)) {
                re += fr;
                im += fi;
                continue;
            }
            if (patch.depth >= maxDepth) {
                failed = 1;
                break;
            }
            // children pushed in reverse so that the first is integrated first
            double ab[3], bc[3], ca[3];
            for (int i = 0; i < 3; ++i) {
                ab[i] = (patch.b[i] + patch.b[3 + i]) * .5;
                bc[i] = (patch.b[3 + i] + patch.b[6 + i]) * .5;
                ca[i] = (patch.b[6 + i] + patch.b[i]) * .5;
            }
            const double *corners[4][3] = {{patch.b, ab, ca}, {ab, patch.b + 3, bc}, {ca, bc, patch.b + 6}, {ab, bc, ca}};
            for (int c = 3; c >= 0; --c) {
                SamplePatch child;
                for (int v = 0; v < 3; ++v)
                    for (int i = 0; i < 3; ++i)
                        child.b[3 * v + i] = corners[c][v][i];
                child.fraction = patch.fraction * .25;
                child.depth = patch.depth + 1;
                stack[top++] = child;
            }
        }
    }
    sA[tid] = re;
    sB[tid] = im;
    sFlag[tid] = failed;
    __syncthreads();
    for (int s = kFieldThreads / 2; s > 0; s >>= 1) {
        if (tid < unsigned(s)) {
            sA[tid] += sA[tid + s];
            sB[tid] += sB[tid + s];
            sFlag[tid] |= sFlag[tid + s];
        }
        __syncthreads();
    }
    if (tid == 0) {
        const bool ok = !sFlag[0] && isfinite(sA[0]) && isfinite(sB[0]);
        status[pt] = ok ? kFieldAir : kFieldNotConverged;
        out[2 * pt] = ok ? sA[0] : 0;
        out[2 * pt + 1] = ok ? sB[0] : 0;
    }
}

}  // namespace

// The field rules (degrees 4, 6, 8, 12, 14) in constant memory, once per
// device (each device has its own copy of the __constant__ table).
void uploadFieldRules(cudaStream_t stream) {
    static PerDeviceOnce once;
    once.run([&]() {
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
    });
}

void samplePressureField(const DPanel *panels, uint32_t T, const double *trace, const double *flux,
                         const double *points, uint32_t count, double k, double minDistance, double tolerance,
                         uint32_t maxDepth, double *pressure, int32_t *status, cudaStream_t stream) {
    if (maxDepth > 12)
        throw std::invalid_argument("Invalid pressure field settings.");
    uploadFieldRules(stream);
    if (!count)
        return;
    pressureFieldKernel<<<count, kFieldThreads, 0, stream>>>(panels, T, trace, flux, points, k, minDistance, tolerance,
                                                           maxDepth, pressure, status);
    check(cudaGetLastError(), "pressure field launch");
}

size_t fieldPartialsBytes(uint32_t T, uint32_t E, uint32_t O, uint32_t B) {
    return size_t(B) * E * O * ((T + kTile - 1) / kTile) * 2 * sizeof(double);
}

void evaluateFieldBatch(const FieldRequest &req, const double *ks, const double *pressure, const double *flux,
                        const uint32_t *batchDegree, double *partials, double *out, int *error, cudaStream_t stream,
                        KernelTimer *timer) {
    uploadFieldRules(stream);
    const uint32_t tiles = (req.T + kTile - 1) / kTile;
    const size_t outputs = size_t(req.B) * req.E * req.O;
    if (!outputs)
        return;
    {
        TimedScope s(timer, "field", stream);
        fieldKernel<<<unsigned(outputs * tiles), 128, 0, stream>>>(req, ks, pressure, flux, batchDegree, partials,
                                                                  error);
    }
    {
        TimedScope s(timer, "field_finish", stream);
        finishKernel<<<unsigned((outputs + 127) / 128), 128, 0, stream>>>(partials, tiles, outputs, out, error);
    }
    check(cudaGetLastError(), "field launch");
}

namespace {
// ---------------------------------------------------------------------------
// Allocation-free observer field.
//
// Some callers cannot allocate device memory at the time they need an
// observer field: an interactive sweep that must not stall on the device-wide
// synchronisation cudaMalloc/cudaFree imply, a host application that hands the
// solver only memory from its own pre-sized arena, or a process that has
// already committed all device memory it may use. This entry point serves
// them: the caller passes every input and output as device memory it already
// owns, and the only extra device memory is the fixed scratch array below,
// which is part of the library's device image (loaded with the module, held
// by every GPU that loads the library until the process exits).
//
// The scratch holds, per call: the panel table built from the caller's raw
// mesh, observers in session coordinates, the wavenumber and rule degree, the
// device error word and the per-tile partial sums. Its maximum is 4 MiB:
// T * 200 B + O * 24 B + O * ceil(T / 256) * 16 B + 256 B must fit.
// Every call reuses the same array and leaves its contents behind; the error
// word is cleared at the start of each call and all other entries are fully
// rewritten. Calls that overlap on the GPU (from several host threads or on
// several streams) race on the array and must be serialised by the caller.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;
static __device__ __align__(256) double gNoAllocScratch[kNoAllocScratchBytes / sizeof(double)];
constexpr int kErrDegenerate = 5;
constexpr int kErrIndex = 6;

// Panel table and observers from the caller's raw arrays, in the session's
// coordinates (centred on vertex 0) and with the session's panel arithmetic.
__global__ void noAllocPrepareKernel(const double *vertices, uint32_t N, const uint32_t *triangles, uint32_t T,
                                     const double *observers, uint32_t O, int farField, double k, uint32_t degree,
                                     DPanel *panels, double *localObservers, double *ks, uint32_t *degrees,
                                     int *error) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const double ox = vertices[0], oy = vertices[1], oz = vertices[2];
    if (i < T) {
        V3 v[3];
        for (int c = 0; c < 3; ++c) {
            const uint32_t n = triangles[3 * i + c];
            if (n >= N) {  // invalid vertex index: flag it and leave the panel unread
                atomicExch(error, kErrIndex);
                return;
            }
            v[c] = V3{vertices[3 * n] - ox, vertices[3 * n + 1] - oy, vertices[3 * n + 2] - oz};
        }
        const V3 ab = v[1] - v[0], ac = v[2] - v[0], bc = v[2] - v[1];
        const V3 av = cross(ab, ac);
        const double twice = norm3d(av.x, av.y, av.z);
        const double maxEdge = fmax(fmax(norm3d(ab.x, ab.y, ab.z), norm3d(ac.x, ac.y, ac.z)), norm3d(bc.x, bc.y, bc.z));
        if (!(twice > 128.0 * 2.220446049250313e-16 * maxEdge * maxEdge))
            atomicExch(error, kErrDegenerate);
        DPanel d;
        const double e1[3] = {ab.x, ab.y, ab.z}, e2[3] = {ac.x, ac.y, ac.z}, v0[3] = {v[0].x, v[0].y, v[0].z};
        for (int c = 0; c < 3; ++c) {
            d.v0[c] = v0[c];
            d.e1[c] = e1[c];
            d.e2[c] = e2[c];
            d.nodes[c] = triangles[3 * i + c];
        }
        d.n[0] = av.x / twice;
        d.n[1] = av.y / twice;
        d.n[2] = av.z / twice;
        for (int c = 0; c < 9; ++c)
            d.curl[c] = 0;  // the field does not use the surface curls
        d.area = 0.5 * twice;
        d.maxEdge = maxEdge;
        d.pad = 0;
        panels[i] = d;
    }
    if (i < O && !farField) {
        localObservers[3 * i] = observers[3 * i] - ox;
        localObservers[3 * i + 1] = observers[3 * i + 1] - oy;
        localObservers[3 * i + 2] = observers[3 * i + 2] - oz;
    }
    if (i == 0) {
        ks[0] = k;
        degrees[0] = degree;
    }
}

// Far-field directions (x - origin)/|x - origin|, origin given in world coordinates.
__global__ void noAllocDirectionsKernel(const double *observers, uint32_t O, double fx, double fy, double fz,
                                        double *directions, int *error) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= O)
        return;
    const double x = observers[3 * i] - fx, y = observers[3 * i + 1] - fy, z = observers[3 * i + 2] - fz;
    const double d = norm3d(x, y, z);
    if (!(d > 0) || !isfinite(d)) {
        atomicExch(error, kErrDistance);
        return;
    }
    directions[3 * i] = x / d;
    directions[3 * i + 1] = y / d;
    directions[3 * i + 2] = z / d;
}

std::mutex gNoAllocMutex;
void *gNoAllocAddress[256] = {};

}  // namespace

// Set-up once per device, with that device current: the host name of the
// array is only a stand-in, so its device address is looked up here and
// passed to the kernels. The first call on a device does this look-up and
// should therefore come before any stream capture on that device. The address
// is kept for the life of the process, which assumes the device's primary
// context lives that long too (no cudaDeviceReset between calls).
static double *noAllocScratch(int device) {
    std::lock_guard<std::mutex> lock(gNoAllocMutex);
    if (device < 0 || device >= 256)
        throw std::runtime_error("CUDA device ordinal out of range for the no-allocation scratch.");
    if (!gNoAllocAddress[device]) {
        void *address = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&address, gNoAllocScratch);
        if (e != cudaSuccess || !address)
            throw std::runtime_error(std::string("no-allocation scratch address: ") + cudaGetErrorString(e));
        gNoAllocAddress[device] = address;
    }
    return static_cast<double *>(gNoAllocAddress[device]);
}

size_t noAllocScratchBytes() { return kNoAllocScratchBytes; }

// Observer pressure of one solved frequency without device allocation; see
// hs_bem_observer_field_noalloc in include/hs_bem.h. Throws on invalid sizes
// before any device work, and on device error codes after the field.
void observerFieldNoAlloc(const double *vertices, size_t vertexCount, const uint32_t *triangles, size_t triangleCount,
                          const double *pressure, const double *flux, const double *observers, size_t observerCount,
                          double k, uint32_t degree, int farField, const double *farOrigin, double farDistance,
                          double tolerance, uint32_t maximumDepth, cudaStream_t stream, double *out) {
    if (!vertices || !triangles || !pressure || !flux || !out || !vertexCount || !triangleCount)
        throw std::invalid_argument("No-allocation field: device inputs and output must be non-null and nonempty.");
    if (observerCount && !observers)
        throw std::invalid_argument("No-allocation field: observers are null.");
    if (degree != 4 && degree != 6 && degree != 8 && degree != 12 && degree != 14)
        throw std::invalid_argument("No-allocation field: rule degree must be 4, 6, 8, 12 or 14.");
    if (!std::isfinite(k) || k <= 0 || !std::isfinite(tolerance) || tolerance <= 0 || maximumDepth > 10 ||
        (farField && (!farOrigin || !std::isfinite(farDistance) || farDistance <= 0)))
        throw std::invalid_argument("No-allocation field: wavenumber, tolerance, depth or far-field settings invalid.");
    if (vertexCount > 0xffffffffu || triangleCount > 0xffffffffu || observerCount > 0xffffffffu)
        throw std::invalid_argument("No-allocation field: sizes exceed 32-bit indexing.");
    if (!observerCount)
        return;
    const uint32_t T = uint32_t(triangleCount), O = uint32_t(observerCount), N = uint32_t(vertexCount);
    const size_t tiles = (T + kTile - 1) / kTile;
    // Scratch layout (doubles): panels | observers | k, degree | error | partials
    const size_t panelDoubles = size_t(T) * (sizeof(DPanel) / sizeof(double));
    const size_t obsOffset = panelDoubles, parOffset = obsOffset + 3 * size_t(O) + 4;
    const size_t needed = (parOffset + 2 * size_t(O) * tiles) * sizeof(double);
    if (needed > kNoAllocScratchBytes)
        throw std::invalid_argument("No-allocation field needs " + std::to_string(needed) + " bytes of scratch for " +
                                    std::to_string(T) + " triangles and " + std::to_string(O) +
                                    " observers; its fixed maximum is " + std::to_string(kNoAllocScratchBytes) +
                                    " bytes (4 MiB).");
    int device = 0;
    check(cudaGetDevice(&device), "no-allocation field device");
    double *scratch = noAllocScratch(device);
    DPanel *panels = reinterpret_cast<DPanel *>(scratch);
    double *localObservers = scratch + obsOffset;
    double *ks = scratch + obsOffset + 3 * size_t(O);
    uint32_t *degrees = reinterpret_cast<uint32_t *>(ks + 1);
    int *error = reinterpret_cast<int *>(ks + 2);
    double *partials = scratch + parOffset;
    check(cudaMemsetAsync(error, 0, sizeof(int), stream), "no-allocation field error reset");
    double origin[3];
    check(cudaMemcpyAsync(origin, vertices, sizeof(origin), cudaMemcpyDeviceToHost, stream), "mesh origin");
    check(cudaStreamSynchronize(stream), "mesh origin");
    const uint32_t threads = std::max(T, O);
    noAllocPrepareKernel<<<(threads + 127) / 128, 128, 0, stream>>>(vertices, N, triangles, T, observers, O, farField,
                                                                   k, degree, panels, localObservers, ks, degrees,
                                                                   error);
    if (farField)
        noAllocDirectionsKernel<<<(O + 127) / 128, 128, 0, stream>>>(observers, O, farOrigin[0], farOrigin[1],
                                                                     farOrigin[2], localObservers, error);
    check(cudaGetLastError(), "no-allocation field preparation");
    // The field kernel indexes the trace through the panel table: stop here on
    // invalid indices or degenerate panels.
    int prepared = 0;
    check(cudaMemcpyAsync(&prepared, error, sizeof(int), cudaMemcpyDeviceToHost, stream), "no-allocation field status");
    check(cudaStreamSynchronize(stream), "no-allocation field preparation");
    if (prepared == kErrIndex)
        throw std::invalid_argument("No-allocation field: a triangle has an invalid vertex index.");
    if (prepared == kErrDegenerate)  // the same input class and message as a session's mesh check
        throw std::invalid_argument("Galerkin triangle is degenerate or numerically unresolved.");
    if (prepared == kErrDistance)
        throw std::invalid_argument("A far-field direction must differ from its origin.");
    FieldRequest req{panels, T, N, 1, O, 1, localObservers, farField,
                     {farField ? farOrigin[0] - origin[0] : 0.0, farField ? farOrigin[1] - origin[1] : 0.0,
                      farField ? farOrigin[2] - origin[2] : 0.0},
                     farField ? farDistance : 1.0, tolerance, maximumDepth};
    evaluateFieldBatch(req, ks, pressure, flux, degrees, partials, out, error, stream, nullptr);
    int code = 0;
    check(cudaMemcpyAsync(&code, error, sizeof(int), cudaMemcpyDeviceToHost, stream), "no-allocation field status");
    check(cudaStreamSynchronize(stream), "no-allocation field");
    if (code == kErrDegenerate)
        throw NumericError("Galerkin triangle is degenerate or numerically unresolved.");
    if (code == kErrDistance)
        throw NumericError("BEM quadrature encountered zero or invalid source distance.");
    if (code == kErrFieldDepth)
        throw NumericError("BEM field integration did not reach its near-field tolerance.");
    if (code)
        throw NumericError("BEM calculation produced a non-finite value.");
}

}  // namespace hsb
