// Test infrastructure only — the FP64 CPU oracle for HornSculpt's dense
// exterior Burton-Miller solve. It restates the reference method entirely in
// FP64: the same P1/DP0 spaces, interaction plan, pair rules, row
// equilibration, LU solve with refinement and observer-field degree loop
// (modules/bem/cuda/cuda_solver.cu:1021-1853 with the FP64 sample of
// panel_integrals.cuh:166-198). Only tests/, the smoke check and bench.py's
// CPU-baseline leg load it; the product never does.
//
// Differences from the product's CUDA path are deliberate and independent:
// singular pairs use the direct Sauter-Schwab points with the radial
// variable inside the transform (pair_quadrature.cpp:809-824) rather than the
// factored radial loop; scatter is a serial sum; LU is a textbook
// partial-pivot elimination.
#include "plan.hpp"

#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <mutex>

namespace oracle {
namespace {

constexpr double kFourPi = 12.56637061435917295385;

struct Moments13 {
    cplx m[9]{}, rhs[3]{}, green{};
};

// panel_integrals.cuh:166-198: G, the double-layer and adjoint kernels, and
// the k^2 (n.n) part of the Maue hypersingular term, alpha = -i/k.
inline void pairSample(Moments13 &acc, const Panel &t, const Panel &s, const PairPoint &p, V3 d, double k,
                       bool coincident) {
    const double r = std::sqrt(norm2(d));
    if (!(r > 0) || !std::isfinite(r))
        throw std::runtime_error("BEM quadrature encountered zero or invalid source distance.");
    const double scale = p.w * (4.0 * t.area * s.area) / (kFourPi * r);
    const cplx g(std::cos(k * r) * scale, -std::sin(k * r) * scale);
    acc.green += g;
    const cplx radial(g.real() - g.imag() * k * r, g.imag() + g.real() * k * r);
    const double inv2 = 1.0 / (r * r);
    const cplx dl = radial * (coincident ? 0.0 : dot(d, s.normal) * inv2);
    const cplx adj = radial * (coincident ? 0.0 : -dot(d, t.normal) * inv2);
    const double nn = dot(t.normal, s.normal);
    const cplx a(-dl.real() - k * nn * g.imag(), -dl.imag() + k * nn * g.real());
    const cplx b(-g.real() - adj.imag() / k, -g.imag() + adj.real() / k);
    for (int i = 0; i < 3; ++i) {
        acc.rhs[i] += b * p.t[i];
        for (int j = 0; j < 3; ++j)
            acc.m[3 * i + j] += a * (p.t[i] * p.s[j]);
    }
}

struct Numerics {
    unsigned quadratureOrder{4}, singularOrder{4};
    double nearRatio{1.0}, nearTol{1e-4};
    unsigned nearDepth{6};
    double residualTol{5e-5};
    unsigned maxRefine{3};
};

struct Problem {
    Space space;
    std::vector<uint32_t> faces;
};

// The 12 complex P1xP1 / P1xDP0 entries of one ordered panel pair.
struct Block {
    cplx m[9]{}, rhs[3]{};
};

Block finishBlock(const Moments13 &mo, const Panel &t, const Panel &s, double k, bool coincident) {
    Block b;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            const double curl = dot(t.curl[i], s.curl[j]);
            b.m[3 * i + j] = mo.m[3 * i + j] + cplx(mo.green.imag() * curl / k, -mo.green.real() * curl / k);
        }
        b.rhs[i] = mo.rhs[i];
        if (coincident)
            b.rhs[i] += cplx(0, t.area / (6 * k));
    }
    return b;
}

struct Rules {
    std::vector<TriPoint> regular[3];  // degree 4, 6, 8
    std::vector<TriPoint> near8, near14;
    std::vector<GaussPoint> gauss;
    std::vector<GaussPoint> inner20;
};

Moments13 singularMoments(const Panel &t, const Panel &s, const Permutation &perm, const Rules &R, double k) {
    Moments13 mo;
    const bool coincident = perm.topology == Coincident;
    for (unsigned sec = 0; sec < sectorCount(perm.topology); ++sec)
        for (const auto &r : R.gauss)
            for (const auto &u : R.gauss)
                for (const auto &v : R.gauss)
                    for (const auto &w : R.gauss) {
                        PairPoint p = sauterSchwab(perm.topology, sec, r.x, u.x, v.x, w.x);
                        p.w *= r.w * u.w * v.w * w.w;
                        p = permute(p, perm);
                        pairSample(mo, t, s, p, pairDelta(t, p.t, s, p.s), k, coincident);
                    }
    return mo;
}

Moments13 tensorPairMoments(const Panel &t, const Panel &s, const std::vector<TriPoint> &rule, double k) {
    Moments13 mo;
    for (const auto &x : rule)
        for (const auto &y : rule) {
            PairPoint p;
            for (int i = 0; i < 3; ++i) {
                p.t[i] = x.b[i];
                p.s[i] = y.b[i];
            }
            p.w = x.w * y.w;
            pairSample(mo, t, s, p, pairDelta(t, p.t, s, p.s), k, false);
        }
    return mo;
}

// cuda_solver.cu:430-518 and near_projection.hpp:228-254: one directed near
// job integrates its plan patches with the degree 8/14 outer rules and the
// 20-point inner projection rule; reverse jobs reuse the patches with test
// and trial barycentrics exchanged.
Moments13 nearMoments(const Panel &t, const Panel &s, const NearJob &job, const Plan &plan, const Rules &R, double k) {
    Moments13 mo;
    const Panel &pa = job.swap ? s : t, &pb = job.swap ? t : s;
    for (uint32_t q = 0; q < job.count; ++q) {
        const Patch &patch = plan.patches[job.first + q];
        const auto &rule = patch.degree == 14 ? R.near14 : R.near8;
        if (!patch.projection) {
            for (const auto &x : rule)
                for (const auto &y : rule) {
                    PairPoint p;
                    p.w = x.w * y.w * patch.areaFraction;
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            p.t[i] += x.b[j] * patch.test[3 * j + i];
                            p.s[i] += y.b[j] * patch.trial[3 * j + i];
                        }
                    if (job.swap)
                        for (int i = 0; i < 3; ++i)
                            std::swap(p.t[i], p.s[i]);
                    pairSample(mo, t, s, p, pairDelta(t, p.t, s, p.s), k, false);
                }
            continue;
        }
        const unsigned iv = patch.intervals;
        std::vector<GaussPoint> g;
        for (unsigned a = 0; a < iv; ++a)
            for (const auto &gp : R.inner20)
                g.push_back({(a + gp.x) / iv, gp.w / iv});
        for (const auto &x : rule) {
            const ProjOuter po = projOuter(x, patch, pa, pb);
            for (unsigned e = 0; e < 3; ++e) {
                const ProjEdge pe = projEdge(po, e, pb);
                for (const auto &u : g) {
                    const ProjRay ray = projRay(po, pe, u);
                    for (const auto &v : g) {
                        PairPoint p = projPoint(po, ray, v);
                        if (job.swap)
                            for (int i = 0; i < 3; ++i)
                                std::swap(p.t[i], p.s[i]);
                        pairSample(mo, t, s, p, pairDelta(t, p.t, s, p.s), k, false);
                    }
                }
            }
        }
    }
    return mo;
}

struct System {
    size_t N{}, T{};
    std::vector<cplx> A;    // row-major N x N, rows scaled by 1/lumped mass
    std::vector<cplx> rhs;  // N x E
};

// Dense assembly of A p = B q (cuda_solver.cu:1408-1471), every pair in FP64.
// q holds E excitation columns of per-panel flux (panel-major within a column).
System assemble(const Problem &P, const Plan &plan, const Rules &R, const Numerics &num, double k,
                const std::vector<cplx> &q, size_t E) {
    const Space &sp = P.space;
    const size_t N = sp.vertices.size(), T = sp.panels.size();
    System S;
    S.N = N;
    S.T = T;
    S.A.assign(N * N, 0);
    S.rhs.assign(N * E, 0);
    std::vector<Bounds> bounds(T);
    for (size_t i = 0; i < T; ++i)
        bounds[i] = makeBounds(sp.panels[i]);
    std::vector<uint8_t> kind(T * T, 0);  // 1 touching, 2 near
    std::vector<const TouchJob *> touchOf(T * T, nullptr);
    std::vector<const NearJob *> nearOf(T * T, nullptr);
    for (const auto &j : plan.touching) {
        kind[size_t(j.test) * T + j.trial] = 1;
        touchOf[size_t(j.test) * T + j.trial] = &j;
    }
    for (const auto &j : plan.near) {
        kind[size_t(j.test) * T + j.trial] = 2;
        nearOf[size_t(j.test) * T + j.trial] = &j;
    }
    const unsigned workers = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    const size_t chunk = 16;
    std::vector<Block> blocks(chunk * T);
    std::vector<std::string> errors(workers);
    for (size_t t0 = 0; t0 < T; t0 += chunk) {
        const size_t t1 = std::min(T, t0 + chunk);
        std::vector<std::thread> pool;
        for (unsigned w = 0; w < workers; ++w)
            pool.emplace_back([&, w]() {
                try {
                    for (size_t idx = w; idx < (t1 - t0) * T; idx += workers) {
                        const size_t t = t0 + idx / T, s = idx % T;
                        const Panel &a = sp.panels[t], &b = sp.panels[s];
                        const uint8_t kd = kind[t * T + s];
                        Moments13 mo;
                        bool coincident = false;
                        if (kd == 1) {
                            const auto &perm = touchOf[t * T + s]->perm;
                            coincident = perm.topology == Coincident;
                            mo = singularMoments(a, b, perm, R, k);
                        } else if (kd == 2) {
                            mo = nearMoments(a, b, *nearOf[t * T + s], plan, R, k);
                        } else {
                            const uint8_t whole = plan.wholePanelDegrees.empty()
                                                      ? 0
                                                      : plan.wholePanelDegrees[unorderedIndex(uint32_t(t), uint32_t(s))];
                            if (whole)
                                mo = tensorPairMoments(a, b, whole == 14 ? R.near14 : R.near8, k);
                            else {
                                const unsigned d = qualifiedDegree(bounds[t], bounds[s], k, num.nearTol, num.quadratureOrder);
                                if (!d)
                                    throw std::runtime_error("BEM dense regular pair escaped its qualified adaptive plan.");
                                mo = tensorPairMoments(a, b, R.regular[d == 4 ? 0 : d == 6 ? 1 : 2], k);
                            }
                        }
                        blocks[idx] = finishBlock(mo, a, b, k, coincident);
                    }
                } catch (const std::exception &e) {
                    errors[w] = e.what();
                }
            });
        for (auto &th : pool)
            th.join();
        for (const auto &e : errors)
            if (!e.empty())
                throw std::runtime_error(e);
        for (size_t t = t0; t < t1; ++t)
            for (size_t s = 0; s < T; ++s) {
                const Block &b = blocks[(t - t0) * T + s];
                const Panel &pt = sp.panels[t], &ps = sp.panels[s];
                for (int i = 0; i < 3; ++i) {
                    const uint32_t row = pt.nodes[i];
                    for (int j = 0; j < 3; ++j)
                        S.A[size_t(row) * N + ps.nodes[j]] += b.m[3 * i + j];
                    for (size_t e = 0; e < E; ++e)
                        S.rhs[size_t(row) * E + e] += b.rhs[i] * q[e * T + s];
                }
            }
    }
    // cuda_solver.cu:519-540: half the P1 mass (the flux half-mass term rides
    // on the coincident block above).
    for (const auto &p : sp.panels)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                S.A[size_t(p.nodes[i]) * N + p.nodes[j]] += p.area * (i == j ? 2.0 : 1.0) / 24.0;
    for (size_t row = 0; row < N; ++row) {
        const double scale = 1.0 / sp.lumpedMass[row];
        for (size_t c = 0; c < N; ++c)
            S.A[row * N + c] *= scale;
        for (size_t e = 0; e < E; ++e)
            S.rhs[row * E + e] *= scale;
    }
    return S;
}

// Optional LAPACK (zgetrf / zgetrs, Fortran calling convention) supplied by
// the caller as function pointers, for the timed CPU baseline: the reference
// factors with a library LU (cusolverDnCgetrf), so the baseline does too. The
// row-major matrix is LAPACK's column-major transpose; A x = b is solved as
// (A^T)^T x = b with trans = 'T'.
using ZgetrfFn = void (*)(int *, int *, cplx *, int *, int *, int *);
using ZgetrsFn = void (*)(char *, int *, int *, cplx *, int *, int *, cplx *, int *, int *);
ZgetrfFn gZgetrf = nullptr;
ZgetrsFn gZgetrs = nullptr;

// Partial-pivot LU in place (row-major), then forward/back substitution.
void luFactor(std::vector<cplx> &A, size_t N, std::vector<size_t> &piv) {
    if (gZgetrf) {
        int n = int(N), info = 0;
        std::vector<int> ipiv(N);
        gZgetrf(&n, &n, A.data(), &n, ipiv.data(), &info);
        if (info != 0)
            throw std::runtime_error("singular Burton-Miller matrix");
        piv.resize(N);
        for (size_t i = 0; i < N; ++i)
            piv[i] = size_t(ipiv[i]);  // 1-based LAPACK pivots mark the LAPACK factors
        return;
    }
    piv.resize(N);
    for (size_t c = 0; c < N; ++c) {
        size_t best = c;
        double bv = std::abs(A[c * N + c]);
        for (size_t r = c + 1; r < N; ++r)
            if (std::abs(A[r * N + c]) > bv) {
                bv = std::abs(A[r * N + c]);
                best = r;
            }
        if (!(bv > 0))
            throw std::runtime_error("singular Burton-Miller matrix");
        piv[c] = best;
        if (best != c)
            for (size_t j = 0; j < N; ++j)
                std::swap(A[c * N + j], A[best * N + j]);
        const cplx inv = 1.0 / A[c * N + c];
        for (size_t r = c + 1; r < N; ++r) {
            const cplx f = A[r * N + c] * inv;
            A[r * N + c] = f;
            if (f != cplx(0))
                for (size_t j = c + 1; j < N; ++j)
                    A[r * N + j] -= f * A[c * N + j];
        }
    }
}
void luSolve(const std::vector<cplx> &LU, size_t N, const std::vector<size_t> &piv, std::vector<cplx> &x) {
    if (gZgetrs) {
        char trans = 'T';
        int n = int(N), one = 1, info = 0;
        std::vector<int> ipiv(piv.begin(), piv.end());
        gZgetrs(&trans, &n, &one, const_cast<cplx *>(LU.data()), &n, ipiv.data(), x.data(), &n, &info);
        if (info != 0)
            throw std::runtime_error("LAPACK zgetrs failed");
        return;
    }
    for (size_t c = 0; c < N; ++c)
        if (piv[c] != c)
            std::swap(x[c], x[piv[c]]);
    for (size_t r = 0; r < N; ++r)
        for (size_t j = 0; j < r; ++j)
            x[r] -= LU[r * N + j] * x[j];
    for (size_t r = N; r-- > 0;) {
        for (size_t j = r + 1; j < N; ++j)
            x[r] -= LU[r * N + j] * x[j];
        x[r] /= LU[r * N + r];
    }
}

// ---- observer fields (panel_integrals.cuh:298-443) ----
struct FieldPatch {
    V3 b[3];
    double fraction;
    unsigned depth;
};
FieldPatch childPatch(const FieldPatch &p, unsigned c) {
    const V3 ab = (p.b[0] + p.b[1]) * .5, ac = (p.b[0] + p.b[2]) * .5, bc = (p.b[1] + p.b[2]) * .5;
    FieldPatch r;
    r.fraction = p.fraction * .25;
    r.depth = p.depth + 1;
    if (c == 0) { r.b[0] = p.b[0]; r.b[1] = ab; r.b[2] = ac; }
    else if (c == 1) { r.b[0] = ab; r.b[1] = p.b[1]; r.b[2] = bc; }
    else if (c == 2) { r.b[0] = ac; r.b[1] = bc; r.b[2] = p.b[2]; }
    else { r.b[0] = ab; r.b[1] = bc; r.b[2] = ac; }
    return r;
}
struct FieldValue {
    cplx value;
    double scale{};
};
FieldValue fieldPatch(V3 obs, const Panel &pn, const FieldPatch &fp, const std::vector<TriPoint> &rule,
                      const cplx *p, cplx flux, double k) {
    FieldValue out;
    for (const auto &q : rule) {
        const V3 l = fp.b[0] * q.b[0] + fp.b[1] * q.b[1] + fp.b[2] * q.b[2];
        const double bary[3] = {l.x, l.y, l.z};
        const V3 d = (obs - pn.v[0]) - localPoint(pn, bary);
        const double r = std::sqrt(norm2(d));
        if (!(r > 0))
            throw std::runtime_error("BEM quadrature encountered zero or invalid source distance.");
        const double scale = 2.0 * pn.area * fp.fraction * q.w / (kFourPi * r);
        const cplx g(std::cos(k * r) * scale, -std::sin(k * r) * scale);
        const double nf = dot(d, pn.normal) / (r * r);
        const cplx dual((g.real() - g.imag() * k * r) * nf, (g.imag() + g.real() * k * r) * nf);
        cplx pp = 0;
        for (int i = 0; i < 3; ++i)
            pp += p[pn.nodes[i]] * bary[i];
        const cplx dp = dual * pp, sq = g * flux;
        out.value += dp - sq;
        out.scale += std::abs(dp) + std::abs(sq);
    }
    return out;
}
cplx nearField(V3 obs, const Panel &pn, const std::vector<TriPoint> &rule, const cplx *p, cplx flux, double k,
               double tol, unsigned maxDepth) {
    std::vector<FieldPatch> stack{{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, 1.0, 0}};
    cplx result = 0;
    while (!stack.empty()) {
        const FieldPatch fp = stack.back();
        stack.pop_back();
        const FieldValue coarse = fieldPatch(obs, pn, fp, rule, p, flux, k);
        FieldValue fine;
        for (unsigned c = 0; c < 4; ++c) {
            const FieldValue v = fieldPatch(obs, pn, childPatch(fp, c), rule, p, flux, k);
            fine.value += v.value;
            fine.scale += v.scale;
        }
        if (std::abs(fine.value - coarse.value) <= tol * std::max(fine.scale, 1e-300))
            result += fine.value;
        else {
            if (fp.depth >= maxDepth || stack.size() + 4 > 34)
                throw std::runtime_error("BEM field integration did not reach its near-field tolerance.");
            for (unsigned c = 0; c < 4; ++c)
                stack.push_back(childPatch(fp, c));
        }
    }
    return result;
}
cplx asymptoticField(V3 dir, V3 origin, const Panel &pn, const std::vector<TriPoint> &rule, const cplx *p, cplx flux,
              double k) {
    cplx out = 0;
    const V3 od = pn.v[0] - origin;
    const double nf = k * dot(dir, pn.normal);
    for (const auto &q : rule) {
        const V3 pos = od + localPoint(pn, q.b);
        const double phase = k * dot(dir, pos);
        const double scale = 2 * pn.area * q.w / kFourPi;
        cplx pp = 0;
        for (int i = 0; i < 3; ++i)
            pp += p[pn.nodes[i]] * q.b[i];
        const cplx integrand(-nf * pp.imag() - flux.real(), nf * pp.real() - flux.imag());
        out += cplx(std::cos(phase) * scale, std::sin(phase) * scale) * integrand;
    }
    return out;
}

// cuda_solver.cu:679-704 — solid-angle inside test for finite observers.
bool insideSolid(const std::vector<Panel> &panels, V3 x) {
    double angle = 0;
    for (const auto &pn : panels) {
        const V3 e0 = pn.v[1] - pn.v[0], e1 = pn.v[2] - pn.v[0], rel = x - pn.v[0];
        const double cs = std::max(std::sqrt(norm2(x)), std::sqrt(norm2(pn.v[0])));
        const double tol = std::max(pn.maxEdge * 1e-10, cs * 32 * std::numeric_limits<double>::epsilon());
        if (std::abs(dot(rel, pn.normal)) <= tol) {
            const double aa = dot(e0, e0), ab = dot(e0, e1), bb = dot(e1, e1), pa = dot(rel, e0), pb = dot(rel, e1);
            const double det = aa * bb - ab * ab, u = (bb * pa - ab * pb) / det, v = (aa * pb - ab * pa) / det;
            if (u >= -1e-10 && v >= -1e-10 && u + v <= 1 + 1e-10)
                return true;
        }
        const V3 a = pn.v[0] - x, b = pn.v[1] - x, c = pn.v[2] - x;
        const double la = std::sqrt(norm2(a)), lb = std::sqrt(norm2(b)), lc = std::sqrt(norm2(c));
        const double den = la * lb * lc + dot(a, b) * lc + dot(b, c) * la + dot(c, a) * lb;
        angle += 2 * std::atan2(dot(a, cross(b, c)), den);
    }
    return std::abs(angle) > 2 * M_PI;
}

Rules makeRules(const Numerics &num) {
    Rules R;
    R.regular[0] = triangleRule(4);
    R.regular[1] = triangleRule(6);
    R.regular[2] = triangleRule(8);
    R.near8 = triangleRule(8);
    R.near14 = triangleRule(14);
    R.gauss = gauss01(num.singularOrder);
    R.inner20 = gauss01(20);
    return R;
}

thread_local std::string lastError;
int fail(const std::exception &e) {
    lastError = e.what();
    return dynamic_cast<const std::invalid_argument *>(&e) ? 1 : 2;
}

Problem makeProblem(const double *verts, size_t nv, const uint32_t *tris, const uint32_t *faces, const uint8_t *driven,
                    size_t nt, V3 *originOut) {
    if (!nv || !nt)
        throw std::invalid_argument("BEM mesh has no vertices.");
    std::vector<V3> v(nv);
    const V3 origin{verts[0], verts[1], verts[2]};
    for (size_t i = 0; i < nv; ++i)
        v[i] = V3{verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]} - origin;
    std::vector<std::array<uint32_t, 3>> t(nt);
    std::vector<uint32_t> f(faces, faces + nt);
    std::vector<uint8_t> d(driven, driven + nt);
    for (size_t i = 0; i < nt; ++i)
        t[i] = {tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]};
    if (originOut)
        *originOut = origin;
    return {buildSpace(v, t, f, d), f};
}

struct PlanHandle {
    Plan plan;
};

}  // namespace
}  // namespace oracle

using namespace oracle;

extern "C" {

struct oracle_numerics {
    unsigned quadrature_order, singular_order;
    double near_ratio, near_tol;
    unsigned near_depth;
    double residual_tol;
    unsigned max_refine;
};

const char *oracle_last_error() { return lastError.c_str(); }

// LAPACK zgetrf / zgetrs for oracle_solve's factorisation (both null: the
// built-in textbook LU).
void oracle_set_lapack(void *zgetrf, void *zgetrs) {
    gZgetrf = reinterpret_cast<ZgetrfFn>(zgetrf);
    gZgetrs = reinterpret_cast<ZgetrsFn>(zgetrs);
}

// Builds the interaction plan for a mesh at planning wavenumber maxK.
int oracle_plan_build(const double *verts, size_t nv, const uint32_t *tris, size_t nt, const oracle_numerics *nm,
                      double maxK, void **out) {
    try {
        std::vector<uint32_t> faces(nt, 0);
        std::vector<uint8_t> drv(nt, 0);
        const Problem P = makeProblem(verts, nv, tris, faces.data(), drv.data(), nt, nullptr);
        PlanSettings st{nm->quadrature_order, nm->singular_order, nm->near_ratio, nm->near_tol, nm->near_depth};
        auto *h = new PlanHandle{makePlan(P.space, st, maxK)};
        *out = h;
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}
void oracle_plan_sizes(void *h, size_t *out) {
    const Plan &p = static_cast<PlanHandle *>(h)->plan;
    out[0] = p.touching.size();
    out[1] = p.near.size();
    out[2] = p.patches.size();
    out[3] = p.wholePanelDegrees.size();
    out[4] = p.nearTrials.size();
    out[5] = p.maxDepth;
}
// touching: 9 u32 per job: test, trial, topology, perm.test[3], perm.trial[3]
void oracle_plan_touching(void *h, uint32_t *out) {
    for (const auto &j : static_cast<PlanHandle *>(h)->plan.touching) {
        *out++ = j.test;
        *out++ = j.trial;
        *out++ = j.perm.topology;
        for (int i = 0; i < 3; ++i)
            *out++ = j.perm.test[i];
        for (int i = 0; i < 3; ++i)
            *out++ = j.perm.trial[i];
    }
}
// near: 5 u32 per job: test, trial, first patch, patch count, swap
void oracle_plan_near(void *h, uint32_t *out) {
    for (const auto &j : static_cast<PlanHandle *>(h)->plan.near) {
        *out++ = j.test;
        *out++ = j.trial;
        *out++ = j.first;
        *out++ = j.count;
        *out++ = j.swap;
    }
}
// patches: 22 doubles each: test[9], trial[9], fraction, degree, projection, intervals
void oracle_plan_patches(void *h, double *out) {
    for (const auto &p : static_cast<PlanHandle *>(h)->plan.patches) {
        for (int i = 0; i < 9; ++i)
            *out++ = p.test[i];
        for (int i = 0; i < 9; ++i)
            *out++ = p.trial[i];
        *out++ = p.areaFraction;
        *out++ = p.degree;
        *out++ = p.projection;
        *out++ = p.intervals;
    }
}
void oracle_plan_whole(void *h, uint8_t *out) {
    const auto &w = static_cast<PlanHandle *>(h)->plan.wholePanelDegrees;
    if (!w.empty())
        std::memcpy(out, w.data(), w.size());
}
void oracle_plan_offsets(void *h, uint32_t *offsets, uint32_t *trials) {
    const Plan &p = static_cast<PlanHandle *>(h)->plan;
    std::memcpy(offsets, p.nearOffsets.data(), p.nearOffsets.size() * 4);
    if (!p.nearTrials.empty())
        std::memcpy(trials, p.nearTrials.data(), p.nearTrials.size() * 4);
}
void oracle_plan_free(void *h) { delete static_cast<PlanHandle *>(h); }

// Patch estimate of one pair (36 complex moments + errors) for unit tests.
int oracle_estimate_patch(const double *tri9a, const double *tri9b, const uint32_t *nodesA, const uint32_t *nodesB,
                          const double *patch22, double k, double *moments72, double *errors3) {
    try {
        std::vector<V3> v;
        for (int i = 0; i < 3; ++i)
            v.push_back({tri9a[3 * i], tri9a[3 * i + 1], tri9a[3 * i + 2]});
        for (int i = 0; i < 3; ++i)
            v.push_back({tri9b[3 * i], tri9b[3 * i + 1], tri9b[3 * i + 2]});
        std::vector<std::array<uint32_t, 3>> t = {{0, 1, 2}, {3, 4, 5}};
        const Space sp = buildSpace(v, t, {0, 0}, {0, 0});
        Panel a = sp.panels[0], b = sp.panels[1];
        for (int i = 0; i < 3; ++i) {
            a.nodes[i] = nodesA[i];
            b.nodes[i] = nodesB[i];
        }
        Patch p;
        for (int i = 0; i < 9; ++i) {
            p.test[i] = patch22[i];
            p.trial[i] = patch22[9 + i];
        }
        p.areaFraction = patch22[18];
        p.degree = unsigned(patch22[19]);
        p.projection = unsigned(patch22[20]);
        p.intervals = unsigned(patch22[21]);
        const Estimate e = estimatePatch(a, b, p, k);
        for (int i = 0; i < 36; ++i) {
            moments72[2 * i] = e.integral[i].real();
            moments72[2 * i + 1] = e.integral[i].imag();
        }
        errors3[0] = e.error;
        errors3[1] = e.inner;
        errors3[2] = e.outer;
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Integral of 1/|x-y| over a pair of triangles by the singular/regular rules:
// used to check the Sauter-Schwab sectors against closed forms.
int oracle_laplace_pair(const double *tri9a, const uint32_t *nodesA, const double *tri9b, const uint32_t *nodesB,
                        unsigned order, double *value) {
    try {
        Panel a, b;
        for (int i = 0; i < 3; ++i) {
            a.v[i] = {tri9a[3 * i], tri9a[3 * i + 1], tri9a[3 * i + 2]};
            b.v[i] = {tri9b[3 * i], tri9b[3 * i + 1], tri9b[3 * i + 2]};
            a.nodes[i] = nodesA[i];
            b.nodes[i] = nodesB[i];
        }
        auto area = [](const Panel &p) {
            const V3 c = cross(p.v[1] - p.v[0], p.v[2] - p.v[0]);
            return 0.5 * std::sqrt(norm2(c));
        };
        const Permutation perm = classify(a.nodes, b.nodes);
        const auto g = gauss01(order);
        double sum = 0;
        for (unsigned sec = 0; sec < sectorCount(perm.topology); ++sec)
            for (const auto &r : g)
                for (const auto &u : g)
                    for (const auto &v : g)
                        for (const auto &w : g) {
                            PairPoint p = sauterSchwab(perm.topology, sec, r.x, u.x, v.x, w.x);
                            p.w *= r.w * u.w * v.w * w.w;
                            p = permute(p, perm);
                            sum += p.w / std::sqrt(norm2(pairDelta(a, p.t, b, p.s)));
                        }
        *value = sum * 4 * area(a) * area(b);
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Assembled, row-equilibrated system at wavenumber k for one excitation
// (per-panel flux q), the plan built at planK. A is row-major complex.
int oracle_assemble(const double *verts, size_t nv, const uint32_t *tris, size_t nt, const oracle_numerics *nm,
                    double planK, double k, const double *q, double *A, double *rhs) {
    try {
        std::vector<uint32_t> faces(nt, 0);
        std::vector<uint8_t> drv(nt, 0);
        const Problem P = makeProblem(verts, nv, tris, faces.data(), drv.data(), nt, nullptr);
        Numerics num{nm->quadrature_order, nm->singular_order, nm->near_ratio, nm->near_tol, nm->near_depth,
                     nm->residual_tol, nm->max_refine};
        PlanSettings st{num.quadratureOrder, num.singularOrder, num.nearRatio, num.nearTol, num.nearDepth};
        const Plan plan = makePlan(P.space, st, planK);
        const Rules R = makeRules(num);
        std::vector<cplx> qv(nt);
        for (size_t i = 0; i < nt; ++i)
            qv[i] = cplx(q[2 * i], q[2 * i + 1]);
        const System S = assemble(P, plan, R, num, k, qv, 1);
        std::memcpy(A, S.A.data(), S.A.size() * sizeof(cplx));
        std::memcpy(rhs, S.rhs.data(), S.rhs.size() * sizeof(cplx));
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Complete dense solve (cuda_solver.cu:1021-1853) for every frequency and
// excitation. Excitations are given as a CSR list of (face id, velocity).
// Outputs (complex interleaved): trace [F][E][N], surface [F][E][T],
// observer [F][E][O]; residual [F][E]; field degrees [F][E][2] and
// discrepancy [F][E]; refinement steps [F].
int oracle_solve(const double *verts, size_t nv, const uint32_t *tris, const uint32_t *faces, const uint8_t *driven,
                 size_t nt, double density, double soundSpeed, const double *freqs, size_t nf, double planMaxFreq,
                 size_t ne, const size_t *excOffsets, const uint32_t *excFaces, const double *excVel,
                 const double *observers, size_t no, int farField, const double *farOrigin, double farDistance,
                 const oracle_numerics *nm, double *trace, double *surface, double *observed, double *residual,
                 uint32_t *fieldDegrees, double *fieldDiscrepancy, uint32_t *refinements) {
    try {
        V3 origin;
        const Problem P = makeProblem(verts, nv, tris, faces, driven, nt, &origin);
        const Space &sp = P.space;
        const size_t N = sp.vertices.size(), T = sp.panels.size();
        Numerics num{nm->quadrature_order, nm->singular_order, nm->near_ratio, nm->near_tol, nm->near_depth,
                     nm->residual_tol, nm->max_refine};
        double fmax = planMaxFreq;
        for (size_t f = 0; f < nf; ++f)
            if (planMaxFreq <= 0)
                fmax = std::max(fmax, freqs[f]);
        const double maxK = 2 * M_PI * fmax / soundSpeed;
        PlanSettings st{num.quadratureOrder, num.singularOrder, num.nearRatio, num.nearTol, num.nearDepth};
        // The plan of the last call is reused when mesh, settings and planning
        // wavenumber repeat (a sweep's later calls, like a solver session's cache).
        static std::mutex cacheMutex;
        static std::vector<double> cachedVerts;
        static std::vector<uint32_t> cachedTris;
        static std::vector<double> cachedKey;
        static std::shared_ptr<const Plan> cachedPlan;
        std::shared_ptr<const Plan> planPtr;
        {
            const std::vector<double> key{double(num.quadratureOrder), double(num.singularOrder), num.nearRatio,
                                          num.nearTol, double(num.nearDepth), maxK};
            std::lock_guard<std::mutex> lock(cacheMutex);
            if (cachedPlan && key == cachedKey && cachedVerts.size() == 3 * nv && cachedTris.size() == 3 * nt &&
                std::equal(cachedVerts.begin(), cachedVerts.end(), verts) &&
                std::equal(cachedTris.begin(), cachedTris.end(), tris))
                planPtr = cachedPlan;
            else {
                planPtr = std::make_shared<const Plan>(makePlan(sp, st, maxK));
                cachedVerts.assign(verts, verts + 3 * nv);
                cachedTris.assign(tris, tris + 3 * nt);
                cachedKey = key;
                cachedPlan = planPtr;
            }
        }
        const Plan &plan = *planPtr;
        const Rules R = makeRules(num);
        // Per-panel velocity per excitation.
        std::vector<cplx> vel(ne * T, 0);
        for (size_t e = 0; e < ne; ++e) {
            std::map<uint32_t, cplx> m;
            for (size_t i = excOffsets[e]; i < excOffsets[e + 1]; ++i)
                m[excFaces[i]] = cplx(excVel[2 * i], excVel[2 * i + 1]);
            for (size_t t = 0; t < T; ++t) {
                const auto it = m.find(P.faces[t]);
                if (it != m.end())
                    vel[e * T + t] = it->second;
            }
        }
        std::vector<V3> obs(no);
        const V3 fo = farField ? V3{farOrigin[0], farOrigin[1], farOrigin[2]} : origin;
        for (size_t o = 0; o < no; ++o) {
            V3 x = V3{observers[3 * o], observers[3 * o + 1], observers[3 * o + 2]} - fo;
            if (farField) {
                const double d = std::hypot(x.x, x.y, x.z);
                x = {x.x / d, x.y / d, x.z / d};
            } else if (insideSolid(sp.panels, x))
                throw std::invalid_argument("BEM observation points must be finite and outside the solid.");
            obs[o] = x;
        }
        const V3 farLocal = fo - origin;
        for (size_t f = 0; f < nf; ++f) {
            const double omega = 2 * M_PI * freqs[f], k = omega / soundSpeed;
            std::vector<cplx> q(ne * T);
            for (size_t i = 0; i < ne * T; ++i)
                q[i] = cplx(0, -density * omega) * vel[i];
            const System S = assemble(P, plan, R, num, k, q, ne);
            std::vector<cplx> LU = S.A;
            std::vector<size_t> piv;
            luFactor(LU, N, piv);
            std::vector<cplx> p(N * ne);
            unsigned steps = 0;
            std::vector<double> rel(ne);
            std::vector<double> rhsNorm(ne, 0);
            for (size_t e = 0; e < ne; ++e)
                for (size_t r = 0; r < N; ++r)
                    rhsNorm[e] = std::hypot(rhsNorm[e], std::abs(S.rhs[r * ne + e]) * sp.lumpedMass[r]);
            for (size_t e = 0; e < ne; ++e) {
                std::vector<cplx> x(N);
                for (size_t r = 0; r < N; ++r)
                    x[r] = S.rhs[r * ne + e];
                luSolve(LU, N, piv, x);
                for (size_t r = 0; r < N; ++r)
                    p[e * N + r] = x[r];
            }
            for (;;) {
                double largest = 0;
                std::vector<cplx> corr(N * ne);
                for (size_t e = 0; e < ne; ++e) {
                    double nrm = 0;
                    for (size_t r = 0; r < N; ++r) {
                        cplx acc = 0;
                        for (size_t c = 0; c < N; ++c)
                            acc += S.A[r * N + c] * p[e * N + c];
                        corr[e * N + r] = S.rhs[r * ne + e] - acc;
                        nrm = std::hypot(nrm, std::abs(corr[e * N + r]) * sp.lumpedMass[r]);
                    }
                    rel[e] = rhsNorm[e] > 0 ? nrm / rhsNorm[e] : (nrm == 0 ? 0 : INFINITY);
                    largest = std::max(largest, rel[e]);
                }
                if (largest <= num.residualTol)
                    break;
                if (steps >= num.maxRefine)
                    throw std::runtime_error("Burton-Miller residual exceeds tolerance after refinement.");
                for (size_t e = 0; e < ne; ++e) {
                    std::vector<cplx> x(corr.begin() + e * N, corr.begin() + (e + 1) * N);
                    luSolve(LU, N, piv, x);
                    for (size_t r = 0; r < N; ++r)
                        p[e * N + r] += x[r];
                }
                ++steps;
            }
            refinements[f] = steps;
            for (size_t e = 0; e < ne; ++e) {
                residual[f * ne + e] = rel[e];
                for (size_t r = 0; r < N; ++r) {
                    trace[2 * ((f * ne + e) * N + r)] = p[e * N + r].real();
                    trace[2 * ((f * ne + e) * N + r) + 1] = p[e * N + r].imag();
                }
                for (size_t t = 0; t < T; ++t) {
                    cplx avg = 0;
                    for (int i = 0; i < 3; ++i)
                        avg += p[e * N + sp.panels[t].nodes[i]] / 3.0;
                    surface[2 * ((f * ne + e) * T + t)] = avg.real();
                    surface[2 * ((f * ne + e) * T + t) + 1] = avg.imag();
                }
            }
            if (no) {
                double maxKh = 0;
                for (const auto &pn : sp.panels)
                    maxKh = std::max(maxKh, k * pn.maxEdge);
                const double tolField = std::min(num.nearTol, .025 * num.residualTol);
                auto evaluate = [&](unsigned degree) {
                    const auto rule = triangleRule(degree);
                    std::vector<cplx> out(ne * no);
                    for (size_t e = 0; e < ne; ++e)
                        for (size_t o = 0; o < no; ++o) {
                            cplx sum = 0;
                            for (size_t t = 0; t < T; ++t) {
                                const Panel &pn = sp.panels[t];
                                const cplx qq = q[e * T + t];
                                if (farField)
                                    sum += asymptoticField(obs[o], farLocal, pn, rule, &p[e * N], qq, k);
                                else {
                                    const V3 off = obs[o] - pn.centroid;
                                    if (norm2(off) > 4 * pn.maxEdge * pn.maxEdge)
                                        sum += fieldPatch(obs[o], pn, {{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, 1.0, 0}, rule,
                                                          &p[e * N], qq, k)
                                                   .value;
                                    else
                                        sum += nearField(obs[o], pn, rule, &p[e * N], qq, k, tolField, num.nearDepth);
                                }
                            }
                            if (farField)
                                sum *= cplx(std::cos(k * farDistance), -std::sin(k * farDistance)) / farDistance;
                            out[e * no + o] = sum;
                        }
                    return out;
                };
                unsigned degree = endpointDegree(maxKh, num.quadratureOrder);
                auto current = evaluate(degree);
                for (;;) {
                    const unsigned next = refinedDegree(degree);
                    auto refined = evaluate(next);
                    bool passed = true;
                    for (size_t e = 0; e < ne; ++e) {
                        double d2 = 0, n2 = 0;
                        for (size_t o = 0; o < no; ++o) {
                            d2 += std::norm(refined[e * no + o] - current[e * no + o]);
                            n2 += std::norm(refined[e * no + o]);
                        }
                        const double ind = n2 > 0 ? std::sqrt(d2 / n2) : (d2 == 0 ? 0 : INFINITY);
                        fieldDegrees[2 * (f * ne + e)] = degree;
                        fieldDegrees[2 * (f * ne + e) + 1] = next;
                        fieldDiscrepancy[f * ne + e] = ind;
                        passed &= ind <= .025 * num.residualTol;
                    }
                    current = refined;
                    if (passed)
                        break;
                    if (degree == 12)
                        throw std::runtime_error("BEM complex observer-field quadrature 12/14 did not converge.");
                    degree = next;
                }
                for (size_t i = 0; i < ne * no; ++i) {
                    observed[2 * (f * ne * no + i)] = current[i].real();
                    observed[2 * (f * ne * no + i) + 1] = current[i].imag();
                }
            }
        }
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

}  // extern "C"
