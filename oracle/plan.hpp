// Test infrastructure only: the FP64 CPU oracle's restatement of HornSculpt's
// dense interaction plan — triangle distances, the projected near-pair fan,
// the embedded-rule error estimator and the largest-error adaptive state
// machine (galerkin/pair_quadrature.cpp, near_projection.hpp,
// regular_qualification.hpp, interaction_plan.cpp).
#pragma once

#include "geometry.hpp"

#include <algorithm>
#include <map>
#include <vector>

namespace oracle {

using Bary = std::array<double, 3>;
struct Sub {
    std::array<Bary, 3> v{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
    double fraction{1};
};

// galerkin/pair_quadrature.hpp:41-55
struct Patch {
    double test[9]{}, trial[9]{};
    double areaFraction{};
    unsigned degree{8};
    unsigned projection{};
    unsigned intervals{1};
};

// pair_quadrature.cpp:43-71 closest point of a triangle (Ericson's regions).
inline double pointTriangleD2(V3 p, const std::array<V3, 3> &tr) {
    const V3 a = tr[0], b = tr[1], c = tr[2];
    const V3 ab = b - a, ac = c - a, ap = p - a;
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0)
        return norm2(ap);
    const V3 bp = p - b;
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3)
        return norm2(bp);
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0)
        return norm2(p - (a + ab * (d1 / (d1 - d3))));
    const V3 cp = p - c;
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6)
        return norm2(cp);
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0)
        return norm2(p - (a + ac * (d2 / (d2 - d6))));
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        const double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return norm2(p - (b + (c - b) * t));
    }
    const double inv = 1 / (va + vb + vc);
    return norm2(p - (a + (ab * (vb * inv) + ac * (vc * inv))));
}
// pair_quadrature.cpp:73-88 segment-segment distance.
inline double segmentD2(V3 p, V3 q, V3 a, V3 b) {
    const V3 u = q - p, v = b - a, w = p - a;
    const double aa = dot(u, u), bb = dot(u, v), cc = dot(v, v), dd = dot(u, w), ee = dot(v, w);
    const double det = aa * cc - bb * bb;
    double s = det > aa * cc * 1e-14 ? std::clamp((bb * ee - cc * dd) / det, 0.0, 1.0) : 0;
    double t = (bb * s + ee) / cc;
    if (t < 0) {
        t = 0;
        s = std::clamp(-dd / aa, 0.0, 1.0);
    } else if (t > 1) {
        t = 1;
        s = std::clamp((bb - dd) / aa, 0.0, 1.0);
    }
    return norm2((w + u * s) - v * t);
}
inline double triangleDistance(const std::array<V3, 3> &a, const std::array<V3, 3> &b) {
    double d2 = std::numeric_limits<double>::infinity();
    for (int i = 0; i < 3; ++i) {
        d2 = std::min({d2, pointTriangleD2(a[i], b), pointTriangleD2(b[i], a)});
        for (int j = 0; j < 3; ++j)
            d2 = std::min(d2, segmentD2(a[i], a[(i + 1) % 3], b[j], b[(j + 1) % 3]));
    }
    return std::sqrt(d2);
}
// pair_quadrature.cpp:800-807 — distances in the test panel's vertex-0 frame.
inline double panelDistance(const Panel &t, const Panel &s) {
    std::array<V3, 3> a, b;
    for (int i = 0; i < 3; ++i) {
        a[i] = t.v[i] - t.v[0];
        b[i] = s.v[i] - t.v[0];
    }
    return triangleDistance(a, b);
}
// pair_quadrature.cpp:786-798
inline bool isNearPair(const Panel &t, const Panel &s, double ratio) {
    if (ratio == 0)
        return false;
    if (classify(t.nodes, s.nodes).topology != Disjoint)
        return false;
    const double size = std::max(t.maxEdge, s.maxEdge);
    const double bound = ratio * size + t.maxEdge + s.maxEdge;
    if (norm2(t.centroid - s.centroid) >= bound * bound)
        return false;
    return panelDistance(t, s) < ratio * size;
}

// regular_qualification.hpp:20-26, 284-306
struct Bounds {
    V3 center;
    double radius{}, maxEdge{};
    bool qualified{};
};
inline Bounds makeBounds(const Panel &p) {
    Bounds b{p.centroid, 0, p.maxEdge, true};
    double e[3];
    for (int i = 0; i < 3; ++i) {
        const V3 a = p.v[i], c = p.v[(i + 1) % 3];
        e[i] = std::hypot(a.x - c.x, a.y - c.y, a.z - c.z);
        b.radius = std::max(b.radius, std::hypot(a.x - p.centroid.x, a.y - p.centroid.y, a.z - p.centroid.z));
    }
    b.radius = std::nextafter(b.radius * (1 + 8 * std::numeric_limits<double>::epsilon()),
                              std::numeric_limits<double>::infinity());
    constexpr double cos20 = .939692620785908384;
    for (int i = 0; i < 3; ++i) {
        const double a = e[i], bb = e[(i + 1) % 3], c = e[(i + 2) % 3];
        b.qualified &= a > 0 && bb > 0 && (a * a + bb * bb - c * c) <= 2 * a * bb * cos20;
    }
    b.qualified &= std::isfinite(b.radius) && b.maxEdge > 0;
    return b;
}
// regular_qualification.hpp:315-345: measured envelopes of the 4/6/8 Dunavant
// pair rules against separation (in units of h) and k*h; 0 = adaptive.
inline unsigned qualifiedDegree(const Bounds &t, const Bounds &s, double k, double tol, unsigned minDegree) {
    if (!t.qualified || !s.qualified)
        return 0;
    const double h = t.maxEdge > s.maxEdge ? t.maxEdge : s.maxEdge, kh = k * h;
    const double dx = t.center.x - s.center.x, dy = t.center.y - s.center.y, dz = t.center.z - s.center.z;
    const double d2 = dx * dx + dy * dy + dz * dz, rs = t.radius + s.radius, budget = .2 * tol;
    auto separated = [&](double gap) {
        const double b = rs + gap * h;
        return d2 >= b * b;
    };
    constexpr double reserve = 1e-6;
    if (minDegree <= 4 && ((kh <= .5 && separated(3) && reserve + 4 * 2.3e-6 <= budget) ||
                           (kh <= .25 && separated(8) && reserve + 4 * 1e-7 <= budget)))
        return 4;
    if (minDegree <= 6 && ((kh <= 2 && separated(1) && reserve + 4 * 6e-7 <= budget) ||
                           (kh <= 1 && separated(2) && reserve + 4 * 2.4e-8 <= budget)))
        return 6;
    if (minDegree <= 8 && kh <= 2 &&
        ((separated(.5) && reserve + 4 * 7.5e-7 <= budget) || (separated(1) && reserve + 4 * 3.5e-8 <= budget)))
        return 8;
    return 0;
}
// regular_qualification.hpp:360-377
inline unsigned endpointDegree(double maxKh, unsigned requested) {
    if (!std::isfinite(maxKh) || maxKh < 0)
        throw std::invalid_argument("endpoint kh");
    if (maxKh > 3.25)
        throw std::runtime_error("k*h exceeds the qualified electrical range 3.25");
    const unsigned e = maxKh <= .25 ? 4 : maxKh <= 1 ? 6 : maxKh <= 2 ? 8 : 12;
    return std::max(e, requested);
}
inline unsigned refinedDegree(unsigned d) {
    return d < 4 ? 4 : d < 6 ? 6 : d < 8 ? 8 : d < 12 ? 12 : d < 14 ? 14 : 0;
}

// ---- projected near-pair fan (near_projection.hpp:119-216) ----
struct ProjOuter {
    double test[3]{}, proj[3]{};
    V3 rel;
    double height{}, h{}, weight{};
};
struct ProjEdge {
    V3 offset, dir;
    double center{}, width{}, lower{}, upper{};
    unsigned edge{}, next{}, opposite{};
};
struct ProjRay {
    double boundary[3]{};
    double stretch{}, denom{}, fan{}, du{}, aw{};
};
inline ProjOuter projOuter(const TriPoint &o, const Patch &patch, const Panel &t, const Panel &s) {
    ProjOuter p;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            p.test[i] += o.b[j] * patch.test[3 * j + i];
    const V3 e1 = s.v[1] - s.v[0], e2 = s.v[2] - s.v[0];
    const V3 t1 = t.v[1] - t.v[0], t2 = t.v[2] - t.v[0];
    p.rel = t.v[0] - s.v[0];
    p.rel.x += t1.x * p.test[1] + t2.x * p.test[2];
    p.rel.y += t1.y * p.test[1] + t2.y * p.test[2];
    p.rel.z += t1.z * p.test[1] + t2.z * p.test[2];
    const V3 g1 = cross(e2, s.normal), g2 = cross(s.normal, e1);
    p.proj[1] = dot(p.rel, g1) / (2 * s.area);
    p.proj[2] = dot(p.rel, g2) / (2 * s.area);
    p.proj[0] = 1 - p.proj[1] - p.proj[2];
    p.height = dot(p.rel, s.normal);
    p.h = std::fabs(p.height);
    p.weight = o.w * patch.areaFraction;
    return p;
}
inline ProjEdge projEdge(const ProjOuter &o, unsigned edge, const Panel &s) {
    ProjEdge e;
    e.edge = edge;
    e.next = (edge + 1) % 3;
    e.opposite = (edge + 2) % 3;
    const V3 a = s.v[edge] - s.v[0];
    e.dir = s.v[e.next] - s.v[edge];
    e.offset = {a.x - o.rel.x + o.height * s.normal.x, a.y - o.rel.y + o.height * s.normal.y,
                a.z - o.rel.z + o.height * s.normal.z};
    const double l2 = dot(e.dir, e.dir);
    e.center = -dot(e.offset, e.dir) / l2;
    const V3 perp{e.offset.x + e.center * e.dir.x, e.offset.y + e.center * e.dir.y,
                  e.offset.z + e.center * e.dir.z};
    e.width = std::sqrt((dot(perp, perp) + o.h * o.h) / l2);
    e.lower = std::asinh(-e.center / e.width);
    e.upper = std::asinh((1 - e.center) / e.width);
    return e;
}
inline ProjRay projRay(const ProjOuter &o, const ProjEdge &e, GaussPoint ang) {
    ProjRay r;
    const double par = e.lower + (e.upper - e.lower) * ang.x;
    const double u = e.center + e.width * std::sinh(par);
    r.du = e.width * (e.upper - e.lower) * std::cosh(par);
    const V3 ray{e.offset.x + u * e.dir.x, e.offset.y + u * e.dir.y, e.offset.z + u * e.dir.z};
    r.stretch = std::asinh(std::sqrt(dot(ray, ray)) / o.h);
    r.denom = std::sinh(r.stretch);
    for (unsigned i = 0; i < 3; ++i)
        r.boundary[i] = i == e.edge ? 1 - u : (i == e.next ? u : 0);
    r.fan = o.weight * o.proj[e.opposite];
    r.aw = ang.w;
    return r;
}
inline PairPoint projPoint(const ProjOuter &o, const ProjRay &r, GaussPoint rad) {
    PairPoint p;
    const double t = r.stretch == 0 ? rad.x : std::sinh(r.stretch * rad.x) / r.denom;
    const double dt = r.stretch == 0 ? 1 : r.stretch * std::cosh(r.stretch * rad.x) / r.denom;
    for (int i = 0; i < 3; ++i) {
        p.t[i] = o.test[i];
        p.s[i] = o.proj[i] + t * (r.boundary[i] - o.proj[i]);
    }
    p.w = r.fan * t * dt * r.du * r.aw * rad.w;
    return p;
}

// ---- embedded-rule patch estimator (pair_quadrature.cpp:143-226, 644-683) ----
using Moments36 = std::array<cplx, 36>;

inline std::array<cplx, 4> pointKernels(V3 d, double k, double scale) {
    const double r = std::sqrt(norm2(d));
    if (!(r > 0))
        throw std::invalid_argument("disjoint quadrature panels intersect");
    const cplx g = std::exp(cplx(0, -k * r)) / r;
    const cplx der = -g * cplx(1, k * r) * (scale / (r * r));
    return {g, der * d.x, der * d.y, der * d.z};
}
inline PairPoint mappedPoint(const TriPoint &x, const TriPoint &y, const Sub &a, const Sub &b) {
    PairPoint p;
    p.w = x.w * y.w * a.fraction * b.fraction;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            p.t[i] += x.b[j] * a.v[j][i];
            p.s[i] += y.b[j] * b.v[j][i];
        }
    return p;
}
inline Moments36 tensorMoments(const Panel &t, const Panel &s, const Sub &a, const Sub &b,
                               const std::vector<TriPoint> &rule, double k, double scale) {
    Moments36 m{};
    for (const auto &x : rule)
        for (const auto &y : rule) {
            const PairPoint p = mappedPoint(x, y, a, b);
            const auto ker = pointKernels(pairDelta(t, p.t, s, p.s), k, scale);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double w = p.w * p.t[i] * p.s[j];
                    for (int c = 0; c < 4; ++c)
                        m[c * 9 + i * 3 + j] += ker[c] * w;
                }
        }
    return m;
}
inline Moments36 projectionMoments(const Panel &t, const Panel &s, const Sub &a,
                                   const std::vector<TriPoint> &outer, unsigned order, unsigned intervals,
                                   double k, double scale) {
    Patch patch;
    patch.projection = 1;
    patch.areaFraction = a.fraction;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            patch.test[3 * i + j] = a.v[i][j];
    const auto base = gauss01(order);
    std::vector<GaussPoint> g;
    for (unsigned iv = 0; iv < intervals; ++iv)
        for (const auto &p : base)
            g.push_back({(iv + p.x) / intervals, p.w / intervals});
    Moments36 m{};
    const V3 offset = t.v[0] - s.v[0];
    for (const auto &x : outer) {
        const ProjOuter po = projOuter(x, patch, t, s);
        const V3 lt = localPoint(t, po.test);
        std::array<cplx, 12> inner{};
        for (unsigned e = 0; e < 3; ++e) {
            const ProjEdge pe = projEdge(po, e, s);
            for (const auto &u : g) {
                const ProjRay ray = projRay(po, pe, u);
                for (const auto &v : g) {
                    const PairPoint p = projPoint(po, ray, v);
                    const V3 d = offset + (lt - localPoint(s, p.s));
                    const auto ker = pointKernels(d, k, scale);
                    for (int j = 0; j < 3; ++j)
                        for (int c = 0; c < 4; ++c)
                            inner[3 * c + j] += ker[c] * (p.w * p.s[j]);
                }
            }
        }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int c = 0; c < 4; ++c)
                    m[9 * c + 3 * i + j] += po.test[i] * inner[3 * c + j];
    }
    return m;
}
inline double maxNorm(const Moments36 &m) {
    double r = 0;
    for (const auto &v : m) {
        const double a = std::abs(v);
        if (!std::isfinite(a))
            throw std::runtime_error("non-finite moment");
        r = std::max(r, a);
    }
    return r;
}
struct Estimate {
    Moments36 integral{};
    double error{}, inner{}, outer{};
};
inline Estimate estimatePatch(const Panel &t, const Panel &s, const Patch &patch, double k) {
    static const auto r6 = triangleRule(6), r8 = triangleRule(8), r12 = triangleRule(12), r14 = triangleRule(14);
    Sub a, b;
    a.fraction = patch.areaFraction;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            a.v[i][j] = patch.test[3 * i + j];
            b.v[i][j] = patch.trial[3 * i + j];
        }
    const double scale = std::max(t.maxEdge, s.maxEdge);
    const auto &lo = patch.degree == 8 ? r6 : r12;
    const auto &hi = patch.degree == 8 ? r8 : r14;
    const Moments36 low = patch.projection ? projectionMoments(t, s, a, lo, 20, patch.intervals, k, scale)
                                           : tensorMoments(t, s, a, b, lo, k, scale);
    const Moments36 high = patch.projection ? projectionMoments(t, s, a, hi, 20, patch.intervals, k, scale)
                                            : tensorMoments(t, s, a, b, hi, k, scale);
    Moments36 diff;
    for (int i = 0; i < 36; ++i)
        diff[i] = high[i] - low[i];
    (void)maxNorm(high);
    const double outer = maxNorm(diff);
    double inner = 0;
    if (patch.projection) {
        const Moments36 il = projectionMoments(t, s, a, hi, 14, patch.intervals, k, scale);
        for (int i = 0; i < 36; ++i)
            diff[i] = high[i] - il[i];
        inner = maxNorm(diff);
    }
    return {high, outer + inner, inner, outer};
}

// pair_quadrature.cpp:231-296: split the test triangle along the projected
// trial edge lines (keeping both halves), fan-triangulate the polygons.
inline std::vector<Sub> projectionPartition(const Panel &t, const Panel &s) {
    Bary proj[3];
    for (int i = 0; i < 3; ++i) {
        const V3 rel = t.v[i] - s.v[0];
        proj[i][1] = dot(rel, s.grad[1]);
        proj[i][2] = dot(rel, s.grad[2]);
        proj[i][0] = 1 - proj[i][1] - proj[i][2];
    }
    using Poly = std::vector<Bary>;
    std::vector<Poly> polys{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
    for (int e = 0; e < 3; ++e) {
        auto val = [&](const Bary &p) { return p[0] * proj[0][e] + p[1] * proj[1][e] + p[2] * proj[2][e]; };
        std::vector<Poly> kids;
        for (const auto &poly : polys) {
            bool pos = false, neg = false;
            for (const auto &p : poly) {
                pos |= val(p) > 0;
                neg |= val(p) < 0;
            }
            if (!(pos && neg)) {
                kids.push_back(poly);
                continue;
            }
            Poly plus, minus;
            for (size_t i = 0; i < poly.size(); ++i) {
                const Bary a = poly[i], b = poly[(i + 1) % poly.size()];
                const double va = val(a), vb = val(b);
                if (va >= 0)
                    plus.push_back(a);
                if (va <= 0)
                    minus.push_back(a);
                if ((va < 0 && vb > 0) || (va > 0 && vb < 0)) {
                    const double tt = va / (va - vb);
                    Bary x;
                    for (int j = 0; j < 3; ++j)
                        x[j] = a[j] + tt * (b[j] - a[j]);
                    plus.push_back(x);
                    minus.push_back(x);
                }
            }
            if (plus.size() >= 3)
                kids.push_back(plus);
            if (minus.size() >= 3)
                kids.push_back(minus);
        }
        polys = std::move(kids);
    }
    std::vector<Sub> out;
    double area = 0;
    for (const auto &poly : polys)
        for (size_t i = 1; i + 1 < poly.size(); ++i) {
            const Bary a = poly[0], b = poly[i], c = poly[i + 1];
            const double f = std::abs((b[1] - a[1]) * (c[2] - a[2]) - (b[2] - a[2]) * (c[1] - a[1]));
            if (f > 0) {
                out.push_back({{a, b, c}, f});
                area += f;
            }
        }
    if (std::abs(area - 1) > 1024 * std::numeric_limits<double>::epsilon())
        throw std::runtime_error("projected partition lost area");
    return out;
}
// pair_quadrature.cpp:298-317
inline bool useProjection(const Panel &t, const Panel &s, double scale) {
    if (panelDistance(t, s) >= .025 * scale)
        return false;
    const double eps = 128 * std::numeric_limits<double>::epsilon() * scale;
    double lo = std::numeric_limits<double>::infinity(), hi = -lo;
    for (int i = 0; i < 3; ++i) {
        const double h = dot(t.v[i] - s.v[0], s.normal);
        lo = std::min(lo, h);
        hi = std::max(hi, h);
    }
    return (lo >= -eps && hi > eps) || (hi <= eps && lo < -eps);
}

inline std::array<Sub, 4> subdivide(const Sub &s) {
    auto mid = [](const Bary &a, const Bary &b) { return Bary{(a[0] + b[0]) * .5, (a[1] + b[1]) * .5, (a[2] + b[2]) * .5}; };
    const Bary a = s.v[0], b = s.v[1], c = s.v[2], ab = mid(a, b), bc = mid(b, c), ca = mid(c, a);
    const double f = s.fraction * .25;
    return {{{{a, ab, ca}, f}, {{ab, b, bc}, f}, {{ca, bc, c}, f}, {{ab, bc, ca}, f}}};
}
inline double subDiameter(const Panel &p, const Sub &s, V3 origin) {
    const V3 off = p.v[0] - origin;
    V3 q[3];
    for (int i = 0; i < 3; ++i)
        q[i] = off + localPoint(p, s.v[i].data());
    return std::sqrt(std::max({norm2(q[0] - q[1]), norm2(q[1] - q[2]), norm2(q[2] - q[0])}));
}

struct PairRule {
    std::vector<Patch> patches;
    unsigned maxDepth{};
    double relError{};
};

// pair_quadrature.cpp:329-575: refine the leaf with the largest embedded
// error estimate until the summed error is below 0.2*tol of the pair's
// largest moment; degree-8 leaves at the depth limit (or a far root) are
// promoted to degree 14, projected leaves may double their inner intervals.
inline PairRule adaptivePair(const Panel &t, const Panel &s, double tol, unsigned maxDepth, double k) {
    struct Leaf {
        Sub a, b;
        Moments36 integral{};
        double error{}, da{}, db{}, inner{}, outer{};
        unsigned depth{}, degree{8}, intervals{1};
    };
    auto less = [](const Leaf &x, const Leaf &y) { return x.error < y.error; };
    const bool projection = useProjection(t, s, std::max(t.maxEdge, s.maxEdge));
    const bool promoteRoot = !projection && !isNearPair(t, s, 1.0);
    std::vector<Sub> initial = projection ? projectionPartition(t, s) : std::vector<Sub>{Sub{}};
    auto leaf = [&](const Sub &a, const Sub &b, unsigned depth, unsigned degree, unsigned intervals) {
        Leaf l;
        l.a = a;
        l.b = b;
        l.da = subDiameter(t, a, t.v[0]);
        l.db = subDiameter(s, b, t.v[0]);
        l.depth = depth;
        l.degree = degree;
        l.intervals = intervals;
        return l;
    };
    auto patchOf = [&](const Leaf &l) {
        Patch p;
        p.degree = l.degree;
        p.projection = projection ? 1 : 0;
        p.intervals = l.intervals;
        p.areaFraction = l.a.fraction * l.b.fraction;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                p.test[3 * i + j] = l.a.v[i][j];
                p.trial[3 * i + j] = l.b.v[i][j];
            }
        return p;
    };
    std::vector<Leaf> pending, atLimit, requested;
    Moments36 integral{};
    double absError = 0;
    size_t nextInitial = 0;
    PairRule result;
    auto requestInitial = [&]() {
        requested.clear();
        while (nextInitial < initial.size() && requested.size() < 4)
            requested.push_back(leaf(initial[nextInitial++], Sub{}, 0, 8, 1));
    };
    requestInitial();
    for (;;) {
        for (auto &l : requested) {
            const Estimate e = estimatePatch(t, s, patchOf(l), k);
            l.integral = e.integral;
            l.error = e.error;
            l.inner = e.inner;
            l.outer = e.outer;
        }
        for (auto &l : requested) {
            absError += l.error;
            for (int i = 0; i < 36; ++i)
                integral[i] += l.integral[i];
            const bool outerLimit = l.depth == maxDepth && l.degree == 14;
            const unsigned nextInner = l.intervals * 2;
            const bool innerLimit = nextInner > (1u << maxDepth) ||
                                    uint64_t(192) * 400 * nextInner * nextInner > std::numeric_limits<unsigned>::max();
            if ((!projection && outerLimit) || (projection && (l.inner > l.outer ? innerLimit : outerLimit)))
                atLimit.push_back(l);
            else {
                pending.push_back(l);
                std::push_heap(pending.begin(), pending.end(), less);
            }
        }
        requested.clear();
        if (nextInitial < initial.size()) {
            requestInitial();
            continue;
        }
        if (absError <= tol * .2 * maxNorm(integral)) {
            for (const auto &l : atLimit) {
                result.maxDepth = std::max(result.maxDepth, l.depth);
                result.patches.push_back(patchOf(l));
            }
            while (!pending.empty()) {
                result.maxDepth = std::max(result.maxDepth, pending.front().depth);
                result.patches.push_back(patchOf(pending.front()));
                std::pop_heap(pending.begin(), pending.end(), less);
                pending.pop_back();
            }
            const double ref = maxNorm(integral);
            result.relError = absError / ref;
            if (!(ref > 0) || !(result.relError <= tol))
                throw std::runtime_error("near-pair quadrature exceeds its tolerance");
            return result;
        }
        if (pending.empty())
            throw std::runtime_error("near-pair quadrature did not converge before the subdivision limit");
        const Leaf v = pending.front();
        std::pop_heap(pending.begin(), pending.end(), less);
        pending.pop_back();
        absError = std::max(0.0, absError - v.error);
        for (int i = 0; i < 36; ++i)
            integral[i] -= v.integral[i];
        if (projection && v.inner > v.outer)
            requested.push_back(leaf(v.a, v.b, v.depth, v.degree, v.intervals * 2));
        else if (v.degree == 8 && (v.depth == maxDepth || (promoteRoot && v.depth == 0)))
            requested.push_back(leaf(v.a, v.b, v.depth, 14, v.intervals));
        else {
            if (pending.size() + atLimit.size() + 4 > 50000)
                throw std::runtime_error("near-pair quadrature exceeds the patch limit");
            if (projection || v.da >= v.db)
                for (const auto &c : subdivide(v.a))
                    requested.push_back(leaf(c, v.b, v.depth + 1, 8, v.intervals));
            else
                for (const auto &c : subdivide(v.b))
                    requested.push_back(leaf(v.a, c, v.depth + 1, 8, 1));
        }
    }
}

// galerkin/interaction_plan.hpp:25-53
struct TouchJob {
    uint32_t test, trial;
    Permutation perm;
};
struct NearJob {
    uint32_t test, trial, first, count, swap;
};
struct Plan {
    std::vector<TouchJob> touching;
    std::vector<NearJob> near;
    std::vector<Patch> patches;
    std::vector<uint8_t> wholePanelDegrees;
    std::vector<uint32_t> nearOffsets, nearTrials;
    unsigned maxDepth{};
    double maxRelError{};
};
inline size_t unorderedIndex(uint32_t a, uint32_t b) {
    const size_t lo = a < b ? a : b, hi = a < b ? b : a;
    return hi * (hi - 1) / 2 + lo;
}
struct PlanSettings {
    unsigned regularOrder{4}, singularOrder{4};
    double nearRatio{1.0}, tol{1e-4};
    unsigned maxDepth{6};
};

// interaction_plan.cpp:228-504, restated serially. Every unordered disjoint
// pair is examined (the reference prunes with a conservative spatial grid,
// which selects the same near set).
inline Plan makePlan(const Space &sp, const PlanSettings &st, double maxK) {
    Plan plan;
    const size_t T = sp.panels.size();
    std::vector<Bounds> bounds(T);
    bool allPairs = !((1e-6 + 4 * 3.5e-8) <= .2 * st.tol);
    for (size_t i = 0; i < T; ++i) {
        bounds[i] = makeBounds(sp.panels[i]);
        allPairs |= !bounds[i].qualified || maxK * sp.panels[i].maxEdge > 2;
    }
    if (allPairs)
        plan.wholePanelDegrees.assign(T * (T - 1) / 2, 0);
    plan.nearOffsets.assign(T + 1, 0);
    for (size_t t = 0; t < T; ++t) {
        std::vector<uint32_t> adj;
        for (int i = 0; i < 3; ++i) {
            const uint32_t n = sp.panels[t].nodes[i];
            for (size_t o = sp.incOffsets[n]; o < sp.incOffsets[n + 1]; ++o)
                adj.push_back(sp.incPanels[o]);
        }
        std::sort(adj.begin(), adj.end());
        adj.erase(std::unique(adj.begin(), adj.end()), adj.end());
        for (auto s : adj)
            plan.touching.push_back({uint32_t(t), s, classify(sp.panels[t].nodes, sp.panels[s].nodes)});
    }
    struct Planned {
        uint32_t a, b;
        PairRule rule;
    };
    std::vector<Planned> planned;
    for (uint32_t i = 0; i < T; ++i)
        for (uint32_t j = i + 1; j < T; ++j) {
            const Panel &t = sp.panels[i], &s = sp.panels[j];
            if (classify(t.nodes, s.nodes).topology != Disjoint)
                continue;
            const unsigned degree = qualifiedDegree(bounds[i], bounds[j], maxK, st.tol, st.regularOrder);
            const double h = std::max(t.maxEdge, s.maxEdge);
            const double limit = bounds[i].radius + bounds[j].radius + st.nearRatio * h;
            const double dx = t.centroid.x - s.centroid.x, dy = t.centroid.y - s.centroid.y,
                         dz = t.centroid.z - s.centroid.z;
            const bool geometricNear = degree && st.nearRatio > 0 && dx * dx + dy * dy + dz * dz < limit * limit &&
                                       isNearPair(t, s, st.nearRatio);
            if (degree && !geometricNear)
                continue;
            PairRule rule = adaptivePair(t, s, st.tol, st.maxDepth, maxK);
            if (allPairs && rule.maxDepth == 0 && rule.patches.size() == 1 && !rule.patches.front().projection) {
                plan.wholePanelDegrees[unorderedIndex(i, j)] = uint8_t(rule.patches.front().degree);
                plan.maxRelError = std::max(plan.maxRelError, rule.relError);
                continue;
            }
            planned.push_back({i, j, std::move(rule)});
        }
    for (auto &e : planned) {
        const uint32_t first = uint32_t(plan.patches.size()), n = uint32_t(e.rule.patches.size());
        plan.patches.insert(plan.patches.end(), e.rule.patches.begin(), e.rule.patches.end());
        plan.near.push_back({e.a, e.b, first, n, 0});
        plan.near.push_back({e.b, e.a, first, n, 1});
        plan.maxDepth = std::max(plan.maxDepth, e.rule.maxDepth);
        plan.maxRelError = std::max(plan.maxRelError, e.rule.relError);
    }
    std::sort(plan.near.begin(), plan.near.end(), [](const NearJob &x, const NearJob &y) {
        return std::pair{x.test, x.trial} < std::pair{y.test, y.trial};
    });
    for (const auto &j : plan.near) {
        ++plan.nearOffsets[j.test + 1];
        plan.nearTrials.push_back(j.trial);
    }
    for (size_t r = 1; r < plan.nearOffsets.size(); ++r)
        plan.nearOffsets[r] += plan.nearOffsets[r - 1];
    return plan;
}

}  // namespace oracle
