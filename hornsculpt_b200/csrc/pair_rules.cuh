// Host/device geometry and pair-quadrature maps shared by the host planner
// and the sm_100a assembly kernels.
//
// The Sauter-Schwab sector maps, the shared-node permutation and the
// projected near-pair fan keep the reference's exact formulas
// (modules/bem/galerkin/pair_quadrature.hpp:57-215,
// modules/bem/galerkin/near_projection.hpp:119-216) because the interaction
// plan and the quadrature points must be identical for parity.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define HS_HD __host__ __device__ __forceinline__
#else
#define HS_HD inline
#endif

namespace hsb {

struct V3 {
    double x, y, z;
};
HS_HD V3 v3(double x, double y, double z) { return V3{x, y, z}; }
HS_HD V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
HS_HD V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
HS_HD V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
HS_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HS_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
HS_HD double norm2(V3 a) { return dot(a, a); }

struct GaussPoint {
    double x, w;
};
struct TriPoint {
    double b[3];
    double w;
};
struct PairPoint {
    double t[3], s[3];
    double w;
};

enum Topology : uint32_t { kDisjoint = 0, kSharedVertex = 1, kSharedEdge = 2, kCoincident = 3 };

struct Permutation {
    uint32_t topology;
    uint8_t test[3], trial[3];
};

// Shared node ids in ascending order first, then the other local indices
// (pair_quadrature.hpp:57-97).
HS_HD Permutation classifyNodes(const uint32_t *a, const uint32_t *b) {
    Permutation r{kDisjoint, {0, 1, 2}, {0, 1, 2}};
    uint32_t shared[3] = {0, 0, 0};
    unsigned n = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (a[i] == b[j] && n < 3)
                shared[n++] = a[i];
    for (unsigned i = 1; i < n; ++i)
        for (unsigned j = i; j > 0 && shared[j] < shared[j - 1]; --j) {
            const uint32_t tmp = shared[j];
            shared[j] = shared[j - 1];
            shared[j - 1] = tmp;
        }
    r.topology = n == 3 ? kCoincident : n == 2 ? kSharedEdge : n == 1 ? kSharedVertex : kDisjoint;
    unsigned tx = 0, ty = 0;
    for (unsigned s = 0; s < n; ++s)
        for (int i = 0; i < 3; ++i) {
            if (a[i] == shared[s])
                r.test[tx++] = uint8_t(i);
            if (b[i] == shared[s])
                r.trial[ty++] = uint8_t(i);
        }
    for (int i = 0; i < 3; ++i) {
        bool sa = false, sb = false;
        for (unsigned s = 0; s < n; ++s) {
            sa = sa || a[i] == shared[s];
            sb = sb || b[i] == shared[s];
        }
        if (!sa)
            r.test[tx++] = uint8_t(i);
        if (!sb)
            r.trial[ty++] = uint8_t(i);
    }
    return r;
}

HS_HD unsigned sectorCount(uint32_t topo) {
    return topo == kCoincident ? 6u : topo == kSharedEdge ? 5u : topo == kSharedVertex ? 2u : 1u;
}

// Sauter-Schwab sector maps of (r,u,v,w) for touching panels; barycentrics
// in canonical (shared-first) local order; weight = 4-D Jacobian.
HS_HD PairPoint sauterSchwab(uint32_t topo, unsigned sector, double r, double u, double v, double w) {
    double xs = 0, xt = 0, ys = 0, yt = 0, jac = 0, tmp;
    if (topo == kSharedVertex) {
        xs = r; xt = r * u; ys = r * v; yt = r * v * w; jac = r * r * r * v;
        if (sector == 1) { tmp = xs; xs = ys; ys = tmp; tmp = xt; xt = yt; yt = tmp; }
    } else if (topo == kSharedEdge) {
        jac = r * r * r * u * u;
        if (sector == 0) { xs = r; xt = r * u * w; ys = r * (1 - u * v); yt = r * u * (1 - v); }
        else if (sector == 1) { xs = r; xt = r * u; ys = r * (1 - u * v * w); yt = r * u * v * (1 - w); jac *= v; }
        else if (sector == 2) { xs = r * (1 - u * v); xt = r * u * (1 - v); ys = r; yt = r * u * v * w; jac *= v; }
        else if (sector == 3) { xs = r * (1 - u * v * w); xt = r * u * v * (1 - w); ys = r; yt = r * u; jac *= v; }
        else { xs = r * (1 - u * v * w); xt = r * u * (1 - v * w); ys = r; yt = r * u * v; jac *= v; }
    } else if (topo == kCoincident) {
        jac = r * r * r * u * u * v;
        const unsigned d = sector % 3;
        if (d == 0) { xs = r; xt = r * (1 - u + u * v); ys = r * (1 - u * v * w); yt = r * (1 - u); }
        else if (d == 1) { xs = r; xt = r * u * (1 - v + v * w); ys = r * (1 - u * v); yt = r * u * (1 - v); }
        else { xs = r * (1 - u * v * w); xt = r * u * (1 - v * w); ys = r; yt = r * u * (1 - v); }
        if (sector >= 3) { tmp = xs; xs = ys; ys = tmp; tmp = xt; xt = yt; yt = tmp; }
    } else {
        xs = r; xt = r * u; ys = v; yt = v * w; jac = r * v;
    }
    PairPoint p;
    p.t[0] = 1 - xs; p.t[1] = xs - xt; p.t[2] = xt;
    p.s[0] = 1 - ys; p.s[1] = ys - yt; p.s[2] = yt;
    p.w = jac;
    return p;
}

HS_HD PairPoint permutePoint(const PairPoint &p, const Permutation &perm) {
    PairPoint r;
    r.w = p.w;
    for (int i = 0; i < 3; ++i) {
        r.t[perm.test[i]] = p.t[i];
        r.s[perm.trial[i]] = p.s[i];
    }
    return r;
}

// One near-pair quadrature patch (pair_quadrature.hpp:41-55): child triangle
// vertices in parent barycentrics, area fraction, outer degree (8/14),
// projected flag and inner interval count.
struct Patch {
    double test[9], trial[9];
    double areaFraction;
    uint32_t degree, projection, intervals, pad;
};

// Panel geometry needed by the projected fan (vertices, unit normal, area).
struct FanPanel {
    V3 v[3];
    V3 n;
    double area;
};

// Exact oriented fan decomposition of the trial triangle about the
// orthogonal projection of a test point, with sinh-clustered angular and
// radial maps (near_projection.hpp:109-216).
struct ProjOuter {
    double test[3], proj[3];
    V3 rel;
    double height, h, weight;
};
struct ProjEdge {
    V3 offset, dir;
    double center, width, lower, upper;
    unsigned edge, next, opposite;
};
struct ProjRay {
    double boundary[3];
    double stretch, denom, fan, du, aw;
};

HS_HD ProjOuter projOuter(const double *outerBary, double outerWeight, const Patch &patch, const FanPanel &t,
                          const FanPanel &s) {
    ProjOuter p;
    for (int i = 0; i < 3; ++i) {
        p.test[i] = 0;
        for (int j = 0; j < 3; ++j)
            p.test[i] += outerBary[j] * patch.test[3 * j + i];
    }
    const V3 e1 = s.v[1] - s.v[0], e2 = s.v[2] - s.v[0];
    const V3 t1 = t.v[1] - t.v[0], t2 = t.v[2] - t.v[0];
    p.rel = t.v[0] - s.v[0];
    p.rel.x += t1.x * p.test[1] + t2.x * p.test[2];
    p.rel.y += t1.y * p.test[1] + t2.y * p.test[2];
    p.rel.z += t1.z * p.test[1] + t2.z * p.test[2];
    const V3 g1 = cross(e2, s.n), g2 = cross(s.n, e1);
    p.proj[1] = dot(p.rel, g1) / (2 * s.area);
    p.proj[2] = dot(p.rel, g2) / (2 * s.area);
    p.proj[0] = 1 - p.proj[1] - p.proj[2];
    p.height = dot(p.rel, s.n);
    p.h = fabs(p.height);
    p.weight = outerWeight * patch.areaFraction;
    return p;
}

HS_HD ProjEdge projEdge(const ProjOuter &o, unsigned edge, const FanPanel &s) {
    ProjEdge e;
    e.edge = edge;
    e.next = (edge + 1) % 3;
    e.opposite = (edge + 2) % 3;
    const V3 a = s.v[edge] - s.v[0];
    e.dir = s.v[e.next] - s.v[edge];
    e.offset = V3{a.x - o.rel.x + o.height * s.n.x, a.y - o.rel.y + o.height * s.n.y, a.z - o.rel.z + o.height * s.n.z};
    const double l2 = dot(e.dir, e.dir);
    e.center = -dot(e.offset, e.dir) / l2;
    const V3 perp{e.offset.x + e.center * e.dir.x, e.offset.y + e.center * e.dir.y, e.offset.z + e.center * e.dir.z};
    e.width = sqrt((dot(perp, perp) + o.h * o.h) / l2);
    e.lower = asinh(-e.center / e.width);
    e.upper = asinh((1 - e.center) / e.width);
    return e;
}

HS_HD ProjRay projRay(const ProjOuter &o, const ProjEdge &e, GaussPoint ang) {
    ProjRay r;
    const double par = e.lower + (e.upper - e.lower) * ang.x;
    const double u = e.center + e.width * sinh(par);
    r.du = e.width * (e.upper - e.lower) * cosh(par);
    const V3 ray{e.offset.x + u * e.dir.x, e.offset.y + u * e.dir.y, e.offset.z + u * e.dir.z};
    r.stretch = asinh(sqrt(dot(ray, ray)) / o.h);
    r.denom = sinh(r.stretch);
    for (unsigned i = 0; i < 3; ++i)
        r.boundary[i] = i == e.edge ? 1 - u : (i == e.next ? u : 0);
    r.fan = o.weight * o.proj[e.opposite];
    r.aw = ang.w;
    return r;
}

HS_HD PairPoint projPoint(const ProjOuter &o, const ProjRay &r, GaussPoint rad) {
    PairPoint p;
    const double t = r.stretch == 0 ? rad.x : sinh(r.stretch * rad.x) / r.denom;
    const double dt = r.stretch == 0 ? 1 : r.stretch * cosh(r.stretch * rad.x) / r.denom;
    for (int i = 0; i < 3; ++i) {
        p.t[i] = o.test[i];
        p.s[i] = o.proj[i] + t * (r.boundary[i] - o.proj[i]);
    }
    p.w = r.fan * t * dt * r.du * r.aw * rad.w;
    return p;
}

// Regular-rule qualification (regular_qualification.hpp:274-345): a
// conservative enclosing ball per panel plus the measured separation / k*h
// envelopes of the 4/6/8 Dunavant pair rules; 0 selects adaptive quadrature.
struct Bounds {
    V3 center;
    double radius, maxEdge;
    uint32_t qualified, pad;
};

HS_HD unsigned qualifiedDegree(const Bounds &t, const Bounds &s, double k, double tol, unsigned minDegree) {
    if (!t.qualified || !s.qualified)
        return 0;
    const double h = t.maxEdge > s.maxEdge ? t.maxEdge : s.maxEdge, kh = k * h;
    const double dx = t.center.x - s.center.x, dy = t.center.y - s.center.y, dz = t.center.z - s.center.z;
    const double d2 = dx * dx + dy * dy + dz * dz, rs = t.radius + s.radius, budget = .2 * tol;
    const double reserve = 1e-6;
#define HS_SEPARATED(gap) (d2 >= (rs + (gap) * h) * (rs + (gap) * h))
    if (minDegree <= 4 && ((kh <= .5 && HS_SEPARATED(3) && reserve + 4 * 2.3e-6 <= budget) ||
                           (kh <= .25 && HS_SEPARATED(8) && reserve + 4 * 1e-7 <= budget)))
        return 4;
    if (minDegree <= 6 && ((kh <= 2 && HS_SEPARATED(1) && reserve + 4 * 6e-7 <= budget) ||
                           (kh <= 1 && HS_SEPARATED(2) && reserve + 4 * 2.4e-8 <= budget)))
        return 6;
    if (minDegree <= 8 && kh <= 2 &&
        ((HS_SEPARATED(.5) && reserve + 4 * 7.5e-7 <= budget) || (HS_SEPARATED(1) && reserve + 4 * 3.5e-8 <= budget)))
        return 8;
#undef HS_SEPARATED
    return 0;
}

// Packed index of an unordered distinct panel pair (interaction_plan.hpp:19-22).
HS_HD uint64_t unorderedPairIndex(uint32_t a, uint32_t b) {
    const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
    return hi * (hi - 1) / 2 + lo;
}

}  // namespace hsb
