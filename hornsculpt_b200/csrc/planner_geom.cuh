// Pair geometry of the interaction planner, shared by the host planner
// (planner.cpp) and the device planner (plan_device.cu) so that both make
// every geometric decision with the same IEEE operations: closest distances
// (Ericson's point-triangle and segment-segment routines,
// pair_quadrature.cpp:43-101, 786-807), the geometric near test, the
// projected-patch test, sub-triangle diameters and quartering
// (pair_quadrature.cpp:231-575).
//
// Every function is a sequence of single IEEE additions, multiplications,
// divisions and square roots; device code that includes this header is
// compiled without floating-point contraction (nvcc -fmad=false), so host and
// device results agree bit for bit.
#pragma once

#include "host_mesh.hpp"

#include <cmath>

namespace hsb {

constexpr double kPlanEps = 0x1p-52;  // DBL_EPSILON

HS_HD double minD(double a, double b) { return b < a ? b : a; }  // std::min
HS_HD double maxD(double a, double b) { return a < b ? b : a; }  // std::max
HS_HD double clampD(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }  // std::clamp

// A sub-triangle of a panel: vertices in the panel's barycentrics and its area
// fraction.
struct Sub {
    double v[3][3];
    double fraction;
};
HS_HD Sub wholeSub() { return Sub{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, 1}; }

HS_HD V3 localPoint(const HostPanel &p, const double *b) {
    return (p.v[1] - p.v[0]) * b[1] + (p.v[2] - p.v[0]) * b[2];
}

HS_HD double pointTriangleD2(V3 p, const V3 *tr) {
    const V3 a = tr[0], b = tr[1], c = tr[2], ab = b - a, ac = c - a, ap = p - a;
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

HS_HD double segmentD2(V3 p, V3 q, V3 a, V3 b) {
    const V3 u = q - p, v = b - a, w = p - a;
    const double aa = dot(u, u), bb = dot(u, v), cc = dot(v, v), dd = dot(u, w), ee = dot(v, w);
    const double det = aa * cc - bb * bb;
    double s = det > aa * cc * 1e-14 ? clampD((bb * ee - cc * dd) / det, 0.0, 1.0) : 0;
    double t = (bb * s + ee) / cc;
    if (t < 0) {
        t = 0;
        s = clampD(-dd / aa, 0.0, 1.0);
    } else if (t > 1) {
        t = 1;
        s = clampD((bb - dd) / aa, 0.0, 1.0);
    }
    return norm2((w + u * s) - v * t);
}

HS_HD double panelDistance(const HostPanel &t, const HostPanel &s) {
    V3 a[3], b[3];
    for (int i = 0; i < 3; ++i) {
        a[i] = t.v[i] - t.v[0];
        b[i] = s.v[i] - t.v[0];
    }
    double d2 = INFINITY;
    for (int i = 0; i < 3; ++i) {
        d2 = minD(d2, pointTriangleD2(a[i], b));
        d2 = minD(d2, pointTriangleD2(b[i], a));
        for (int j = 0; j < 3; ++j)
            d2 = minD(d2, segmentD2(a[i], a[(i + 1) % 3], b[j], b[(j + 1) % 3]));
    }
    return sqrt(d2);
}

HS_HD bool panelsDisjoint(const HostPanel &t, const HostPanel &s) {
    return classifyNodes(t.nodes, s.nodes).topology == kDisjoint;
}

HS_HD bool isNearPair(const HostPanel &t, const HostPanel &s, double ratio) {
    if (ratio == 0 || !panelsDisjoint(t, s))
        return false;
    const double size = maxD(t.maxEdge, s.maxEdge);
    const double bound = ratio * size + t.maxEdge + s.maxEdge;
    if (norm2(t.centroid - s.centroid) >= bound * bound)
        return false;
    return panelDistance(t, s) < ratio * size;
}

// A test vertex nearly on the trial plane with the others on one side
// (pair_quadrature.cpp:329-340): the pair is integrated on projected patches.
HS_HD bool useProjection(const HostPanel &t, const HostPanel &s, double scale) {
    if (panelDistance(t, s) >= .025 * scale)
        return false;
    const double eps = 128 * kPlanEps * scale;
    double lo = INFINITY, hi = -lo;
    for (int i = 0; i < 3; ++i) {
        const double h = dot(t.v[i] - s.v[0], s.n);
        lo = minD(lo, h);
        hi = maxD(hi, h);
    }
    return (lo >= -eps && hi > eps) || (hi <= eps && lo < -eps);
}

// Child c of a sub-triangle's halving (0..2 at its corners, 3 the middle),
// vertices as midpoints of the parent's edges ab, bc, ca.
HS_HD void quarterChild(const Sub &s, int c, Sub &out) {
    const auto mid = [&](int e, double *m) {  // midpoint of edge e (v_e, v_e+1)
        const int f = e == 2 ? 0 : e + 1;
        for (int i = 0; i < 3; ++i)
            m[i] = (s.v[e][i] + s.v[f][i]) * .5;
    };
    if (c == 0) {
        for (int i = 0; i < 3; ++i)
            out.v[0][i] = s.v[0][i];
        mid(0, out.v[1]);
        mid(2, out.v[2]);
    } else if (c == 1) {
        mid(0, out.v[0]);
        for (int i = 0; i < 3; ++i)
            out.v[1][i] = s.v[1][i];
        mid(1, out.v[2]);
    } else if (c == 2) {
        mid(2, out.v[0]);
        mid(1, out.v[1]);
        for (int i = 0; i < 3; ++i)
            out.v[2][i] = s.v[2][i];
    } else {
        mid(0, out.v[0]);
        mid(1, out.v[1]);
        mid(2, out.v[2]);
    }
    out.fraction = s.fraction * .25;
}

HS_HD void quarter(const Sub &s, Sub *out) {
    for (int c = 0; c < 4; ++c)
        quarterChild(s, c, out[c]);
}

HS_HD double subDiameter(const HostPanel &p, const Sub &s, V3 origin) {
    const V3 off = p.v[0] - origin;
    V3 q[3];
    for (int i = 0; i < 3; ++i)
        q[i] = off + localPoint(p, s.v[i]);
    double d = norm2(q[0] - q[1]);
    d = maxD(d, norm2(q[1] - q[2]));
    d = maxD(d, norm2(q[2] - q[0]));
    return sqrt(d);
}

}  // namespace hsb
