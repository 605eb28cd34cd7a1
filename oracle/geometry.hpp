// Test infrastructure only: the FP64 CPU oracle for the dense Burton-Miller
// solve. Nothing in the product links, imports or runs this directory.
//
// Geometry, quadrature rules and pair transforms restated from HornSculpt's
// galerkin module (file:line citations refer to the reference project tree).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <vector>

namespace oracle {

using cplx = std::complex<double>;

struct V3 {
    double x{}, y{}, z{};
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double norm2(V3 a) { return dot(a, a); }

// galerkin/space.hpp:11-26 — one flat triangle with its P1 data.
struct Panel {
    uint32_t nodes[3]{};
    V3 v[3];
    V3 centroid, normal;
    double area{}, maxEdge{};
    V3 grad[3], curl[3];
    uint32_t face{};
    uint8_t driven{};
};

// galerkin/space.hpp:33-42
struct Space {
    std::vector<V3> vertices;
    std::vector<Panel> panels;
    std::vector<size_t> incOffsets;
    std::vector<uint32_t> incPanels;
    std::vector<double> lumpedMass;
};

// galerkin/space.cpp:75-154: areas, unit normals, P1 gradients and surface
// curls (n x grad), lumped mass A/3 per incident vertex, incidence CSR.
inline Space buildSpace(const std::vector<V3> &vertices, const std::vector<std::array<uint32_t, 3>> &tris,
                        const std::vector<uint32_t> &faces, const std::vector<uint8_t> &driven) {
    if (vertices.empty() || tris.empty())
        throw std::invalid_argument("empty mesh");
    Space s;
    s.vertices = vertices;
    s.incOffsets.assign(vertices.size() + 1, 0);
    s.lumpedMass.assign(vertices.size(), 0.0);
    for (size_t t = 0; t < tris.size(); ++t) {
        Panel p;
        for (int i = 0; i < 3; ++i) {
            if (tris[t][i] >= vertices.size())
                throw std::invalid_argument("invalid vertex index");
            p.nodes[i] = tris[t][i];
            p.v[i] = vertices[tris[t][i]];
        }
        p.face = faces[t];
        p.driven = driven[t];
        const V3 ab = p.v[1] - p.v[0], ac = p.v[2] - p.v[0], bc = p.v[2] - p.v[1];
        const V3 av = cross(ab, ac);
        const double twice = std::hypot(av.x, av.y, av.z);
        p.maxEdge = std::max({std::hypot(ab.x, ab.y, ab.z), std::hypot(ac.x, ac.y, ac.z),
                              std::hypot(bc.x, bc.y, bc.z)});
        if (!(twice > 128.0 * std::numeric_limits<double>::epsilon() * p.maxEdge * p.maxEdge))
            throw std::invalid_argument("degenerate triangle");
        p.area = 0.5 * twice;
        p.normal = {av.x / twice, av.y / twice, av.z / twice};
        p.centroid = {p.v[0].x + (ab.x + ac.x) / 3.0, p.v[0].y + (ab.y + ac.y) / 3.0,
                      p.v[0].z + (ab.z + ac.z) / 3.0};
        const V3 opposite[3] = {bc, p.v[0] - p.v[2], ab};
        for (int i = 0; i < 3; ++i) {
            const V3 g = cross(p.normal, opposite[i]);
            p.grad[i] = {g.x / twice, g.y / twice, g.z / twice};
            p.curl[i] = cross(p.normal, p.grad[i]);
            ++s.incOffsets[p.nodes[i] + 1];
            s.lumpedMass[p.nodes[i]] += p.area / 3.0;
        }
        s.panels.push_back(p);
    }
    for (size_t v = 0; v < vertices.size(); ++v) {
        if (s.incOffsets[v + 1] == 0)
            throw std::invalid_argument("orphan vertex");
        s.incOffsets[v + 1] += s.incOffsets[v];
    }
    s.incPanels.resize(s.incOffsets.back());
    auto cursor = s.incOffsets;
    for (size_t t = 0; t < s.panels.size(); ++t)
        for (int i = 0; i < 3; ++i)
            s.incPanels[cursor[s.panels[t].nodes[i]]++] = static_cast<uint32_t>(t);
    return s;
}

struct GaussPoint {
    double x, w;
};
// galerkin/pair_quadrature.cpp:685-713: Gauss-Legendre nodes on [0,1] by
// Newton iteration on the three-term Legendre recurrence.
inline std::vector<GaussPoint> gauss01(unsigned n) {
    if (n < 2 || n > 20)
        throw std::invalid_argument("gauss order");
    std::vector<GaussPoint> r(n);
    for (unsigned i = 0; i < (n + 1) / 2; ++i) {
        double x = std::cos(M_PI * (double(i) + .75) / (double(n) + .5)), dp = 0;
        for (unsigned it = 0; it < 32; ++it) {
            double p0 = 1, p1 = x;
            for (unsigned d = 2; d <= n; ++d) {
                const double p = ((2 * d - 1) * x * p1 - (d - 1) * p0) / d;
                p0 = p1;
                p1 = p;
            }
            dp = n * (x * p1 - p0) / (x * x - 1);
            const double dx = p1 / dp;
            x -= dx;
            if (std::abs(dx) < 4 * std::numeric_limits<double>::epsilon())
                break;
        }
        const double w = 1 / ((1 - x * x) * dp * dp);
        r[i] = {(1 - x) * .5, w};
        r[n - 1 - i] = {(1 + x) * .5, w};
    }
    return r;
}

struct TriPoint {
    double b[3];
    double w;
};
// galerkin/pair_quadrature.cpp:715-769: Dunavant (1985) positive rules of
// degree 2/4/6/8 and collapsed tensor Gauss rules of degree 12/14 on the
// reference triangle (weights sum to 1/2).
inline std::vector<TriPoint> triangleRule(unsigned degree) {
    std::vector<TriPoint> r;
    if (degree == 12 || degree == 14) {
        const auto g = gauss01((degree + 2) / 2);
        for (const auto &u : g)
            for (const auto &v : g)
                r.push_back({{(1 - u.x) * (1 - v.x), u.x, (1 - u.x) * v.x}, u.w * v.w * (1 - u.x)});
        return r;
    }
    if (degree == 2) {
        r.push_back({{2.0 / 3, 1.0 / 6, 1.0 / 6}, 1.0 / 6});
        r.push_back({{1.0 / 6, 2.0 / 3, 1.0 / 6}, 1.0 / 6});
        r.push_back({{1.0 / 6, 1.0 / 6, 2.0 / 3}, 1.0 / 6});
        return r;
    }
    auto orbit3 = [&](double a, double b, double w) {
        for (int i = 0; i < 3; ++i) {
            TriPoint p{{a, a, a}, w};
            p.b[i] = b;
            r.push_back(p);
        }
    };
    auto orbit6 = [&](double a, double b, double c, double w) {
        const double c3[3] = {a, b, c};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                if (i != j)
                    r.push_back({{c3[i], c3[j], c3[3 - i - j]}, w});
    };
    if (degree == 4) {
        orbit3(.445948490915965, .108103018168070, .1116907948390055);
        orbit3(.091576213509771, .816847572980459, .054975871827661);
    } else if (degree == 6) {
        orbit3(.249286745170910, .501426509658179, .0583931378631895);
        orbit3(.063089014491502, .873821971016996, .0254224531851035);
        orbit6(.310352451033785, .636502499121399, .053145049844816, .041425537809187);
    } else if (degree == 8) {
        r.push_back({{1.0 / 3, 1.0 / 3, 1.0 / 3}, .0721578038388935});
        orbit3(.459292588292723, .081414823414554, .0475458171336425);
        orbit3(.170569307751760, .658861384496480, .051608685267359);
        orbit3(.050547228317031, .898905543365938, .016229248811599);
        orbit6(.263112829634638, .728492392955404, .008394777409958, .0136151570872175);
    } else
        throw std::invalid_argument("triangle rule degree");
    return r;
}

enum Topology : uint8_t { Disjoint = 0, SharedVertex = 1, SharedEdge = 2, Coincident = 3 };
struct Permutation {
    uint8_t topology{Disjoint};
    uint8_t test[3]{0, 1, 2}, trial[3]{0, 1, 2};
};
// galerkin/pair_quadrature.hpp:57-97: shared node ids in ascending order
// first, then the remaining local indices.
inline Permutation classify(const uint32_t *a, const uint32_t *b) {
    Permutation r;
    uint32_t shared[3];
    unsigned n = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (a[i] == b[j] && n < 3)
                shared[n++] = a[i];
    for (unsigned i = 1; i < n; ++i)
        for (unsigned j = i; j > 0 && shared[j] < shared[j - 1]; --j)
            std::swap(shared[j], shared[j - 1]);
    r.topology = n == 3 ? Coincident : n == 2 ? SharedEdge : n == 1 ? SharedVertex : Disjoint;
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
            sa |= a[i] == shared[s];
            sb |= b[i] == shared[s];
        }
        if (!sa)
            r.test[tx++] = uint8_t(i);
        if (!sb)
            r.trial[ty++] = uint8_t(i);
    }
    return r;
}

struct PairPoint {
    double t[3]{}, s[3]{};
    double w{};
};
inline unsigned sectorCount(uint8_t topo) {
    return topo == Coincident ? 6 : topo == SharedEdge ? 5 : topo == SharedVertex ? 2 : 1;
}
// galerkin/pair_quadrature.hpp:121-204: Sauter-Schwab / Duffy sector maps of
// (r,u,v,w) in [0,1]^4 to reference-triangle pairs, with the 4-D Jacobian.
// The sector formulas follow Sauter & Schwab's published transformations.
inline PairPoint sauterSchwab(uint8_t topo, unsigned sector, double r, double u, double v, double w) {
    double xs{}, xt{}, ys{}, yt{}, jac{};
    if (topo == Disjoint) {
        xs = r; xt = r * u; ys = v; yt = v * w; jac = r * v;
    } else if (topo == SharedVertex) {
        xs = r; xt = r * u; ys = r * v; yt = r * v * w; jac = r * r * r * v;
        if (sector == 1) { std::swap(xs, ys); std::swap(xt, yt); }
    } else if (topo == SharedEdge) {
        jac = r * r * r * u * u;
        switch (sector) {
        case 0: xs = r; xt = r * u * w; ys = r * (1 - u * v); yt = r * u * (1 - v); break;
        case 1: xs = r; xt = r * u; ys = r * (1 - u * v * w); yt = r * u * v * (1 - w); jac *= v; break;
        case 2: xs = r * (1 - u * v); xt = r * u * (1 - v); ys = r; yt = r * u * v * w; jac *= v; break;
        case 3: xs = r * (1 - u * v * w); xt = r * u * v * (1 - w); ys = r; yt = r * u; jac *= v; break;
        default: xs = r * (1 - u * v * w); xt = r * u * (1 - v * w); ys = r; yt = r * u * v; jac *= v; break;
        }
    } else {
        jac = r * r * r * u * u * v;
        switch (sector % 3) {
        case 0: xs = r; xt = r * (1 - u + u * v); ys = r * (1 - u * v * w); yt = r * (1 - u); break;
        case 1: xs = r; xt = r * u * (1 - v + v * w); ys = r * (1 - u * v); yt = r * u * (1 - v); break;
        default: xs = r * (1 - u * v * w); xt = r * u * (1 - v * w); ys = r; yt = r * u * (1 - v); break;
        }
        if (sector >= 3) { std::swap(xs, ys); std::swap(xt, yt); }
    }
    PairPoint p;
    p.t[0] = 1 - xs; p.t[1] = xs - xt; p.t[2] = xt;
    p.s[0] = 1 - ys; p.s[1] = ys - yt; p.s[2] = yt;
    p.w = jac;
    return p;
}
// galerkin/pair_quadrature.hpp:206-215: canonical local order back to the
// panels' original local node order.
inline PairPoint permute(const PairPoint &p, const Permutation &perm) {
    PairPoint r;
    r.w = p.w;
    for (int i = 0; i < 3; ++i) {
        r.t[perm.test[i]] = p.t[i];
        r.s[perm.trial[i]] = p.s[i];
    }
    return r;
}

inline V3 localPoint(const Panel &p, const double *b) {
    return (p.v[1] - p.v[0]) * b[1] + (p.v[2] - p.v[0]) * b[2];
}
// galerkin/pair_quadrature.cpp:34-41: panel-origin difference first, then
// the local offsets, so that remote placements keep their small gaps.
inline V3 pairDelta(const Panel &t, const double *bt, const Panel &s, const double *bs) {
    return (t.v[0] - s.v[0]) + (localPoint(t, bt) - localPoint(s, bs));
}

}  // namespace oracle
