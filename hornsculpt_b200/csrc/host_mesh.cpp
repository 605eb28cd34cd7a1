// Host-side mesh validation, Galerkin space and quadrature rules.
#include "host_mesh.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <map>
#include <numeric>
#include <unordered_map>

namespace hsb {
namespace {

double len(V3 a) { return std::hypot(a.x, a.y, a.z); }

struct EdgeUse {
    int count = 0, orientation = 0;
};

// Separating-axis test of two triangles with no common vertex: the 2 face
// normals, the 9 edge-edge cross products and the 6 in-plane edge normals
// (the last separate coplanar triangles, for which every other axis is the
// common normal). Touching within `eps` counts as intersecting.
bool trianglesIntersect(const V3 *a, const V3 *b, double eps) {
    auto separated = [&](V3 axis) {
        const double l = len(axis);
        if (!(l > 0))
            return false;
        axis = axis * (1 / l);
        double amin = INFINITY, amax = -INFINITY, bmin = INFINITY, bmax = -INFINITY;
        for (int i = 0; i < 3; ++i) {
            const double pa = dot(a[i], axis), pb = dot(b[i], axis);
            amin = std::min(amin, pa);
            amax = std::max(amax, pa);
            bmin = std::min(bmin, pb);
            bmax = std::max(bmax, pb);
        }
        return amax < bmin - eps || bmax < amin - eps;
    };
    const V3 ea[3] = {a[1] - a[0], a[2] - a[1], a[0] - a[2]};
    const V3 eb[3] = {b[1] - b[0], b[2] - b[1], b[0] - b[2]};
    const V3 na = cross(ea[0], ea[1]), nb = cross(eb[0], eb[1]);
    if (separated(na) || separated(nb))
        return false;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (separated(cross(ea[i], eb[j])))
                return false;
    for (int i = 0; i < 3; ++i)
        if (separated(cross(na, ea[i])) || separated(cross(nb, eb[i])))
            return false;
    return true;
}

int root(std::vector<uint32_t> &parent, uint32_t v) {
    while (parent[v] != v) {
        parent[v] = parent[parent[v]];
        v = parent[v];
    }
    return int(v);
}

}  // namespace

void validateExteriorSurface(const MeshInput &mesh) {
    const size_t nv = mesh.vertices.size(), nt = mesh.faces.size();
    if (!nv || !nt)
        throw InvalidArgument("The surface mesh is empty.");
    V3 lo = mesh.vertices[0], hi = lo;
    for (const V3 &p : mesh.vertices) {
        if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.z))
            throw InvalidArgument("BEM mesh coordinates are not finite.");
        lo = {std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
        hi = {std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
    }
    const double areaTol = norm2(hi - lo) * 1e-14;
    std::map<std::pair<uint32_t, uint32_t>, EdgeUse> edges;
    std::map<std::array<uint32_t, 3>, int> unique;
    std::vector<std::vector<uint32_t>> vertexTris(nv);
    for (size_t t = 0; t < nt; ++t) {
        const uint32_t *tri = &mesh.triangles[3 * t];
        for (int i = 0; i < 3; ++i)
            if (tri[i] >= nv)
                throw InvalidArgument("Triangle index outside vertex array.");
        std::array<uint32_t, 3> key{tri[0], tri[1], tri[2]};
        std::sort(key.begin(), key.end());
        if (++unique[key] > 1)
            throw InvalidArgument("The mesh contains duplicate triangles.");
        const V3 a = mesh.vertices[tri[0]], b = mesh.vertices[tri[1]], c = mesh.vertices[tri[2]];
        if (len(cross(b - a, c - a)) <= areaTol || tri[0] == tri[1] || tri[1] == tri[2] || tri[0] == tri[2])
            throw InvalidArgument("BEM requires a closed, outward-oriented, non-intersecting mesh.");
        for (int j = 0; j < 3; ++j) {
            const uint32_t i0 = tri[j], i1 = tri[(j + 1) % 3];
            auto &use = edges[{std::min(i0, i1), std::max(i0, i1)}];
            ++use.count;
            use.orientation += i0 < i1 ? 1 : -1;
            vertexTris[tri[j]].push_back(uint32_t(t));
        }
    }
    for (const auto &[e, use] : edges)
        if (use.count != 2 || use.orientation != 0)
            throw InvalidArgument("BEM requires a closed, outward-oriented, non-intersecting mesh.");
    // Manifold vertices: the triangles around each vertex form one edge-connected fan.
    for (size_t v = 0; v < nv; ++v) {
        const auto &fan = vertexTris[v];
        if (fan.empty())
            throw InvalidArgument("Galerkin mesh contains an orphan pressure vertex.");
        std::vector<uint32_t> parent(fan.size());
        std::iota(parent.begin(), parent.end(), 0u);
        std::map<uint32_t, uint32_t> otherToFan;  // neighbour vertex -> first fan triangle using edge (v, other)
        for (uint32_t f = 0; f < fan.size(); ++f) {
            const uint32_t *tri = &mesh.triangles[3 * fan[f]];
            for (int j = 0; j < 3; ++j) {
                if (tri[j] == v)
                    continue;
                const auto [it, inserted] = otherToFan.emplace(tri[j], f);
                if (!inserted)
                    parent[root(parent, f)] = uint32_t(root(parent, it->second));
            }
        }
        for (uint32_t f = 1; f < fan.size(); ++f)
            if (root(parent, f) != root(parent, 0))
                throw InvalidArgument("BEM requires a closed, outward-oriented, non-intersecting mesh.");
    }
    // Self-intersections between triangles without a common vertex
    // (sweep-and-prune on x, then separating axes).
    struct Box {
        double lo[3], hi[3];
        uint32_t t;
    };
    std::vector<Box> boxes(nt);
    double maxEdge = 0;
    for (size_t t = 0; t < nt; ++t) {
        Box b;
        b.t = uint32_t(t);
        for (int k = 0; k < 3; ++k) {
            b.lo[k] = INFINITY;
            b.hi[k] = -INFINITY;
        }
        for (int j = 0; j < 3; ++j) {
            const V3 p = mesh.vertices[mesh.triangles[3 * t + j]];
            const double c[3] = {p.x, p.y, p.z};
            for (int k = 0; k < 3; ++k) {
                b.lo[k] = std::min(b.lo[k], c[k]);
                b.hi[k] = std::max(b.hi[k], c[k]);
            }
            maxEdge = std::max(maxEdge, len(p - mesh.vertices[mesh.triangles[3 * t + (j + 1) % 3]]));
        }
        boxes[t] = b;
    }
    std::sort(boxes.begin(), boxes.end(), [](const Box &a, const Box &b) { return a.lo[0] < b.lo[0]; });
    const double eps = 1e-12 * std::max(maxEdge, std::sqrt(norm2(hi - lo)));
    for (size_t i = 0; i < nt; ++i)
        for (size_t j = i + 1; j < nt && boxes[j].lo[0] <= boxes[i].hi[0] + eps; ++j) {
            const Box &a = boxes[i], &b = boxes[j];
            if (a.lo[1] > b.hi[1] + eps || b.lo[1] > a.hi[1] + eps || a.lo[2] > b.hi[2] + eps || b.lo[2] > a.hi[2] + eps)
                continue;
            const uint32_t *ta = &mesh.triangles[3 * a.t], *tb = &mesh.triangles[3 * b.t];
            bool sharesVertex = false;
            for (int x = 0; x < 3; ++x)
                for (int y = 0; y < 3; ++y)
                    sharesVertex = sharesVertex || ta[x] == tb[y];
            if (sharesVertex)
                continue;
            const V3 pa[3] = {mesh.vertices[ta[0]], mesh.vertices[ta[1]], mesh.vertices[ta[2]]};
            const V3 pb[3] = {mesh.vertices[tb[0]], mesh.vertices[tb[1]], mesh.vertices[tb[2]]};
            if (trianglesIntersect(pa, pb, eps))
                throw InvalidArgument("BEM requires a closed, outward-oriented, non-intersecting mesh.");
        }
    // Components: positive volume each (outward winding), none nested.
    std::vector<uint32_t> parent(nv);
    std::iota(parent.begin(), parent.end(), 0u);
    for (size_t t = 0; t < nt; ++t) {
        const uint32_t *tri = &mesh.triangles[3 * t];
        const int first = root(parent, tri[0]);
        for (int j = 1; j < 3; ++j)
            parent[root(parent, tri[j])] = uint32_t(first);
    }
    std::unordered_map<int, std::vector<uint32_t>> comps;
    for (size_t t = 0; t < nt; ++t)
        comps[root(parent, mesh.triangles[3 * t])].push_back(uint32_t(t));
    struct Comp {
        std::vector<uint32_t> tris;
        V3 lo, hi;
    };
    std::vector<Comp> list;
    for (auto &[r, tris] : comps) {
        Comp c{tris, mesh.vertices[mesh.triangles[3 * tris[0]]], mesh.vertices[mesh.triangles[3 * tris[0]]]};
        for (auto t : tris)
            for (int j = 0; j < 3; ++j) {
                const V3 p = mesh.vertices[mesh.triangles[3 * t + j]];
                c.lo = {std::min(c.lo.x, p.x), std::min(c.lo.y, p.y), std::min(c.lo.z, p.z)};
                c.hi = {std::max(c.hi.x, p.x), std::max(c.hi.y, p.y), std::max(c.hi.z, p.z)};
            }
        double vol = 0, comp = 0;
        for (auto t : tris) {
            const V3 a = mesh.vertices[mesh.triangles[3 * t]] - c.lo, b = mesh.vertices[mesh.triangles[3 * t + 1]] - c.lo,
                     d = mesh.vertices[mesh.triangles[3 * t + 2]] - c.lo;
            const double y = dot(a, cross(b, d)) / 6 - comp, s = vol + y;
            comp = (s - vol) - y;
            vol = s;
        }
        if (!(vol > 0) || !std::isfinite(vol))
            throw InvalidArgument("Every exterior surface component must have outward winding.");
        list.push_back(std::move(c));
    }
    for (size_t inner = 0; inner < list.size(); ++inner) {
        const V3 q = mesh.vertices[mesh.triangles[3 * list[inner].tris[0]]];
        for (size_t outer = 0; outer < list.size(); ++outer) {
            if (inner == outer)
                continue;
            const Comp &c = list[outer];
            if (q.x < c.lo.x || q.x > c.hi.x || q.y < c.lo.y || q.y > c.hi.y || q.z < c.lo.z || q.z > c.hi.z)
                continue;
            double angle = 0;
            for (auto t : c.tris) {
                V3 r[3];
                for (int j = 0; j < 3; ++j) {
                    r[j] = mesh.vertices[mesh.triangles[3 * t + j]] - q;
                    r[j] = r[j] * (1 / len(r[j]));
                }
                angle += 2 * std::atan2(dot(r[0], cross(r[1], r[2])), 1 + dot(r[0], r[1]) + dot(r[1], r[2]) + dot(r[2], r[0]));
            }
            if (std::abs(angle) > 2 * M_PI)
                throw InvalidArgument("Nested surface components and sealed air cavities are not supported by exterior BEM.");
        }
    }
}

Space buildSpace(const MeshInput &mesh) {
    const size_t nv = mesh.vertices.size(), nt = mesh.faces.size();
    if (!nv || !nt)
        throw InvalidArgument("Galerkin space requires a nonempty surface mesh.");
    if (nv > std::numeric_limits<uint32_t>::max() || nt > std::numeric_limits<uint32_t>::max())
        throw InvalidArgument("Galerkin mesh exceeds the 32-bit panel index limit.");
    Space s;
    s.vertices = mesh.vertices;
    s.incOffsets.assign(nv + 1, 0);
    s.lumpedMass.assign(nv, 0);
    s.panels.resize(nt);
    double comp = 0;
    for (size_t t = 0; t < nt; ++t) {
        HostPanel &p = s.panels[t];
        for (int i = 0; i < 3; ++i) {
            p.nodes[i] = mesh.triangles[3 * t + i];
            if (p.nodes[i] >= nv)
                throw InvalidArgument("Galerkin triangle has an invalid vertex index.");
            p.v[i] = mesh.vertices[p.nodes[i]];
        }
        p.face = mesh.faces[t];
        p.driven = mesh.driven[t];
        const V3 ab = p.v[1] - p.v[0], ac = p.v[2] - p.v[0], bc = p.v[2] - p.v[1];
        const V3 av = cross(ab, ac);
        const double twice = len(av);
        p.maxEdge = std::max({len(ab), len(ac), len(bc)});
        if (!std::isfinite(twice) || !std::isfinite(p.maxEdge) ||
            !(twice > 128.0 * std::numeric_limits<double>::epsilon() * p.maxEdge * p.maxEdge))
            throw InvalidArgument("Galerkin triangle is degenerate or numerically unresolved.");
        p.area = 0.5 * twice;
        p.n = V3{av.x / twice, av.y / twice, av.z / twice};
        p.centroid = V3{p.v[0].x + (ab.x + ac.x) / 3.0, p.v[0].y + (ab.y + ac.y) / 3.0, p.v[0].z + (ab.z + ac.z) / 3.0};
        const V3 opposite[3] = {bc, p.v[0] - p.v[2], ab};
        for (int i = 0; i < 3; ++i) {
            const V3 g = cross(p.n, opposite[i]);
            p.grad[i] = V3{g.x / twice, g.y / twice, g.z / twice};
            p.curl[i] = cross(p.n, p.grad[i]);
            ++s.incOffsets[p.nodes[i] + 1];
            s.lumpedMass[p.nodes[i]] += p.area / 3.0;
        }
        const double y = p.area - comp, sum = s.surfaceArea + y;
        comp = (sum - s.surfaceArea) - y;
        s.surfaceArea = sum;
    }
    for (size_t v = 0; v < nv; ++v) {
        if (s.incOffsets[v + 1] == 0)
            throw InvalidArgument("Galerkin mesh contains an orphan pressure vertex.");
        s.incOffsets[v + 1] += s.incOffsets[v];
    }
    s.incPanel.resize(s.incOffsets.back());
    s.incLocal.resize(s.incOffsets.back());
    std::vector<uint32_t> cursor(s.incOffsets.begin(), s.incOffsets.end() - 1);
    for (size_t t = 0; t < nt; ++t)
        for (int i = 0; i < 3; ++i) {
            const uint32_t slot = cursor[s.panels[t].nodes[i]]++;
            s.incPanel[slot] = uint32_t(t);
            s.incLocal[slot] = uint8_t(i);
        }
    return s;
}

std::vector<GaussPoint> gaussLegendre01(unsigned n) {
    if (n < 2 || n > 20)
        throw InvalidArgument("Gauss order must be between 2 and 20.");
    std::vector<GaussPoint> r(n);
    for (unsigned i = 0; i < (n + 1) / 2; ++i) {
        double x = std::cos(M_PI * (double(i) + .75) / (double(n) + .5)), dp = 0;
        for (unsigned it = 0;; ++it) {
            double p0 = 1, p1 = x;
            for (unsigned d = 2; d <= n; ++d) {
                const double p = ((2 * d - 1) * x * p1 - (d - 1) * p0) / d;
                p0 = p1;
                p1 = p;
            }
            dp = n * (x * p1 - p0) / (x * x - 1);
            const double step = p1 / dp;
            x -= step;
            if (std::abs(step) < 4 * std::numeric_limits<double>::epsilon())
                break;
            if (it == 31)
                throw NumericError("Gauss-Legendre roots did not converge.");
        }
        const double w = 1 / ((1 - x * x) * dp * dp);
        r[i] = {(1 - x) * .5, w};
        r[n - 1 - i] = {(1 + x) * .5, w};
    }
    return r;
}

std::vector<TriPoint> triangleRule(unsigned degree) {
    std::vector<TriPoint> r;
    if (degree == 12 || degree == 14) {
        const auto g = gaussLegendre01((degree + 2) / 2);
        for (const auto &u : g)
            for (const auto &v : g)
                r.push_back({{(1 - u.x) * (1 - v.x), u.x, (1 - u.x) * v.x}, u.w * v.w * (1 - u.x)});
        return r;
    }
    if (degree == 2) {
        for (int i = 0; i < 3; ++i) {
            TriPoint p{{1.0 / 6, 1.0 / 6, 1.0 / 6}, 1.0 / 6};
            p.b[i] = 2.0 / 3;
            r.push_back(p);
        }
        return r;
    }
    // Dunavant (1985) symmetric orbits: (a,a,b) in 3 positions, (a,b,c) in 6.
    const auto orbit3 = [&](double a, double b, double w) {
        for (int i = 0; i < 3; ++i) {
            TriPoint p{{a, a, a}, w};
            p.b[i] = b;
            r.push_back(p);
        }
    };
    const auto orbit6 = [&](double a, double b, double c, double w) {
        const double v[3] = {a, b, c};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                if (i != j)
                    r.push_back({{v[i], v[j], v[3 - i - j]}, w});
    };
    switch (degree) {
    case 4:
        orbit3(.445948490915965, .108103018168070, .1116907948390055);
        orbit3(.091576213509771, .816847572980459, .054975871827661);
        break;
    case 6:
        orbit3(.249286745170910, .501426509658179, .0583931378631895);
        orbit3(.063089014491502, .873821971016996, .0254224531851035);
        orbit6(.310352451033785, .636502499121399, .053145049844816, .041425537809187);
        break;
    case 8:
        r.push_back({{1.0 / 3, 1.0 / 3, 1.0 / 3}, .0721578038388935});
        orbit3(.459292588292723, .081414823414554, .0475458171336425);
        orbit3(.170569307751760, .658861384496480, .051608685267359);
        orbit3(.050547228317031, .898905543365938, .016229248811599);
        orbit6(.263112829634638, .728492392955404, .008394777409958, .0136151570872175);
        break;
    default:
        throw InvalidArgument("Triangle quadrature degree must be 2, 4, 6, 8, 12 or 14.");
    }
    return r;
}

}  // namespace hsb
