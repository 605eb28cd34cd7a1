// Support octree and near/far partition of the fast-multipole form; the rules
// are those of makeSupportTree (fmm/support_tree.cpp:27-415), restated.
#include "fmm_tree.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>

namespace hsb {

bool FmmNode::leaf() const {
    return std::all_of(child.begin(), child.end(), [](uint32_t c) { return c == kNoNode; });
}

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

FmmBox emptyBox() { return {{kInf, kInf, kInf}, {-kInf, -kInf, -kInf}, 0.0}; }

void grow(FmmBox &a, const FmmBox &b) {
    for (int d = 0; d < 3; ++d) {
        a.lo[d] = std::min(a.lo[d], b.lo[d]);
        a.hi[d] = std::max(a.hi[d], b.hi[d]);
    }
    a.edge = std::max(a.edge, b.edge);
}

// Euclidean gap between two boxes (0 when they overlap).
double boxGap(const FmmBox &a, const FmmBox &b) {
    double g[3];
    for (int d = 0; d < 3; ++d)
        g[d] = std::max({0.0, a.lo[d] - b.hi[d], b.lo[d] - a.hi[d]});
    return std::hypot(g[0], g[1], g[2]);
}

double dist(const double *a, const double *b) { return std::hypot(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }

class TreeBuilder {
  public:
    TreeBuilder(const double *V, uint32_t N, const uint32_t *tri, uint32_t T, const FmmTreeSettings &s)
        : V_(V), N_(N), tri_(tri), T_(T), s_(s) {}

    FmmTree build() {
        // panel (flux) supports: bounds of the three vertices, anchor at the centroid
        panelBox_.resize(T_);
        anchorF_.resize(3 * size_t(T_));
        FmmBox all = emptyBox();
        for (uint32_t t = 0; t < T_; ++t) {
            FmmBox b = emptyBox();
            double edge = 0;
            for (int a = 0; a < 3; ++a) {
                const double *p = V_ + 3 * size_t(tri_[3 * t + a]), *q = V_ + 3 * size_t(tri_[3 * t + (a + 1) % 3]);
                for (int d = 0; d < 3; ++d) {
                    if (!std::isfinite(p[d]))
                        throw std::invalid_argument("Wideband support coordinates are not finite.");
                    b.lo[d] = std::min(b.lo[d], p[d]);
                    b.hi[d] = std::max(b.hi[d], p[d]);
                    anchorF_[3 * t + d] += p[d] / 3.0;
                }
                edge = std::max(edge, dist(p, q));
            }
            b.edge = edge;
            panelBox_[t] = b;
            grow(all, b);
        }
        // vertex (pressure) supports: the union of the incident panels
        incOffsets_.assign(N_ + 1, 0);
        for (size_t i = 0; i < 3 * size_t(T_); ++i)
            ++incOffsets_[tri_[i] + 1];
        for (uint32_t v = 0; v < N_; ++v)
            incOffsets_[v + 1] += incOffsets_[v];
        incPanel_.resize(3 * size_t(T_));
        std::vector<uint32_t> cursor(incOffsets_.begin(), incOffsets_.end() - 1);
        for (uint32_t t = 0; t < T_; ++t)
            for (int a = 0; a < 3; ++a)
                incPanel_[cursor[tri_[3 * t + a]]++] = t;
        vertexBox_.assign(N_, emptyBox());
        for (uint32_t v = 0; v < N_; ++v) {
            if (incOffsets_[v] == incOffsets_[v + 1])
                throw std::invalid_argument("Wideband pressure support has invalid incidences.");
            for (uint32_t j = incOffsets_[v]; j < incOffsets_[v + 1]; ++j)
                grow(vertexBox_[v], panelBox_[incPanel_[j]]);
        }
        tree_.pressureOrder.resize(N_);
        tree_.fluxOrder.resize(T_);
        for (uint32_t i = 0; i < N_; ++i)
            tree_.pressureOrder[i] = i;
        for (uint32_t i = 0; i < T_; ++i)
            tree_.fluxOrder[i] = i;
        tree_.pressureLeaf.assign(N_, kNoNode);
        tree_.fluxLeaf.assign(T_, kNoNode);
        double center[3], half = 0;
        for (int d = 0; d < 3; ++d) {
            center[d] = 0.5 * (all.lo[d] + all.hi[d]);
            half = std::max(half, 0.5 * (all.hi[d] - all.lo[d]));
        }
        if (!(half > 0) || !std::isfinite(half))
            throw std::invalid_argument("Wideband root bounds are invalid.");
        makeNode(center, std::nextafter(half, kInf), 0, kNoNode, 0, N_, 0, T_);
        // inner radii enclose the child balls (children follow their parent in the node list)
        for (size_t i = tree_.nodes.size(); i-- > 1;) {
            const FmmNode &c = tree_.nodes[i];
            FmmNode &p = tree_.nodes[c.parent];
            const double d = dist(c.center, p.center);
            if (c.countP)
                p.radiusP = std::max(p.radiusP, std::nextafter(d + c.radiusP, kInf));
            if (c.countF)
                p.radiusF = std::max(p.radiusF, std::nextafter(d + c.radiusF, kInf));
        }
        partition(0, 0, false, tree_.ppNear, tree_.ppFar);
        partition(0, 0, true, tree_.pfNear, tree_.pfFar);
        return std::move(tree_);
    }

  private:
    // Octant of an anchor relative to a cell centre: bit d set when coordinate d >= centre.
    static unsigned octant(const double *p, const double *c) {
        return unsigned(p[0] >= c[0]) | (unsigned(p[1] >= c[1]) << 1) | (unsigned(p[2] >= c[2]) << 2);
    }

    // Stable split of order[first, first + count) by octant; returns the 9 span boundaries.
    std::array<uint32_t, 9> split(std::vector<uint32_t> &order, bool flux, uint32_t first, uint32_t count,
                                  const double *c) {
        std::array<uint32_t, 9> off{};
        const auto anchor = [&](uint32_t id) { return flux ? &anchorF_[3 * size_t(id)] : V_ + 3 * size_t(id); };
        for (uint32_t i = first; i < first + count; ++i)
            ++off[octant(anchor(order[i]), c) + 1];
        off[0] = first;
        for (int i = 1; i < 9; ++i)
            off[i] += off[i - 1];
        std::array<uint32_t, 9> cur = off;
        std::vector<uint32_t> sorted(count);
        for (uint32_t i = first; i < first + count; ++i)
            sorted[cur[octant(anchor(order[i]), c)]++ - first] = order[i];
        std::copy(sorted.begin(), sorted.end(), order.begin() + first);
        return off;
    }

    double panelRadius(uint32_t t, const double *c) const {
        double r = 0;
        for (int a = 0; a < 3; ++a)
            r = std::max(r, dist(V_ + 3 * size_t(tri_[3 * t + a]), c));
        return r;
    }

    uint32_t makeNode(const double *center, double half, uint32_t level, uint32_t parent, uint32_t fp, uint32_t np,
                      uint32_t fq, uint32_t nq) {
        if (tree_.nodes.size() >= kNoNode)
            throw std::overflow_error("Wideband node index overflow.");
        FmmNode n{};
        std::copy(center, center + 3, n.center);
        n.half = half;
        n.level = level;
        n.parent = parent;
        n.child.fill(kNoNode);
        n.firstP = fp;
        n.countP = np;
        n.firstF = fq;
        n.countF = nq;
        n.boxP = emptyBox();
        n.boxF = emptyBox();
        for (uint32_t i = fp; i < fp + np; ++i)
            grow(n.boxP, vertexBox_[tree_.pressureOrder[i]]);
        for (uint32_t i = fq; i < fq + nq; ++i)
            grow(n.boxF, panelBox_[tree_.fluxOrder[i]]);
        const bool leaf = (np <= s_.leafCapacity && nq <= s_.leafCapacity) || level == s_.maximumDepth;
        if (leaf) {
            // complete-support balls: every vertex of every support panel
            double rp = 0, rq = 0;
            for (uint32_t i = fp; i < fp + np; ++i) {
                const uint32_t v = tree_.pressureOrder[i];
                for (uint32_t j = incOffsets_[v]; j < incOffsets_[v + 1]; ++j)
                    rp = std::max(rp, panelRadius(incPanel_[j], center));
            }
            for (uint32_t i = fq; i < fq + nq; ++i)
                rq = std::max(rq, panelRadius(tree_.fluxOrder[i], center));
            n.radiusP = np ? std::nextafter(rp, kInf) : 0.0;
            n.radiusF = nq ? std::nextafter(rq, kInf) : 0.0;
        }
        const uint32_t id = uint32_t(tree_.nodes.size());
        tree_.nodes.push_back(n);
        if (tree_.levels.size() <= level)
            tree_.levels.resize(level + 1);
        tree_.levels[level].push_back(id);
        if (leaf) {
            for (uint32_t i = fp; i < fp + np; ++i)
                tree_.pressureLeaf[tree_.pressureOrder[i]] = id;
            for (uint32_t i = fq; i < fq + nq; ++i)
                tree_.fluxLeaf[tree_.fluxOrder[i]] = id;
            return id;
        }
        const auto po = split(tree_.pressureOrder, false, fp, np, center);
        const auto qo = split(tree_.fluxOrder, true, fq, nq, center);
        for (unsigned o = 0; o < 8; ++o) {
            if (po[o] == po[o + 1] && qo[o] == qo[o + 1])
                continue;
            const double h = 0.5 * half;
            const double c[3] = {center[0] + ((o & 1) ? h : -h), center[1] + ((o & 2) ? h : -h),
                                 center[2] + ((o & 4) ? h : -h)};
            const uint32_t child = makeNode(c, h, level + 1, id, po[o], po[o + 1] - po[o], qo[o], qo[o + 1] - qo[o]);
            tree_.nodes[id].child[o] = child;
        }
        return id;
    }

    void partition(uint32_t ti, uint32_t si, bool flux, std::vector<FmmLink> &nearOut, std::vector<FmmLink> &farOut) {
        const FmmNode &t = tree_.nodes[ti], &s = tree_.nodes[si];
        const uint32_t ns = flux ? s.countF : s.countP;
        if (!t.countP || !ns)
            return;
        const FmmBox &sb = flux ? s.boxF : s.boxP;
        const double sr = flux ? s.radiusF : s.radiusP;
        const double gap = boxGap(t.boxP, sb);
        const bool far = t.level == s.level && gap > 0 && gap > s_.nearDistanceRatio * std::max(t.boxP.edge, sb.edge) &&
                         dist(t.center, s.center) > s_.separationRatio * (t.radiusP + sr);
        const bool tl = t.leaf(), sl = s.leaf();
        if (far || (tl && sl)) {
            (far ? farOut : nearOut).push_back({ti, si});
            return;
        }
        const std::array<uint32_t, 8> tc = t.child, sc = s.child;
        const uint32_t tLevel = t.level, sLevel = s.level;
        if (!tl && (sl || tLevel < sLevel)) {
            for (uint32_t c : tc)
                if (c != kNoNode)
                    partition(c, si, flux, nearOut, farOut);
        } else if (!sl && (tl || sLevel < tLevel)) {
            for (uint32_t c : sc)
                if (c != kNoNode)
                    partition(ti, c, flux, nearOut, farOut);
        } else {
            for (uint32_t a : tc)
                if (a != kNoNode)
                    for (uint32_t b : sc)
                        if (b != kNoNode)
                            partition(a, b, flux, nearOut, farOut);
        }
    }

    const double *V_;
    uint32_t N_;
    const uint32_t *tri_;
    uint32_t T_;
    FmmTreeSettings s_;
    std::vector<FmmBox> panelBox_, vertexBox_;
    std::vector<double> anchorF_ = {};
    std::vector<uint32_t> incOffsets_, incPanel_;
    FmmTree tree_;
};

}  // namespace

FmmTree buildSupportTree(const double *vertices, uint32_t N, const uint32_t *triangles, uint32_t T,
                         const FmmTreeSettings &settings) {
    if (!settings.leafCapacity || settings.maximumDepth > 30 || !std::isfinite(settings.separationRatio) ||
        settings.separationRatio <= 1 || !std::isfinite(settings.nearDistanceRatio) || settings.nearDistanceRatio < 0)
        throw std::invalid_argument("Wideband support tree settings are invalid.");
    if (!N || !T)
        throw std::invalid_argument("Wideband support geometry is empty or invalid.");
    TreeBuilder b(vertices, N, triangles, T, settings);
    return b.build();
}

}  // namespace hsb
