// Support octree, near/far partition and translation plan of the fast-multipole
// form (host side, once per mesh).
//
// The tree follows makeSupportTree (fmm/support_tree.cpp:407): P1 pressure
// supports are vertex stars anchored at the vertex, DP0 flux supports are
// panels anchored at the centroid; anchors select dyadic cells of a cube
// around all support bounds, a cell is a leaf when it holds at most
// `leafCapacity` supports of each kind (or at `maximumDepth`), and a node's
// radius about its cell centre encloses every vertex of its complete supports
// (leaves) or every child ball (inner nodes). Two nodes interact in the far
// field when they are on the same level, their support boxes have a gap
// larger than `nearDistanceRatio` longest panel edges, and their centre
// distance exceeds `separationRatio` times the sum of their radii
// (support_tree.cpp:340-351); leaf pairs that fail this are near, the rest
// recurse into children (:352-373).
#pragma once

#include <array>
#include <cstdint>
#include <vector>

namespace hsb {

constexpr uint32_t kNoNode = 0xffffffffu;

struct FmmBox {
    double lo[3], hi[3], edge;  // axis-aligned bounds and longest panel edge of the supports
};

struct FmmNode {
    double center[3];
    double half;
    uint32_t level, parent;
    std::array<uint32_t, 8> child;
    uint32_t firstP, countP, firstF, countF;  // spans of pressureOrder / fluxOrder
    FmmBox boxP, boxF;
    double radiusP, radiusF;
    bool leaf() const;
};

struct FmmLink {
    uint32_t target, source;
};

struct FmmTreeSettings {
    uint32_t leafCapacity = 32, maximumDepth = 20;
    double separationRatio = 1.5, nearDistanceRatio = 2.0;
};

struct FmmTree {
    std::vector<FmmNode> nodes;
    std::vector<uint32_t> pressureOrder, fluxOrder;  // supports sorted by leaf
    std::vector<uint32_t> pressureLeaf, fluxLeaf;    // leaf of each support
    std::vector<std::vector<uint32_t>> levels;       // node ids per level
    // Near links join leaves (possibly of different levels); far links join
    // nodes of one level. pp: pressure x pressure (the operator), pf: pressure
    // x flux (the right-hand side).
    std::vector<FmmLink> ppNear, ppFar, pfNear, pfFar;
};

// vertices N x 3, triangles T x 3 (vertex ids). Throws std::invalid_argument
// for empty or non-finite input and invalid settings.
FmmTree buildSupportTree(const double *vertices, uint32_t N, const uint32_t *triangles, uint32_t T,
                         const FmmTreeSettings &settings);

}  // namespace hsb
