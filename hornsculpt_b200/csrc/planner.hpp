// Host interaction plan for dense assembly: touching jobs, adaptive
// near-pair patches and the all-pairs whole-panel degree table
// (modules/bem/galerkin/interaction_plan.hpp:25-71).
#pragma once

#include "host_mesh.hpp"

#include <vector>

namespace hsb {

struct TouchJob {
    uint32_t test, trial;
    Permutation perm;
};
struct NearJob {
    uint32_t test, trial, first, count, swap;
};
struct Plan {
    std::vector<TouchJob> touching;           // ordered (test, trial), self and both directions
    std::vector<NearJob> near;                // ordered near jobs sorted by (test, trial)
    std::vector<Patch> patches;
    std::vector<uint8_t> wholePanelDegrees;   // all-pairs mode only: unordered pair -> 8/14
    std::vector<uint32_t> nearOffsets, nearTrials;
    unsigned maxDepth{};
    double maxRelError{};
};

struct PlanSettings {
    unsigned regularOrder{4}, singularOrder{4};
    double nearRatio{1.0}, tol{1e-4};
    unsigned maxDepth{6};
};

Bounds makeBounds(const HostPanel &p);
// Parallel over host threads (at most `threads`, 0 = hardware concurrency).
// The result does not depend on the thread count.
Plan makePlan(const Space &space, const PlanSettings &settings, double maxK, unsigned threads,
              const volatile int32_t *cancel);

}  // namespace hsb
