// Host interaction plan for dense assembly: touching jobs, adaptive
// near-pair patches and the all-pairs whole-panel degree table
// (modules/bem/galerkin/interaction_plan.hpp:25-71).
#pragma once

#include "host_mesh.hpp"

#include <memory>
#include <new>
#include <type_traits>
#include <utility>
#include <vector>

namespace hsb {

// Allocator that leaves elements default-initialised (for Patch: uninitialised)
// when a vector grows by resize: a plan's patch array is sized once and then
// filled in parallel, so zeroing hundreds of megabytes on one thread first
// would only cost time.
template <class T> struct UninitAllocator : std::allocator<T> {
    using value_type = T;
    template <class U> struct rebind {
        using other = UninitAllocator<U>;
    };
    UninitAllocator() noexcept = default;
    template <class U> UninitAllocator(const UninitAllocator<U> &) noexcept {}
    template <class U> void construct(U *p) noexcept(std::is_nothrow_default_constructible_v<U>) {
        ::new (static_cast<void *>(p)) U;
    }
    template <class U, class... Args> void construct(U *p, Args &&...args) {
        ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
    }
};
template <class T, class U> bool operator==(const UninitAllocator<T> &, const UninitAllocator<U> &) { return true; }
template <class T, class U> bool operator!=(const UninitAllocator<T> &, const UninitAllocator<U> &) { return false; }

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
    std::vector<Patch, UninitAllocator<Patch>> patches;
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

// One pair's adaptive rule: patches in the reference's output order (patches
// at the depth limit first, then the rest by decreasing error estimate).
struct PairRule {
    std::vector<Patch> patches;
    unsigned maxDepth{};
    double relError{};
};

// The frequency-independent frame of a plan: validated settings, panel
// bounds, the all-pairs switch (interaction_plan.cpp:186-196), touching jobs
// and, outside the all-pairs mode, the grid candidates sorted by (first,
// second).
struct PlanFrame {
    Plan plan;
    std::vector<Bounds> bounds;
    bool allPairs{};
    std::vector<std::pair<uint32_t, uint32_t>> candidates;
};

Bounds makeBounds(const HostPanel &p);
PlanFrame beginPlan(const Space &space, const PlanSettings &settings, double maxK);
// Appends one pair's rule in flattening order: a single depth-0 tensor patch
// becomes a whole-panel degree in the all-pairs mode, anything else a near job
// in both orientations.
void appendPairRule(Plan &plan, bool allPairs, uint32_t first, uint32_t second, const Patch *patches, uint32_t count,
                    unsigned maxDepth, double relError);
// Sorts the near jobs by (test, trial) and builds the near CSR.
void finishPlan(Plan &plan, size_t triangleCount);
// The host planner's adaptive refinement of the listed pairs (first < second,
// pairs known to need it), on host threads; errors carry the host planner's
// messages.
std::vector<PairRule> planPairsOnHost(const Space &space, const PlanSettings &settings, double maxK,
                                      const std::vector<std::pair<uint32_t, uint32_t>> &pairs, unsigned threads,
                                      const volatile int32_t *cancel);
// The host planner's embedded-rule error estimate of one tensor patch of the
// pair (t, s), bit for bit the value its refinement compares.
double hostPatchError(const HostPanel &t, const HostPanel &s, const Patch &patch, double k);
// Parallel over host threads (at most `threads`, 0 = hardware concurrency).
// The result does not depend on the thread count.
Plan makePlan(const Space &space, const PlanSettings &settings, double maxK, unsigned threads,
              const volatile int32_t *cancel);

}  // namespace hsb
