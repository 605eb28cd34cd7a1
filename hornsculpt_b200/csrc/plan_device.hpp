// Interaction planning on the GPU (the reference plans on host threads,
// modules/bem/galerkin/interaction_plan.cpp:156-504 with the adaptive pair
// rule of pair_quadrature.cpp:329-575 and the embedded-rule estimator of
// pair_quadrature.cpp:143-226, 644-683).
//
// The device decides, for every candidate (or, in the all-pairs mode, every)
// panel pair, whether it needs an adaptive rule, and runs the largest-error
// refinement of tensor-rule pairs with one warp per pair. The plan must equal
// the host planner's bit for bit, and the host's decisions compare error
// estimates that carry glibc's rounding. The device therefore bounds, for
// every estimate, how far its value can be from the host's, and a pair for
// which any comparison falls inside that bound (a tie, a termination test at
// the threshold, an order of two leaves), that overflows the device arena, or
// that raises an error is handed to the host planner's code, as are the pairs
// integrated on projected patches. Every other pair's patch list is exact:
// the patches are sub-triangles built by halving, identical on both sides.
#pragma once

#include "planner.hpp"

#include <cuda_runtime.h>

namespace hsb {

struct DevicePlanStats {
    size_t devicePairs{};      // pairs refined on the device
    size_t projectedPairs{};   // pairs with projected patches (host)
    size_t flaggedPairs{};     // device pairs handed back to the host
    size_t wholePanelPairs{};  // all-pairs mode: single whole-panel rules decided on the device
    size_t resolvedPairs{};    // device pairs whose patch order the host settled by its own estimates
    unsigned long long samples{};  // kernel samples the refinement evaluated (both rules of every estimate)
    double refineKernelMs{};       // CUDA-event time of the refinement launches (root pre-pass included)
    size_t rootSettledPairs{};     // all-pairs mode: pairs the root pre-pass settled
    double deviceMs{}, hostMs{};
    // frame (validation, bounds, touching jobs, candidates), classification,
    // refinement, readback, host part (runs, host pairs, flattening)
    double phaseMs[5]{};
    // the host part: ordering runs, host pairs, flattening, patch fill, near CSR
    double hostPhaseMs[5]{};
};

// The plan of makePlan, with the adaptive pairs refined on the current CUDA
// device (stream `stream`). `emulate` runs the device algorithm on the host
// instead (one lane per warp; a test hook that needs no GPU).
Plan makePlanOnDevice(const Space &space, const PlanSettings &settings, double maxK, cudaStream_t stream,
                      const volatile int32_t *cancel, DevicePlanStats *stats, bool emulate = false);

}  // namespace hsb
