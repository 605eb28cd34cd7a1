// Solver session orchestration (cuda_solver.cu:1021-1853, dense form).
#include "session.hpp"

#include "autotune.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <limits>
#include <map>
#include <set>
#include <sstream>

namespace hsb {
namespace {

using Clock = std::chrono::steady_clock;
double msSince(Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }

void cuda(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        throw OutOfMemory(std::string(what) + ": " + cudaGetErrorString(e));
    if (e != cudaSuccess)
        throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T, class A> void upload(DeviceBuffer &buf, const std::vector<T, A> &v, cudaStream_t s) {
    buf.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
    if (!v.empty())
        cuda(cudaMemcpyAsync(buf.as<void>(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
}

bool sameNumerics(const hs_numerics &a, const hs_numerics &b) {
    return a.quadrature_order == b.quadrature_order && a.singular_order == b.singular_order &&
           a.near_distance_ratio == b.near_distance_ratio && a.near_relative_tolerance == b.near_relative_tolerance &&
           a.near_maximum_depth == b.near_maximum_depth;
}

// cuda_solver.cu:679-704: solid-angle inside test of a finite observer.
bool insideSolid(const Space &sp, V3 x) {
    double angle = 0;
    for (const auto &pn : sp.panels) {
        const V3 e0 = pn.v[1] - pn.v[0], e1 = pn.v[2] - pn.v[0], rel = x - pn.v[0];
        const double scale = std::max(std::sqrt(norm2(x)), std::sqrt(norm2(pn.v[0])));
        const double tol = std::max(pn.maxEdge * 1e-10, scale * 32 * std::numeric_limits<double>::epsilon());
        if (std::abs(dot(rel, pn.n)) <= tol) {
            const double aa = dot(e0, e0), ab = dot(e0, e1), bb = dot(e1, e1), pa = dot(rel, e0), pb = dot(rel, e1);
            const double det = aa * bb - ab * ab, u = (bb * pa - ab * pb) / det, v = (aa * pb - ab * pa) / det;
            if (u >= -1e-10 && v >= -1e-10 && u + v <= 1 + 1e-10)
                return true;
        }
        const V3 a = pn.v[0] - x, b = pn.v[1] - x, c = pn.v[2] - x;
        const double la = std::sqrt(norm2(a)), lb = std::sqrt(norm2(b)), lc = std::sqrt(norm2(c));
        const double den = la * lb * lc + dot(a, b) * lc + dot(b, c) * la + dot(c, a) * lb;
        angle += 2 * std::atan2(dot(a, cross(b, c)), den);
    }
    return std::abs(angle) > 2 * M_PI;
}

// regular_qualification.hpp:370-377
uint32_t refinedDegreeOf(uint32_t d) { return d < 4 ? 4 : d < 6 ? 6 : d < 8 ? 8 : d < 12 ? 12 : d < 14 ? 14 : 0; }

// planning_frequencies.hpp:14-38
double planningWavenumber(const hs_request &r) {
    if (!r.frequency_count || !std::isfinite(r.sound_speed) || r.sound_speed <= 0)
        throw InvalidArgument("Interaction planning requires frequencies and sound speed.");
    std::set<double> raster;
    double maximum = 0;
    for (size_t i = 0; i < r.plan_frequency_count; ++i) {
        const double f = r.plan_frequencies[i];
        if (!std::isfinite(f) || f <= 0 || !raster.insert(f).second)
            throw InvalidArgument("Interaction planning frequencies must be finite, positive and unique.");
        maximum = std::max(maximum, f);
    }
    for (size_t i = 0; i < r.frequency_count; ++i) {
        const double f = r.frequencies[i];
        if (!std::isfinite(f) || f <= 0 || (r.plan_frequency_count && !raster.count(f)))
            throw InvalidArgument("Solved frequency is invalid or absent from its interaction planning raster.");
        if (!r.plan_frequency_count)
            maximum = std::max(maximum, f);
    }
    const double k = 2 * M_PI * maximum / r.sound_speed;
    if (!std::isfinite(k))
        throw InvalidArgument("Interaction planning wavenumber overflows.");
    return k;
}

void validateRequest(const hs_request &r) {
    const hs_numerics &o = r.numerics;
    const bool fmm = o.acceleration == HS_FAST_MULTIPOLE;
    const unsigned w = o.fmm_preconditioner_block_width;
    if ((o.acceleration != HS_DENSE && !fmm) ||
        (fmm && ((o.fmm_leaf_support_capacity != 0 && o.fmm_leaf_support_capacity < 4) ||
                 o.fmm_leaf_support_capacity > 256 ||
                 !std::isfinite(o.fmm_separation_ratio) || o.fmm_separation_ratio < 1.5 || o.fmm_separation_ratio > 10 ||
                 o.fmm_maximum_iterations < 1 || o.fmm_maximum_iterations > 10000 || o.fmm_restart_length < 2 ||
                 o.fmm_restart_length > 300 ||
                 (w != 32 && w != 64 && w != 128 && w != 256 && w != 512 && w != 1024 && w != 2048))))
        throw InvalidArgument("Invalid Fast Multipole or GMRES settings.");
    if (o.precision == HS_PRECISION_MIXED && (o.fmm_maximum_iterations < 1 || o.fmm_maximum_iterations > 10000 ||
                                               o.fmm_restart_length < 2 || o.fmm_restart_length > 300))
        throw InvalidArgument("Invalid Fast Multipole or GMRES settings.");
    if (!std::isfinite(r.density) || r.density <= 0 || !std::isfinite(r.sound_speed) || r.sound_speed <= 0 ||
        !r.frequency_count || !r.excitation_count || (o.quadrature_order != 2 && o.quadrature_order != 4) ||
        o.singular_order < 2 || o.singular_order > 20 || !std::isfinite(o.near_distance_ratio) ||
        o.near_distance_ratio < 0 || o.near_distance_ratio > 10 || !std::isfinite(o.near_relative_tolerance) ||
        o.near_relative_tolerance < 1e-10 || o.near_relative_tolerance > .01 || o.near_maximum_depth > 10 ||
        !std::isfinite(o.relative_residual_tolerance) || o.relative_residual_tolerance < 1e-7 ||
        o.relative_residual_tolerance > .01 || o.maximum_refinement_steps > 10)
        throw InvalidArgument("Invalid BEM medium, frequencies, excitation or Galerkin settings.");
    if (o.precision != HS_PRECISION_FP64 && o.precision != HS_PRECISION_MIXED)
        throw InvalidArgument("Invalid BEM precision form.");
    if (r.excitation_count > 1024 || r.observer_count > 100000)
        throw InvalidArgument("BEM request exceeds indexing limits.");
}

}  // namespace

void *DeviceBuffer::ensure(size_t bytes) {
    if (bytes <= bytes_)
        return ptr_;
    release();
    void *p = nullptr;
    cuda(cudaMalloc(&p, bytes), "CUDA allocation");
    ptr_ = p;
    bytes_ = bytes;
    return ptr_;
}
void DeviceBuffer::release() {
    if (ptr_)
        cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
}

Session::Session(const MeshInput &mesh, uint32_t residency) : mesh_(mesh), residency_(residency) {
    if (residency > HS_RESIDENCY_MAPPED_HOST)
        throw InvalidArgument("Invalid CUDA quadrature storage policy.");
    if (mesh_.vertices.empty())
        throw InvalidArgument("BEM mesh has no vertices.");
    origin_ = mesh_.vertices.front();
    for (auto &v : mesh_.vertices) {
        v = v - origin_;
        if (!std::isfinite(v.x) || !std::isfinite(v.y) || !std::isfinite(v.z))
            throw InvalidArgument("BEM mesh coordinates are not finite.");
    }
    validateExteriorSurface(mesh_);
    space_ = buildSpace(mesh_);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        throw CudaError("No CUDA device is available.");
    cuda(cudaStreamCreateWithFlags(&own_, cudaStreamNonBlocking), "CUDA stream");
    uploadGeometry();
}

void Session::releaseMappedPatches() {
    if (mappedPatchesHost_) {
        cudaStreamSynchronize(stream());  // no kernel may still read the mapped range
        cudaFreeHost(mappedPatchesHost_);
        mappedPatchesHost_ = nullptr;
        patches_ = nullptr;
    }
}

Session::~Session() {
    dropGraphs();
    releaseMappedPatches();
    if (own_) {
        cudaStreamSynchronize(own_);
        cudaStreamDestroy(own_);
    }
    if (phaseReady_)
        for (cudaEvent_t e : {phase_.batch, phase_.assembled, phase_.factored, phase_.solved, phase_.refine0,
                              phase_.refine1})
            cudaEventDestroy(e);
}

Session::PhaseEvents &Session::phaseEvents() {
    if (!phaseReady_) {
        for (cudaEvent_t *e : {&phase_.batch, &phase_.assembled, &phase_.factored, &phase_.solved, &phase_.refine0,
                               &phase_.refine1})
            cuda(cudaEventCreate(e), "phase event");
        phaseReady_ = true;
    }
    return phase_;
}

void Session::setStream(cudaStream_t s) {
    cuda(cudaStreamSynchronize(stream()), "CUDA synchronization");
    external_ = s;
}

void Session::uploadGeometry() {
    const size_t T = space_.panels.size(), N = space_.vertices.size();
    std::vector<DPanel> panels(T);
    std::vector<Bounds> bounds(T);
    for (size_t t = 0; t < T; ++t) {
        const HostPanel &p = space_.panels[t];
        DPanel &d = panels[t];
        const V3 e1 = p.v[1] - p.v[0], e2 = p.v[2] - p.v[0];
        const double v0[3] = {p.v[0].x, p.v[0].y, p.v[0].z}, a[3] = {e1.x, e1.y, e1.z}, b[3] = {e2.x, e2.y, e2.z},
                     n[3] = {p.n.x, p.n.y, p.n.z};
        for (int i = 0; i < 3; ++i) {
            d.v0[i] = v0[i];
            d.e1[i] = a[i];
            d.e2[i] = b[i];
            d.n[i] = n[i];
            d.curl[3 * i] = p.curl[i].x;
            d.curl[3 * i + 1] = p.curl[i].y;
            d.curl[3 * i + 2] = p.curl[i].z;
            d.nodes[i] = p.nodes[i];
        }
        d.area = p.area;
        d.maxEdge = p.maxEdge;
        d.pad = 0;
        bounds[t] = makeBounds(p);
    }
    std::vector<double> scale(N);
    for (size_t v = 0; v < N; ++v)
        scale[v] = 1.0 / space_.lumpedMass[v];
    const cudaStream_t s = stream();
    std::vector<MixedPanel> mixedPanels(T);
    for (size_t t = 0; t < T; ++t)
        mixedPanels[t] = makeMixedPanel(panels[t], bounds[t]);
    upload(dPanels_, panels, s);
    upload(dBounds_, bounds, s);
    upload(dMixedPanels_, mixedPanels, s);
    upload(dIncOffsets_, space_.incOffsets, s);
    upload(dIncPanel_, space_.incPanel, s);
    upload(dIncLocal_, space_.incLocal, s);
    upload(dRowScale_, scale, s);
    upload(dMass_, space_.lumpedMass, s);
    dError_.ensure(16);
    cuda(cudaMemsetAsync(dError_.as<void>(), 0, 16, s), "error reset");
    uploadRuleTables(s);
    cuda(cudaStreamSynchronize(s), "CUDA synchronization");
}

const Plan &Session::plan(const hs_numerics &numerics, double maxK, const volatile int32_t *cancel) {
    preparePlan(numerics, maxK, cancel);
    return plan_;
}

// cuda_solver.cu:800-940: the plan is rebuilt only when its settings or the
// planning wavenumber change; otherwise the session's device copy is reused.
void Session::preparePlan(const hs_numerics &o, double maxK, const volatile int32_t *cancel) {
    if (planValid_ && sameNumerics(planNumerics_, o) && planK_ == maxK) {
        planMs_ = 0;
        return;
    }
    planValid_ = false;
    dropGraphs();  // captured chains hold the old plan's counts and rules
    const auto start = Clock::now();
    PlanSettings st{o.quadrature_order, o.singular_order, o.near_distance_ratio, o.near_relative_tolerance,
                    o.near_maximum_depth};
    planStats_ = DevicePlanStats{};
    plan_ = planner_ == HS_PLANNER_HOST ? makePlan(space_, st, maxK, 0, cancel)
                                        : makePlanOnDevice(space_, st, maxK, stream(), cancel, &planStats_);
    const uint32_t T = uint32_t(space_.panels.size());
    const size_t pairs = size_t(T) * (T - 1) / 2;
    std::vector<uint8_t> code(pairs, kPairRegular);
    for (const auto &j : plan_.touching)
        if (j.test != j.trial)
            code[unorderedPairIndex(j.test, j.trial)] = kPairTouching;
    // Near pairs with only tensor patches first, those with projected patches last.
    std::vector<NearPairJob> nearPairs, projectedPairs;
    for (const auto &j : plan_.near) {
        code[unorderedPairIndex(j.test, j.trial)] = kPairNear;
        if (j.swap)
            continue;
        bool projected = false;
        for (uint32_t q = 0; q < j.count; ++q)
            projected = projected || plan_.patches[j.first + q].projection;
        (projected ? projectedPairs : nearPairs).push_back({j.test, j.trial, j.first, j.count});
    }
    projectedPairCount_ = uint32_t(projectedPairs.size());
    nearPairs.insert(nearPairs.end(), projectedPairs.begin(), projectedPairs.end());
    if (!plan_.wholePanelDegrees.empty())
        for (size_t u = 0; u < pairs; ++u)
            if (code[u] == kPairRegular && plan_.wholePanelDegrees[u])
                code[u] = plan_.wholePanelDegrees[u] == 14 ? kPairWhole14 : kPairWhole8;
    std::vector<TouchingJob> touching(plan_.touching.size());
    for (size_t i = 0; i < touching.size(); ++i) {
        const auto &j = plan_.touching[i];
        TouchingJob &d = touching[i];
        d.test = j.test;
        d.trial = j.trial;
        d.topology = j.perm.topology;
        for (int c = 0; c < 3; ++c) {
            d.permTest[c] = j.perm.test[c];
            d.permTrial[c] = j.perm.trial[c];
        }
        d.pad[0] = d.pad[1] = 0;
    }
    const auto gauss = gaussLegendre01(o.singular_order);
    std::vector<double> g(2 * gauss.size());
    for (size_t i = 0; i < gauss.size(); ++i) {
        g[2 * i] = gauss[i].x;
        g[2 * i + 1] = gauss[i].w;
    }
    const cudaStream_t s = stream();
    upload(dPairCode_, code, s);
    upload(dTouching_, touching, s);
    upload(dNearPairs_, nearPairs, s);
    // Near-pair quadrature patches: device memory, or mapped pinned host memory
    // that the kernels read over the bus (CudaCacheResidency, cuda_solver.cu:112-160,
    // 899-903): always for HS_RESIDENCY_MAPPED_HOST; for AUTOMATIC when the
    // patches would take more than a quarter of the free device memory.
    {
        const size_t patchBytes = plan_.patches.size() * sizeof(Patch);
        size_t freeBytes = 0, totalBytes = 0;
        cuda(cudaMemGetInfo(&freeBytes, &totalBytes), "CUDA memory query");
        const bool mapped = patchBytes && (residency_ == HS_RESIDENCY_MAPPED_HOST ||
                                           (residency_ == HS_RESIDENCY_AUTOMATIC && patchBytes > freeBytes / 4));
        releaseMappedPatches();
        if (mapped) {
            int device = 0, canMap = 0;
            cuda(cudaGetDevice(&device), "CUDA device query");
            cuda(cudaDeviceGetAttribute(&canMap, cudaDevAttrCanMapHostMemory, device), "CUDA host mapping query");
            if (!canMap)
                throw CudaError("CUDA device does not support mapped quadrature storage.");
            cuda(cudaHostAlloc(&mappedPatchesHost_, patchBytes, cudaHostAllocMapped), "CUDA mapped patch allocation");
            std::memcpy(mappedPatchesHost_, plan_.patches.data(), patchBytes);
            void *alias = nullptr;
            cuda(cudaHostGetDevicePointer(&alias, mappedPatchesHost_, 0), "CUDA mapped patch pointer");
            patches_ = static_cast<const Patch *>(alias);
            dPatches_.release();
        } else {
            upload(dPatches_, plan_.patches, s);
            patches_ = dPatches_.as<Patch>();
        }
    }
    upload(dGauss_, g, s);
    upload(dSingularTable_, buildSingularTable(o.singular_order), s);
    cuda(cudaStreamSynchronize(s), "CUDA synchronization");
    singularSamples_ = 0;
    for (const auto &j : plan_.touching)
        singularSamples_ += uint64_t(sectorCount(j.perm.topology)) * o.singular_order * o.singular_order *
                            o.singular_order * o.singular_order;
    nearSamples_ = 0;
    for (const auto &j : nearPairs)
        for (uint32_t q = 0; q < j.patchCount; ++q) {
            const Patch &p = plan_.patches[j.firstPatch + q];
            const uint64_t n = p.degree == 14 ? 64 : 16, inner = 20ull * p.intervals;
            nearSamples_ += p.projection ? n * 3 * inner * inner : n * n;
        }
    touchingCount_ = uint32_t(touching.size());
    nearPairCount_ = uint32_t(nearPairs.size());
    planNumerics_ = o;
    planK_ = maxK;
    planValid_ = true;
    planMs_ = msSince(start);
}

namespace {
uint64_t perFrequencyBytes(uint64_t T, uint64_t N, uint32_t E, uint32_t O, bool mixed, uint32_t restart) {
    return assemblyWorkspaceBytes(uint32_t(T), uint32_t(N), E, 1, mixed) + 2 * N * N * 16 + 4 * E * N * 16 +
           E * T * 16 + E * N * 16 + 8 * N + fieldPartialsBytes(uint32_t(T), E, O, 1) +
           (mixed ? gmresWorkspaceBytes(uint32_t(N), E, restart) + luPackBytes(uint32_t(N), 1) : 0) + 64;
}
}  // namespace

size_t solveFootprint(size_t T, size_t N, uint32_t E, uint32_t O, uint32_t B, bool mixed, uint32_t restart) {
    // geometry (panels, bounds, FP32 panels, incidence, scales) and plan
    // (pair codes, touching jobs, near pairs and patches at about a dozen
    // neighbours per panel)
    const size_t geometry = T * (200 + 48 + 112 + 16) + N * 24, plan = T * (T - 1) / 2 + T * 16 * 40 + T * 16 * 220;
    return geometry + plan + B * perFrequencyBytes(T, N, E, O, mixed, restart);
}

size_t fmmSolveFootprint(size_t T, size_t N, uint32_t E, uint32_t O, uint32_t restart) {
    // geometry and plan as for the dense form; near records and their pair
    // lists at about 700 near panel pairs per panel, near CSR values, GMRES
    // basis and the expansion tables (a fixed allowance)
    const size_t geometry = T * (200 + 48 + 112 + 16) + N * 24, plan = T * (T - 1) / 2 + T * 16 * 40 + T * 16 * 220;
    const size_t nearField = T * 700 * (kRecordDoubles * 8 + 4 + 8 + 8) + N * 500 * 20;
    const size_t solve = size_t(E) * N * 16 * (restart + 12) + N * 6 * 1024 * 16 * 2;
    const size_t fields = fieldPartialsBytes(uint32_t(T), E, O, 1) + size_t(E) * T * 16;
    return geometry + plan + nearField + solve + fields + (size_t(256) << 20);
}

size_t Session::residentBytes() const {
    size_t bytes = 0;
    for (const DeviceBuffer *b : {&dPanels_, &dBounds_, &dMixedPanels_, &dIncOffsets_, &dIncPanel_, &dIncLocal_,
                                  &dRowScale_, &dMass_, &dPairCode_, &dTouching_, &dNearPairs_, &dPatches_, &dGauss_,
                                  &dSingularTable_, &dRecords_, &dColumns_, &dPanelRhs_, &dBins_, &dBinCounts_, &dBinOffsets_, &dA_,
                                  &dLU_, &dRhs_, &dX_, &dCorr_, &dNorms_, &dPivots_, &dKs_, &dFlux_, &dObservers_,
                                  &dPartials_, &dField_, &dDegrees_, &dWork32_, &dGmres_, &dLuPack_, &dSolveScratch_})
        bytes += b->bytes();
    return bytes;
}

uint32_t Session::chooseBatch(uint32_t F, uint32_t E, uint32_t O, bool mixed, uint32_t restart) const {
    const uint64_t T = space_.panels.size(), N = space_.vertices.size();
    const uint64_t perFrequency = perFrequencyBytes(T, N, E, O, mixed, restart);
    size_t free = 0, total = 0;
    cuda(cudaMemGetInfo(&free, &total), "CUDA memory query");
    // the batch workspace this session already holds is reused (or freed before it grows)
    size_t held = 0;
    for (const DeviceBuffer *b : {&dRecords_, &dColumns_, &dPanelRhs_, &dBins_, &dBinCounts_, &dBinOffsets_, &dA_, &dLU_, &dRhs_,
                                  &dX_, &dCorr_, &dNorms_, &dPivots_, &dKs_, &dFlux_, &dPartials_, &dField_, &dDegrees_,
                                  &dWork32_, &dGmres_, &dLuPack_, &dSolveScratch_})
        held += b->bytes();
    uint64_t budget = uint64_t(double(free + held) * .6);
    if (perFrequency > budget)  // one frequency at a time may take up to 90 %
        budget = uint64_t(double(free + held) * .9);
    if (memoryBudget_)
        budget = std::min<uint64_t>(budget, memoryBudget_);
    if (perFrequency > budget)
        throw OutOfMemory("BEM dense workspace of " + std::to_string(perFrequency >> 20) + " MiB per frequency exceeds the " +
                          std::to_string(budget >> 20) + " MiB device budget.");
    return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>({uint64_t(F), budget / perFrequency, 32})));
}

void Session::ensureWorkspace(uint32_t B, uint32_t E, uint32_t O, bool mixed, uint32_t restart) {
    const size_t T = space_.panels.size(), N = space_.vertices.size();
    const size_t pairs = T * (T - 1) / 2;
    dRecords_.ensure(std::max<size_t>(B * recordBytes(uint32_t(T), mixed), 16));
    if (gatherUsesColumns(uint32_t(T)))
        dColumns_.ensure(B * N * 6 * T * (mixed ? 4 : 8));
    if (mixed) {
        dGmres_.ensure(gmresWorkspaceBytes(uint32_t(N), B * E, restart));
        dLuPack_.ensure(std::max<size_t>(luPackBytes(uint32_t(N), B), 16));
    }
    dPanelRhs_.ensure(B * E * 6 * T * 8);
    dBins_.ensure(std::max<size_t>(B * (T > kExactBinsT ? 1 : kBins) * pairs * sizeof(uint2), 16));
    dBinCounts_.ensure(B * kBins * sizeof(uint32_t));
    if (T > kExactBinsT)
        dBinOffsets_.ensure(B * kBins * sizeof(uint64_t));
    dA_.ensure(B * N * N * 16);
    dLU_.ensure(B * N * N * 16);
    dRhs_.ensure(B * E * N * 16);
    dX_.ensure(B * E * N * 16);
    dCorr_.ensure(B * E * N * 16);
    dNorms_.ensure(2 * B * E * 8 + 2 * B * E * N * 8);
    dPivots_.ensure(luWorkspaceBytes(uint32_t(N), B));
    dSolveScratch_.ensure(B * E * N * 16);
    dInfo_.ensure(16);
    dKs_.ensure(B * 8);
    dFlux_.ensure(B * E * T * 16);
    dObservers_.ensure(std::max<size_t>(O * 3 * 8, 16));
    dPartials_.ensure(std::max<size_t>(fieldPartialsBytes(uint32_t(T), E, O, B), 16));
    dField_.ensure(std::max<size_t>(B * E * O * 16, 16));
    dDegrees_.ensure(B * 4);
    dWork32_.ensure(B * E * N * 8);
    size_t bytes = 0;
    for (const DeviceBuffer *b : {&dPanels_, &dBounds_, &dMixedPanels_, &dIncOffsets_, &dIncPanel_, &dIncLocal_, &dRowScale_, &dMass_,
                                  &dPairCode_, &dTouching_, &dNearPairs_, &dPatches_, &dGauss_, &dSingularTable_, &dRecords_, &dColumns_,
                                  &dPanelRhs_, &dBins_, &dBinCounts_, &dBinOffsets_, &dA_, &dLU_, &dRhs_, &dX_, &dCorr_, &dNorms_,
                                  &dPivots_, &dKs_, &dFlux_, &dObservers_, &dPartials_, &dField_, &dDegrees_,
                                  &dWork32_, &dGmres_, &dLuPack_, &dSolveScratch_})
        bytes += b->bytes();
    peakBytes_ = std::max(peakBytes_, bytes);
}

void Session::pressureField(double frequency, double soundSpeed, const double *trace, const double *normalDerivative,
                            const double *points, size_t count, const hs_field_settings &st, double *pressure,
                            int32_t *status) {
    // checks and messages of evaluatePressureField (field_evaluation.cpp:334-356)
    if (!std::isfinite(frequency) || frequency <= 0 || !std::isfinite(soundSpeed) || soundSpeed <= 0 ||
        !std::isfinite(st.minimum_boundary_distance) || st.minimum_boundary_distance <= 0 ||
        !std::isfinite(st.relative_quadrature_tolerance) || st.relative_quadrature_tolerance <= 0 ||
        st.relative_quadrature_tolerance > .01 || st.maximum_quadrature_depth > 12)
        throw InvalidArgument("Invalid pressure field settings.");
    const size_t T = space_.panels.size(), N = space_.vertices.size();
    for (size_t i = 0; i < 2 * N; ++i)
        if (!std::isfinite(trace[i]))
            throw InvalidArgument("Non-finite pressure trace.");
    for (size_t i = 0; i < 2 * T; ++i)
        if (!std::isfinite(normalDerivative[i]))
            throw InvalidArgument("Non-finite derivative trace.");
    if (count > 0x7fffffffu)
        throw InvalidArgument("Too many pressure field points.");
    std::vector<double> local(3 * count);
    for (size_t i = 0; i < count; ++i) {
        if (!std::isfinite(points[3 * i]) || !std::isfinite(points[3 * i + 1]) || !std::isfinite(points[3 * i + 2]))
            throw InvalidArgument("Invalid pressure field point.");
        local[3 * i] = points[3 * i] - origin_.x;  // session coordinates are centred on vertex 0
        local[3 * i + 1] = points[3 * i + 1] - origin_.y;
        local[3 * i + 2] = points[3 * i + 2] - origin_.z;
    }
    if (!count)
        return;
    const cudaStream_t s = stream();
    dSamplePoints_.ensure(local.size() * 8);
    dSampleTrace_.ensure(N * 16);
    dSampleFlux_.ensure(T * 16);
    dSampleOut_.ensure(count * 16);
    dSampleStatus_.ensure(count * 4);
    cuda(cudaMemcpyAsync(dSamplePoints_.as<void>(), local.data(), local.size() * 8, cudaMemcpyHostToDevice, s),
         "field points upload");
    cuda(cudaMemcpyAsync(dSampleTrace_.as<void>(), trace, N * 16, cudaMemcpyHostToDevice, s), "trace upload");
    cuda(cudaMemcpyAsync(dSampleFlux_.as<void>(), normalDerivative, T * 16, cudaMemcpyHostToDevice, s),
         "derivative upload");
    const double k = 2 * M_PI * frequency / soundSpeed;
    samplePressureField(dPanels_.as<DPanel>(), uint32_t(T), dSampleTrace_.as<double>(), dSampleFlux_.as<double>(),
                        dSamplePoints_.as<double>(), uint32_t(count), k, st.minimum_boundary_distance,
                        st.relative_quadrature_tolerance, st.maximum_quadrature_depth, dSampleOut_.as<double>(),
                        dSampleStatus_.as<int32_t>(), s);
    cuda(cudaMemcpyAsync(pressure, dSampleOut_.as<void>(), count * 16, cudaMemcpyDeviceToHost, s), "field download");
    cuda(cudaMemcpyAsync(status, dSampleStatus_.as<void>(), count * 4, cudaMemcpyDeviceToHost, s), "field download");
    cuda(cudaStreamSynchronize(s), "CUDA pressure field");
}

void Session::checkDeviceError(const char *where) {
    int code = 0;
    cuda(cudaMemcpyAsync(&code, dError_.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, stream()), where);
    cuda(cudaStreamSynchronize(stream()), where);
    if (!code)
        return;
    cuda(cudaMemsetAsync(dError_.as<int>(), 0, sizeof(int), stream()), "error reset");
    if (code == kErrDistance)
        throw NumericError("BEM quadrature encountered zero or invalid source distance.");
    if (code == kErrNonFinite)
        throw NumericError("BEM calculation produced a non-finite value.");
    if (code == kErrFieldDepth)
        throw NumericError("BEM field integration did not reach its near-field tolerance.");
    if (code == kErrEscapedPlan)
        throw NumericError("BEM dense regular pair escaped its qualified adaptive plan.");
    throw NumericError("BEM device error code " + std::to_string(code));
}

std::unique_ptr<Result> Session::solve(const hs_request &r, const volatile int32_t *cancel, hs_progress_fn progress,
                                       void *user, const SolveHooks *hooks, const CouplingNetwork *coupling) {
    const auto checkCancel = [&]() {
        if (cancel && *cancel)
            throw Cancelled();
    };
    checkCancel();
    validateRequest(r);
    const hs_numerics &o = r.numerics;
    const double maxK = planningWavenumber(r);
    const uint32_t T = uint32_t(space_.panels.size()), N = uint32_t(space_.vertices.size());
    const uint32_t E = uint32_t(r.excitation_count), O = uint32_t(r.observer_count);
    const uint32_t F = uint32_t(r.frequency_count);
    // Far-field origin and observers in session coordinates (cuda_solver.cu:1087-1137).
    V3 farOrigin{0, 0, 0};
    if (r.far_field) {
        const V3 fo{r.far_origin[0], r.far_origin[1], r.far_origin[2]};
        farOrigin = fo - origin_;
        if (!std::isfinite(fo.x) || !std::isfinite(fo.y) || !std::isfinite(fo.z) || !std::isfinite(farOrigin.x) ||
            !std::isfinite(farOrigin.y) || !std::isfinite(farOrigin.z) || !std::isfinite(r.far_reference_distance) ||
            r.far_reference_distance <= 0 || !std::isfinite(maxK * r.far_reference_distance))
            throw InvalidArgument("Far-field origin and positive reference distance must be finite.");
    }
    std::vector<double> observers(3 * size_t(O));
    for (uint32_t i = 0; i < O; ++i) {
        const V3 w{r.observers[3 * i], r.observers[3 * i + 1], r.observers[3 * i + 2]};
        V3 p = w - (r.far_field ? V3{r.far_origin[0], r.far_origin[1], r.far_origin[2]} : origin_);
        if (!std::isfinite(w.x) || !std::isfinite(w.y) || !std::isfinite(w.z) || !std::isfinite(p.x) ||
            !std::isfinite(p.y) || !std::isfinite(p.z))
            throw InvalidArgument("BEM observation coordinates must be finite.");
        if (r.far_field) {
            const double d = std::hypot(p.x, p.y, p.z);
            if (!(d > 0) || !std::isfinite(d))
                throw InvalidArgument("A far-field direction must differ from its origin.");
            p = V3{p.x / d, p.y / d, p.z / d};
        } else if (insideSolid(space_, p))
            throw InvalidArgument("BEM observation points must be finite and outside the solid.");
        observers[3 * i] = p.x;
        observers[3 * i + 1] = p.y;
        observers[3 * i + 2] = p.z;
    }
    // Per-face boundary conditions and per-panel velocities (cuda_solver.cu:1165-1212).
    std::map<uint32_t, uint8_t> conditions;
    for (const auto &p : space_.panels) {
        const auto [it, inserted] = conditions.emplace(p.face, p.driven);
        if (!inserted && it->second != p.driven)
            throw InvalidArgument("Conflicting boundary conditions on one face.");
    }
    std::vector<cplx> velocity(size_t(E) * T);
    std::vector<std::map<uint32_t, cplx>> faceVelocity(E);
    bool nonzero = false;
    for (uint32_t e = 0; e < E; ++e) {
        for (size_t i = r.excitation_face_offsets[e]; i < r.excitation_face_offsets[e + 1]; ++i) {
            const uint32_t face = r.excitation_face_ids[i];
            const cplx v(r.excitation_velocities[2 * i], r.excitation_velocities[2 * i + 1]);
            const auto c = conditions.find(face);
            if (c == conditions.end() || c->second != HS_DRIVEN || !std::isfinite(v.real()) || !std::isfinite(v.imag()) ||
                !faceVelocity[e].emplace(face, v).second)
                throw InvalidArgument("Excitation must assign each known Driven face at most once.");
            nonzero = nonzero || v != cplx(0);
        }
        if (faceVelocity[e].empty())
            throw InvalidArgument("Each excitation needs at least one assigned Driven face.");
        for (uint32_t t = 0; t < T; ++t) {
            const auto it = faceVelocity[e].find(space_.panels[t].face);
            if (it != faceVelocity[e].end())
                velocity[size_t(e) * T + t] = it->second;
        }
    }
    // LEM coupling (cuda_solver.cu:1584-1667): the excitations are the unit-flow
    // basis, one per port; panel -> port and its velocity per unit flow.
    std::vector<int32_t> panelPort;
    std::vector<double> panelUnitVelocity;
    if (coupling) {
        if (o.acceleration == HS_FAST_MULTIPOLE)
            throw Unsupported("LEM-coupled fast-multipole solves are not part of this build; use a dense form.");
        panelPort.assign(T, -1);
        panelUnitVelocity.assign(T, 0.0);
        std::map<uint32_t, std::pair<uint32_t, double>> facePort;
        for (uint32_t e = 0; e < E; ++e)
            for (size_t i = r.excitation_face_offsets[e]; i < r.excitation_face_offsets[e + 1]; ++i) {
                const double vr = r.excitation_velocities[2 * i], vi = r.excitation_velocities[2 * i + 1];
                if (vi != 0 || !(vr > 0) || !std::isfinite(vr) ||
                    !facePort.emplace(r.excitation_face_ids[i], std::make_pair(e, vr)).second)
                    throw InvalidArgument("Coupled ports need positive real unit-flow velocities and disjoint faces.");
            }
        for (uint32_t t = 0; t < T; ++t) {
            const auto it = facePort.find(space_.panels[t].face);
            if (it != facePort.end()) {
                panelPort[t] = int32_t(it->second.first);
                panelUnitVelocity[t] = it->second.second;
            }
        }
    }
    if (progress) {
        hs_progress p{0, F, r.frequencies[0], HS_PHASE_PREPARING};
        progress(&p, user);
    }
    preparePlan(o, maxK, cancel);
    const double planMs = planMs_;
    checkCancel();
    const cudaStream_t s = stream();
    const bool mixedForm = o.precision == HS_PRECISION_MIXED;
    const uint32_t restart = o.fmm_restart_length;
    const bool fmmRequest = o.acceleration == HS_FAST_MULTIPOLE;
    // The fast-multipole form runs one frequency at a time on its own sparse
    // near-field workspace (no dense records or matrices).
    const uint32_t Bmax = fmmRequest ? 1 : chooseBatch(F, E, O, mixedForm, restart);
    if (fmmRequest)
        ensureFmmWorkspace(o, E, O, maxK);
    else
        ensureWorkspace(Bmax, E, O, mixedForm, restart);
    if (O)
        cuda(cudaMemcpyAsync(dObservers_.as<void>(), observers.data(), observers.size() * 8, cudaMemcpyHostToDevice, s),
             "observer upload");
    auto result = std::make_unique<Result>();
    result->T = T;
    result->N = N;
    result->O = O;
    result->E = coupling ? 1 : E;
    result->frequencies.resize(F);
    AssemblyGeometry geo{dPanels_.as<DPanel>(), dBounds_.as<Bounds>(), dPairCode_.as<uint8_t>(),
                         dTouching_.as<TouchingJob>(), dNearPairs_.as<NearPairJob>(), patches_,
                         dIncOffsets_.as<uint32_t>(), dIncPanel_.as<uint32_t>(), dIncLocal_.as<uint8_t>(),
                         dRowScale_.as<double>(), T, N, touchingCount_, nearPairCount_, projectedPairCount_,
                         o.near_relative_tolerance,
                         o.quadrature_order, o.singular_order, dSingularTable_.as<float4>(),
                         dMixedPanels_.as<MixedPanel>()};
    double maxEdge = 0;
    for (const auto &p : space_.panels)
        maxEdge = std::max(maxEdge, p.maxEdge);
    // Device span of the whole sweep (profiling on): from the first upload to
    // the last result download, host-side control included.
    const size_t span = timer_.start("solve_span", s);
    // frequencies in solve order: the request's, plus those a serving hook adds
    std::vector<double> freqList(r.frequencies, r.frequencies + F);
    for (uint32_t f0 = 0, B = 0; f0 < freqList.size(); f0 += B) {
        checkCancel();
        if (hooks && hooks->more) {
            const std::vector<double> extra = hooks->more();
            for (double f : extra)
                if (!std::isfinite(f) || f <= 0 || 2 * M_PI * f / r.sound_speed > maxK * (1 + 1e-12))
                    throw InvalidArgument("A frequency joining a running solve lies outside its interaction plan.");
            freqList.insert(freqList.begin() + f0, extra.begin(), extra.end());
            result->frequencies.insert(result->frequencies.begin() + f0, extra.size(), FrequencyResult{});
        }
        const uint32_t Ftotal = uint32_t(freqList.size());
        B = std::min<uint32_t>(Bmax, Ftotal - f0);
        // Phase times come from events on the session stream; the host waits for the
        // device only where it needs data (residual norms, GMRES estimates, fields).
        PhaseEvents &ev = phaseEvents();
        cuda(cudaEventRecord(ev.batch, s), "phase event");
        std::vector<double> ks(B);
        std::vector<cplx> flux(size_t(B) * E * T);
        for (uint32_t b = 0; b < B; ++b) {
            const double omega = 2 * M_PI * freqList[f0 + b];
            ks[b] = omega / r.sound_speed;
            for (size_t i = 0; i < size_t(E) * T; ++i)
                flux[size_t(b) * E * T + i] = cplx(0, -r.density * omega) * velocity[i];
        }
        cuda(cudaMemcpyAsync(dKs_.as<void>(), ks.data(), B * 8, cudaMemcpyHostToDevice, s), "k upload");
        cuda(cudaMemcpyAsync(dFlux_.as<void>(), flux.data(), flux.size() * 16, cudaMemcpyHostToDevice, s), "flux upload");
        AssemblyWorkspace ws{dRecords_.as<void>(), dColumns_.as<void>(), dPanelRhs_.as<double>(), dBins_.as<uint2>(),
                             dBinCounts_.as<uint32_t>(), size_t(T) * (T - 1) / 2,
                             T > kExactBinsT ? dBinOffsets_.as<uint64_t>() : nullptr};
        const bool mixed = o.precision == HS_PRECISION_MIXED;
        const bool fmmForm = o.acceleration == HS_FAST_MULTIPOLE;
        if (!fmmForm)  // assembly, LU and initial solves: launches only, no host waits
            runDenseChain(geo, ws, B, E, mixed, s);
        else
            cuda(cudaEventRecord(ev.assembled, s), "phase event");
        // the assembly error word is checked with the first residual norms
        const auto countWork = [&]() {
            std::vector<uint32_t> counts(size_t(B) * kBins);
            cuda(cudaMemcpy(counts.data(), dBinCounts_.as<void>(), counts.size() * 4, cudaMemcpyDeviceToHost),
                 "bin counts");
            for (uint32_t b = 0; b < B; ++b)
                for (int bin = 0; bin < kBins; ++bin) {
                    const uint64_t c = counts[size_t(b) * kBins + bin];
                    work[bin] += c;
                    work[4] += c * uint64_t(kBinPoints[bin]) * kBinPoints[bin];
                }
            work[5] += uint64_t(B) * singularSamples_;
            work[6] += uint64_t(B) * nearSamples_;
            work[7] += B;
        };
        checkCancel();
        double assemblyMs = 0, factorMs = 0, triMs = 0, residualMs = 0;
        std::vector<uint32_t> steps(B, 0), krylov(size_t(B) * E, 0), cycle;
        std::vector<double> relative(size_t(B) * E, 0);
        // the dense mixed form refines to 1e-10; the fast-multipole forms (FP64, or
        // GMRES-IR over the FP32 operator) solve to the request's tolerance
        const double target =
            mixed && !fmmForm ? std::min(o.relative_residual_tolerance, 1e-10) : o.relative_residual_tolerance;
        if (fmmForm) {
            // Fast-multipole form: per frequency the exact near support pairs
            // (records of the near panel pairs only), the right-hand side as
            // near part plus expansion far field, block-Jacobi on the leaf
            // blocks and GMRES on near + expansion far field
            // (support_fmm_solve.cu:401-525).
            FmmOperator &op = fmmOperator(o, maxK, fmmTuneTolerance(o));
            const NearFieldLayout layout{dPanelRow_.as<uint32_t>(), dPanelCol_.as<uint32_t>(), op.nearPanelCol().size(),
                                         dPanelPairs_.as<uint2>(), op.nearPanelPairs().size(),
                                         fmmSystem_->nearRowDevice(), fmmSystem_->nearColDevice()};
            // working expansions at 1 % of the target (the audit checks them against
            // expansions ten times finer)
            const double expansionTolerance = std::clamp(.01 * target, 1e-10, 1e-6);
            const auto solveStart = Clock::now();
            std::vector<double> rel;
            std::vector<uint32_t> its;
            // mixed: the inner operator of GMRES-IR, FP32 translations at expansions
            // for 1e-5 (its cycles win at most four digits each)
            FmmOperator *inner = mixed ? &fmmInnerOperator(o) : nullptr;
            for (uint32_t b = 0; b < B; ++b) {
                checkCancel();
                if (op.panelDegree() != 4)  // a promotion of an earlier, failed audit
                    op.setPanelDegree(4, s);
                op.prepare(ks[b], expansionTolerance, s);
                if (inner)
                    inner->prepare(ks[b], std::max(expansionTolerance, 1e-5), s);
                // near support pairs and the near right-hand side from the near panel-pair records
                double *rhsB = dRhs_.as<double>() + size_t(b) * E * N * 2;
                const double *fluxB = dFlux_.as<double>() + size_t(b) * E * T * 2;
                const size_t reals = size_t(E) * N * 2;
                double *nearRhs = dNearRhs_.as<double>();
                assembleNearField(geo, dKs_.as<double>() + b, dGauss_.as<double>(), fluxB, E, layout,
                                  dNearWork_.as<void>(), fmmSystem_->nearValues(), nearRhs, dError_.as<int>(), s,
                                  &timer_);
                if (inner)
                    fmmSystem_->roundNearValues(s);
                cuda(cudaEventRecord(ev.assembled, s), "phase event");
                // right-hand side with the operator's current far-field panel rule
                const auto buildRhs = [&](double *dst) {
                    TimedScope scope(&timer_, "fmm_rhs_far", s);
                    cuda(cudaMemcpyAsync(dst, nearRhs, reals * 8, cudaMemcpyDeviceToDevice, s), "near rhs copy");
                    op.applyFarRhs(fluxB, E, dCorr_.as<double>(), s, &timer_);
                    fmmSystem_->addScaled(dst, dCorr_.as<double>(), E, s);
                };
                buildRhs(rhsB);
                cuda(cudaEventRecord(ev.factored, s), "phase event");
                fmmSystem_->factorBlocks(s, &timer_);
                double *xB = dX_.as<double>() + size_t(b) * E * N * 2;
                // working solve to half the target, leaving the audit its margin
                fmmSystem_->solve(rhsB, xB, E, .5 * target, o.fmm_restart_length, o.fmm_maximum_iterations, s, &timer_,
                                  rel, its, inner);
                for (uint32_t e = 0; e < E; ++e)
                    krylov[size_t(b) * E + e] = its[e];
                const auto download = [&](const double *src) {
                    std::vector<cplx> v(size_t(E) * N);
                    cuda(cudaMemcpyAsync(v.data(), src, reals * 8, cudaMemcpyDeviceToHost, s), "audit download");
                    return v;
                };
                const auto massNorm = [&](const std::vector<cplx> &v, uint32_t e) {
                    double acc = 0;
                    for (size_t i = 0; i < N; ++i)
                        acc += space_.lumpedMass[i] * std::norm(v[size_t(e) * N + i]);
                    return std::sqrt(acc);
                };
                // defect correction: x += A_work^-1 r with the working expansions. The
                // correction solve is relative to r, whose norm is rRel of the
                // right-hand side's: it aims at half the target relative to the
                // right-hand side, not to r (which would ask for digits below the
                // FP64 operator's rounding once r is small).
                const auto correct = [&](const double *r, double workTolerance, double rRel) {
                    op.prepare(ks[b], workTolerance, s);
                    const double relTarget = rRel > 0 ? std::clamp(.5 * target / rRel, .5 * target, .5) : .5;
                    fmmSystem_->solve(r, dCorr_.as<double>(), E, relTarget, o.fmm_restart_length,
                                      o.fmm_maximum_iterations, s, &timer_, rel, its, inner);
                    fmmSystem_->add(xB, dCorr_.as<double>(), reals, s);
                    for (uint32_t e = 0; e < E; ++e)
                        krylov[size_t(b) * E + e] += its[e];
                };
                double tau = expansionTolerance;
                // Direct Galerkin audit (preferSupportDirectAudit, support_fmm_solve.cu:79-114;
                // directFar, support_direct_audit.cu:26) where assembling the dense
                // operator costs less than two expansion operators: the residual of
                // the exact FP64 dense system, defect-corrected with the working
                // fast-multipole operator.
                if (preferDirectAudit(op)) {
                    TimedScope scope(&timer_, "fmm_direct_audit", s);
                    double *directA = nullptr, *directB = nullptr;
                    directAuditFrequency_ = b;
                    directAuditSystem(geo, ks[b], fluxB, E, directA, directB);
                    for (uint32_t round = 0;; ++round) {
                        residualBatch(directA, directB, xB, dMass_.as<double>(), N, 1, E, dAuditFine_.as<double>(),
                                      dNorms_.as<double>(), s, nullptr);
                        std::vector<double> norms(2 * size_t(E));
                        cuda(cudaMemcpyAsync(norms.data(), dNorms_.as<void>(), norms.size() * 8, cudaMemcpyDeviceToHost,
                                             s),
                             "direct audit norms");
                        cuda(cudaStreamSynchronize(s), "CUDA direct audit");
                        bool accept = true;
                        double worst = 0;
                        for (uint32_t e = 0; e < E; ++e) {
                            const double r = norms[2 * e + 1] > 0 ? norms[2 * e] / norms[2 * e + 1] : 0.0;
                            relative[size_t(b) * E + e] = r;
                            accept = accept && r <= target;
                            worst = std::max(worst, r);
                        }
                        if (accept)
                            break;
                        if (round >= std::max<uint32_t>(o.maximum_refinement_steps, 3))
                            throw NoConvergence("Direct Galerkin audit residual exceeds the tolerance; bounded "
                                                "fast-multipole defect corrections did not converge.");
                        correct(dAuditFine_.as<double>(), tau, worst);
                    }
                    directAudits_ += 1;
                } else
                    for (unsigned degree = op.panelDegree();;) {
                        // Audit against a ten times finer expansion operator and defect-correct
                        // (SupportFmmLinearSolver::solve / improve, support_fmm_solve.cu:324-343,
                        // 575-634): accept when the audited residual meets the target and the two
                        // operators differ on x by at most a quarter of it; otherwise tighten the
                        // working tolerance and solve for the audited residual's correction.
                        std::vector<double> relWork, relAudit;
                        for (uint32_t round = 0;; ++round) {
                            TimedScope scope(&timer_, "fmm_audit", s);
                            op.prepare(ks[b], tau, s);
                            fmmSystem_->residual(rhsB, xB, E, dAuditWork_.as<double>(), relWork, s, &timer_);
                            op.prepare(ks[b], .1 * tau, s);
                            fmmSystem_->residual(rhsB, xB, E, dAuditFine_.as<double>(), relAudit, s, &timer_);
                            const auto rWork = download(dAuditWork_.as<double>());
                            const auto rAudit = download(dAuditFine_.as<double>());
                            const auto rhsHost = download(rhsB);
                            cuda(cudaStreamSynchronize(s), "CUDA fast-multipole audit");
                            bool accept = true;
                            for (uint32_t e = 0; e < E; ++e) {
                                double dd = 0, bb = 0;
                                for (size_t i = 0; i < N; ++i) {
                                    const double m = space_.lumpedMass[i];
                                    dd += m * std::norm(rAudit[size_t(e) * N + i] - rWork[size_t(e) * N + i]);
                                    bb += m * std::norm(rhsHost[size_t(e) * N + i]);
                                }
                                const double disc = bb > 0 ? std::sqrt(dd / bb) : 0.0;
                                relative[size_t(b) * E + e] = relAudit[e];
                                accept = accept && relAudit[e] <= target && disc <= .25 * target;
                            }
                            if (accept)
                                break;
                            if (round >= 3)
                                throw NoConvergence("Fast-multipole audit did not meet the residual tolerance after 4 "
                                                    "expansion refinements.");
                            tau = std::max(.1 * tau, 1e-12);
                            correct(dAuditFine_.as<double>(), tau, *std::max_element(relAudit.begin(), relAudit.end()));
                        }
                        // Far-field panel rule (compareQuadrature, support_fmm_solve.cu:525-560):
                        // at the verification expansions, the operator and right-hand side with
                        // the next panel rule must differ from the current ones by at most
                        // 0.025 of the target, and the next rule's residual meet the target;
                        // otherwise the rule is promoted (4 -> 6 -> 8 -> 12), the solution
                        // defect-corrected and both audits repeated.
                        TimedScope scope(&timer_, "fmm_quadrature_audit", s);
                        const unsigned next = degree < 6 ? 6 : degree < 8 ? 8 : 12;
                        op.prepare(ks[b], .1 * tau, s);
                        fmmSystem_->apply(xB, size_t(N) * 2, E, dAuditWork_.as<double>(), s, &timer_);
                        const auto axNow = download(dAuditWork_.as<double>());
                        const auto bNow = download(rhsB);
                        op.setPanelDegree(next, s);
                        buildRhs(dAuditB_.as<double>());
                        fmmSystem_->apply(xB, size_t(N) * 2, E, dAuditWork_.as<double>(), s, &timer_);
                        const auto axNext = download(dAuditWork_.as<double>());
                        const auto bNext = download(dAuditB_.as<double>());
                        cuda(cudaStreamSynchronize(s), "CUDA quadrature audit");
                        bool accept = true;
                        for (uint32_t e = 0; e < E; ++e) {
                            std::vector<cplx> db(size_t(E) * N), da(size_t(E) * N), rn(size_t(E) * N);
                            for (size_t i = size_t(e) * N; i < size_t(e + 1) * N; ++i) {
                                db[i] = bNext[i] - bNow[i];
                                da[i] = axNext[i] - axNow[i];
                                rn[i] = bNext[i] - axNext[i];
                            }
                            const double bn = massNorm(bNext, e);
                            const double disc = bn > 0 ? (massNorm(db, e) + massNorm(da, e)) / bn : 0.0;
                            const double res = bn > 0 ? massNorm(rn, e) / bn : 0.0;
                            accept = accept && disc <= .025 * target && res <= target;
                        }
                        if (accept) {
                            op.setPanelDegree(4, s);  // the next frequency starts from the base rule again
                            break;
                        }
                        if (degree == 12)
                            throw NoConvergence("BEM endpoint quadrature 12/14 did not converge: the fast-multipole "
                                                "far-field panel rules disagree beyond 0.025*residualTolerance; "
                                                "refine the mesh.");
                        // promoted: the next rule's right-hand side, then a defect correction
                        degree = next;
                        ++quadraturePromotions_;
                        cuda(cudaMemcpyAsync(rhsB, dAuditB_.as<void>(), reals * 8, cudaMemcpyDeviceToDevice, s),
                             "promoted rhs");
                        fmmSystem_->residual(rhsB, xB, E, dAuditFine_.as<double>(), relAudit, s, &timer_);
                        correct(dAuditFine_.as<double>(), tau, *std::max_element(relAudit.begin(), relAudit.end()));
                    }
            }
            cuda(cudaEventRecord(ev.solved, s), "phase event");
            cuda(cudaStreamSynchronize(s), "CUDA fast-multipole solve");
            checkDeviceError("CUDA Galerkin near-field assembly");
            float a = 0, c = 0;
            cuda(cudaEventElapsedTime(&a, ev.batch, ev.assembled), "phase time");
            cuda(cudaEventElapsedTime(&c, ev.factored, ev.solved), "phase time");
            assemblyMs = a;
            triMs = c;
            residualMs = msSince(solveStart);
            if (timer_.enabled())
                countWork();
        } else {
        const size_t vectorReals = size_t(B) * E * N * 2;
        float *LU32 = dLU_.as<float>();
        bool refining = false;  // a refinement solve between ev.refine0 and ev.refine1 awaits its time
        // FP64 refinement (cuda_solver.cu:1519-1581), per frequency. The mixed
        // form refines against the FP64 residual to min(tolerance, 1e-10).
        const uint32_t maxSteps = mixed ? std::max<uint32_t>(o.maximum_refinement_steps, 10) : o.maximum_refinement_steps;
        const auto residualStart = Clock::now();
        std::vector<double> norms(2 * size_t(B) * E);
        bool statusChecked = false;
        for (int pass = 0; pass < (coupling ? 2 : 1); ++pass) {
        if (pass == 1)  // the coupled field: superposed basis, then its own refinement
            coupleBatch(*coupling, freqList, f0, B, E, r.density, panelPort, panelUnitVelocity, result->frequencies);
        for (;;) {
            checkCancel();
            residualBatch(dA_.as<double>(), dRhs_.as<double>(), dX_.as<double>(), dMass_.as<double>(), N, B, E,
                          dCorr_.as<double>(), dNorms_.as<double>(), s, &timer_);
            cuda(cudaMemcpyAsync(norms.data(), dNorms_.as<void>(), norms.size() * 8, cudaMemcpyDeviceToHost, s),
                 "residual norms");
            cuda(cudaStreamSynchronize(s), "CUDA FP64 physical residual");
            if (refining) {
                float ms = 0;
                cuda(cudaEventElapsedTime(&ms, ev.refine0, ev.refine1), "phase time");
                triMs += ms;
                refining = false;
            } else if (!statusChecked) {  // first residual: assembly and factorisation status, phase times
                statusChecked = true;
                checkDeviceError("CUDA Galerkin assembly");
                int info = 0;
                cuda(cudaMemcpy(&info, dInfo_.as<int>(), sizeof(int), cudaMemcpyDeviceToHost), "LU info");
                if (info < 0)
                    throw NumericError("CUDA Burton-Miller factorization: a tensor-core trailing update did not complete.");
                if (info)
                    throw NumericError("CUDA Burton-Miller factorization failed at pivot " + std::to_string(info));
                float a = 0, b = 0, c = 0;
                cuda(cudaEventElapsedTime(&a, ev.batch, ev.assembled), "phase time");
                cuda(cudaEventElapsedTime(&b, ev.assembled, ev.factored), "phase time");
                cuda(cudaEventElapsedTime(&c, ev.factored, ev.solved), "phase time");
                assemblyMs = a;
                factorMs = b;
                triMs = c;
                if (timer_.enabled())
                    countWork();
            }
            bool any = false;
            for (uint32_t b = 0; b < B; ++b) {
                double largest = 0;
                for (uint32_t e = 0; e < E; ++e) {
                    const double res = norms[2 * (size_t(b) * E + e)], rhs = norms[2 * (size_t(b) * E + e) + 1];
                    const double rel = rhs > 0 ? res / rhs : (res == 0 ? 0 : std::numeric_limits<double>::infinity());
                    if (!std::isfinite(rel))
                        throw NumericError("Burton-Miller residual is not finite.");
                    relative[size_t(b) * E + e] = rel;
                    largest = std::max(largest, rel);
                }
                const bool need = largest > target;
                if (need && steps[b] >= maxSteps) {
                    std::ostringstream msg;
                    msg << std::setprecision(9) << "Burton-Miller residual " << largest << " exceeds tolerance "
                        << target << " at " << freqList[f0 + b] << " Hz after " << steps[b]
                        << " refinement steps.";
                    throw NoConvergence(msg.str());
                }
                if (need) {
                    ++steps[b];
                    any = true;
                } else
                    cuda(cudaMemsetAsync(dCorr_.as<char>() + size_t(b) * E * N * 16, 0, size_t(E) * N * 16, s),
                         "converged correction");
            }
            if (!any)
                break;
            cuda(cudaEventRecord(ev.refine0, s), "phase event");
            if (mixed) {
                // GMRES-IR: one FP64 GMRES cycle on A d = r per system, preconditioned
                // by the FP32 LU, reducing each system's preconditioned residual far
                // enough that it lands a hundredfold below the target.
                std::vector<double> tolerances(relative.size());
                for (size_t q = 0; q < relative.size(); ++q)
                    tolerances[q] = relative[q] > 0 ? std::clamp(.01 * target / relative[q], 1e-13, .5) : .5;
                gmresCycleBatch(dA_.as<double>(), LU32, dPivots_.as<int>(), N, B, E, dCorr_.as<double>(),
                                dX_.as<double>(), restart, tolerances, dGmres_.as<void>(), s, &timer_, cycle);
                for (size_t q = 0; q < cycle.size(); ++q)
                    krylov[q] += cycle[q];
            } else {
                luSolveBatch(dLU_.as<double>(), dPivots_.as<int>(), N, B, E, dCorr_.as<double>(),
                             dSolveScratch_.as<void>(), s, &timer_);
                TimedScope scope(&timer_, "add_correction", s);
                addCorrectionBatch(dX_.as<double>(), dCorr_.as<double>(), vectorReals, s);
            }
            cuda(cudaEventRecord(ev.refine1, s), "phase event");
            refining = true;
        }
        }
        residualMs = msSince(residualStart);
        }
        // Observer fields with the degree-comparison loop (cuda_solver.cu:1717-1799).
        const auto fieldStart = Clock::now();
        std::vector<cplx> field(size_t(B) * E * O, 0);
        std::vector<uint32_t> degree(B), fieldDeg(size_t(B) * E), fieldNext(size_t(B) * E);
        std::vector<double> fieldDisc(size_t(B) * E, 0);
        if (O && nonzero) {
            if (progress)
                for (uint32_t b = 0; b < B; ++b) {
                    hs_progress p{f0 + b, Ftotal, freqList[f0 + b], HS_PHASE_FIELD_EVALUATION};
                    progress(&p, user);
                }
            for (uint32_t b = 0; b < B; ++b) {
                const double kh = ks[b] * maxEdge;
                if (kh > 3.25) {
                    std::ostringstream msg;
                    msg << "BEM panel quadrature: maximum k*h=" << kh
                        << " exceeds the qualified electrical range 3.25; refine the mesh.";
                    throw NumericError(msg.str());
                }
                const unsigned electrical = kh <= .25 ? 4 : kh <= 1 ? 6 : kh <= 2 ? 8 : 12;
                degree[b] = std::max(electrical, o.quadrature_order);
            }
            FieldRequest fr{dPanels_.as<DPanel>(), T, N, E, O, B, dObservers_.as<double>(), r.far_field,
                            {farOrigin.x, farOrigin.y, farOrigin.z}, r.far_field ? r.far_reference_distance : 1.0,
                            std::min(o.near_relative_tolerance, .025 * o.relative_residual_tolerance),
                            o.near_maximum_depth};
            const auto evaluate = [&](const std::vector<uint32_t> &deg) {
                cuda(cudaMemcpyAsync(dDegrees_.as<void>(), deg.data(), B * 4, cudaMemcpyHostToDevice, s), "degrees");
                evaluateFieldBatch(fr, dKs_.as<double>(), dX_.as<double>(), dFlux_.as<double>(), dDegrees_.as<uint32_t>(),
                                   dPartials_.as<double>(), dField_.as<double>(), dError_.as<int>(), s, &timer_);
                std::vector<cplx> out(size_t(B) * E * O);
                cuda(cudaMemcpyAsync(out.data(), dField_.as<void>(), out.size() * 16, cudaMemcpyDeviceToHost, s),
                     "field download");
                checkDeviceError("CUDA P1 field evaluation");
                return out;
            };
            std::vector<cplx> current = evaluate(degree);
            std::vector<bool> done(B, false);
            for (;;) {
                checkCancel();
                std::vector<uint32_t> next(B);
                for (uint32_t b = 0; b < B; ++b)
                    next[b] = done[b] ? degree[b] : refinedDegreeOf(degree[b]);
                const std::vector<cplx> refined = evaluate(next);
                bool all = true;
                for (uint32_t b = 0; b < B; ++b) {
                    if (done[b])
                        continue;
                    bool passed = true;
                    for (uint32_t e = 0; e < E; ++e) {
                        double d2 = 0, n2 = 0;
                        for (uint32_t q = 0; q < O; ++q) {
                            const size_t i = (size_t(b) * E + e) * O + q;
                            d2 += std::norm(refined[i] - current[i]);
                            n2 += std::norm(refined[i]);
                        }
                        const double ind = n2 > 0 ? std::sqrt(d2 / n2) : (d2 == 0 ? 0 : std::numeric_limits<double>::infinity());
                        fieldDeg[size_t(b) * E + e] = degree[b];
                        fieldNext[size_t(b) * E + e] = next[b];
                        fieldDisc[size_t(b) * E + e] = ind;
                        passed = passed && ind <= .025 * o.relative_residual_tolerance;
                    }
                    for (uint32_t e = 0; e < E; ++e)
                        for (uint32_t q = 0; q < O; ++q) {
                            const size_t i = (size_t(b) * E + e) * O + q;
                            field[i] = refined[i];
                        }
                    if (passed)
                        done[b] = true;
                    else if (degree[b] == 12)
                        throw NoConvergence("BEM complex observer-field quadrature 12/14 did not converge within "
                                            "0.025*residualTolerance; refine the mesh or observer separation. "
                                            "Equation residuals do not bound field quadrature.");
                    else
                        degree[b] = next[b];
                    all = all && done[b];
                }
                current = refined;
                if (all)
                    break;
            }
        }
        const double fieldMs = msSince(fieldStart);
        // Boundary data and impedances (cuda_solver.cu:1800-1846).
        std::vector<cplx> x(size_t(B) * E * N);
        cuda(cudaMemcpyAsync(x.data(), dX_.as<void>(), x.size() * 16, cudaMemcpyDeviceToHost, s), "trace download");
        cuda(cudaStreamSynchronize(s), "CUDA synchronization");
        for (uint32_t b = 0; b < B; ++b) {
            FrequencyResult &fr = result->frequencies[f0 + b];
            const double omega = 2 * M_PI * freqList[f0 + b];
            fr.frequency = freqList[f0 + b];
            fr.info.frequency = fr.frequency;
            fr.info.assembly_ms = assemblyMs / B;
            fr.info.factorization_ms = factorMs / B;
            fr.info.triangular_solve_ms = triMs / B;
            fr.info.residual_check_ms = residualMs / B;
            fr.info.solve_ms = (factorMs + triMs + residualMs) / B;
            fr.info.field_ms = fieldMs / B;
            fr.info.interaction_plan_ms = (f0 + b == 0) ? planMs : 0;
            fr.info.interaction_plan_reused = planMs == 0;
            const uint32_t Eout = coupling ? 1 : E;  // a coupled solve reports its one coupled field
            fr.excitations.resize(Eout);
            // coupled face velocities: each port's unit-flow velocities times its flow
            std::map<uint32_t, cplx> coupledFaces;
            if (coupling)
                for (uint32_t e = 0; e < E; ++e)
                    for (size_t i = r.excitation_face_offsets[e]; i < r.excitation_face_offsets[e + 1]; ++i)
                        coupledFaces[r.excitation_face_ids[i]] =
                            fr.portFlow[e] * cplx(r.excitation_velocities[2 * i], r.excitation_velocities[2 * i + 1]);
            for (uint32_t e = 0; e < Eout; ++e) {
                ExcitationResult &er = fr.excitations[e];
                const std::map<uint32_t, cplx> &velocities = coupling ? coupledFaces : faceVelocity[e];
                er.trace.assign(x.begin() + (size_t(b) * E + e) * N, x.begin() + (size_t(b) * E + e + 1) * N);
                er.residual = relative[size_t(b) * E + e];
                er.refinements = steps[b];
                er.iterations = krylov[size_t(b) * E + e];
                er.fieldDegree = fieldDeg[size_t(b) * E + e];
                er.fieldNext = fieldNext[size_t(b) * E + e];
                er.fieldDiscrepancy = fieldDisc[size_t(b) * E + e];
                er.surface.resize(T);
                er.normalDerivative.resize(T);
                for (uint32_t t = 0; t < T; ++t) {
                    const HostPanel &p = space_.panels[t];
                    cplx avg = 0;
                    for (int i = 0; i < 3; ++i)
                        avg += er.trace[p.nodes[i]] / 3.0;
                    if (!std::isfinite(avg.real()) || !std::isfinite(avg.imag()))
                        throw NumericError("Burton-Miller pressure is not finite.");
                    er.surface[t] = avg;
                    const auto it = velocities.find(p.face);
                    er.normalDerivative[t] = it == velocities.end() ? cplx(0) : cplx(0, -r.density * omega) * it->second;
                }
                if (coupling) {
                    // validateCouplingClosure (lem_coupling.cpp:97-120): the coupled field's
                    // power-dual mean pressure per port against the network's port pressure
                    std::vector<cplx> means(E, 0.0);
                    std::vector<double> mags(E, 0.0);
                    for (uint32_t t = 0; t < T; ++t)
                        if (panelPort[t] >= 0) {
                            const double w = space_.panels[t].area * panelUnitVelocity[t];
                            means[panelPort[t]] += w * er.surface[t];
                            mags[panelPort[t]] += w * std::abs(er.surface[t]);
                        }
                    for (uint32_t i = 0; i < E; ++i) {
                        const double scale = std::max(mags[i], std::abs(fr.portPressure[i]));
                        const double diff = std::abs(means[i] - fr.portPressure[i]);
                        if (!std::isfinite(scale) || !std::isfinite(diff) || diff > 1e-3 * scale)
                            throw NumericError("BEM and LEM port pressures fail the feedback consistency check.");
                    }
                }
                er.observer.assign(field.begin() + (size_t(b) * E + e) * O, field.begin() + (size_t(b) * E + e + 1) * O);
                std::vector<std::pair<uint32_t, cplx>> drive;
                if (coupling)
                    drive.assign(coupledFaces.begin(), coupledFaces.end());
                else
                    for (size_t i = r.excitation_face_offsets[e]; i < r.excitation_face_offsets[e + 1]; ++i)
                        drive.emplace_back(r.excitation_face_ids[i],
                                           cplx(r.excitation_velocities[2 * i], r.excitation_velocities[2 * i + 1]));
                for (const auto &[face, v] : drive) {
                    if (std::abs(v) == 0)
                        continue;
                    double area = 0;
                    cplx integrated = 0;
                    for (uint32_t t = 0; t < T; ++t)
                        if (space_.panels[t].face == face) {
                            area += space_.panels[t].area;
                            integrated += er.surface[t] * space_.panels[t].area;
                        }
                    const cplx mean = integrated / area, volume = v * area, z = mean / volume;
                    er.impedances.push_back(
                        {face, area, {mean.real(), mean.imag()}, {volume.real(), volume.imag()}, {z.real(), z.imag()}});
                }
            }
            if (progress) {
                hs_progress p{f0 + b + 1, Ftotal, fr.frequency, HS_PHASE_FREQUENCY_COMPLETE};
                progress(&p, user);
            }
            if (hooks && hooks->done)
                hooks->done(fr);
        }
    }
    timer_.stop(span, s);
    result->peakDeviceBytes = peakBytes_;
    return result;
}

// LEM coupling of one batch (cuda_solver.cu:1584-1667): per frequency the port
// impedance Z from the refined unit-flow basis solves (power-dual DP0 mean
// pressure at port i per unit flow at port j), the network's port flows, and the
// superposed pressure, right-hand side and flux of the coupled field written to
// excitation slot 0 (the other slots zeroed), ready for its own refinement with
// the retained factors.
void Session::coupleBatch(const CouplingNetwork &network, const std::vector<double> &freqList, uint32_t f0, uint32_t B,
                          uint32_t E, double density, const std::vector<int32_t> &panelPort,
                          const std::vector<double> &panelUnitVelocity, std::vector<FrequencyResult> &out) {
    (void)density;
    const cudaStream_t s = stream();
    const size_t N = space_.vertices.size(), T = space_.panels.size();
    std::vector<cplx> x(size_t(B) * E * N), b(size_t(B) * E * N), q(size_t(B) * E * T);
    cuda(cudaMemcpyAsync(x.data(), dX_.as<void>(), x.size() * 16, cudaMemcpyDeviceToHost, s), "coupling download");
    cuda(cudaMemcpyAsync(b.data(), dRhs_.as<void>(), b.size() * 16, cudaMemcpyDeviceToHost, s), "coupling download");
    cuda(cudaMemcpyAsync(q.data(), dFlux_.as<void>(), q.size() * 16, cudaMemcpyDeviceToHost, s), "coupling download");
    cuda(cudaStreamSynchronize(s), "CUDA coupling");
    for (uint32_t bb = 0; bb < B; ++bb) {
        std::vector<cplx> Z(size_t(E) * E, 0.0), Q, P;
        for (size_t t = 0; t < T; ++t) {
            const int port = panelPort[t];
            if (port < 0)
                continue;
            const HostPanel &pn = space_.panels[t];
            const double w = pn.area * panelUnitVelocity[t];
            for (uint32_t j = 0; j < E; ++j) {
                const cplx *xj = x.data() + (size_t(bb) * E + j) * N;
                Z[size_t(port) * E + j] += (xj[pn.nodes[0]] + xj[pn.nodes[1]] + xj[pn.nodes[2]]) / 3.0 * w;
            }
        }
        network(freqList[f0 + bb], Z, Q, P);
        if (Q.size() != E || P.size() != E)
            throw InvalidArgument("LEM result port count does not match its BEM basis.");
        for (uint32_t j = 0; j < E; ++j)
            if (!std::isfinite(Q[j].real()) || !std::isfinite(Q[j].imag()) || !std::isfinite(P[j].real()) ||
                !std::isfinite(P[j].imag()))
                throw NumericError("LEM port flows or pressures are not finite.");
        const auto superpose = [&](std::vector<cplx> &v, size_t n) {
            std::vector<cplx> sum(n, 0.0);
            for (uint32_t j = 0; j < E; ++j)
                for (size_t i = 0; i < n; ++i)
                    sum[i] += Q[j] * v[(size_t(bb) * E + j) * n + i];
            std::fill(v.begin() + size_t(bb) * E * n, v.begin() + size_t(bb + 1) * E * n, cplx(0));
            std::copy(sum.begin(), sum.end(), v.begin() + size_t(bb) * E * n);
        };
        superpose(x, N);
        superpose(b, N);
        superpose(q, T);
        FrequencyResult &fr = out[f0 + bb];
        fr.portImpedance = std::move(Z);
        fr.portFlow = std::move(Q);
        fr.portPressure = std::move(P);
    }
    cuda(cudaMemcpyAsync(dX_.as<void>(), x.data(), x.size() * 16, cudaMemcpyHostToDevice, s), "coupling upload");
    cuda(cudaMemcpyAsync(dRhs_.as<void>(), b.data(), b.size() * 16, cudaMemcpyHostToDevice, s), "coupling upload");
    cuda(cudaMemcpyAsync(dFlux_.as<void>(), q.data(), q.size() * 16, cudaMemcpyHostToDevice, s), "coupling upload");
    cuda(cudaStreamSynchronize(s), "CUDA coupling");
}

// Assembly, LU and initial solves of one frequency batch (launches only; the
// phase events are recorded with `eventFlags`, external inside a capture).
void Session::denseChain(const AssemblyGeometry &geo, const AssemblyWorkspace &ws, uint32_t B, uint32_t E, bool mixed,
                         cudaStream_t s, KernelTimer *timer, unsigned eventFlags) {
    const uint32_t N = geo.N;
    PhaseEvents &ev = phaseEvents();
    assembleBatch(geo, dKs_.as<double>(), dGauss_.as<double>(), dFlux_.as<double>(), E, B, ws, dA_.as<double>(),
                  dRhs_.as<double>(), dError_.as<int>(), s, timer, mixed);
    cuda(cudaEventRecordWithFlags(ev.assembled, s, eventFlags), "phase event");
    // LU of every matrix of the batch (FP64, or an FP32 copy in the mixed
    // form), then the initial solves.
    const size_t matrixReals = size_t(B) * N * N * 2, vectorReals = size_t(B) * E * N * 2;
    float *LU32 = dLU_.as<float>(), *work32 = dWork32_.as<float>();
    if (mixed) {
        {
            TimedScope scope(timer, "round_fp32", s);
            roundToFloat(dA_.as<double>(), LU32, matrixReals, s);
        }
        luFactorBatch(LU32, N, B, dPivots_.as<int>(), dInfo_.as<int>(), s, timer, dLuPack_.as<float>());
    } else {
        cuda(cudaMemcpyAsync(dLU_.as<void>(), dA_.as<void>(), matrixReals * 8, cudaMemcpyDeviceToDevice, s),
             "factorization copy");
        luFactorBatch(dLU_.as<double>(), N, B, dPivots_.as<int>(), dInfo_.as<int>(), s, timer);
    }
    cuda(cudaEventRecordWithFlags(ev.factored, s, eventFlags), "phase event");
    // the LU status is checked with the first residual norms
    if (mixed) {
        {
            TimedScope scope(timer, "round_fp32", s);
            roundToFloat(dRhs_.as<double>(), work32, vectorReals, s);
        }
        luSolveBatch(LU32, dPivots_.as<int>(), N, B, E, work32, dSolveScratch_.as<void>(), s, timer);
        cuda(cudaMemsetAsync(dX_.as<void>(), 0, vectorReals * 8, s), "solution reset");
        TimedScope scope(timer, "add_correction", s);
        addCorrectionBatch(dX_.as<double>(), work32, vectorReals, s);
    } else {
        cuda(cudaMemcpyAsync(dX_.as<void>(), dRhs_.as<void>(), vectorReals * 8, cudaMemcpyDeviceToDevice, s),
             "rhs copy");
        luSolveBatch(dLU_.as<double>(), dPivots_.as<int>(), N, B, E, dX_.as<double>(), dSolveScratch_.as<void>(), s,
                     timer);
    }
    cuda(cudaEventRecordWithFlags(ev.solved, s, eventFlags), "phase event");
}

// The dense chain of a batch shape (B, E, form) is captured as a CUDA graph on
// its second use with the same workspaces and plan, and replayed from then on.
// With kernel profiling on the chain runs as plain launches, so that every
// kernel family keeps its own timing.
void Session::runDenseChain(const AssemblyGeometry &geo, const AssemblyWorkspace &ws, uint32_t B, uint32_t E,
                            bool mixed, cudaStream_t s) {
    const bool capturable = s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread;
    if (!graphs_ || timer_.enabled() || !capturable) {
        denseChain(geo, ws, B, E, mixed, s, &timer_, cudaEventRecordDefault);
        return;
    }
    // a graph is valid while every buffer it captured sits at the same address
    // (buffers only grow, so the captured extents stay inside them)
    uint64_t signature = generation_ * 0x9e3779b97f4a7c15ull;
    for (const DeviceBuffer *b :
         {&dPanels_, &dBounds_, &dMixedPanels_, &dIncOffsets_, &dIncPanel_, &dIncLocal_, &dRowScale_, &dError_,
          &dPairCode_, &dTouching_, &dNearPairs_, &dPatches_, &dGauss_, &dSingularTable_, &dRecords_, &dColumns_,
          &dPanelRhs_, &dBins_, &dBinCounts_, &dBinOffsets_, &dA_, &dLU_, &dRhs_, &dX_, &dPivots_, &dInfo_, &dKs_,
          &dFlux_, &dWork32_, &dLuPack_, &dSolveScratch_})
        signature = (signature ^ reinterpret_cast<uintptr_t>(b->as<void>())) * 0x100000001b3ull;
    signature = (signature ^ reinterpret_cast<uintptr_t>(patches_)) * 0x100000001b3ull;
    DenseGraph *hit = nullptr;
    for (auto &g : denseGraphs_)
        if (g.B == B && g.E == E && g.mixed == mixed && g.signature == signature)
            hit = &g;
    if (!hit) {
        // graphs of superseded buffers are released
        for (auto &g : denseGraphs_)
            if (g.signature != signature && g.exec) {
                cudaGraphExecDestroy(g.exec);
                g.exec = nullptr;
            }
        std::erase_if(denseGraphs_, [&](const DenseGraph &g) { return g.signature != signature; });
        denseGraphs_.push_back({B, E, mixed, signature, 0, nullptr});
        hit = &denseGraphs_.back();
    }
    if (!hit->exec && hit->uses++ == 0) {
        denseChain(geo, ws, B, E, mixed, s, &timer_, cudaEventRecordDefault);
        return;
    }
    if (!hit->exec) {
        cudaGraph_t g = nullptr;
        cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "dense chain capture");
        try {
            denseChain(geo, ws, B, E, mixed, s, nullptr, cudaEventRecordExternal);
        } catch (...) {
            cudaStreamEndCapture(s, &g);
            if (g)
                cudaGraphDestroy(g);
            throw;
        }
        cuda(cudaStreamEndCapture(s, &g), "dense chain capture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        cuda(e, "dense chain graph instantiation");
        hit->exec = exec;
    }
    cuda(cudaGraphLaunch(hit->exec, s), "dense chain graph launch");
    ++graphLaunches_;
}

void Session::dropGraphs() {
    for (auto &g : denseGraphs_)
        if (g.exec)
            cudaGraphExecDestroy(g.exec);
    denseGraphs_.clear();
    ++generation_;
}

void Session::setPlaneWaveThreshold(double threshold) {
    planeWaveThreshold_ = threshold;
    if (fmm_)
        fmm_->setHfThreshold(threshold);
}

void Session::setPlanner(uint32_t planner) {
    if (planner != HS_PLANNER_DEVICE && planner != HS_PLANNER_HOST)
        throw InvalidArgument("Interaction planner must be HS_PLANNER_DEVICE or HS_PLANNER_HOST.");
    planner_ = planner;
}

void Session::setGroupedM2l(bool enabled) {
    groupedM2l_ = enabled;
    if (fmm_)
        fmm_->setGroupedM2l(enabled);
    if (fmmInner_)
        fmmInner_->setGroupedM2l(enabled);
}

void Session::setGraphs(bool enabled) {
    graphs_ = enabled;
    dropGraphs();
    if (fmm_)
        fmm_->setGraphs(enabled);
    if (fmmInner_)
        fmmInner_->setGraphs(enabled);
}

void Session::debugAssemble(const hs_numerics &o, double planK, double k, const double *flux, double *matrix,
                            double *rhs) {
    preparePlan(o, planK, nullptr);
    const uint32_t T = uint32_t(space_.panels.size()), N = uint32_t(space_.vertices.size());
    ensureWorkspace(1, 1, 0, o.precision == HS_PRECISION_MIXED, o.fmm_restart_length);
    const cudaStream_t s = stream();
    cuda(cudaMemcpyAsync(dKs_.as<void>(), &k, 8, cudaMemcpyHostToDevice, s), "k upload");
    cuda(cudaMemcpyAsync(dFlux_.as<void>(), flux, size_t(T) * 16, cudaMemcpyHostToDevice, s), "flux upload");
    AssemblyGeometry geo{dPanels_.as<DPanel>(), dBounds_.as<Bounds>(), dPairCode_.as<uint8_t>(),
                         dTouching_.as<TouchingJob>(), dNearPairs_.as<NearPairJob>(), patches_,
                         dIncOffsets_.as<uint32_t>(), dIncPanel_.as<uint32_t>(), dIncLocal_.as<uint8_t>(),
                         dRowScale_.as<double>(), T, N, touchingCount_, nearPairCount_, projectedPairCount_,
                         o.near_relative_tolerance,
                         o.quadrature_order, o.singular_order, dSingularTable_.as<float4>(),
                         dMixedPanels_.as<MixedPanel>()};
    AssemblyWorkspace ws{dRecords_.as<void>(), dColumns_.as<void>(), dPanelRhs_.as<double>(), dBins_.as<uint2>(),
                         dBinCounts_.as<uint32_t>(), size_t(T) * (T - 1) / 2,
                         T > kExactBinsT ? dBinOffsets_.as<uint64_t>() : nullptr};
    assembleBatch(geo, dKs_.as<double>(), dGauss_.as<double>(), dFlux_.as<double>(), 1, 1, ws, dA_.as<double>(),
                  dRhs_.as<double>(), dError_.as<int>(), s, &timer_, o.precision == HS_PRECISION_MIXED);
    checkDeviceError("CUDA Galerkin assembly");
    cuda(cudaMemcpyAsync(matrix, dA_.as<void>(), size_t(N) * N * 16, cudaMemcpyDeviceToHost, s), "matrix download");
    cuda(cudaMemcpyAsync(rhs, dRhs_.as<void>(), size_t(N) * 16, cudaMemcpyDeviceToHost, s), "rhs download");
    cuda(cudaStreamSynchronize(s), "CUDA synchronization");
}

// Expansion tolerance the leaf-size tuning measures at: the working tolerance
// of the solve (1 % of its residual target, as in the batch loop).
double Session::fmmTuneTolerance(const hs_numerics &o) {
    return std::clamp(.01 * o.relative_residual_tolerance, 1e-10, 1e-6);
}

void Session::ensureFmmWorkspace(const hs_numerics &o, uint32_t E, uint32_t O, double maxK) {
    const size_t T = space_.panels.size(), N = space_.vertices.size();
    FmmOperator &op = fmmOperator(o, maxK, fmmTuneTolerance(o));
    if (!fmmSystem_ || fmmSystemOp_ != &op || fmmBlockWidth_ != o.fmm_preconditioner_block_width) {
        fmmSystem_.reset();
        fmmBlockWidth_ = o.fmm_preconditioner_block_width;
        fmmSystem_ = std::make_unique<FmmSystem>(op, dRowScale_.as<double>(), dMass_.as<double>(),
                                                 o.fmm_preconditioner_block_width);
        fmmSystemOp_ = &op;
        const cudaStream_t s = stream();
        const auto put = [&](DeviceBuffer &b, const void *src, size_t bytes) {
            b.ensure(std::max<size_t>(bytes, 16));
            if (bytes)
                cuda(cudaMemcpyAsync(b.as<void>(), src, bytes, cudaMemcpyHostToDevice, s), "near panel upload");
        };
        put(dPanelRow_, op.nearPanelRow().data(), op.nearPanelRow().size() * 4);
        put(dPanelCol_, op.nearPanelCol().data(), op.nearPanelCol().size() * 4);
        put(dPanelPairs_, op.nearPanelPairs().data(), op.nearPanelPairs().size() * 8);
        cuda(cudaStreamSynchronize(s), "near panel upload");
    }
    dNearWork_.ensure(nearFieldWorkspaceBytes(op.nearPanelCol().size(), op.nearPanelPairs().size()));
    dAuditWork_.ensure(E * N * 16);
    dAuditFine_.ensure(E * N * 16);
    dNearRhs_.ensure(E * N * 16);
    dAuditB_.ensure(E * N * 16);
    dRhs_.ensure(E * N * 16);
    dX_.ensure(E * N * 16);
    dCorr_.ensure(E * N * 16);
    dNorms_.ensure(2 * E * 8 + 2 * E * N * 8);
    dBinCounts_.ensure(kBins * sizeof(uint32_t));
    dKs_.ensure(8);
    dFlux_.ensure(E * T * 16);
    dObservers_.ensure(std::max<size_t>(O * 3 * 8, 16));
    dPartials_.ensure(std::max<size_t>(fieldPartialsBytes(uint32_t(T), E, O, 1), 16));
    dField_.ensure(std::max<size_t>(E * O * 16, 16));
    dDegrees_.ensure(4);
    size_t bytes = 0;
    for (const DeviceBuffer *b : {&dPanels_, &dBounds_, &dMixedPanels_, &dIncOffsets_, &dIncPanel_, &dIncLocal_, &dRowScale_,
                                  &dMass_, &dPairCode_, &dTouching_, &dNearPairs_, &dPatches_, &dGauss_, &dSingularTable_,
                                  &dNearWork_, &dPanelRow_, &dPanelCol_, &dPanelPairs_, &dRhs_, &dX_, &dCorr_, &dNorms_,
                                  &dKs_, &dFlux_, &dObservers_, &dPartials_, &dField_, &dDegrees_})
        bytes += b->bytes();
    peakBytes_ = std::max(peakBytes_, bytes);
}

FmmOperator &Session::fmmOperator(const hs_numerics &o, double tuneK, double tuneTolerance) {
    FmmTreeSettings st;
    st.leafCapacity = o.fmm_leaf_support_capacity ? o.fmm_leaf_support_capacity : 32;
    st.separationRatio = std::isfinite(o.fmm_separation_ratio) && o.fmm_separation_ratio > 1 ? o.fmm_separation_ratio : 1.5;
    if (o.fmm_leaf_support_capacity == 0 && tuneK > 0)
        st.leafCapacity = tunedLeafCapacity(st.separationRatio, tuneK, tuneTolerance);
    if (!fmm_ || st.leafCapacity != fmmSettings_.leafCapacity || st.separationRatio != fmmSettings_.separationRatio) {
        fmmSystem_.reset();
        fmmSystemOp_ = nullptr;
        fmm_.reset();
        fmm_ = std::make_unique<FmmOperator>(space_, st);
        fmm_->setGraphs(graphs_);
        fmm_->setHfThreshold(planeWaveThreshold_);
        fmm_->setGroupedM2l(groupedM2l_);
        fmmSettings_ = st;
    }
    return *fmm_;
}

// Whether the direct Galerkin audit is cheaper than two expansion operators
// (preferSupportDirectAudit, support_fmm_solve.cu:79-114, restated): dense
// regular work T^2 (9 + q^2 (13 + 1/r)) with q the panel rule's points and r
// the FP32:FP64 throughput ratio, against, per far level, the pairs times the
// rotation-coaxial-rotation work (or the plane-wave samples) plus the O(n^4)
// coaxial preparation per distance class; at most 20 000 panels.
bool Session::preferDirectAudit(const FmmOperator &op) const {
    const size_t T = space_.panels.size(), N = space_.vertices.size();
    if (fmmAuditMode_ == 2)
        return true;
    if (!T || T > 20000 || op.levels().empty() || fmmAuditMode_ == 1)
        return false;
    size_t freeBytes = 0, totalBytes = 0;  // the dense system must fit beside the fast-multipole state
    if (cudaMemGetInfo(&freeBytes, &totalBytes) != cudaSuccess ||
        recordBytes(uint32_t(T), false) + 2 * N * N * 16 > freeBytes / 2)
        return false;
    const long double q = 6, ratio = 2;  // degree-4 Dunavant rule; B200 FP32 : FP64
    const long double direct = (long double)T * T * (9.L + q * q * (13.L + 1.L / ratio));
    const FmmTree &tree = op.tree();
    std::vector<long double> pairs(tree.levels.size(), 0);
    for (const auto *list : {&tree.ppFar, &tree.pfFar})
        for (const auto &lk : *list)
            pairs[tree.nodes[lk.target].level] += 1;
    long double multipole = 0;
    for (const auto &lv : op.levels()) {
        const long double p = lv.order, n = p + 1;
        if (lv.planeWave)
            multipole += pairs[lv.level] * 2.L * (1.5L * p + 1) * (3 * p + 2);
        else {
            const long double rotation = n * (4 * p * p + 8 * p + 3) / 3, axial = n * n + p * n * (2 * p + 1) / 3;
            multipole += pairs[lv.level] * (2 * rotation + axial) + n * n * n * n;
        }
    }
    return direct <= 2 * multipole;
}

// The exact FP64 dense system of one frequency for the direct audit: matrix
// into dA_, right-hand side into dAuditB_ (the dense assembly of the plain form).
void Session::directAuditSystem(const AssemblyGeometry &geo, double k, const double *flux, uint32_t E, double *&A,
                                double *&b) {
    (void)k;
    const uint32_t T = geo.T;
    ensureWorkspace(1, E, 0, false, 2);
    AssemblyWorkspace ws{dRecords_.as<void>(), dColumns_.as<void>(), dPanelRhs_.as<double>(), dBins_.as<uint2>(),
                         dBinCounts_.as<uint32_t>(), size_t(T) * (T - 1) / 2,
                         T > kExactBinsT ? dBinOffsets_.as<uint64_t>() : nullptr};
    assembleBatch(geo, dKs_.as<double>() + directAuditFrequency_, dGauss_.as<double>(), flux, E, 1, ws,
                  dA_.as<double>(), dAuditB_.as<double>(), dError_.as<int>(), stream(), nullptr, false);
    A = dA_.as<double>();
    b = dAuditB_.as<double>();
}

// The mixed form's inner operator: the same tree and partition as the FP64
// operator (built from the same settings), translations in FP32 on scaled
// expansions.
FmmOperator &Session::fmmInnerOperator(const hs_numerics &o) {
    if (!fmmInner_ || fmmInnerSettings_.leafCapacity != fmmSettings_.leafCapacity ||
        fmmInnerSettings_.separationRatio != fmmSettings_.separationRatio) {
        fmmInner_.reset();
        fmmInner_ = std::make_unique<FmmOperator>(space_, fmmSettings_);
        fmmInner_->setFp32(true);
        fmmInner_->setGraphs(graphs_);
        fmmInner_->setGroupedM2l(groupedM2l_);
        fmmInnerSettings_ = fmmSettings_;
    }
    (void)o;
    return *fmmInner_;
}

// Leaf support capacity of the fast-multipole tree picked by the autotuner
// (requests with capacity 0): per mesh size class and electrical size class,
// each candidate tree is built and its operator apply (far expansions plus the
// near product) timed at the request's top wavenumber; the fastest is kept for
// the class. The leaf size moves work between the exact near part and the
// expansions, so results differ between candidates within the expansion
// tolerance, as for any explicit capacity.
uint32_t Session::tunedLeafCapacity(double separation, double k, double tolerance) {
    static constexpr uint32_t kCandidates[] = {8, 16, 32};
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (const auto &v : space_.vertices)
        for (int d = 0; d < 3; ++d) {
            const double x = d == 0 ? v.x : d == 1 ? v.y : v.z;
            lo[d] = std::min(lo[d], x);
            hi[d] = std::max(hi[d], x);
        }
    const double diameter = std::hypot(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    const uint32_t T = uint32_t(space_.panels.size());
    const int kd = int(std::floor(std::log2(std::max(1.0, k * diameter))));
    const std::string key = "fmm_leaf_T2^" + std::to_string(31 - __builtin_clz(T | 1u)) + "_kD2^" + std::to_string(kd) +
                            "_sep" + std::to_string(int(std::lround(separation * 10)));
    Autotuner &tuner = Autotuner::instance();
    const int known = tuner.choice(key);
    if (known >= 0)
        return kCandidates[known];
    if (!tuner.enabled() || timer_.enabled())
        return 16;
    const cudaStream_t s = stream();
    const size_t N = space_.vertices.size();
    DeviceBuffer in, out;
    in.ensure(N * 16);
    out.ensure(N * 16);
    cuda(cudaMemsetAsync(in.as<void>(), 0, N * 16, s), "tuning input");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cuda(cudaEventCreate(&e0), "tuning event");
    cuda(cudaEventCreate(&e1), "tuning event");
    std::vector<double> ms;
    int best = 0;
    try {
        for (uint32_t cap : kCandidates) {
            FmmTreeSettings st;
            st.leafCapacity = cap;
            st.separationRatio = separation;
            FmmOperator op(space_, st);
            FmmSystem system(op, dRowScale_.as<double>(), dMass_.as<double>(), 32);
            cuda(cudaMemsetAsync(system.nearValues(), 0, std::max<size_t>(op.nearCols().size(), 1) * 16, s),
                 "tuning near values");
            op.setGraphs(false);
            op.prepare(k, tolerance, s);
            system.apply(in.as<double>(), 2 * N, 1, out.as<double>(), s, nullptr);  // warm-up
            cuda(cudaEventRecord(e0, s), "tuning event");
            system.apply(in.as<double>(), 2 * N, 1, out.as<double>(), s, nullptr);
            cuda(cudaEventRecord(e1, s), "tuning event");
            cuda(cudaEventSynchronize(e1), "tuning");
            float t = 0;
            cuda(cudaEventElapsedTime(&t, e0, e1), "tuning time");
            ms.push_back(t);
            if (t < ms[size_t(best)])
                best = int(ms.size() - 1);
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tuner.record(key, best, ms);
    return kCandidates[best];
}

void Session::debugFmmFar(const hs_numerics &o, double k, double tolerance, const double *pressure, double *far,
                          std::vector<uint32_t> &nearRow, std::vector<uint32_t> &nearCol,
                          std::vector<FmmLevelInfo> &levels) {
    // HS_PRECISION_MIXED: the mixed form's FP32 operator on the same tree
    FmmOperator &op = o.precision == HS_PRECISION_MIXED ? (fmmOperator(o), fmmInnerOperator(o)) : fmmOperator(o);
    const cudaStream_t s = stream();
    const size_t N = space_.vertices.size();
    op.prepare(k, tolerance, s);
    dFmmIn_.ensure(N * 16);
    dFmmOut_.ensure(N * 16);
    cuda(cudaMemcpyAsync(dFmmIn_.as<void>(), pressure, N * 16, cudaMemcpyHostToDevice, s), "pressure upload");
    op.applyFar(dFmmIn_.as<double>(), 2 * N, 1, dFmmOut_.as<double>(), s, &timer_);
    cuda(cudaMemcpyAsync(far, dFmmOut_.as<void>(), N * 16, cudaMemcpyDeviceToHost, s), "far download");
    cuda(cudaStreamSynchronize(s), "CUDA fast multipole");
    for (size_t i = 0; i < N; ++i) {  // row equilibration 1 / lumped mass
        far[2 * i] /= space_.lumpedMass[i];
        far[2 * i + 1] /= space_.lumpedMass[i];
    }
    nearRow = op.nearRowStart();
    nearCol = op.nearCols();
    levels = op.levels();
}

}  // namespace hsb
