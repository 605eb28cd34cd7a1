// Solver session: one validated mesh with its device geometry, cached
// interaction plan and reusable device workspaces
// (CudaBemSolver::Implementation, cuda_solver.cu:742-987).
#pragma once

#include "device_types.cuh"
#include "fmm.hpp"
#include "hs_bem.h"
#include "kernel_timer.hpp"
#include "plan_device.hpp"
#include "planner.hpp"

#include <complex>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace hsb {

class DeviceBuffer {
  public:
    DeviceBuffer() = default;
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    void *ensure(size_t bytes);  // grows (never shrinks) the allocation
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr_); }
    size_t bytes() const { return bytes_; }

  private:
    void *ptr_ = nullptr;
    size_t bytes_ = 0;
};

using cplx = std::complex<double>;

struct ExcitationResult {
    std::vector<cplx> trace, surface, normalDerivative, observer;
    double residual{};
    uint32_t refinements{}, iterations{}, fieldDegree{}, fieldNext{};
    double fieldDiscrepancy{};
    std::vector<hs_face_impedance> impedances;
};
struct FrequencyResult {
    double frequency{};
    hs_frequency_info info{};
    std::vector<ExcitationResult> excitations;
    // LEM-coupled solves: port impedance Z (ports x ports, row i col j) and the
    // network's port flows and pressures
    std::vector<cplx> portImpedance, portFlow, portPressure;
};
struct Result {
    size_t T{}, N{}, O{}, E{}, peakDeviceBytes{};
    std::vector<FrequencyResult> frequencies;
};

// Continuous batching hooks of a solve (serving): before each frequency batch
// `more` may hand in further frequencies (solved next, ahead of the remaining
// ones; they must lie within the solve's interaction plan), and `done` sees
// every frequency result as soon as its batch completes.
struct SolveHooks {
    std::function<std::vector<double>()> more;
    std::function<void(const FrequencyResult &)> done;
};

// The lumped network of a coupled solve (lem::solve in the reference): from the
// frequency and the port impedance matrix Z (ports x ports, row i col j: mean
// pressure at port i per unit flow at port j) the port flows Q and pressures P.
using CouplingNetwork = std::function<void(double frequency, const std::vector<cplx> &Z, std::vector<cplx> &Q,
                                           std::vector<cplx> &P)>;

class Session {
  public:
    Session(const MeshInput &mesh, uint32_t residency);
    ~Session();
    void setStream(cudaStream_t stream);
    std::unique_ptr<Result> solve(const hs_request &request, const volatile int32_t *cancel, hs_progress_fn progress,
                                  void *user, const SolveHooks *hooks = nullptr,
                                  const CouplingNetwork *coupling = nullptr);
    const Plan &plan(const hs_numerics &numerics, double maxK, const volatile int32_t *cancel);
    void debugAssemble(const hs_numerics &numerics, double planK, double k, const double *flux, double *matrix,
                       double *rhs);
    // Far part of the fast-multipole operator (row-equilibrated like the dense
    // matrix) applied to a P1 vector, with the near support-pair pattern.
    void debugFmmFar(const hs_numerics &numerics, double k, double tolerance, const double *pressure, double *far,
                     std::vector<uint32_t> &nearRow, std::vector<uint32_t> &nearCol,
                     std::vector<FmmLevelInfo> &levels);
    KernelTimer &timer() { return timer_; }
    // Replay of the per-batch dense chain and of the fast-multipole far-field
    // apply as captured CUDA graphs (on by default); graph launches so far.
    void setGraphs(bool enabled);
    void setPlaneWaveThreshold(double threshold);
    void setGroupedM2l(bool enabled);
    // Interaction planner: on the device (default) or the host's threads;
    // both give the same plan bit for bit. The statistics are the last device
    // plan's.
    void setPlanner(uint32_t planner);
    const DevicePlanStats &planStats() const { return planStats_; }
    uint64_t graphLaunches() const { return graphLaunches_; }
    // Device bytes a solve may hold beyond the resident geometry and plan
    // (0: 60 % of free memory); bounds the frequency batch.
    void setMemoryBudget(size_t bytes) { memoryBudget_ = bytes; }
    // Pressure samples at world points from a solution's traces (hs_bem_pressure_field).
    void pressureField(double frequency, double soundSpeed, const double *trace, const double *normalDerivative,
                       const double *points, size_t count, const hs_field_settings &settings, double *pressure,
                       int32_t *status);
    // Device bytes held now (geometry, plan and grown workspaces).
    size_t residentBytes() const;
    // regular pairs per bin (4), regular samples, touching samples, near samples, frequencies
    std::vector<uint64_t> work = std::vector<uint64_t>(8, 0);
    std::mutex mutex;

  private:
    struct Batch;
    void uploadGeometry();
    void preparePlan(const hs_numerics &numerics, double maxK, const volatile int32_t *cancel);
    void ensureWorkspace(uint32_t B, uint32_t E, uint32_t O, bool mixed, uint32_t restart);
    uint32_t chooseBatch(uint32_t F, uint32_t E, uint32_t O, bool mixed, uint32_t restart) const;
    void checkDeviceError(const char *where);
    // Events at the phase boundaries of a frequency batch (created on first use).
    struct PhaseEvents {
        cudaEvent_t batch{}, assembled{}, factored{}, solved{}, refine0{}, refine1{};
    };
    PhaseEvents &phaseEvents();
    PhaseEvents phase_{};
    bool phaseReady_ = false;
    cudaStream_t stream() const { return external_ ? external_ : own_; }
    void denseChain(const AssemblyGeometry &geo, const AssemblyWorkspace &ws, uint32_t B, uint32_t E, bool mixed,
                    cudaStream_t s, KernelTimer *timer, unsigned eventFlags);
    void runDenseChain(const AssemblyGeometry &geo, const AssemblyWorkspace &ws, uint32_t B, uint32_t E, bool mixed,
                       cudaStream_t s);
    void dropGraphs();
    void coupleBatch(const CouplingNetwork &network, const std::vector<double> &freqList, uint32_t f0, uint32_t B,
                     uint32_t E, double density, const std::vector<int32_t> &panelPort,
                     const std::vector<double> &panelUnitVelocity, std::vector<FrequencyResult> &out);
    struct DenseGraph {
        uint32_t B, E;
        bool mixed;
        uint64_t signature;
        uint32_t uses;
        cudaGraphExec_t exec;
    };
    std::vector<DenseGraph> denseGraphs_;
    uint64_t generation_ = 0, graphLaunches_ = 0;
    bool graphs_ = true;
    double planeWaveThreshold_ = 8.0;
    bool groupedM2l_ = true;

    MeshInput mesh_;
    V3 origin_{};
    Space space_;
    uint32_t residency_;
    cudaStream_t own_ = nullptr, external_ = nullptr;
    KernelTimer timer_;

    // geometry (frequency independent)
    DeviceBuffer dSamplePoints_, dSampleTrace_, dSampleFlux_, dSampleOut_, dSampleStatus_;
    DeviceBuffer dPanels_, dBounds_, dMixedPanels_, dIncOffsets_, dIncPanel_, dIncLocal_, dRowScale_, dMass_, dError_;
    // plan cache
    bool planValid_ = false;
    hs_numerics planNumerics_{};
    double planK_ = -1;
    Plan plan_;
    double planMs_ = 0;
    uint32_t planner_ = HS_PLANNER_DEVICE;
    DevicePlanStats planStats_;
    DeviceBuffer dPairCode_, dTouching_, dNearPairs_, dPatches_, dGauss_, dSingularTable_;
    // patches as the kernels see them: dPatches_, or the device alias of mapped
    // pinned host memory (residency)
    const Patch *patches_ = nullptr;
    void *mappedPatchesHost_ = nullptr;
    void releaseMappedPatches();
public:
    bool patchesMapped() const { return mappedPatchesHost_ != nullptr; }
private:
    uint32_t touchingCount_ = 0, nearPairCount_ = 0, projectedPairCount_ = 0;
    uint64_t singularSamples_ = 0, nearSamples_ = 0;
    // workspaces (grow only)
    DeviceBuffer dRecords_, dColumns_, dPanelRhs_, dBins_, dBinCounts_, dBinOffsets_, dA_, dLU_, dRhs_, dX_, dCorr_, dNorms_,
        dPivots_, dInfo_, dKs_, dFlux_, dObservers_, dPartials_, dField_, dDegrees_, dWork32_, dGmres_, dLuPack_, dSolveScratch_;
    size_t peakBytes_ = 0;
    size_t memoryBudget_ = 0;
    // fast-multipole form: operator on the support tree (built on first use
    // for a tree setting) and its workspaces
    // tuneK > 0: a capacity of 0 asks the autotuner (at wavenumber tuneK and
    // expansion tolerance tuneTolerance) for the leaf size.
    FmmOperator &fmmOperator(const hs_numerics &numerics, double tuneK = 0, double tuneTolerance = 1e-8);
    uint32_t tunedLeafCapacity(double separation, double k, double tolerance);
    static double fmmTuneTolerance(const hs_numerics &numerics);
    std::unique_ptr<FmmOperator> fmm_, fmmInner_;
    FmmTreeSettings fmmInnerSettings_{};
    FmmOperator &fmmInnerOperator(const hs_numerics &numerics);
    bool preferDirectAudit(const FmmOperator &op) const;
    void directAuditSystem(const AssemblyGeometry &geo, double k, const double *flux, uint32_t E, double *&A,
                           double *&b);
    uint32_t directAuditFrequency_ = 0;
    DeviceBuffer dNearRhs_, dAuditB_;
  public:
    // fast-multipole audit evidence of the session: direct audits, panel-rule promotions
    uint64_t directAudits_ = 0, quadraturePromotions_ = 0;
    // 0: the reference's policy (direct audit where cheaper), 1: expansion and
    // panel-rule audits only, 2: direct audit always
    uint32_t fmmAuditMode_ = 0;
  private:
    std::unique_ptr<FmmSystem> fmmSystem_;
    const FmmOperator *fmmSystemOp_ = nullptr;
    uint32_t fmmBlockWidth_ = 0;
    FmmTreeSettings fmmSettings_{};
    DeviceBuffer dFmmIn_, dFmmOut_, dNearWork_, dPanelRow_, dPanelCol_, dPanelPairs_, dAuditWork_, dAuditFine_;
    void ensureFmmWorkspace(const hs_numerics &numerics, uint32_t E, uint32_t O, double maxK);
};

// Device bytes of one solve of F frequencies on a mesh with T panels and N
// vertices, batched B at a time: workspace of the batch plus the session's
// geometry and plan (for admission before a session exists).
size_t solveFootprint(size_t T, size_t N, uint32_t E, uint32_t O, uint32_t B, bool mixed, uint32_t restart);
// The same for the fast-multipole form (one frequency at a time, sparse near field).
size_t fmmSolveFootprint(size_t T, size_t N, uint32_t E, uint32_t O, uint32_t restart);

}  // namespace hsb
