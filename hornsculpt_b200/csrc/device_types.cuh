// Device-resident data layout of a solver session and the launch interface
// of the sm_100a kernels (assembly.cu, dense_lu.cu, field.cu).
#pragma once

#include "pair_rules.cuh"

#include <cstddef>
#include <cstdint>
#include <functional>
#include <vector>
#include <cuda_runtime.h>

namespace hsb {

// One flat panel in HBM (200 B): local-origin vertex 0, edge vectors, unit
// normal, P1 surface curls, area, longest edge and node ids.
struct DPanel {
    double v0[3], e1[3], e2[3], n[3];
    double curl[9];
    double area, maxEdge;
    uint32_t nodes[3], pad;
};

// Pair-block record of one ordered (test, trial) panel pair: the 3x3 P1xP1
// Burton-Miller block (curl term included) and the 3 P1xDP0 right-hand-side
// moments, 12 complex values (24 reals: FP64 in the plain form, FP32 in the
// mixed form). Slot = trial * T + test. A frequency's records form four
// planes of T*T slots with 3 complex values each: plane j < 3 holds column j
// of the block (rows i = 0..2), plane 3 the right-hand-side moments, so the
// trial-vertex gather reads one contiguous column per (trial, test) slot and
// consecutive test panels are adjacent.
constexpr int kRecordDoubles = 24;

// Offset (in reals) of record element e of a slot: e < 9 is block entry
// (row e / 3, column e % 3), e >= 9 right-hand-side row e - 9.
HS_HD size_t recordOffset(uint32_t T, size_t slot, int e) {
    const int plane = e < 9 ? e % 3 : 3, row = e < 9 ? e / 3 : e - 9;
    return ((size_t(plane) * T * T + slot) * 3 + row) * 2;
}

// Stored (test, trial) slots of the record planes: all T*T ordered pairs
// (row == nullptr, slot = trial * T + test) or, for the fast-multipole near
// field, the pairs of a CSR over test panels (columns sorted), slot = the
// CSR position. planeSlots: slots per plane (T*T or the CSR size).
struct SlotMap {
    const uint32_t *row = nullptr, *col = nullptr;
    size_t planeSlots = 0;
};
constexpr size_t kNoSlot = ~size_t(0);
HS_HD size_t mapSlot(const SlotMap &m, uint32_t T, uint32_t test, uint32_t trial) {
    if (!m.row)
        return size_t(trial) * T + test;
    uint32_t lo = m.row[test], hi = m.row[test + 1];
    const uint32_t end = hi;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (m.col[mid] < trial)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < end && m.col[lo] == trial ? size_t(lo) : kNoSlot;
}
// Offset (in reals) of record element e of a slot in a plane set of planeSlots slots.
HS_HD size_t mapOffset(size_t planeSlots, size_t slot, int e) {
    const int plane = e < 9 ? e % 3 : 3, row = e < 9 ? e / 3 : e - 9;
    return ((size_t(plane) * planeSlots + slot) * 3 + row) * 2;
}

// Device error word codes (cuda_solver.cu:705-715).
enum DeviceError : int {
    kErrDistance = 1,      // zero or invalid source distance
    kErrNonFinite = 2,     // non-finite assembled value
    kErrFieldDepth = 3,    // observer near field missed its tolerance
    kErrEscapedPlan = 4,   // regular pair without a qualified rule
};

// Unordered-pair codes of the session plan.
enum PairCode : uint8_t { kPairRegular = 0, kPairTouching = 1, kPairNear = 2, kPairWhole8 = 8, kPairWhole14 = 14 };

// Regular-rule bins: Dunavant degree 4 (6 pts), 6 (12), 8 (16) and the
// collapsed tensor degree-14 rule (64 pts) of accepted whole-panel pairs.
constexpr int kBins = 4;
constexpr int kBinPoints[kBins] = {6, 12, 16, 64};

struct NearPairJob {
    uint32_t first, second, firstPatch, patchCount;
};
struct TouchingJob {
    uint32_t test, trial;
    uint32_t topology;
    uint8_t permTest[3], permTrial[3], pad[2];
};

// FP32 view of a panel for the mixed form (112 B): first vertex minus the
// bounding-ball centre and the area, the edges e1 = v1 - v0, e2 = v2 - v0
// with |e1|^2 and |e2|^2, the normal with e1.e2, and the P1 basis curls.
struct MixedPanel {
    float4 offset, e1, e2, n;
    float4 curl[3];
};

inline MixedPanel makeMixedPanel(const DPanel &p, const Bounds &b) {
    MixedPanel m{};
    const double o[3] = {p.v0[0] - b.center.x, p.v0[1] - b.center.y, p.v0[2] - b.center.z};
    const double e11 = p.e1[0] * p.e1[0] + p.e1[1] * p.e1[1] + p.e1[2] * p.e1[2];
    const double e22 = p.e2[0] * p.e2[0] + p.e2[1] * p.e2[1] + p.e2[2] * p.e2[2];
    const double e12 = p.e1[0] * p.e2[0] + p.e1[1] * p.e2[1] + p.e1[2] * p.e2[2];
    m.offset = make_float4(float(o[0]), float(o[1]), float(o[2]), float(p.area));
    m.e1 = make_float4(float(p.e1[0]), float(p.e1[1]), float(p.e1[2]), float(e11));
    m.e2 = make_float4(float(p.e2[0]), float(p.e2[1]), float(p.e2[2]), float(e22));
    m.n = make_float4(float(p.n[0]), float(p.n[1]), float(p.n[2]), float(e12));
    for (int i = 0; i < 3; ++i)
        m.curl[i] = make_float4(float(p.curl[3 * i]), float(p.curl[3 * i + 1]), float(p.curl[3 * i + 2]), 0.f);
    return m;
}

struct AssemblyGeometry {
    const DPanel *panels;
    const Bounds *bounds;
    const uint8_t *pairCode;        // T(T-1)/2 unordered pair codes
    const TouchingJob *touching;
    const NearPairJob *nearPairs;
    const Patch *patches;
    const uint32_t *incOffsets;     // vertex -> (panel, local) incidence
    const uint32_t *incPanel;
    const uint8_t *incLocal;
    const double *rowScale;         // 1 / lumped mass
    uint32_t T, N;
    uint32_t touchingCount, nearPairCount;
    uint32_t projectedPairCount;    // the last near pairs, those with projected patches
    double nearTolerance;
    uint32_t minimumDegree, singularOrder;
    const float4 *singularTable;    // mixed-form touching tuples (buildSingularTable)
    const MixedPanel *mixedPanels;  // FP32 panel view of the mixed form
};


// Quadrature tables copied to __constant__ memory at first use.
void uploadRuleTables(cudaStream_t stream);

// Touching-pair tuples of the mixed form for one singular order: per
// (topology block vertex|edge|coincident, sector, u, v, w) twelve floats
// (canonical test and trial barycentrics at radius 1, displacement
// coefficients a1 a2 b1 b2, weight, pad), then per radial node (r, r^3 w, 1/r, 1 - r).
std::vector<float> buildSingularTable(unsigned order);

// Per-batch assembly of B frequencies. ks[B]; flux q[B][E][T] complex;
// outputs A[B][N*N] (column-major) and rhs[B][E][N] complex. Workspace:
// records [B][T*T][24], gathered columns C[B][N][3T] complex, per-panel rhs
// partials R[B][E][3T] complex, pair bins [B][4][pairs] and counters.
struct AssemblyWorkspace {
    void *records;                  // double (plain form) or float (mixed form) records
    void *columns;                  // trial-gathered columns, the record type
    double *panelRhs;
    uint2 *bins;
    uint32_t *binCounts;
    size_t binCapacity;
    // Set for meshes above kExactBinsT triangles: the bins of each frequency are packed
    // into `pairs` entries, bin b of frequency f starting at binOffsets[f * kBins + b]
    // (B * kBins entries, filled by the assembly: count pass, scan, fill pass). Null:
    // every bin has binCapacity entries.
    uint64_t *binOffsets = nullptr;
};
constexpr uint32_t kExactBinsT = 10000;
size_t assemblyWorkspaceBytes(uint32_t T, uint32_t N, uint32_t E, uint32_t B, bool mixed);
// Record bytes of one frequency; whether the gather needs the columns buffer
// (meshes whose 3T column entries exceed the fused gather's shared memory).
size_t recordBytes(uint32_t T, bool mixed);
bool gatherUsesColumns(uint32_t T);
// mixed: FP32 samples and records (phases kept exact: centre phase in FP64 for
// regular pairs, FP64 displacement and phase for near pairs), FP64 matrix.
void assembleBatch(const AssemblyGeometry &geo, const double *ks, const double *gaussSingular, const double *flux,
                   uint32_t E, uint32_t B, const AssemblyWorkspace &ws, double *A, double *rhs, int *error,
                   cudaStream_t stream, class KernelTimer *timer, bool mixed = false);

// Fast-multipole near field of one frequency (assembly.cu): the records of
// the near panel pairs (pairRow/pairCol: CSR over test panels, pairList: the
// unordered pairs i < j to classify), reduced into the near support-pair
// values (nearRow/nearCol, row-equilibrated) and the near right-hand side
// rhsNear[E][N] (row-equilibrated). The workspace holds
// nearFieldWorkspaceBytes(pairSlots, pairCount) bytes.
struct NearFieldLayout {
    const uint32_t *pairRow, *pairCol;
    size_t pairSlots;
    const uint2 *pairList;
    uint64_t pairCount;
    const uint32_t *nearRow, *nearCol;
};
size_t nearFieldWorkspaceBytes(size_t pairSlots, uint64_t pairCount);
void assembleNearField(const AssemblyGeometry &g, const double *k, const double *gaussSingular, const double *flux,
                       uint32_t E, const NearFieldLayout &nf, void *workspace, double *vals, double *rhsNear,
                       int *error, cudaStream_t stream, class KernelTimer *timer);

// Batched dense LU (partial pivoting) and solves, complex column-major. The
// pivot buffer holds luWorkspaceBytes(N, B): the LAPACK-style interchanges
// of each matrix, then their composition as a permutation. A solve needs
// B * E * N complex elements of scratch.
size_t luWorkspaceBytes(uint32_t N, uint32_t B);
void luFactorBatch(double *LU, uint32_t N, uint32_t B, int *pivots, int *info, cudaStream_t stream,
                   class KernelTimer *timer);
// FP32 factorisation: `pack` holds luPackBytes(N, B) of operand tiles for the
// tensor-core trailing updates.
size_t luPackBytes(uint32_t N, uint32_t B);
void luFactorBatch(float *LU, uint32_t N, uint32_t B, int *pivots, int *info, cudaStream_t stream,
                   class KernelTimer *timer, float *pack);
void luSolveBatch(const double *LU, const int *pivots, uint32_t N, uint32_t B, uint32_t E, double *x,
                  void *scratch, cudaStream_t stream, class KernelTimer *timer);
// Test hook: factors B host matrices (complex column-major, interleaved) with
// the batched kernels above, FP64 or FP32 (FP32 in, rounded from the FP64
// input), and returns the factors (as doubles), the 0-based interchange
// sequence and the breakdown word (first zero pivot + 1, -1 for a tensor-core
// timeout, 0 when every pivot is nonzero).
void debugLuFactor(bool fp32, uint32_t N, uint32_t B, const double *matrices, double *factors, int *pivots,
                   int *info);
void luSolveBatch(const float *LU, const int *pivots, uint32_t N, uint32_t B, uint32_t E, float *x,
                  void *scratch, cudaStream_t stream, class KernelTimer *timer);
// r = b - A x (FP64); writes the correction rhs into `correction` and the
// mass-scaled residual norm and rhs norm per (batch, excitation) into norms[2].
void residualBatch(const double *A, const double *b, const double *x, const double *mass, uint32_t N, uint32_t B,
                   uint32_t E, double *correction, double *norms, cudaStream_t stream, class KernelTimer *timer);
void addCorrectionBatch(double *x, const double *correction, size_t count, cudaStream_t stream);
void addCorrectionBatch(double *x, const float *correction, size_t count, cudaStream_t stream);
void roundToFloat(const double *in, float *out, size_t count, cudaStream_t stream);

// One left-preconditioned GMRES cycle (at most m Arnoldi steps) per system of
// a batch: solves A_f d = r_s with M = the FP32 LU of A_f and adds d to x_s
// (systems s = f * E + e; a zero r_s is left alone). Stops system s once its
// preconditioned residual estimate is at most tolerances[s] relative to its
// start, so each system's result does not depend on the others in the batch.
// Returns the Arnoldi steps taken by the batch; stepsOut[s] holds each
// system's. The workspace holds gmresWorkspaceBytes(N, B * E, m) bytes.
size_t gmresWorkspaceBytes(uint32_t N, uint32_t S, uint32_t m);
uint32_t gmresCycleBatch(const double *A, const float *LU32, const int *pivots, uint32_t N, uint32_t B, uint32_t E,
                         const double *r, double *x, uint32_t m, const std::vector<double> &tolerances,
                         void *workspace, cudaStream_t stream, KernelTimer *timer, std::vector<uint32_t> &stepsOut);
// The same cycle with a caller-supplied operator and preconditioner (gmres.cu).
uint32_t gmresCycleOperator(uint32_t N, uint32_t S, const double *r, double *x, uint32_t m,
                            const std::vector<double> &tolerances, void *workspace, cudaStream_t stream,
                            KernelTimer *timer, std::vector<uint32_t> &stepsOut,
                            const std::function<void(const double *, size_t, double *)> &apply,
                            const std::function<void(const double *, double *)> &precondition);

// Observer fields of one rule degree for every (batch, excitation, observer).
struct FieldRequest {
    const DPanel *panels;
    uint32_t T, N, E, O, B;
    const double *observers;     // O x 3 local points or unit directions
    int farField;
    double farOrigin[3];
    double farDistance;
    double tolerance;
    uint32_t maximumDepth;
};
// Post-solve pressure samples at points (local coordinates, count x 3): for
// each point a status (0 air, 1 boundary, 2 excluded, 3 quadrature not
// converged) and, for air, the pressure from the P1 trace and DP0 flux.
void samplePressureField(const DPanel *panels, uint32_t T, const double *trace, const double *flux,
                         const double *points, uint32_t count, double k, double minDistance, double tolerance,
                         uint32_t maxDepth, double *pressure, int32_t *status, cudaStream_t stream);
void evaluateFieldBatch(const FieldRequest &req, const double *ks, const double *pressure, const double *flux,
                        const uint32_t *batchDegree, double *partials, double *out, int *error,
                        cudaStream_t stream, class KernelTimer *timer);
size_t fieldPartialsBytes(uint32_t T, uint32_t E, uint32_t O, uint32_t B);

// Allocation-free observer field (field.cu): all inputs/outputs are caller
// device memory, scratch is a fixed static device array.
void observerFieldNoAlloc(const double *vertices, size_t vertexCount, const uint32_t *triangles, size_t triangleCount,
                          const double *pressure, const double *flux, const double *observers, size_t observerCount,
                          double k, uint32_t degree, int farField, const double *farOrigin, double farDistance,
                          double tolerance, uint32_t maximumDepth, cudaStream_t stream, double *out);
size_t noAllocScratchBytes();

}  // namespace hsb
