// Far-field operator of the fast-multipole form (fmm.cu) on the support tree
// of fmm_tree.cpp.
//
// The operator splits the Burton-Miller matrix by support pairs: entries of
// near support pairs (leaf pairs of the partition) are exact Galerkin entries,
// the rest are applied through spherical-wave expansions of the fields
//   V(x) = sum_j p_j int G(x, y) n(y) phi_j(y) dy,   W(x) = sum_j p_j int G(x, y) curl phi_j(y) dy,
// tested as  y_i = int phi_i (div V + i k n.V) - (i / k) int curl phi_i . W,
// the far part of the record formula of the dense form (double layer
// d/dn_y G = -n.grad_x G, so its field is -div V; Maue curl term with
// alpha = -i / k). Panel integrals use the degree-4 Dunavant rule.
#pragma once

#include "fmm_tree.hpp"
#include "host_mesh.hpp"

#include <cuda_runtime.h>
#include <memory>
#include <utility>
#include <vector>

namespace hsb {

class KernelTimer;

struct FmmLevelInfo {
    uint32_t level, order, nodes, m2lLinks;
    double radius;
    uint32_t planeWave;  // 1: M2L in the plane-wave (diagonal) form at this level
};

class FmmOperator {
  public:
    FmmOperator(const Space &space, const FmmTreeSettings &settings);
    ~FmmOperator();
    FmmOperator(const FmmOperator &) = delete;
    FmmOperator &operator=(const FmmOperator &) = delete;

    // Expansion orders and translation tables for one wavenumber; the orders
    // follow the wideband excess-bandwidth rule p = kD + 1.8 d^(2/3) (kD)^(1/3)
    // (wideband_transfer.cpp:285-303) with d = -log10(tolerance), floored by a
    // low-frequency order.
    void prepare(double k, double tolerance, cudaStream_t stream);
    // y[s] = far part of the raw (not row-equilibrated) operator applied to
    // p[s] for S systems (complex, interleaved; system stride `stride` reals).
    void applyFar(const double *p, size_t stride, uint32_t S, double *y, cudaStream_t stream, KernelTimer *timer);
    // y[s] = far part of the raw right-hand side -S q - alpha K' q for per-panel
    // flux q[s] (T complex each): each panel's flux is emitted through its three
    // vertex supports (1/3 each), so the near part pairs with it exactly.
    void applyFarRhs(const double *q, uint32_t S, double *y, cudaStream_t stream, KernelTimer *timer);
    // Near panel pairs: CSR over test panels (sorted trials) of every (a, s) with a
    // vertex pair in a near support pair, and its unordered pairs a < s.
    const std::vector<uint32_t> &nearPanelRow() const { return panelRow_; }
    const std::vector<uint32_t> &nearPanelCol() const { return panelCol_; }
    const std::vector<std::pair<uint32_t, uint32_t>> &nearPanelPairs() const { return panelPairs_; }

    const FmmTree &tree() const { return tree_; }
    const std::vector<FmmLevelInfo> &levels() const { return levelInfo_; }
    // Near support pairs (pressure x pressure) as CSR over rows i, columns sorted.
    const std::vector<uint32_t> &nearRowStart() const { return nearRow_; }
    const std::vector<uint32_t> &nearCols() const { return nearCol_; }
    double wavenumber() const { return k_; }
    // Replay of the far-field apply as a captured CUDA graph (on by default).
    void setGraphs(bool enabled);
    // Mixed form: translations in FP32 on scaled expansions (P2M and L2P stay
    // FP64); takes effect at the next prepare().
    void setFp32(bool enabled);
    // k times the shortest M2L distance from which a level translates in the
    // plane-wave form (default 12; a large value keeps every level rotational).
    void setHfThreshold(double threshold);
    // Rotational M2L grouped by translation class (default) or per target node;
    // takes effect at the next prepare().
    void setGroupedM2l(bool enabled);
    // Far-field panel rule (Dunavant degree 4 by default; the audit promotes it
    // 4 -> 6 -> 8 -> 12 like the reference's compareQuadrature).
    void setPanelDegree(unsigned degree, cudaStream_t stream);
    unsigned panelDegree() const;

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
    FmmTree tree_;
    std::vector<FmmLevelInfo> levelInfo_;
    std::vector<uint32_t> nearRow_, nearCol_;
    std::vector<uint32_t> panelRow_, panelCol_;
    std::vector<std::pair<uint32_t, uint32_t>> panelPairs_;
    double k_ = 0;
    void run(const double *src, bool rhs, double *y, cudaStream_t stream, KernelTimer *timer);
    void launchApply(const double *src, bool rhs, double *y, cudaStream_t stream, KernelTimer *timer);
    void prepareHf(cudaStream_t stream);
    void planeWaveM2L(int level, int nch, cudaStream_t stream);
};

// The fast-multipole linear system of one frequency: A = N + R F, with N the
// exact near support-pair entries (CSR of the operator's pattern), F the far
// expansion operator and R = 1 / lumped mass the row equilibration. Solved by
// restarted GMRES (CGS2, Givens) left-preconditioned by block Jacobi on
// spatially ordered diagonal blocks of N (SupportBlockJacobi,
// cuda/support_preconditioner.cu:33-191: spatially ordered diagonal blocks of
// the near matrix, inverted once per frequency).
class FmmSystem {
  public:
    // blockWidth: supports per preconditioner block (at most 64); consecutive
    // leaves in tree order are merged up to it.
    FmmSystem(FmmOperator &op, const double *rowScale, const double *mass, uint32_t blockWidth);
    ~FmmSystem();
    // Device storage of the near values (CSR order of the operator's pattern),
    // filled directly by the near-field assembly; device near CSR arrays.
    double *nearValues();
    const uint32_t *nearRowDevice() const;
    const uint32_t *nearColDevice() const;
    // b_s += rowScale * far_s for S systems (N complex each).
    void addScaled(double *b, const double *far, uint32_t S, cudaStream_t stream);
    // r_s = b_s - A x_s with the operator as currently prepared; relative[s] its
    // mass-weighted norm over that of b_s.
    void residual(const double *b, const double *x, uint32_t S, double *r, std::vector<double> &relative,
                  cudaStream_t stream, KernelTimer *timer);
    // x += d (reals values).
    void add(double *x, const double *d, size_t reals, cudaStream_t stream);
    void factorBlocks(cudaStream_t stream, KernelTimer *timer);
    void apply(const double *x, size_t stride, uint32_t S, double *y, cudaStream_t stream, KernelTimer *timer);
    void precondition(const double *in, double *out, uint32_t S, cudaStream_t stream);
    // x_s = A^{-1} b_s to mass-weighted relative residual `target` (x starts at 0).
    // relative[s]: final relative residual of the operator; iterations[s]: Arnoldi steps.
    // With `inner` (an operator on the same tree in FP32 mode, prepared for the
    // same wavenumber) the solve is GMRES-IR: Krylov cycles on the FP32 operator
    // and FP32 near values (roundNearValues first), residuals of the FP64 one.
    void solve(const double *b, double *x, uint32_t S, double target, uint32_t restart, uint32_t maxIterations,
               cudaStream_t stream, KernelTimer *timer, std::vector<double> &relative,
               std::vector<uint32_t> &iterations, FmmOperator *inner = nullptr);
    // FP32 copy of the near values for the inner operator of the mixed form.
    void roundNearValues(cudaStream_t stream);
    void applyInner(FmmOperator &inner, const double *x, size_t stride, uint32_t S, double *y, cudaStream_t stream,
                    KernelTimer *timer);

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
    FmmOperator &op_;
};

// Host self-test of the expansion primitives (special functions, Wigner
// rotations, Gaunt-built coaxial translations, coefficient derivatives)
// against direct kernel sums. Returns the largest relative error.
double fmmSelfTest();

}  // namespace hsb
