/*
 * hs_bem.h — C ABI of the B200-native exterior Burton-Miller solve.
 *
 * Drop-in boundary for HornSculpt's `hornsculpt::CudaBemSolver`
 * (modules/bem/include/hornsculpt/bem.hpp:367-388; implementation
 * modules/bem/cuda/cuda_solver.cu:1021-1853). Plain pointers and sizes only.
 * A session holds one closed surface mesh (its geometry, interaction plan and
 * device workspaces) across calls, like the reference solver object; a solve
 * call takes a request (medium, frequencies, excitations, observers,
 * numerics) and returns a host-owned result.
 *
 * Conventions follow the reference (bem.hpp:357-360): exp(+i omega t) RMS
 * phasors, outgoing exp(-ikr), flux q = dp/dn = -i rho omega v on Driven
 * faces, Burton-Miller coupling alpha = -i/k, P1 pressure per mesh vertex,
 * DP0 flux per triangle. Complex arrays are interleaved (re, im) doubles.
 *
 * Every function returns an hs_status; on failure hs_last_error() holds the
 * message of the calling thread's last failure. Invalid inputs that the
 * reference rejects with std::invalid_argument return HS_E_INVALID; device,
 * numerical and convergence failures that it reports with
 * std::runtime_error return HS_E_CUDA / HS_E_NUMERIC / HS_E_NOCONVERGE /
 * HS_E_NOMEM / HS_E_CANCELLED.
 */
#ifndef HS_BEM_H
#define HS_BEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hs_status {
    HS_OK = 0,
    HS_E_INVALID = 1,     /* std::invalid_argument in the reference */
    HS_E_CUDA = 2,        /* CUDA runtime failure (cuda_solver.cu:35-38) */
    HS_E_NUMERIC = 3,     /* quadrature / non-finite codes (cuda_solver.cu:705-715) */
    HS_E_NOCONVERGE = 4,  /* refinement or field-degree loop exhausted (cuda_solver.cu:1559-1565, 1792-1796) */
    HS_E_NOMEM = 5,       /* memory preflight (cuda_solver.cu:1161-1163, 1261-1264) */
    HS_E_CANCELLED = 6,   /* "BEM calculation cancelled." (cuda_solver.cu:49-52) */
    HS_E_UNSUPPORTED = 7  /* sub-domain, baffle, axisymmetric or mixed-precision fast-multipole requests */
} hs_status;

typedef enum hs_boundary { HS_WALL = 0, HS_DRIVEN = 1 } hs_boundary;   /* mesh.hpp:17 */
/* HS_FAST_MULTIPOLE: FP64 support-tree FMM + GMRES (precision must be HS_PRECISION_FP64). */
typedef enum hs_acceleration { HS_DENSE = 0, HS_FAST_MULTIPOLE = 1 } hs_acceleration; /* bem.hpp:38 */
typedef enum hs_precision {
    HS_PRECISION_FP64 = 0,  /* plain form: the reference method evaluated entirely in FP64 */
    HS_PRECISION_MIXED = 1  /* FP32 regular/near samples (FP64 displacement and phase), FP64 touching
                               pairs, FP32 LU, FP64 iterative refinement to min(tolerance, 1e-10) */
} hs_precision;
/* Interaction planner of a session (hs_bem_session_set_planner). */
typedef enum hs_planner { HS_PLANNER_DEVICE = 0, HS_PLANNER_HOST = 1 } hs_planner;
typedef enum hs_residency { HS_RESIDENCY_AUTOMATIC = 0, HS_RESIDENCY_DEVICE = 1, HS_RESIDENCY_MAPPED_HOST = 2 } hs_residency; /* bem.hpp:361-365 */

/* BemNumerics + FastMultipoleSettings (bem.hpp:61-72, 113-123). */
typedef struct hs_numerics {
    uint32_t quadrature_order;            /* 2 or 4 (default 4) */
    uint32_t singular_order;              /* 2..20 (default 4) */
    double near_distance_ratio;           /* [0, 10] (default 1) */
    double near_relative_tolerance;       /* [1e-10, 1e-2] (default 1e-4) */
    uint32_t near_maximum_depth;          /* <= 10 (default 6) */
    double relative_residual_tolerance;   /* [1e-7, 1e-2] (default 5e-5) */
    uint32_t maximum_refinement_steps;    /* <= 10 (default 3) */
    uint32_t acceleration;                /* hs_acceleration */
    uint32_t precision;                   /* hs_precision */
    uint32_t fmm_leaf_support_capacity;   /* 16; 0: chosen by the autotuner (below) */
    double fmm_separation_ratio;          /* 1.5 */
    uint32_t fmm_maximum_iterations;      /* 300 */
    uint32_t fmm_restart_length;          /* 40 */
    uint32_t fmm_preconditioner_block_width; /* 32 */
} hs_numerics;

/* BemRequest (bem.hpp:163-191), exterior single-domain subset. Excitation e
 * assigns velocities to Driven faces excitation_face_ids[o] for
 * o in [excitation_face_offsets[e], excitation_face_offsets[e+1]). */
typedef struct hs_request {
    double density;                       /* kg/m^3 (AcousticMedium, default 1.21) */
    double sound_speed;                   /* m/s (default 343) */
    const double *frequencies;            /* Hz, finite, > 0 */
    size_t frequency_count;
    const double *plan_frequencies;       /* interactionPlanFrequencies; may be NULL */
    size_t plan_frequency_count;
    size_t excitation_count;              /* 1..1024 */
    const size_t *excitation_face_offsets;/* excitation_count + 1 */
    const uint32_t *excitation_face_ids;
    const double *excitation_velocities;  /* complex RMS normal velocity per face entry */
    const double *observers;              /* xyz world points, or far-field directions */
    size_t observer_count;
    int32_t far_field;                    /* nonzero: FarFieldObservation */
    double far_origin[3];
    double far_reference_distance;        /* metres; result includes exp(-ik R)/R */
    hs_numerics numerics;
} hs_request;

/* BemProgress (bem.hpp:334-355). */
typedef enum hs_phase {
    HS_PHASE_PREPARING = 0,
    HS_PHASE_NEAR_CONSTRUCTION = 1,
    HS_PHASE_FAR_PREPARATION = 2,
    HS_PHASE_KRYLOV_SOLVE = 3,
    HS_PHASE_RESIDUAL_AUDIT = 4,
    HS_PHASE_FIELD_EVALUATION = 5,
    HS_PHASE_FREQUENCY_COMPLETE = 6
} hs_phase;
typedef struct hs_progress {
    size_t completed_frequencies, total_frequencies;
    double frequency;
    uint32_t phase;
} hs_progress;
typedef void (*hs_progress_fn)(const hs_progress *progress, void *user);

typedef struct hs_bem_session hs_bem_session;
typedef struct hs_result hs_result;

/* Per-excitation result scalars (BemExcitationResult, bem.hpp:231-301). */
typedef struct hs_excitation_info {
    double boundary_residual;             /* relative L2 residual of the unscaled equation */
    uint32_t refinement_steps;
    uint32_t iterations;                  /* 0 for dense LU */
    uint32_t field_comparison_degree, field_verification_degree;
    double field_discrepancy;
    size_t impedance_count;
} hs_excitation_info;

/* FaceImpedance (bem.hpp:193-199). */
typedef struct hs_face_impedance {
    uint32_t face_id;
    double area;
    double mean_pressure[2];
    double volume_velocity[2];
    double volume_impedance[2];
} hs_face_impedance;

/* BemFrequencyResult timings (bem.hpp:303-317), milliseconds. */
typedef struct hs_frequency_info {
    double frequency;
    double assembly_ms, factorization_ms, triangular_solve_ms, solve_ms, field_ms, residual_check_ms;
    double interaction_plan_ms;
    int32_t interaction_plan_reused;
} hs_frequency_info;

/* ---- numerics ---- */
void hs_numerics_default(hs_numerics *out);                 /* BemNumerics{} defaults */

/* ---- session (CudaBemSolver ctor / dtor, bem.hpp:369-378) ----
 * vertices: vertex_count x 3 doubles; triangles: triangle_count x 3 vertex
 * indices; face_ids, boundary (hs_boundary) one per triangle. The mesh is
 * copied and centred on vertex 0 (cuda_solver.cu:771-781) and validated as a
 * closed, outward-oriented exterior surface (cuda_solver.cu:782-789). */
hs_status hs_bem_session_create(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                                const uint32_t *face_ids, const uint8_t *boundary, size_t triangle_count,
                                uint32_t residency, hs_bem_session **out);
void hs_bem_session_destroy(hs_bem_session *session);

/* Optional: run the session's device work on a caller-owned cudaStream_t
 * (passed as void*). NULL restores the session's own non-blocking stream. */
hs_status hs_bem_session_set_stream(hs_bem_session *session, void *cuda_stream);

/* ---- solve (CudaBemSolver::solve, bem.hpp:381-382) ----
 * cancel: optional flag polled between device batches (std::stop_token);
 * progress: optional callback. Calls on one session are serialised. */
hs_status hs_bem_solve(hs_bem_session *session, const hs_request *request, const volatile int32_t *cancel,
                       hs_progress_fn progress, void *user, hs_result **out);

/* ---- LEM-coupled solve (CudaBemSolver::solve with request.coupling,
 * cuda_solver.cu:1584-1667; lem_coupling.cpp:9-120) ----
 * The request's excitations are the unit-flow basis, one per port: each port's
 * faces (disjoint between ports) with positive real velocities w_f / S_w whose
 * flux integrates to one unit of volume velocity (makeCouplingBasis). Per
 * frequency the library solves the basis, forms the port impedance matrix Z
 * (ports x ports complex, row-major: the power-dual mean pressure at port i per
 * unit flow at port j), calls `network` for the port flows and pressures (the
 * caller's lumped network: lem::solve), superposes the coupled pressure,
 * right-hand side and flux, refines that combined equation with the retained
 * factors, checks the port-pressure closure to 1e-3 (validateCouplingClosure)
 * and evaluates the observers for it. The result has one excitation per
 * frequency, the coupled field; hs_result_coupling returns Z, the flows and the
 * pressures. Dense forms only (fast multipole: HS_E_UNSUPPORTED). `network`
 * returns HS_OK or fails the solve with HS_E_INVALID. */
typedef hs_status (*hs_network_fn)(double frequency, size_t port_count, const double *impedance,
                                   double *volume_velocity, double *pressure, void *user);
hs_status hs_bem_solve_coupled(hs_bem_session *session, const hs_request *request, hs_network_fn network,
                               void *user, const volatile int32_t *cancel, hs_result **out);

/* ---- results (BemResult, bem.hpp:319-332) ---- */
size_t hs_result_frequency_count(const hs_result *r);
size_t hs_result_excitation_count(const hs_result *r);
size_t hs_result_triangle_count(const hs_result *r);
size_t hs_result_pressure_dof_count(const hs_result *r);
size_t hs_result_observer_count(const hs_result *r);
size_t hs_result_peak_device_bytes(const hs_result *r);
hs_status hs_result_frequency_info(const hs_result *r, size_t f, hs_frequency_info *out);
hs_status hs_result_excitation_info(const hs_result *r, size_t f, size_t e, hs_excitation_info *out);
/* BemBoundaryData (bem.hpp:203-214): P1 trace [N], DP0 mean surface pressure
 * [T], DP0 normal derivative [T]; observer pressure [O]. */
hs_status hs_result_pressure_trace(const hs_result *r, size_t f, size_t e, double *out);
hs_status hs_result_surface_pressure(const hs_result *r, size_t f, size_t e, double *out);
hs_status hs_result_normal_derivative(const hs_result *r, size_t f, size_t e, double *out);
hs_status hs_result_observer_pressure(const hs_result *r, size_t f, size_t e, double *out);
hs_status hs_result_impedances(const hs_result *r, size_t f, size_t e, hs_face_impedance *out);
/* The whole result in one call, [frequency][excitation] order with interleaved
 * complex values: traces F*E*N, surface and normal F*E*T, observers F*E*O
 * complex values, excitation infos F*E, frequency infos F. A null pointer
 * skips that part. The per-item getters above return the same values. */
hs_status hs_result_copy_all(const hs_result *r, double *traces, double *surface, double *normal, double *observers,
                             hs_excitation_info *excitation_infos, hs_frequency_info *frequency_infos);
/* Coupled solves: Z (ports x ports complex), port flows and pressures (ports
 * complex each) of frequency f; ports receives the count (0 for uncoupled
 * results). Any output pointer may be NULL. */
hs_status hs_result_coupling(const hs_result *r, size_t f, double *impedance, double *volume_velocity,
                             double *pressure, size_t *ports);
void hs_result_free(hs_result *r);

/* ---- diagnostics ---- */
const char *hs_last_error(void);
/* CudaBemSolver::deviceDescription (bem.hpp:383, cuda_solver.cu:1010-1020). */
hs_status hs_device_description(char *buffer, size_t size);

/* Device work of the last solve on this session, summed per kernel family
 * from CUDA events recorded on the session stream when profiling is on.
 * names: comma-separated family names written to names_buffer; ms/launches:
 * one entry per family (capacity entries at most). */
hs_status hs_bem_session_set_profiling(hs_bem_session *session, int32_t enabled);
hs_status hs_bem_session_profile(const hs_bem_session *session, char *names_buffer, size_t names_size,
                                 double *ms, uint64_t *launches, size_t capacity, size_t *count);

/* CUDA graphs (no reference counterpart beyond its captured M2L chunks,
 * support_m2l_graph.hpp:52-78): a session replays the launch chain of a dense
 * frequency batch (assembly, LU, initial solves) and the fast-multipole
 * far-field apply as captured graphs. A chain is captured on its second use
 * with the same batch shape and buffers (the first use runs its launches
 * directly) and replayed after that; re-planning or regrown buffers retire
 * it. With kernel profiling on, the dense chain runs as plain launches so
 * each kernel family keeps its own time. Results are the same either way (the
 * graph holds the same launches). On by default; graph_launches counts dense
 * chain replays of the session. */
hs_status hs_bem_session_set_graphs(hs_bem_session *session, int32_t enabled);
hs_status hs_bem_session_graph_launches(const hs_bem_session *session, uint64_t *launches);

/* Launch-shape autotuner (process-wide; the reference has no counterpart).
 * For each kernel family and size class (form, rule, batch, mesh size to a
 * power of two) the first solve outside a graph capture and outside a
 * profiled solve times the candidate launch shapes once with CUDA events and
 * keeps the fastest. Candidates spread the same independent work items
 * differently over the grid, so a choice changes speed, never results. A
 * fast-multipole request with fmm_leaf_support_capacity = 0 has its leaf size
 * chosen the same way (per mesh size and electrical size class, by timing one
 * operator apply per candidate tree of 8, 16, 32 supports). The report lists
 * "class=choice:ms/ms/...;" per tuned class (needed: its size with the NUL). */
hs_status hs_autotune_set_enabled(int32_t enabled);
hs_status hs_autotune_clear(void);
hs_status hs_autotune_report(char *buffer, size_t size, size_t *needed);

/* Work counters of the solves since profiling was last enabled, in this
 * order: regular unordered pairs with the 6/12/16/64-point rules (4 values),
 * regular pair samples, touching-pair samples, near-pair samples (each
 * sample evaluates the Green kernel once for both orientations of an
 * unordered pair where applicable), solved frequency points. */
hs_status hs_bem_session_work(const hs_bem_session *session, uint64_t *counters, size_t capacity, size_t *count);

/* Test hooks: the host interaction plan of a mesh (no device needed) and a
 * session's assembled system. hs_bem_debug_plan centres the mesh on vertex 0
 * like a session, plans at wavenumber max_k and writes sizes = {touching,
 * near, patches, whole-panel bytes, near-trial entries, maximum depth}; any
 * array pointer may be NULL to query sizes first. Layouts match the
 * reference's InteractionPlan (interaction_plan.hpp:25-53): touching 9 u32
 * per job (test, trial, topology, test perm[3], trial perm[3]), near 5 u32
 * (test, trial, first patch, count, swap), patches 22 doubles (test[9],
 * trial[9], area fraction, degree, projection, intervals), near offsets
 * triangle_count + 1 u32. hs_bem_debug_assemble writes the row-equilibrated
 * matrix (column-major N x N complex) and right-hand side (N complex) of one
 * excitation with per-triangle flux q (T complex) at wavenumber k, planned
 * at plan_k >= k. */
hs_status hs_bem_debug_plan(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                            size_t triangle_count, const hs_numerics *numerics, double max_k, size_t *sizes,
                            uint32_t *touching, uint32_t *near, double *patches, uint8_t *whole,
                            uint32_t *near_offsets, uint32_t *near_trials);
/* The same plan from the device planner (mode 0: on the current CUDA device;
 * mode 1: its algorithm emulated on the host, one lane per warp, no GPU
 * needed). No reference counterpart beyond makeInteractionPlan itself
 * (interaction_plan.cpp:156): the result equals hs_bem_debug_plan's bit for
 * bit. stats (20 doubles, may be NULL): pairs refined on the device, pairs on
 * projected patches (refined by the host), device pairs handed to the host
 * because a decision fell within its rounding bound, whole-panel pairs
 * decided on the device (all-pairs mode), device milliseconds, host
 * milliseconds, device pairs whose order of nearly equal patches the host
 * settled with its own error estimates, then the milliseconds of the phases:
 * frame (validation, bounds, touching jobs, grid candidates), classification,
 * refinement, readback, host part; then the host part's own phases: ordering
 * runs, host pairs, flattening, patch fill, near CSR; then the kernel samples
 * the refinement evaluated, the CUDA-event time of its launches and, in the
 * all-pairs mode, the pairs settled by their root estimate alone. */
hs_status hs_bem_debug_plan_device(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                                   size_t triangle_count, const hs_numerics *numerics, double max_k, uint32_t mode,
                                   double *stats, size_t *sizes, uint32_t *touching, uint32_t *near,
                                   double *patches, uint8_t *whole, uint32_t *near_offsets, uint32_t *near_trials);
hs_status hs_bem_debug_assemble(hs_bem_session *session, const hs_numerics *numerics, double plan_k, double k,
                                const double *flux, double *matrix, double *rhs);
/* LU test hook: factors `batch` complex n x n matrices (host, column-major,
 * interleaved re/im) with the solver's batched LU kernels — FP64
 * (HS_PRECISION_FP64: the plain form's factorisation) or FP32
 * (HS_PRECISION_MIXED: the input rounded to FP32, the two-level factorisation
 * with tensor-core trailing updates). `factors` (same layout, doubles)
 * receives L (unit diagonal, strictly below it) and U in place, like LAPACK
 * zgetrf / the reference's cusolverDnCgetrf (cuda_solver.cu:1485-1513);
 * `pivots` (batch x n) the row interchange sequence, 0-based (ipiv - 1 in
 * LAPACK terms); `info` one status word for the batch: 0, or the first zero
 * pivot's column + 1 (-1: a tensor-core update did not complete). */
hs_status hs_bem_debug_lu(uint32_t precision, size_t n, size_t batch, const double *matrices, double *factors,
                          int32_t *pivots, int32_t *info);
/* Fast-multipole test hooks. hs_bem_debug_fmm_far applies the far part of the
 * fast-multipole operator (support pairs outside the near leaf pairs of the
 * support tree, row-equilibrated like hs_bem_debug_assemble's matrix) to a P1
 * vector `pressure` (vertex_count complex) at wavenumber k with expansion
 * tolerance `tolerance`, writing `far` (vertex_count complex); near_row_start
 * (vertex_count + 1) and near_cols (capacity near_capacity, sorted per row)
 * receive the near pattern, near_count its size; level_info receives per
 * far-field level {level, order, nodes, M2L links, plane wave} (capacity
 * level_capacity rows of 5 u32; plane wave 1 when the level's M2L runs in the
 * diagonal plane-wave form), level_count their number. Pointers after `far`
 * may be NULL. With numerics.precision = HS_PRECISION_MIXED the hook applies
 * the mixed form's operator (scaled expansions, FP32 translations).
 * hs_bem_debug_fmm_selftest checks the expansion primitives (Bessel and
 * Legendre recurrences, Wigner rotations, Gaunt-built coaxial translations)
 * against a direct kernel sum on the host and writes the relative error. */
hs_status hs_bem_debug_fmm_far(hs_bem_session *session, const hs_numerics *numerics, double k, double tolerance,
                               const double *pressure, double *far, uint32_t *near_row_start, uint32_t *near_cols,
                               size_t near_capacity, size_t *near_count, uint32_t *level_info, size_t level_capacity,
                               size_t *level_count);
hs_status hs_bem_debug_fmm_selftest(double *error);
/* Interaction planner of a session (makeInteractionPlan,
 * interaction_plan.cpp:156): HS_PLANNER_DEVICE (default) classifies the
 * panel pairs and runs the adaptive near-pair refinement on the session's
 * device, handing the pairs on projected patches and any pair whose decisions
 * fall within the device's rounding bounds to the host planner's code;
 * HS_PLANNER_HOST plans on host threads like the reference. Both give the
 * same plan bit for bit. hs_bem_session_plan_stats writes the last device
 * plan's statistics (20 doubles, the layout of hs_bem_debug_plan_device). */
hs_status hs_bem_session_set_planner(hs_bem_session *session, uint32_t planner);
hs_status hs_bem_session_plan_stats(hs_bem_session *session, double *stats);
/* Fast-multipole LF/HF switch (wideband_transfer.cpp:266-310): a level's M2L
 * runs in the diagonal plane-wave form when k times its shortest M2L distance
 * is at least `threshold` (default 8) and its order is at least 8; below, the
 * rotate-coaxial-rotate form. A very large threshold keeps every level
 * rotational. Applies to the FP64 operator; the mixed form's FP32 inner
 * operator stays rotational. */
hs_status hs_bem_session_set_plane_wave_threshold(hs_bem_session *session, double threshold);
/* Rotational M2L schedule of the fast-multipole operators: grouped by
 * translation class (enabled != 0, the default: the links sharing a rotation
 * and a coaxial table are translated together, each into its own slot, and the
 * slots summed per target in link order) or one CTA per target node walking
 * its links (enabled == 0). Both give the same operator to rounding; the
 * switch exists for tests and measurements. The reference's M2L batches its
 * chunks under graphs (support_m2l_graph.hpp:52-78). */
hs_status hs_bem_session_set_fmm_grouped_m2l(hs_bem_session *session, int enabled);
/* Acceptance audit of fast-multipole solves (SupportFmmLinearSolver::solve,
 * support_fmm_solve.cu:324-634). mode 0 (default), the reference's policy:
 * where assembling the dense system costs less than two expansion operators
 * (preferSupportDirectAudit, :79-114; at most 20 000 panels and within half the
 * free memory) the residual is that of the exact FP64 dense system, with
 * fast-multipole defect corrections (directFar, support_direct_audit.cu:26);
 * otherwise a ten times finer expansion operator audits the working one and
 * the far-field panel rule is compared with the next one and promoted
 * 4 -> 6 -> 8 -> 12 until they agree to 0.025 of the residual target
 * (compareQuadrature). mode 1: always the expansion and panel-rule audits;
 * mode 2: always the direct audit. The counts report the session's direct
 * audits and panel-rule promotions so far. */
hs_status hs_bem_session_set_fmm_audit(hs_bem_session *session, uint32_t mode);
hs_status hs_bem_session_fmm_audit_counts(const hs_bem_session *session, uint64_t *direct_audits,
                                          uint64_t *quadrature_promotions);
/* The support tree of the fast-multipole form (host only): the mesh centred on
 * vertex 0 like a session; sizes = {nodes, levels, pressure-pressure near,
 * pressure-pressure far, pressure-flux near, pressure-flux far} and links the
 * (target, source) node pairs of the four lists in that order (capacity pairs
 * at most; NULL to query sizes). */
hs_status hs_bem_debug_fmm_tree(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                                size_t triangle_count, uint32_t leaf_capacity, double separation_ratio,
                                double near_distance_ratio, size_t *sizes, uint32_t *links, size_t capacity);

/* Allocation-free observer field. No counterpart in the reference: it is an
 * addition for callers that cannot allocate device memory when they need a
 * field — an interactive sweep that must not stall on the device-wide
 * synchronisation of cudaMalloc/cudaFree, or a host that gives the solver only
 * memory from its own pre-sized arena. All pointers except far_origin are
 * DEVICE memory the caller owns: vertices (vertex_count x 3), triangles
 * (triangle_count x 3), the solved P1 trace (vertex_count complex), the DP0
 * flux q = -i rho omega v (triangle_count complex), observers
 * (observer_count x 3 world points, or far-field points when far_field is
 * nonzero), and the output (observer_count complex). The same quantity as a
 * solve's observer pressure at rule degree `degree` (4, 6, 8, 12 or 14) with
 * near-field tolerance `tolerance` and depth `maximum_depth`. The function
 * calls no cudaMalloc, cudaFree or allocating library routine; its scratch is
 * a fixed 4 MiB static device array of the library, which limits
 * triangle_count * 200 + observer_count * 24 +
 * observer_count * ceil(triangle_count / 256) * 16 + 256 bytes to 4 MiB (larger
 * requests return HS_E_INVALID). The first call on a device looks up that
 * array's device address and keeps it until the process exits, so do not
 * reset the device between calls. All calls share the array: calls that
 * overlap on the GPU race and must be serialised. The call reads status words
 * back and waits for `cuda_stream`, so it returns after the work on that
 * stream has finished and cannot be captured in a CUDA graph. A
 * degenerate triangle returns HS_E_INVALID, as at session creation. */
hs_status hs_bem_observer_field_noalloc(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                                        size_t triangle_count, const double *pressure_trace, const double *flux,
                                        const double *observers, size_t observer_count, double wavenumber,
                                        uint32_t degree, int32_t far_field, const double *far_origin,
                                        double far_reference_distance, double tolerance, uint32_t maximum_depth,
                                        void *cuda_stream, double *observer_pressure);

/* Post-solve pressure samples at arbitrary points. Replaces
 * hornsculpt::evaluatePressureField (field_evaluation.hpp:29-33,
 * field_evaluation.cpp:330-463) for the exterior closed-surface form (no
 * baffle, sub-domains, symmetry or axisymmetric contract): from a solution's
 * P1 pressure trace (vertex_count complex, interleaved re/im) and DP0 outward
 * normal derivative (triangle_count complex), at `point_count` world points
 * (x, y, z), with the session's mesh. Per point a status (enum below) and, for
 * air points, the pressure D p - S q with the reference's adaptive quadrature
 * (degree 4 against degree 8 per patch, quartering to maximum_quadrature_depth).
 * Host buffers; runs on the session's stream and returns when done. Invalid
 * settings (minimum_boundary_distance <= 0, tolerance outside (0, 0.01],
 * depth > 12, frequency or sound speed not positive), non-finite traces or
 * points return HS_E_INVALID with the reference's messages. */
enum { HS_FIELD_AIR = 0, HS_FIELD_BOUNDARY = 1, HS_FIELD_EXCLUDED = 2, HS_FIELD_NOT_CONVERGED = 3 };
typedef struct hs_field_settings {
    double minimum_boundary_distance;     /* m; default 1e-4 */
    double relative_quadrature_tolerance; /* default 1e-4 */
    uint32_t maximum_quadrature_depth;    /* default 8 */
} hs_field_settings;
hs_status hs_field_settings_default(hs_field_settings *out);
hs_status hs_bem_pressure_field(hs_bem_session *session, double frequency, double sound_speed,
                                const double *pressure_trace, const double *normal_derivative, const double *points,
                                size_t point_count, const hs_field_settings *settings, double *pressure,
                                int32_t *status);

/* ---------------------------------------------------------------------------
 * Serving form (no reference counterpart; the reference solves one request per
 * CudaBemSolver::solve call): a persistent request loop on the current device.
 * Requests (mesh + request) are submitted at any time and admitted in arrival
 * order as device memory allows (by the estimated footprint of the solve);
 * `workers` requests run at once, each on its own CUDA stream, so requests on
 * different meshes overlap on the GPU. Sessions stay resident per mesh
 * (geometry, plan, workspaces; least recently used evicted), and queued
 * requests on the same mesh with the same settings are solved in one call with
 * their frequencies batched. With planning_frequency > 0 every request plans
 * its interactions at that frequency, so a result is the same whatever it was
 * batched with (frequencies above it are rejected).
 * ------------------------------------------------------------------------- */
typedef struct hs_server hs_server;

typedef struct hs_serve_options {
    uint32_t workers;                     /* requests on the device at once (default 4) */
    double memory_fraction;               /* share of the device memory free at creation that
                                             admitted requests may hold (default 0.6) */
    uint32_t resident_meshes;             /* sessions kept for reuse (default 8) */
    double planning_frequency;            /* Hz; 0 plans per request (default 0) */
    uint32_t max_batch_frequencies;       /* frequencies factored together (1..32, default 32) */
} hs_serve_options;

typedef struct hs_serve_timing {
    double queue_ms;                      /* arrival to start on a worker */
    double run_ms;                        /* start to finish */
    double latency_ms;                    /* arrival to finish */
    size_t footprint_bytes;               /* device bytes reserved at admission */
    uint32_t batched_requests;            /* requests solved in the same session call */
} hs_serve_timing;

void hs_serve_options_default(hs_serve_options *options);
hs_status hs_serve_create(const hs_serve_options *options, hs_server **out);
/* Copies the mesh and request; validates the mesh and frequencies at once. */
hs_status hs_serve_submit(hs_server *server, const double *vertices, size_t vertex_count, const uint32_t *triangles,
                          const uint32_t *face_ids, const uint8_t *boundary, size_t triangle_count,
                          const hs_request *request, uint64_t *ticket);
/* Blocks until the request is done; returns its result (free with
 * hs_result_free) or its error status. Each ticket is collected once. */
hs_status hs_serve_wait(hs_server *server, uint64_t ticket, hs_result **out, hs_serve_timing *timing);
/* Cancels queued requests, finishes running ones, releases the device state. */
void hs_serve_destroy(hs_server *server);

#ifdef __cplusplus
}
#endif
#endif /* HS_BEM_H */
