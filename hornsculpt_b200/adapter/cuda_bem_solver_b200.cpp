// Reference-side adapter: HornSculpt's `hornsculpt::CudaBemSolver`
// (modules/bem/include/hornsculpt/bem.hpp:367-388) implemented over this
// library's C ABI (include/hs_bem.h), for the single exterior domain. It
// replaces modules/bem/cuda/cuda_solver.cu in a HornSculpt build: compile it
// with the reference's include directories and link libhs_bem.so. It uses the
// reference's types as they are declared there and needs nothing else of the
// reference at link time.
#include <hornsculpt/bem.hpp>
#include "hs_bem.h"
#include <stdexcept>

namespace hornsculpt {
namespace {
void check(hs_status s) {
    if (s == HS_OK) return;
    if (s == HS_E_INVALID) throw std::invalid_argument(hs_last_error());
    throw std::runtime_error(hs_last_error());
}
}  // namespace

class CudaBemSolver::Implementation {
  public:
    Implementation(const SurfaceMesh &mesh, CudaStorageOptions storage) : faces(mesh.triangles.size()) {
        std::vector<double> v; std::vector<uint32_t> t, f; std::vector<uint8_t> b;
        for (auto p : mesh.vertices) v.insert(v.end(), {p.x, p.y, p.z});
        for (auto &tri : mesh.triangles) {
            t.insert(t.end(), tri.vertices.begin(), tri.vertices.end());
            f.push_back(tri.faceId);
            b.push_back(tri.boundary == BoundaryCondition::driven ? HS_DRIVEN : HS_WALL);
        }
        check(hs_bem_session_create(v.data(), mesh.vertices.size(), t.data(), f.data(), b.data(),
                                    mesh.triangles.size(), static_cast<uint32_t>(storage.quadraturePatches),
                                    &session));
    }
    ~Implementation() { hs_bem_session_destroy(session); }
    hs_bem_session *session{};
    size_t faces;
};

CudaBemSolver::CudaBemSolver(SurfaceMesh mesh) : CudaBemSolver(std::move(mesh), CudaStorageOptions{}) {}
CudaBemSolver::CudaBemSolver(SurfaceMesh mesh, CudaStorageOptions storage)
    : implementation_(std::make_unique<Implementation>(mesh, storage)) {}
CudaBemSolver::~CudaBemSolver() = default;

BemResult CudaBemSolver::solve(const BemRequest &request, std::stop_token stop,
                               std::function<void(const BemProgress &)> progress) {
    if (request.subdomains || request.infiniteBaffle || request.axisymmetric || request.coupling)
        throw std::invalid_argument("This build implements the single exterior domain.");
    hs_request r{};
    r.density = request.medium.density;
    r.sound_speed = request.medium.soundSpeed;
    r.frequencies = request.frequencies.data();
    r.frequency_count = request.frequencies.size();
    r.plan_frequencies = request.interactionPlanFrequencies.data();
    r.plan_frequency_count = request.interactionPlanFrequencies.size();
    std::vector<size_t> offsets{0}; std::vector<uint32_t> ids; std::vector<double> vel;
    for (auto &e : request.excitations) {
        for (auto &fv : e.faces) {
            ids.push_back(fv.faceId);
            vel.insert(vel.end(), {fv.normalVelocity.real(), fv.normalVelocity.imag()});
        }
        offsets.push_back(ids.size());
    }
    r.excitation_count = request.excitations.size();
    r.excitation_face_offsets = offsets.data();
    r.excitation_face_ids = ids.data();
    r.excitation_velocities = vel.data();
    std::vector<double> obs;
    for (auto p : request.observers) obs.insert(obs.end(), {p.x, p.y, p.z});
    r.observers = obs.data();
    r.observer_count = request.observers.size();
    if (request.farField) {
        r.far_field = 1;
        r.far_origin[0] = request.farField->origin.x;
        r.far_origin[1] = request.farField->origin.y;
        r.far_origin[2] = request.farField->origin.z;
        r.far_reference_distance = request.farField->referenceDistance;
    }
    hs_numerics_default(&r.numerics);
    const auto &n = request.numerics;
    r.numerics.quadrature_order = n.quadratureOrder;
    r.numerics.singular_order = n.singularOrder;
    r.numerics.near_distance_ratio = n.nearDistanceRatio;
    r.numerics.near_relative_tolerance = n.nearRelativeTolerance;
    r.numerics.near_maximum_depth = n.nearMaximumDepth;
    r.numerics.relative_residual_tolerance = n.relativeResidualTolerance;
    r.numerics.maximum_refinement_steps = n.maximumRefinementSteps;
    r.numerics.acceleration = n.acceleration == BemAcceleration::dense ? HS_DENSE : HS_FAST_MULTIPOLE;
    // FastMultipoleSettings (bem.hpp:61-72), field by field
    r.numerics.fmm_leaf_support_capacity = n.fastMultipole.leafSupportCapacity;
    r.numerics.fmm_separation_ratio = n.fastMultipole.separationRatio;
    r.numerics.fmm_maximum_iterations = n.fastMultipole.maximumIterations;
    r.numerics.fmm_restart_length = n.fastMultipole.restartLength;
    r.numerics.fmm_preconditioner_block_width = n.fastMultipole.preconditionerBlockWidth;
    volatile int32_t cancel = 0;
    std::stop_callback onStop(stop, [&] { cancel = 1; });
    struct Ctx { std::function<void(const BemProgress &)> *fn; } ctx{&progress};
    auto bridge = [](const hs_progress *p, void *u) {
        auto *c = static_cast<Ctx *>(u);
        if (*c->fn) (*c->fn)(BemProgress{p->completed_frequencies, p->total_frequencies, p->frequency,
                                         static_cast<BemSolvePhase>(p->phase)});
    };
    hs_result *out = nullptr;
    check(hs_bem_solve(implementation_->session, &r, &cancel, bridge, &ctx, &out));
    BemResult result;
    char name[256];
    hs_device_description(name, sizeof name);
    result.device = name;
    result.triangleCount = hs_result_triangle_count(out);
    result.pressureDofCount = hs_result_pressure_dof_count(out);
    result.peakDeviceBytes = hs_result_peak_device_bytes(out);
    const size_t N = result.pressureDofCount, T = result.triangleCount, O = hs_result_observer_count(out);
    for (size_t f = 0; f < hs_result_frequency_count(out); ++f) {
        hs_frequency_info fi; check(hs_result_frequency_info(out, f, &fi));
        BemFrequencyResult frame;
        frame.frequency = fi.frequency;
        frame.assemblyMilliseconds = fi.assembly_ms;
        frame.solveMilliseconds = fi.solve_ms;
        frame.factorizationMilliseconds = fi.factorization_ms;
        frame.triangularSolveMilliseconds = fi.triangular_solve_ms;
        frame.fieldMilliseconds = fi.field_ms;
        frame.residualCheckMilliseconds = fi.residual_check_ms;
        frame.interactionPlanMilliseconds = fi.interaction_plan_ms;
        frame.interactionPlanReused = fi.interaction_plan_reused;
        for (size_t e = 0; e < request.excitations.size(); ++e) {
            hs_excitation_info xi; check(hs_result_excitation_info(out, f, e, &xi));
            BemExcitationResult ex;
            ex.name = request.excitations[e].name;
            ex.refinementSteps = xi.refinement_steps;
            ex.boundaryResidual = xi.boundary_residual;
            ex.fieldQuadratureComparisonDegree = xi.field_comparison_degree;
            ex.fieldQuadratureVerificationDegree = xi.field_verification_degree;
            ex.fieldQuadratureDiscrepancy = xi.field_discrepancy;
            BemBoundaryData b;
            b.pressureTrace.resize(N); b.surfacePressure.resize(T); b.normalDerivative.resize(T);
            ex.observerPressure.resize(O);
            check(hs_result_pressure_trace(out, f, e, reinterpret_cast<double *>(b.pressureTrace.data())));
            check(hs_result_surface_pressure(out, f, e, reinterpret_cast<double *>(b.surfacePressure.data())));
            check(hs_result_normal_derivative(out, f, e, reinterpret_cast<double *>(b.normalDerivative.data())));
            check(hs_result_observer_pressure(out, f, e, reinterpret_cast<double *>(ex.observerPressure.data())));
            std::vector<hs_face_impedance> z(xi.impedance_count);
            check(hs_result_impedances(out, f, e, z.data()));
            for (auto &i : z)
                ex.impedances.push_back({i.face_id, i.area, {i.mean_pressure[0], i.mean_pressure[1]},
                                         {i.volume_velocity[0], i.volume_velocity[1]},
                                         {i.volume_impedance[0], i.volume_impedance[1]}});
            ex.solvedVelocities = request.excitations[e].faces;
            ex.setBoundary(std::move(b));
            frame.excitations.push_back(std::move(ex));
        }
        result.frequencies.push_back(std::move(frame));
    }
    hs_result_free(out);
    return result;
}

std::string CudaBemSolver::deviceDescription() {
    char name[256];
    check(hs_device_description(name, sizeof name));
    return name;
}
}  // namespace hornsculpt
