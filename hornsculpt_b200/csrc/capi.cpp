// extern "C" entry points of include/hs_bem.h: exceptions of the session
// layer become hs_status codes plus a thread-local message.
#include "hs_bem.h"
#include "autotune.hpp"
#include "plan_device.hpp"
#include "serve.hpp"
#include "session.hpp"

#include <cmath>
#include <cstring>
#include <string>

using namespace hsb;

struct hs_bem_session {
    std::unique_ptr<Session> impl;
};
struct hs_result {
    std::unique_ptr<Result> impl;
};
struct hs_server {
    std::unique_ptr<Server> impl;
};

namespace {
thread_local std::string lastError;

hs_status fail(hs_status code, const char *message) {
    lastError = message;
    return code;
}

template <class F> hs_status guarded(F &&f) {
    try {
        f();
        return HS_OK;
    } catch (const InvalidArgument &e) {
        return fail(HS_E_INVALID, e.what());
    } catch (const std::invalid_argument &e) {
        return fail(HS_E_INVALID, e.what());
    } catch (const Cancelled &e) {
        return fail(HS_E_CANCELLED, e.what());
    } catch (const NoConvergence &e) {
        return fail(HS_E_NOCONVERGE, e.what());
    } catch (const OutOfMemory &e) {
        return fail(HS_E_NOMEM, e.what());
    } catch (const Unsupported &e) {
        return fail(HS_E_UNSUPPORTED, e.what());
    } catch (const NumericError &e) {
        return fail(HS_E_NUMERIC, e.what());
    } catch (const std::bad_alloc &) {
        return fail(HS_E_NOMEM, "Host allocation failed.");
    } catch (const std::exception &e) {
        return fail(HS_E_CUDA, e.what());
    }
}

const ExcitationResult *excitation(const hs_result *r, size_t f, size_t e) {
    if (!r || !r->impl || f >= r->impl->frequencies.size() || e >= r->impl->frequencies[f].excitations.size())
        return nullptr;
    return &r->impl->frequencies[f].excitations[e];
}
hs_status copyComplex(const std::vector<cplx> &v, double *out) {
    if (!out && !v.empty())
        return fail(HS_E_INVALID, "Output buffer is null.");
    if (!v.empty())
        std::memcpy(out, v.data(), v.size() * sizeof(cplx));
    return HS_OK;
}
}  // namespace

extern "C" {

void hs_numerics_default(hs_numerics *o) {
    if (!o)
        return;
    *o = hs_numerics{};
    o->quadrature_order = 4;
    o->singular_order = 4;
    o->near_distance_ratio = 1.0;
    o->near_relative_tolerance = 1e-4;
    o->near_maximum_depth = 6;
    o->relative_residual_tolerance = 5e-5;
    o->maximum_refinement_steps = 3;
    o->acceleration = HS_DENSE;
    o->precision = HS_PRECISION_FP64;
    o->fmm_leaf_support_capacity = 16;
    o->fmm_separation_ratio = 1.5;
    o->fmm_maximum_iterations = 300;
    o->fmm_restart_length = 40;
    o->fmm_preconditioner_block_width = 32;
}

hs_status hs_bem_session_create(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                                const uint32_t *face_ids, const uint8_t *boundary, size_t triangle_count,
                                uint32_t residency, hs_bem_session **out) {
    if (!out)
        return fail(HS_E_INVALID, "Session output pointer is null.");
    *out = nullptr;
    if ((!vertices && vertex_count) || (!triangle_count || !triangles || !face_ids || !boundary))
        return fail(HS_E_INVALID, "BEM mesh has no vertices.");
    return guarded([&]() {
        MeshInput mesh;
        mesh.vertices.resize(vertex_count);
        for (size_t i = 0; i < vertex_count; ++i)
            mesh.vertices[i] = V3{vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]};
        mesh.triangles.assign(triangles, triangles + 3 * triangle_count);
        mesh.faces.assign(face_ids, face_ids + triangle_count);
        mesh.driven.resize(triangle_count);
        for (size_t t = 0; t < triangle_count; ++t) {
            if (boundary[t] > HS_DRIVEN)
                throw InvalidArgument("Triangle boundary must be wall (0) or driven (1).");
            mesh.driven[t] = boundary[t];
        }
        auto s = std::make_unique<hs_bem_session>();
        s->impl = std::make_unique<Session>(mesh, residency);
        *out = s.release();
    });
}

void hs_bem_session_destroy(hs_bem_session *s) { delete s; }

hs_status hs_bem_session_set_stream(hs_bem_session *s, void *stream) {
    if (!s)
        return fail(HS_E_INVALID, "Session is null.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        s->impl->setStream(static_cast<cudaStream_t>(stream));
    });
}

hs_status hs_field_settings_default(hs_field_settings *out) {
    if (!out)
        return fail(HS_E_INVALID, "Settings pointer is null.");
    *out = hs_field_settings{1e-4, 1e-4, 8};  // PressureFieldSettings defaults (field_evaluation.hpp:14-20)
    return HS_OK;
}

hs_status hs_bem_pressure_field(hs_bem_session *s, double frequency, double sound_speed, const double *pressure_trace,
                                const double *normal_derivative, const double *points, size_t point_count,
                                const hs_field_settings *settings, double *pressure, int32_t *status) {
    if (!s || !pressure_trace || !normal_derivative || !settings || (point_count && (!points || !pressure || !status)))
        return fail(HS_E_INVALID, "Session, traces, settings, points and outputs must be non-null.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        s->impl->pressureField(frequency, sound_speed, pressure_trace, normal_derivative, points, point_count,
                               *settings, pressure, status);
    });
}

hs_status hs_bem_solve(hs_bem_session *s, const hs_request *request, const volatile int32_t *cancel,
                       hs_progress_fn progress, void *user, hs_result **out) {
    if (!s || !request || !out)
        return fail(HS_E_INVALID, "Session, request and result pointers must be non-null.");
    *out = nullptr;
    if ((request->frequency_count && !request->frequencies) ||
        (request->plan_frequency_count && !request->plan_frequencies) ||
        (request->excitation_count && !request->excitation_face_offsets) ||
        (request->observer_count && !request->observers))
        return fail(HS_E_INVALID, "Invalid BEM medium, frequencies, excitation or Galerkin settings.");
    if (request->excitation_count) {
        const size_t faces = request->excitation_face_offsets[request->excitation_count];
        if (faces && (!request->excitation_face_ids || !request->excitation_velocities))
            return fail(HS_E_INVALID, "Excitation must assign each known Driven face at most once.");
        for (size_t e = 0; e < request->excitation_count; ++e)
            if (request->excitation_face_offsets[e] > request->excitation_face_offsets[e + 1])
                return fail(HS_E_INVALID, "Excitation face offsets must be nondecreasing.");
    }
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        auto r = std::make_unique<hs_result>();
        r->impl = s->impl->solve(*request, cancel, progress, user);
        *out = r.release();
    });
}

size_t hs_result_frequency_count(const hs_result *r) { return r && r->impl ? r->impl->frequencies.size() : 0; }
size_t hs_result_excitation_count(const hs_result *r) { return r && r->impl ? r->impl->E : 0; }
size_t hs_result_triangle_count(const hs_result *r) { return r && r->impl ? r->impl->T : 0; }
size_t hs_result_pressure_dof_count(const hs_result *r) { return r && r->impl ? r->impl->N : 0; }
size_t hs_result_observer_count(const hs_result *r) { return r && r->impl ? r->impl->O : 0; }
size_t hs_result_peak_device_bytes(const hs_result *r) { return r && r->impl ? r->impl->peakDeviceBytes : 0; }

hs_status hs_result_frequency_info(const hs_result *r, size_t f, hs_frequency_info *out) {
    if (!r || !r->impl || !out || f >= r->impl->frequencies.size())
        return fail(HS_E_INVALID, "Result index out of range.");
    *out = r->impl->frequencies[f].info;
    return HS_OK;
}
hs_status hs_result_excitation_info(const hs_result *r, size_t f, size_t e, hs_excitation_info *out) {
    const ExcitationResult *x = excitation(r, f, e);
    if (!x || !out)
        return fail(HS_E_INVALID, "Result index out of range.");
    out->boundary_residual = x->residual;
    out->refinement_steps = x->refinements;
    out->iterations = x->iterations;
    out->field_comparison_degree = x->fieldDegree;
    out->field_verification_degree = x->fieldNext;
    out->field_discrepancy = x->fieldDiscrepancy;
    out->impedance_count = x->impedances.size();
    return HS_OK;
}
hs_status hs_result_pressure_trace(const hs_result *r, size_t f, size_t e, double *out) {
    const ExcitationResult *x = excitation(r, f, e);
    return x ? copyComplex(x->trace, out) : fail(HS_E_INVALID, "Result index out of range.");
}
hs_status hs_result_surface_pressure(const hs_result *r, size_t f, size_t e, double *out) {
    const ExcitationResult *x = excitation(r, f, e);
    return x ? copyComplex(x->surface, out) : fail(HS_E_INVALID, "Result index out of range.");
}
hs_status hs_result_normal_derivative(const hs_result *r, size_t f, size_t e, double *out) {
    const ExcitationResult *x = excitation(r, f, e);
    return x ? copyComplex(x->normalDerivative, out) : fail(HS_E_INVALID, "Result index out of range.");
}
hs_status hs_result_observer_pressure(const hs_result *r, size_t f, size_t e, double *out) {
    const ExcitationResult *x = excitation(r, f, e);
    return x ? copyComplex(x->observer, out) : fail(HS_E_INVALID, "Result index out of range.");
}
hs_status hs_result_copy_all(const hs_result *r, double *traces, double *surface, double *normal, double *observers,
                             hs_excitation_info *excitation_infos, hs_frequency_info *frequency_infos) {
    if (!r || !r->impl)
        return fail(HS_E_INVALID, "Result handle is null.");
    const auto &fs = r->impl->frequencies;
    const size_t E = r->impl->E, N = r->impl->N, T = r->impl->T, O = r->impl->O;
    for (size_t f = 0; f < fs.size(); ++f) {
        if (frequency_infos)
            frequency_infos[f] = fs[f].info;
        for (size_t e = 0; e < E; ++e) {
            const ExcitationResult *x = excitation(r, f, e);
            if (!x)
                return fail(HS_E_INVALID, "Result index out of range.");
            const size_t q = f * E + e;
            if (traces)
                copyComplex(x->trace, traces + 2 * q * N);
            if (surface)
                copyComplex(x->surface, surface + 2 * q * T);
            if (normal)
                copyComplex(x->normalDerivative, normal + 2 * q * T);
            if (observers)
                copyComplex(x->observer, observers + 2 * q * O);
            if (excitation_infos)
                hs_result_excitation_info(r, f, e, excitation_infos + q);
        }
    }
    return HS_OK;
}
hs_status hs_result_impedances(const hs_result *r, size_t f, size_t e, hs_face_impedance *out) {
    const ExcitationResult *x = excitation(r, f, e);
    if (!x || (!out && !x->impedances.empty()))
        return fail(HS_E_INVALID, "Result index out of range.");
    if (!x->impedances.empty())
        std::memcpy(out, x->impedances.data(), x->impedances.size() * sizeof(hs_face_impedance));
    return HS_OK;
}
void hs_result_free(hs_result *r) { delete r; }

const char *hs_last_error(void) { return lastError.c_str(); }

hs_status hs_device_description(char *buffer, size_t size) {
    int count = 0, dev = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || !count)
        return fail(HS_E_CUDA, "No CUDA device is available.");
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return fail(HS_E_CUDA, "CUDA device properties");
    if (buffer && size) {
        std::strncpy(buffer, prop.name, size - 1);
        buffer[size - 1] = 0;
    }
    return HS_OK;
}

hs_status hs_bem_session_set_profiling(hs_bem_session *s, int32_t enabled) {
    if (!s)
        return fail(HS_E_INVALID, "Session is null.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        s->impl->timer().reset();
        s->impl->timer().enable(enabled != 0);
        std::fill(s->impl->work.begin(), s->impl->work.end(), 0);
    });
}

hs_status hs_bem_solve_coupled(hs_bem_session *s, const hs_request *request, hs_network_fn network, void *user,
                               const volatile int32_t *cancel, hs_result **out) {
    if (!s || !request || !network || !out)
        return fail(HS_E_INVALID, "Coupled solve: session, request, network and output must be non-null.");
    *out = nullptr;
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        const CouplingNetwork bridge = [&](double frequency, const std::vector<cplx> &Z, std::vector<cplx> &Q,
                                           std::vector<cplx> &P) {
            const size_t ports = size_t(std::sqrt(double(Z.size())) + 0.5);
            Q.assign(ports, 0.0);
            P.assign(ports, 0.0);
            const hs_status st = network(frequency, ports, reinterpret_cast<const double *>(Z.data()),
                                         reinterpret_cast<double *>(Q.data()), reinterpret_cast<double *>(P.data()),
                                         user);
            if (st != HS_OK)
                throw InvalidArgument("The lumped network failed for the coupled BEM load.");
        };
        auto result = s->impl->solve(*request, cancel, nullptr, nullptr, nullptr, &bridge);
        *out = new hs_result{std::move(result)};
    });
}

hs_status hs_result_coupling(const hs_result *r, size_t f, double *impedance, double *volume_velocity,
                             double *pressure, size_t *ports) {
    if (!r || !r->impl || f >= r->impl->frequencies.size())
        return fail(HS_E_INVALID, "Result index out of range.");
    const FrequencyResult &fr = r->impl->frequencies[f];
    if (ports)
        *ports = fr.portFlow.size();
    if (impedance && !fr.portImpedance.empty())
        std::memcpy(impedance, fr.portImpedance.data(), fr.portImpedance.size() * sizeof(cplx));
    if (volume_velocity && !fr.portFlow.empty())
        std::memcpy(volume_velocity, fr.portFlow.data(), fr.portFlow.size() * sizeof(cplx));
    if (pressure && !fr.portPressure.empty())
        std::memcpy(pressure, fr.portPressure.data(), fr.portPressure.size() * sizeof(cplx));
    return HS_OK;
}

hs_status hs_bem_session_set_graphs(hs_bem_session *s, int32_t enabled) {
    if (!s)
        return fail(HS_E_INVALID, "Session is null.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        s->impl->setGraphs(enabled != 0);
    });
}

hs_status hs_bem_session_graph_launches(const hs_bem_session *s, uint64_t *launches) {
    if (!s || !launches)
        return fail(HS_E_INVALID, "Session and output must be non-null.");
    *launches = s->impl->graphLaunches();
    return HS_OK;
}

hs_status hs_autotune_set_enabled(int32_t enabled) {
    Autotuner::instance().setEnabled(enabled != 0);
    return HS_OK;
}

hs_status hs_autotune_clear(void) {
    Autotuner::instance().clear();
    return HS_OK;
}

hs_status hs_autotune_report(char *buffer, size_t size, size_t *needed) {
    return guarded([&]() {
        const std::string r = Autotuner::instance().report();
        if (needed)
            *needed = r.size() + 1;
        if (buffer && size) {
            const size_t n = std::min(size - 1, r.size());
            std::memcpy(buffer, r.data(), n);
            buffer[n] = 0;
        }
    });
}

hs_status hs_bem_session_work(const hs_bem_session *s, uint64_t *counters, size_t capacity, size_t *count) {
    if (!s || !count)
        return fail(HS_E_INVALID, "Session is null.");
    std::lock_guard<std::mutex> lock(s->impl->mutex);
    const auto &w = s->impl->work;
    *count = std::min(capacity, w.size());
    for (size_t i = 0; i < *count && counters; ++i)
        counters[i] = w[i];
    return HS_OK;
}

hs_status hs_bem_session_profile(const hs_bem_session *s, char *names, size_t namesSize, double *ms,
                                 uint64_t *launches, size_t capacity, size_t *count) {
    if (!s || !count)
        return fail(HS_E_INVALID, "Session is null.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        auto &timer = s->impl->timer();
        timer.collect();
        std::string joined;
        size_t i = 0;
        for (const auto &[name, total] : timer.totals()) {
            if (i < capacity) {
                if (ms)
                    ms[i] = total.ms;
                if (launches)
                    launches[i] = total.launches;
                joined += (i ? "," : "") + name;
            }
            ++i;
        }
        *count = std::min(i, capacity);
        if (names && namesSize) {
            std::strncpy(names, joined.c_str(), namesSize - 1);
            names[namesSize - 1] = 0;
        }
    });
}

namespace {
// Writes a plan into hs_bem_debug_plan's output layout.
void writePlan(const hsb::Plan &p, size_t *sizes, uint32_t *touching, uint32_t *near, double *patches,
               uint8_t *whole, uint32_t *near_offsets, uint32_t *near_trials) {
    sizes[0] = p.touching.size();
    sizes[1] = p.near.size();
    sizes[2] = p.patches.size();
    sizes[3] = p.wholePanelDegrees.size();
    sizes[4] = p.nearTrials.size();
    sizes[5] = p.maxDepth;
    if (touching)
        for (const auto &j : p.touching) {
            *touching++ = j.test;
            *touching++ = j.trial;
            *touching++ = j.perm.topology;
            for (int i = 0; i < 3; ++i)
                *touching++ = j.perm.test[i];
            for (int i = 0; i < 3; ++i)
                *touching++ = j.perm.trial[i];
        }
    if (near)
        for (const auto &j : p.near) {
            *near++ = j.test;
            *near++ = j.trial;
            *near++ = j.first;
            *near++ = j.count;
            *near++ = j.swap;
        }
    if (patches)
        for (const auto &q : p.patches) {
            for (int i = 0; i < 9; ++i)
                *patches++ = q.test[i];
            for (int i = 0; i < 9; ++i)
                *patches++ = q.trial[i];
            *patches++ = q.areaFraction;
            *patches++ = q.degree;
            *patches++ = q.projection;
            *patches++ = q.intervals;
        }
    if (whole && !p.wholePanelDegrees.empty())
        std::memcpy(whole, p.wholePanelDegrees.data(), p.wholePanelDegrees.size());
    if (near_offsets)
        std::memcpy(near_offsets, p.nearOffsets.data(), p.nearOffsets.size() * 4);
    if (near_trials && !p.nearTrials.empty())
        std::memcpy(near_trials, p.nearTrials.data(), p.nearTrials.size() * 4);
}

hsb::Space debugSpace(const double *vertices, size_t vertex_count, const uint32_t *triangles, size_t triangle_count) {
    MeshInput mesh;
    const V3 origin{vertices[0], vertices[1], vertices[2]};
    for (size_t i = 0; i < vertex_count; ++i)
        mesh.vertices.push_back(V3{vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]} - origin);
    mesh.triangles.assign(triangles, triangles + 3 * triangle_count);
    mesh.faces.assign(triangle_count, 0);
    mesh.driven.assign(triangle_count, 0);
    return buildSpace(mesh);
}

hsb::PlanSettings planSettings(const hs_numerics *n) {
    return hsb::PlanSettings{n->quadrature_order, n->singular_order, n->near_distance_ratio,
                             n->near_relative_tolerance, n->near_maximum_depth};
}
}  // namespace

hs_status hs_bem_debug_plan(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                            size_t triangle_count, const hs_numerics *numerics, double max_k, size_t *sizes,
                            uint32_t *touching, uint32_t *near, double *patches, uint8_t *whole,
                            uint32_t *near_offsets, uint32_t *near_trials) {
    if (!vertices || !vertex_count || !triangles || !triangle_count || !numerics || !sizes)
        return fail(HS_E_INVALID, "Mesh, numerics and sizes must be non-null.");
    return guarded([&]() {
        const Space space = debugSpace(vertices, vertex_count, triangles, triangle_count);
        const Plan p = makePlan(space, planSettings(numerics), max_k, 0, nullptr);
        writePlan(p, sizes, touching, near, patches, whole, near_offsets, near_trials);
    });
}

namespace {
// The last device plan of this thread, so that the size query and the fill
// call of hs_bem_debug_plan_device plan once. Keyed by the inputs' bytes.
struct DevicePlanCache {
    uint64_t key = 0;
    bool valid = false;
    hsb::Plan plan;
    hsb::DevicePlanStats stats;
};
thread_local DevicePlanCache tDevicePlanCache;

uint64_t hashBytes(uint64_t h, const void *data, size_t bytes) {
    const unsigned char *p = static_cast<const unsigned char *>(data);
    for (size_t i = 0; i < bytes; ++i)
        h = (h ^ p[i]) * 1099511628211ull;
    return h;
}
}  // namespace

hs_status hs_bem_debug_plan_device(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                                   size_t triangle_count, const hs_numerics *numerics, double max_k, uint32_t mode,
                                   double *stats, size_t *sizes, uint32_t *touching, uint32_t *near,
                                   double *patches, uint8_t *whole, uint32_t *near_offsets, uint32_t *near_trials) {
    if (!vertices || !vertex_count || !triangles || !triangle_count || !numerics || !sizes || mode > 1)
        return fail(HS_E_INVALID, "Mesh, numerics and sizes must be non-null and the mode 0 or 1.");
    return guarded([&]() {
        uint64_t key = 1469598103934665603ull;
        key = hashBytes(key, vertices, vertex_count * 3 * sizeof(double));
        key = hashBytes(key, triangles, triangle_count * 3 * sizeof(uint32_t));
        key = hashBytes(key, numerics, sizeof(hs_numerics));
        key = hashBytes(key, &max_k, sizeof(max_k));
        key = hashBytes(key, &mode, sizeof(mode));
        DevicePlanCache &c = tDevicePlanCache;
        if (!c.valid || c.key != key) {
            c.valid = false;
            const Space space = debugSpace(vertices, vertex_count, triangles, triangle_count);
            c.stats = DevicePlanStats{};
            c.plan = makePlanOnDevice(space, planSettings(numerics), max_k, nullptr, nullptr, &c.stats, mode == 1);
            if (mode == 0) {
                const cudaError_t e = cudaDeviceSynchronize();
                if (e != cudaSuccess)
                    throw CudaError(std::string("CUDA synchronization: ") + cudaGetErrorString(e));
            }
            c.key = key;
            c.valid = true;
        }
        const DevicePlanStats &st = c.stats;
        if (stats) {
            stats[0] = double(st.devicePairs);
            stats[1] = double(st.projectedPairs);
            stats[2] = double(st.flaggedPairs);
            stats[3] = double(st.wholePanelPairs);
            stats[4] = st.deviceMs;
            stats[5] = st.hostMs;
            stats[6] = double(st.resolvedPairs);
            for (int i = 0; i < 5; ++i) {
                stats[7 + i] = st.phaseMs[i];
                stats[12 + i] = st.hostPhaseMs[i];
            }
            stats[17] = double(st.samples);
            stats[18] = st.refineKernelMs;
            stats[19] = double(st.rootSettledPairs);
        }
        writePlan(c.plan, sizes, touching, near, patches, whole, near_offsets, near_trials);
        if (touching || near || patches || whole || near_offsets || near_trials)
            c.valid = false;  // filled: the next call plans again
    });
}

hs_status hs_bem_debug_assemble(hs_bem_session *s, const hs_numerics *numerics, double plan_k, double k,
                                const double *flux, double *matrix, double *rhs) {
    if (!s || !numerics || !flux || !matrix || !rhs)
        return fail(HS_E_INVALID, "Debug assembly pointers must be non-null.");
    if (!std::isfinite(k) || k <= 0 || !std::isfinite(plan_k) || plan_k < k)
        return fail(HS_E_INVALID, "Debug assembly needs 0 < k <= plan_k.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        s->impl->debugAssemble(*numerics, plan_k, k, flux, matrix, rhs);
    });
}

hs_status hs_bem_debug_lu(uint32_t precision, size_t n, size_t batch, const double *matrices, double *factors,
                          int32_t *pivots, int32_t *info) {
    if (!matrices || !factors || !pivots || !info)
        return fail(HS_E_INVALID, "Debug LU pointers must be non-null.");
    if (precision != HS_PRECISION_FP64 && precision != HS_PRECISION_MIXED)
        return fail(HS_E_INVALID, "Debug LU precision must be HS_PRECISION_FP64 or HS_PRECISION_MIXED.");
    if (n == 0 || batch == 0 || n > 65536 || batch > 64)
        return fail(HS_E_INVALID, "Debug LU needs 1 <= n <= 65536 and 1 <= batch <= 64.");
    return guarded([&]() {
        debugLuFactor(precision == HS_PRECISION_MIXED, uint32_t(n), uint32_t(batch), matrices, factors, pivots, info);
    });
}

hs_status hs_bem_debug_fmm_far(hs_bem_session *s, const hs_numerics *numerics, double k, double tolerance,
                               const double *pressure, double *far, uint32_t *near_row_start, uint32_t *near_cols,
                               size_t near_capacity, size_t *near_count, uint32_t *level_info, size_t level_capacity,
                               size_t *level_count) {
    if (!s || !numerics || !pressure || !far)
        return fail(HS_E_INVALID, "Debug fast-multipole pointers must be non-null.");
    if (!std::isfinite(k) || k <= 0 || !std::isfinite(tolerance) || tolerance <= 0 || tolerance >= 1)
        return fail(HS_E_INVALID, "Debug fast multipole needs k > 0 and 0 < tolerance < 1.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        std::vector<uint32_t> row, col;
        std::vector<hsb::FmmLevelInfo> levels;
        s->impl->debugFmmFar(*numerics, k, tolerance, pressure, far, row, col, levels);
        if (near_count)
            *near_count = col.size();
        if (near_row_start)
            std::copy(row.begin(), row.end(), near_row_start);
        if (near_cols)
            std::copy(col.begin(), col.begin() + std::min(col.size(), near_capacity), near_cols);
        if (level_count)
            *level_count = levels.size();
        if (level_info)
            for (size_t i = 0; i < std::min(levels.size(), level_capacity); ++i) {
                level_info[5 * i] = levels[i].level;
                level_info[5 * i + 1] = levels[i].order;
                level_info[5 * i + 2] = levels[i].nodes;
                level_info[5 * i + 3] = levels[i].m2lLinks;
                level_info[5 * i + 4] = levels[i].planeWave;
            }
    });
}

hs_status hs_bem_session_set_plane_wave_threshold(hs_bem_session *s, double threshold) {
    if (!s || !(threshold > 0))
        return fail(HS_E_INVALID, "Plane-wave threshold must be positive.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        s->impl->setPlaneWaveThreshold(threshold);
    });
}

hs_status hs_bem_session_set_planner(hs_bem_session *s, uint32_t planner) {
    if (!s)
        return fail(HS_E_INVALID, "Session handle is null.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        s->impl->setPlanner(planner);
    });
}

hs_status hs_bem_session_plan_stats(hs_bem_session *s, double *stats) {
    if (!s || !stats)
        return fail(HS_E_INVALID, "Session handle and statistics must be non-null.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        const DevicePlanStats &st = s->impl->planStats();
        stats[0] = double(st.devicePairs);
        stats[1] = double(st.projectedPairs);
        stats[2] = double(st.flaggedPairs);
        stats[3] = double(st.wholePanelPairs);
        stats[4] = st.deviceMs;
        stats[5] = st.hostMs;
        stats[6] = double(st.resolvedPairs);
        for (int i = 0; i < 5; ++i) {
            stats[7 + i] = st.phaseMs[i];
            stats[12 + i] = st.hostPhaseMs[i];
        }
        stats[17] = double(st.samples);
        stats[18] = st.refineKernelMs;
        stats[19] = double(st.rootSettledPairs);
    });
}

hs_status hs_bem_session_set_fmm_grouped_m2l(hs_bem_session *s, int enabled) {
    if (!s)
        return fail(HS_E_INVALID, "Session handle is null.");
    return guarded([&]() {
        std::lock_guard<std::mutex> lock(s->impl->mutex);
        s->impl->setGroupedM2l(enabled != 0);
    });
}

hs_status hs_bem_session_set_fmm_audit(hs_bem_session *s, uint32_t mode) {
    if (!s || mode > 2)
        return fail(HS_E_INVALID, "Fast-multipole audit mode must be 0, 1 or 2.");
    std::lock_guard<std::mutex> lock(s->impl->mutex);
    s->impl->fmmAuditMode_ = mode;
    return HS_OK;
}

hs_status hs_bem_session_fmm_audit_counts(const hs_bem_session *s, uint64_t *direct_audits,
                                          uint64_t *quadrature_promotions) {
    if (!s || !direct_audits || !quadrature_promotions)
        return fail(HS_E_INVALID, "Session and outputs must be non-null.");
    *direct_audits = s->impl->directAudits_;
    *quadrature_promotions = s->impl->quadraturePromotions_;
    return HS_OK;
}

hs_status hs_bem_debug_fmm_selftest(double *error) {
    if (!error)
        return fail(HS_E_INVALID, "Self-test error pointer must be non-null.");
    return guarded([&]() { *error = hsb::fmmSelfTest(); });
}

hs_status hs_bem_debug_fmm_tree(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                                size_t triangle_count, uint32_t leaf_capacity, double separation_ratio,
                                double near_distance_ratio, size_t *sizes, uint32_t *links, size_t capacity) {
    if (!vertices || !triangles || !sizes || !vertex_count || !triangle_count)
        return fail(HS_E_INVALID, "Debug tree needs a mesh and a sizes array.");
    return guarded([&]() {
        std::vector<double> v(vertices, vertices + 3 * vertex_count);
        for (size_t i = 0; i < vertex_count; ++i)
            for (int d = 0; d < 3; ++d)
                v[3 * i + d] = vertices[3 * i + d] - vertices[d];
        hsb::FmmTreeSettings st;
        st.leafCapacity = leaf_capacity;
        st.separationRatio = separation_ratio;
        st.nearDistanceRatio = near_distance_ratio;
        const hsb::FmmTree tree = hsb::buildSupportTree(v.data(), uint32_t(vertex_count), triangles,
                                                        uint32_t(triangle_count), st);
        sizes[0] = tree.nodes.size();
        sizes[1] = tree.levels.size();
        sizes[2] = tree.ppNear.size();
        sizes[3] = tree.ppFar.size();
        sizes[4] = tree.pfNear.size();
        sizes[5] = tree.pfFar.size();
        size_t at = 0;
        for (const auto *list : {&tree.ppNear, &tree.ppFar, &tree.pfNear, &tree.pfFar})
            for (const auto &lk : *list) {
                if (links && at < capacity) {
                    links[2 * at] = lk.target;
                    links[2 * at + 1] = lk.source;
                }
                ++at;
            }
    });
}

hs_status hs_bem_observer_field_noalloc(const double *vertices, size_t vertex_count, const uint32_t *triangles,
                                        size_t triangle_count, const double *pressure_trace, const double *flux,
                                        const double *observers, size_t observer_count, double wavenumber,
                                        uint32_t degree, int32_t far_field, const double *far_origin,
                                        double far_reference_distance, double tolerance, uint32_t maximum_depth,
                                        void *cuda_stream, double *observer_pressure) {
    return guarded([&]() {
        observerFieldNoAlloc(vertices, vertex_count, triangles, triangle_count, pressure_trace, flux, observers,
                             observer_count, wavenumber, degree, far_field, far_origin, far_reference_distance,
                             tolerance, maximum_depth, static_cast<cudaStream_t>(cuda_stream), observer_pressure);
    });
}

void hs_serve_options_default(hs_serve_options *o) {
    if (!o)
        return;
    *o = hs_serve_options{};
    o->workers = 4;
    o->memory_fraction = 0.6;
    o->resident_meshes = 8;
    o->planning_frequency = 0;
    o->max_batch_frequencies = 32;
}

hs_status hs_serve_create(const hs_serve_options *options, hs_server **out) {
    if (!options || !out)
        return fail(HS_E_INVALID, "Serving options and output pointer must be non-null.");
    *out = nullptr;
    return guarded([&]() {
        auto s = std::make_unique<hs_server>();
        s->impl = std::make_unique<Server>(*options);
        *out = s.release();
    });
}

hs_status hs_serve_submit(hs_server *server, const double *vertices, size_t vertex_count, const uint32_t *triangles,
                          const uint32_t *face_ids, const uint8_t *boundary, size_t triangle_count,
                          const hs_request *request, uint64_t *ticket) {
    if (!server || !request || !ticket)
        return fail(HS_E_INVALID, "Server, request and ticket pointers must be non-null.");
    if ((!vertices && vertex_count) || (!triangle_count || !triangles || !face_ids || !boundary))
        return fail(HS_E_INVALID, "BEM mesh has no vertices.");
    if (!request->frequency_count || !request->frequencies || (request->observer_count && !request->observers) ||
        !request->excitation_count || !request->excitation_face_offsets)
        return fail(HS_E_INVALID, "Invalid BEM medium, frequencies, excitation or Galerkin settings.");
    const size_t faces = request->excitation_face_offsets[request->excitation_count];
    if (faces && (!request->excitation_face_ids || !request->excitation_velocities))
        return fail(HS_E_INVALID, "Excitation must assign each known Driven face at most once.");
    return guarded([&]() {
        MeshInput mesh;
        mesh.vertices.resize(vertex_count);
        for (size_t i = 0; i < vertex_count; ++i)
            mesh.vertices[i] = V3{vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]};
        mesh.triangles.assign(triangles, triangles + 3 * triangle_count);
        mesh.faces.assign(face_ids, face_ids + triangle_count);
        mesh.driven.resize(triangle_count);
        for (size_t t = 0; t < triangle_count; ++t) {
            if (boundary[t] > HS_DRIVEN)
                throw InvalidArgument("Triangle boundary must be wall (0) or driven (1).");
            mesh.driven[t] = boundary[t];
        }
        *ticket = server->impl->submit(std::move(mesh), *request);
    });
}

hs_status hs_serve_wait(hs_server *server, uint64_t ticket, hs_result **out, hs_serve_timing *timing) {
    if (!server || !out)
        return fail(HS_E_INVALID, "Server and result pointers must be non-null.");
    *out = nullptr;
    return guarded([&]() {
        hs_serve_timing t{};
        auto r = std::make_unique<hs_result>();
        try {
            r->impl = server->impl->wait(ticket, t);
        } catch (...) {
            if (timing)
                *timing = t;
            throw;
        }
        if (timing)
            *timing = t;
        *out = r.release();
    });
}

void hs_serve_destroy(hs_server *server) { delete server; }

}  // extern "C"
