// Test infrastructure only: a C entry layer over HornSculpt's own CPU
// galerkin code (space.cpp, pair_quadrature.cpp, interaction_plan.cpp) and its
// post-solve field evaluation (field_evaluation.cpp), compiled from the
// reference tree by oracle/Makefile into oracle/_ref/. It exposes the
// reference's interaction plan and patch estimator with the same flat layout
// as the restated oracle so tests can compare them exactly, and
// evaluatePressureField for the GPU point-sampling parity tests, and the
// fast-multipole support tree (fmm/support_tree.cpp) for the tree parity test.
#include "galerkin/interaction_plan.hpp"
#include <hornsculpt/field_evaluation.hpp>
#include "galerkin/pair_quadrature.hpp"
#include "galerkin/space.hpp"
#include "fmm/support_tree.hpp"

#include <cstring>
#include <string>

using namespace hornsculpt;
using namespace hornsculpt::galerkin;

namespace {
thread_local std::string lastError;
struct Handle {
    InteractionPlan plan;
};
SurfaceMesh makeMesh(const double *verts, size_t nv, const uint32_t *tris, size_t nt) {
    SurfaceMesh m;
    // The solver session centres the mesh on vertex 0 before planning
    // (cuda_solver.cu:771-781); do the same so plans are comparable.
    const Vec3 origin{verts[0], verts[1], verts[2]};
    for (size_t i = 0; i < nv; ++i)
        m.vertices.push_back({verts[3 * i] - origin.x, verts[3 * i + 1] - origin.y, verts[3 * i + 2] - origin.z});
    for (size_t i = 0; i < nt; ++i)
        m.triangles.push_back({{tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]}, 0, BoundaryCondition::wall});
    return m;
}
}  // namespace

extern "C" {
struct ref_numerics {
    unsigned quadrature_order, singular_order;
    double near_ratio, near_tol;
    unsigned near_depth;
    double residual_tol;
    unsigned max_refine;
};
const char *ref_last_error() { return lastError.c_str(); }

int ref_plan_build(const double *verts, size_t nv, const uint32_t *tris, size_t nt, const ref_numerics *nm,
                   double maxK, unsigned threads, void **out) {
    try {
        const Space space = buildSpace(makeMesh(verts, nv, tris, nt));
        PairQuadratureSettings st;
        st.regularOrder = nm->quadrature_order;
        st.singularOrder = nm->singular_order;
        st.nearDistanceRatio = nm->near_ratio;
        st.relativeTolerance = nm->near_tol;
        st.maximumSubdivisionDepth = nm->near_depth;
        auto *h = new Handle{makeInteractionPlan(space, st, maxK, {}, threads)};
        *out = h;
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return 2;
    }
}
void ref_plan_sizes(void *h, size_t *out) {
    const auto &p = static_cast<Handle *>(h)->plan;
    out[0] = p.touching.size();
    out[1] = p.near.size();
    out[2] = p.patches.size();
    out[3] = p.wholePanelDegrees.size();
    out[4] = p.nearTrials.size();
    out[5] = p.maximumDepth;
}
void ref_plan_touching(void *h, uint32_t *out) {
    for (const auto &j : static_cast<Handle *>(h)->plan.touching) {
        *out++ = j.test;
        *out++ = j.trial;
        *out++ = static_cast<uint32_t>(j.permutation.topology);
        for (int i = 0; i < 3; ++i)
            *out++ = j.permutation.test[i];
        for (int i = 0; i < 3; ++i)
            *out++ = j.permutation.trial[i];
    }
}
void ref_plan_near(void *h, uint32_t *out) {
    for (const auto &j : static_cast<Handle *>(h)->plan.near) {
        *out++ = j.test;
        *out++ = j.trial;
        *out++ = j.firstPatch;
        *out++ = j.patchCount;
        *out++ = j.swapBarycentric;
    }
}
void ref_plan_patches(void *h, double *out) {
    for (const auto &p : static_cast<Handle *>(h)->plan.patches) {
        for (int i = 0; i < 9; ++i)
            *out++ = p.test[i];
        for (int i = 0; i < 9; ++i)
            *out++ = p.trial[i];
        *out++ = p.areaFraction;
        *out++ = p.degree;
        *out++ = p.projection;
        *out++ = p.projectionIntervals;
    }
}
void ref_plan_whole(void *h, uint8_t *out) {
    const auto &w = static_cast<Handle *>(h)->plan.wholePanelDegrees;
    if (!w.empty())
        std::memcpy(out, w.data(), w.size());
}
void ref_plan_offsets(void *h, uint32_t *offsets, uint32_t *trials) {
    const auto &p = static_cast<Handle *>(h)->plan;
    std::memcpy(offsets, p.nearOffsets.data(), p.nearOffsets.size() * 4);
    if (!p.nearTrials.empty())
        std::memcpy(trials, p.nearTrials.data(), p.nearTrials.size() * 4);
}
void ref_plan_free(void *h) { delete static_cast<Handle *>(h); }

int ref_triangle_rule(unsigned degree, double *out, size_t *count) {
    try {
        const auto r = triangleRule(degree);
        *count = r.size();
        if (out)
            for (const auto &p : r) {
                *out++ = p.barycentric[0];
                *out++ = p.barycentric[1];
                *out++ = p.barycentric[2];
                *out++ = p.weight;
            }
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return 1;
    }
}
int ref_gauss(unsigned order, double *out) {
    try {
        for (const auto &g : gaussLegendre01(order)) {
            *out++ = g.position;
            *out++ = g.weight;
        }
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return 1;
    }
}
int ref_estimate_patch(const double *tri9a, const double *tri9b, const uint32_t *nodesA, const uint32_t *nodesB,
                       const double *patch22, double k, double *moments72, double *errors3) {
    try {
        SurfaceMesh m;
        for (int i = 0; i < 3; ++i)
            m.vertices.push_back({tri9a[3 * i], tri9a[3 * i + 1], tri9a[3 * i + 2]});
        for (int i = 0; i < 3; ++i)
            m.vertices.push_back({tri9b[3 * i], tri9b[3 * i + 1], tri9b[3 * i + 2]});
        m.triangles.push_back({{0, 1, 2}, 0, BoundaryCondition::wall});
        m.triangles.push_back({{3, 4, 5}, 0, BoundaryCondition::wall});
        const Space space = buildSpace(m);
        Panel a = space.panels[0], b = space.panels[1];
        for (int i = 0; i < 3; ++i) {
            a.nodes[i] = nodesA[i];
            b.nodes[i] = nodesB[i];
        }
        PairQuadraturePatch p;
        for (int i = 0; i < 9; ++i) {
            p.test[i] = patch22[i];
            p.trial[i] = patch22[9 + i];
        }
        p.areaFraction = patch22[18];
        p.degree = unsigned(patch22[19]);
        p.projection = unsigned(patch22[20]);
        p.projectionIntervals = unsigned(patch22[21]);
        const auto e = estimatePairPatchCpu(a, b, p, k);
        for (int i = 0; i < 36; ++i) {
            moments72[2 * i] = e.integral[i].real();
            moments72[2 * i + 1] = e.integral[i].imag();
        }
        errors3[0] = e.absoluteError;
        errors3[1] = e.innerError;
        errors3[2] = e.outerError;
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return 2;
    }
}

// evaluatePressureField (field_evaluation.cpp:330-463) on an exterior closed
// mesh (world coordinates, as given): P1 trace nv and DP0 derivative nt
// complex (interleaved); per point the pressure and the FieldPointStatus.
int ref_pressure_field(const double *verts, size_t nv, const uint32_t *tris, size_t nt, const double *trace,
                       const double *derivative, double frequency, double soundSpeed, const double *points, size_t np,
                       double minDistance, double tolerance, unsigned depth, double *out, int *status) {
    try {
        SurfaceMesh m;
        for (size_t i = 0; i < nv; ++i)
            m.vertices.push_back({verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]});
        for (size_t i = 0; i < nt; ++i)
            m.triangles.push_back({{tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]}, 0, BoundaryCondition::wall});
        BemRequest request;
        request.medium.soundSpeed = soundSpeed;
        BemBoundaryData boundary;
        for (size_t i = 0; i < nv; ++i)
            boundary.pressureTrace.emplace_back(trace[2 * i], trace[2 * i + 1]);
        for (size_t i = 0; i < nt; ++i)
            boundary.normalDerivative.emplace_back(derivative[2 * i], derivative[2 * i + 1]);
        BemExcitationResult solution;
        solution.setBoundary(std::move(boundary));
        std::vector<Vec3> pts;
        for (size_t i = 0; i < np; ++i)
            pts.push_back({points[3 * i], points[3 * i + 1], points[3 * i + 2]});
        PressureFieldSettings settings;
        settings.minimumBoundaryDistance = minDistance;
        settings.relativeQuadratureTolerance = tolerance;
        settings.maximumQuadratureDepth = depth;
        const auto samples = evaluatePressureField(m, request, frequency, solution, pts, settings);
        for (size_t i = 0; i < np; ++i) {
            out[2 * i] = samples[i].pressure.real();
            out[2 * i + 1] = samples[i].pressure.imag();
            status[i] = int(samples[i].status);
        }
        return 0;
    } catch (const std::invalid_argument &e) {
        lastError = e.what();
        return 1;
    } catch (const std::exception &e) {
        lastError = e.what();
        return 2;
    }
}

// makeSupportTree on the centred mesh: sizes = {nodes, levels, pp near, pp far,
// pf near, pf far}; links = (target, source) pairs of the four lists in that
// order (capacity pairs at most).
int ref_support_tree(const double *verts, size_t nv, const uint32_t *tris, size_t nt, unsigned leafCapacity,
                     double separationRatio, double nearDistanceRatio, size_t *sizes, uint32_t *links,
                     size_t capacity) {
    try {
        const Space space = buildSpace(makeMesh(verts, nv, tris, nt));
        wideband::SupportTreeSettings st;
        st.leafCapacity = leafCapacity;
        st.separationRatio = separationRatio;
        st.nearDistanceRatio = nearDistanceRatio;
        const auto tree = wideband::makeSupportTree(space, st);
        sizes[0] = tree.nodes.size();
        sizes[1] = tree.levels.size();
        sizes[2] = tree.pressurePressure.nearInteractions.size();
        sizes[3] = tree.pressurePressure.farInteractions.size();
        sizes[4] = tree.pressureFlux.nearInteractions.size();
        sizes[5] = tree.pressureFlux.farInteractions.size();
        size_t at = 0;
        for (const auto *list : {&tree.pressurePressure.nearInteractions, &tree.pressurePressure.farInteractions,
                                 &tree.pressureFlux.nearInteractions, &tree.pressureFlux.farInteractions})
            for (const auto &lk : *list) {
                if (at < capacity) {
                    links[2 * at] = lk.target;
                    links[2 * at + 1] = lk.source;
                }
                ++at;
            }
        return 0;
    } catch (const std::exception &e) {
        lastError = e.what();
        return 1;
    }
}
}
