// Host-side mesh validation, Galerkin space and quadrature rules.
#pragma once

#include "pair_rules.cuh"

#include <stdexcept>
#include <string>
#include <vector>

namespace hsb {

// Error classes mapped onto hs_status codes at the C boundary.
struct InvalidArgument : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
struct NumericError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct NoConvergence : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct OutOfMemory : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct Cancelled : std::runtime_error {
    Cancelled() : std::runtime_error("BEM calculation cancelled.") {}
};
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// P1/DP0 panel (galerkin/space.hpp:11-26).
struct HostPanel {
    uint32_t nodes[3];
    V3 v[3];
    V3 centroid, n;
    double area, maxEdge;
    V3 grad[3], curl[3];
    uint32_t face;
    uint8_t driven;
};

// Pressure DOF i = mesh vertex i, flux DOF t = triangle t (galerkin/space.hpp:33-42).
struct Space {
    std::vector<V3> vertices;
    std::vector<HostPanel> panels;
    std::vector<uint32_t> incOffsets;  // vertex -> incident (panel, local) CSR
    std::vector<uint32_t> incPanel;
    std::vector<uint8_t> incLocal;
    std::vector<double> lumpedMass;
    double surfaceArea{};
};

struct MeshInput {
    std::vector<V3> vertices;
    std::vector<uint32_t> triangles;  // 3 per triangle
    std::vector<uint32_t> faces;
    std::vector<uint8_t> driven;
};

// Watertight, outward and non-nested exterior surface: the reference's
// inspectMesh().watertight() and validateExteriorComponents
// (modules/meshing/src/mesh_quality.cpp:34-38, galerkin/exterior_domain.cpp:72-141).
void validateExteriorSurface(const MeshInput &mesh);
Space buildSpace(const MeshInput &mesh);

// Gauss-Legendre on [0,1] (pair_quadrature.cpp:685-713), order 2..20.
std::vector<GaussPoint> gaussLegendre01(unsigned order);
// Dunavant degree 2/4/6/8 and collapsed tensor Gauss degree 12/14 triangle rules.
std::vector<TriPoint> triangleRule(unsigned degree);

}  // namespace hsb
