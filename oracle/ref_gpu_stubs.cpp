// Test infrastructure only. Link stubs for the reference's GPU solver harness
// (oracle/refgpu.mk): the two meshing functions its CudaBemSolver links that
// need CGAL, which this image lacks. The harness only solves meshes generated
// and validated here (closed, outward, self-intersection free by
// hornsculpt_b200.meshes and this library's own checks), so the embedding check
// reports none; chart meshing belongs to sub-domain partitioning, which the
// harness never reaches.
#include "frontal_delaunay.hpp"
#include "mesh_validation.hpp"

#include <stdexcept>

namespace hornsculpt::detail {

EmbeddingValidation validateEmbedding(const SurfaceMesh &, std::vector<std::pair<std::size_t, std::size_t>> *) {
    return {};
}

FrontalChartMesh meshFrontalChart(const SurfaceChart &, std::span<const Vec3>, const MeshingOptions &,
                                  std::stop_token) {
    throw std::logic_error("chart meshing is not part of the reference GPU harness");
}

}  // namespace hornsculpt::detail
