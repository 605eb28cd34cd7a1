// Drives one solve through the reference-side adapter: a hornsculpt::SurfaceMesh
// and hornsculpt::BemRequest (the reference's own types) handed to
// hornsculpt::CudaBemSolver (cuda_bem_solver_b200.cpp over libhs_bem.so), the
// way a HornSculpt caller does (apps/desktop/simulation_dock.cpp:2550-2575).
//
//   adapter_solve <input> <output>
// input (native endianness): u64 N, T, F, O; f64 vertices[3N]; u32 triangles[3T];
// u32 faceIds[T]; u8 driven[T]; f64 frequencies[F]; f64 observers[3O];
// f64 density, soundSpeed, relativeResidualTolerance; u64 repeats. The
// excitation drives face 1 at 1 m/s; the solve runs `repeats` times on one
// solver object (the first plans, later ones reuse the plan like a sweep).
// output: per frequency of the last solve the pressure trace (N complex), the
// observer pressure (O complex) and the boundary residual; stdout: one JSON
// line with the wall-clock milliseconds of every solve call.
#include <hornsculpt/bem.hpp>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <exception>
#include <vector>

namespace {
template <class T> bool get(std::FILE *f, T *dst, size_t n) { return std::fread(dst, sizeof(T), n, f) == n; }
}  // namespace

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: adapter_solve <input> <output>\n");
        return 2;
    }
    try {
        std::FILE *in = std::fopen(argv[1], "rb");
        if (!in)
            throw std::runtime_error("cannot open input");
        uint64_t dims[4];
        if (!get(in, dims, 4))
            throw std::runtime_error("short input");
        const size_t N = dims[0], T = dims[1], F = dims[2], O = dims[3];
        std::vector<double> v(3 * N), freqs(F), obs(3 * O), medium(3);
        uint64_t repeats = 1;
        std::vector<uint32_t> tri(3 * T), faces(T);
        std::vector<uint8_t> driven(T);
        if (!get(in, v.data(), v.size()) || !get(in, tri.data(), tri.size()) || !get(in, faces.data(), T) ||
            !get(in, driven.data(), T) || !get(in, freqs.data(), F) || !get(in, obs.data(), obs.size()) ||
            !get(in, medium.data(), 3) || !get(in, &repeats, 1))
            throw std::runtime_error("short input");
        std::fclose(in);
        hornsculpt::SurfaceMesh mesh;
        for (size_t i = 0; i < N; ++i)
            mesh.vertices.push_back({v[3 * i], v[3 * i + 1], v[3 * i + 2]});
        for (size_t t = 0; t < T; ++t) {
            hornsculpt::Triangle tr;
            tr.vertices = {tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]};
            tr.faceId = faces[t];
            tr.boundary = driven[t] ? hornsculpt::BoundaryCondition::driven : hornsculpt::BoundaryCondition::wall;
            mesh.triangles.push_back(tr);
        }
        hornsculpt::BemRequest request;
        request.medium = {medium[0], medium[1]};
        request.frequencies = freqs;
        request.excitations = {{"unit", {{1u, {1.0, 0.0}}}}};
        for (size_t o = 0; o < O; ++o)
            request.observers.push_back({obs[3 * o], obs[3 * o + 1], obs[3 * o + 2]});
        request.numerics.relativeResidualTolerance = medium[2];
        hornsculpt::CudaBemSolver solver(std::move(mesh));
        hornsculpt::BemResult result;
        std::vector<double> wall;
        for (uint64_t rep = 0; rep < std::max<uint64_t>(repeats, 1); ++rep) {
            const auto t0 = std::chrono::steady_clock::now();
            result = solver.solve(request);
            wall.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
        }
        std::FILE *out = std::fopen(argv[2], "wb");
        if (!out)
            throw std::runtime_error("cannot open output");
        for (const auto &frame : result.frequencies) {
            const auto &e = frame.excitations.at(0);
            const auto &b = *e.boundary();
            std::fwrite(b.pressureTrace.data(), sizeof(b.pressureTrace[0]), b.pressureTrace.size(), out);
            std::fwrite(e.observerPressure.data(), sizeof(e.observerPressure[0]), e.observerPressure.size(), out);
            std::fwrite(&e.boundaryResidual, sizeof(double), 1, out);
        }
        std::fclose(out);
        std::printf("{\"device\": \"%s\", \"frequencies\": %zu, \"triangles\": %zu, \"wall_ms\": [",
                    hornsculpt::CudaBemSolver::deviceDescription().c_str(), result.frequencies.size(),
                    size_t(result.triangleCount));
        for (size_t i = 0; i < wall.size(); ++i)
            std::printf("%s%.4f", i ? ", " : "", wall[i]);
        std::printf("]}\n");
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "adapter_solve: %s\n", e.what());
        return 1;
    }
}
