// Host-side arena mesh build: validation, uu -> bt conversion, per-triangle normals and bounds, device upload.
#include "rg_mesh.h"

#include <cuda_runtime.h>

#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>

namespace rg {

namespace {
// Positions beyond this (uu, any axis) are rejected, as the reference's ValidateArenaLayout does
// (include/rocketgpu/rocketgpu.h:915, src/rocketgpu.cpp:792-828).
constexpr float kMaxCoordUu = 11500.0f;
}  // namespace

MeshHost build_mesh_host(const float* v, int64_t nv, const int32_t* idx, int64_t ni) {
    if (!v || !idx || nv <= 0 || ni <= 0) throw std::invalid_argument("a custom arena needs a triangle mesh");
    if (ni % 3 != 0) throw std::invalid_argument("a custom arena mesh needs a whole number of triangles (three indices each)");
    for (int64_t i = 0; i < 3 * nv; ++i) {
        if (!std::isfinite(v[i]) || std::fabs(v[i]) > kMaxCoordUu)
            throw std::invalid_argument("ArenaLayout mesh vertex must be finite and within 11500 uu of the origin");
    }
    MeshHost h;
    const int64_t nt = ni / 3;
    h.tris.resize(static_cast<size_t>(nt));
    V3 mn{INFINITY, INFINITY, INFINITY}, mx{-INFINITY, -INFINITY, -INFINITY};
    for (int64_t t = 0; t < nt; ++t) {
        V3 p[3];
        for (int k = 0; k < 3; ++k) {
            const int32_t j = idx[3 * t + k];
            if (j < 0 || j >= nv) throw std::invalid_argument("custom arena mesh triangle index out of range");
            // uu -> bt as the reference's CustomArenaMeshSources: v * (1 / 50) (src/rocketgpu.cpp:680-685)
            p[k] = V3{v[3 * j] * (1.0f / 50.0f), v[3 * j + 1] * (1.0f / 50.0f), v[3 * j + 2] * (1.0f / 50.0f)};
        }
        MeshTri& tri = h.tris[static_cast<size_t>(t)];
        tri.a = p[0];
        tri.b = p[1];
        tri.c = p[2];
        tri.normal = V3{0, 0, 1};
        tri.min = vmin(p[0], vmin(p[1], p[2]));
        tri.max = vmax(p[0], vmax(p[1], p[2]));
        tri.edge_angle[0] = tri.edge_angle[1] = tri.edge_angle[2] = 0.0f;
        tri.edge_flags = 0;
        mn = vmin(mn, tri.min);
        mx = vmax(mx, tri.max);
    }
    h.aabb_min = mn;
    h.aabb_max = mx;
    return h;
}

MeshDevice upload_mesh(const MeshHost& h) {
    MeshDevice d;
    MeshTri* tris = nullptr;
    const size_t bytes = h.tris.size() * sizeof(MeshTri);
    cudaError_t e = cudaMalloc(&tris, bytes);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaMalloc mesh: ") + cudaGetErrorString(e));
    e = cudaMemcpy(tris, h.tris.data(), bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(tris);
        throw std::runtime_error(std::string("upload mesh: ") + cudaGetErrorString(e));
    }
    d.tris = tris;
    d.tri_count = static_cast<int32_t>(h.tris.size());
    return d;
}

void free_mesh(MeshDevice& d) {
    if (d.tris) cudaFree(const_cast<MeshTri*>(d.tris));
    d = MeshDevice{};
}

}  // namespace rg
