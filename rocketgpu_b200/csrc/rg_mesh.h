// Arena mesh: host-side preprocessing of the ArenaLayout triangle mesh and its device copy.
#pragma once

#include <cstdint>
#include <vector>

#include "rg_math.cuh"

namespace rg {

// One triangle in Bullet units (uu / 50).
struct MeshTri {
    V3 a, b, c;
    V3 normal;
    V3 min, max;
    float edge_angle[3];  // v0v1, v1v2, v2v0 (0 = open edge)
    uint32_t edge_flags;
};

struct MeshHost {
    std::vector<MeshTri> tris;
    V3 aabb_min{0, 0, 0}, aabb_max{0, 0, 0};
};

// Device view (plain pointers; lives in the rg_batch).
struct MeshDevice {
    const MeshTri* tris = nullptr;
    int32_t tri_count = 0;
};

MeshHost build_mesh_host(const float* vertices_uu, int64_t vertex_count, const int32_t* indices, int64_t index_count);
MeshDevice upload_mesh(const MeshHost& h);
void free_mesh(MeshDevice& d);

}  // namespace rg
