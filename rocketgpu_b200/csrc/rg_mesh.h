// Arena mesh: host-side preprocessing of the ArenaLayout triangle mesh and its device copy.
//
// Host build (rg_mesh.cpp), following the reference's custom-arena loader (src/arena/mesh_loader.cpp:1263-1411):
//   1. triangles in Bullet units with their normal and bounds;
//   2. btInternalEdgeUtility-style edge angles between triangles that share an edge (mesh_loader.cpp:57-206);
//   3. the Bullet-style quantized BVH (mesh_loader.cpp:210-396), built only for its leaf order: the reference visits
//      a query's triangles in that order and contact manifolds depend on it.
// Device layout: triangles re-indexed by BVH leaf rank (80 B records, one per rank), and a uniform query grid whose
// cells list, in rank order, every triangle whose quantized bounds overlap the cell grown by kQueryExtentBt. A query
// box no larger than kQueryExtentBt reads exactly one cell, already in the reference's visit order.
#pragma once

#include <cstdint>
#include <vector>

#include "rg_math.cuh"

namespace rg {

// Edge flags (reference ArenaTriangleEdgeFlags, include/rocketgpu/detail/arena/mesh_bvh.hpp:280-288).
constexpr uint32_t kEdgeV0V1Convex = 1u << 0, kEdgeV1V2Convex = 1u << 1, kEdgeV2V0Convex = 1u << 2,
                   kEdgeV0V1Swap = 1u << 3, kEdgeV1V2Swap = 1u << 4, kEdgeV2V0Swap = 1u << 5;

// One triangle as the tick reads it (Bullet units). 80 bytes, 16-byte aligned.
struct alignas(16) DevTri {
    V3 a, b, c;
    V3 normal;
    float edge_angle[3];  // v0v1, v1v2, v2v0; 0 = concave-or-open marker as in the reference
    uint32_t edge_flags;
    uint16_t qmin[3], qmax[3];  // quantized leaf bounds
    int32_t source_index;       // triangle index in the caller's mesh
};
static_assert(sizeof(DevTri) == 80, "DevTri is five 16-byte words");

struct Quantization {
    V3 aabb_min, aabb_max, scale;
};

// Host-side triangle before reordering (reference ArenaMeshTriangle fields the build uses).
struct HostTri {
    V3 a, b, c, normal, min, max;
    float edge_angle[3];
    uint32_t edge_flags;
    uint16_t qmin[3], qmax[3];
};

constexpr float kQueryCellBt = 4.0f;
constexpr float kQueryExtentBt = 4.0f;

// One query-grid entry: a triangle's quantized leaf bounds and its rank, so the overlap test needs no triangle load.
struct alignas(16) CellEntry {
    uint16_t qmin[3], qmax[3];
    int32_t rank;
};
static_assert(sizeof(CellEntry) == 16, "CellEntry is one 16-byte word");

struct MeshHost {
    std::vector<HostTri> tris;          // caller order
    std::vector<int32_t> leaf_order;    // BVH leaf rank -> caller triangle index
    std::vector<DevTri> dev_tris;       // rank order
    Quantization quant{};
    V3 aabb_min{0, 0, 0}, aabb_max{0, 0, 0};
    // query grid
    V3 grid_lo{0, 0, 0};
    int32_t grid_dims[3] = {0, 0, 0};
    std::vector<int32_t> cell_start;       // grid cell -> first entry, size cells + 1
    std::vector<CellEntry> cell_entries;   // per cell, in rank order
    std::vector<CellEntry> rank_entries;   // every triangle in rank order (queries larger than one cell)
};

// Device view (plain pointers; lives in the rg_batch).
struct MeshDevice {
    const DevTri* tris = nullptr;
    int32_t tri_count = 0;
    Quantization quant{};
    V3 aabb_min{0, 0, 0}, aabb_max{0, 0, 0};
    V3 grid_lo{0, 0, 0};
    int32_t grid_dims[3] = {0, 0, 0};
    const int32_t* cell_start = nullptr;
    const CellEntry* cell_entries = nullptr;
    const CellEntry* rank_entries = nullptr;
};

MeshHost build_mesh_host(const float* vertices_uu, int64_t vertex_count, const int32_t* indices, int64_t index_count);
MeshDevice upload_mesh(const MeshHost& h);
void free_mesh(MeshDevice& d);

// Quantizes a point into the BVH's 16-bit grid (reference QuantizeArenaMeshBvhPoint, mesh_bvh.hpp:395-410):
// min corners round down to even, max corners up to odd.
RG_HDI void quantize_point(const Quantization& q, V3 p, int is_max, uint16_t out[3]) {
    V3 c = vmax(p, q.aabb_min);
    c = vmin(c, q.aabb_max);
    const V3 v{(c.x - q.aabb_min.x) * q.scale.x, (c.y - q.aabb_min.y) * q.scale.y, (c.z - q.aabb_min.z) * q.scale.z};
    if (is_max) {
        out[0] = static_cast<uint16_t>(static_cast<uint16_t>(v.x + 1.0f) | 1u);
        out[1] = static_cast<uint16_t>(static_cast<uint16_t>(v.y + 1.0f) | 1u);
        out[2] = static_cast<uint16_t>(static_cast<uint16_t>(v.z + 1.0f) | 1u);
    } else {
        out[0] = static_cast<uint16_t>(static_cast<uint16_t>(v.x) & 0xfffeu);
        out[1] = static_cast<uint16_t>(static_cast<uint16_t>(v.y) & 0xfffeu);
        out[2] = static_cast<uint16_t>(static_cast<uint16_t>(v.z) & 0xfffeu);
    }
}

}  // namespace rg
