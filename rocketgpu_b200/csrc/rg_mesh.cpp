// Host-side arena mesh build (see rg_mesh.h): validation, uu -> bt, normals and bounds, internal-edge angles, the
// Bullet-style quantized BVH's leaf order, the rank-ordered device triangles and the query grid, and the upload.
#include "rg_mesh.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>

#include "rg_ucrt.cuh"

namespace rg {

namespace {
// Positions beyond this (uu, any axis) are rejected, as the reference's ValidateArenaLayout does
// (include/rocketgpu/rocketgpu.h:915, src/rocketgpu.cpp:792-828).
constexpr float kMaxCoordUu = 11500.0f;
constexpr float kTwoPi = 6.28318548f;  // 2 * Pi() as a float

// Unit vector or fallback (reference Normalize, include/rocketgpu/detail/math.hpp:697-704).
V3 normalize_or(V3 v, V3 fallback) {
    const float l2 = dot(v, v);
    if (l2 <= 1e-12f) return fallback;
    const float inv = 1.0f / sqrtf(l2);
    return v * inv;
}
// Same with the plain x*x + y*y + z*z grouping (reference mesh_loader.cpp:33-40).
V3 normalize_sse_or(V3 v, V3 fallback) {
    const float l2 = v.x * v.x + v.y * v.y + v.z * v.z;
    if (l2 <= 1e-12f) return fallback;
    const float inv = 1.0f / sqrtf(l2);
    return V3{v.x * inv, v.y * inv, v.z * inv};
}

// Bullet quaternion from axis and angle, and quaternion rotation (reference math.hpp:876-895).
Q4 quat_axis_angle(V3 axis, float angle) {
    const float d = len(axis);
    const float s = game_sinf(angle * 0.5f) / d;
    return Q4{game_cosf(angle * 0.5f), axis.x * s, axis.y * s, axis.z * s};
}
V3 quat_rotate(Q4 q, V3 v) {
    const float rx = q.w * v.x + q.y * v.z - q.z * v.y;
    const float ry = q.w * v.y + q.z * v.x - q.x * v.z;
    const float rz = q.w * v.z + q.x * v.y - q.y * v.x;
    const float rw = -q.x * v.x - q.y * v.y - q.z * v.z;
    const float cx = -q.x, cy = -q.y, cz = -q.z, cw = q.w;
    return V3{rw * cx + rx * cw + ry * cz - rz * cy, rw * cy + ry * cw + rz * cx - rx * cz,
              rw * cz + rz * cw + rx * cy - ry * cx};
}

// Internal-edge angle between triangle a and its neighbour b across their shared edge, stored on a: Bullet's
// btInternalEdgeUtility (reference PopulateTriangleInternalEdgeInfo, src/arena/mesh_loader.cpp:57-206).
void edge_info(std::vector<HostTri>& tris, int ia, int ib) {
    constexpr float kEqualVertexThresholdSq = 1.0e-4f * 1.0e-4f;
    const HostTri& ta = tris[ia];
    const HostTri& tb = tris[ib];
    const V3 va[3] = {ta.a, ta.b, ta.c};
    const V3 vb[3] = {tb.a, tb.b, tb.c};
    int sa[2] = {-1, -1}, sb[2] = {-1, -1};
    int shared = 0;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            const V3 d = va[i] - vb[j];
            if (dot(d, d) < kEqualVertexThresholdSq) {
                sa[shared] = i;
                sb[shared] = j;
                ++shared;
                if (shared >= 3) return;
                break;
            }
        }
        if (shared >= 3) return;
    }
    if (shared != 2) return;
    if (sa[0] == 0 && sa[1] == 2) {
        std::swap(sa[0], sa[1]);
        std::swap(sb[0], sb[1]);
    }
    HostTri& wa = tris[ia];
    const int sum_a = sa[0] + sa[1];
    const int other_a = 3 - sum_a;
    const int other_b = 3 - (sb[0] + sb[1]);
    V3 edge = va[sa[1]] - va[sa[0]];
    if (dot(edge, edge) <= 1.0e-12f) return;
    edge = normalize_sse_or(edge, V3{1, 0, 0});
    const V3 normal_a = normalize_sse_or(cross(va[1] - va[0], va[2] - va[0]), V3{0, 0, 1});
    const V3 b0 = vb[sb[1]], b1 = vb[sb[0]], b2 = vb[other_b];
    const V3 normal_b = normalize_sse_or(cross(b1 - b0, b2 - b0), normalize_or(tb.normal, V3{0, 0, 1}));
    V3 ecross_a = normalize_sse_or(cross(edge, normal_a), normal_a);
    if (dot(ecross_a, va[other_a] - va[sa[0]]) < 0.0f) ecross_a = -ecross_a;
    V3 ecross_b = normalize_sse_or(cross(edge, normal_b), normal_b);
    if (dot(ecross_b, vb[other_b] - vb[sb[0]]) < 0.0f) ecross_b = -ecross_b;
    float corrected = 0.0f;
    bool convex = false;
    const V3 calc_edge = cross(ecross_a, ecross_b);
    if (dot(calc_edge, calc_edge) >= 0.0001f) {
        const V3 calc_edge_unit = normalize_sse_or(calc_edge, edge);
        const V3 calc_normal_a = normalize_sse_or(cross(calc_edge_unit, ecross_a), normal_a);
        const float angle2 = ucrt_atan2f(dot(ecross_b, calc_normal_a), dot(ecross_b, ecross_a));
        const float ang4 = 3.14159274f - angle2;
        convex = dot(normal_a, ecross_b) < 0.0f;
        corrected = convex ? ang4 : -ang4;
    }
    auto set = [&](int slot, uint32_t convex_flag, uint32_t swap_flag, V3 axis) {
        V3 nb = quat_rotate(quat_axis_angle(axis, -corrected), normal_a);
        if (dot(nb, normal_b) < 0.0f) wa.edge_flags |= swap_flag;
        wa.edge_angle[slot] = -corrected;
        if (convex) wa.edge_flags |= convex_flag;
    };
    switch (sum_a) {
        case 1: set(0, kEdgeV0V1Convex, kEdgeV0V1Swap, va[0] - va[1]); break;
        case 2: set(2, kEdgeV2V0Convex, kEdgeV2V0Swap, va[2] - va[0]); break;
        case 3: set(1, kEdgeV1V2Convex, kEdgeV1V2Swap, va[1] - va[2]); break;
        default: break;
    }
}

// BVH quantization over the mesh bounds with a 1 bt margin, snapped so the bounds land on quantization steps
// (reference SetArenaMeshBvhQuantization with legacy_282, include/rocketgpu/detail/arena/mesh_bvh.hpp:323-360).
Quantization make_quantization(V3 mn, V3 mx) {
    const V3 clamp{1.0f, 1.0f, 1.0f};
    Quantization q;
    q.aabb_min = mn - clamp;
    q.aabb_max = mx + clamp;
    V3 size = q.aabb_max - q.aabb_min;
    q.scale = V3{65533.0f / size.x, 65533.0f / size.y, 65533.0f / size.z};
    uint16_t qmin[3];
    const V3 cur_min = q.aabb_min;
    quantize_point(q, cur_min, 0, qmin);
    const V3 unq_min{static_cast<float>(qmin[0]) / q.scale.x, static_cast<float>(qmin[1]) / q.scale.y,
                     static_cast<float>(qmin[2]) / q.scale.z};
    q.aabb_min = vmin(cur_min, cur_min + unq_min - clamp);
    const V3 new_min = q.aabb_min;
    const V3 cur_max = q.aabb_max;
    const float qx = (cur_max.x - new_min.x) * q.scale.x;
    const float qy = (cur_max.y - new_min.y) * q.scale.y;
    const float qz = (cur_max.z - new_min.z) * q.scale.z;
    const uint16_t qmax[3] = {static_cast<uint16_t>(static_cast<uint16_t>(static_cast<int>(qx + 1.0f)) | 1),
                              static_cast<uint16_t>(static_cast<uint16_t>(static_cast<int>(qy + 1.0f)) | 1),
                              static_cast<uint16_t>(static_cast<uint16_t>(static_cast<int>(qz + 1.0f)) | 1)};
    const V3 unq_max{static_cast<float>(qmax[0]) / q.scale.x, static_cast<float>(qmax[1]) / q.scale.y,
                     static_cast<float>(qmax[2]) / q.scale.z};
    q.aabb_max = vmax(cur_max, new_min + unq_max + clamp);
    size = q.aabb_max - q.aabb_min;
    q.scale = V3{65533.0f / size.x, 65533.0f / size.y, 65533.0f / size.z};
    return q;
}

V3 unquantize(const Quantization& q, const uint16_t in[3]) {
    return V3{q.aabb_min.x + static_cast<float>(in[0]) / q.scale.x, q.aabb_min.y + static_cast<float>(in[1]) / q.scale.y,
              q.aabb_min.z + static_cast<float>(in[2]) / q.scale.z};
}

struct Leaf {
    uint16_t qmin[3], qmax[3];
    int32_t tri;
};

// Leaf order of Bullet's quantized BVH build (btQuantizedBvh::buildTree: split on the axis of largest centre
// variance at the mean, fall back to the middle when unbalanced; reference mesh_loader.cpp:210-396). Only the leaf
// sequence is kept: it is the order every query visits triangles in.
void bvh_leaf_order(const Quantization& q, std::vector<Leaf>& leaves, int start, int end) {
    const int n = end - start;
    if (n == 1) return;
    auto center = [&](const Leaf& l) { return (unquantize(q, l.qmax) + unquantize(q, l.qmin)) * 0.5f; };
    V3 means{0, 0, 0}, var{0, 0, 0};
    for (int i = start; i < end; ++i) means = means + center(leaves[i]);
    means = means * (1.0f / static_cast<float>(n));
    for (int i = start; i < end; ++i) {
        V3 d = center(leaves[i]) - means;
        d = V3{d.x * d.x, d.y * d.y, d.z * d.z};
        var = var + d;
    }
    var = var * (1.0f / static_cast<float>(n - 1));
    const int axis = var.x < var.y ? (var.y < var.z ? 2 : 1) : (var.x < var.z ? 2 : 0);
    // sort and split
    V3 m2{0, 0, 0};
    for (int i = start; i < end; ++i) m2 = m2 + center(leaves[i]);
    m2 = m2 * (1.0f / static_cast<float>(n));
    const float split_value = axis == 0 ? m2.x : (axis == 1 ? m2.y : m2.z);
    int split = start;
    for (int i = start; i < end; ++i) {
        const V3 c = center(leaves[i]);
        const float cv = axis == 0 ? c.x : (axis == 1 ? c.y : c.z);
        if (cv > split_value) {
            std::swap(leaves[i], leaves[split]);
            ++split;
        }
    }
    const int balanced = n / 3;
    if (split <= start + balanced || split >= end - 1 - balanced) split = start + (n >> 1);
    bvh_leaf_order(q, leaves, start, split);
    bvh_leaf_order(q, leaves, split, end);
}

}  // namespace

MeshHost build_mesh_host(const float* v, int64_t nv, const int32_t* idx, int64_t ni) {
    if (!v || !idx || nv <= 0 || ni <= 0) throw std::invalid_argument("a custom arena needs a triangle mesh");
    if (ni % 3 != 0)
        throw std::invalid_argument("a custom arena mesh needs a whole number of triangles (three indices each)");
    for (int64_t i = 0; i < 3 * nv; ++i) {
        if (!std::isfinite(v[i]) || std::fabs(v[i]) > kMaxCoordUu)
            throw std::invalid_argument("ArenaLayout mesh vertex must be finite and within 11500 uu of the origin");
    }
    MeshHost h;
    const int64_t nt = ni / 3;
    if (nt > (1 << 24)) throw std::invalid_argument("custom arena mesh has too many triangles");
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
        HostTri& tri = h.tris[static_cast<size_t>(t)];
        tri.a = p[0];
        tri.b = p[1];
        tri.c = p[2];
        tri.normal = normalize_or(cross(p[1] - p[0], p[2] - p[0]), V3{0, 0, 1});
        tri.min = V3{fmin_(p[0].x, fmin_(p[1].x, p[2].x)), fmin_(p[0].y, fmin_(p[1].y, p[2].y)),
                     fmin_(p[0].z, fmin_(p[1].z, p[2].z))};
        tri.max = V3{fmax_(p[0].x, fmax_(p[1].x, p[2].x)), fmax_(p[0].y, fmax_(p[1].y, p[2].y)),
                     fmax_(p[0].z, fmax_(p[1].z, p[2].z))};
        tri.edge_angle[0] = tri.edge_angle[1] = tri.edge_angle[2] = kTwoPi;
        tri.edge_flags = 0;
        mn = vmin(mn, tri.min);
        mx = vmax(mx, tri.max);
    }
    h.aabb_min = mn;
    h.aabb_max = mx;

    // internal-edge angles: candidate neighbours share a 0.001 bt vertex cell (reference mesh_loader.cpp:1317-1367)
    {
        constexpr float kCell = 1.0e-3f;
        auto key = [](int64_t x, int64_t y, int64_t z) {
            return (static_cast<uint64_t>(x & 0x1fffff) << 42) | (static_cast<uint64_t>(y & 0x1fffff) << 21) |
                   static_cast<uint64_t>(z & 0x1fffff);
        };
        auto cell_of = [&](V3 p, int64_t c[3]) {
            c[0] = static_cast<int64_t>(std::floor(p.x / kCell));
            c[1] = static_cast<int64_t>(std::floor(p.y / kCell));
            c[2] = static_cast<int64_t>(std::floor(p.z / kCell));
        };
        std::unordered_map<uint64_t, std::vector<int32_t>> by_cell;
        for (int32_t t = 0; t < nt; ++t) {
            const HostTri& tri = h.tris[t];
            for (const V3* p : {&tri.a, &tri.b, &tri.c}) {
                int64_t c[3];
                cell_of(*p, c);
                auto& list = by_cell[key(c[0], c[1], c[2])];
                if (list.empty() || list.back() != t) list.push_back(t);
            }
        }
        std::vector<int32_t> cand;
        for (int32_t ta = 0; ta < nt; ++ta) {
            const HostTri& A = h.tris[ta];
            cand.clear();
            for (const V3* p : {&A.a, &A.b, &A.c}) {
                int64_t c[3];
                cell_of(*p, c);
                for (int dx = -1; dx <= 1; ++dx)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dz = -1; dz <= 1; ++dz) {
                            auto it = by_cell.find(key(c[0] + dx, c[1] + dy, c[2] + dz));
                            if (it != by_cell.end()) cand.insert(cand.end(), it->second.begin(), it->second.end());
                        }
            }
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            for (int32_t tb : cand) {
                if (tb == ta) continue;
                const HostTri& B = h.tris[tb];
                if (A.max.x < B.min.x || A.min.x > B.max.x || A.max.y < B.min.y || A.min.y > B.max.y ||
                    A.max.z < B.min.z || A.min.z > B.max.z)
                    continue;
                edge_info(h.tris, ta, tb);
            }
        }
        for (HostTri& t : h.tris)
            for (float& a : t.edge_angle)
                if (a == kTwoPi) a = 0.0f;
    }

    // quantization, leaf bounds (degenerate extents widened to 0.002 bt, mesh_loader.cpp:217-238), leaf order
    h.quant = make_quantization(mn, mx);
    std::vector<Leaf> leaves(static_cast<size_t>(nt));
    for (int32_t t = 0; t < nt; ++t) {
        HostTri& tri = h.tris[t];
        V3 lo = tri.min, hi = tri.max;
        if (hi.x - lo.x < 0.002f) { hi.x += 0.001f; lo.x -= 0.001f; }
        if (hi.y - lo.y < 0.002f) { hi.y += 0.001f; lo.y -= 0.001f; }
        if (hi.z - lo.z < 0.002f) { hi.z += 0.001f; lo.z -= 0.001f; }
        quantize_point(h.quant, lo, 0, leaves[t].qmin);
        quantize_point(h.quant, hi, 1, leaves[t].qmax);
        leaves[t].tri = t;
        for (int a = 0; a < 3; ++a) {
            tri.qmin[a] = leaves[t].qmin[a];
            tri.qmax[a] = leaves[t].qmax[a];
        }
    }
    bvh_leaf_order(h.quant, leaves, 0, static_cast<int>(nt));
    h.leaf_order.resize(static_cast<size_t>(nt));
    h.dev_tris.resize(static_cast<size_t>(nt));
    for (int32_t r = 0; r < nt; ++r) {
        const int32_t t = leaves[r].tri;
        h.leaf_order[r] = t;
        const HostTri& s = h.tris[t];
        DevTri& d = h.dev_tris[r];
        d.a = s.a;
        d.b = s.b;
        d.c = s.c;
        d.normal = s.normal;
        for (int k = 0; k < 3; ++k) d.edge_angle[k] = s.edge_angle[k];
        d.edge_flags = s.edge_flags;
        for (int a = 0; a < 3; ++a) {
            d.qmin[a] = s.qmin[a];
            d.qmax[a] = s.qmax[a];
        }
        d.source_index = t;
    }

    // query grid over the quantized leaf bounds, each cell grown by the largest single-cell query
    h.grid_lo = h.quant.aabb_min;
    const V3 span = h.quant.aabb_max - h.quant.aabb_min;
    h.grid_dims[0] = static_cast<int32_t>(std::ceil(span.x / kQueryCellBt)) + 1;
    h.grid_dims[1] = static_cast<int32_t>(std::ceil(span.y / kQueryCellBt)) + 1;
    h.grid_dims[2] = static_cast<int32_t>(std::ceil(span.z / kQueryCellBt)) + 1;
    const int64_t cells = static_cast<int64_t>(h.grid_dims[0]) * h.grid_dims[1] * h.grid_dims[2];
    std::vector<std::vector<int32_t>> lists(static_cast<size_t>(cells));
    for (int32_t r = 0; r < nt; ++r) {
        const DevTri& d = h.dev_tris[r];
        const V3 lo = unquantize(h.quant, d.qmin);
        const V3 hi = unquantize(h.quant, d.qmax);
        int c0[3], c1[3];
        const float lo3[3] = {lo.x - h.grid_lo.x, lo.y - h.grid_lo.y, lo.z - h.grid_lo.z};
        const float hi3[3] = {hi.x - h.grid_lo.x, hi.y - h.grid_lo.y, hi.z - h.grid_lo.z};
        for (int a = 0; a < 3; ++a) {
            // a cell c serves queries whose min corner lies in it; such a query reaches at most
            // (c + 1) * cell + extent, so the triangle belongs to every cell from (lo - extent) / cell to hi / cell.
            c0[a] = std::max(0, static_cast<int>(std::floor((lo3[a] - kQueryExtentBt) / kQueryCellBt)) - 1);
            c1[a] = std::min(h.grid_dims[a] - 1, static_cast<int>(std::floor(hi3[a] / kQueryCellBt)) + 1);
        }
        for (int z = c0[2]; z <= c1[2]; ++z)
            for (int y = c0[1]; y <= c1[1]; ++y)
                for (int x = c0[0]; x <= c1[0]; ++x)
                    lists[(static_cast<size_t>(z) * h.grid_dims[1] + y) * h.grid_dims[0] + x].push_back(r);
    }
    h.cell_start.assign(static_cast<size_t>(cells) + 1, 0);
    for (int64_t c = 0; c < cells; ++c) h.cell_start[c + 1] = h.cell_start[c] + static_cast<int32_t>(lists[c].size());
    auto entry_of = [&](int32_t r) {
        CellEntry e;
        for (int a = 0; a < 3; ++a) {
            e.qmin[a] = h.dev_tris[r].qmin[a];
            e.qmax[a] = h.dev_tris[r].qmax[a];
        }
        e.rank = r;
        return e;
    };
    h.cell_entries.reserve(static_cast<size_t>(h.cell_start[cells]));
    for (auto& l : lists)
        for (int32_t r : l) h.cell_entries.push_back(entry_of(r));
    h.rank_entries.reserve(static_cast<size_t>(nt));
    for (int32_t r = 0; r < nt; ++r) h.rank_entries.push_back(entry_of(r));
    return h;
}

namespace {
template <class T>
T* upload_array(const std::vector<T>& v, const char* what) {
    T* p = nullptr;
    const size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e));
    if (!v.empty()) {
        e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(p);
            throw std::runtime_error(std::string("upload ") + what + ": " + cudaGetErrorString(e));
        }
    }
    return p;
}
}  // namespace

MeshDevice upload_mesh(const MeshHost& h) {
    MeshDevice d;
    d.tris = upload_array(h.dev_tris, "mesh triangles");
    d.tri_count = static_cast<int32_t>(h.dev_tris.size());
    d.quant = h.quant;
    d.aabb_min = h.aabb_min;
    d.aabb_max = h.aabb_max;
    d.grid_lo = h.grid_lo;
    for (int a = 0; a < 3; ++a) d.grid_dims[a] = h.grid_dims[a];
    d.cell_start = upload_array(h.cell_start, "mesh grid");
    d.cell_entries = upload_array(h.cell_entries, "mesh grid lists");
    d.rank_entries = upload_array(h.rank_entries, "mesh rank list");
    return d;
}

void free_mesh(MeshDevice& d) {
    if (d.tris) cudaFree(const_cast<DevTri*>(d.tris));
    if (d.cell_start) cudaFree(const_cast<int32_t*>(d.cell_start));
    if (d.cell_entries) cudaFree(const_cast<CellEntry*>(d.cell_entries));
    if (d.rank_entries) cudaFree(const_cast<CellEntry*>(d.rank_entries));
    d = MeshDevice{};
}

}  // namespace rg
