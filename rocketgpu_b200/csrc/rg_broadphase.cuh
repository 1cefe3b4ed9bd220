// The arena's broadphase history and persistent-manifold list, host+device.
//
// The solver visits contact rows in the order of the world's persistent manifolds after Bullet's island sort, so that
// order is part of the result. The reference keeps it by emulating Bullet 2.8x's btAxisSweep3 pair cache and the
// dispatcher's manifold array per arena (BuildBulletManifoldList, include/rocketgpu/detail/step/arena_geometry.hpp:
// 4162-5010; the sweep helpers :695-830, 4036-4160; body proxies ComputeBulletBodyProxy :3873-4035; island sort
// SortBulletManifoldListByIsland, env_step.hpp:4269-4303, with QuickSortSharedContactOrderIndices,
// arena_geometry.hpp:5278-5326). This file restates that integer bookkeeping for one arena:
//   * a sweep over three axes of 16-bit quantized edges with one static handle (the arena mesh) and one handle per
//     body (ball = body 0, car slot i = body i + 1), whose edge crossings add and remove overlapping pairs;
//   * the manifold list: a pair's manifold appears once its bodies' child AABBs overlap (for a new car/car or
//     ball/car pair also their boxes, for a new car/mesh pair the compound child test) and leaves with the overlap;
//     each tick's predictive (CCD) contacts are appended as their own entries and dropped the next tick;
//   * islands: bodies joined by ball/car or car/car pairs, and the quicksort of the list by island id.
// Arrays are sized for this port's limits: one static mesh handle and at most 9 bodies.
#pragma once

#include "rg_math.cuh"

namespace rg {

constexpr int kBpBodies = 9;                    // ball + up to 8 car slots
constexpr int kBpHandles = 1 + 1 + kBpBodies;   // handle 0 is the sentinel, handle 1 the mesh
constexpr int kBpEdges = 2 * (kBpHandles - 1) + 2;
constexpr int kBpMaxEntries = 96;               // the reference's kMaxContactOrder
constexpr int kBpPredictiveId = 99;             // static id of a predictive (CCD) manifold
constexpr float kSweepHalfExtentBt = 10485.740234375f;

// Manifold / pair keys: kind 0 ball-static, 1 ball-car, 2 car-static, 3 car-car (reference PackBulletPairKey).
RG_HD uint32_t bp_key(int kind, int body_a, int body_b, int static_id) {
    return (static_cast<uint32_t>(kind) & 3u) | ((static_cast<uint32_t>(body_a + 1) & 15u) << 2) |
           ((static_cast<uint32_t>(body_b + 1) & 15u) << 6) | ((static_cast<uint32_t>(static_id) & 0xffffu) << 16);
}
RG_HD int bp_kind(uint32_t k) { return static_cast<int>(k & 3u); }
RG_HD int bp_body_a(uint32_t k) { return static_cast<int>((k >> 2) & 15u) - 1; }
RG_HD int bp_body_b(uint32_t k) { return static_cast<int>((k >> 6) & 15u) - 1; }
RG_HD int bp_static(uint32_t k) { return static_cast<int>(static_cast<int16_t>(k >> 16)); }
// The body whose island an entry belongs to (the ball for kinds 0 and 1).
RG_HD int bp_entry_body(uint32_t k) { return bp_kind(k) <= 1 ? 0 : bp_body_a(k) + 1; }

// Persistent per arena (reference BulletSweepHistory + BulletBroadphaseHistory). Zero = never swept.
struct alignas(16) Broadphase {
    uint8_t handle_count, static_count, next_fresh, free_count;
    uint8_t obj_count, pair_count, manifold_count, predictive_count;
    uint8_t free_[kBpBodies];
    uint8_t body_handle[kBpBodies];
    uint8_t obj[kBpBodies];
    uint8_t edge_handle[3][kBpEdges];
    uint8_t min_edge[kBpHandles][3];
    uint8_t max_edge[kBpHandles][3];
    uint8_t pad0[3];
    int16_t static_id[kBpHandles];
    uint16_t edge_pos[3][kBpEdges];
    uint32_t pairs[kBpMaxEntries];
    uint32_t manifolds[kBpMaxEntries];
    uint32_t predictive[kBpBodies];
    uint32_t pad1[3];
    // each body's swept AABB as the last sweep saw it (Bullet units: min xyz, max xyz) and which entries hold one;
    // suspension rays skip bodies whose box misses them (reference sap_body_aabb, arena_geometry.hpp:712-721)
    float body_aabb[kBpBodies][6];
    uint16_t body_aabb_valid;
    uint16_t pad2[7];
};

// A body's broadphase proxy for this tick (reference BulletBroadphaseProxy).
struct BpProxy {
    V3 aabb_min, aabb_max;            // swept AABB (now and predicted) grown by the contact threshold
    V3 child_min, child_max;          // the collision shape's AABB now
    V3 child_center, child_half;
    V3 axis[3];                       // car basis columns
    V3 local_min, local_max, origin;  // car child box in body space, body origin
    uint8_t valid, is_ball;
};

RG_HD uint16_t sweep_quantize(float v, int is_max) {
    const float q = 65535.0f / (kSweepHalfExtentBt + kSweepHalfExtentBt);
    float s = (v + kSweepHalfExtentBt) * q;
    s = s >= 0.0f ? (s < 65535.0f ? s : 65535.0f) : 0.0f;
    return static_cast<uint16_t>((static_cast<int>(s) & 0xfffe) | is_max);
}
RG_HD bool aabb_overlap(V3 a0, V3 a1, V3 b0, V3 b1) {
    return !(a1.x < b0.x || a0.x > b1.x || a1.y < b0.y || a0.y > b1.y || a1.z < b0.z || a0.z > b1.z);
}

// ---- proxies (reference ComputeBulletBodyProxy) -----------------------------------------------------------------
RG_HDI void ball_proxy(BpProxy& p, V3 pos_bt, V3 predict_vel_bt, float ball_radius_uu, float dt) {
    constexpr float kThr = 0.02f, kExtra = 0.08f;
    const V3 pred = pos_bt + predict_vel_bt * dt;
    const float extent = ball_radius_uu * (1.0f / 50.0f) + kExtra;
    const float pe = (ball_radius_uu * (1.0f / 50.0f) + 0.5f * kExtra) + 0.5f * kExtra;
    p.aabb_min = V3{fmin_(pos_bt.x, pred.x) - pe - kThr, fmin_(pos_bt.y, pred.y) - pe - kThr,
                    fmin_(pos_bt.z, pred.z) - pe - kThr};
    p.aabb_max = V3{fmax_(pos_bt.x, pred.x) + pe + kThr, fmax_(pos_bt.y, pred.y) + pe + kThr,
                    fmax_(pos_bt.z, pred.z) + pe + kThr};
    p.child_min = V3{pos_bt.x - extent, pos_bt.y - extent, pos_bt.z - extent};
    p.child_max = V3{pos_bt.x + extent, pos_bt.y + extent, pos_bt.z + extent};
    p.child_center = pos_bt;
    p.child_half = V3{extent, extent, extent};
    p.valid = 1;
    p.is_ball = 1;
}
// A car: its box (half extents with margin `half_bt`, centre `child_bt` in body space) now and at the pose this
// tick's velocities predict (`pred_*` basis columns).
RG_HDI void car_proxy(BpProxy& p, V3 origin, V3 ax, V3 ay, V3 az, V3 pred_ax, V3 pred_ay, V3 pred_az,
                      V3 predict_vel_bt, V3 child_bt, V3 half_bt, float dt) {
    constexpr float kThr = 0.02f;
    const V3 pred_origin = origin + predict_vel_bt * dt;
    auto center = [](V3 o, V3 x, V3 y, V3 z, V3 l) {
        return V3{(x.x * l.x + y.x * l.y) + z.x * l.z + o.x, (x.y * l.x + y.y * l.y) + z.y * l.z + o.y,
                  (x.z * l.x + y.z * l.y) + z.z * l.z + o.z};
    };
    auto extent = [](V3 x, V3 y, V3 z, V3 h) {
        return V3{fabs_(x.x) * h.x + fabs_(y.x) * h.y + fabs_(z.x) * h.z,
                  fabs_(x.y) * h.x + fabs_(y.y) * h.y + fabs_(z.y) * h.z,
                  fabs_(x.z) * h.x + fabs_(y.z) * h.y + fabs_(z.z) * h.z};
    };
    const V3 cn = center(origin, ax, ay, az, child_bt);
    const V3 en = extent(ax, ay, az, half_bt);
    p.child_min = cn - en;
    p.child_max = cn + en;
    const V3 lmin = child_bt - half_bt, lmax = child_bt + half_bt;
    const V3 lc = (lmax + lmin) * 0.5f, lh = (lmax - lmin) * 0.5f;
    const V3 on = center(origin, ax, ay, az, lc);
    const V3 op = center(pred_origin, pred_ax, pred_ay, pred_az, lc);
    const V3 eon = extent(ax, ay, az, lh);
    const V3 eop = extent(pred_ax, pred_ay, pred_az, lh);
    p.aabb_min = V3{fmin_(on.x - eon.x, op.x - eop.x) - kThr, fmin_(on.y - eon.y, op.y - eop.y) - kThr,
                    fmin_(on.z - eon.z, op.z - eop.z) - kThr};
    p.aabb_max = V3{fmax_(on.x + eon.x, op.x + eop.x) + kThr, fmax_(on.y + eon.y, op.y + eop.y) + kThr,
                    fmax_(on.z + eon.z, op.z + eop.z) + kThr};
    p.child_center = cn;
    p.axis[0] = ax;
    p.axis[1] = ay;
    p.axis[2] = az;
    p.child_half = half_bt;
    p.local_min = lmin;
    p.local_max = lmax;
    p.origin = origin;
    p.valid = 1;
    p.is_ball = 0;
}

// ---- the sweep -----------------------------------------------------------------------------------------------------
struct Sweep {
    Broadphase& h;
    int body_count;
    RG_HD int find(const uint32_t* list, int n, uint32_t key) const {
        for (int i = 0; i < n; ++i)
            if (list[i] == key) return i;
        return -1;
    }
    RG_HD static void swap_remove(uint32_t* list, uint8_t& n, int i) {
        if (i >= 0) list[i] = list[--n];
    }
    // The pair key of two handles, false when the pair is not between a body and something else.
    RG_HD bool pair_key(int ha, int hb, uint32_t& key) const {
        if (ha > hb) {
            const int t = ha;
            ha = hb;
            hb = t;
        }
        if (h.static_id[hb] >= 0) return false;
        int body_b = -1 - h.static_id[hb];
        if (body_b < 0 || body_b >= body_count) return false;
        if (h.static_id[ha] >= 0) {
            key = bp_key(body_b == 0 ? 0 : 2, body_b - 1, -1, h.static_id[ha]);
        } else {
            int body_a = -1 - h.static_id[ha];
            if (body_a > body_b) {
                const int t = body_a;
                body_a = body_b;
                body_b = t;
            }
            key = bp_key(body_a == 0 ? 1 : 3, body_a == 0 ? body_b - 1 : body_a - 1, body_a == 0 ? -1 : body_b - 1,
                         -1);
        }
        return true;
    }
    RG_HD void add_pair(int ha, int hb) {
        uint32_t key = 0;
        if (pair_key(ha, hb, key) && find(h.pairs, h.pair_count, key) < 0 && h.pair_count < kBpMaxEntries)
            h.pairs[h.pair_count++] = key;
    }
    RG_HD void remove_pair(int ha, int hb) {
        uint32_t key = 0;
        if (!pair_key(ha, hb, key)) return;
        const int at = find(h.pairs, h.pair_count, key);
        if (at >= 0) {
            swap_remove(h.pairs, h.pair_count, at);
            swap_remove(h.manifolds, h.manifold_count, find(h.manifolds, h.manifold_count, key));
        }
    }
    // Edge-index overlap of two handles on the two axes other than `axis`.
    RG_HD bool overlap_2d(int a, int b, int axis) const {
        const int a1 = (1 << axis) & 3;
        const int a2 = (1 << a1) & 3;
        return !(h.max_edge[a][a1] < h.min_edge[b][a1] || h.max_edge[b][a1] < h.min_edge[a][a1] ||
                 h.max_edge[a][a2] < h.min_edge[b][a2] || h.max_edge[b][a2] < h.min_edge[a][a2]);
    }
    RG_HD uint8_t& edge_ref(int handle, int axis, bool is_max) {
        return is_max ? h.max_edge[handle][axis] : h.min_edge[handle][axis];
    }
    RG_HDI void sort_down(int axis, int index, bool is_max, bool update) {
        const uint8_t owner = h.edge_handle[axis][index];
        const uint16_t pos = h.edge_pos[axis][index];
        const int start = index;
        while (index > 0 && pos < h.edge_pos[axis][index - 1]) {
            const uint8_t prev = h.edge_handle[axis][index - 1];
            const uint16_t prev_pos = h.edge_pos[axis][index - 1];
            const bool prev_max = (prev_pos & 1) != 0;
            if (update && prev_max != is_max && overlap_2d(owner, prev, axis)) {
                if (is_max)
                    remove_pair(owner, prev);
                else
                    add_pair(owner, prev);
            }
            ++edge_ref(prev, axis, prev_max);
            --edge_ref(owner, axis, is_max);
            h.edge_pos[axis][index] = prev_pos;
            h.edge_handle[axis][index] = prev;
            --index;
        }
        if (index != start) {
            h.edge_pos[axis][index] = pos;
            h.edge_handle[axis][index] = owner;
        }
    }
    RG_HDI void sort_up(int axis, int index, bool is_max, bool update) {
        const uint8_t owner = h.edge_handle[axis][index];
        const uint16_t pos = h.edge_pos[axis][index];
        const int start = index;
        const int n = 2 * h.handle_count + 2;
        while (index + 1 < n && h.edge_handle[axis][index + 1] != 0 && pos >= h.edge_pos[axis][index + 1]) {
            const uint8_t next = h.edge_handle[axis][index + 1];
            const uint16_t next_pos = h.edge_pos[axis][index + 1];
            const bool next_max = (next_pos & 1) != 0;
            if (update && next_max != is_max && overlap_2d(owner, next, axis)) {
                if (is_max)
                    add_pair(owner, next);
                else
                    remove_pair(owner, next);
            }
            --edge_ref(next, axis, next_max);
            ++edge_ref(owner, axis, is_max);
            h.edge_pos[axis][index] = next_pos;
            h.edge_handle[axis][index] = next;
            ++index;
        }
        if (index != start) {
            h.edge_pos[axis][index] = pos;
            h.edge_handle[axis][index] = owner;
        }
    }
    // A new handle's two edges enter just below the top sentinel and sort down; pairs are made on the last axis.
    RG_HDI void add_handle(V3 mn, V3 mx, int16_t id, bool update_pairs) {
        const float lo[3] = {mn.x, mn.y, mn.z}, hi[3] = {mx.x, mx.y, mx.z};
        const int handle = h.free_count > 0 ? h.free_[--h.free_count] : h.next_fresh++;
        const int limit = 2 * ++h.handle_count;
        h.static_id[handle] = id;
        for (int axis = 0; axis < 3; ++axis) {
            h.max_edge[0][axis] = static_cast<uint8_t>(h.max_edge[0][axis] + 2);
            h.edge_pos[axis][limit + 1] = h.edge_pos[axis][limit - 1];
            h.edge_handle[axis][limit + 1] = h.edge_handle[axis][limit - 1];
            h.edge_pos[axis][limit - 1] = sweep_quantize(lo[axis], 0);
            h.edge_handle[axis][limit - 1] = static_cast<uint8_t>(handle);
            h.edge_pos[axis][limit] = sweep_quantize(hi[axis], 1);
            h.edge_handle[axis][limit] = static_cast<uint8_t>(handle);
            h.min_edge[handle][axis] = static_cast<uint8_t>(limit - 1);
            h.max_edge[handle][axis] = static_cast<uint8_t>(limit);
        }
        for (int axis = 0; axis < 3; ++axis) {
            sort_down(axis, h.min_edge[handle][axis], false, update_pairs && axis == 2);
            sort_down(axis, h.max_edge[handle][axis], true, update_pairs && axis == 2);
        }
    }
    // The static handles of a fresh sweep: the arena mesh (reference BulletSweepAddStatics with planes off).
    RG_HDI void add_statics(V3 mesh_min, V3 mesh_max) {
        h.next_fresh = 1;
        h.free_count = 0;
        h.handle_count = 0;
        for (int axis = 0; axis < 3; ++axis) {
            h.edge_pos[axis][0] = 0;
            h.edge_handle[axis][0] = 0;
            h.edge_pos[axis][1] = 0xffff;
            h.edge_handle[axis][1] = 0;
            h.min_edge[0][axis] = 0;
            h.max_edge[0][axis] = 1;
        }
        add_handle(mesh_min, mesh_max, 0, false);
        h.static_count = h.handle_count;
    }
    static RG_HD bool key_has_body(uint32_t key, int body) {
        const int kind = bp_kind(key);
        const int a = static_cast<int>((key >> 2) & 15u), b = static_cast<int>((key >> 6) & 15u);
        if (kind == 0) return body == 0;
        if (kind == 1) return body == 0 || body == a;
        return body == a || (kind == 3 && body == b);
    }
    // reference BulletSweepRemoveBody
    RG_HDI void remove_body(int body) {
        const int handle = h.body_handle[body];
        if (handle == 0) return;
        for (int i = 0; i < h.pair_count; ++i) {
            const uint32_t key = h.pairs[i];
            if (!key_has_body(key, body)) continue;
            for (int m = 0; m < h.manifold_count; ++m) {
                if (h.manifolds[m] == key) {
                    h.manifolds[m] = h.manifolds[--h.manifold_count];
                    break;
                }
            }
        }
        for (int i = 0; i < h.pair_count;) {
            if (key_has_body(h.pairs[i], body))
                h.pairs[i] = h.pairs[--h.pair_count];
            else
                ++i;
        }
        const int limit = 2 * h.handle_count;
        for (int axis = 0; axis < 3; ++axis) h.max_edge[0][axis] = static_cast<uint8_t>(h.max_edge[0][axis] - 2);
        for (int axis = 0; axis < 3; ++axis) {
            for (int is_max = 1; is_max >= 0; --is_max) {
                int index = is_max ? h.max_edge[handle][axis] : h.min_edge[handle][axis];
                h.edge_pos[axis][index] = 0xffff;
                while (h.edge_handle[axis][index + 1] != 0 && h.edge_pos[axis][index] >= h.edge_pos[axis][index + 1]) {
                    const int next = h.edge_handle[axis][index + 1];
                    const bool next_max = (h.edge_pos[axis][index + 1] & 1) != 0;
                    --edge_ref(next, axis, next_max);
                    ++edge_ref(handle, axis, is_max != 0);
                    const uint16_t pos = h.edge_pos[axis][index];
                    h.edge_pos[axis][index] = h.edge_pos[axis][index + 1];
                    h.edge_handle[axis][index] = h.edge_handle[axis][index + 1];
                    h.edge_pos[axis][index + 1] = pos;
                    h.edge_handle[axis][index + 1] = static_cast<uint8_t>(handle);
                    ++index;
                }
            }
            h.edge_handle[axis][limit - 1] = 0;
            h.edge_pos[axis][limit - 1] = 0xffff;
        }
        h.free_[h.free_count++] = static_cast<uint8_t>(handle);
        h.handle_count = static_cast<uint8_t>(h.handle_count - 1);
        h.body_handle[body] = 0;
        h.body_aabb_valid = static_cast<uint16_t>(h.body_aabb_valid & ~(1u << body));
        for (int i = 0; i < h.obj_count; ++i) {
            if (h.obj[i] == body) {
                h.obj[i] = h.obj[--h.obj_count];
                break;
            }
        }
    }
    // Bodies of a fresh sweep enter together: their edges are merged into the static edges, then each pair with a
    // static or an earlier body is found by scanning the last axis (reference add_bodies_merged).
    RG_HDI void add_bodies_merged(const BpProxy* proxies) {
        uint8_t new_handle[kBpBodies], new_body[kBpBodies];
        uint16_t q[kBpBodies][2][3];
        const int old_count = 2 * h.handle_count + 2;
        int n = 0;
        for (int body = 0; body < body_count; ++body) {
            const BpProxy& p = proxies[body];
            if (!p.valid) continue;
            const int handle = h.free_count > 0 ? h.free_[--h.free_count] : h.next_fresh++;
            ++h.handle_count;
            h.body_handle[body] = static_cast<uint8_t>(handle);
            h.static_id[handle] = static_cast<int16_t>(-1 - body);
            h.obj[h.obj_count++] = static_cast<uint8_t>(body);
            const float lo[3] = {p.child_min.x, p.child_min.y, p.child_min.z};
            const float hi[3] = {p.child_max.x, p.child_max.y, p.child_max.z};
            for (int a = 0; a < 3; ++a) {
                q[n][0][a] = sweep_quantize(lo[a], 0);
                q[n][1][a] = sweep_quantize(hi[a], 1);
            }
            new_handle[n] = static_cast<uint8_t>(handle);
            new_body[n++] = static_cast<uint8_t>(body);
        }
        const int new_count = 2 * n;
        for (int axis = 0; axis < 3; ++axis) {
            uint32_t key[2 * kBpBodies];
            for (int e = 0; e < new_count; ++e) {
                const uint32_t v = (static_cast<uint32_t>(q[e >> 1][e & 1][axis]) << 5) | static_cast<uint32_t>(e);
                int j = e;
                for (; j > 0 && key[j - 1] < v; --j) key[j] = key[j - 1];
                key[j] = v;
            }
            // merge from the top: the old edges stay where they are below the last new edge
            uint16_t old_pos[kBpEdges];
            uint8_t old_handle[kBpEdges];
            for (int e = 0; e < old_count; ++e) {
                old_pos[e] = h.edge_pos[axis][e];
                old_handle[e] = h.edge_handle[axis][e];
            }
            int old = old_count - 1;
            int dst = old_count + new_count - 1;
            h.edge_pos[axis][dst] = old_pos[old];
            h.edge_handle[axis][dst] = old_handle[old];
            h.max_edge[old_handle[old]][axis] = static_cast<uint8_t>(dst);
            --old;
            --dst;
            for (int e = 0; e < new_count; --dst) {
                uint16_t pos = old_pos[old];
                uint8_t handle;
                if (pos > static_cast<uint16_t>(key[e] >> 5)) {
                    handle = old_handle[old--];
                } else {
                    pos = static_cast<uint16_t>(key[e] >> 5);
                    handle = new_handle[(key[e++] & 31u) >> 1];
                }
                h.edge_pos[axis][dst] = pos;
                h.edge_handle[axis][dst] = handle;
                edge_ref(handle, axis, (pos & 1) != 0) = static_cast<uint8_t>(dst);
            }
        }
        const int top = old_count + new_count - 2;
        for (int k = 0; k < n; ++k) {
            const int moving = new_handle[k];
            const int min_id = -1 - new_body[k];
            const uint8_t m0 = h.min_edge[moving][0], m1 = h.min_edge[moving][1];
            const uint8_t x0 = h.max_edge[moving][0], x1 = h.max_edge[moving][1];
            for (int is_max = 0; is_max < 2; ++is_max) {
                const uint16_t pos = q[k][is_max][2];
                for (int i = top; i >= 0; --i) {
                    const uint16_t p = h.edge_pos[2][i];
                    if (!(p > pos)) break;
                    const int o = h.edge_handle[2][i];
                    if ((p & 1) != is_max && h.static_id[o] > min_id &&
                        !(x0 < h.min_edge[o][0] || h.max_edge[o][0] < m0 || x1 < h.min_edge[o][1] ||
                          h.max_edge[o][1] < m1)) {
                        if (is_max)
                            remove_pair(moving, o);
                        else
                            add_pair(moving, o);
                    }
                }
            }
        }
    }
    RG_HDI void add_body(int body, const BpProxy& p) {
        if (p.valid && h.body_handle[body] == 0 && h.handle_count < kBpHandles - 1) {
            h.body_handle[body] = h.free_count > 0 ? h.free_[h.free_count - 1] : h.next_fresh;
            add_handle(p.child_min, p.child_max, static_cast<int16_t>(-1 - body), true);
            h.obj[h.obj_count++] = static_cast<uint8_t>(body);
        }
    }
    // Each body's swept AABB moves its edges; crossings update the pairs (reference update_aabbs).
    RG_HDI void update_aabbs(const BpProxy* proxies) {
        for (int o = 0; o < h.obj_count; ++o) {
            const int body = h.obj[o];
            if (body >= body_count) continue;
            const BpProxy& p = proxies[body];
            const int handle = h.body_handle[body];
            if (!p.valid || handle == 0) continue;
            const float lo[3] = {p.aabb_min.x, p.aabb_min.y, p.aabb_min.z};
            const float hi[3] = {p.aabb_max.x, p.aabb_max.y, p.aabb_max.z};
            for (int a = 0; a < 3; ++a) {
                h.body_aabb[body][a] = lo[a];
                h.body_aabb[body][a + 3] = hi[a];
            }
            h.body_aabb_valid = static_cast<uint16_t>(h.body_aabb_valid | (1u << body));
            for (int axis = 0; axis < 3; ++axis) {
                const uint16_t qmin = sweep_quantize(lo[axis], 0), qmax = sweep_quantize(hi[axis], 1);
                const int emin = h.min_edge[handle][axis], emax = h.max_edge[handle][axis];
                const int dmin = static_cast<int>(qmin) - static_cast<int>(h.edge_pos[axis][emin]);
                const int dmax = static_cast<int>(qmax) - static_cast<int>(h.edge_pos[axis][emax]);
                if (dmin == 0 && dmax == 0) continue;
                if (dmin != 0) h.edge_pos[axis][emin] = qmin;
                if (dmax != 0) h.edge_pos[axis][emax] = qmax;
                if (dmin < 0) sort_down(axis, emin, false, true);
                if (dmax > 0) sort_up(axis, emax, true, true);
                if (dmin > 0) sort_up(axis, emin, false, true);
                if (dmax < 0) sort_down(axis, emax, true, true);
            }
        }
    }
};

// Kickoff reset: demolished cars leave, then the ball and every car leave the sweep (reference BulletSweepNewRound /
// BulletSweepRemoveRoundBodies).
RG_HDI void bp_new_round(Broadphase& h, int car_count, const uint8_t* car_demoed) {
    if (h.handle_count == 0) return;
    const int n = car_count < kBpBodies - 1 ? car_count : kBpBodies - 1;
    Sweep s{h, kBpBodies};
    for (int slot = 0; slot < n; ++slot)
        if (car_demoed[slot]) s.remove_body(slot + 1);
    s.remove_body(0);
    for (int slot = 0; slot < n; ++slot) s.remove_body(slot + 1);
}

// One manifold-list entry after the island sort.
struct BpEntry {
    uint32_t key;
    int32_t island;
};

// The tick's manifold list (reference BuildBulletManifoldList<0> then SortBulletManifoldListByIsland). `mesh_min`,
// `mesh_max`: the arena mesh's bounds (Bullet units); `pred_mask`: bodies with a predictive contact this tick;
// `ball_static_skipped`: the ball sleeps, so its static pairs make no new manifold. Fills `out` (sorted) and returns
// its length.
RG_NOINL int bp_build_manifold_list(Broadphase& h, const BpProxy* proxies, int body_count, V3 mesh_min, V3 mesh_max,
                                  uint32_t pred_mask, bool ball_static_skipped, BpEntry* out) {
    Sweep s{h, body_count};
    const bool fresh = h.handle_count == 0;
    if (fresh) s.add_statics(mesh_min, mesh_max);
    for (int body = 1; body < body_count; ++body)
        if (!proxies[body].valid && h.body_handle[body] != 0) s.remove_body(body);
    bool round_cached = false;
    if (fresh) {
        bool empty = h.pair_count == 0 && h.manifold_count == 0 && h.obj_count == 0;
        for (int body = 0; empty && body < body_count; ++body) empty = h.body_handle[body] == 0;
        round_cached = !empty;
    }
    if (fresh && !round_cached) {
        s.add_bodies_merged(proxies);
    } else {
        for (int body = 0; body < body_count; ++body) s.add_body(body, proxies[body]);
    }
    if (round_cached) {
        s.remove_body(0);
        for (int slot = 0; slot < body_count - 1; ++slot) s.remove_body(slot + 1);
        for (int body = 0; body < body_count; ++body) s.add_body(body, proxies[body]);
    }
    // last tick's predictive manifolds leave; this tick's are appended in sweep-object order
    for (int i = 0; i < h.predictive_count; ++i)
        Sweep::swap_remove(h.manifolds, h.manifold_count, s.find(h.manifolds, h.manifold_count, h.predictive[i]));
    h.predictive_count = 0;
    for (int o = 0; o < h.obj_count && pred_mask != 0u; ++o) {
        const int body = h.obj[o];
        if (body >= body_count || ((pred_mask >> body) & 1u) == 0u || h.manifold_count >= kBpMaxEntries) continue;
        const uint32_t key = bp_key(body == 0 ? 0 : 2, body - 1, -1, kBpPredictiveId);
        h.manifolds[h.manifold_count++] = key;
        h.predictive[h.predictive_count++] = key;
    }
    s.update_aabbs(proxies);
    // pairs -> manifolds
    auto proxy_of = [&](int body) -> const BpProxy* {
        return body >= 0 && body < body_count && proxies[body].valid ? &proxies[body] : nullptr;
    };
    for (int i = 0; i < h.pair_count; ++i) {
        const uint32_t key = h.pairs[i];
        const int kind = bp_kind(key);
        const int at = s.find(h.manifolds, h.manifold_count, key);
        bool want;
        const BpProxy* pa = proxy_of(kind <= 1 ? 0 : bp_body_a(key) + 1);
        if (kind == 0) {
            want = proxy_of(0) != nullptr;
        } else if (pa == nullptr) {
            want = false;
        } else if (kind == 1 || kind == 3) {
            const BpProxy* pb = proxy_of(kind == 1 ? bp_body_a(key) + 1 : bp_body_b(key) + 1);
            want = pb != nullptr && aabb_overlap(pa->child_min, pa->child_max, pb->child_min, pb->child_max);
        } else {
            want = aabb_overlap(pa->child_min, pa->child_max, mesh_min, mesh_max);
        }
        if (want && at < 0 && (kind == 1 || kind == 3)) {
            // a new car/ball or car/car manifold needs the boxes to overlap on the first body's axes
            int a = bp_body_a(key) + 1;
            int b = kind == 1 ? 0 : bp_body_b(key) + 1;
            if (kind == 3 && h.body_handle[b] < h.body_handle[a]) {
                const int t = a;
                a = b;
                b = t;
            }
            const BpProxy* qa = proxy_of(a);
            const BpProxy* qb = proxy_of(b);
            bool local = qa != nullptr && qb != nullptr;
            if (local) {
                const V3 d = qb->child_center - qa->child_center;
                const float ha[3] = {qa->child_half.x, qa->child_half.y, qa->child_half.z};
                const float hb[3] = {qb->child_half.x, qb->child_half.y, qb->child_half.z};
                for (int k = 0; k < 3 && local; ++k) {
                    const V3 ak = qa->axis[k];
                    float e = hb[k];
                    if (!qb->is_ball)
                        e = fabs_(dot(ak, qb->axis[0])) * hb[0] + fabs_(dot(ak, qb->axis[1])) * hb[1] +
                            fabs_(dot(ak, qb->axis[2])) * hb[2];
                    if (fabs_(dot(d, ak)) > ha[k] + e) local = false;
                }
            }
            if (!local) continue;
        }
        if (want && at < 0 && kind == 2 && bp_static(key) < 100) {
            // compound child test: the mesh bounds in the car's frame against the child box
            const V3* r = pa->axis;
            const V3 no{-pa->origin.x, -pa->origin.y, -pa->origin.z};
            const V3 c = (mesh_max + mesh_min) * 0.5f;
            const V3 hh = (mesh_max - mesh_min) * 0.5f;
            const float lo[3] = {pa->local_min.x, pa->local_min.y, pa->local_min.z};
            const float hi[3] = {pa->local_max.x, pa->local_max.y, pa->local_max.z};
            bool tree = true;
            for (int k = 0; k < 3 && tree; ++k) {
                const float io = (r[k].x * no.x + r[k].y * no.y) + r[k].z * no.z;
                const float ctr = (r[k].x * c.x + r[k].y * c.y) + r[k].z * c.z + io;
                const float ext = (hh.x * fabs_(r[k].x) + hh.y * fabs_(r[k].y)) + hh.z * fabs_(r[k].z);
                if (!(ctr - ext <= hi[k] && ctr + ext >= lo[k])) tree = false;
            }
            if (!tree) continue;
        }
        if (want && at < 0 && kind == 0 && ball_static_skipped) continue;
        if (want && at < 0) {
            h.manifolds[h.manifold_count++] = key;
        } else if (!want) {
            Sweep::swap_remove(h.manifolds, h.manifold_count, at);
        }
    }
    // islands: bodies joined through ball/car and car/car pairs; ids are sweep-object positions
    int tag[kBpBodies];
    for (int b = 0; b < kBpBodies; ++b) tag[b] = -1;
    for (int o = 0; o < h.obj_count; ++o) tag[h.obj[o]] = o;
    int parent[kBpBodies];
    bool joined = false;
    auto root = [&](int i) {
        while (parent[i] != i) i = parent[i];
        return i;
    };
    for (int i = 0; i < h.pair_count; ++i) {
        const uint32_t key = h.pairs[i];
        const int kind = bp_kind(key);
        if (kind != 1 && kind != 3) continue;
        int b0 = kind == 1 ? 0 : bp_body_a(key) + 1;
        int b1 = kind == 1 ? bp_body_a(key) + 1 : bp_body_b(key) + 1;
        if (h.body_handle[b0] > h.body_handle[b1]) {
            const int t = b0;
            b0 = b1;
            b1 = t;
        }
        if (tag[b0] < 0 || tag[b1] < 0) continue;
        if (!joined) {
            for (int k = 0; k < kBpBodies; ++k) parent[k] = k;
            joined = true;
        }
        const int ra = root(tag[b0]), rb = root(tag[b1]);
        if (ra != rb) parent[ra] = rb;
    }
    int island_of[kBpBodies];
    for (int b = 0; b < kBpBodies; ++b) island_of[b] = joined && tag[b] >= 0 ? root(tag[b]) : tag[b];
    const int n = h.manifold_count < kBpMaxEntries ? h.manifold_count : kBpMaxEntries;
    int8_t ids[kBpMaxEntries];
    for (int i = 0; i < n; ++i) {
        out[i].key = h.manifolds[i];
        out[i].island = island_of[bp_entry_body(h.manifolds[i])];
        ids[i] = static_cast<int8_t>(out[i].island);
    }
    if (n == 2) {
        if (ids[1] <= ids[0]) {
            const BpEntry t = out[0];
            out[0] = out[1];
            out[1] = t;
        }
    } else if (n > 2) {
        // Bullet's quicksort of the manifolds by island id (btAlignedObjectArray::quickSortInternal)
        int8_t order[kBpMaxEntries];
        for (int i = 0; i < n; ++i) order[i] = static_cast<int8_t>(i);
        int8_t range_lo[32], range_hi[32];
        int depth = 0;
        range_lo[depth] = 0;
        range_hi[depth] = static_cast<int8_t>(n - 1);
        ++depth;
        while (depth > 0) {
            --depth;
            int i = range_lo[depth], j = range_hi[depth];
            const int lo = i, hi = j;
            const int pivot = ids[order[(lo + hi) / 2]];
            do {
                while (ids[order[i]] < pivot) ++i;
                while (pivot < ids[order[j]]) --j;
                if (i <= j) {
                    const int8_t t = order[i];
                    order[i] = order[j];
                    order[j] = t;
                    ++i;
                    --j;
                }
            } while (i <= j);
            const bool right_first = hi - i < j - lo;
            for (int side = 0; side < 2; ++side) {
                const bool right = (side == 0) != right_first;
                const int a = right ? i : lo, b = right ? hi : j;
                if (a < b && depth < 32) {
                    range_lo[depth] = static_cast<int8_t>(a);
                    range_hi[depth] = static_cast<int8_t>(b);
                    ++depth;
                }
            }
        }
        BpEntry sorted[kBpMaxEntries];
        for (int i = 0; i < n; ++i) sorted[i] = out[order[i]];
        for (int i = 0; i < n; ++i) out[i] = sorted[i];
    }
    return n;
}

}  // namespace rg
