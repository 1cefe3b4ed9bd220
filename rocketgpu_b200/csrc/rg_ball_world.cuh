// Ball vs arena mesh: query, narrowphase, persistent manifold, contact rows and the ball's PGS solves (host+device).
//
// Reference behaviour reproduced (custom-mesh soccar arena, one mesh group, ball rotation off):
//   * AppendBallWorldSpecialContactRows, include/rocketgpu/detail/step/arena_ball.hpp:1868-2466 (mesh branch);
//   * BallMeshTriangleHit :1389-1462, DetectBallMeshTriangleContactEx arena_geometry.hpp:1913-1998;
//   * MaybeAdjustArenaTriangleInternalEdgeContactT raycast_wheels_and_contact_prep.hpp:5044-5170 (game edge rules);
//   * the 4-point manifold: Insert/Sort/Remove/Refresh, arena_ball.hpp:1137-1297;
//   * rows: InitializeBallSplitContactRow arena_geometry.hpp:6588-6715, InitializeBallVelocityContactRow :2013-2140,
//     InitializeBallFrictionContactRow :2141-2271, AppendBallVelocityContactRows :2272-2403;
//   * solves: SolveUnifiedVelocityContactRowsGeneral :5527-5867 (ball rows in Bullet units, at most 10 iterations,
//     stopping early when no impulse changed) and SolveUnifiedSplitContactRows :5035-5279 (split-impulse position
//     push, Bullet-unit accumulators).
// Triangles are visited in the BVH's leaf order (rank order of rg_mesh), which is the order the reference inserts
// manifold points in.
#pragma once

#include "rg_math.cuh"
#include "rg_mesh.h"
#include "rg_state.cuh"
#include "rg_ucrt.cuh"

namespace rg {

constexpr float kSimdEpsilon = 1.1920928955078125e-7f;
constexpr float kPiF = 3.14159274f;

struct BallManifoldPt {
    V3 normal;
    float pen_uu;
    V3 local_a;
    V3 local_b;
    int32_t tri;
    float rel_len;
    V3 rel_pos1;
    float distance;
};

// Per-arena state kept between ticks: the ball's persistent contact manifold with the arena mesh, and the world's
// persistent manifold list as far as the ball-only world has entries in it: the ball/mesh pair and the ball's
// predictive contact, in list order (kListMesh / kListPredictive). The reference keeps that list in its broadphase
// history (BuildBulletManifoldList, arena_geometry.hpp:4862-4905) and its order decides the solver's row order.
constexpr uint8_t kListMesh = 1, kListPredictive = 2;
struct BallWorldScratch {
    BallManifoldPt pts[4];
    int32_t count;
    uint8_t list[2];
    uint8_t list_count;
    uint8_t pad0;
    int32_t pad[2];
};

RG_HDI void ball_basis(const BallState& b, V3& x, V3& y, V3& z) {
    if (b.basis_authoritative) {
        x = b.basis_forward;
        y = b.basis_right;
        z = b.basis_up;
        return;
    }
    upload_basis_from_rot(b.rot, x, y, z);
}

// --- narrowphase ---------------------------------------------------------------------------------------------------
RG_HDI bool point_in_triangle(V3 p, V3 a, V3 b, V3 c, V3 n) {
    const float r1 = dot(cross(b - a, n), p - a);
    const float r2 = dot(cross(c - b, n), p - b);
    const float r3 = dot(cross(a - c, n), p - c);
    return (r1 > 0.0f && r2 > 0.0f && r3 > 0.0f) || (r1 <= 0.0f && r2 <= 0.0f && r3 <= 0.0f);
}

RG_HDI bool nearest_edge_point(V3 p, V3 a, V3 b, V3 c, float max_dist_sq, V3& out) {
    const V3 from[3] = {a, b, c};
    const V3 to[3] = {b, c, a};
    bool found = false;
    for (int i = 0; i < 3; ++i) {
        V3 diff = p - from[i];
        const V3 v = to[i] - from[i];
        float t = dot(v, diff);
        if (t > 0.0f) {
            const float vv = dot(v, v);
            if (t < vv) {
                t /= vv;
                diff = diff - v * t;
            } else {
                t = 1.0f;
                diff = diff - v;
            }
        } else {
            t = 0.0f;
        }
        const float d2 = dot(diff, diff);
        if (d2 < max_dist_sq) {
            max_dist_sq = d2;
            out = from[i] + v * t;
            found = true;
        }
    }
    return found;
}

// Sphere vs triangle (Bullet SphereTriangleDetector with back faces rejected, as the game's ball does).
RG_HDI bool sphere_triangle(V3 center, float radius, float threshold, V3 ta, V3 tb, V3 tc, V3& out_normal,
                            float& out_pen_uu, V3& out_on_tri, float& out_depth) {
    const float rwt = radius + threshold;
    V3 n = cross(tb - ta, tc - ta);
    const float l2 = dot(n, n);
    if (l2 < kSimdEpsilon * kSimdEpsilon) return false;
    n = n * (1.0f / sqrtf(l2));
    const V3 p1c = center - ta;
    const float dist = dot(p1c, n);
    if (dist < 0.0f) return false;
    if (dist >= rwt) return false;
    V3 cp{0, 0, 0};
    bool has = false;
    if (point_in_triangle(center, ta, tb, tc, n)) {
        has = true;
        cp = center - n * dist;
    } else {
        has = nearest_edge_point(center, ta, tb, tc, rwt * rwt, cp);
    }
    if (!has) return false;
    const V3 c2c = center - cp;
    const float d2 = dot(c2c, c2c);
    if (d2 >= rwt * rwt) return false;
    if (d2 > kSimdEpsilon) {
        const float d = sqrtf(d2);
        out_normal = c2c * (1.0f / d);
        out_pen_uu = (radius - d) * 50.0f;
        out_depth = -(radius - d);
    } else {
        out_normal = n;
        out_pen_uu = radius * 50.0f;
        out_depth = -radius;
    }
    out_on_tri = cp;
    return true;
}

// Rotation by a Bullet quaternion through its matrix (reference BulletMatrixRotate, math.hpp:929-938).
RG_HDI V3 quat_matrix_rotate(Q4 q, V3 v) {
    V3 c0, c1, c2;
    game_basis_from_rot(q, c0, c1, c2);
    return V3{c0.x * v.x + c1.x * v.y + c2.x * v.z, c0.y * v.x + c1.y * v.y + c2.y * v.z,
              c0.z * v.x + c1.z * v.y + c2.z * v.z};
}
RG_HDI Q4 quat_from_axis_angle(V3 axis, float angle) {
    const float d = len(axis);
    const float s = game_sinf(angle * 0.5f) / d;
    return Q4{game_cosf(angle * 0.5f), axis.x * s, axis.y * s, axis.z * s};
}
RG_HDI V3 quat_rotate_vec(Q4 q, V3 v) {
    const float rx = q.w * v.x + q.y * v.z - q.z * v.y;
    const float ry = q.w * v.y + q.z * v.x - q.x * v.z;
    const float rz = q.w * v.z + q.x * v.y - q.y * v.x;
    const float rw = -q.x * v.x - q.y * v.y - q.z * v.z;
    const float cx = -q.x, cy = -q.y, cz = -q.z, cw = q.w;
    return V3{rw * cx + rx * cw + ry * cz - rz * cy, rw * cy + ry * cw + rz * cx - rx * cz,
              rw * cz + rz * cw + rx * cy - ry * cx};
}

RG_HDI float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

RG_HDI V3 closest_on_segment(V3 p, V3 a, V3 b, float t_lo, float t_hi) {
    const V3 seg = b - a;
    const float l2 = dot(seg, seg);
    if (l2 <= 1.0e-12f) return a;
    const float t = clampf(dot(p - a, seg) / l2, t_lo, t_hi);
    return a + seg * t;
}

RG_HDI V3 normalize_or(V3 v, V3 fallback) {
    const float l2 = dot(v, v);
    if (l2 <= 1e-12f) return fallback;
    return v * (1.0f / sqrtf(l2));
}

RG_HDI bool clamp_edge_normal(V3 edge, V3 tri_normal, V3 contact_normal, float corrected, V3& out) {
    const V3 edge_cross = normalize_or(cross(edge, tri_normal), tri_normal);
    const float cur = ucrt_atan2f(dot(contact_normal, edge_cross), dot(contact_normal, tri_normal));
    if (corrected < 0.0f) {
        if (cur < corrected) {
            out = quat_matrix_rotate(quat_from_axis_angle(edge, corrected - cur), contact_normal);
            return true;
        }
    } else if (cur > corrected) {
        out = quat_matrix_rotate(quat_from_axis_angle(edge, corrected - cur), contact_normal);
        return true;
    }
    return false;
}

// Internal-edge correction of a triangle contact (Bullet btAdjustInternalEdgeContacts, reference
// MaybeAdjustArenaTriangleInternalEdgeContactT, raycast_wheels_and_contact_prep.hpp:5044-5170, with the game's edge
// rules: a soccar layout installs its local triangle copy, cal_arena_local_tris, src/rocketgpu.cpp:1152-1156, and that
// selects them for custom meshes too). Returns whether the contact was near an internal edge.
RG_HDI bool adjust_internal_edge(const DevTri& t, V3 point_on_a, float distance, V3& io_point_b, V3& io_normal) {
    constexpr float t_lo = 1.0e-5f, t_hi = 1.0f - 1.0e-5f;
    constexpr float kEdgeDistanceThreshold = 0.1f;
    constexpr float kMaxEdgeAngle = 2.0f * kPiF;
    const V3 tri_normal = t.normal;
    const float cl2 = dot(io_normal, io_normal);
    V3 contact_normal = tri_normal;
    if (cl2 > 1e-12f) contact_normal = io_normal * (1.0f / sqrtf(cl2));
    const V3 contact = io_point_b;
    const V3 es[3] = {t.a, t.b, t.c};
    const V3 ee[3] = {t.b, t.c, t.a};
    int best = -1;
    float best_d = 1.0e30f;
    uint32_t on_edge = 0u;
    for (int e = 0; e < 3; ++e) {
        if (fabs_(t.edge_angle[e]) >= kMaxEdgeAngle) continue;
        const V3 nearest = closest_on_segment(contact, es[e], ee[e], t_lo, t_hi);
        const float d = len(contact - nearest);
        if (d < 1.1920928955078125e-07f) on_edge |= 1u << e;
        if (d < best_d) {
            best_d = d;
            best = e;
        }
    }
    if (best < 0) return false;
    bool near_edge = false;
    int concave_hits = 0;
    const uint32_t convex_flag[3] = {kEdgeV0V1Convex, kEdgeV1V2Convex, kEdgeV2V0Convex};
    const uint32_t swap_flag[3] = {kEdgeV0V1Swap, kEdgeV1V2Swap, kEdgeV2V0Swap};
    for (int e = 0; e < 3; ++e) {
        if (best != e && (on_edge & (1u << e)) == 0u) continue;
        const float ang = t.edge_angle[e];
        if (fabs_(ang) >= kMaxEdgeAngle) continue;
        const V3 nearest = closest_on_segment(contact, es[e], ee[e], 0.0f, 1.0f);
        if (len(contact - nearest) >= kEdgeDistanceThreshold) continue;
        near_edge = true;
        if (ang == 0.0f) {
            ++concave_hits;
            continue;
        }
        const bool convex = (t.edge_flags & convex_flag[e]) != 0;
        const float swap = convex ? 1.0f : -1.0f;
        const V3 nA = tri_normal * swap;
        const V3 edge = es[e] - ee[e];
        V3 nb = quat_rotate_vec(quat_from_axis_angle(edge, ang), tri_normal);
        if ((t.edge_flags & swap_flag[e]) != 0) nb = -nb;
        const V3 nB = nb * swap;
        if (dot(contact_normal, nA) < 0.0f && dot(contact_normal, nB) < 0.0f) {
            ++concave_hits;
            continue;
        }
        V3 clamped{0.0f, 0.0f, 1.0f};
        const bool did = clamp_edge_normal(edge, tri_normal * swap, e == 0 ? contact_normal : io_normal, ang, clamped);
        if (did && dot(clamped, tri_normal) > 0.0f) {
            io_normal = clamped;
            io_point_b = point_on_a - io_normal * distance;
        }
    }
    if (!near_edge) return false;
    if (concave_hits > 0) {
        if (dot(tri_normal, contact_normal) < 0.0f) return false;
        io_normal = tri_normal;
        io_point_b = point_on_a - io_normal * distance;
    }
    return true;
}

// --- manifold ------------------------------------------------------------------------------------------------------
RG_HDI int manifold_replace_index(const BallManifoldPt* c, const BallManifoldPt& p) {
    int max_i = -1;
    float max_pen = p.pen_uu;
    for (int i = 0; i < 4; ++i) {
        if (c[i].pen_uu > max_pen) {
            max_i = i;
            max_pen = c[i].pen_uu;
        }
    }
    float r0 = 0.0f, r1 = 0.0f, r2 = 0.0f, r3 = 0.0f;
    if (max_i != 0) {
        const V3 x = cross(p.local_a - c[1].local_a, c[3].local_a - c[2].local_a);
        r0 = dot(x, x);
    }
    if (max_i != 1) {
        const V3 x = cross(p.local_a - c[0].local_a, c[3].local_a - c[2].local_a);
        r1 = dot(x, x);
    }
    if (max_i != 2) {
        const V3 x = cross(p.local_a - c[0].local_a, c[3].local_a - c[1].local_a);
        r2 = dot(x, x);
    }
    if (max_i != 3) {
        const V3 x = cross(p.local_a - c[0].local_a, c[2].local_a - c[1].local_a);
        r3 = dot(x, x);
    }
    int big = 0;
    float best = r0;
    if (r1 > best) { best = r1; big = 1; }
    if (r2 > best) { best = r2; big = 2; }
    if (r3 > best) { best = r3; big = 3; }
    return big;
}

RG_HDI void manifold_insert(BallManifoldPt* c, int& count, const BallManifoldPt& p, float merge) {
    float shortest = merge * merge;
    int nearest = -1;
    for (int i = 0; i < count; ++i) {
        const V3 d = c[i].local_a - p.local_a;
        const float dd = dot(d, d);
        if (dd < shortest) {
            shortest = dd;
            nearest = i;
        }
    }
    if (nearest >= 0) {
        c[nearest] = p;
        return;
    }
    int at = count;
    if (at == 4) {
        at = manifold_replace_index(c, p);
    } else {
        ++count;
    }
    c[at] = p;
}

RG_HDI BallManifoldPt manifold_empty_point() {
    BallManifoldPt z;
    z.normal = V3{0.0f, 0.0f, 1.0f};
    z.pen_uu = 0.0f;
    z.local_a = V3{0, 0, 0};
    z.local_b = V3{0, 0, 0};
    z.tri = -1;
    z.rel_len = 0.0f;
    z.rel_pos1 = V3{0, 0, 0};
    z.distance = 0.0f;
    return z;
}

// Re-evaluates every retained point at the ball's new pose; drops those beyond the breaking threshold, along the
// normal or sideways (swap-remove, as the reference does for retained ball-mesh points).
RG_HDI void manifold_refresh(BallManifoldPt* c, int& count, V3 center, const BallState& b, float threshold) {
    V3 bx, by, bz;
    ball_basis(b, bx, by, bz);
    for (int i = count - 1; i >= 0; --i) {
        BallManifoldPt& m = c[i];
        const V3 rot_a{bx.x * m.local_a.x + by.x * m.local_a.y + bz.x * m.local_a.z,
                       bx.y * m.local_a.x + by.y * m.local_a.y + bz.y * m.local_a.z,
                       bx.z * m.local_a.x + by.z * m.local_a.y + bz.z * m.local_a.z};
        const V3 wa = rot_a + center;
        const V3 wb = m.local_b;
        const float d = dot(wa - wb, m.normal);
        m.pen_uu = -d * 50.0f;
        m.distance = d;
        m.rel_pos1 = wa - center;
        m.rel_len = len(wa - center);
        if (d > threshold) {
            c[i] = c[count - 1];
            c[count - 1] = manifold_empty_point();
            --count;
            continue;
        }
        const V3 proj = wa - m.normal * d;
        const V3 pd = wb - proj;
        if (dot(pd, pd) > threshold * threshold) {
            c[i] = c[count - 1];
            c[count - 1] = manifold_empty_point();
            --count;
        }
    }
}

// --- rows ----------------------------------------------------------------------------------------------------------
// Rows are kept in Bullet units only: the reference builds uu and Bullet-unit copies and solves the ball's rows in
// Bullet units (ConvertRowUnits, arena_geometry.hpp:5498-5526); the uu copies only feed the denominators below.
struct BallSplitRow {
    V3 normal;
    V3 rel_cross_bt;  // rel_ball x normal
    V3 ang_bt;        // ball angular component
    float inv_mass;
    float jac_inv_bt;
    float rhs_bt;
    float applied_bt;
    int32_t static_id;
};

struct BallVelRow {
    V3 normal;
    V3 rel_cross;
    V3 ang;
    float inv_mass;
    float jac_inv;
    float rhs;
    float applied;
    int32_t predictive;
};

struct BallFricRow {
    V3 tangent;
    V3 rel_cross;
    V3 ang;
    float inv_mass;
    float jac_inv;
    float rhs;
    float friction;
    float applied;
    int32_t normal_row;
};

constexpr int kMaxBallSplitRows = 5;  // 4 manifold points + 1 predictive
constexpr int kMaxBallVelRows = 2;    // the manifold's averaged row + 1 predictive
constexpr int32_t kPredictiveStaticId = 99;

struct BallContactRows {
    int split_count;
    int vel_count;
    int fric_count;
    BallSplitRow split[kMaxBallSplitRows];
    BallVelRow vel[kMaxBallVelRows];
    BallFricRow fric[kMaxBallVelRows];
};

RG_HDI V3 ball_inv_inertia_world(float mass, float radius, V3 torque) {
    const float inertia = 0.4f * mass * radius * radius;
    return inertia > 0.0f ? (torque / inertia) : V3{0, 0, 0};
}

// Inverse inertia in Bullet units through the tick-start basis (reference ApplyInverseBallInertiaWorldBtBall /
// ApplyInverseBallInertiaWorldBtColumns, host_validation_and_contact_debug.hpp:1040-1083).
RG_HDI V3 ball_inv_inertia_bt(const BallState& b, float mass, float radius_uu, V3 torque_bt) {
    if (b.restored_inv_inertia_valid) {
        return mul3(b.restored_inv_inertia_bt[0], b.restored_inv_inertia_bt[1], b.restored_inv_inertia_bt[2],
                    torque_bt);
    }
    V3 f{1, 0, 0}, r{0, 1, 0}, u{0, 0, 1};
    if (b.inertia_basis_valid) {
        f = b.inertia_basis_forward;
        r = b.inertia_basis_right;
        u = b.inertia_basis_up;
    }
    const float radius_bt = radius_uu * (1.0f / 50.0f);
    const float inertia_bt = 0.4f * mass * radius_bt * radius_bt;
    const float inv = inertia_bt != 0.0f ? (1.0f / inertia_bt) : 0.0f;
    const float b00 = f.x, b01 = r.x, b02 = u.x;
    const float b10 = f.y, b11 = r.y, b12 = u.y;
    const float b20 = f.z, b21 = r.z, b22 = u.z;
    const float s00 = b00 * inv, s01 = b01 * inv, s02 = b02 * inv;
    const float s10 = b10 * inv, s11 = b11 * inv, s12 = b12 * inv;
    const float s20 = b20 * inv, s21 = b21 * inv, s22 = b22 * inv;
    const V3 row0{s00 * b00 + s01 * b01 + s02 * b02, s00 * b10 + s01 * b11 + s02 * b12,
                  s00 * b20 + s01 * b21 + s02 * b22};
    const V3 row1{s10 * b00 + s11 * b01 + s12 * b02, s10 * b10 + s11 * b11 + s12 * b12,
                  s10 * b20 + s11 * b21 + s12 * b22};
    const V3 row2{s20 * b00 + s21 * b01 + s22 * b02, s20 * b10 + s21 * b11 + s22 * b12,
                  s20 * b20 + s21 * b21 + s22 * b22};
    return mul3(row0, row1, row2, torque_bt);
}

RG_HDI V3 orthonormal_tangent(V3 n) {
    const V3 axis = fabs_(n.z) < 0.70710678f ? V3{0.0f, 0.0f, 1.0f} : V3{1.0f, 0.0f, 0.0f};
    return normalize_or(cross(axis, n), V3{1.0f, 0.0f, 0.0f});
}

// Static split row (reference AppendBallStaticSplitRow / InitializeBallSplitContactRow, arena_geometry.hpp:6588-6715):
// only penetrating contacts push.
RG_HDI void append_split_row(BallContactRows& rows, float pen_uu, V3 normal, V3 rel_uu, const TickConfig& c,
                             V3 rel_bt, float pen_bt, V3 ang_bt, float dt, int32_t static_id) {
    if (rows.split_count >= kMaxBallSplitRows) return;
    if (pen_uu <= 0.0f || dt <= 0.0f) return;
    const float inv_mass = 1.0f / c.ball_mass;
    const V3 ang = ball_inv_inertia_world(c.ball_mass, c.ball_radius, cross(rel_uu, normal));
    float denom = 0.0f;
    if (inv_mass > 0.0f) denom += inv_mass + dot(normal, cross(ang, rel_uu));
    if (denom <= 1e-8f) return;
    const float jac_inv = 1.0f / denom;
    float denom_bt = 0.0f;
    if (inv_mass > 0.0f) denom_bt += inv_mass + dot(normal, cross(ang_bt, rel_bt));
    BallSplitRow& row = rows.split[rows.split_count++];
    row.jac_inv_bt = denom_bt > 1e-8f ? (1.0f / denom_bt) : jac_inv;
    const float p_bt = pen_bt > 0.0f ? pen_bt : pen_uu * (1.0f / 50.0f);
    row.rhs_bt = ((p_bt * 0.8f) / dt) * row.jac_inv_bt;
    row.normal = normal;
    row.rel_cross_bt = cross(rel_bt, normal);
    row.ang_bt = ang_bt;
    row.inv_mass = inv_mass;
    row.applied_bt = 0.0f;
    row.static_id = static_id;
}

// Normal + friction rows of a ball contact against the (static) arena, restitution without Bullet's velocity
// threshold (reference AppendBallVelocityContactRows with the Bullet-unit overrides, arena_geometry.hpp:2013-2403).
// `basis_bt` is the relative velocity the tangent is taken from; `lin_bt` the ball's solver start velocity.
RG_HDI void append_velocity_rows(BallContactRows& rows, V3 normal, float restitution, float friction, float inv_mass,
                                 V3 rel_uu, V3 ang_n_uu, V3 ang_t_uu, V3 rel_bt, V3 ang_n_bt, V3 ang_t_bt,
                                 V3 lin_bt, V3 ext_delta_uu, V3 ang_w, V3 basis_bt, bool predictive) {
    if (rows.vel_count >= kMaxBallVelRows) return;
    const V3 zero{0, 0, 0};
    float denom = 0.0f;
    if (inv_mass > 0.0f) denom += inv_mass + dot(normal, cross(ang_n_uu, rel_uu));
    if (denom <= 1e-8f) return;
    float jac = 1.0f / denom;
    {
        float bden = 0.0f;
        if (inv_mass > 0.0f) bden += inv_mass + dot(normal, cross(ang_n_bt, rel_bt));
        if (bden > 1e-8f) jac = 1.0f / bden;
    }
    const V3 rcn_bt = cross(rel_bt, normal);
    const V3 ext_bt = uu_to_bt_div(ext_delta_uu);
    const V3 rhs_lin = lin_bt + ext_bt;
    const float rhs_ball_n = dot(rhs_lin, normal) + dot(rcn_bt, ang_w + zero);
    const float rhs_other_n = dot(zero + zero, normal) + dot(cross(zero, normal), zero + zero);
    const float rhs_rel_n = rhs_ball_n - rhs_other_n;
    const V3 pt_vel = lin_bt + cross(ang_w, rel_bt);
    const V3 other_pt = zero + cross(zero, zero);
    const float rest_rel_n = dot(pt_vel - other_pt, normal);
    const float curve = fmax_(restitution * -rest_rel_n, 0.0f);
    const float verr = curve - rhs_rel_n;
    const int ni = rows.vel_count++;
    BallVelRow& vr = rows.vel[ni];
    vr.normal = normal;
    vr.rel_cross = rcn_bt;
    vr.ang = ang_n_bt;
    vr.inv_mass = inv_mass;
    vr.jac_inv = jac;
    vr.rhs = verr * jac;
    vr.applied = 0.0f;
    vr.predictive = predictive ? 1 : 0;

    if (rows.fric_count >= kMaxBallVelRows) return;
    V3 tangent;
    {
        const float vn = dot(normal, basis_bt);
        const V3 lat = basis_bt - normal * vn;
        const float lat2 = dot(lat, lat);
        tangent = lat2 > 1.1920928955078125e-7f ? lat * (1.0f / sqrtf(lat2)) : orthonormal_tangent(normal);
    }
    if (friction <= 0.0f) return;
    const V3 naxis = -tangent;
    const float den1 = inv_mass > 0.0f ? inv_mass + dot(naxis, cross(-ang_t_uu, rel_uu)) : 0.0f;
    const float fden = 0.0f + den1;
    if (fden <= 1e-8f) return;
    float fjac = 1.0f / fden;
    {
        const float b1 = inv_mass > 0.0f ? inv_mass + dot(naxis, cross(-ang_t_bt, rel_bt)) : 0.0f;
        const float bden = 0.0f + b1;
        if (bden > 1e-8f) fjac = 1.0f / bden;
    }
    const V3 rpcn = cross(rel_bt, tangent);
    const float v1 = dot(tangent, lin_bt + ext_bt) + dot(rpcn, ang_w);
    const float frel = v1 + 0.0f;
    BallFricRow& fr = rows.fric[rows.fric_count++];
    fr.tangent = tangent;
    fr.rel_cross = rpcn;
    fr.ang = ang_t_bt;
    fr.inv_mass = inv_mass;
    fr.jac_inv = fjac;
    fr.rhs = -frel * fjac;
    fr.friction = friction;
    fr.applied = 0.0f;
    fr.normal_row = ni;
}

// --- queries -------------------------------------------------------------------------------------------------------
// Visits, in BVH leaf order, every triangle whose quantized bounds overlap the box [lo, hi] (Bullet units).
template <class F>
RG_HDI void mesh_query_box(const MeshDevice& m, V3 lo, V3 hi, F&& visit) {
    // Clamp to the quantization bounds first, exactly as quantize_point does: the box quantizes to the same cells, a
    // box reaching past the mesh shrinks to the part it can overlap, and a box with a non-finite coordinate (a car
    // whose state went NaN, which the reference's EPA can produce on a flat landing) collapses onto the bounds' corner
    // like the reference's quantized BVH walk does, instead of scanning every triangle in one lane.
    lo = vmin(vmax(lo, m.quant.aabb_min), m.quant.aabb_max);
    hi = vmin(vmax(hi, m.quant.aabb_min), m.quant.aabb_max);
    uint16_t qmin[3], qmax[3];
    quantize_point(m.quant, lo, 0, qmin);
    quantize_point(m.quant, hi, 1, qmax);
    const float l3[3] = {lo.x - m.grid_lo.x, lo.y - m.grid_lo.y, lo.z - m.grid_lo.z};
    const bool small = (hi.x - lo.x) <= kQueryExtentBt && (hi.y - lo.y) <= kQueryExtentBt &&
                       (hi.z - lo.z) <= kQueryExtentBt;
    int begin = 0, end = m.tri_count;
    const CellEntry* list = m.rank_entries;
    if (small) {
        int cell[3];
        for (int a = 0; a < 3; ++a) {
            int ci = x86_f2i(floorf(l3[a] / kQueryCellBt));
            ci = ci < 0 ? 0 : (ci >= m.grid_dims[a] ? m.grid_dims[a] - 1 : ci);
            cell[a] = ci;
        }
        const int ci = (cell[2] * m.grid_dims[1] + cell[1]) * m.grid_dims[0] + cell[0];
        begin = m.cell_start[ci];
        end = m.cell_start[ci + 1];
        list = m.cell_entries;
    }
    // entries are tested four at a time: the four 16-byte loads are independent, so their latencies overlap
    auto overlaps = [&](const CellEntry& t) {
        return !(qmin[0] > t.qmax[0] || qmax[0] < t.qmin[0] || qmin[1] > t.qmax[1] || qmax[1] < t.qmin[1] ||
                 qmin[2] > t.qmax[2] || qmax[2] < t.qmin[2]);
    };
    for (int e = begin; e < end; e += 4) {
        int rank[4];
        unsigned hits = 0u;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const CellEntry en = list[e + k < end ? e + k : e];
            rank[k] = en.rank;
            hits |= (e + k < end && overlaps(en)) ? (1u << k) : 0u;
        }
        while (hits != 0u) {
            const int k = ctz32(hits);
            hits &= hits - 1u;
            const int r = k == 0 ? rank[0] : (k == 1 ? rank[1] : (k == 2 ? rank[2] : rank[3]));
            visit(m.tris[r]);
        }
    }
}

// Bullet's ray-vs-leaf-box test of the quantized BVH walk: the ray must cross the leaf's dequantized bounds within its
// length (reference ArenaMeshBvhRayLeaf, include/rocketgpu/detail/arena/mesh_bvh.hpp:522-558, and the same slab test
// in HostRayCastArenaMeshBlocks, host_validation_and_contact_debug.hpp:1591-1602).
struct RayLeaf {
    V3 src, inv;
    float lambda_max;
};
RG_HDI RayLeaf make_ray_leaf(V3 from, V3 to) {
    RayLeaf r;
    const V3 d = to - from;
    const float rl = 1.0f / sqrtf(d.y * d.y + d.x * d.x + d.z * d.z);
    const V3 n{d.x * rl, d.y * rl, d.z * rl};
    r.lambda_max = n.x * d.x + n.y * d.y + n.z * d.z;
    r.inv = V3{n.x == 0.0f ? 1e18f : 1.0f / n.x, n.y == 0.0f ? 1e18f : 1.0f / n.y, n.z == 0.0f ? 1e18f : 1.0f / n.z};
    r.src = from;
    return r;
}
RG_HDI bool ray_leaf_hits(const Quantization& q, const RayLeaf& r, const uint16_t* qmin, const uint16_t* qmax) {
    const V3 lo{q.aabb_min.x + static_cast<float>(qmin[0]) / q.scale.x,
                q.aabb_min.y + static_cast<float>(qmin[1]) / q.scale.y,
                q.aabb_min.z + static_cast<float>(qmin[2]) / q.scale.z};
    const V3 hi{q.aabb_min.x + static_cast<float>(qmax[0]) / q.scale.x,
                q.aabb_min.y + static_cast<float>(qmax[1]) / q.scale.y,
                q.aabb_min.z + static_cast<float>(qmax[2]) / q.scale.z};
    const float tmin = ((r.inv.x < 0.0f ? hi.x : lo.x) - r.src.x) * r.inv.x;
    const float tmax = ((r.inv.x < 0.0f ? lo.x : hi.x) - r.src.x) * r.inv.x;
    const float tymin = ((r.inv.y < 0.0f ? hi.y : lo.y) - r.src.y) * r.inv.y;
    const float tymax = ((r.inv.y < 0.0f ? lo.y : hi.y) - r.src.y) * r.inv.y;
    if (!(tmin <= tymax) || !(tymin <= tmax)) return false;
    const float t0 = tymin <= tmin ? tmin : tymin;
    const float t1 = tmax <= tymax ? tmax : tymax;
    const float tzmin = ((r.inv.z < 0.0f ? hi.z : lo.z) - r.src.z) * r.inv.z;
    const float tzmax = ((r.inv.z < 0.0f ? lo.z : hi.z) - r.src.z) * r.inv.z;
    if (!(t0 <= tzmax) || !(tzmin <= t1)) return false;
    return (tzmin <= t0 ? t0 : tzmin) < r.lambda_max && 0.0f < (t1 <= tzmax ? t1 : tzmax);
}

// Closest hit of the segment from -> to against the mesh, Bullet's triangle ray test in the reference's arithmetic
// (btTriangleRaycastCallback as evaluated by HostRayCastArenaMeshBlocks, host_validation_and_contact_debug.hpp:
// 1603-1690): returns the hit fraction and the hit triangle, ties kept by the first triangle in leaf order.
RG_HDI bool mesh_ray_closest(const MeshDevice& m, V3 from, V3 to, float& out_fraction, const DevTri*& out_tri) {
    bool hit = false;
    float hit_fraction = 0.0f;
    float fraction = 1.0f;
    const DevTri* win = nullptr;
    const RayLeaf leaf = make_ray_leaf(from, to);
    mesh_query_box(m, vmin(from, to), vmax(from, to), [&](const DevTri& t) {
        if (!ray_leaf_hits(m.quant, leaf, t.qmin, t.qmax)) return;
        const V3 n = cross(t.b - t.a, t.c - t.a);
        const float plane = dot(t.a, n);
        const float dist_a = ((n.x * from.x + n.y * from.y) + n.z * from.z) - plane;
        const float dist_b = ((n.x * to.x + n.y * to.y) + n.z * to.z) - plane;
        if (dist_a * dist_b >= 0.0f) return;
        const float proj = dist_a - dist_b;
        if (proj == 0.0f) return;
        const float d = dist_a / proj;
        const float keep = 1.0f - d;
        const V3 p{keep * from.x + d * to.x, keep * from.y + d * to.y, keep * from.z + d * to.z};
        const float tol = -0.0001f * dot(n, n);
        const V3 v0 = t.a - p, v1 = t.b - p, v2 = t.c - p;
        auto edge_ok = [&](V3 u, V3 w) {
            const V3 c{u.y * w.z - u.z * w.y, u.z * w.x - u.x * w.z, u.x * w.y - u.y * w.x};
            return !(((c.x * n.x + c.y * n.y) + c.z * n.z) < tol);
        };
        if (!(edge_ok(v0, v1) && edge_ok(v1, v2) && edge_ok(v2, v0))) return;
        if (d >= fraction) return;
        if (!(d < 0.0f || d > 1.0f) && (!hit || d < hit_fraction)) {
            hit = true;
            hit_fraction = d;
            win = &t;
        }
        fraction = hit ? hit_fraction : 1.0f;
    });
    out_fraction = hit_fraction;
    out_tri = win;
    return hit;
}

// The ray of a body's motion this tick, from `cur` (backed off 0.04 bt) to `to`, against the mesh; a hit gives the hit
// plane's normal (facing the ray's start) and the motion's signed distance past it (reference
// PredictiveContactRayForBody tail, env_step.hpp:4075-4127).
RG_HDI bool predictive_ray(const MeshDevice& m, V3 cur, V3 to, V3& out_n, float& out_dist) {
    constexpr float kCcdMotionThresholdBt = 0.02f;
    constexpr float kRayBackoffBt = 0.04f;
    const V3 mv{to.x - cur.x, to.y - cur.y, to.z - cur.z};
    const float m2 = mv.x * mv.x + mv.y * mv.y + mv.z * mv.z;
    if (!(m2 > kCcdMotionThresholdBt * kCcdMotionThresholdBt)) return false;
    const float inv_len = 1.0f / sqrtf(m2);
    const V3 from{cur.x - inv_len * mv.x * kRayBackoffBt, cur.y - inv_len * mv.y * kRayBackoffBt,
                  cur.z - inv_len * mv.z * kRayBackoffBt};
    const V3 delta{to.x - from.x, to.y - from.y, to.z - from.z};
    if (!(len(delta) * 50.0f > 0.0f) || m.tri_count == 0) return false;
    float f = 0.0f;
    const DevTri* t = nullptr;
    if (!mesh_ray_closest(m, from, from + delta, f, t) || !(f < 1.0f)) return false;
    V3 n = cross(t->b - t->a, t->c - t->a);
    const bool behind = dot(n, from) - dot(t->a, n) <= 0.0f;
    const float il = 1.0f / sqrtf((n.y * n.y + n.x * n.x) + n.z * n.z);
    n = V3{n.x * il, n.y * il, n.z * il};
    if (behind) n = -n;
    const V3 d{delta.x * f, delta.y * f, delta.z * f};
    const float d_len = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
    const float s = d_len > kRayBackoffBt ? d_len - kRayBackoffBt : 0.0f;
    const float inv_d = 1.0f / d_len;
    const V3 ds{inv_d * d.x * s, inv_d * d.y * s, inv_d * d.z * s};
    out_n = n;
    out_dist = ((delta.y - ds.y) * n.y + (delta.x - ds.x) * n.x) + (delta.z - ds.z) * n.z;
    return true;
}
// Predictive (continuous) contact of the ball: its centre's motion this tick (reference PredictiveContactRayForBody
// body 0, env_step.hpp:3894-4128).
RG_HDI bool ball_predictive_hit(const BallState& b, const MeshDevice& m, float dt, V3& out_n, float& out_dist) {
    return predictive_ray(m, b.pos_bt, b.pos_bt + b.vel_bt * dt, out_n, out_dist);
}

// --- the ball's arena contact stage ---------------------------------------------------------------------------------
// Builds the ball's mesh manifold and its contact rows for this tick (the mesh branch of
// AppendBallWorldSpecialContactRows). `solver_vel_bt` is the ball's linear velocity the solver starts from;
// `ext_delta` the external (gravity) velocity change in uu/s.
// event_env >= 0: each triangle the ball meets is a ball-world event of that arena, with the triangle's own normal
// (reference AppendBallWorldSpecialContactRows, arena_ball.hpp:1927-1936, 2195-2240).
RG_NOINL void ball_mesh_contacts(const BallState& b, BallWorldScratch& s, const TickConfig& c, const MeshDevice& m,
                               V3 ext_delta, V3 solver_vel_bt, float dt, BallContactRows& rows, int event_env = -1) {
    const float radius_bt = c.ball_radius * (1.0f / 50.0f);
    const float threshold = (radius_bt + 0.08f) * 0.02f;
    const float rwt = radius_bt + threshold;
    const V3 center = b.pos_bt;
    int count = s.count;
    if (m.tri_count > 0) {
        V3 bx, by, bz;
        ball_basis(b, bx, by, bz);
        mesh_query_box(m, V3{center.x - rwt, center.y - rwt, center.z - rwt},
                       V3{center.x + rwt, center.y + rwt, center.z + rwt}, [&](const DevTri& t) {
            V3 n, on_tri;
            float pen_uu, depth;
            if (!sphere_triangle(center, radius_bt, threshold, t.a, t.b, t.c, n, pen_uu, on_tri, depth)) return;
            if (event_env >= 0 && c.events.windows) {
                PhysicsEvent e = new_event(kEventBallWorldContact);
                e.position = b.pos;
                e.normal = n;
                e.ball_position = b.pos;
                e.ball_velocity = b.vel;
                emit_event(c.events, static_cast<uint32_t>(event_env), e);
            }
            const V3 on_a = on_tri + n * depth;
            const V3 rel = on_a - center;
            BallManifoldPt p;
            p.local_a = V3{dot(rel, bx), dot(rel, by), dot(rel, bz)};
            p.rel_len = len(rel);
            V3 io_n = n;
            V3 io_b = on_tri;
            adjust_internal_edge(t, on_a, depth, io_b, io_n);
            p.normal = io_n;
            p.pen_uu = pen_uu;
            p.local_b = io_b;
            p.tri = t.source_index;
            p.rel_pos1 = V3{0, 0, 0};
            p.distance = 0.0f;
            manifold_insert(s.pts, count, p, threshold);
        });
    }
    manifold_refresh(s.pts, count, center, b, threshold);
    s.count = count;
    if (count == 0) return;

    // one split row per penetrating point, one averaged normal row and its friction row for the manifold
    V3 normal_sum{0, 0, 0};
    float rel_len_sum = 0.0f;
    for (int i = 0; i < count; ++i) {
        normal_sum = normal_sum + s.pts[i].normal;
        rel_len_sum += s.pts[i].rel_len;
    }
    for (int i = 0; i < count; ++i) {
        const BallManifoldPt& q = s.pts[i];
        const V3 ang_bt = ball_inv_inertia_bt(b, c.ball_mass, c.ball_radius, cross(q.rel_pos1, q.normal));
        append_split_row(rows, q.pen_uu, q.normal, (-q.normal) * c.ball_radius, c, q.rel_pos1, -q.distance, ang_bt,
                         dt, 0);
    }
    const float inv_count = 1.0f / static_cast<float>(count);
    V3 normal = normal_sum;
    float dist_bt = rel_len_sum;
    float friction = c.ball_friction;
    float restitution = b.constrained_2d ? 0.0f : c.ball_restitution;
    if (count > 1) {
        float fs = friction, rs = restitution;
        for (int i = 1; i < count; ++i) {
            fs += friction;
            rs += restitution;
        }
        friction = inv_count * fs;
        restitution = inv_count * rs;
        const float l2 = dot(normal, normal);
        normal = l2 >= kSimdEpsilon * kSimdEpsilon ? normal * (1.0f / sqrtf(l2)) : V3{1.0f, 0.0f, 0.0f};
        dist_bt = inv_count * dist_bt;
    }
    const V3 rel_bt = normal * (-dist_bt);
    const V3 rel_uu = rel_bt * 50.0f;
    const float inv_mass = 1.0f / c.ball_mass;
    const V3 ang_n_uu = ball_inv_inertia_world(c.ball_mass, c.ball_radius, cross(rel_uu, normal));
    const V3 basis_bt = (solver_vel_bt + uu_to_bt_div(ext_delta)) + cross(b.ang_vel, rel_bt);
    V3 tangent;
    {
        const float vn = dot(normal, basis_bt);
        const V3 lat = basis_bt - normal * vn;
        const float lat2 = dot(lat, lat);
        tangent = lat2 > 1.1920928955078125e-7f ? lat * (1.0f / sqrtf(lat2)) : orthonormal_tangent(normal);
    }
    const V3 ang_t_uu = ball_inv_inertia_world(c.ball_mass, c.ball_radius, cross(rel_uu, tangent));
    const V3 ang_n_bt = ball_inv_inertia_bt(b, c.ball_mass, c.ball_radius, cross(rel_bt, normal));
    const V3 ang_t_bt = ball_inv_inertia_bt(b, c.ball_mass, c.ball_radius, cross(rel_bt, tangent));
    append_velocity_rows(rows, normal, restitution, friction, inv_mass, rel_uu, ang_n_uu, ang_t_uu, rel_bt, ang_n_bt,
                         ang_t_bt, solver_vel_bt, ext_delta, b.ang_vel, basis_bt, false);
}

// The predictive contact's rows (reference AppendPredictiveContactRows body 0, env_step.hpp:4182-4207).
RG_HDI void ball_predictive_rows(const BallState& b, const TickConfig& c, V3 n, float distance_bt, V3 ext_delta,
                                 V3 solver_vel_bt, float dt, BallContactRows& rows) {
    const V3 zero{0, 0, 0};
    const float pen_bt = -distance_bt;
    append_split_row(rows, pen_bt * 50.0f, n, zero, c, zero, pen_bt, zero, dt, kPredictiveStaticId);
    const V3 basis_bt = solver_vel_bt + uu_to_bt_div(ext_delta);
    append_velocity_rows(rows, n, 0.0f, c.ball_friction, 1.0f / c.ball_mass, zero, zero, zero, zero, zero, zero,
                         solver_vel_bt, ext_delta, b.ang_vel, basis_bt, true);
}

RG_HDI float bt_dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// PGS over the ball's normal and friction rows at the velocity level, in the order of the sorted manifold list
// (predictive rows first when the predictive manifold is listed, then the rest in row order; each normal row's
// friction rows follow it), at most 10 iterations, stopping when no impulse changed. Returns the velocity deltas.
RG_HDI void ball_solve_velocity(BallContactRows& rows, bool pred_listed, V3& d_lin, V3& d_ang) {
    d_lin = V3{0, 0, 0};
    d_ang = V3{0, 0, 0};
    if (rows.vel_count == 0 && rows.fric_count == 0) return;
    int norder[kMaxBallVelRows];
    int forder[kMaxBallVelRows];
    int nn = 0, nf = 0;
    if (rows.vel_count <= 1 && rows.fric_count <= 1) {
        if (rows.vel_count == 1) norder[nn++] = 0;
        if (rows.fric_count == 1) forder[nf++] = 0;
    } else {
        bool used[kMaxBallVelRows] = {false, false};
        if (pred_listed) {
            for (int r = 0; r < rows.vel_count; ++r)
                if (rows.vel[r].predictive) {
                    used[r] = true;
                    norder[nn++] = r;
                }
        }
        for (int r = 0; r < rows.vel_count; ++r)
            if (!used[r]) norder[nn++] = r;
        bool fused[kMaxBallVelRows] = {false, false};
        for (int k = 0; k < nn; ++k)
            for (int f = 0; f < rows.fric_count; ++f)
                if (!fused[f] && rows.fric[f].normal_row == norder[k]) {
                    fused[f] = true;
                    forder[nf++] = f;
                }
        for (int f = 0; f < rows.fric_count; ++f)
            if (!fused[f]) forder[nf++] = f;
    }
    for (int iter = 0; iter < 10; ++iter) {
        bool changed = false;
        for (int k = 0; k < nn; ++k) {
            BallVelRow& r = rows.vel[norder[k]];
            float di = r.rhs;
            const float dv = bt_dot(r.normal, d_lin) + bt_dot(r.rel_cross, d_ang);
            di = di - dv * r.jac_inv;
            const float before = r.applied;
            const float sum = before + di;
            if (sum < 0.0f) {
                di = -before;
                r.applied = 0.0f;
            } else {
                r.applied = sum;
            }
            if (di == 0.0f) {
                changed = (f2u(before) != f2u(r.applied)) || changed;
                continue;
            }
            d_lin = d_lin + (r.normal * r.inv_mass) * di;
            d_ang = d_ang + r.ang * di;
            changed = true;
        }
        for (int k = 0; k < nf; ++k) {
            BallFricRow& r = rows.fric[forder[k]];
            const float total = rows.vel[r.normal_row].applied;
            if (total <= 0.0f) continue;
            const float maxi = r.friction * total;
            float di = r.rhs;
            const float dv = bt_dot(r.tangent, d_lin) + bt_dot(r.rel_cross, d_ang);
            di = di - dv * r.jac_inv;
            const float before = r.applied;
            const float sum = before + di;
            if (sum < -maxi) {
                di = -maxi - before;
                r.applied = -maxi;
            } else if (sum > maxi) {
                di = maxi - before;
                r.applied = maxi;
            } else {
                r.applied = sum;
            }
            if (di == 0.0f) {
                changed = (f2u(before) != f2u(r.applied)) || changed;
                continue;
            }
            d_lin = d_lin + (r.tangent * r.inv_mass) * di;
            d_ang = d_ang + r.ang * di;
            changed = true;
        }
        if (!changed) break;
    }
}

// Split-impulse position push (Bullet units) over the ball's split rows in manifold-list order: the rows of each
// listed static id in turn (`order_ids`, -1 terminated), then the rest in row order. Returns the push velocity.
RG_HDI V3 ball_solve_split(BallContactRows& rows, const int32_t* order_ids, int n_ids) {
    V3 push{0, 0, 0}, turn{0, 0, 0};
    if (rows.split_count == 0) return push;
    int order[kMaxBallSplitRows];
    int no = 0;
    if (rows.split_count > 1 && n_ids > 0) {
        bool used[kMaxBallSplitRows] = {false, false, false, false, false};
        for (int k = 0; k < n_ids; ++k)
            for (int r = 0; r < rows.split_count; ++r)
                if (!used[r] && rows.split[r].static_id >= 0 && rows.split[r].static_id == order_ids[k]) {
                    used[r] = true;
                    order[no++] = r;
                }
        for (int r = 0; r < rows.split_count; ++r)
            if (!used[r]) order[no++] = r;
    } else {
        for (int r = 0; r < rows.split_count; ++r) order[no++] = r;
    }
    for (int iter = 0; iter < 10; ++iter) {
        bool changed = false;
        for (int k = 0; k < no; ++k) {
            BallSplitRow& r = rows.split[order[k]];
            const float before = r.applied_bt;
            float di = r.rhs_bt;
            const float term = (bt_dot(r.normal, push) + bt_dot(r.rel_cross_bt, turn)) * r.jac_inv_bt;
            di -= term;
            const float sum = r.applied_bt + di;
            if (sum < 0.0f) {
                di = -r.applied_bt;
                r.applied_bt = 0.0f;
            } else {
                r.applied_bt = sum;
            }
            if (di == 0.0f) {
                changed = (f2u(before) != f2u(r.applied_bt)) || changed;
                continue;
            }
            push = push + (r.normal * r.inv_mass) * di;
            turn = turn + r.ang_bt * di;
            changed = true;
        }
        if (!changed) break;
    }
    return push;
}

}  // namespace rg
