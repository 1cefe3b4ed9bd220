// Car-ball contacts, host+device: the contact geometry (box-sphere GJK/EPA with a closest-point fallback), the
// retained 4-point manifold per car, the two-body contact rows, and the ball-hit bookkeeping with the game's extra
// hit impulse.
//
// Reference: the world step's ball-car stage (include/rocketgpu/detail/step/env_step.hpp:5074-5133);
// AppendBallCarContactRowsRetained (triangle_and_carcar.hpp:1700-1779) with RefreshBallCarRetainedManifold /
// AddBallCarRetainedPoint (:1571-1650); ComputeBallCarContactGeometry (:1102-1146, GJK :626-821, sphere-box
// fallback :994-1100); AppendBallCarContactRows (:1342-1550) with InitializeBallVelocityContactRow /
// InitializeBallFrictionContactRow / InitializeBallSplitContactRow / AppendBallCarSplitRow (arena_geometry.hpp:
// 2013-2271, 6588-6760); CommitBallCarHit(FromManifold) (triangle_and_carcar.hpp:1178-1331); ApplyBallExtraHits
// (env_step.hpp:6929-6948).
#pragma once

#include "rg_ball_world.cuh"
#include "rg_car.cuh"
#include "rg_car_world.cuh"
#include "rg_gjk.cuh"
#include "rg_vehicle.cuh"

namespace rg {

// One retained car-ball contact point (reference BallCarRetainedPoint): body-space points on the ball and the car,
// their world positions at the last refresh, the normal (car toward ball) and the separation.
struct BallCarPoint {
    V3 local_a, local_b, pos_a, pos_b, normal;
    float distance;
};
// Persistent per car slot (reference BallCarRetainedManifold).
struct alignas(16) BallCarScratch {
    BallCarPoint pts[4];
    int32_t count;
    int32_t pad[3];
};

// ---- shapes and thresholds ------------------------------------------------------------------------------------------
// reference BallCarShapeMargin (arena_geometry.hpp:137-141), in uu
RG_HDI float ball_car_shape_margin(const CarConfig& cfg) {
    const V3 h = bullet_hitbox_size(cfg) * 0.5f;
    return fmin_(2.0f, fmin_(h.x, fmin_(h.y, h.z)) * 0.1f);
}
// reference BallCarContactBreakingThresholdBT (triangle_and_carcar.hpp:823-832)
RG_HDI float ball_car_threshold_bt(const CarConfig& cfg, float ball_radius) {
    const float m = ball_car_shape_margin(cfg);
    const V3 half_uu = (bullet_hitbox_size(cfg) * 0.5f) - V3{m, m, m} + V3{m, m, m};
    const float car_disc = len(half_uu * (1.0f / 50.0f)) + len(cfg.hitbox_offset) * (1.0f / 50.0f);
    const float sphere_disc = ball_radius * (1.0f / 50.0f) + 0.08f;
    return fmin_(car_disc, sphere_disc) * 0.02f;
}

// A fresh contact this tick, before it is merged into the retained manifold.
struct BallCarGeom {
    V3 normal;
    float penetration_uu;
    V3 rel_ball_uu, rel_car_uu;
    bool exact;
    V3 rel_ball_bt, rel_car_bt, ball_local_bt, car_local_bt;
};

// Closest point of the car's box (shrunk by the ball-car margin, in the car frame) to the ball centre
// (reference ComputeBallCarContactGeometrySphereBox).
RG_HDI bool ball_car_sphere_box(const BallState& b, const CarState& c, const CarConfig& cfg, float ball_radius,
                                float max_contact_bt, BallCarGeom& g) {
    V3 f, r, u;
    car_basis(c, f, r, u);
    const V3 off = cfg.hitbox_offset * (1.0f / 50.0f);
    const V3 box_origin = c.pos_bt + rotate_via_basis(f, r, u, off);
    const V3 d = b.pos_bt - box_origin;
    const V3 rel{dot(f, d), dot(r, d), dot(u, d)};
    const float radius_bt = ball_radius * (1.0f / 50.0f);
    const float margin_bt = ball_car_shape_margin(cfg) * (1.0f / 50.0f);
    const V3 raw_half = (bullet_hitbox_size(cfg) * 0.5f) * (1.0f / 50.0f);
    const V3 hb = (bullet_hitbox_size(cfg) * (1.0f / 50.0f)) / 2.0f;
    const float safe = 0.1f * fmin_(hb.x, fmin_(hb.y, hb.z));
    const float inset = safe < 0.04f ? safe : 0.04f;
    const V3 half{raw_half.x - inset, raw_half.y - inset, raw_half.z - inset};
    auto clampf_ = [](float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); };
    V3 closest{clampf_(rel.x, -half.x, half.x), clampf_(rel.y, -half.y, half.y), clampf_(rel.z, -half.z, half.z)};
    V3 nl = rel - closest;
    const float inter = radius_bt + margin_bt;
    const float contact = inter + max_contact_bt;
    const float d2 = len2(nl);
    if (d2 > contact * contact) return false;
    float dist;
    if (d2 <= 1.1920929e-7f) {
        float fd = half.x - rel.x;
        float mn = fd;
        closest = rel;
        closest.x = half.x;
        nl = V3{1.0f, 0.0f, 0.0f};
        fd = half.x + rel.x;
        if (fd < mn) {
            mn = fd;
            closest = rel;
            closest.x = -half.x;
            nl = V3{-1.0f, 0.0f, 0.0f};
        }
        fd = half.y - rel.y;
        if (fd < mn) {
            mn = fd;
            closest = rel;
            closest.y = half.y;
            nl = V3{0.0f, 1.0f, 0.0f};
        }
        fd = half.y + rel.y;
        if (fd < mn) {
            mn = fd;
            closest = rel;
            closest.y = -half.y;
            nl = V3{0.0f, -1.0f, 0.0f};
        }
        fd = half.z - rel.z;
        if (fd < mn) {
            mn = fd;
            closest = rel;
            closest.z = half.z;
            nl = V3{0.0f, 0.0f, 1.0f};
        }
        fd = half.z + rel.z;
        if (fd < mn) {
            mn = fd;
            closest = rel;
            closest.z = -half.z;
            nl = V3{0.0f, 0.0f, -1.0f};
        }
        dist = -mn;
    } else {
        dist = sqrtf(d2);
        nl = nl * (1.0f / dist);
    }
    const V3 point_box_local = closest + nl * margin_bt;
    const float pen_depth = dist - inter;
    g.penetration_uu = -pen_depth * 50.0f;
    const V3 point_box_world = box_origin + rotate_via_basis(f, r, u, point_box_local);
    g.normal = rotate_via_basis(f, r, u, nl);
    g.rel_ball_uu = -g.normal * ball_radius;
    g.rel_car_uu = point_box_world * 50.0f - c.pos;
    g.exact = false;
    return true;
}

// reference ComputeBallCarContactGeometry: the GJK/EPA contact, else the closest-point fallback.
RG_HDI bool ball_car_geometry(const BallState& b, const CarState& c, const CarConfig& cfg, float ball_radius,
                              float threshold_bt, BallCarGeom& g) {
    V3 f, r, u, bx, by, bz;
    car_basis(c, f, r, u);
    ball_basis(b, bx, by, bz);
    gjk::BallBoxContact bc;
    const V3 raw_half = (bullet_hitbox_size(cfg) * 0.5f) * (1.0f / 50.0f);
    if (gjk::ball_box_contact(f, r, u, c.pos_bt, cfg.hitbox_offset * (1.0f / 50.0f), raw_half, bx, by, bz, b.pos_bt,
                              ball_radius * (1.0f / 50.0f), threshold_bt, bc)) {
        g.normal = bc.normal;
        g.penetration_uu = -bc.distance_bt * 50.0f;
        g.rel_ball_uu = bc.rel_ball_bt * 50.0f;
        g.rel_car_uu = bc.rel_car_bt * 50.0f;
        g.exact = true;
        g.rel_ball_bt = bc.rel_ball_bt;
        g.rel_car_bt = bc.rel_car_bt;
        g.ball_local_bt = bc.ball_local_bt;
        g.car_local_bt = bc.car_local_bt;
        return true;
    }
    return ball_car_sphere_box(b, c, cfg, ball_radius, fmax_(0.0f, threshold_bt), g);
}

// ---- the retained manifold ---------------------------------------------------------------------------------------
RG_HDI V3 ball_world_point(V3 bx, V3 by, V3 bz, V3 pos, V3 l) {
    return V3{bx.x * l.x + by.x * l.y + bz.x * l.z, bx.y * l.x + by.y * l.y + bz.y * l.z,
              bx.z * l.x + by.z * l.y + bz.z * l.z} + pos;
}
RG_HDI void ball_car_refresh(BallCarPoint* pts, int& count, const BallState& b, const CarState& c, float thr) {
    V3 bx, by, bz, f, r, u;
    ball_basis(b, bx, by, bz);
    car_basis(c, f, r, u);
    for (int i = 0; i < count; ++i) {
        BallCarPoint& p = pts[i];
        p.pos_a = ball_world_point(bx, by, bz, b.pos_bt, p.local_a);
        p.pos_b = car_world_point(f, r, u, c.pos_bt, p.local_b);
        p.distance = dot(p.pos_a - p.pos_b, p.normal);
    }
    const float thr2 = thr * thr;
    int kept = count;
    for (int i = count - 1; i >= 0; --i) {
        const BallCarPoint p = pts[i];
        bool remove = p.distance > thr;
        if (!remove) {
            const V3 proj = p.pos_a - p.normal * p.distance;
            const V3 diff = p.pos_b - proj;
            remove = dot(diff, diff) > thr2;
        }
        if (remove) {
            pts[i] = pts[kept - 1];
            --kept;
        }
    }
    count = kept;
}
RG_HD float ball_car_res(V3 l, V3 p1, V3 p2, V3 p3) {
    const V3 c = cross(l - p1, p2 - p3);
    return dot(c, c);
}
RG_HDI void ball_car_add(BallCarScratch& m, const BallCarPoint& p, float thr) {
    const int count = m.count;
    float shortest = thr * thr;
    int nearest = -1;
    for (int i = 0; i < count; ++i) {
        const V3 d = m.pts[i].local_b - p.local_b;
        const float dd = dot(d, d);
        if (dd < shortest) {
            shortest = dd;
            nearest = i;
        }
    }
    if (nearest >= 0) {
        m.pts[nearest] = p;
        return;
    }
    if (count < 4) {
        m.pts[count] = p;
        m.count = count + 1;
        return;
    }
    int max_i = 4;
    float max_pen = p.distance;
    for (int i = 0; i < 4; ++i) {
        if (m.pts[i].distance < max_pen) {
            max_i = i;
            max_pen = m.pts[i].distance;
        }
    }
    const V3 l = p.local_b, p0 = m.pts[0].local_b, p1 = m.pts[1].local_b, p2 = m.pts[2].local_b,
             p3 = m.pts[3].local_b;
    const float r0 = max_i == 0 ? 0.0f : ball_car_res(l, p1, p3, p2);
    const float r1 = max_i == 1 ? 0.0f : ball_car_res(l, p0, p3, p2);
    const float r2 = max_i == 2 ? 0.0f : ball_car_res(l, p0, p3, p1);
    const float r3 = max_i == 3 ? 0.0f : ball_car_res(l, p0, p2, p1);
    int best = 0;
    float area = r0;
    if (r1 > area) {
        best = 1;
        area = r1;
    }
    if (r2 > area) {
        best = 2;
        area = r2;
    }
    if (r3 > area) best = 3;
    m.pts[best] = p;
}

// ---- two-body rows (ball = body b, car = body a of Bullet's pair) -----------------------------------------------------
struct BcVelRow {
    V3 normal, rel_ball_cross, ball_ang, rel_car_cross, car_ang;
    float ball_inv_mass, car_inv_mass, jac, rhs, applied;
    int32_t car;
};
struct BcFricRow {
    V3 tangent, rel_ball_cross, ball_ang, rel_car_cross, car_ang;
    float ball_inv_mass, car_inv_mass, jac, rhs, applied, friction;
    int32_t car, normal_row;
};
struct BcSplitRow {
    V3 normal, rel_ball_cross, ball_ang, rel_car_cross, car_ang;
    float ball_inv_mass, car_inv_mass, jac, rhs, applied;
    int32_t car;
};
constexpr int kMaxBallCarRows = 4 * 8;
struct BallCarRows {
    BcVelRow vel[kMaxBallCarRows];
    BcFricRow fric[kMaxBallCarRows];
    BcSplitRow split[kMaxBallCarRows];
    int nv, nf, ns;
};

// The rows of one retained contact point (reference AppendBallCarContactRows with the retained override).
// `ball_ext_uu`: the ball's external (gravity) velocity change; `ball_lin_bt`: the ball's solver start velocity.
RG_HDI void ball_car_point_rows(BallCarRows& rows, const BallState& b, const CarState& c, const CarConfig& cfg,
                                const TickConfig& tc, int car, const BallCarPoint& p, V3 ball_ext_uu, V3 ball_lin_bt,
                                float dt) {
    const V3 normal = p.normal;
    const float pen_uu = -p.distance * 50.0f;
    const V3 rel_ball_bt = p.pos_a - b.pos_bt;
    const V3 rel_car_bt = p.pos_b - c.pos_bt;
    const V3 rel_ball_uu = rel_ball_bt * 50.0f;
    const V3 rel_car_uu = rel_car_bt * 50.0f;
    const float split_pen_bt = -p.distance;
    V3 i0, i1, i2, u0, u1, u2;
    car_inv_inertia_world_bt(c, cfg, tc.car_mass, i0, i1, i2);
    car_inv_inertia_uu(c, cfg, tc.car_mass, u0, u1, u2);
    const float ball_inv = 1.0f / tc.ball_mass, car_inv = 1.0f / tc.car_mass;
    // split row (reference AppendBallCarSplitRow / InitializeBallSplitContactRow)
    if (!(pen_uu * 1.0f <= 0.0f || dt <= 0.0f) && rows.ns < kMaxBallCarRows) {
        const float pen = pen_uu * 1.0f;
        const V3 car_ang_bt = mul_rows(i0, i1, i2, -cross(rel_car_bt, normal));
        const V3 ball_ang_bt = ball_inv_inertia_bt(b, tc.ball_mass, tc.ball_radius, cross(rel_ball_bt, normal));
        const V3 ball_ang_uu = ball_inv_inertia_world(tc.ball_mass, tc.ball_radius, cross(rel_ball_uu, normal));
        const V3 car_ang_uu = mul_rows(u0, u1, u2, -cross(rel_car_uu, normal));
        float denom = 0.0f;
        if (ball_inv > 0.0f) denom += ball_inv + dot(normal, cross(ball_ang_uu, rel_ball_uu));
        if (car_inv > 0.0f) denom += car_inv + dot(normal, cross(-car_ang_uu, rel_car_uu));
        if (denom > 1e-8f) {
            const float jac_uu = 1.0f / denom;
            float denom_bt = 0.0f;
            if (ball_inv > 0.0f) denom_bt += ball_inv + dot(normal, cross(ball_ang_bt, rel_ball_bt));
            if (car_inv > 0.0f) denom_bt += car_inv + dot(normal, cross(-car_ang_bt, rel_car_bt));
            BcSplitRow& s = rows.split[rows.ns++];
            s.jac = denom_bt > 1e-8f ? (1.0f / denom_bt) : jac_uu;
            const float pbt = split_pen_bt > 0.0f ? split_pen_bt : pen * (1.0f / 50.0f);
            s.rhs = ((pbt * 0.8f) / dt) * s.jac;
            s.normal = normal;
            s.rel_ball_cross = cross(rel_ball_bt, normal);
            s.rel_car_cross = -cross(rel_car_bt, normal);
            s.ball_ang = ball_ang_bt;
            s.car_ang = car_ang_bt;
            s.ball_inv_mass = ball_inv;
            s.car_inv_mass = car_inv;
            s.applied = 0.0f;
            s.car = car;
        }
    }
    // velocity rows
    const V3 ball_w = b.ang_vel;
    const V3 car_w = c.ang_vel;
    const V3 ball_rhs_lin = ball_lin_bt + uu_to_bt_div(ball_ext_uu);
    const V3 car_ext_bt = c.ext_force_impulse_bt_valid ? c.ext_force_impulse_bt : V3{0.0f, 0.0f, 0.0f};
    const V3 car_ext_w = c.ext_force_impulse_bt_valid ? c.ext_torque_impulse : V3{0.0f, 0.0f, 0.0f};
    const V3 car_rhs_lin = c.vel_bt + car_ext_bt;
    const V3 car_rhs_w = car_w + car_ext_w;
    const V3 basis = (ball_rhs_lin + cross(ball_w, rel_ball_bt)) - (car_rhs_lin + cross(car_rhs_w, rel_car_bt));
    const V3 ball_n_uu = ball_inv_inertia_world(tc.ball_mass, tc.ball_radius, cross(rel_ball_uu, normal));
    const V3 ball_n_bt = ball_inv_inertia_bt(b, tc.ball_mass, tc.ball_radius, cross(rel_ball_bt, normal));
    const V3 car_n_bt = mul_rows(i0, i1, i2, cross(rel_car_bt, -normal));
    const V3 car_n_uu = car_n_bt * (1.0f / 50.0f);
    V3 tangent;
    {
        const float rn = dot(normal, basis);
        const V3 lat = basis - normal * rn;
        const float l2 = dot(lat, lat);
        tangent = l2 > 1.1920928955078125e-7f ? lat * (1.0f / sqrtf(l2)) : orthonormal_tangent(normal);
    }
    const V3 ball_t_uu = ball_inv_inertia_world(tc.ball_mass, tc.ball_radius, cross(rel_ball_uu, tangent));
    const V3 ball_t_bt = ball_inv_inertia_bt(b, tc.ball_mass, tc.ball_radius, cross(rel_ball_bt, tangent));
    const V3 car_t_bt = mul_rows(i0, i1, i2, cross(rel_car_bt, -tangent));
    const V3 car_t_uu = car_t_bt * (1.0f / 50.0f);
    if (rows.nv >= kMaxBallCarRows) return;
    // normal row (reference InitializeBallVelocityContactRow)
    float denom = 0.0f;
    if (ball_inv > 0.0f) denom += ball_inv + dot(normal, cross(ball_n_uu, rel_ball_uu));
    if (car_inv > 0.0f) denom += car_inv + dot(normal, cross(-car_n_uu, rel_car_uu));
    if (denom <= 1e-8f) return;
    float jac = 1.0f / denom;
    {
        float bd = 0.0f;
        if (ball_inv > 0.0f) bd += ball_inv + dot(normal, cross(ball_n_bt, rel_ball_bt));
        if (car_inv > 0.0f) bd += car_inv + dot(normal, cross(-car_n_bt, rel_car_bt));
        if (bd > 1e-8f) jac = 1.0f / bd;
    }
    const V3 rbc = cross(rel_ball_bt, normal);
    const V3 rcc = cross(rel_car_bt, normal);
    const float rhs_ball = dot(ball_rhs_lin, normal) + dot(rbc, ball_w + V3{0.0f, 0.0f, 0.0f});
    const float rhs_car = dot(car_rhs_lin, normal) + dot(rcc, car_rhs_w);
    const float rhs_rel = rhs_ball - rhs_car;
    const V3 rest_ball = ball_lin_bt + cross(ball_w, rel_ball_bt);
    const V3 rest_car = c.vel_bt + cross(car_w, rel_car_bt);
    const float rest_n = dot(rest_ball - rest_car, normal);
    // CarBallCollisionRestitution is 0, with Bullet's 0.2 bt/s threshold
    const float rest_raw = fabs_(rest_n) < 0.2f ? 0.0f : (0.0f * -rest_n);
    const float rest = rest_raw > 0.0f ? rest_raw : 0.0f;
    const int vi = rows.nv++;
    BcVelRow& v = rows.vel[vi];
    v.normal = normal;
    v.rel_ball_cross = rbc;
    v.rel_car_cross = -rcc;
    v.ball_ang = ball_n_bt;
    v.car_ang = car_n_bt;
    v.ball_inv_mass = ball_inv;
    v.car_inv_mass = car_inv;
    v.jac = jac;
    v.rhs = (rest - rhs_rel) * jac;
    v.applied = 0.0f;
    v.car = car;
    // friction row (reference InitializeBallFrictionContactRow, CarBallCollisionFriction = 2)
    constexpr float kFriction = 2.0f;
    if (rows.nf >= kMaxBallCarRows) return;
    const V3 na = -tangent;
    const float d0 = car_inv > 0.0f ? car_inv + dot(na, cross(car_t_uu, rel_car_uu)) : 0.0f;
    const float d1 = ball_inv > 0.0f ? ball_inv + dot(na, cross(-ball_t_uu, rel_ball_uu)) : 0.0f;
    if (d0 + d1 <= 1e-8f) return;
    float fjac = 1.0f / (d0 + d1);
    {
        const float b0 = car_inv > 0.0f ? car_inv + dot(na, cross(car_t_bt, rel_car_bt)) : 0.0f;
        const float b1 = ball_inv > 0.0f ? ball_inv + dot(na, cross(-ball_t_bt, rel_ball_bt)) : 0.0f;
        if (b0 + b1 > 1e-8f) fjac = 1.0f / (b0 + b1);
    }
    const V3 n1 = -tangent;
    const V3 r1c = cross(rel_car_bt, n1);
    const V3 r2c = cross(rel_ball_bt, tangent);
    const float vel1 = dot(n1, c.vel_bt + car_ext_bt) + dot(r1c, car_w);
    const float vel2 = dot(tangent, ball_lin_bt + uu_to_bt_div(ball_ext_uu)) + dot(r2c, ball_w);
    const float relv = vel1 + vel2;
    BcFricRow& fr = rows.fric[rows.nf++];
    fr.tangent = tangent;
    fr.rel_ball_cross = cross(rel_ball_bt, tangent);
    fr.rel_car_cross = -cross(rel_car_bt, tangent);
    fr.ball_ang = ball_t_bt;
    fr.car_ang = car_t_bt;
    fr.ball_inv_mass = ball_inv;
    fr.car_inv_mass = car_inv;
    fr.jac = fjac;
    fr.rhs = (-relv) * fjac;
    fr.applied = 0.0f;
    fr.friction = kFriction;
    fr.car = car;
    fr.normal_row = vi;
}

// The geometry half of a car's ball contact: this tick's fresh contact merged into the retained manifold. It reads
// only the two bodies' poses.
RG_HDI void ball_car_manifold_update(BallCarScratch& m, const BallState& b, const CarState& c, const CarConfig& cfg,
                                     const TickConfig& tc) {
    const float thr = ball_car_threshold_bt(cfg, tc.ball_radius);
    BallCarGeom g;
    const bool fresh = ball_car_geometry(b, c, cfg, tc.ball_radius, thr, g);
    int count = m.count;
    ball_car_refresh(m.pts, count, b, c, thr);
    m.count = count;
    if (fresh) {
        V3 f, r, u;
        car_basis(c, f, r, u);
        const V3 rel_ball = g.exact ? g.rel_ball_bt : uu_to_bt_div(g.rel_ball_uu);
        const V3 rel_car = g.exact ? g.rel_car_bt
                                   : car_world_point(f, r, u, c.pos_bt,
                                                     car_local_point(f, r, u, c.pos_bt,
                                                                     c.pos_bt + g.rel_car_uu * (1.0f / 50.0f))) -
                                         c.pos_bt;
        const V3 pos_a = b.pos_bt + rel_ball;
        const V3 pos_b = c.pos_bt + rel_car;
        const float depth = dot(pos_a - pos_b, g.normal);
        if (depth <= thr) {
            BallCarPoint fp[4];
            fp[0].normal = g.normal;
            if (g.exact) {
                fp[0].local_a = g.ball_local_bt;
                fp[0].local_b = g.car_local_bt;
            } else {
                V3 bx, by, bz;
                ball_basis(b, bx, by, bz);
                const V3 rel = pos_a - b.pos_bt;
                fp[0].local_a = V3{dot(rel, bx), dot(rel, by), dot(rel, bz)};
                fp[0].local_b = car_local_point(f, r, u, c.pos_bt, pos_b);
            }
            fp[0].distance = depth;
            int fc = 1;
            ball_car_refresh(fp, fc, b, c, thr);
            for (int i = 0; i < fc; ++i) ball_car_add(m, fp[i], thr);
        }
    }
}

// The rows half: the rows of every retained point, from the bodies' velocities at the world step.
RG_HDI void ball_car_manifold_rows(const BallCarScratch& m, const BallState& b, const CarState& c, const CarConfig& cfg,
                                   const TickConfig& tc, int car, V3 ball_ext_uu, V3 ball_lin_bt, float dt,
                                   BallCarRows& rows) {
    for (int i = 0; i < m.count; ++i) ball_car_point_rows(rows, b, c, cfg, tc, car, m.pts[i], ball_ext_uu, ball_lin_bt, dt);
}

// The car's contact with the ball this tick: fresh geometry merged into the retained manifold, rows per point
// (reference AppendBallCarContactRowsRetained).
RG_NOINL void ball_car_contacts(BallCarScratch& m, const BallState& b, const CarState& c, const CarConfig& cfg,
                              const TickConfig& tc, int car, V3 ball_ext_uu, V3 ball_lin_bt, float dt,
                              BallCarRows& rows) {
    ball_car_manifold_update(m, b, c, cfg, tc);
    ball_car_manifold_rows(m, b, c, cfg, tc, car, ball_ext_uu, ball_lin_bt, dt, rows);
}

// ---- the ball hit ------------------------------------------------------------------------------------------------
RG_HD V3 ue3_safe_normal(V3 v) {
    const float l2 = len2(v);
    if (l2 == 1.0f) return v;
    if (l2 < 1e-8f) return V3{0.0f, 0.0f, 0.0f};
    const float s = 1.0f / sqrtf(l2);
    return V3{v.x * s, v.y * s, v.z * s};
}
RG_HDI V3 ue3_rotator_forward(const Ue3Rotator& r) {
    const float cp = ue3_rotator_sin(r.pitch + 16384);
    return V3{cp * ue3_rotator_sin(r.yaw + 16384), cp * ue3_rotator_sin(r.yaw), ue3_rotator_sin(r.pitch)};
}
// v rotated by the inverse of q (reference InverseRotate = Rotate(Inverse(q), v), math.hpp:779-874)
RG_HDI V3 quat_inverse_rotate(Q4 q, V3 v) {
    auto inverse = [](Q4 a) {
        const float l2 = a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z;
        if (l2 <= 1e-12f) return Q4{1.0f, 0.0f, 0.0f, 0.0f};
        const float s = 1.0f / l2;
        return Q4{a.w * s, -a.x * s, -a.y * s, -a.z * s};
    };
    auto mul = [](Q4 a, Q4 b) {
        return Q4{a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
                  a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
    };
    const Q4 qi = inverse(q);
    const Q4 p{0.0f, v.x, v.y, v.z};
    const Q4 r = mul(mul(qi, p), inverse(qi));
    return V3{r.x, r.y, r.z};
}
// Bookkeeping of a car's ball touch: touch start, the hit record and the game's extra hit impulse
// (reference CommitBallCarHit). `car_pos` / `car_rot` / `ball_pos`: the bodies at the world step's start;
// `car_start_vel` / `ball_start_vel`: their velocities at the tick start (uu).
// A touch start is a ball-touch event of the car (team `team`) when `events` is on (reference :1216-1227).
RG_HDI void commit_ball_hit(BallState& b, CarState& c, uint32_t car_id, uint64_t env_tick, V3 normal, V3 rel_ball_uu,
                            V3 rel_car_uu, V3 car_pos, Q4 car_rot, V3 ball_pos, V3 car_start_vel,
                            V3 ball_start_vel, uint8_t team, const EventStream& events) {
    const bool started = !c.ball_contact_last_tick && !c.ball_contact_this_tick;
    if (started) {
        c.previous_ball_contact_start = c.last_ball_contact_start;
        c.first_world_after_previous_ball = c.first_world_after_last_ball;
        c.last_ball_contact_start = c.tick_count_since_update;
        c.first_world_after_last_ball = kNoTick;
        c.last_ball_started_with_world = c.last_world_surface_contact == c.tick_count_since_update;
        c.latest_touch_tick = env_tick;
        c.latest_touch_location = car_pos + rel_car_uu;
        c.latest_touch_normal = normal;
    }
    c.ball_contact_this_tick = 1;
    if (started && events.windows) {
        PhysicsEvent e = new_event(kEventBallTouchStart);
        e.car_id = car_id;
        e.team = team;
        e.car_on_ground = c.is_on_ground;
        e.position = c.pos;
        e.car_velocity = c.vel;
        e.ball_position = b.pos;
        e.ball_velocity = b.vel;
        emit_event_for_car(events, car_id, e);
    }
    BallHitInfo& h = c.ball_hit_info;
    const uint8_t had_prior = h.is_valid;
    const uint64_t prev_extra = h.tick_count_when_extra_impulse_applied;
    h.is_valid = 1;
    h.tick_count_when_hit = env_tick;
    h.hit_car_id = car_id;
    h.relative_pos_on_ball = quat_inverse_rotate(b.rot, rel_ball_uu);
    h.ball_pos = ball_pos;
    h.extra_hit_vel = V3{0.0f, 0.0f, 0.0f};
    const bool can_apply = !had_prior || (h.extra_tick_is_previous ? prev_extra != env_tick
                                                                   : (prev_extra > env_tick) ||
                                                                         ((prev_extra + 1ull) < env_tick));
    if (!can_apply) return;
    const V3 rel_pos = ball_pos - car_pos;
    const V3 rel_vel = ball_start_vel - car_start_vel;
    const float rel_speed = fmin_(len(rel_vel), 4600.0f);
    if (!(rel_speed > 0.0f)) return;
    const V3 fwd = ue3_rotator_forward(ue3_quat_to_rotator(car_rot));
    V3 dir = ue3_safe_normal(rel_pos);
    dir.z *= 0.35f;
    dir = ue3_safe_normal(dir);
    const V3 adj = (fwd * dot(dir, fwd)) * (1.0f - 0.65f);
    dir = ue3_safe_normal(dir - adj);
    const float in[5] = {0.0f, 500.0f, 1400.0f, 2300.0f, 4600.0f};
    const float out[5] = {0.65f, 0.65f, 0.6f, 0.55f, 0.30f};
    const V3 added = ((dir * rel_speed) * interp_curve(in, out, fabs_(rel_speed))) * 1.0f;
    h.extra_pending = 1;
    b.tick_count_when_extra_impulse_applied = env_tick;
    h.tick_count_when_extra_impulse_applied = env_tick;
    h.extra_tick_is_previous = 0;
    h.extra_hit_vel = added;
}
// The hit from the retained manifold's averaged point (reference CommitBallCarHitFromManifold).
RG_HDI void commit_ball_hit_from_manifold(BallState& b, CarState& c, const BallCarScratch& m, uint32_t car_id,
                                          uint64_t env_tick, V3 car_pos, Q4 car_rot, V3 ball_pos, V3 car_start_vel,
                                          V3 ball_start_vel, uint8_t team, const EventStream& events) {
    if (m.count == 0) return;
    V3 pa{0.0f, 0.0f, 0.0f}, pb{0.0f, 0.0f, 0.0f}, n{0.0f, 0.0f, 0.0f};
    for (int k = 0; k < m.count; ++k) {
        pa = pa + m.pts[k].pos_a;
        pb = pb + m.pts[k].pos_b;
        n = n + m.pts[k].normal;
    }
    const float inv = 1.0f / static_cast<float>(m.count);
    commit_ball_hit(b, c, car_id, env_tick, ue3_safe_normal(n * inv), (pa * inv - b.pos_bt) * 50.0f,
                    (pb * inv - c.pos_bt) * 50.0f, car_pos, car_rot, ball_pos, car_start_vel, ball_start_vel, team,
                    events);
}
}  // namespace rg
