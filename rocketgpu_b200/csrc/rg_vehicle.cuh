// The vehicle update of one car (suspension rays, tyre forces, steering, sticky force, flip torque, air control,
// jump state, auto-roll, boost) and the car's part of the world step (deferred forces, transform integration) and of
// the post-tick (timers, impulse caches, the RLBot-facing report fields).
//
// Restates the reference's PreTickCar (include/rocketgpu/detail/step/env_step.hpp:3115-3484) and the functions it
// calls in raycast_wheels_and_contact_prep.hpp, for a car that always has a wheel record and a force-queueing frame
// (how BatchSim runs it). Three-wheel (Psyclops) cars and per-wheel state-set normals are not built.
#pragma once

#include "rg_broadphase.cuh"
#include "rg_car.cuh"

namespace rg {

constexpr float kWheelSuspensionStiffness = 500.0f;  // reference host_validation_and_contact_debug.hpp:1-3
constexpr float kWheelDampingCompression = 25.0f;
constexpr float kWheelDampingRelaxation = 40.0f;

constexpr uint8_t kRayHitUnknown = 0, kRayHitArenaMesh = 3, kRayHitCar = 4, kRayHitBall = 5;

// One wheel for one tick (reference WheelStepState, host_validation_and_contact_debug.hpp:5-37).
struct WheelStep {
    V3 ray_source_bt, wheel_dir_ws, wheel_axle_ws, contact_point_bt, contact_normal_ws;
    float wheel_trace_len_bt, suspension_len_bt, suspension_relative_velocity_bt, suspension_relative_velocity;
    float clipped_inv_contact_dot_suspension, extra_pushback, wheel_radius, suspension_rest_length;
    float max_suspension_travel, suspension_force_scale;
    V3 cal_axle_dir, cal_forward_dir;
    float cal_rolling_friction, cal_lat_friction, cal_long_friction, cal_friction_scale;
    int32_t ground_car_idx, ground_static_id;
    uint8_t ground_kind, is_front_wheel, is_in_contact, is_in_contact_with_world;
};

// ---- curves (reference constants.hpp:114-160) ---------------------------------------------------------------------
template <int N>
RG_HDI float interp_curve(const float (&in)[N], const float (&out)[N], float x) {
    if (N < 2 || in[0] >= x) return out[0];
    if (x >= in[N - 1]) return out[N - 1];
    for (int i = 1; i < N; ++i) {
        if (in[i] > x) return (out[i] - out[i - 1]) * ((x - in[i - 1]) / (in[i] - in[i - 1])) + out[i - 1];
    }
    return out[N - 1];
}
RG_HDI float steer_angle_from_speed(const float (&c)[6], float speed_abs) {
    const float in[6] = {0.0f, 500.0f, 1000.0f, 1500.0f, 1750.0f, 3000.0f};
    return interp_curve(in, c, fabs_(speed_abs));
}
RG_HDI float powerslide_steer_angle_from_speed(const float (&c)[2], float speed_abs) {
    const float in[2] = {0.0f, 2500.0f};
    return interp_curve(in, c, fabs_(speed_abs));
}
RG_HDI float drive_torque_factor(float forward_speed) {
    const float in[5] = {-1410.0f, -1400.0f, 0.0f, 1400.0f, 1410.0f};
    const float out[5] = {0.0f, 0.1f, 1.0f, 0.1f, 0.0f};
    return interp_curve(in, out, forward_speed);
}
RG_HDI float non_sticky_friction_factor(float normal_z) {
    const float in[3] = {0.0f, 0.707f, 1.0f};
    const float out[3] = {0.1f, 0.5f, 1.0f};
    return interp_curve(in, out, normal_z);
}
RG_HDI float lat_friction_curve(float x) {
    const float in[2] = {0.0f, 1.0f};
    const float out[2] = {1.0f, 0.2f};
    return interp_curve(in, out, x);
}
RG_HDI float handbrake_long_friction_factor(float x) {
    const float in[2] = {0.0f, 1.0f};
    const float out[2] = {0.5f, 0.9f};
    return interp_curve(in, out, x);
}

// ---- wheel geometry (reference raycast_wheels_and_contact_prep.hpp:420-457, 614-640) -------------------------------
RG_HDI void wheel_bone_z(const CarConfig& cfg, float& front, float& back) {
    front = floorf((cfg.hitbox_offset.z - (cfg.front_suspension_rest - 12.0f)) * 100.0f + 0.5f) / 100.0f;
    back = (cfg.back_suspension_rest == cfg.front_suspension_rest)
               ? front
               : (floorf((cfg.hitbox_offset.z - (cfg.back_suspension_rest - 12.0f)) * 100.0f + 0.5f) / 100.0f);
}
RG_HDI float min_wheel_hit_dist_sq_bt(const CarConfig& cfg) {
    const float d = (cfg.hitbox_size.z * 0.5f - 2.25f) * kUuToBt;
    return d * d;
}
RG_HDI void suspension_force_scales(const CarConfig& cfg, float car_mass, float& front, float& back) {
    const float mass = 1.0f / (1.0f / car_mass);
    const float front_x = cfg.front_wheels_offset.x * kUuToBt;
    const float back_x = -(cfg.back_wheels_offset.x * kUuToBt);
    if (front_x < 0.0f || back_x < 0.0f) {
        front = back = (mass * 0.5f) * 0.5f;
    } else {
        const float back_share = (front_x / (back_x + front_x)) * mass;
        front = (mass - back_share) * 0.5f;
        back = back_share * 0.5f;
    }
}
RG_HDI void init_wheel(WheelStep& w, const CarState& c, const CarConfig& cfg, int i, const CarFrame& f, float bone_z) {
    const bool front = i < 2;
    const bool left = (i % 2) != 0;
    V3 offset = front ? cfg.front_wheels_offset : cfg.back_wheels_offset;
    if (left) offset.y = -offset.y;
    offset.z = cfg.hitbox_offset.z;
    w.ray_source_bt = c.pos_bt + rotate_via_basis(f.fwd, f.right, f.up, offset * kUuToBt);
    w.wheel_dir_ws = -f.up;
    w.wheel_axle_ws = -f.right;
    w.contact_point_bt = V3{0.0f, 0.0f, 0.0f};
    w.wheel_trace_len_bt = w.suspension_len_bt = 0.0f;
    w.suspension_relative_velocity_bt = w.suspension_relative_velocity = 0.0f;
    w.clipped_inv_contact_dot_suspension = 1.0f;
    w.extra_pushback = 0.0f;
    w.wheel_radius = front ? cfg.front_wheel_radius : cfg.back_wheel_radius;
    w.suspension_rest_length = offset.z - bone_z;
    w.max_suspension_travel = 14.5f;
    w.suspension_force_scale = 1.0f;
    w.cal_axle_dir = V3{0.0f, -1.0f, 0.0f};
    w.cal_forward_dir = V3{1.0f, 0.0f, 0.0f};
    w.cal_rolling_friction = w.cal_lat_friction = w.cal_long_friction = w.cal_friction_scale = 0.0f;
    w.ground_car_idx = -1;
    w.ground_static_id = -1;
    w.ground_kind = kRayHitUnknown;
    w.is_front_wheel = front ? 1 : 0;
    w.is_in_contact = w.is_in_contact_with_world = 0;
    w.contact_normal_ws = -w.wheel_dir_ws;
}
RG_HDI void wheel_ray_miss(WheelStep& w) {
    w.suspension_relative_velocity = 0.0f;
    w.clipped_inv_contact_dot_suspension = 1.0f;
    w.extra_pushback = 0.0f;
    w.is_in_contact = 0;
    w.is_in_contact_with_world = 0;
    w.ground_kind = kRayHitUnknown;
    w.ground_car_idx = -1;
    w.contact_normal_ws = -w.wheel_dir_ws;
}
// reference ComputeWheelRayVelocityTerms (:847-862)
RG_HDI void wheel_ray_velocity_terms(const CarState& c, V3 car_up, V3 hit_point_bt, WheelStep& w) {
    const float denominator = dot(w.contact_normal_ws, car_up);
    const V3 relpos_bt = hit_point_bt - c.pos_bt;
    const V3 vel_at_contact_bt = c.vel_bt + cross(c.ang_vel, relpos_bt);
    const float proj_vel_bt = dot(w.contact_normal_ws, vel_at_contact_bt);
    if (denominator > 0.1f) {
        w.clipped_inv_contact_dot_suspension = 1.0f / denominator;
        w.suspension_relative_velocity_bt = proj_vel_bt * w.clipped_inv_contact_dot_suspension;
        w.suspension_relative_velocity = w.suspension_relative_velocity_bt * 50.0f;
    } else {
        w.clipped_inv_contact_dot_suspension = 10.0f;
        w.suspension_relative_velocity = 0.0f;
        w.suspension_relative_velocity_bt = 0.0f;
    }
}

// ---- ray casts ----------------------------------------------------------------------------------------------------
// Closest mesh hit of a segment, rejecting hits nearer than sqrt(min_fraction_sq) of it; returns the hit fraction,
// the triangle and the source's signed plane distance (reference HostRayCastArenaMeshBlocks,
// host_validation_and_contact_debug.hpp:1603-1672, as CastArenaRayDeltaBt runs it).
RG_NOINL bool mesh_ray_cast(const MeshDevice& m, V3 from, V3 to, float min_fraction_sq, float& out_fraction,
                          const DevTri*& out_tri, float& out_dist_a) {
    bool hit = false;
    float hit_fraction = 0.0f, win_dist_a = 0.0f;
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
        if (!(d < 0.0f || d > 1.0f) && !(min_fraction_sq > 0.0f && d * d < min_fraction_sq) &&
            (!hit || d < hit_fraction)) {
            hit = true;
            hit_fraction = d;
            win = &t;
            win_dist_a = dist_a;
        }
        fraction = hit ? hit_fraction : 1.0f;
    });
    out_fraction = hit_fraction;
    out_tri = win;
    out_dist_a = win_dist_a;
    return hit;
}

struct RayHit {
    float t;
    V3 point_bt, normal;
    uint8_t hit, kind;
    int32_t mesh_index;
};

// Bullet's ray-vs-sphere conservative advancement (reference CastGjkRayVsSphere, :206-264).
RG_HDI bool gjk_ray_vs_sphere(V3 from, V3 to, V3 center, float radius, float& out_fraction, V3& out_normal) {
    constexpr float kRadius = 0.001f;
    constexpr int kMaxIterations = 64;
    auto closest = [&](V3 p, V3 c, float& dist, V3& n) {
        const V3 offset = (p + c) * 0.5f;
        const V3 w = (p - offset) - (c - offset);
        const float l2 = dot(w, w);
        if (!(l2 > 1.1920929e-7f * 1.1920929e-7f)) return false;
        const float rlen = 1.0f / sqrtf(l2);
        n = w * rlen;
        dist = (1.0f / rlen) - radius;
        return true;
    };
    const V3 r = to - from;
    float lambda = 0.0f, last_lambda = 0.0f, dist = 0.0f;
    V3 n{0.0f, 0.0f, 0.0f};
    if (!closest(from, center, dist, n)) return false;
    int iter = 0;
    while (dist > kRadius) {
        if (++iter > kMaxIterations) return false;
        lambda = lambda - dist / dot(r, n);
        if (lambda > 1.0f || lambda < 0.0f || lambda <= last_lambda) return false;
        last_lambda = lambda;
        const V3 p = from * (1.0f - lambda) + to * lambda;
        const V3 c = center * lambda + center * (1.0f - lambda);
        float next_dist = 0.0f;
        if (!closest(p, c, next_dist, n)) return false;
        if (next_dist < 0.0f) {
            out_fraction = last_lambda;
            out_normal = n;
            return true;
        }
        dist = next_dist;
    }
    if (dot(n, r) >= 0.0f) return false;
    out_fraction = lambda;
    out_normal = n;
    return true;
}
// reference CastWheelRayAgainstBall (:266-327)
RG_HDI bool wheel_ray_vs_ball(V3 src_bt, V3 dir, float max_len, const BallState& b, float ball_radius,
                              float max_len_bt, RayHit& out) {
    const V3 center = b.pos_bt;
    const float radius_bt = ball_radius * kUuToBt;
    {
        const V3 d = center - src_bt;
        const float reject = radius_bt + max_len_bt + 1.0e-4f;
        if (dot(d, d) > reject * reject) return false;
    }
    const V3 to = src_bt + dir * max_len_bt;
    float fraction = 0.0f;
    V3 normal{0.0f, 0.0f, 0.0f};
    const bool hit = gjk_ray_vs_sphere(src_bt, to, center, radius_bt, fraction, normal);
    const float nl2 = dot(normal, normal);
    if (!hit || nl2 <= 0.0001f) return false;
    normal = normal * (1.0f / sqrtf(nl2));
    if (fraction >= 1.0f) return false;
    const float t_hit = fraction * max_len;
    const V3 p = src_bt * (1.0f - fraction) + to * fraction;
    if (max_len <= 0.0f || t_hit < 0.0f || t_hit > max_len) return false;
    out.hit = 1;
    out.t = t_hit;
    out.point_bt = p;
    out.normal = normal;
    out.kind = kRayHitBall;
    out.mesh_index = -1;
    return true;
}

// The other cars of the arena a wheel ray may land on (null `cars`: none can be reached, see arena_free_cars),
// and the bodies (bit 0 the ball, bit i + 1 car slot i) the car's rays skip this tick (wheel_ray_excluded_bodies).
struct WheelOthers {
    CarState* cars;
    const CarConfig* cfgs;
    int count, self;
    uint32_t excluded;
};

// The bodies a car's suspension rays skip this tick: those whose swept AABB from the arena's last sweep misses the
// box around all four of the car's rays (reference WheelRayExcludedBodies with WheelRaysWhole,
// raycast_wheels_and_contact_prep.hpp:9-25, 508-606, as StepEnvVehicleUpdateCarInline calls it, env_step.hpp:6232).
// The ball is body 0, car slot i body i + 1; bodies without a stored box (not yet swept, or left the sweep) are tested.
RG_HDI uint32_t wheel_ray_excluded_bodies(const CarState& c, const CarConfig& cfg, const Broadphase* bp, int self,
                                          int count) {
    const int bodies = count + 1 < kBpBodies ? count + 1 : kBpBodies;
    const uint32_t mask = (bp != nullptr && bodies > 0)
                              ? (bp->body_aabb_valid & ((1u << bodies) - 1u) & ~(1u << (self + 1)))
                              : 0u;
    if (mask == 0u) return 0u;
    V3 fw, rt, up;
    car_basis(c, fw, rt, up);
    const V3 dir = -up;
    const float oz = cfg.hitbox_offset.z;
    float front_bone, back_bone;
    wheel_bone_z(cfg, front_bone, back_bone);
    const float front_len_bt =
        ((oz - front_bone) * kUuToBt + cfg.front_wheel_radius * kUuToBt) + ((14.5f - kWheelSuspensionSubtraction) * kUuToBt);
    const float back_len_bt =
        ((oz - back_bone) * kUuToBt + cfg.back_wheel_radius * kUuToBt) + ((14.5f - kWheelSuspensionSubtraction) * kUuToBt);
    V3 mn{0.0f, 0.0f, 0.0f}, mx{0.0f, 0.0f, 0.0f};
    for (int i = 0; i < 4; ++i) {
        V3 offset = i < 2 ? cfg.front_wheels_offset : cfg.back_wheels_offset;
        if (i % 2) offset.y = -offset.y;
        offset.z = oz;
        const V3 from = c.pos_bt + rotate_via_basis(fw, rt, up, offset * kUuToBt);
        const V3 to = from + dir * (i < 2 ? front_len_bt : back_len_bt);
        const V3 lo = vmin(from, to), hi = vmax(from, to);
        mn = i == 0 ? lo : vmin(mn, lo);
        mx = i == 0 ? hi : vmax(mx, hi);
    }
    uint32_t excluded = 0u;
    for (int body = 0; body < bodies; ++body) {
        if (!((mask >> body) & 1u)) continue;
        const float* a = bp->body_aabb[body];
        if (a[3] < mn.x || mx.x < a[0] || a[4] < mn.y || mx.y < a[1] || a[5] < mn.z || mx.z < a[2])
            excluded |= 1u << body;
    }
    return excluded;
}

// Distance from a point to a car's hitbox (core box plus margin) by Bullet's GJK pair detector with the Voronoi
// simplex solver; keeps the result only when it is nearer than `out_distance` (reference WheelGjkPointBoxClosest,
// raycast_wheels_and_contact_prep.hpp:4758-4855).
RG_HDI bool wheel_point_box_closest(V3 point_a, V3 box_origin, V3 f, V3 r, V3 u, V3 core, float margin_in,
                                    bool& has_result, float& out_distance, V3& out_normal) {
    constexpr float kRelError2 = 1.0e-6f;
    constexpr float kEps = 1.1920929e-7f;
    const V3 offset = (point_a + box_origin) * 0.5f;
    const V3 la = point_a - offset, lb = box_origin - offset;
    const float margin = 0.0f + margin_in;
    V3 axis{0.0f, 1.0f, 0.0f};
    float sq = 1.0e18f;
    gjk::VoronoiSimplex sx;
    sx.reset();
    bool check = false;
    int iter = 0;
    const V3 pw = V3{0.0f, 0.0f, 0.0f} + la;
    while (true) {
        const V3 sb{dot(f, axis), dot(r, axis), dot(u, axis)};
        const V3 ql{sb.x >= 0.0f ? core.x : -core.x, sb.y >= 0.0f ? core.y : -core.y, sb.z >= 0.0f ? core.z : -core.z};
        const V3 qw{(f.x * ql.x + r.x * ql.y) + u.x * ql.z + lb.x, (f.y * ql.x + r.y * ql.y) + u.y * ql.z + lb.y,
                    (f.z * ql.x + r.z * ql.y) + u.z * ql.z + lb.z};
        const V3 w = pw - qw;
        const float delta = dot(axis, w);
        if (delta > 0.0f && delta * delta > sq * 1.0e18f) {
            check = true;
            break;
        }
        if (sx.in_simplex(w)) {
            check = true;
            break;
        }
        const float f0 = sq - delta, f1 = sq * kRelError2;
        if (f0 <= f1) {
            check = true;
            break;
        }
        sx.add(w, pw, qw);
        if (!sx.update()) {
            check = true;
            break;
        }
        const V3 na = sx.cv;
        if (len2(na) < kRelError2) {
            axis = na;
            check = true;
            break;
        }
        const float prev = sq;
        sq = len2(na);
        if (prev - sq <= kEps * prev) {
            check = true;
            break;
        }
        axis = na;
        if (iter++ > 1000) break;
        if (sx.full()) break;
    }
    if (!check) return has_result;
    sx.update();
    const float l2 = len2(axis);
    if (!(l2 > kEps * kEps)) return has_result;
    const float rlen = 1.0f / sqrtf(l2);
    V3 normal = axis * rlen;
    const float distance = (1.0f / rlen) - margin;
    if (!(distance < 0.0f || distance * distance < 1.0e18f)) return has_result;
    const V3 hm = core + V3{margin_in, margin_in, margin_in};
    const V3 ext{(hm.x * fabs_(f.x) + hm.y * fabs_(r.x)) + hm.z * fabs_(u.x),
                 (hm.x * fabs_(f.y) + hm.y * fabs_(r.y)) + hm.z * fabs_(u.y),
                 (hm.x * fabs_(f.z) + hm.y * fabs_(r.z)) + hm.z * fabs_(u.z)};
    const V3 pos_a = ((la + V3{0.0f, 0.0f, 0.0f}) + (la - V3{0.0f, 0.0f, 0.0f})) * 0.5f;
    const V3 pos_b = ((lb - ext) + (lb + ext)) * 0.5f;
    if (dot(pos_a - pos_b, normal) < 0.0f) normal = normal * -1.0f;
    if (distance < out_distance) {
        has_result = true;
        out_normal = normal;
        out_distance = distance;
    }
    return has_result;
}

// A suspension ray against another car's hitbox: slab test in the box frame, then conservative advancement with the
// point-box distance (reference CastWheelRayAgainstCarHitboxGjkCast, raycast_wheels_and_contact_prep.hpp:4857-4977).
RG_HDI bool wheel_ray_vs_car_box(V3 src, V3 dir, float max_len, float max_len_bt, const CarState& o,
                                 const CarConfig& ocfg, RayHit& out) {
    constexpr float kRadius = 0.001f;
    const V3 to = src + dir * max_len_bt;
    const V3 half_raw = bullet_hitbox_size(ocfg) * (0.5f * kUuToBt);
    const float margin = fmin_(0.1f * fmin_(half_raw.x, fmin_(half_raw.y, half_raw.z)), 0.04f);
    const V3 inner = half_raw - V3{margin, margin, margin};
    V3 f{1.0f, 0.0f, 0.0f}, rt{0.0f, 1.0f, 0.0f}, u{0.0f, 0.0f, 1.0f};
    car_basis(o, f, rt, u);
    const V3 center = o.pos_bt + rotate_via_basis(f, rt, u, ocfg.hitbox_offset * kUuToBt);
    {
        const float rr = len(half_raw) + max_len_bt + 1.0e-3f;
        if (len2(center - src) > rr * rr) return false;
    }
    {
        const V3 rf = src - o.pos_bt, rto = to - o.pos_bt;
        const V3 lf{dot(rf, f), dot(rf, rt), dot(rf, u)}, lt{dot(rto, f), dot(rto, rt), dot(rto, u)};
        const V3 off = ocfg.hitbox_offset * kUuToBt;
        const V3 ext = inner + V3{margin, margin, margin};
        const V3 bmin = off - ext, bmax = off + ext;
        if ((lf.x < bmin.x && lt.x < bmin.x) || (lf.x > bmax.x && lt.x > bmax.x) || (lf.y < bmin.y && lt.y < bmin.y) ||
            (lf.y > bmax.y && lt.y > bmax.y) || (lf.z < bmin.z && lt.z < bmin.z) || (lf.z > bmax.z && lt.z > bmax.z))
            return false;
        V3 d = lt - lf;
        const float dl = len(d);
        if (!(dl > 0.0f)) return false;
        d = d * (1.0f / dl);
        const float lambda_max = dot(d, lt - lf);
        const float inv[3] = {d.x == 0.0f ? 1.0e30f : 1.0f / d.x, d.y == 0.0f ? 1.0e30f : 1.0f / d.y,
                              d.z == 0.0f ? 1.0e30f : 1.0f / d.z};
        const float from[3] = {lf.x, lf.y, lf.z};
        const float lo[3] = {bmin.x, bmin.y, bmin.z}, hi[3] = {bmax.x, bmax.y, bmax.z};
        float tmin = ((inv[0] < 0.0f ? hi[0] : lo[0]) - from[0]) * inv[0];
        float tmax = ((inv[0] < 0.0f ? lo[0] : hi[0]) - from[0]) * inv[0];
        for (int a = 1; a < 3; ++a) {
            const float t0 = ((inv[a] < 0.0f ? hi[a] : lo[a]) - from[a]) * inv[a];
            const float t1 = ((inv[a] < 0.0f ? lo[a] : hi[a]) - from[a]) * inv[a];
            if (tmin > t1 || t0 > tmax) return false;
            if (t0 > tmin) tmin = t0;
            if (t1 < tmax) tmax = t1;
        }
        if (!(tmin < lambda_max && tmax > 0.0f)) return false;
    }
    const V3 rv{to.x - src.x - (center.x - center.x), to.y - src.y - (center.y - center.y),
                to.z - src.z - (center.z - center.z)};
    bool has = false;
    float dist = 1.0e18f;
    V3 n{0.0f, 0.0f, 0.0f};
    if (!wheel_point_box_closest(src, center, f, rt, u, inner, margin, has, dist, n)) return false;
    float lambda = 0.0f;
    int iter = 0;
    while (true) {
        if (dist <= kRadius) {
            if (-0.0f <= dot(rv, n)) return false;
            break;
        }
        if (++iter > 64) return false;
        const float nl = lambda - dist / dot(rv, n);
        if (nl > 1.0f || nl < 0.0f || nl <= lambda) return false;
        const float s = 1.0f - nl;
        const V3 pa{nl * to.x + s * src.x, nl * to.y + s * src.y, nl * to.z + s * src.z};
        const V3 bo{nl * center.x + s * center.x, nl * center.y + s * center.y, nl * center.z + s * center.z};
        if (!wheel_point_box_closest(pa, bo, f, rt, u, inner, margin, has, dist, n)) return false;
        lambda = nl;
        if (!(0.0f <= dist)) break;
    }
    const float nl2 = len2(n);
    if (!(nl2 > 1.0e-4f) || !(lambda < 1.0f)) return false;
    const float il = 1.0f / sqrtf(nl2);
    const float s = 1.0f - lambda;
    out.t = lambda * max_len;
    out.normal = V3{n.x * il, n.y * il, n.z * il};
    out.point_bt = V3{s * src.x + lambda * to.x, s * src.y + lambda * to.y, s * src.z + lambda * to.z};
    out.hit = 1;
    out.kind = kRayHitCar;
    out.mesh_index = -1;
    return true;
}

// One suspension ray against the arena mesh, the arena's other cars and the ball (reference RayCastWheelAgainstArena,
// :641-845, with CastWheelRayAgainstCars :329-421, on a meshes-only arena).
// The arena-mesh part of a wheel's suspension ray. It reads only the wheel's ray (the car's pose and config), which
// nothing changes between the car's tick start and its vehicle update, so it may run ahead of the update.
RG_HDI void wheel_mesh_ray(const WheelStep& w, const MeshDevice& mesh, float min_hit_dist_sq_bt, RayHit& hit) {
    const float real_ray_length =
        w.suspension_rest_length + w.max_suspension_travel + w.wheel_radius - kWheelSuspensionSubtraction;
    const float real_ray_length_bt = (w.suspension_rest_length * kUuToBt + w.wheel_radius * kUuToBt) +
                                     (w.max_suspension_travel - kWheelSuspensionSubtraction) * kUuToBt;
    hit.hit = 0;
    hit.t = 0.0f;
    hit.point_bt = hit.normal = V3{0.0f, 0.0f, 0.0f};
    hit.kind = kRayHitUnknown;
    hit.mesh_index = -1;
    {
        const float max_len_bt = real_ray_length_bt > 0.0f ? real_ray_length_bt : real_ray_length * kUuToBt;
        const V3 delta = w.wheel_dir_ws * max_len_bt;
        const V3 to = w.ray_source_bt + delta;
        float min_fraction_sq = 0.0f;
        if (min_hit_dist_sq_bt > 0.0f) min_fraction_sq = min_hit_dist_sq_bt / len2(to - w.ray_source_bt);
        float d = 0.0f, dist_a = 0.0f;
        const DevTri* t = nullptr;
        if (real_ray_length > 0.0f && mesh.tri_count > 0 &&
            mesh_ray_cast(mesh, w.ray_source_bt, to, min_fraction_sq, d, t, dist_a)) {
            const V3 n = cross(t->b - t->a, t->c - t->a);
            const float l2 = len2(n);
            V3 normal = l2 <= 1e-12f ? t->normal : n * (1.0f / sqrtf(l2));
            if (dist_a <= 0.0f) normal = -normal;
            hit.hit = 1;
            hit.t = d * real_ray_length;
            hit.point_bt = (1.0f - d) * w.ray_source_bt + d * to;
            hit.normal = normal;
            hit.kind = kRayHitArenaMesh;
            hit.mesh_index = 0;
        }
    }
}

// The closest of the other cars' boxes a wheel's suspension ray hits (best.hit = 0: none), skipping the cars the
// broadphase excludes and demolished ones. It reads only the cars' poses, configs and demolition flags.
RG_HDI void wheel_ray_vs_cars(const WheelStep& w, float min_hit_dist_sq_bt, const WheelOthers& oth, RayHit& best,
                              int& best_idx, bool& best_nr) {
    const float real_ray_length =
        w.suspension_rest_length + w.max_suspension_travel + w.wheel_radius - kWheelSuspensionSubtraction;
    const float real_ray_length_bt = (w.suspension_rest_length * kUuToBt + w.wheel_radius * kUuToBt) +
                                     (w.max_suspension_travel - kWheelSuspensionSubtraction) * kUuToBt;
    best.hit = 0;
    best.t = 0.0f;
    best_idx = -1;
    best_nr = false;
    for (int i = 0; i < oth.count; ++i) {
        if (i == oth.self || ((oth.excluded >> (i + 1)) & 1u)) continue;
        const CarState& o = oth.cars[i];
        if (o.is_demoed) continue;
        {
            const CarConfig& ocfg = oth.cfgs[i];
            const float reach = 0.5f * (fabs_(ocfg.hitbox_size.x) + fabs_(ocfg.hitbox_size.y) +
                                        fabs_(ocfg.hitbox_size.z)) +
                                fabs_(ocfg.hitbox_offset.x) + fabs_(ocfg.hitbox_offset.y) + fabs_(ocfg.hitbox_offset.z);
            const float rr = reach * kUuToBt + real_ray_length_bt + 1.0e-2f;
            if (len2(o.pos_bt - w.ray_source_bt) > rr * rr) continue;
        }
        RayHit h;
        if (!wheel_ray_vs_car_box(w.ray_source_bt, w.wheel_dir_ws, real_ray_length, real_ray_length_bt, o, oth.cfgs[i],
                                  h))
            continue;
        if (min_hit_dist_sq_bt > 0.0f && len2(h.point_bt - w.ray_source_bt) < min_hit_dist_sq_bt) continue;
        if (!best.hit || h.t < best.t) {
            best = h;
            best_idx = i;
            best_nr = o.demo_no_contact_response != 0;
        }
    }
}

// A wheel's suspension ray against the arena mesh (or its result `mesh_hit`, cast ahead by wheel_mesh_ray), the
// other cars' boxes and the ball; the closest hit becomes the wheel's contact.
RG_HDI void wheel_ray_cast(const CarState& c, WheelStep& w, const BallState& ball, const TickConfig& tc,
                           const MeshDevice& mesh, float min_hit_dist_sq_bt, const WheelOthers& oth,
                           const RayHit* mesh_hit = nullptr) {
    const float real_ray_length =
        w.suspension_rest_length + w.max_suspension_travel + w.wheel_radius - kWheelSuspensionSubtraction;
    const float real_ray_length_bt = (w.suspension_rest_length * kUuToBt + w.wheel_radius * kUuToBt) +
                                     (w.max_suspension_travel - kWheelSuspensionSubtraction) * kUuToBt;
    RayHit hit;
    if (mesh_hit) {
        hit = *mesh_hit;
    } else {
        wheel_mesh_ray(w, mesh, min_hit_dist_sq_bt, hit);
    }
    bool hit_world = hit.hit != 0;
    int32_t ground_car_idx = -1;
    bool selected_no_response = false;
    if (oth.cars) {
        RayHit best;
        int best_idx = -1;
        bool best_nr = false;
        wheel_ray_vs_cars(w, min_hit_dist_sq_bt, oth, best, best_idx, best_nr);
        if (best.hit && (!hit.hit || best.t < hit.t)) {
            hit = best;
            hit_world = false;
            ground_car_idx = best_idx;
            selected_no_response = best_nr;
        }
    }
    if (!(oth.excluded & 1u)) {
        RayHit bh;
        if (wheel_ray_vs_ball(w.ray_source_bt, w.wheel_dir_ws, real_ray_length, ball, tc.ball_radius,
                              real_ray_length_bt, bh)) {
            const bool too_close = min_hit_dist_sq_bt > 0.0f && len2(bh.point_bt - w.ray_source_bt) < min_hit_dist_sq_bt;
            if (!too_close && (!hit.hit || bh.t < hit.t)) {
                hit = bh;
                ground_car_idx = -1;
                hit_world = false;
                selected_no_response = false;
            }
        }
    }
    if (selected_no_response) {
        hit.hit = 0;
        hit_world = false;
        ground_car_idx = -1;
    }
    const V3 car_up = -w.wheel_dir_ws;
    if (hit.hit) {
        w.contact_point_bt = hit.point_bt;
        w.contact_normal_ws = hit.normal;
        w.is_in_contact = 1;
        w.is_in_contact_with_world = hit_world ? 1 : 0;
        w.ground_kind = hit.kind;
        w.ground_car_idx = ground_car_idx;
        w.ground_static_id = hit_world ? hit.mesh_index : -1;
        const float trace_len_bt = dot(w.ray_source_bt - hit.point_bt, car_up);
        const float radius_bt = w.wheel_radius * kUuToBt;
        w.wheel_trace_len_bt = trace_len_bt;
        w.suspension_len_bt = trace_len_bt - radius_bt;
        wheel_ray_velocity_terms(c, car_up, hit.point_bt, w);
    } else {
        wheel_ray_miss(w);
    }
}

// Push-back of a wheel pressed into the world (reference SetWorldWheelPushback, :2050-2072, with
// ResolveStaticCollisionImpulseMagnitudeBtInputs / BodyImpulseDenominatorBt, host_validation_and_contact_debug.hpp:
// 394-459).
RG_HDI void world_wheel_pushback(const CarState& c, const TickConfig& tc, WheelStep& w, const CarFrame& f) {
    const float solver_dt = 1.0f / 60.0f;
    const float thresh = (w.suspension_rest_length * kUuToBt + w.wheel_radius * kUuToBt) -
                         kWheelSuspensionSubtraction * kUuToBt;
    const float trace = w.wheel_trace_len_bt;
    if (trace < thresh) {
        const float distance_bt = trace - thresh;
        const V3 rel_bt = w.contact_point_bt - c.pos_bt;
        const V3 vel_at_contact_bt = c.vel_bt + cross(c.ang_vel, rel_bt);
        const float rel_vel_bt = dot(w.contact_normal_ws, vel_at_contact_bt);
        const V3 rel2 = w.contact_point_bt - c.pos_bt;
        const V3 c0 = cross(rel2, w.contact_normal_ws);
        const V3 ang = vec_mul3x3(c0, f.inv_w0, f.inv_w1, f.inv_w2);
        const float denom = 1.0f / tc.car_mass + dot(w.contact_normal_ws, cross(ang, rel2));
        float impulse = 0.0f;
        if (!(denom <= 0.0f || solver_dt <= 0.0f)) {
            const float jac = 1.0f / denom;
            const float positional_error_bt = 0.2f * -distance_bt / solver_dt;
            const float velocity_error_bt = -rel_vel_bt;
            const float normal_impulse = positional_error_bt * jac + velocity_error_bt * jac;
            impulse = normal_impulse > 0.0f ? normal_impulse : 0.0f;
        }
        w.extra_pushback = impulse / 4.0f;
    }
}

// ---- drive (reference :1501-1535, 1697-1796) ----------------------------------------------------------------------
RG_HDI V3 wheel_steered_right_col(const WheelStep& w, float steer_angle) {
    const V3 up = -w.wheel_dir_ws;
    const V3 right = w.wheel_axle_ws;
    const float half_angle = steer_angle * 0.5f;
    const float sin_scale = (half_angle == 0.0f && len2(up) > 0.0f) ? half_angle : (game_sinf(half_angle) / len(up));
    const float cos_half = (half_angle == 0.0f) ? 1.0f : game_cosf(half_angle);
    const Q4 q{cos_half, up.x * sin_scale, up.y * sin_scale, up.z * sin_scale};
    const float s = 2.0f / (((q.x * q.x + q.y * q.y) + q.z * q.z) + q.w * q.w);
    const float xs = q.x * s, ys = q.y * s, zs = q.z * s;
    const float wx = q.w * xs, wy = q.w * ys, wz = q.w * zs;
    const float xx = q.x * xs, xy = q.x * ys, xz = q.x * zs;
    const float yy = q.y * ys, yz = q.y * zs, zz = q.z * zs;
    const V3 c0{1.0f - (yy + zz), xy + wz, xz - wy};
    const V3 c1{xy - wz, 1.0f - (xx + zz), yz + wx};
    const V3 c2{xz + wy, yz - wx, 1.0f - (xx + yy)};
    const V3 nr = -right;
    return V3{c0.x * nr.x + c1.x * nr.y + c2.x * nr.z, c0.y * nr.x + c1.y * nr.y + c2.y * nr.z,
              c0.z * nr.x + c1.z * nr.y + c2.z * nr.z};
}
struct DriveShared {
    V3 front_right_col, back_right_col;
    float next_steer_angle, drive_engine_force, drive_brake_force, real_throttle, friction_scale;
};
RG_HDI void wheel_drive_setup(const CarState& c, const DriveShared& s, WheelStep& w, int i, WheelRuntime& wr,
                              float dt) {
    const float prev_lat = wr.lat_friction[i];
    const float prev_long = wr.long_friction[i];
    const float steer = w.is_front_wheel ? s.next_steer_angle : 0.0f;
    wr.engine_force[i] = s.drive_engine_force;
    wr.brake[i] = s.drive_brake_force;
    wr.steer_angle[i] = steer;
    float lat = prev_lat, lng = prev_long;
    V3 right_col{0.0f, 0.0f, 0.0f};
    if (w.is_in_contact) {
        right_col = w.is_front_wheel ? s.front_right_col : s.back_right_col;
        const V3 wheel_delta_bt = w.ray_source_bt - c.pos_bt;
        const V3 cv = (cross(c.ang_vel, wheel_delta_bt) + c.vel_bt) * 50.0f;
        const V3 long_dir = cross(right_col, w.contact_normal_ws);
        const float base_friction = fabs_(dot(cv, right_col));
        const float longitudinal = fabs_(dot(cv, long_dir));
        float curve_input = 0.0f;
        if (base_friction > 5.0f) curve_input = base_friction / (longitudinal + base_friction);
        lat = lat_friction_curve(curve_input);
        lng = 1.0f;
        if (c.handbrake_val > 0.0f) {
            lat *= (0.1f - 1.0f) * c.handbrake_val + 1.0f;
            lng *= (handbrake_long_friction_factor(curve_input) - 1.0f) * c.handbrake_val + 1.0f;
        } else {
            lng = 1.0f;
        }
        const bool sticky = s.real_throttle != 0.0f && w.is_in_contact_with_world;
        if (!sticky) {
            const float ns = non_sticky_friction_factor(w.contact_normal_ws.z);
            lat *= ns;
            lng *= ns;
        }
    }
    wr.lat_friction[i] = lat;
    wr.long_friction[i] = lng;
    if (!w.is_in_contact) return;
    const V3 cc = cross(w.contact_normal_ws, right_col);
    const V3 forward_dir = cc * (1.0f / sqrtf(len2(cc)));
    float rolling = 0.0f;
    if (s.drive_engine_force == 0.0f) {
        if (s.drive_brake_force != 0.0f) {
            const V3 rel = w.contact_point_bt - c.pos_bt;
            const V3 cvel = c.vel_bt + cross(c.ang_vel, rel);
            float rel_vel = dot(cvel, forward_dir);
            if (dt > (1.0f / 80.0f)) {
                const float threshold = -(1.0f / (dt * 150.0f)) + 0.8f;
                if (fabs_(rel_vel) < threshold) rel_vel = 0.0f;
            }
            const float v = -rel_vel * 113.73963f;
            const float b = s.drive_brake_force;
            rolling = (v < -b ? -b : (v > b ? b : v)) * (dt * s.friction_scale);
        }
    } else {
        rolling = -s.drive_engine_force * dt;
    }
    w.cal_axle_dir = right_col;
    w.cal_forward_dir = forward_dir;
    w.cal_rolling_friction = rolling;
    w.cal_lat_friction = lat;
    w.cal_long_friction = lng;
    w.cal_friction_scale = s.friction_scale;
}

// ---- suspension and tyre impulses (reference :1089-1300, 1475-1499) ------------------------------------------------
struct WheelImpulse {
    V3 dv_bt, dw;
    bool applied;
};
RG_HDI WheelImpulse wheel_impulse_at(float mass, const CarFrame& f, V3 impulse_bt, V3 rel_bt) {
    WheelImpulse o;
    o.dv_bt = impulse_bt * (1.0f / mass);
    const V3 torque_bt = cross(rel_bt, impulse_bt);
    o.dw = V3{dot(f.inv_w0, torque_bt), dot(f.inv_w1, torque_bt), dot(f.inv_w2, torque_bt)};
    o.applied = true;
    return o;
}
RG_HDI void combine_wheel_impulses(CarState& c, const WheelImpulse* o) {
    V3 vel_bt = c.vel_bt;
    V3 ang_vel = c.ang_vel;
    bool any = false;
    for (int k = 0; k < 4; ++k) {
        const int i = k ^ 1;
        if (!o[i].applied) continue;
        vel_bt = vel_bt + o[i].dv_bt;
        ang_vel += o[i].dw;
        any = true;
    }
    if (any) {
        car_set_vel_bt(c, vel_bt);
        c.vel_touched_solve_stage = 1;
        c.ang_vel = ang_vel;
    }
}
RG_HDI void wheel_suspension_and_friction(CarState& c, const TickConfig& tc, WheelStep* wh, const CarFrame& f) {
    if (!(wh[0].is_in_contact || wh[1].is_in_contact || wh[2].is_in_contact || wh[3].is_in_contact)) return;
    const float dt = tc.tick_dt;
    WheelImpulse o[4];
    for (int i = 0; i < 4; ++i) {
        WheelStep& w = wh[i];
        o[i].applied = false;
        if (!w.is_in_contact) continue;
        const float force_bt = (w.suspension_rest_length * kUuToBt - w.suspension_len_bt) *
                               kWheelSuspensionStiffness * w.clipped_inv_contact_dot_suspension;
        const float damping =
            w.suspension_relative_velocity < 0.0f ? kWheelDampingCompression : kWheelDampingRelaxation;
        float susp = (force_bt - damping * w.suspension_relative_velocity_bt) * w.suspension_force_scale;
        if (susp < 0.0f) susp = 0.0f;
        if (susp * 50.0f > 0.0f) {
            const V3 rel_bt = w.contact_point_bt - c.pos_bt;
            const float scale = (susp * dt) + w.extra_pushback;
            o[i] = wheel_impulse_at(tc.car_mass, f, w.contact_normal_ws * scale, rel_bt);
        }
    }
    combine_wheel_impulses(c, o);
    // the bilateral body after the suspension impulses (reference MakeBilateralCarBodyBt)
    const V3 com = c.pos_bt, lin = c.vel_bt, ang = c.ang_vel;
    const float inv_mass = tc.car_mass != 0.0f ? 1.0f / tc.car_mass : 0.0f;
    for (int i = 0; i < 4; ++i) {
        WheelStep& w = wh[i];
        o[i].applied = false;
        if (!w.is_in_contact) continue;
        float side_impulse = 0.0f;
        {
            const V3 rel_pos1 = w.contact_point_bt - com;
            const V3 vel = lin + cross(ang, rel_pos1);
            const V3 cj = cross(rel_pos1, w.cal_axle_dir);
            const V3 a_j{dot(f.fwd, cj), dot(f.right, cj), dot(f.up, cj)};
            const V3 minv{f.inv_inertia_local_bt.x * a_j.x, f.inv_inertia_local_bt.y * a_j.y,
                          f.inv_inertia_local_bt.z * a_j.z};
            const float a_diag = inv_mass + dot(minv, a_j);
            const float rel_vel = dot(w.cal_axle_dir, vel);
            if (!(a_diag <= 0.0f)) side_impulse = -0.2f * rel_vel * (1.0f / a_diag);
        }
        const float roll = w.cal_rolling_friction * w.cal_long_friction;
        const float side = (side_impulse * (dt * w.cal_friction_scale)) * w.cal_lat_friction;
        const V3 imp{roll * w.cal_forward_dir.x + side * w.cal_axle_dir.x,
                     roll * w.cal_forward_dir.y + side * w.cal_axle_dir.y,
                     roll * w.cal_forward_dir.z + side * w.cal_axle_dir.z};
        if (len2(imp) == 0.0f) continue;
        const V3 car_up = f.up;
        const V3 rel = w.contact_point_bt - c.pos_bt;
        const V3 wheel_rel = rel - car_up * dot(car_up, rel);
        o[i] = wheel_impulse_at(tc.car_mass, f, imp, wheel_rel);
    }
    combine_wheel_impulses(c, o);
}

// ---- auto-roll (reference ApplyAutoRollReference, :1021-1087) ------------------------------------------------------
RG_HDI void queue_first_force_and_torque(CarFrame& f, V3 force_bt, V3 torque_bt) {
    if (f.n_force_items > 4 || f.n_torque_items > 4) {
        queue_force(f, force_bt);
        queue_torque(f, torque_bt);
        return;
    }
    V3 force = force_bt;
    for (int k = 0; k < f.n_force_items; ++k) force += f.force_items[k];
    V3 torque = torque_bt;
    for (int k = 0; k < f.n_torque_items; ++k) torque += f.torque_items[k];
    f.queued_force = force;
    f.queued_torque_bt = torque;
    f.n_force_items = 5;
    f.n_torque_items = 5;
}
RG_HDI void apply_auto_roll(const CarState& c, const CarConfig& cfg, const TickConfig& tc, int contacts,
                            V3 normal_sum, CarFrame& f) {
    const V3 ground_up = contacts > 0 ? (len2(normal_sum) >= 1e-8f ? normal_sum * (1.0f / sqrtf(len2(normal_sum)))
                                                                   : V3{0.0f, 0.0f, 0.0f})
                                      : c.world_contact.contact_normal;
    const V3 ground_down = -ground_up;
    const V3 force_bt = ((ground_down * 100.0f) * kUuToBt) * tc.car_mass;
    V3 F, R, U;
    ue_quat_axes(c.rot, F, R, U);
    const V3& G = ground_up;
    const float crx = F.z * G.y - F.y * G.z;
    const float cry = F.x * G.z - F.z * G.x;
    const float crz = F.y * G.x - F.x * G.y;
    auto clamp01 = [](float v) { return 0.0f <= v ? (1.0f <= v ? 1.0f : v) : 0.0f; };
    const float r_dot = clamp01((crx * R.x + R.y * cry) + R.z * crz);
    const float nx = -G.x, ny = -G.y, nz = -G.z;
    const float f_dot =
        clamp01(((ny * crz - nz * cry) * F.x + (crx * nz - nx * crz) * F.y) + (nx * cry - crx * ny) * F.z);
    const V3 f_axis = 0.0f <= (R.y * G.y + R.x * G.x) + R.z * G.z ? V3{-F.x, -F.y, -F.z} : F;
    const V3 r_axis = (F.y * G.y + F.x * G.x) + F.z * G.z < 0.0f ? V3{-R.x, -R.y, -R.z} : R;
    const float rf = (1.0f - r_dot) * 80.0f;
    const float ff = (1.0f - f_dot) * 80.0f;
    const V3 t_game{ff * r_axis.x + rf * f_axis.x, ff * r_axis.y + rf * f_axis.y, ff * r_axis.z + rf * f_axis.z};
    V3 i0, i1, i2;
    frame_inertia(&f, c, cfg, tc.car_mass, i0, i1, i2);
    queue_first_force_and_torque(f, force_bt, mul3x3(i0, i1, i2, t_game));
}

// ---- flip torque, air control, jump (reference :3042-3241, 3399-3484, 3629-3652) ------------------------------------
RG_HDI V3 flip_torque(CarState& c, const CarControls& k, const CarConfig& cfg, const TickConfig& tc, float raw_pitch,
                      const CarFrame& f) {
    if (c.is_flipping) c.is_flipping = (c.has_flipped && c.internal_flip_time < tc.flip_torque_time) ? 1 : 0;
    if (!c.is_flipping) return V3{0.0f, 0.0f, 0.0f};
    const V3 rel = c.flip_rel_torque;
    float torque_y = rintf(rel.y * tc.flip_torque_y);
    float cancel_raw;
    {
        const float pitch = raw_pitch <= 1.0f ? raw_pitch : k.pitch;
        cancel_raw = c.internal_flip_time >= 0.041f ? pitch : 0.0f;
    }
    const float cancel_pitch = -quantize_axis(-cancel_raw);
    if (rel.y != 0.0f && cancel_pitch != 0.0f && sgnf(rel.y) == sgnf(cancel_pitch))
        torque_y *= (1.0f - fmin_(fabs_(cancel_pitch), 1.0f));
    const V3 t{rintf(rel.x * tc.flip_torque_x), torque_y, 0.0f};
    V3 uf, ur, uu;
    ue_quat_axes(c.rot, uf, ur, uu);
    const V3 tw{((t.y * ur.x + t.x * uf.x) + t.z * uu.x) + 0.0f * 0.0f,
                ((t.y * ur.y + t.x * uf.y) + t.z * uu.y) + 0.0f * 0.0f,
                ((t.y * ur.z + t.x * uf.z) + t.z * uu.z) + 0.0f * 0.0f};
    constexpr float kGate = 1.0e-4f;
    if (fabs_(tw.x) >= kGate || fabs_(tw.y) >= kGate || fabs_(tw.z) >= kGate) {
        V3 i0, i1, i2;
        frame_inertia(&f, c, cfg, tc.car_mass, i0, i1, i2);
        return mul3x3(i0, i1, i2, tw);
    }
    return V3{0.0f, 0.0f, 0.0f};
}
RG_HDI void air_control(const CarState& c, const CarControls& k, const CarConfig& cfg, const TickConfig& tc,
                        bool update_air_control, bool air_throttle, float pitchlock_restart_time, V3 damp_ang_vel,
                        CarFrame& f) {
    if (!update_air_control && !air_throttle) return;
    V3 ue_f{0.0f, 0.0f, 0.0f};
    bool have_ue_axes = false;
    if (update_air_control) {
        float pitch_scale = 1.0f;
        if (c.is_flipping) {
            pitch_scale = 0.0f;
        } else if (c.has_flipped && c.internal_flip_time < (tc.flip_torque_time + tc.flip_pitchlock_extra_time)) {
            pitch_scale = 0.0f;
        } else if (pitchlock_restart_time >= 0.0f && pitchlock_restart_time < tc.flip_pitchlock_extra_time) {
            pitch_scale = 0.0f;
        }
        V3 ue_r, ue_u;
        ue_quat_axes(c.rot, ue_f, ue_r, ue_u);
        have_ue_axes = true;
        constexpr float kGate = 1.0e-4f;
        const float in_pitch = k.pitch * pitch_scale;
        const float a_p = (tc.car_air_control_pitch * -in_pitch) * kUeRot;
        const float a_y = (tc.car_air_control_yaw * k.yaw) * kUeRot;
        const float a_r = (-tc.car_air_control_roll * k.roll) * kUeRot;
        const V3 t_in{(((a_p * ue_r.x + 0.0f) + a_y * ue_u.x) + a_r * ue_f.x) * 1000.0f,
                      (((a_p * ue_r.y + 0.0f) + a_y * ue_u.y) + a_r * ue_f.y) * 1000.0f,
                      (((a_p * ue_r.z + 0.0f) + a_y * ue_u.z) + a_r * ue_f.z) * 1000.0f};
        const float d_p = (1.0f - fabs_(in_pitch)) * (dot(damp_ang_vel, ue_r) * (tc.car_air_damp_pitch * kUeRot));
        const float d_y = (1.0f - fabs_(k.yaw)) * (dot(damp_ang_vel, ue_u) * (tc.car_air_damp_yaw * kUeRot));
        const float d_r = (1.0f * dot(damp_ang_vel, ue_f)) * (tc.car_air_damp_roll * kUeRot);
        const V3 t_damp{(((0.0f - d_p * ue_r.x) - d_y * ue_u.x) - d_r * ue_f.x) * 1000.0f,
                        (((0.0f - d_p * ue_r.y) - d_y * ue_u.y) - d_r * ue_f.y) * 1000.0f,
                        (((0.0f - d_p * ue_r.z) - d_y * ue_u.z) - d_r * ue_f.z) * 1000.0f};
        const bool apply_in = fabs_(t_in.x) >= kGate || fabs_(t_in.y) >= kGate || fabs_(t_in.z) >= kGate;
        const bool apply_damp = fabs_(t_damp.x) >= kGate || fabs_(t_damp.y) >= kGate || fabs_(t_damp.z) >= kGate;
        if (apply_in || apply_damp) {
            V3 i0, i1, i2;
            frame_inertia(&f, c, cfg, tc.car_mass, i0, i1, i2);
            if (apply_in) queue_torque(f, mul3x3(i0, i1, i2, t_in));
            if (apply_damp) queue_torque(f, mul3x3(i0, i1, i2, t_damp));
        }
    }
    const float input = c.is_boosting ? 1.0f : k.throttle;
    if (input != 0.0f && air_throttle) {
        if (!have_ue_axes) {
            V3 r_, u_;
            ue_quat_axes(c.rot, ue_f, r_, u_);
        }
        const float force = tc.car_air_throttle_accel * tc.car_mass;
        queue_force(f, ((ue_f * force) * input) * kUuToBt);
    }
}
RG_HDI void update_jump_state(CarState& c, const CarControls& k, const TickConfig& tc, CarFrame& f) {
    if (c.is_on_ground && !c.is_jumping) {
        if (!(c.has_jumped && c.internal_jump_time < tc.jump_min_time + tc.jump_reset_time_pad)) {
            c.has_jumped = 0;
            c.internal_jump_time = 0.0f;
        }
    }
    for (int pass = 0; pass < 2; ++pass) {  // UpdateJumpState then ContinueJump test the same condition
        if (c.is_jumping) {
            if (!(c.internal_jump_time < tc.jump_min_time ||
                  (k.jump && !c.jump_hold_broken && c.internal_jump_time < tc.jump_max_time)))
                c.is_jumping = 0;
        }
    }
    if (c.is_jumping) {
        c.has_jumped = 1;
        f.queued_jump_force = game_jump_up_scaled_bt(c, tc.jump_accel * tc.car_mass);
        f.has_queued_jump_force = true;
    }
    if (c.is_jumping || c.has_jumped) c.internal_jump_time += tc.tick_dt;
}

// ---- boost (reference ApplyBoost, :3242-3305) ---------------------------------------------------------------------
RG_HDI void apply_boost(CarState& c, const CarControls& k, const TickConfig& tc, CarFrame& f) {
    const float dt = tc.tick_dt;
    c.rlbotv5_boost_hold = 0;
    if (c.is_demoed) return;  // a demolished car never reaches the vehicle update
    bool push;
    if (c.is_boosting) {
        car_set_boost_amount(c, fmax_(0.0f, car_boost_amount(c) - (tc.boost_used_per_second / 100.0f) * dt));
        const bool latch_expired = !k.boost && c.boosting_time >= tc.boost_min_time;
        push = !(c.boost == 0.0f || latch_expired);
    } else {
        push = k.boost && c.boost > 0.0f;
    }
    c.is_boosting = push ? 1 : 0;
    if (push) {
        const V3 dir = ue_quat_rotate(c.rot, V3{1.0f, 0.0f, 0.0f});
        const float force = tc.boost_accel_ground * tc.car_mass;
        queue_force(f, (force * dir) * kUuToBt);
        c.boosting_time += dt;
        c.time_since_boosted = 0.0f;
    } else {
        c.boosting_time = 0.0f;
        c.time_since_boosted += dt;
        if (tc.recharge_boost_enabled && c.time_since_boosted >= tc.recharge_boost_delay)
            car_set_boost_amount(c, car_boost_amount(c) + (tc.recharge_boost_per_second / 100.0f) * dt);
    }
    if (c.boost < 0.0f || c.boost > tc.boost_max)
        car_set_boost_amount(c, fmin_(fmax_(c.boost, 0.0f), tc.boost_max) / 100.0f);
}

// ---- the vehicle update -------------------------------------------------------------------------------------------
// reference PreTickCar (env_step.hpp:3115-3484) with PreTickVehicleDynamics (raycast_wheels_and_contact_prep.hpp:
// 2618-2953), WheelRayPhase (:2074-2238) and CombineWheelContacts (:2240-2282).
// The contact impulse denominator of a body at a point, inverse inertia applied column-wise (reference
// BodyImpulseDenominatorBt with ApplyInverseBodyInertiaWorldBtColumnDot, host_validation_and_contact_debug.hpp:333-411).
RG_HDI float car_impulse_denominator_bt(const CarState& c, const CarConfig& cfg, float mass, V3 p, V3 n) {
    const V3 rel = p - c.pos_bt;
    const V3 c0 = cross(rel, n);
    V3 r0, r1, r2;
    car_inv_inertia_world_bt(c, cfg, mass, r0, r1, r2);
    const V3 ang{r0.x * c0.x + r1.x * c0.y + r2.x * c0.z, r0.y * c0.x + r1.y * c0.y + r2.y * c0.z,
                 r0.z * c0.x + r1.z * c0.y + r2.z * c0.z};
    return 1.0f / mass + dot(n, cross(ang, rel));
}
RG_HDI float car_car_wheel_pushback(const CarState& c, const CarConfig& cfg, const CarState& o, const CarConfig& ocfg,
                                    float mass, V3 p, V3 n, float distance_bt, float dt) {
    const V3 v1 = c.vel_bt + cross(c.ang_vel, p - c.pos_bt);
    const V3 v2 = o.vel_bt + cross(o.ang_vel, p - o.pos_bt);
    const float rel = dot(n, v1 - v2);
    const float d0 = car_impulse_denominator_bt(c, cfg, mass, p, n);
    const float d1 = car_impulse_denominator_bt(o, ocfg, mass, p, n);
    if (dt <= 0.0f || d0 + d1 <= 0.0f) return 0.0f;
    const float jac = 1.0f / (d0 + d1);
    const float imp = (0.2f * -distance_bt / dt) * jac + -rel * jac;
    return imp > 0.0f ? imp : 0.0f;
}
RG_HDI void car_impulse_at_point_bt(CarState& c, const CarConfig& cfg, float mass, V3 impulse, V3 rel) {
    car_set_vel_bt(c, c.vel_bt + impulse * (1.0f / mass));
    c.vel_touched_solve_stage = 1;
    const V3 torque = cross(rel, impulse);
    V3 r0, r1, r2;
    car_inv_inertia_world_bt(c, cfg, mass, r0, r1, r2);
    c.ang_vel = c.ang_vel + V3{dot(r0, torque), dot(r1, torque), dot(r2, torque)};
}

// Wheel rays that landed on the ball this tick, in the car's wheel order: each pushes the ball down along the hit
// normal. Nothing else in a car's vehicle update reads the ball's velocity, so the pushes are recorded and applied
// afterwards in the arena's car order, which keeps the reference's floating-point order (reference WheelRayPhase,
// raycast_wheels_and_contact_prep.hpp:2200-2207) while the cars' updates run independently.
struct WheelBallPushes {
    int32_t count;
    V3 point_bt[4], normal[4];
    // the update's car-world event (a wheel newly on the arena, when events are on), which the arena emits in the
    // game's car order: its normal, and the car's position, velocity and ground flag after the update
    uint32_t world_event;
    uint8_t world_event_on_ground;
    V3 world_event_normal, world_event_pos, world_event_vel;
};
RG_HDI void apply_wheel_ball_pushes(BallState& ball, const WheelBallPushes& p, const TickConfig& tc) {
    for (int k = 0; k < p.count; ++k) {
        ball.sleeping |= 4u;
        const V3 push_bt = -p.normal[k];
        ball.vel_bt = ball.vel_bt + push_bt * (1.0f / tc.ball_mass);
        ball.vel = ball.vel_bt * 50.0f;
        ball.ang_vel = ball.ang_vel + ball_inv_inertia_bt(ball, tc.ball_mass, tc.ball_radius,
                                                          cross(p.point_bt[k] - ball.pos_bt, push_bt));
    }
}

// The update's car-world event: the wheel on the arena with the most upward normal, unless a wheel stood on the same
// triangle with the same normal last tick (reference PreTickCar, env_step.hpp:3426-3469). Kept out of line: only a
// batch with an event stream calls it.
RG_NOINL void wheel_world_event(const CarState& c, const WheelRuntime& wr, const WheelStep* wh,
                                WheelBallPushes& pushes) {
    bool has = false;
    V3 normal{0.0f, 0.0f, 0.0f};
    int32_t id = -1;
    for (int i = 0; i < 4; ++i) {
        if (wh[i].is_in_contact && wh[i].is_in_contact_with_world && (!has || wh[i].contact_normal_ws.z > normal.z)) {
            has = true;
            normal = wh[i].contact_normal_ws;
            id = wh[i].ground_static_id;
        }
    }
    bool previous = false;
    if (has && c.tick_count_since_update != 0) {
        for (int i = 0; i < 4; ++i) {
            const V3 old = wr.event_world_normals[i];
            previous = previous || (wr.event_world_ids[i] == id && old.x == normal.x && old.y == normal.y &&
                                    old.z == normal.z);
        }
    }
    pushes.world_event = has && !previous ? 1u : 0u;
    pushes.world_event_normal = normal;
    pushes.world_event_pos = c.pos;
    pushes.world_event_vel = c.vel;
    pushes.world_event_on_ground = c.is_on_ground;
}

// `mesh_hits`: the four wheels' arena-mesh rays cast ahead (wheel_mesh_ray_ahead), or null to cast them here.
RG_NOINL void vehicle_update(CarState& c, CarControls k_raw, const CarConfig& cfg, const TickConfig& tc,
                           WheelRuntime& wr, const BallState& ball, const MeshDevice& mesh, const WheelOthers& oth,
                           WheelBallPushes& pushes, const RayHit* mesh_hits = nullptr) {
    pushes.count = 0;
    pushes.world_event = 0u;
    const float dt = tc.tick_dt;
    c.demo_no_contact_response = c.is_demoed ? 1 : 0;
    if (c.is_demoed) return;
    float raw_pitch = 2.0f;
    const CarControls k = pre_tick_controls(c, k_raw, raw_pitch);
    const uint8_t cal_pre = c.cal_pre_flags;
    CarFrame f;
    make_car_frame(f, c, cfg, tc.car_mass);
    f.queue_forces = true;
    wr.pre_solve_rot = c.rot;
    wr.pre_solve_basis_forward = c.tick_start_basis_forward;
    wr.pre_solve_basis_right = c.tick_start_basis_right;
    wr.pre_solve_basis_up = c.tick_start_basis_up;
    wr.pre_solve_basis_authoritative = 1;
    const uint8_t flipping_at_start = (cal_pre & kCalPreFlippingAtStart) ? 1 : 0;
    const bool flip_started = (cal_pre & kCalPreFlipStarted) != 0;
    const float pitchlock_restart_time = c.cal_pre_pitchlock_restart_time;
    const bool air_jump_started = (cal_pre & kCalPreAirJumpStarted) != 0;
    const uint8_t was_jumping = (cal_pre & kCalPreWasJumping) ? 1 : 0;
    float forward_speed_uu = c.cal_pre_forward_speed_uu;
    const uint8_t air_jump_used_before = (cal_pre & kCalPreAirJumpUsedBefore) ? 1 : 0;
    const bool set_v3_tick = (cal_pre & kCalPreSetV3Tick) != 0;
    const int prev_wheel_contacts = (c.wheels_with_contact[0] != 0) + (c.wheels_with_contact[1] != 0) +
                                    (c.wheels_with_contact[2] != 0) + (c.wheels_with_contact[3] != 0);
    const bool autoroll_prev_contact = c.tick_count_since_update != 0;
    V3 autoroll_normal_sum = autoroll_prev_contact ? wr.cal_prev_wheel_normal_sum : V3{0.0f, 0.0f, 0.0f};
    int autoroll_world_contacts = autoroll_prev_contact ? wr.cal_prev_world_wheel_contacts : 0;

    // -- PreTickVehicleDynamics
    WheelStep wh[4];
    int num_contact = 0;
    bool wheel_world_contact = false;
    float abs_snapshot_forward_speed;
    {
        c.world_contact.wheel_ball_mask = 0;
        const uint8_t sticky_prev_world_contacts = wr.cal_prev_world_wheel_contacts;
        const V3 sticky_prev_world_normal_sum = wr.cal_prev_wheel_normal_sum;
        float front_scale, back_scale, front_bone, back_bone;
        suspension_force_scales(cfg, tc.car_mass, front_scale, back_scale);
        const float min_hit_dist_sq = min_wheel_hit_dist_sq_bt(cfg);
        wheel_bone_z(cfg, front_bone, back_bone);
        uint32_t flags[4];
        for (int kk = 0; kk < 4; ++kk) {
            const int i = kk ^ 1;
            WheelStep& w = wh[i];
            init_wheel(w, c, cfg, i, f, i < 2 ? front_bone : back_bone);
            w.suspension_force_scale = w.is_front_wheel ? front_scale : back_scale;
            w.extra_pushback = wr.extra_pushback[i];
            wheel_ray_cast(c, w, ball, tc, mesh, min_hit_dist_sq, oth, mesh_hits ? mesh_hits + i : nullptr);
            if (w.is_in_contact) w.extra_pushback = 0.0f;
            if (w.is_in_contact_with_world) world_wheel_pushback(c, tc, w, f);
            if (w.is_in_contact && !w.is_in_contact_with_world && w.ground_kind == kRayHitCar && oth.cars &&
                w.ground_car_idx >= 0 && w.ground_car_idx < oth.count && w.ground_car_idx != oth.self) {
                // a wheel on another car pushes that car down (and back out when pressed in) at once (reference
                // WheelRayPhase, :2196-2219; ResolveCarCarWheelPushbackMagnitudeBtInputs, ApplyImpulseAtPointBt-
                // RoundtripBtInputs, host_validation_and_contact_debug.hpp:413-482)
                CarState& o = oth.cars[w.ground_car_idx];
                const CarConfig& ocfg = oth.cfgs[w.ground_car_idx];
                const V3 n_bt = w.contact_normal_ws, cp_bt = w.contact_point_bt;
                const float solver_dt = 1.0f / 60.0f;
                const float thresh = (w.suspension_rest_length * kUuToBt + w.wheel_radius * kUuToBt) - 0.05f;
                w.extra_pushback = 0.0f;
                if (w.wheel_trace_len_bt < thresh)
                    w.extra_pushback = car_car_wheel_pushback(c, cfg, o, ocfg, tc.car_mass, cp_bt, n_bt,
                                                              w.wheel_trace_len_bt - thresh, solver_dt) /
                                       4.0f;
                if (w.extra_pushback > 0.0f) {
                    const float full = w.extra_pushback * 4.0f;
                    car_impulse_at_point_bt(o, ocfg, tc.car_mass, -n_bt * full, cp_bt - o.pos_bt);
                }
                car_impulse_at_point_bt(o, ocfg, tc.car_mass, -n_bt, cp_bt - o.pos_bt);
            } else if (w.is_in_contact && !w.is_in_contact_with_world && w.ground_kind == kRayHitBall) {
                // the ray pushes the ball down (reference WheelRayPhase, :2200-2207); the caller applies the push in
                // the arena's car order (apply_wheel_ball_pushes)
                pushes.point_bt[pushes.count] = w.contact_point_bt;
                pushes.normal[pushes.count] = w.contact_normal_ws;
                ++pushes.count;
            }
            wr.extra_pushback[i] = w.extra_pushback;
            flags[i] = (w.is_in_contact ? 1u : 0u) | (w.is_in_contact_with_world ? 2u : 0u) |
                       (w.ground_kind == kRayHitBall ? 4u : 0u);
        }
        // CombineWheelContacts
        V3 world_normal_sum{0.0f, 0.0f, 0.0f};
        int world_contacts = 0;
        for (int kk = 0; kk < 4; ++kk) {
            const int i = kk ^ 1;
            const bool in_contact = (flags[i] & 1u) != 0;
            c.wheels_with_contact[i] = in_contact;
            c.world_contact.wheel_ball_mask |= static_cast<uint8_t>((in_contact && (flags[i] & 4u)) << i);
            num_contact += in_contact ? 1 : 0;
        }
        c.is_on_ground = num_contact >= 3 ? 1 : 0;
        for (int kk = 0; kk < 4; ++kk) {
            const int i = kk ^ 1;
            if ((flags[i] & 1u) && (flags[i] & 2u)) {
                world_normal_sum += wh[i].contact_normal_ws;
                ++world_contacts;
            }
        }
        wr.cal_prev_wheel_normal_sum = world_normal_sum;
        wr.cal_prev_world_wheel_contacts = static_cast<uint8_t>(world_contacts);
        wheel_world_contact = world_contacts > 0;

        abs_snapshot_forward_speed = fabs_(forward_speed_uu);
        {
            // FreshCarRbSnapshot (:940-988)
            V3 v = c.vel_bt * 50.0f;
            const float l2 = (v.y * v.y + v.x * v.x) + v.z * v.z;
            if (tc.car_max_speed > 0.0f && tc.car_max_speed * tc.car_max_speed < l2) {
                const float inv = 1.0f / sqrtf(l2);
                v = V3{tc.car_max_speed * (inv * v.x), tc.car_max_speed * (inv * v.y), tc.car_max_speed * (inv * v.z)};
            }
            const V3 snap_vel{quant_trunc_offset(v.x, 100.0f), quant_trunc_offset(v.y, 100.0f),
                              quant_trunc_offset(v.z, 100.0f)};
            const Q4 snap_rot = game_quantize_quat(game_rot_from_basis(f.fwd, f.right, f.up));
            forward_speed_uu = snapshot_forward_speed(snap_rot, snap_vel);
        }
        const float abs_forward_speed = fabs_(forward_speed_uu);
        const float friction_scale = tc.car_mass / 3.0f;
        if (k.handbrake) {
            c.handbrake_val = clampf(c.handbrake_val + 5.0f * dt, 0.0f, 1.0f);
        } else {
            c.handbrake_val = clampf(c.handbrake_val - 2.0f * dt, 0.0f, 1.0f);
        }
        const float real_throttle = k.throttle;
        float real_brake = 0.0f;
        float engine_throttle = c.driving_disabled ? 0.0f : real_throttle;
        if (!k.handbrake && !c.driving_disabled) {
            const float abs_throttle = fabs_(real_throttle);
            if (abs_throttle > 0.01f) {
                if (abs_forward_speed > 25.0f && sgnf(real_throttle) != sgnf(forward_speed_uu)) {
                    real_brake = 1.0f;
                    if (abs_forward_speed > 0.01f) engine_throttle = 0.0f;
                }
            } else {
                engine_throttle = 0.0f;
                real_brake = abs_forward_speed < 25.0f ? 1.0f : 0.15f;
            }
        }
        const float drive_speed_scale = engine_throttle != 0.0f ? drive_torque_factor(forward_speed_uu) : 1.0f;
        float engine_uu = (drive_speed_scale * (engine_throttle * 288000.0f)) * 0.25f;
        if (num_contact < 3) engine_uu *= 0.25f;
        DriveShared ds;
        ds.drive_engine_force = engine_uu * kUuToBt;
        ds.drive_brake_force = ((real_brake * 10500.0f) * 0.25f) * kUuToBt;
        {
            float steer_deg = steer_angle_from_speed(cfg.steer_angle_curve_deg, abs_forward_speed);
            if (c.handbrake_val > 0.0f)
                steer_deg +=
                    (powerslide_steer_angle_from_speed(cfg.powerslide_steer_angle_curve_deg, abs_forward_speed) -
                     steer_deg) *
                    c.handbrake_val;
            ds.next_steer_angle = (steer_deg * k.steer) * kSteerDegToRad;
        }
        ds.real_throttle = real_throttle;
        ds.friction_scale = friction_scale;
        ds.front_right_col = ds.back_right_col = V3{0.0f, 0.0f, 0.0f};
        const bool front_in = wh[0].is_in_contact || wh[1].is_in_contact;
        const bool back_in = wh[2].is_in_contact || wh[3].is_in_contact;
        if (front_in) ds.front_right_col = wheel_steered_right_col(wh[0], ds.next_steer_angle);
        if (back_in) {
            const bool positive_zero = ds.next_steer_angle == 0.0f && !signbit(ds.next_steer_angle);
            if (front_in && positive_zero) {
                ds.back_right_col = ds.front_right_col;
            } else {
                ds.back_right_col = wheel_steered_right_col(wh[2], 0.0f);
            }
        }
        for (int i = 0; i < 4; ++i) wheel_drive_setup(c, ds, wh[i], i, wr, dt);
        // sticky force
        V3 sticky_sum = sticky_prev_world_normal_sum;
        bool gate = sticky_prev_world_contacts > 0;
        if (c.tick_count_since_update == 0) {
            sticky_sum = world_normal_sum;
            gate = world_contacts > 0;
        }
        if (gate) {
            const float l2 = len2(sticky_sum);
            const V3 up = l2 >= 1e-8f ? sticky_sum * (1.0f / sqrtf(l2)) : V3{0.0f, 0.0f, 0.0f};
            const bool full_stick = (k.throttle != 0.0f) || (abs_snapshot_forward_speed > 25.0f);
            const float base = 0.5f;
            const float full = base + 1.0f;
            const float target = full_stick ? full : base;
            const float scale = fabs_(up.z) * (base - target) + target;
            const float accel = (tc.gravity_z * scale) * (tc.gravity_z > 0.0f ? -1.0f : 1.0f);
            queue_force(f, ((accel * up) * kUuToBt) * tc.car_mass);
        }
    }

    if (wheel_world_contact) car_record_world_surface(c, false);
    if (car_has_flip_or_jump(c) && !c.flip_or_jump_last_tick) c.last_flip_or_jump_start = c.tick_count_since_update;
    const int air_gate_contacts = (c.tick_count_since_update != 0 || set_v3_tick)
                                      ? prev_wheel_contacts
                                      : (prev_wheel_contacts > num_contact ? prev_wheel_contacts : num_contact);
    const int landing_prev_contacts = (c.tick_count_since_update == 0 && !set_v3_tick)
                                          ? (num_contact > prev_wheel_contacts ? num_contact : prev_wheel_contacts)
                                          : prev_wheel_contacts;
    const uint8_t flipping_before_air = c.is_flipping;
    const V3 air_damp_ang_vel = c.cal_tick_start_ang_vel;
    if (air_gate_contacts < 3) {
        const V3 dodge_torque_bt = flip_torque(c, k, cfg, tc, raw_pitch, f);
        if (!c.driving_disabled)
            air_control(c, k, cfg, tc, landing_prev_contacts == 0, landing_prev_contacts == 0, pitchlock_restart_time,
                        air_damp_ang_vel, f);
        if (dodge_torque_bt.x != 0.0f || dodge_torque_bt.y != 0.0f || dodge_torque_bt.z != 0.0f)
            queue_torque(f, dodge_torque_bt);
    } else {
        c.is_flipping = 0;
        if (landing_prev_contacts == 0 && !c.driving_disabled)
            air_control(c, k, cfg, tc, true, true, pitchlock_restart_time, air_damp_ang_vel, f);
    }
    const bool flip_ended = air_gate_contacts < 3 && flipping_before_air && !c.is_flipping;
    update_jump_state(c, k, tc, f);
    if ((c.is_jumping && !was_jumping) || (!air_jump_used_before && (c.has_double_jumped || c.has_flipped)))
        wr.cal_game_jumped = 1;
    if (!air_jump_used_before && (c.has_double_jumped || c.has_flipped)) wr.cal_game_double_jumped = 1;
    wr.cal_jump_inactive_time = c.is_jumping ? 0.0f : wr.cal_jump_inactive_time + dt;
    const bool jump_changed = air_jump_started || (was_jumping && !c.is_jumping);
    const bool flip_changed = flip_started || c.is_flipping != flipping_at_start;
    if (jump_changed || !c.just_respawned) {
        const float jump_ticks = rintf(c.jump_time / dt) + 1.0f;
        c.jump_time = jump_changed ? dt : (jump_ticks <= 1024.0f ? c.jump_time + dt : jump_ticks * dt);
    }
    if (flip_changed || !c.just_respawned) c.flip_time = flip_changed ? dt : c.flip_time + dt;
    if (air_jump_started) {
        c.jump_hold_broken = 0;
    } else if (was_jumping && !k.jump) {
        c.jump_hold_broken = 1;
    }
    // auto-roll
    if (!autoroll_prev_contact) {
        autoroll_normal_sum = wr.cal_prev_wheel_normal_sum;
        autoroll_world_contacts = wr.cal_prev_world_wheel_contacts;
    }
    int autoroll_contacts = autoroll_world_contacts;
    bool autoroll_gate = autoroll_contacts < 4 && (autoroll_contacts > 0 || c.world_contact.has_contact);
    if (!autoroll_prev_contact && prev_wheel_contacts > 0 && prev_wheel_contacts < 4) {
        const bool sticky = autoroll_world_contacts > 0;
        autoroll_gate = sticky || c.world_contact.has_contact;
        autoroll_contacts = sticky ? prev_wheel_contacts : 0;
    }
    if (k.throttle && !c.is_flipping && !flipping_at_start && !flip_ended && autoroll_gate)
        apply_auto_roll(c, cfg, tc, autoroll_contacts, autoroll_normal_sum, f);
    c.set_wheel_normals_mask = 0;
    c.world_contact.has_contact = 0;
    if (!c.just_respawned) wheel_suspension_and_friction(c, tc, wh, f);
    apply_boost(c, k, tc, f);
    if (f.has_queued_jump_force) f.queued_force += f.queued_jump_force;
    wr.accumulated_force = f.queued_force;
    wr.accumulated_ang_accel = f.queued_ang_accel;
    wr.accumulated_torque_bt = f.queued_torque_bt;
    wr.solver_time_step = dt;
    if (tc.events.windows) wheel_world_event(c, wr, wh, pushes);
    for (int i = 0; i < 4; ++i) {
        const bool world = wh[i].is_in_contact && wh[i].is_in_contact_with_world;
        wr.event_world_ids[i] = world ? wh[i].ground_static_id : -1;
        wr.event_world_normals[i] = world ? wh[i].contact_normal_ws : V3{0.0f, 0.0f, 0.0f};
    }
}

// ---- world step: the car's external forces and integration (reference env_step.hpp:3737-3806,
// host_validation_and_contact_debug.hpp:971-1022) ------------------------------------------------------------------
struct PreContactCar {
    Q4 rot;
    V3 vel, vel_bt, ang_vel;
    uint8_t is_demoed;
};
// Wheel `i`'s arena-mesh ray as the car's vehicle update casts it (the same wheel set-up from the car's pose and
// config), for running the rays of every car ahead of the updates, one thread per wheel.
// Also reports whether the ray meets another car's box (`oth`: the arena's cars with this car's broadphase
// exclusions), which is when the update can push that car and must run in the arena's car order.
RG_HDI void wheel_mesh_ray_ahead(const CarState& c, const CarConfig& cfg, const MeshDevice& mesh, int i,
                                 const WheelOthers& oth, RayHit& hit, uint8_t& meets_car) {
    CarFrame f;
    car_basis(c, f.fwd, f.right, f.up);
    float front_bone, back_bone;
    wheel_bone_z(cfg, front_bone, back_bone);
    WheelStep w;
    init_wheel(w, c, cfg, i, f, i < 2 ? front_bone : back_bone);
    const float min_hit_dist_sq = min_wheel_hit_dist_sq_bt(cfg);
    wheel_mesh_ray(w, mesh, min_hit_dist_sq, hit);
    RayHit best;
    int best_idx;
    bool best_nr;
    wheel_ray_vs_cars(w, min_hit_dist_sq, oth, best, best_idx, best_nr);
    meets_car = best.hit ? 1 : 0;
}

RG_HDI void car_world_prestep(CarState& c, const CarConfig& cfg, const WheelRuntime& wr, const TickConfig& tc,
                              float sub_dt, PreContactCar& pre) {
    const bool inactive = c.is_demoed || c.just_respawned;
    V3 ext_force{0.0f, 0.0f, 0.0f};
    if (!inactive) {
        const float inv_mass = 1.0f / tc.car_mass;
        const V3 gravity_force_bt{0.0f, 0.0f, (tc.gravity_z * kUuToBt) * tc.car_mass};
        const V3 total = wr.accumulated_force + gravity_force_bt;
        ext_force = (total * inv_mass) * sub_dt;
    }
    V3 ext_torque{0.0f, 0.0f, 0.0f};
    if (!inactive) {
        const V3 t_bt = wr.accumulated_torque_bt;
        if (t_bt.x != 0.0f || t_bt.y != 0.0f || t_bt.z != 0.0f) {
            V3 r0, r1, r2;
            if (c.restored_inv_inertia_valid) {
                car_inv_inertia_world_bt(c, cfg, tc.car_mass, r0, r1, r2);
            } else {
                inv_inertia_world_from_columns(wr.pre_solve_basis_forward, wr.pre_solve_basis_right,
                                               wr.pre_solve_basis_up, car_inv_inertia_local_bt(cfg, tc.car_mass), r0,
                                               r1, r2);
            }
            ext_torque = vec_mul3x3(t_bt, r0, r1, r2) * sub_dt;
        }
    }
    pre.rot = c.rot;
    pre.vel = c.vel;
    pre.vel_bt = c.vel_bt;
    pre.ang_vel = c.ang_vel;
    pre.is_demoed = c.is_demoed;
    c.ext_force_impulse_bt = ext_force;
    c.ext_force_impulse_bt_valid = 1;
    c.solve_delta_linear_bt = V3{0.0f, 0.0f, 0.0f};
    c.solve_delta_angular = V3{0.0f, 0.0f, 0.0f};
    c.ext_torque_impulse = ext_torque;
}
RG_HDI void car_world_finish(CarState& c, const PreContactCar& pre, float sub_dt) {
    if (pre.is_demoed) return;
    if (c.just_respawned) return;
    // A car demolished during this step's car pairs takes the reference's fallback (ComputeOfficialExternalForce-
    // ImpulseBt from the same wheel record), which yields the impulses the prestep stored
    // (ApplyDeferredVelocityDeltas, host_validation_and_contact_debug.hpp:986-1023).
    if (c.ext_force_impulse_bt_valid) {
        car_set_vel_bt(c, c.vel_bt + c.ext_force_impulse_bt);
        c.ang_vel += c.ext_torque_impulse;
    }
    if (!is_zero(c.vel_bt)) car_set_pos_bt(c, c.pos_bt + c.vel_bt * sub_dt);
    game_integrate_orientation(c.basis_forward, c.basis_right, c.basis_up, c.rot, c.ang_vel, sub_dt);
}

// ---- post tick (reference env_step.hpp:5822-5912, raycast_wheels_and_contact_prep.hpp:3961-3992, 4033-4041) ------
RG_HDI void car_post_tick(CarState& c, const CarControls& k, float dt) {
    if (c.is_demoed) return;
    if (c.car_contact.cooldown_timer > 0.0f) c.car_contact.cooldown_timer = fmax_(0.0f, c.car_contact.cooldown_timer - dt);
    c.last_controls = k;
}
RG_HDI void car_finish_tick(CarState& c) {
    c.restored_inv_inertia_valid = 0;
    if (car_has_flip_or_jump(c) && !c.flip_or_jump_last_tick) c.last_flip_or_jump_start = c.tick_count_since_update;
    c.flip_or_jump_last_tick = car_has_flip_or_jump(c);
    c.ball_contact_last_tick = c.ball_contact_this_tick;
    if (c.is_demoed) return;
    if (c.pending_bump_count > 0) {
        V3 vel_bt = c.vel_bt;
        for (int i = 0; i < c.pending_bump_count; ++i) vel_bt = vel_bt + c.pending_bump_bt[i];
        car_set_vel_bt(c, vel_bt);
        c.pending_bump_count = 0;
        c.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
        c.vel_impulse_cache_bt = V3{0.0f, 0.0f, 0.0f};
    } else if (len2(c.vel_impulse_cache_bt) > 0.0f) {
        car_set_vel_bt(c, c.vel_bt + c.vel_impulse_cache_bt);
        c.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
        c.vel_impulse_cache_bt = V3{0.0f, 0.0f, 0.0f};
    } else if (len2(c.vel_impulse_cache) > 0.0f) {
        car_set_vel_uu(c, c.vel + c.vel_impulse_cache);
        c.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
    }
    c.tick_count_since_update += 1;
}
RG_HDI void report_rlbot_fields(CarState& c, const WheelRuntime& w, const TickConfig& tc) {
    const float dt = tc.tick_dt;
    if (c.is_demoed && c.tick_count_since_update == 0) {
        c.reported_flags = 0;
        return;
    }
    const bool dj_started = c.has_double_jumped && !c.internal_has_double_jumped;
    c.internal_vel = c.vel;
    c.internal_ang_vel = c.ang_vel;
    c.internal_has_jumped = c.has_jumped;
    c.internal_has_double_jumped = c.has_double_jumped;
    c.internal_has_flipped = c.has_flipped;
    c.internal_is_supersonic = c.is_supersonic;
    c.double_jump_ticks =
        !c.has_double_jumped ? 255 : (dj_started ? 0 : (c.double_jump_ticks < 255 ? c.double_jump_ticks + 1 : 255));
    const bool on_ground_state = c.is_on_ground && !c.is_jumping && !c.is_flipping;
    if (c.is_jumping) {
        c.game_has_jumped = 1;
    } else if (on_ground_state &&
               (!c.has_jumped || c.internal_jump_time - dt > tc.jump_min_time + tc.jump_reset_time_pad)) {
        c.game_has_jumped = 0;
    }
    bool game_jumped = w.cal_game_jumped != 0;
    bool game_double_jumped = w.cal_game_double_jumped != 0;
    if (!w.cal_frame_open && !w.cal_cached_ground &&
        (c.wheels_with_contact[0] != 0) + (c.wheels_with_contact[1] != 0) + (c.wheels_with_contact[2] != 0) +
                (c.wheels_with_contact[3] != 0) >=
            3) {
        game_jumped = game_double_jumped = false;
    }
    c.has_jumped = game_jumped;
    c.has_double_jumped = game_double_jumped && c.internal_has_double_jumped;
    c.has_flipped = game_double_jumped && !c.has_double_jumped;
    const uint8_t air_state =
        c.is_jumping ? 1 : (c.is_flipping ? 3 : (c.is_on_ground ? 0 : (c.double_jump_ticks < 13 ? 2 : 4)));
    c.air_state = air_state;
    const bool flipped = c.internal_has_flipped != 0;
    const bool dodged = (c.rlbotv5_dodged || flipped) && air_state != 0;
    c.rlbotv5_dodged = dodged ? 1 : 0;
    const float jump_inactive = w.cal_jump_inactive_time;
    const bool dodge_window = !c.is_on_ground && !c.is_jumping && c.game_has_jumped && !c.internal_has_double_jumped &&
                              !dodged && jump_inactive < tc.doublejump_max_delay - 0.5f * dt;
    c.dodge_timeout = dodge_window ? tc.doublejump_max_delay - jump_inactive : -1.0f;
    c.dodge_elapsed = (flipped && !on_ground_state) ? c.internal_flip_time : (dodged ? c.dodge_elapsed + dt : 0.0f);
    c.dodge_dir_x = c.flip_rel_torque.y;
    c.dodge_dir_y = -c.flip_rel_torque.x;
    c.reported_vel = c.vel;
    c.reported_ang_vel = c.ang_vel;
    c.reported_flags = kReportedValid | (c.has_jumped ? kReportedHasJumped : 0) |
                       (c.has_double_jumped ? kReportedHasDoubleJumped : 0) |
                       (c.has_flipped ? kReportedHasFlipped : 0) | (c.is_supersonic ? kReportedIsSupersonic : 0);
}
RG_HDI void advance_rlbot_fields(CarState& c, const WheelRuntime& w, const TickConfig& tc) {
    const float dt = tc.tick_dt;
    if (!(len2(c.vel_bt) < 1.0e38f && len2(c.ang_vel) < 1.0e38f)) {
        report_rlbot_fields(c, w, tc);
        return;
    }
    c.reported_flags = 0;
    if (c.is_demoed && c.tick_count_since_update == 0) return;
    const bool dj_started = c.has_double_jumped && !c.internal_has_double_jumped;
    c.internal_has_double_jumped = c.has_double_jumped;
    c.double_jump_ticks =
        !c.has_double_jumped ? 255 : (dj_started ? 0 : (c.double_jump_ticks < 255 ? c.double_jump_ticks + 1 : 255));
    const bool on_ground_state = c.is_on_ground && !c.is_jumping && !c.is_flipping;
    if (c.is_jumping) {
        c.game_has_jumped = 1;
    } else if (on_ground_state &&
               (!c.has_jumped || c.internal_jump_time - dt > tc.jump_min_time + tc.jump_reset_time_pad)) {
        c.game_has_jumped = 0;
    }
}

}  // namespace rg
