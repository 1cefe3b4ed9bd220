// Car dynamics of one arena tick, host+device: the pre-tick control, jump, flip, auto-flip, boost and air-control
// logic, the suspension rays and drive setup of the vehicle update, the deferred-force application and transform
// integration of the world step, and the post-tick bookkeeping including the RLBot-facing report fields.
//
// Each function restates one reference function (file:line given on it) in the same float operation order; the
// reference evaluates these scalar on its device build and through 4-wide host lanes on its CPU build, and both give
// the results written here. Cars live in global memory and are edited in place through references.
#pragma once

#include "rg_ball_world.cuh"
#include "rg_car_state.cuh"
#include "rg_math.cuh"
#include "rg_mesh.h"
#include "rg_state.cuh"
#include "rg_ucrt.cuh"

namespace rg {

constexpr float kUuToBt = 1.0f / 50.0f;
constexpr float kCarTorqueScale = (2.0f * kPiF / 65536.0f) * 1000.0f;  // reference constants.hpp:18
constexpr float kUeRot = 2.0f * kPiF / 65536.0f;
constexpr float kSteerDegToRad = 0.01745329238474369f;  // reference constants.hpp:112
constexpr float kWheelSuspensionSubtraction = 2.5f;
constexpr uint64_t kNoTick = ~0ull;
constexpr int kKickoffSpawnOverridePlus1 = 5;  // reference rocketgpu.h:529
constexpr int kRespawnOffsetOverridePlus1 = 128;  // reference rocketgpu.h:533

// Pre-tick flags the vehicle update reads back (reference env_step.hpp:2978-2979).
constexpr uint8_t kCalPreAirJumpStarted = 1, kCalPreFlipStarted = 2, kCalPreFlipVelChanged = 4,
                  kCalPreAirJumpUsedBefore = 8, kCalPreSetV3Tick = 16, kCalPreFlippingAtStart = 32,
                  kCalPreWasJumping = 64;

RG_HD float sgnf(float v) { return static_cast<float>((v > 0.0f) - (v < 0.0f)); }
RG_HD V3& operator+=(V3& a, V3 b) {
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
    return a;
}
RG_HD V3 mul3x3(V3 r0, V3 r1, V3 r2, V3 v) { return V3{dot(r0, v), dot(r1, v), dot(r2, v)}; }
// v^T M for a matrix given by rows (reference VecMul3x3, host_validation_and_contact_debug.hpp:585-591)
RG_HD V3 vec_mul3x3(V3 v, V3 r0, V3 r1, V3 r2) {
    return V3{r0.x * v.x + r1.x * v.y + r2.x * v.z, r0.y * v.x + r1.y * v.y + r2.y * v.z,
              r0.z * v.x + r1.z * v.y + r2.z * v.z};
}
RG_HD V3 rotate_via_basis(V3 f, V3 r, V3 u, V3 v) { return (f * v.x + r * v.y) + u * v.z; }
RG_HD V3 clamp_length(V3 v, float max_len) {
    const float l2 = len2(v);
    if (l2 <= max_len * max_len) return v;
    return (v * (1.0f / sqrtf(l2))) * max_len;
}
RG_HD V3 normalize_fallback(V3 v, V3 fallback) {
    const float l2 = len2(v);
    if (l2 <= 1e-12f) return fallback;
    return v * (1.0f / sqrtf(l2));
}

// The reference MutatorConfig's car-side defaults (include/rocketgpu/rocketgpu.h:733-817).
inline void fill_car_constants(TickConfig& t) {
    t.car_air_throttle_accel = 200.0f / 3.0f;
    t.boost_max = 100.0f;
    t.boost_used_per_second = 33.3f;
    t.boost_min_time = 0.10f;
    t.boost_accel_ground = 2975.0f / 3.0f;
    t.boost_spawn_amount = 33.3f;
    t.recharge_boost_per_second = 10.0f;
    t.recharge_boost_delay = 0.25f;
    t.recharge_boost_enabled = 0;
    t.jump_accel = 4375.0f / 3.0f;
    t.jump_immediate_speed = 875.0f / 3.0f;
    t.jump_min_time = 0.0249f;
    t.jump_reset_time_pad = 1.0f / 40.0f;
    t.jump_max_time = 0.20f;
    t.doublejump_max_delay = 1.25f;
    t.flip_torque_time = 0.65f;
    t.flip_pitchlock_extra_time = 0.30f;
    t.flip_initial_vel_scale = 500.0f;
    t.flip_torque_x = 260.0f;
    t.flip_torque_y = 224.0f;
    t.flip_forward_impulse_max_speed_scale = 1.0f;
    t.flip_side_impulse_max_speed_scale = 1.9f;
    t.flip_backward_impulse_max_speed_scale = 2.5f;
    t.flip_backward_impulse_scale_x = 16.0f / 15.0f;
    t.unlimited_flips = 0;
    t.unlimited_double_jumps = 0;
    t.supersonic_start_speed = 2200.0f;
    t.supersonic_maintain_min_speed = 2100.0f;
    t.supersonic_maintain_max_time = 1.0f;
    t.car_air_control_pitch = 130.0f;
    t.car_air_control_yaw = 95.0f;
    t.car_air_control_roll = 400.0f;
    t.car_air_damp_pitch = 30.0f;
    t.car_air_damp_yaw = 20.0f;
    t.car_air_damp_roll = 50.0f;
    t.boost_pad_cooldown_small = 4.0f;
    t.boost_pad_cooldown_big = 10.0f;
    t.demo_respawn_time = 3.0f;
    t.arena_friction = 0.30f;
    t.arena_restitution = 0.30f;
}

// ---- setters (reference arena_geometry.hpp:1799-1821) ------------------------------------------------------------
RG_HD void car_set_pos_bt(CarState& c, V3 p) {
    c.pos_bt = p;
    c.pos = p * 50.0f;
}
RG_HD void car_set_vel_bt(CarState& c, V3 v) {
    c.vel_bt = v;
    c.vel = v * 50.0f;
}
RG_HD void car_set_vel_uu(CarState& c, V3 v) {
    c.vel = v;
    c.vel_bt = v * kUuToBt;
    c.vel_touched_solve_stage = 1;
}

// reference CarBoostAmount / SetCarBoostAmount (raycast_wheels_and_contact_prep.hpp:3242-3250)
RG_HDI float car_boost_amount(const CarState& c) {
    const float amount = c.boost_amount;
    return amount * 100.0f == c.boost ? amount : c.boost / 100.0f;
}
RG_HDI void car_set_boost_amount(CarState& c, float amount) {
    c.boost_amount = amount;
    c.boost = amount * 100.0f;
}
RG_HD bool car_has_flip_or_jump(const CarState& c) {
    return c.is_on_ground || (!c.has_flipped && !c.has_double_jumped && c.air_time_since_jump < 1.25f);
}

// reference CarState::RecordWorldSurface (rocketgpu.h:239-246)
RG_HD void car_record_world_surface(CarState& c, bool body_contact) {
    c.last_world_surface_contact = c.tick_count_since_update;
    if (body_contact && c.last_ball_contact_start == c.tick_count_since_update) c.last_ball_started_with_world = 1;
    if (c.last_ball_contact_start != kNoTick && c.first_world_after_last_ball == kNoTick &&
        c.tick_count_since_update > c.last_ball_contact_start)
        c.first_world_after_last_ball = c.tick_count_since_update;
}

// reference CarState::RestoreWorkingFields / ReReportFields (rocketgpu.h:398-448): the report fields a caller sees
// are swapped back for the working values the tick continues from, unless the caller overwrote them.
RG_HD void restore_flag(const CarState& c, uint8_t& field, uint8_t internal, uint8_t bit, uint8_t& kept) {
    if ((field != 0) == ((c.reported_flags & bit) != 0)) {
        field = internal;
        kept |= bit;
    }
}
RG_HD uint8_t car_restore_working_fields(CarState& c) {
    if (!(c.reported_flags & kReportedValid)) return 0;
    uint8_t kept = kReportedValid;
    if (c.vel.x == c.reported_vel.x && c.vel.y == c.reported_vel.y && c.vel.z == c.reported_vel.z) {
        c.vel = c.internal_vel;
        kept |= kReportedVel;
    }
    if (c.ang_vel.x == c.reported_ang_vel.x && c.ang_vel.y == c.reported_ang_vel.y &&
        c.ang_vel.z == c.reported_ang_vel.z) {
        c.ang_vel = c.internal_ang_vel;
        kept |= kReportedAngVel;
    }
    restore_flag(c, c.has_jumped, c.internal_has_jumped, kReportedHasJumped, kept);
    restore_flag(c, c.has_double_jumped, c.internal_has_double_jumped, kReportedHasDoubleJumped, kept);
    restore_flag(c, c.has_flipped, c.internal_has_flipped, kReportedHasFlipped, kept);
    restore_flag(c, c.is_supersonic, c.internal_is_supersonic, kReportedIsSupersonic, kept);
    return kept;
}
RG_HD void re_report_flag(const CarState& c, uint8_t& field, uint8_t bit, uint8_t kept, uint8_t& flags) {
    if (kept & bit) field = (c.reported_flags & bit) ? 1 : 0;
    if (field) flags |= bit;
}
RG_HD void car_re_report_fields(CarState& c, uint8_t kept) {
    if (!(kept & kReportedValid)) return;
    c.internal_vel = c.vel;
    c.internal_ang_vel = c.ang_vel;
    c.internal_has_jumped = c.has_jumped;
    c.internal_has_double_jumped = c.has_double_jumped;
    c.internal_has_flipped = c.has_flipped;
    c.internal_is_supersonic = c.is_supersonic;
    if (kept & kReportedVel)
        c.vel = c.reported_vel;
    else
        c.reported_vel = c.vel;
    if (kept & kReportedAngVel)
        c.ang_vel = c.reported_ang_vel;
    else
        c.reported_ang_vel = c.ang_vel;
    uint8_t flags = kReportedValid;
    re_report_flag(c, c.has_jumped, kReportedHasJumped, kept, flags);
    re_report_flag(c, c.has_double_jumped, kReportedHasDoubleJumped, kept, flags);
    re_report_flag(c, c.has_flipped, kReportedHasFlipped, kept, flags);
    re_report_flag(c, c.is_supersonic, kReportedIsSupersonic, kept, flags);
    c.reported_flags = flags;
}

// reference CarState::ResetTrainingHistory (rocketgpu.h:230-238)
RG_HD void car_reset_training_history(CarState& c) {
    c.restored_inv_inertia_valid = 0;
    c.world_contact.wheel_ball_mask = 0;
    c.previous_ball_contact_start = c.last_ball_contact_start = c.last_world_surface_contact = kNoTick;
    c.first_world_after_previous_ball = c.first_world_after_last_ball = kNoTick;
    c.last_flip_or_jump_start = c.last_directional_flip_start = kNoTick;
    c.ball_contact_last_tick = c.ball_contact_this_tick = c.last_ball_started_with_world = 0;
    c.flip_or_jump_last_tick = car_has_flip_or_jump(c);
}

// ---- rotation helpers (reference math.hpp:940-1000, 1092-1150, 1392-1420, 1442-1530) -----------------------------
// Bullet's quaternion from a rotation matrix given by its columns (reference BulletQuatFromBasisColumns).
RG_HDI Q4 bullet_quat_from_basis(V3 fwd, V3 right, V3 up) {
    const float m00 = fwd.x, m01 = right.x, m02 = up.x;
    const float m10 = fwd.y, m11 = right.y, m12 = up.y;
    const float m20 = fwd.z, m21 = right.z, m22 = up.z;
    const float trace = m00 + m11 + m22;
    float r0, r1, r2, r3, x;
    if (trace > 0.0f) {
        x = trace + 1.0f;
        r0 = m21 - m12;
        r1 = m02 - m20;
        r2 = m10 - m01;
        r3 = x;
    } else {
        const int i = m00 < m11 ? (m11 < m22 ? 2 : 1) : (m00 < m22 ? 2 : 0);
        if (i == 0) {
            x = m00 - m11 - m22 + 1.0f;
            r0 = x;
            r1 = m10 + m01;
            r2 = m20 + m02;
            r3 = m21 - m12;
        } else if (i == 1) {
            x = m11 - m22 - m00 + 1.0f;
            r0 = m01 + m10;
            r1 = x;
            r2 = m21 + m12;
            r3 = m02 - m20;
        } else {
            x = m22 - m00 - m11 + 1.0f;
            r0 = m02 + m20;
            r1 = m12 + m21;
            r2 = x;
            r3 = m10 - m01;
        }
    }
    const float s = sqrtf(x);
    const float scale = 0.5f / s;
    return Q4{r3 * scale, r0 * scale, r1 * scale, r2 * scale};
}

// The game's axes of a quaternion (reference GameUeQuatAxes).
RG_HDI void ue_quat_axes(Q4 q, V3& fwd, V3& right, V3& up) {
    const float z2 = q.z + q.z, y2 = q.y + q.y;
    const float x2x = (q.x + q.x) * q.x, x2w = (q.x + q.x) * q.w;
    fwd = V3{1.0f - (z2 * q.z + y2 * q.y), z2 * q.w + y2 * q.x, z2 * q.x - y2 * q.w};
    right = V3{y2 * q.x - z2 * q.w, 1.0f - (z2 * q.z + x2x), x2w + z2 * q.y};
    up = V3{y2 * q.w + z2 * q.x, z2 * q.y - x2w, 1.0f - (y2 * q.y + x2x)};
}

// The game's rotation of a vector by a quaternion (reference GameUeQuatRotateVector).
RG_HDI V3 ue_quat_rotate(Q4 q, V3 v) {
    const float qq = (q.y * q.y + q.x * q.x) + q.z * q.z;
    const float d = q.w * q.w - qq;
    const float w2 = q.w + q.w;
    const float dt = (v.x * q.x + v.y * q.y) + v.z * q.z;
    const float t = dt + dt;
    const float cx = v.z * q.y - v.y * q.z, cy = v.x * q.z - v.z * q.x, cz = v.y * q.x - v.x * q.y;
    return V3{(cx * w2 + d * v.x) + t * q.x, (cy * w2 + d * v.y) + t * q.y, (cz * w2 + d * v.z) + t * q.z};
}

// UE3 rotator units: 65536 per turn. The sine table is evaluated, not stored (reference Ue3SinTab).
RG_HDI float ue3_sin_tab(int j) {
    const float a = ((static_cast<float>(j) + static_cast<float>(j)) * 3.14159274f) * 6.103515625e-05f;
    return ucrt_sinf(a);
}
RG_HDI float ue3_rotator_sin(int a) { return ue3_sin_tab((a >> 2) & 16383); }
struct Ue3Rotator {
    int pitch, yaw, roll;
};
RG_HDI int ue3_round(float v) { return x86_f2i(rintf(v + v + 0.5f)) >> 1; }
// reference Ue3QuatToRotator (math.hpp:1492-1512)
RG_HDI Ue3Rotator ue3_quat_to_rotator(Q4 q) {
    const float x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
    const float xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
    const float yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
    const float wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    const V3 fwd{1.0f - (yy + zz), xy + wz, xz - wy};
    const V3 right{xy - wz, 1.0f - (xx + zz), yz + wx};
    const V3 up{xz + wy, yz - wx, 1.0f - (xx + yy)};
    Ue3Rotator r;
    r.yaw = ue3_round(ucrt_atan2f(fwd.y, fwd.x) * 32768.0f / 3.14159274f);
    const float fwd_xy = static_cast<float>(sqrt(static_cast<double>(fwd.y * fwd.y + fwd.x * fwd.x)));
    r.pitch = ue3_round(ucrt_atan2f(fwd.z, fwd_xy) * 32768.0f / 3.14159274f);
    const float sy = ue3_rotator_sin(r.yaw);
    const float cy = ue3_rotator_sin(r.yaw + 16384);
    const float z_dot = (up.y * cy + up.x * -sy) + up.z * -0.0f;
    const float y_dot = (right.y * cy + right.x * -sy) + right.z * -0.0f;
    r.roll = ue3_round(ucrt_atan2f(z_dot, y_dot) * 32768.0f / 3.14159274f);
    return r;
}
// reference Ue3RotatorUpAxis (math.hpp:1524-1533)
RG_HDI V3 ue3_rotator_up_axis(const Ue3Rotator& r) {
    const float sy = ue3_rotator_sin(r.yaw);
    const float cy = ue3_rotator_sin(r.yaw + 16384);
    const float sp = ue3_rotator_sin(r.pitch);
    const float cp = ue3_rotator_sin(r.pitch + 16384);
    const float sr = ue3_rotator_sin(r.roll);
    const float cr = ue3_rotator_sin(r.roll + 16384);
    const float cr_sp = cr * sp;
    return V3{-(cr_sp * cy + sy * sr), cy * sr - cr_sp * sy, cp * cr};
}
// reference Ue3QuatFromYawRotator (math.hpp:1455-1477)
RG_HDI Q4 ue3_quat_from_yaw(int yaw) {
    const float sy = ue3_rotator_sin(yaw), cy = ue3_rotator_sin(yaw + 16384);
    const float cp = ue3_rotator_sin(16384);
    const float m[3][3] = {{cy * cp, cp * sy, 0.0f}, {-(cp * sy), cy * cp, -0.0f}, {-0.0f, 0.0f, cp * cp}};
    const float tr = (m[1][1] + m[0][0]) + m[2][2];
    if (tr > 0.0f) {
        const float inv_s = 1.0f / sqrtf(tr + 1.0f);
        const float s = inv_s * 0.5f;
        return Q4{0.5f / inv_s, (m[1][2] - m[2][1]) * s, (m[2][0] - m[0][2]) * s, (m[0][1] - m[1][0]) * s};
    }
    int i = m[0][0] < m[1][1] ? 1 : 0;
    if (m[i][i] <= m[2][2] && m[2][2] != m[i][i]) i = 2;
    const int j = i == 2 ? 0 : i + 1, k = j == 2 ? 0 : j + 1;
    const float inv_s = 1.0f / sqrtf(((m[i][i] - m[j][j]) - m[k][k]) + 1.0f);
    const float s = inv_s * 0.5f;
    float v[3];
    v[i] = 0.5f / inv_s;
    v[j] = (m[i][j] + m[j][i]) * s;
    v[k] = (m[i][k] + m[k][i]) * s;
    return Q4{(m[j][k] - m[k][j]) * s, v[0], v[1], v[2]};
}
// reference SpawnInertiaBasis (math.hpp:1514-1518)
RG_HDI void spawn_inertia_basis(Q4 spawn_rot, V3& fwd, V3& right, V3& up) {
    V3 f, r, u;
    ue_quat_axes(ue3_quat_from_yaw(ue3_quat_to_rotator(spawn_rot).yaw), f, r, u);
    game_basis_from_rot(game_rot_from_basis(f, r, u), fwd, right, up);
}

RG_HD void car_basis(const CarState& c, V3& f, V3& r, V3& u) {
    if (c.basis_authoritative) {
        f = c.basis_forward;
        r = c.basis_right;
        u = c.basis_up;
        return;
    }
    upload_basis_from_rot(c.rot, f, r, u);
}
RG_HD V3 car_rotate(const CarState& c, V3 v) {
    if (!c.basis_authoritative) {
        V3 f, r, u;
        upload_basis_from_rot(c.rot, f, r, u);
        return rotate_via_basis(f, r, u, v);
    }
    return rotate_via_basis(c.basis_forward, c.basis_right, c.basis_up, v);
}

// Orientation step of the game's integrator (reference GameIntegrateOrientationBasisColumns, math.hpp:1202-1228).
RG_HDI void game_integrate_orientation(V3& fwd, V3& right, V3& up, Q4& q_mirror, V3 w, float dt) {
    constexpr float kAngularMotionThreshold = 0.5f * kPiF * 0.5f;
    float angle = sqrtf((w.x * w.x + w.y * w.y) + w.z * w.z);
    if (angle * dt > kAngularMotionThreshold) angle = kAngularMotionThreshold / dt;
    float f;
    if (angle < 0.001f) {
        f = dt * 0.5f - ((((dt * dt) * dt) * 0.020833333333f) * angle) * angle;
    } else {
        const float half_angle = (angle * 0.5f) * dt;
        f = game_sinf(half_angle) / angle;
    }
    const float ax = w.x * f, ay = w.y * f, az = w.z * f;
    const float c = game_cosf((angle * dt) * 0.5f);
    const Q4 o = game_rot_from_basis(fwd, right, up);
    const Q4 p{((c * o.w - ax * o.x) - ay * o.y) - az * o.z, ((ax * o.w + c * o.x) + ay * o.z) - az * o.y,
               ((c * o.y + ay * o.w) + az * o.x) - ax * o.z, ((c * o.z + az * o.w) + ax * o.y) - ay * o.x};
    q_mirror = game_quat_normalize(p, -1.0f);
    game_basis_from_rot(q_mirror, fwd, right, up);
}

// ---- inertia (reference host_validation_and_contact_debug.hpp:156-175, 222-297, 530-700) -------------------------
RG_HDI V3 box_inertia_diag_bt(const CarConfig& cfg, float mass) {
    const V3 sized = cfg.hitbox_published + V3{2.5f, 2.5f, 2.5f};
    const bool has_published =
        sized.x == cfg.hitbox_size.x && sized.y == cfg.hitbox_size.y && sized.z == cfg.hitbox_size.z;
    const V3 published = has_published ? cfg.hitbox_published : cfg.hitbox_size - V3{2.5f, 2.5f, 2.5f};
    const V3 setup_half = (published * 0.02f) * 0.5f + V3{0.025f, 0.025f, 0.025f};
    const V3 box_half = (setup_half * 50.0f) * 0.02f;
    const float margin = fmin_(0.04f, 0.1f * fmin_(fmin_(box_half.x, box_half.y), box_half.z));
    const V3 margin_v{margin, margin, margin};
    const V3 half_extent = (box_half - margin_v) + margin_v;
    const float x = half_extent.x * 2.0f, y = half_extent.y * 2.0f, z = half_extent.z * 2.0f;
    const float x2 = x * x, y2 = y * y, z2 = z * z;
    const float scale = mass / 12.0f;
    return V3{scale * (y2 + z2), scale * (x2 + z2), scale * (x2 + y2)};
}
RG_HDI V3 car_inv_inertia_local_bt(const CarConfig& cfg, float mass) {
    const V3 i = box_inertia_diag_bt(cfg, mass);
    return V3{i.x != 0.0f ? 1.0f / i.x : 0.0f, i.y != 0.0f ? 1.0f / i.y : 0.0f, i.z != 0.0f ? 1.0f / i.z : 0.0f};
}
RG_HDI void inv_inertia_world_from_columns(V3 fc, V3 rc, V3 uc, V3 il, V3& o0, V3& o1, V3& o2) {
    const float b00 = fc.x, b01 = rc.x, b02 = uc.x;
    const float b10 = fc.y, b11 = rc.y, b12 = uc.y;
    const float b20 = fc.z, b21 = rc.z, b22 = uc.z;
    const float s00 = b00 * il.x, s01 = b01 * il.y, s02 = b02 * il.z;
    const float s10 = b10 * il.x, s11 = b11 * il.y, s12 = b12 * il.z;
    const float s20 = b20 * il.x, s21 = b21 * il.y, s22 = b22 * il.z;
    o0 = V3{s00 * b00 + s01 * b01 + s02 * b02, s00 * b10 + s01 * b11 + s02 * b12, s00 * b20 + s01 * b21 + s02 * b22};
    o1 = V3{s10 * b00 + s11 * b01 + s12 * b02, s10 * b10 + s11 * b11 + s12 * b12, s10 * b20 + s11 * b21 + s12 * b22};
    o2 = V3{s20 * b00 + s21 * b01 + s22 * b02, s20 * b10 + s21 * b11 + s22 * b12, s20 * b20 + s21 * b21 + s22 * b22};
}
// reference InverseMatrix3x3BulletStyle (host_validation_and_contact_debug.hpp:530-554)
RG_HDI void inverse3x3(V3 r0, V3 r1, V3 r2, V3& o0, V3& o1, V3& o2) {
    const float co_x = r1.y * r2.z - r1.z * r2.y;
    const float co_y = r1.z * r2.x - r1.x * r2.z;
    const float co_z = r1.x * r2.y - r1.y * r2.x;
    const float det = r0.x * co_x + r0.y * co_y + r0.z * co_z;
    const float s = det != 0.0f ? 1.0f / det : 0.0f;
    o0 = V3{co_x * s, (r0.z * r2.y - r0.y * r2.z) * s, (r0.y * r1.z - r0.z * r1.y) * s};
    o1 = V3{co_y * s, (r0.x * r2.z - r0.z * r2.x) * s, (r0.z * r1.x - r0.x * r1.z) * s};
    o2 = V3{co_z * s, (r0.y * r2.x - r0.x * r2.y) * s, (r0.x * r1.y - r0.y * r1.x) * s};
}
RG_HDI void car_inv_inertia_world_bt(const CarState& c, const CarConfig& cfg, float mass, V3& o0, V3& o1, V3& o2) {
    if (c.restored_inv_inertia_valid) {
        o0 = c.restored_inv_inertia_bt[0];
        o1 = c.restored_inv_inertia_bt[1];
        o2 = c.restored_inv_inertia_bt[2];
        return;
    }
    inv_inertia_world_from_columns(c.tick_start_basis_forward, c.tick_start_basis_right, c.tick_start_basis_up,
                                   car_inv_inertia_local_bt(cfg, mass), o0, o1, o2);
}

// The per-tick car frame of the vehicle update: tick-start basis, inverse inertia, queued forces
// (reference CarFrame / MakeCarFrame, host_validation_and_contact_debug.hpp:184-297).
struct CarFrame {
    V3 fwd, right, up;
    V3 inv_inertia_local_bt;
    V3 inv_w0, inv_w1, inv_w2;  // world inverse inertia rows (Bullet units)
    bool has_inertia;
    V3 in0, in1, in2;  // its inverse, built on first use
    bool queue_forces;
    V3 queued_force, queued_ang_accel, queued_torque_bt;
    bool has_queued_jump_force;
    V3 queued_jump_force;
    int n_force_items, n_torque_items;
    V3 force_items[4], torque_items[4];
};
RG_HDI void make_car_frame(CarFrame& f, const CarState& c, const CarConfig& cfg, float mass) {
    car_basis(c, f.fwd, f.right, f.up);
    f.inv_inertia_local_bt = car_inv_inertia_local_bt(cfg, mass);
    if (c.restored_inv_inertia_valid) {
        f.inv_w0 = c.restored_inv_inertia_bt[0];
        f.inv_w1 = c.restored_inv_inertia_bt[1];
        f.inv_w2 = c.restored_inv_inertia_bt[2];
    } else {
        inv_inertia_world_from_columns(c.tick_start_basis_forward, c.tick_start_basis_right, c.tick_start_basis_up,
                                       f.inv_inertia_local_bt, f.inv_w0, f.inv_w1, f.inv_w2);
    }
    f.has_inertia = false;
    f.queue_forces = false;
    f.queued_force = f.queued_ang_accel = f.queued_torque_bt = V3{0.0f, 0.0f, 0.0f};
    f.has_queued_jump_force = false;
    f.queued_jump_force = V3{0.0f, 0.0f, 0.0f};
    f.n_force_items = f.n_torque_items = 0;
}
RG_HD void frame_basis(const CarFrame* f, const CarState& c, V3& fw, V3& r, V3& u) {
    if (f) {
        fw = f->fwd;
        r = f->right;
        u = f->up;
        return;
    }
    car_basis(c, fw, r, u);
}
// World inertia tensor (Bullet units) = inverse of the frame's inverse-inertia rows
// (reference BuildInertiaTensorWorldBtInverse, host_validation_and_contact_debug.hpp:870-930).
RG_HDI void frame_inertia(const CarFrame* f, const CarState& c, const CarConfig& cfg, float mass, V3& o0, V3& o1,
                          V3& o2) {
    if (f) {
        CarFrame& m = const_cast<CarFrame&>(*f);
        if (!m.has_inertia) {
            inverse3x3(m.inv_w0, m.inv_w1, m.inv_w2, m.in0, m.in1, m.in2);
            m.has_inertia = true;
        }
        o0 = m.in0;
        o1 = m.in1;
        o2 = m.in2;
        return;
    }
    V3 i0, i1, i2;
    car_inv_inertia_world_bt(c, cfg, mass, i0, i1, i2);
    inverse3x3(i0, i1, i2, o0, o1, o2);
}
RG_HDI void frame_inv_inertia(const CarFrame* f, const CarState& c, const CarConfig& cfg, float mass, V3& o0, V3& o1,
                              V3& o2) {
    if (f) {
        o0 = f->inv_w0;
        o1 = f->inv_w1;
        o2 = f->inv_w2;
        return;
    }
    car_inv_inertia_world_bt(c, cfg, mass, o0, o1, o2);
}

// Force queues (reference QueueCentralForce / QueueOfficialTorqueBt, host_validation_and_contact_debug.hpp:726-790).
// The tick always runs with a wheel record and a frame that queues, so the queue lives in the frame.
RG_HD void queue_force(CarFrame& f, V3 force_bt) {
    f.queued_force += force_bt;
    if (f.n_force_items < 4) f.force_items[f.n_force_items] = force_bt;
    ++f.n_force_items;
}
RG_HD void queue_torque(CarFrame& f, V3 torque_bt) {
    f.queued_torque_bt += torque_bt;
    if (f.n_torque_items < 4) f.torque_items[f.n_torque_items] = torque_bt;
    ++f.n_torque_items;
}

// ---- impulses (reference host_validation_and_contact_debug.hpp:488-509) -------------------------------------------
RG_HD void car_apply_central_impulse_bt(CarState& c, V3 impulse_bt, float car_mass) {
    const float inv_mass = 1.0f / car_mass;
    if (!c.vel_touched_solve_stage && !c.is_on_ground) {
        car_set_vel_bt(c, c.vel_bt + impulse_bt * inv_mass);
        return;
    }
    const bool was_touched = c.vel_touched_solve_stage != 0;
    car_set_vel_bt(c, c.vel_bt + impulse_bt * inv_mass);
    if (was_touched || c.is_on_ground) c.vel_touched_solve_stage = 1;
}
RG_HD V3 game_jump_up_scaled_bt(const CarState& c, float scale_uu) {
    V3 f, r, u;
    ue_quat_axes(c.rot, f, r, u);
    return V3{(scale_uu * u.x) * 0.02f, (scale_uu * u.y) * 0.02f, (scale_uu * u.z) * 0.02f};
}

// ---- controls (reference raycast_wheels_and_contact_prep.hpp:2956-3046, arena_ball.hpp:2467-2476) ---------------
RG_HD float clamp1(float v) { return v < -1.0f ? -1.0f : (v > 1.0f ? 1.0f : v); }
RG_HDI float quantize_axis(float x) {
    const float c = clamp1(x);
    const float y = c < 0.0f ? fmax_(c * 128.0f, -128.0f) : fmin_(c * 127.0f, 127.0f);
    const float w = ((y + 128.0f) + (y + 128.0f)) + 0.5f;
    const int byte = (x86_f2i(rintf(w)) >> 1) & 0xFF;
    const float s = static_cast<float>(byte) - 128.0f;
    constexpr float kInv127 = 1.0f / 127.0f;
    const float q = s * kInv127;
    const float s_over_127 = fmaf(fmaf(-127.0f, q, s), kInv127, q);
    return byte < 0x80 ? s * (1.0f / 128.0f) : s_over_127;
}
// Clamp, byte-quantize the axes, and zero everything but throttle while driving is disabled
// (reference PreTickCarControls, env_step.hpp:2958-2976). raw_pitch is the clamped pitch before quantization.
RG_HDI CarControls pre_tick_controls(const CarState& c, CarControls k, float& raw_pitch) {
    k.throttle = clamp1(k.throttle);
    k.steer = clamp1(k.steer);
    k.pitch = clamp1(k.pitch);
    k.yaw = clamp1(k.yaw);
    k.roll = clamp1(k.roll);
    k.jump = k.jump ? 1 : 0;
    k.boost = k.boost ? 1 : 0;
    k.handbrake = k.handbrake ? 1 : 0;
    raw_pitch = k.pitch;
    k.throttle = quantize_axis(k.throttle);
    k.steer = quantize_axis(k.steer);
    k.pitch = quantize_axis(k.pitch);
    k.yaw = quantize_axis(k.yaw);
    k.roll = quantize_axis(k.roll);
    if (c.driving_disabled) {
        const float throttle = k.throttle;
        memset(&k, 0, sizeof(k));
        k.throttle = throttle;
    }
    return k;
}

// ---- tick start (reference env_step.hpp:5914-5926, 6751-6853; raycast_wheels_and_contact_prep.hpp:3677-3700,
// 3917-4028) -------------------------------------------------------------------------------------------------------
RG_HDI float cal_accumulated_ticks(int n, float dt) {
    if (n > 1024) return static_cast<float>(n) * dt;
    float t = 0.0f;
    for (int i = 0; i < n; ++i) t += dt;
    return t;
}
RG_HDI void cal_internal_timers_from_set_state(CarState& c, const TickConfig& tc) {
    const float dt = tc.tick_dt;
    c.internal_jump_time = (c.is_jumping || c.has_jumped) ? c.jump_time : 0.0f;
    const float flip_ticks = rintf(c.flip_time / dt);
    const int m = flip_ticks >= 0.0f ? x86_f2i(fmin_(flip_ticks, 1.0e6f)) : 0;
    if (c.is_flipping) {
        c.internal_flip_time = cal_accumulated_ticks(m > 1 ? m - 1 : 0, dt);
    } else if (c.has_flipped) {
        c.internal_flip_time = cal_accumulated_ticks(m + x86_f2i(rintf(tc.flip_torque_time / dt)), dt);
    } else {
        c.internal_flip_time = c.flip_time;
    }
}
RG_HDI void restore_step_fields(CarState& c) {
    if (c.tick_count_since_update != 0) {
        car_restore_working_fields(c);
        return;
    }
    if (c.supersonic_time > 0.0f) c.is_supersonic = 1;
    c.internal_has_double_jumped = c.has_double_jumped;
    c.game_has_jumped = c.has_jumped;
    c.double_jump_ticks = 255;
}
// Speed caps then the game's replicated-state quantization; saves the tick-start basis (reference
// CalTickStartLimitAndQuantizeCar + QuantizeCarState v3_exact).
RG_HDI void car_tick_start_quantize(CarState& c, const TickConfig& tc) {
    if (c.is_demoed) return;
    V3 vel_uu = c.vel_bt * 50.0f;
    const float l2 = len2(vel_uu);
    if (l2 > tc.car_max_speed * tc.car_max_speed) {
        vel_uu = (vel_uu * (1.0f / sqrtf(l2))) * tc.car_max_speed;
        car_set_vel_bt(c, vel_uu * kUuToBt);
    }
    c.ang_vel = clamp_length(c.ang_vel, tc.car_max_ang_speed);
    const uint8_t touched = c.vel_touched_solve_stage;
    const V3 p = c.pos_bt * 50.0f;
    const V3 qp{quant_round_pos(p.x, 100.0f), quant_round_pos(p.y, 100.0f), quant_round_pos(p.z, 100.0f)};
    car_set_pos_bt(c, qp * kUuToBt);
    c.pos = qp;
    const V3 q{quant_trunc_offset(vel_uu.x, 100.0f), quant_trunc_offset(vel_uu.y, 100.0f),
               quant_trunc_offset(vel_uu.z, 100.0f)};
    car_set_vel_bt(c, q * kUuToBt);
    c.vel = q;
    c.vel_touched_solve_stage = touched;
    c.ang_vel = V3{quant_trunc_offset(c.ang_vel.x, 10000.0f), quant_trunc_offset(c.ang_vel.y, 10000.0f),
                   quant_trunc_offset(c.ang_vel.z, 10000.0f)};
    V3 fwd, right, up;
    car_basis(c, fwd, right, up);
    c.tick_start_basis_forward = fwd;
    c.tick_start_basis_right = right;
    c.tick_start_basis_up = up;
    c.rot = game_quantize_basis(fwd, right, up);
    c.basis_forward = fwd;
    c.basis_right = right;
    c.basis_up = up;
    c.basis_authoritative = 1;
}
RG_HDI void cal_flip_z_damp_prepass(CarState& c, const TickConfig& tc) {
    if (c.is_demoed || c.is_on_ground || !c.is_flipping) return;
    const float flip_time = c.internal_flip_time + tc.tick_dt;
    if (!(flip_time >= 0.15f && flip_time <= tc.flip_torque_time)) return;
    if (c.vel_bt.z < 0.0f || flip_time < 0.21f) {
        const float dv_uu = (-c.vel.z) * 0.35f;
        if (fabs_(dv_uu) >= 1.0e-4f) {
            const float inv_mass = 1.0f / tc.car_mass;
            const float impulse = (dv_uu * 0.02f) * (1.0f / inv_mass);
            const V3 v = c.vel_bt;
            car_set_vel_bt(c, V3{v.x, v.y, v.z + impulse * inv_mass});
        }
    }
}
// reference BodyDampingClampCar (env_step.hpp:2916-2940)
RG_HDI int car_body_damping_clamp(CarState& c, const TickConfig& tc) {
    int clamped = 0;
    {
        const V3 v = c.vel_bt;
        const float max_lin = tc.car_max_speed * 0.02f;
        const float vsq = (v.x * v.x + v.y * v.y) + v.z * v.z;
        if (0.0f < max_lin && max_lin * max_lin < vsq) {
            const float s = 1.0f / sqrtf(vsq);
            c.vel_bt = V3{(v.x * s) * max_lin, (v.y * s) * max_lin, (v.z * s) * max_lin};
            clamped |= 1;
        }
    }
    {
        const V3 w = c.ang_vel;
        const float max_ang = tc.car_max_ang_speed;
        const float lsq = (w.x * w.x + w.y * w.y) + w.z * w.z;
        if (0.0f < max_ang && max_ang * max_ang < lsq) {
            const float s = 1.0f / sqrtf(lsq);
            c.ang_vel = V3{(w.x * s) * max_ang, (w.y * s) * max_ang, (w.z * s) * max_ang};
            clamped |= 2;
        }
    }
    return clamped;
}

// ---- pre-physics: supersonic, jump, double jump / dodge, auto-flip -------------------------------------------------
// reference UpdateSupersonicCalDemo (arena_ball.hpp:3168-3181)
RG_HDI void update_supersonic(CarState& c, V3 vel_uu, const TickConfig& tc) {
    const float speed_sq = len2(vel_uu);
    if (speed_sq >= (tc.supersonic_start_speed * tc.supersonic_start_speed)) {
        c.is_supersonic = 1;
        c.supersonic_time = 0.0f;
    } else if (c.is_supersonic) {
        c.supersonic_time += tc.tick_dt;
        if (c.supersonic_time >= tc.supersonic_maintain_max_time ||
            speed_sq < (tc.supersonic_maintain_min_speed * tc.supersonic_maintain_min_speed)) {
            c.is_supersonic = 0;
            c.supersonic_time = 0.0f;
        }
    }
}
// Forward speed from a rotation + velocity snapshot (reference SnapshotForwardSpeed, :1000-1016).
RG_HDI float snapshot_forward_speed(Q4 q, V3 v) {
    const float w2 = q.w + q.w;
    const float s = q.w * q.w - ((q.y * q.y + q.x * q.x) + q.z * q.z);
    float d = (1.0f * q.x + 0.0f * q.y) + 0.0f * q.z;
    d = d + d;
    const V3 fwd{((0.0f * q.y - 0.0f * q.z) * w2 + s * 1.0f) + d * q.x,
                 ((1.0f * q.z - 0.0f * q.x) * w2 + s * 0.0f) + d * q.y,
                 ((0.0f * q.x - 1.0f * q.y) * w2 + s * 0.0f) + d * q.z};
    return (fwd.x * v.x + fwd.y * v.y) + fwd.z * v.z;
}
// reference AutoFlipGate (:3485-3489)
RG_HDI bool auto_flip_gate(const CarState& c) {
    return c.world_contact.has_contact && c.world_contact.contact_normal.z > 0.707f &&
           dot(c.world_contact.contact_normal, ue3_rotator_up_axis(ue3_quat_to_rotator(c.rot))) < -0.966f;
}
// reference StartJump (:3388-3397); the three-wheel jump torque is not built
RG_HDI void start_jump(CarState& c, const TickConfig& tc) {
    c.is_jumping = 1;
    c.internal_jump_time = 0.0f;
    car_apply_central_impulse_bt(c, game_jump_up_scaled_bt(c, tc.jump_immediate_speed * tc.car_mass), tc.car_mass);
}
// reference CalFlipRestartTimeOnGround (:3654-3675)
RG_HDI float cal_flip_restart_time_on_ground(const CarState& c, const TickConfig& tc) {
    const float dt = tc.tick_dt;
    if (c.is_flipping) return 0.0f;
    if (!c.has_flipped) return c.internal_flip_time;
    if (c.internal_flip_time < tc.flip_torque_time) return 0.0f;
    int k = x86_f2i(rintf(c.internal_flip_time / dt)) - x86_f2i(rintf(tc.flip_torque_time / dt));
    if (k < 1) k = 1;
    if (k > 64) return static_cast<float>(k) * dt;
    float t = 0.0f;
    for (int i = 0; i < k; ++i) t += dt;
    return t;
}
// reference TryDoubleJumpOrFlip (:3546-3627)
RG_HDI bool try_double_jump_or_flip(CarState& c, const CarControls& k_in, const CarConfig& cfg, const TickConfig& tc,
                                    float forward_speed_uu, float raw_pitch) {
    CarControls k = k_in;
    k.pitch = -quantize_axis(-(raw_pitch <= 1.0f ? raw_pitch : k.pitch));
    const float input_magnitude = fabs_(k.yaw) + fabs_(k.pitch) + fabs_(k.roll);
    const bool is_flip_input = input_magnitude >= cfg.dodge_deadzone;
    bool can_use;
    if (is_flip_input) {
        can_use = ((!c.has_double_jumped && !c.has_flipped) || tc.unlimited_flips) && !c.is_auto_flipping;
    } else {
        can_use = ((!c.has_double_jumped && !c.has_flipped) || tc.unlimited_double_jumps) && !c.is_auto_flipping;
    }
    if (!can_use) return false;
    if (is_flip_input) {
        c.internal_flip_time = 0.0f;
        c.flip_timer_live = 1;
        c.last_directional_flip_start = c.tick_count_since_update;
        c.has_flipped = 1;
        c.is_flipping = 1;
        V3 dodge_dir{-k.pitch, k.yaw + k.roll, 0.0f};
        if (fabs_(k.yaw + k.roll) < 0.1f && fabs_(k.pitch) < 0.1f) {
            dodge_dir = V3{0.0f, 0.0f, 0.0f};
        } else {
            dodge_dir = normalize_fallback(dodge_dir, V3{0.0f, 0.0f, 0.0f});
        }
        c.flip_rel_torque = V3{-dodge_dir.y, dodge_dir.x, 0.0f};
        if (fabs_(dodge_dir.x) < 0.1f) dodge_dir.x = 0.0f;
        if (fabs_(dodge_dir.y) < 0.1f) dodge_dir.y = 0.0f;
        if (len2(dodge_dir) > 0.0f) {
            const float forward_speed_ratio = fabs_(forward_speed_uu) / tc.car_max_speed;
            bool backwards;
            if (fabs_(forward_speed_uu) < 100.0f) {
                backwards = dodge_dir.x < 0.0f;
            } else {
                backwards = ((dodge_dir.x >= 0.0f) != (forward_speed_uu >= 0.0f));
            }
            const float dodge_imp = tc.flip_initial_vel_scale * tc.car_mass;
            const float dodge_imp_x = backwards ? rintf(dodge_imp * tc.flip_backward_impulse_scale_x) : dodge_imp;
            V3 initial{dodge_dir.x * dodge_imp_x, dodge_dir.y * dodge_imp, 0.0f};
            const float max_speed_scale_x =
                backwards ? tc.flip_backward_impulse_max_speed_scale : tc.flip_forward_impulse_max_speed_scale;
            initial.x *= ((max_speed_scale_x - 1.0f) * forward_speed_ratio) + 1.0f;
            initial.y *= ((tc.flip_side_impulse_max_speed_scale - 1.0f) * forward_speed_ratio) + 1.0f;
            const int dodge_yaw = ue3_quat_to_rotator(c.rot).yaw;
            const int idx = (dodge_yaw >> 2) & 16383;
            const V3 fwd2{ue3_sin_tab((idx + 4096) & 16383), ue3_sin_tab(idx), 0.0f};
            const V3 right2{-fwd2.y, fwd2.x, 0.0f};
            const V3 final_delta_vel = fwd2 * initial.x + right2 * initial.y;
            car_apply_central_impulse_bt(c, final_delta_vel * 0.02f, tc.car_mass);
        }
    } else {
        car_apply_central_impulse_bt(c, game_jump_up_scaled_bt(c, tc.jump_immediate_speed * tc.car_mass), tc.car_mass);
        c.has_double_jumped = 1;
    }
    return is_flip_input;
}
// reference UpdateDoubleJumpOrFlipState (:3701-3750)
RG_HDI void update_double_jump_or_flip(CarState& c, const CarControls& k, const CarConfig& cfg, const TickConfig& tc,
                                       bool jump_pressed, float forward_speed_uu, bool press_as_air, float raw_pitch,
                                       bool& flip_started) {
    const float dt = tc.tick_dt;
    if (c.is_on_ground && !press_as_air) {
        c.has_double_jumped = 0;
        c.internal_flip_time = cal_flip_restart_time_on_ground(c, tc);
        c.has_flipped = 0;
        c.air_time = 0.0f;
        c.air_time_since_jump = 0.0f;
    } else {
        if (c.is_on_ground) {
            c.has_double_jumped = 0;
            c.internal_flip_time = cal_flip_restart_time_on_ground(c, tc);
            c.has_flipped = 0;
            c.air_time = 0.0f;
            c.air_time_since_jump = 0.0f;
        }
        c.air_time += dt;
        if (c.has_jumped && !c.is_jumping) {
            c.air_time_since_jump += dt;
        } else {
            c.air_time_since_jump = 0.0f;
        }
        if (jump_pressed && c.air_time_since_jump < tc.doublejump_max_delay) {
            if (try_double_jump_or_flip(c, k, cfg, tc, forward_speed_uu, raw_pitch)) flip_started = true;
            if (c.is_flipping && c.internal_flip_time == 0.0f) c.internal_flip_time = -dt;
        }
    }
    if (c.is_flipping) {
        c.internal_flip_time += dt;
    } else if (c.has_flipped || c.flip_timer_live || (c.internal_flip_time != 0.0f)) {
        c.internal_flip_time += dt;
    }
}
// reference ApplyAutoFlip (:3490-3544)
RG_HDI void apply_auto_flip(CarState& c, const CarConfig& cfg, const TickConfig& tc, bool starts, const CarFrame* f) {
    if (starts) {
        V3 fw, rg_, up;
        frame_basis(f, c, fw, rg_, up);
        const float roll = -ucrt_atan2f(rg_.z, up.z);
        const float abs_roll = fabs_(roll);
        const float flip_time = cfg.three_wheels ? 0.2f : 0.4f;
        c.auto_flip_timer =
            static_cast<float>(static_cast<double>(flip_time) * (static_cast<double>(abs_roll) / 3.14159265358979323846));
        c.auto_flip_torque_scale = (roll > 0.0f) ? 1.0f : -1.0f;
        c.is_auto_flipping = 1;
        V3 af, ar, au;
        ue_quat_axes(c.rot, af, ar, au);
        car_apply_central_impulse_bt(c, ((-au) * 200.0f) * kUuToBt * tc.car_mass, tc.car_mass);
    }
    if (c.is_auto_flipping) {
        if (c.auto_flip_timer <= 0.0f) {
            c.is_auto_flipping = 0;
            c.auto_flip_timer = 0.0f;
        } else {
            V3 af, ar, au;
            ue_quat_axes(c.rot, af, ar, au);
            const V3 t_flip = (af * 1000.0f) * c.auto_flip_torque_scale;
            V3 m0, m1, m2, i0, i1, i2;
            frame_inv_inertia(f, c, cfg, tc.car_mass, m0, m1, m2);
            frame_inertia(f, c, cfg, tc.car_mass, i0, i1, i2);
            c.ang_vel += mul3x3(m0, m1, m2, mul3x3(i0, i1, i2, t_flip));
            c.auto_flip_timer -= tc.tick_dt;
        }
    }
}

// Everything the tick does to a car before the vehicle update (reference PreTickCarPrePhysics, env_step.hpp:2981-3113),
// for a car that always has a wheel record.
RG_NOINL void car_pre_physics(CarState& c, CarControls k, const CarConfig& cfg, const TickConfig& tc, WheelRuntime& w,
                            Q4 snap_rot, V3 snap_vel_uu) {
    const float dt = tc.tick_dt;
    c.cal_pre_flags = 0;
    const uint8_t start_is_flipping = c.is_flipping;
    const uint8_t start_has_flipped = c.has_flipped;
    const uint8_t start_has_jumped = c.has_jumped;
    const uint8_t start_has_double_jumped = c.has_double_jumped;
    const uint8_t start_is_jumping = c.is_jumping;
    const uint8_t start_is_on_ground = c.is_on_ground;
    const float start_internal_flip_time = c.internal_flip_time;
    const float start_internal_jump_time = c.internal_jump_time;
    const bool start_last_jump = c.last_controls.jump;
    const uint64_t start_ticks = c.tick_count_since_update;
    const int start_wheel_contacts = (c.wheels_with_contact[0] != 0) + (c.wheels_with_contact[1] != 0) +
                                     (c.wheels_with_contact[2] != 0) + (c.wheels_with_contact[3] != 0);
    c.demo_no_contact_response = c.is_demoed ? 1 : 0;
    if (c.is_demoed) return;
    if (c.driving_disabled) k.jump = 0;
    const bool set_v3_tick = c.supersonic_set_v3 && start_ticks == 0;
    if (c.supersonic_set_v3) {
        c.supersonic_set_v3 = 0;
    } else {
        update_supersonic(c, snap_vel_uu, tc);
    }
    c.vel_touched_solve_stage = 0;
    bool flip_started = false;
    const bool jump_pressed = k.jump && !start_last_jump;
    const bool flip_over_starts = jump_pressed && !start_is_flipping && !c.is_auto_flipping && auto_flip_gate(c);
    const bool flip_over_takes_press = jump_pressed && !start_is_flipping && (c.is_auto_flipping || flip_over_starts);
    const bool need_pre_frame = cfg.three_wheels != 0 || c.is_auto_flipping != 0 ||
                                (jump_pressed && c.world_contact.has_contact && c.world_contact.contact_normal.z > 0.707f);
    CarFrame frame_store;
    const CarFrame* frame = nullptr;
    if (need_pre_frame) {
        make_car_frame(frame_store, c, cfg, tc.car_mass);
        frame = &frame_store;
    }
    if (start_ticks == 0 && w.cal_restored) c.flip_timer_live = 1;
    const float pitchlock_restart_time =
        (!start_has_flipped && !start_is_flipping && (start_internal_flip_time > 0.0f || c.flip_timer_live))
            ? start_internal_flip_time
            : -1.0f;
    bool air_jump_started = false;
    const bool jump_g = start_wheel_contacts >= 3;
    if (start_ticks == 0 && !w.cal_restored) {
        w.cal_game_jumped = start_has_jumped ? 1 : 0;
        w.cal_game_double_jumped = (start_has_double_jumped || start_has_flipped) && !jump_g ? 1 : 0;
        w.cal_cached_ground = jump_g ? 1 : 0;
        w.cal_jump_inactive_time = start_is_jumping ? 0.0f : start_internal_jump_time;
        w.cal_frame_open = 0;
    }
    w.cal_restored = 0;
    if (!w.cal_frame_open) {
        if (jump_g && !w.cal_cached_ground) {
            w.cal_game_jumped = 0;
            w.cal_game_double_jumped = 0;
        }
        w.cal_cached_ground = jump_g ? 1 : 0;
    }
    const bool jump_blocked = w.cal_game_jumped != 0;
    if (w.cal_game_jumped && jump_g && !start_is_jumping && w.cal_jump_inactive_time >= 0.125f) {
        w.cal_game_jumped = 0;
        w.cal_game_double_jumped = 0;
        w.cal_cached_ground = 1;
    }
    w.cal_frame_open = tc.frame_frac < 0.0f ? 1 : 0;
    const uint8_t was_jumping = start_is_jumping;
    const float forward_speed_uu = snapshot_forward_speed(snap_rot, snap_vel_uu);
    if (jump_pressed && start_is_on_ground && !start_is_jumping && !jump_blocked && !flip_over_takes_press) {
        start_jump(c, tc);
        air_jump_started = true;
    }
    const bool air_window_closed =
        w.cal_game_double_jumped || (w.cal_game_jumped && w.cal_jump_inactive_time > tc.doublejump_max_delay);
    const bool air_jump_pressed = jump_pressed && !jump_g && !air_window_closed && !flip_over_takes_press;
    const bool press_as_air = !jump_g && jump_pressed && !air_window_closed && !flip_over_takes_press;
    const uint8_t air_jump_used_before = (c.has_double_jumped || c.has_flipped) ? 1 : 0;
    bool flip_vel_changed = false;
    {
        const bool try_air_jump = air_jump_pressed && !air_jump_started;
        float raw_pitch = 2.0f;
        if (try_air_jump) k = pre_tick_controls(c, k, raw_pitch);
        const float fbw_speed = try_air_jump ? snapshot_forward_speed(c.rot, c.vel) : 0.0f;
        const V3 fbw_vel_bt = c.vel_bt;
        update_double_jump_or_flip(c, k, cfg, tc, try_air_jump, fbw_speed, press_as_air && !air_jump_started,
                                   raw_pitch, flip_started);
        flip_vel_changed = c.vel_bt.x != fbw_vel_bt.x || c.vel_bt.y != fbw_vel_bt.y || c.vel_bt.z != fbw_vel_bt.z;
    }
    apply_auto_flip(c, cfg, tc, flip_over_starts, frame);
    c.cal_pre_flags = static_cast<uint8_t>(
        (air_jump_started ? kCalPreAirJumpStarted : 0) | (flip_started ? kCalPreFlipStarted : 0) |
        (flip_vel_changed ? kCalPreFlipVelChanged : 0) | (air_jump_used_before ? kCalPreAirJumpUsedBefore : 0) |
        (set_v3_tick ? kCalPreSetV3Tick : 0) | (start_is_flipping ? kCalPreFlippingAtStart : 0) |
        (was_jumping ? kCalPreWasJumping : 0));
    c.cal_pre_forward_speed_uu = forward_speed_uu;
    c.cal_pre_pitchlock_restart_time = pitchlock_restart_time;
}

}  // namespace rg
