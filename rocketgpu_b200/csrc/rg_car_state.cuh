// Device views of the car-side public structs (byte-identical to the C ABI's rg_car_state / rg_car_config /
// rg_car_controls / rg_boost_pad_state, which are byte-identical to the reference's CarState, CarConfig, CarControls
// and BoostPadState, include/rocketgpu/rocketgpu.h:135-516) and of the per-car wheel record the tick keeps between
// ticks (the reference's WheelRuntimeState, include/rocketgpu/detail/step/arena_geometry.hpp:1545-1578).
#pragma once

#include <stddef.h>

#include "rg_math.cuh"
#include "rocketgpu_b200.h"

namespace rg {

struct CarControls {
    float throttle, steer, pitch, yaw, roll;
    uint8_t jump, boost, handbrake, pad_;
};
static_assert(sizeof(CarControls) == sizeof(rg_car_controls), "CarControls layout");

struct CarConfig {
    V3 hitbox_size, hitbox_published, hitbox_offset, front_wheels_offset, back_wheels_offset;
    float front_wheel_radius, back_wheel_radius;
    float front_suspension_rest, back_suspension_rest;
    float dodge_deadzone;
    uint8_t three_wheels;
    uint16_t body;
    float steer_angle_curve_deg[6];
    float powerslide_steer_angle_curve_deg[2];
    float spawn_z;
};
static_assert(sizeof(CarConfig) == sizeof(rg_car_config), "CarConfig layout");
static_assert(offsetof(CarConfig, steer_angle_curve_deg) == offsetof(rg_car_config, steer_angle_curve_deg), "layout");

struct BallHitInfo {
    uint8_t is_valid, extra_pending, extra_tick_is_previous, reserved2;
    uint64_t tick_count_when_hit;
    uint64_t tick_count_when_extra_impulse_applied;
    uint32_t hit_car_id;
    V3 relative_pos_on_ball, ball_pos, extra_hit_vel;
};

struct CarState {
    V3 pos;
    Q4 rot;
    V3 vel, ang_vel, flip_rel_torque;
    float jump_time, flip_time, air_time, air_time_since_jump, boost, time_since_boosted, boosting_time,
        supersonic_time, handbrake_val, auto_flip_timer, boost_amount, demo_respawn_timer;
    uint64_t tick_count_since_update;
    uint8_t ball_contact_last_tick, ball_contact_this_tick;
    uint8_t is_on_ground;
    uint8_t wheels_with_contact[4];
    uint8_t has_jumped, has_double_jumped, has_flipped, is_flipping, is_jumping, is_boosting, is_supersonic,
        is_auto_flipping, is_demoed, just_respawned;
    uint8_t demo_no_contact_response, respawn_slot_override_plus1, rlbotv5_boost_hold;
    struct {
        uint8_t has_contact, wheel_ball_mask, reserved1, reserved2;
        V3 contact_normal;
    } world_contact;
    struct {
        uint32_t other_car_id;
        float cooldown_timer;
    } car_contact;
    V3 vel_impulse_cache;
    BallHitInfo ball_hit_info;
    CarControls last_controls;
    V3 pos_bt, vel_bt, tick_start_pos_bt, pad_frame_pos_bt;
    uint8_t vel_touched_solve_stage, basis_authoritative, ext_force_impulse_bt_valid, pad_frame_pos_valid;
    V3 basis_forward, basis_right, basis_up;
    V3 ext_force_impulse_bt, ext_torque_impulse, solve_delta_linear_bt, vel_impulse_cache_bt, solve_delta_angular;
    uint8_t bump_event_bumps[7], bump_event_demos[7];
    uint8_t boost_pad_touching, bump_event_reserved1;
    uint64_t previous_ball_contact_start, last_ball_contact_start, last_world_surface_contact,
        first_world_after_previous_ball, first_world_after_last_ball, last_flip_or_jump_start,
        last_directional_flip_start;
    uint8_t last_ball_started_with_world, flip_or_jump_last_tick;
    float internal_jump_time, internal_flip_time;
    uint8_t flip_timer_live;
    uint8_t air_state;
    uint16_t driving_disabled;
    float dodge_timeout, dodge_elapsed, dodge_dir_x, dodge_dir_y;
    uint64_t latest_touch_tick;
    V3 latest_touch_location, latest_touch_normal;
    V3 internal_vel, internal_ang_vel, reported_vel, reported_ang_vel;
    uint8_t internal_has_jumped, internal_has_double_jumped, internal_has_flipped, internal_is_supersonic,
        reported_flags, game_has_jumped, double_jump_ticks, jump_hold_broken, supersonic_set_v3, rlbotv5_dodged;
    V3 set_wheel_normals[4];
    uint8_t set_wheel_normals_mask, cal_pre_flags;
    float cal_pre_forward_speed_uu, cal_pre_pitchlock_restart_time;
    V3 cal_tick_start_ang_vel, tick_start_basis_forward, tick_start_basis_right, tick_start_basis_up;
    V3 restored_inv_inertia_bt[3];
    uint8_t restored_inv_inertia_valid;
    V3 pending_bump_bt[7];
    uint32_t pending_bump_hitter[7];
    uint8_t pending_bump_count;
    float auto_flip_torque_scale;
};
static_assert(sizeof(CarState) == sizeof(rg_car_state), "CarState layout");
static_assert(offsetof(CarState, tick_count_since_update) == offsetof(rg_car_state, tick_count_since_update), "layout");
static_assert(offsetof(CarState, pos_bt) == offsetof(rg_car_state, pos_bt), "layout");
static_assert(offsetof(CarState, basis_forward) == offsetof(rg_car_state, basis_forward), "layout");
static_assert(offsetof(CarState, previous_ball_contact_start) == offsetof(rg_car_state, previous_ball_contact_start),
              "layout");
static_assert(offsetof(CarState, internal_vel) == offsetof(rg_car_state, internal_vel), "layout");
static_assert(offsetof(CarState, cal_tick_start_ang_vel) == offsetof(rg_car_state, cal_tick_start_ang_vel), "layout");
static_assert(offsetof(CarState, auto_flip_torque_scale) == offsetof(rg_car_state, auto_flip_torque_scale), "layout");

// Reported-field flags (reference CarState::kReported*, rocketgpu.h:395-396).
constexpr uint8_t kReportedVel = 1, kReportedAngVel = 2, kReportedHasJumped = 4, kReportedHasDoubleJumped = 8,
                  kReportedHasFlipped = 16, kReportedIsSupersonic = 32, kReportedValid = 128;

struct PadState {
    float cooldown;
    uint8_t is_active, is_big;
    uint16_t pickup_frac_q;
    uint32_t prev_locked_car_id, cur_locked_car_id;
};
static_assert(sizeof(PadState) == sizeof(rg_boost_pad_state), "PadState layout");

// Per-car wheel and jump bookkeeping kept between ticks (292 bytes, the reference's layout).
struct WheelRuntime {
    int32_t event_world_ids[4];
    V3 event_world_normals[4];
    float steer_angle[4], engine_force[4], brake[4], lat_friction[4], long_friction[4], extra_pushback[4];
    float solver_time_step;
    V3 accumulated_force, accumulated_ang_accel, accumulated_torque_bt;
    Q4 pre_solve_rot;
    V3 pre_solve_basis_forward, pre_solve_basis_right, pre_solve_basis_up;
    uint8_t pre_solve_basis_authoritative;
    V3 cal_prev_sticky_dir;
    V3 cal_prev_wheel_normal_sum;
    uint8_t cal_prev_world_wheel_contacts;
    uint8_t cal_game_jumped, cal_game_double_jumped, cal_cached_ground;
    float cal_jump_inactive_time;
    uint8_t cal_frame_open, cal_restored;
};
static_assert(sizeof(WheelRuntime) == 292, "WheelRuntime layout");

// The reference's default WheelRuntimeState (arena_geometry.hpp:1545-1578).
RG_HDI WheelRuntime wheel_runtime_default() {
    WheelRuntime w;
    memset(&w, 0, sizeof(w));
    for (int i = 0; i < 4; ++i) w.event_world_ids[i] = -1;
    w.solver_time_step = 1.0f / 60.0f;
    w.pre_solve_rot = Q4{1.0f, 0.0f, 0.0f, 0.0f};
    w.pre_solve_basis_forward = V3{1.0f, 0.0f, 0.0f};
    w.pre_solve_basis_right = V3{0.0f, 1.0f, 0.0f};
    w.pre_solve_basis_up = V3{0.0f, 0.0f, 1.0f};
    return w;
}

}  // namespace rg
