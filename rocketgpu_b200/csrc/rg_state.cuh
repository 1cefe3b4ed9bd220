// Device views of the public state structs (byte-identical to the C ABI's rg_*_state, which are byte-identical to the
// reference's BallState / EnvState, include/rocketgpu/rocketgpu.h:435-575) plus the per-config constants the tick
// reads.
#pragma once

#include <stddef.h>
#include <string.h>

#include "rg_math.cuh"
#include "rocketgpu_b200.h"

namespace rg {

struct BallState {
    float hs_y_target_dir, hs_cur_target_speed, hs_time_since_hit;
    uint32_t ds_pad0;
    int32_t ds_charge_level;
    float ds_accumulated_hit_force, ds_y_target_dir;
    uint8_t ds_flags[4];
    uint64_t ds_last_damage_tick;
    V3 pos;
    Q4 rot;
    V3 vel;
    V3 ang_vel;
    V3 vel_impulse_cache;
    uint64_t tick_count_when_extra_impulse_applied;
    uint64_t tick_count_since_update;
    V3 pos_bt, vel_bt;
    V3 basis_forward, basis_right, basis_up;
    uint32_t basis_authoritative;
    V3 inertia_basis_forward, inertia_basis_right, inertia_basis_up;
    uint32_t inertia_basis_valid;
    V3 restored_inv_inertia_bt[3];
    uint32_t restored_inv_inertia_valid;
    V3 vel_impulse_cache_bt;
    uint32_t sleeping;
    float deactivation_time;
    uint16_t constrained_2d, reserved_c2d;
};
static_assert(sizeof(BallState) == sizeof(rg_ball_state), "BallState layout");
static_assert(offsetof(BallState, pos) == offsetof(rg_ball_state, pos), "BallState layout");
static_assert(offsetof(BallState, vel_bt) == offsetof(rg_ball_state, vel_bt), "BallState layout");
static_assert(offsetof(BallState, sleeping) == offsetof(rg_ball_state, sleeping), "BallState layout");
static_assert(offsetof(BallState, constrained_2d) == offsetof(rg_ball_state, constrained_2d), "BallState layout");

struct EnvState {
    uint32_t tick, blue_score, orange_score;
    int32_t last_scored_team;
    uint8_t goal_scored_this_tick, car_visit_order_mode, car_visit_present_mask, kickoff_resets;
    uint32_t car_visit_order_packed;
    uint8_t countdown_phase, countdown_fires;
    uint16_t frame_ticks;
    float countdown_count, frame_frac_prev;
    uint16_t kickoff_match_order;
    uint8_t kickoff_match_index, goal_latched, respawn_match_order;
};
static_assert(sizeof(EnvState) == sizeof(rg_env_state), "EnvState layout");
static_assert(offsetof(EnvState, frame_frac_prev) == offsetof(rg_env_state, frame_frac_prev), "EnvState layout");

// Constants of one BatchSim config, resolved on the host (the reference's SimConfig + MutatorConfig fields the tick
// reads, with BatchSim's derived values such as the cached per-tick drag factor).
// A custom arena's spawns, ball spawn and goals (reference ArenaRules, detail/constants.hpp:57-67, made by
// MakeArenaRules, src/rocketgpu.cpp:859-881: goal normals normalized). TickConfig::rules points at one when the
// layout's rules differ from the official ones; null otherwise.
struct ArenaRules {
    V3 kickoff_pos[2][5];
    float kickoff_yaw[2][5];
    V3 respawn_pos[2][4];
    float respawn_yaw[2][4];
    V3 ball_spawn;
    V3 goal_point[2], goal_normal[2], goal_min[2], goal_max[2];
};

struct KickoffSettledRow;  // rg_reset.cuh

// Physics events (reference PhysicsEventType / PhysicsEvent / PhysicsEventWindow / PhysicsEventStream,
// rocketgpu.h:44-98), byte-identical to rg_physics_event / rg_physics_event_window.
enum : uint8_t {
    kEventBallTouchStart = 0,
    kEventBallWorldContact = 1,
    kEventCarWorldContact = 2,
    kEventBoostPickup = 3,
    kEventCarBump = 4,
    kEventGoal = 5,
};
struct PhysicsEvent {
    uint64_t tick;
    uint8_t type;
    uint32_t car_id, other_car_id;
    int32_t team;
    uint32_t pad_index;
    uint8_t car_on_ground, is_big_pad, is_demo;
    V3 position, normal, car_velocity, ball_position, ball_velocity;
    float boost_before, boost_after;
};
struct PhysicsEventWindow {
    uint64_t tick;
    uint32_t count, overflow;
};
static_assert(sizeof(PhysicsEvent) == sizeof(rg_physics_event) && sizeof(PhysicsEvent) == 104, "PhysicsEvent layout");
static_assert(offsetof(PhysicsEvent, position) == 32 && offsetof(PhysicsEvent, boost_after) == 96, "PhysicsEvent");
static_assert(sizeof(PhysicsEventWindow) == sizeof(rg_physics_event_window), "PhysicsEventWindow layout");
// The stream a batch writes: records[env * capacity + k] and windows[env] in device memory; off when windows is null.
struct EventStream {
    PhysicsEvent* records;
    PhysicsEventWindow* windows;
    uint32_t capacity, env_count, cars_per_env, goal_only;
};

struct TickConfig {
    float tick_dt;
    float gravity_z;
    float ball_radius, ball_mass, ball_drag, ball_drag_scale, ball_friction, ball_restitution;
    float ball_max_speed, ball_max_ang_speed;
    float goal_base_threshold_y;
    float frame_frac;
    uint8_t enable_scoring;
    // car-side constants (reference MutatorConfig defaults, include/rocketgpu/rocketgpu.h:708-817)
    uint8_t enable_boost_pads;
    int32_t max_cars;
    int32_t pad_count;
    float car_mass, car_max_speed, car_max_ang_speed, car_air_throttle_accel;
    float boost_max, boost_used_per_second, boost_min_time, boost_accel_ground, boost_spawn_amount;
    float recharge_boost_per_second, recharge_boost_delay;
    uint8_t recharge_boost_enabled, unlimited_flips, unlimited_double_jumps;
    float jump_accel, jump_immediate_speed, jump_min_time, jump_reset_time_pad, jump_max_time, doublejump_max_delay;
    float flip_torque_time, flip_pitchlock_extra_time, flip_initial_vel_scale, flip_torque_x, flip_torque_y;
    float flip_forward_impulse_max_speed_scale, flip_side_impulse_max_speed_scale,
        flip_backward_impulse_max_speed_scale, flip_backward_impulse_scale_x;
    float supersonic_start_speed, supersonic_maintain_min_speed, supersonic_maintain_max_time;
    float car_air_control_pitch, car_air_control_yaw, car_air_control_roll;
    float car_air_damp_pitch, car_air_damp_yaw, car_air_damp_roll;
    float boost_pad_cooldown_small, boost_pad_cooldown_big, demo_respawn_time;
    float arena_friction, arena_restitution;
    // car/car contacts (reference MutatorConfig: bump_force_scale 1, bump_cooldown_time 0.25, team demos off)
    uint8_t enable_car_car, enable_demos, enable_team_demos;
    float bump_force_scale, bump_cooldown_time;
    uint64_t kickoff_seed;  // the last reset_to_kickoff seed: demolished cars' respawn draw (reference Impl::seed)
    const ArenaRules* rules;  // custom spawns and goals (memory the kernels can read), or null
    // Kickoff settling (reference SimConfig::kickoff_settled_*, rocketgpu.h:892-897): per (car config, team) entry
    // and kickoff spot, the car and wheel record the game's countdown leaves, and the ball it leaves; null when off.
    const KickoffSettledRow* settled_rows;
    const int32_t* settled_entry;  // per car slot: its entry, or -1
    const BallState* settled_ball;
    int32_t settled_spawns;  // rows per entry (kickoff spots): max(max_cars_per_env, 5)
    EventStream events;      // physics events, or all zero
};

// A new event of `type` with the reference's member defaults (every field zero, team -1).
RG_HDI PhysicsEvent new_event(uint8_t type) {
    PhysicsEvent e;
    memset(&e, 0, sizeof(e));
    e.type = type;
    e.team = -1;
    return e;
}
// reference PhysicsEventStream::Emit / EmitForCar (rocketgpu.h:83-97): the env's window stamps the tick; a full
// window sets its overflow flag instead.
RG_HDI void emit_event(const EventStream& s, uint32_t env, PhysicsEvent e) {
    if (s.goal_only && e.type != kEventGoal) return;
    if (!s.windows || env >= s.env_count) return;
    PhysicsEventWindow& w = s.windows[env];
    e.tick = w.tick;
    if (w.count >= s.capacity) {
        w.overflow = 1;
        return;
    }
    s.records[static_cast<size_t>(env) * s.capacity + w.count++] = e;
}
RG_HDI void emit_event_for_car(const EventStream& s, uint32_t id, const PhysicsEvent& e) {
    if (id && s.cars_per_env) emit_event(s, (id - 1) / s.cars_per_env, e);
}

}  // namespace rg
