/*
 * rocketgpu_b200 — C ABI of the B200-native batched arena tick.
 *
 * The drop-in boundary for the reference's BatchSim (reference include/rocketgpu/rocketgpu.h:988-1089). Plain C:
 * opaque handle, plain pointers and sizes, int status (0 = ok) plus rg_last_error(), the convention of the
 * reference's C shim (rust/shim/shim.h:57-78). No C++ or torch types cross it, so a pybind module, a Rust crate or a
 * ctypes/cffi binding can sit directly on it.
 *
 * Public state structs are byte-identical to the reference's (same field order, types and padding), so callers pass
 * the arrays they already hold: rg_car_state == rocketgpu::CarState (880 B), rg_ball_state == BallState (288 B),
 * rg_env_state == EnvState (44 B), rg_boost_pad_state == BoostPadState (16 B), rg_car_controls == CarControls (24 B),
 * rg_car_config == CarConfig (120 B), rg_env_command == EnvCommand (16 B).
 *
 * Device side: every rg_batch owns its device memory (one allocation per array at create time, none while stepping).
 * Host pointers are borrowed for the call; device pointers (rg_batch_step_with_device_controls) must stay valid until
 * the given stream has run the step. Errors are reported synchronously for argument checks; a CUDA error raised by
 * an earlier asynchronous launch is reported by the next call that synchronises (rg_batch_synchronize, downloads).
 */
#ifndef ROCKETGPU_B200_H
#define ROCKETGPU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define RG_API __declspec(dllexport)
#else
#define RG_API __attribute__((visibility("default")))
#endif

typedef struct rg_vec3 { float x, y, z; } rg_vec3;
typedef struct rg_quat { float w, x, y, z; } rg_quat;

/* reference rocketgpu.h:127-136 */
typedef struct rg_car_controls {
    float throttle, steer, pitch, yaw, roll;
    uint8_t jump, boost, handbrake;
} rg_car_controls;

/* reference rocketgpu.h:138-171 */
typedef struct rg_car_config {
    rg_vec3 hitbox_size;
    rg_vec3 hitbox_published;
    rg_vec3 hitbox_offset;
    rg_vec3 front_wheels_offset;
    rg_vec3 back_wheels_offset;
    float front_wheel_radius, back_wheel_radius;
    float front_suspension_rest, back_suspension_rest;
    float dodge_deadzone;
    uint8_t three_wheels;
    uint16_t body;
    float steer_angle_curve_deg[6];
    float powerslide_steer_angle_curve_deg[2];
    float spawn_z;
} rg_car_config;

/* reference rocketgpu.h:173-184 */
typedef struct rg_ball_hit_info {
    uint8_t is_valid, extra_pending, extra_tick_is_previous, reserved2;
    uint64_t tick_count_when_hit;
    uint64_t tick_count_when_extra_impulse_applied;
    uint32_t hit_car_id;
    rg_vec3 relative_pos_on_ball, ball_pos, extra_hit_vel;
} rg_ball_hit_info;

/* reference rocketgpu.h:186-433 (field order and meaning as there) */
typedef struct rg_car_state {
    rg_vec3 pos; rg_quat rot; rg_vec3 vel; rg_vec3 ang_vel; rg_vec3 flip_rel_torque;
    float jump_time, flip_time, air_time, air_time_since_jump, boost, time_since_boosted, boosting_time,
        supersonic_time, handbrake_val, auto_flip_timer, boost_amount, demo_respawn_timer;
    uint64_t tick_count_since_update;
    uint8_t ball_contact_last_tick, ball_contact_this_tick;
    uint8_t is_on_ground;
    uint8_t wheels_with_contact[4];
    uint8_t has_jumped, has_double_jumped, has_flipped, is_flipping, is_jumping, is_boosting, is_supersonic,
        is_auto_flipping, is_demoed, just_respawned;
    uint8_t demo_no_contact_response, respawn_slot_override_plus1, rlbotv5_boost_hold;
    struct { uint8_t has_contact, wheel_ball_mask, reserved1, reserved2; rg_vec3 contact_normal; } world_contact;
    struct { uint32_t other_car_id; float cooldown_timer; } car_contact;
    rg_vec3 vel_impulse_cache;
    rg_ball_hit_info ball_hit_info;
    rg_car_controls last_controls;
    rg_vec3 pos_bt, vel_bt, tick_start_pos_bt, pad_frame_pos_bt;
    uint8_t vel_touched_solve_stage, basis_authoritative, ext_force_impulse_bt_valid, pad_frame_pos_valid;
    rg_vec3 basis_forward, basis_right, basis_up;
    rg_vec3 ext_force_impulse_bt, ext_torque_impulse, solve_delta_linear_bt, vel_impulse_cache_bt, solve_delta_angular;
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
    rg_vec3 latest_touch_location, latest_touch_normal;
    rg_vec3 internal_vel, internal_ang_vel, reported_vel, reported_ang_vel;
    uint8_t internal_has_jumped, internal_has_double_jumped, internal_has_flipped, internal_is_supersonic,
        reported_flags, game_has_jumped, double_jump_ticks, jump_hold_broken, supersonic_set_v3, rlbotv5_dodged;
    rg_vec3 set_wheel_normals[4];
    uint8_t set_wheel_normals_mask, cal_pre_flags;
    float cal_pre_forward_speed_uu, cal_pre_pitchlock_restart_time;
    rg_vec3 cal_tick_start_ang_vel, tick_start_basis_forward, tick_start_basis_right, tick_start_basis_up;
    rg_vec3 restored_inv_inertia_bt[3];
    uint8_t restored_inv_inertia_valid;
    rg_vec3 pending_bump_bt[7];
    uint32_t pending_bump_hitter[7];
    uint8_t pending_bump_count;
    float auto_flip_torque_scale;
} rg_car_state;

/* reference rocketgpu.h:435-505 */
typedef struct rg_ball_state {
    struct { float y_target_dir, cur_target_speed, time_since_hit; } hs_info;
    struct {
        int32_t charge_level; float accumulated_hit_force, y_target_dir;
        uint8_t has_damaged, reserved0, reserved1, reserved2;
        uint64_t last_damage_tick;
    } ds_info;
    rg_vec3 pos; rg_quat rot; rg_vec3 vel; rg_vec3 ang_vel; rg_vec3 vel_impulse_cache;
    uint64_t tick_count_when_extra_impulse_applied;
    uint64_t tick_count_since_update;
    rg_vec3 pos_bt, vel_bt;
    rg_vec3 basis_forward, basis_right, basis_up;
    uint32_t basis_authoritative;
    rg_vec3 inertia_basis_forward, inertia_basis_right, inertia_basis_up;
    uint32_t inertia_basis_valid;
    rg_vec3 restored_inv_inertia_bt[3];
    uint32_t restored_inv_inertia_valid;
    rg_vec3 vel_impulse_cache_bt;
    uint32_t sleeping;
    float deactivation_time;
    uint16_t constrained_2d, reserved_c2d;
} rg_ball_state;

/* reference rocketgpu.h:507-516 */
typedef struct rg_boost_pad_state {
    float cooldown;
    uint8_t is_active, is_big;
    uint16_t pickup_frac_q;
    uint32_t prev_locked_car_id, cur_locked_car_id;
} rg_boost_pad_state;

/* reference rocketgpu.h:535-575 */
typedef struct rg_env_state {
    uint32_t tick, blue_score, orange_score;
    int32_t last_scored_team;
    uint8_t goal_scored_this_tick, car_visit_order_mode, car_visit_present_mask, kickoff_resets;
    uint32_t car_visit_order_packed;
    uint8_t countdown_phase, countdown_fires;
    uint16_t frame_ticks;
    float countdown_count, frame_frac_prev;
    uint16_t kickoff_match_order;
    uint8_t kickoff_match_index, goal_latched, respawn_match_order;
} rg_env_state;

/* reference rocketgpu.h:683-706 */
typedef struct rg_env_command {
    uint8_t reset_to_kickoff, reset_scoreboard, reset_tick_count, kickoff_seed_mode, new_round_bodies, keep_boost_pads;
    uint16_t kickoff_countdown_ticks;
    uint64_t kickoff_seed;
} rg_env_command;

/* reference PhysicsEvent / PhysicsEventWindow (rocketgpu.h:44-70; types: 0 ball touch start, 1 ball-world contact,
 * 2 car-world contact, 3 boost pickup, 4 car bump, 5 goal). Fields an event does not set are 0, team -1. */
typedef struct rg_physics_event {
    uint64_t tick;
    uint8_t type;
    uint32_t car_id, other_car_id;
    int32_t team;
    uint32_t pad_index;
    uint8_t car_on_ground, is_big_pad, is_demo;
    rg_vec3 position, normal, car_velocity, ball_position, ball_velocity;
    float boost_before, boost_after;
} rg_physics_event;
typedef struct rg_physics_event_window {
    uint64_t tick;
    uint32_t count, overflow;
} rg_physics_event_window;

/* The BatchSim configuration subset this path takes (reference SimConfig, rocketgpu.h:842-909, and the
 * MutatorConfig fields the tick reads, rocketgpu.h:708-840). Zero-initialise, then call rg_sim_config_default. */
typedef struct rg_sim_config {
    int32_t env_count;
    int32_t max_cars_per_env;       /* 0..6 (the reference allows 8; 7- and 8-car arenas are refused here) */
    float tick_dt;                   /* 1/120 */
    uint8_t enable_boost_pads, enable_car_car_collisions, enable_demos, enable_scoring;
    uint64_t respawn_rng_seed;
    /* mutator */
    float gravity_z, ball_radius, ball_mass, car_mass, ball_drag, ball_friction, ball_restitution, ball_max_speed,
        ball_max_ang_speed, car_max_speed, car_max_ang_speed, arena_friction, arena_restitution,
        goal_base_threshold_y;
    /* reference MutatorConfig::kickoff_settled (rocketgpu.h:831, default 1 there and here). 1: a kickoff without a
     * countdown puts each car into the state the game's countdown leaves at its spot (and the ball into the state it
     * leaves), recorded once per (car config, team) by stepping a countdown kickoff (src/rocketgpu.cpp:1439-1612);
     * recorded at create and before a reset after set_car_configs / set_teams / set_env_car_count. A batch with 1
     * takes no further geometry (rg_batch_add_mesh) and the server takes 0. */
    uint8_t kickoff_settled;
    uint8_t reserved[7];
} rg_sim_config;

/* reference ArenaSpawn (rocketgpu.h:929-933): pos.z is the ground under the car (its spawn_z is added); yaw in rad */
typedef struct rg_arena_spawn { rg_vec3 pos; float yaw; } rg_arena_spawn;
/* reference ArenaGoal (rocketgpu.h:935-942): the other team scores when the ball's centre is at least the ball radius
 * past the plane through point (normal into the goal) and inside [min, max] */
typedef struct rg_arena_goal { rg_vec3 point, normal, min, max; } rg_arena_goal;
/* reference BoostPadConfig (rocketgpu.h:518-524) */
typedef struct rg_boost_pad_config { rg_vec3 pos; uint8_t is_big, reserved0, reserved1, reserved2; } rg_boost_pad_config;
/* The rules part of reference ArenaLayout (goals[2], kickoff_spawns[2][5], respawn_spawns[2][4], ball_spawn); teams
 * index the arrays (0 blue, 1 orange). rg_default_arena_rules fills the official ones. */
typedef struct rg_arena_rules {
    rg_arena_goal goals[2];
    rg_arena_spawn kickoff_spawns[2][5];
    rg_arena_spawn respawn_spawns[2][4];
    rg_vec3 ball_spawn;
} rg_arena_rules;

/* A custom arena (reference ArenaLayout, rocketgpu.h:943-959): one triangle mesh in uu, optional rules and pads.
 * Rules equal to the official ones behave as null, as the reference's SameArenaRules test makes them
 * (src/rocketgpu.cpp:834-849); positions are validated as ValidateArenaLayout does (finite, within 11,500 uu, spawn
 * yaw within 8 pi, goal normal nonzero, goal bounds not NaN). Planes and mesh directories are not built. */
typedef struct rg_arena_layout {
    const float* vertices_uu;   /* 3 * vertex_count */
    int64_t vertex_count;
    const int32_t* indices;     /* 3 per triangle */
    int64_t index_count;
    const rg_arena_rules* rules;            /* null: the official goals, spawns and ball spawn */
    const rg_boost_pad_config* boost_pads;  /* null: the 34 soccar pads */
    int32_t boost_pad_count;                /* with boost_pads: 0..48 (reference kMaxBoostPads) */
    int32_t reserved;
} rg_arena_layout;
/* The official rules (reference ArenaLayout::ArenaLayout, src/rocketgpu.cpp:2754-2775). */
RG_API void rg_default_arena_rules(rg_arena_rules* out);

typedef struct rg_batch rg_batch;

/* Last error of this thread, "" if none. */
RG_API const char* rg_last_error(void);
/* Library version string. */
RG_API const char* rg_version(void);

/* Fills a config with the reference's SimConfig/MutatorConfig defaults. */
RG_API void rg_sim_config_default(rg_sim_config* cfg);
/* Reference-default public states (the reference's member initialisers), for callers building uploads. */
RG_API void rg_default_ball_state(rg_ball_state* out);
RG_API void rg_default_env_state(rg_env_state* out);
/* CarState{} and CarConfig{} (the Octane preset) — reference rocketgpu.h:135-175, 190-502. */
RG_API void rg_default_car_state(rg_car_state* out);
RG_API void rg_default_car_config(rg_car_config* out);
/* The hitbox presets: 0 Octane (= rg_default_car_config), 1 Dominus, 2 Plank, 3 Breakout, 4 Hybrid, 5 Merc
 * (reference OctaneConfig .. MercConfig, src/rocketgpu.cpp:417-490; Python binding OctaneConfig() ..). out_of_range
 * for any other index. */
RG_API int rg_car_preset(int32_t preset, rg_car_config* out);

/* BatchSim(config, layout) — reference rocketgpu.h:990-992, src/rocketgpu.cpp:1019-1250. Validates the config
 * (env_count > 0, 0 <= max_cars_per_env <= 8) and layout (finite, within 11,500 uu), builds the mesh BVH on the
 * host, uploads it and allocates every device array. */
RG_API int rg_batch_create(const rg_sim_config* cfg, const rg_arena_layout* layout, int device, rg_batch** out);
/* ~BatchSim */
RG_API void rg_batch_destroy(rg_batch* b);

RG_API int64_t rg_batch_env_count(const rg_batch* b);    /* BatchSim::env_count (rocketgpu.h:1012) */
RG_API int64_t rg_batch_car_capacity(const rg_batch* b); /* BatchSim::car_capacity (rocketgpu.h:1011) */

/* BatchSim::set_env_car_count (rocketgpu.h:1017; range checks src/rocketgpu.cpp:2920-2932). */
RG_API int rg_batch_set_env_car_count(rg_batch* b, const int32_t* host_counts, size_t count, void* stream);
/* BatchSim::upload_ball_states / download_ball_states (rocketgpu.h:1023-1046). */
RG_API int rg_batch_upload_ball_states(rg_batch* b, const rg_ball_state* host, size_t count, void* stream);
RG_API int rg_batch_download_ball_states(rg_batch* b, rg_ball_state* host, size_t count, void* stream);
/* BatchSim::upload_env_states / download_env_states (rocketgpu.h:1027,1047). */
RG_API int rg_batch_upload_env_states(rg_batch* b, const rg_env_state* host, size_t count, void* stream);
RG_API int rg_batch_download_env_states(rg_batch* b, rg_env_state* host, size_t count, void* stream);
/* BatchSim::upload_car_states in PublicState mode / download_car_states (rocketgpu.h:1028,1036; src/rocketgpu.cpp:
 * 2952-2965 with the import canonicalisation of src/rocketgpu.cpp:355-379). Slot j of env e is index
 * e * max_cars_per_env + j. */
RG_API int rg_batch_upload_car_states(rg_batch* b, const rg_car_state* host, size_t count, void* stream);
RG_API int rg_batch_download_car_states(rg_batch* b, rg_car_state* host, size_t count, void* stream);
/* BatchSim::boost_pad_capacity / upload_boost_pad_states / download_boost_pad_states (rocketgpu.h:1019,1034,1048):
 * 34 pads per env (the layout's default soccar pads), pad p of env e at index e * 34 + p. */
RG_API int64_t rg_batch_pad_capacity(const rg_batch* b);
RG_API int rg_batch_upload_pad_states(rg_batch* b, const rg_boost_pad_state* host, size_t count, void* stream);
RG_API int rg_batch_download_pad_states(rg_batch* b, rg_boost_pad_state* host, size_t count, void* stream);
/* BatchSim::set_car_configs (rocketgpu.h:1025). Three-wheel configs are rejected (invalid_argument): that car
 * model is not built. */
RG_API int rg_batch_set_car_configs(rg_batch* b, const rg_car_config* host, size_t count, void* stream);
/* BatchSim::set_teams (rocketgpu.h:1024): team per car slot, 0 blue / 1 orange (the reference's Team enum). */
RG_API int rg_batch_set_teams(rg_batch* b, const uint8_t* host, size_t count, void* stream);
/* BatchSim::reset_to_kickoff (rocketgpu.h:1070; src/rocketgpu.cpp:2085-2132, ResetEnvToKickoff arena_ball.hpp:
 * 3054-3085): every arena to kickoff, the spot order drawn from `seed` (0: from the arena's reset count). Car
 * contact state and the ball's manifolds are cleared; wheel records are kept, as the reference keeps them.
 * rg_batch_create ends with reset_to_kickoff(0). With kickoff_settled = 1 the cars and the ball take their settled
 * states (rg_sim_config). */
RG_API int rg_batch_reset_to_kickoff(rg_batch* b, uint64_t seed, void* stream);
/* BatchSim::upload_controls (rocketgpu.h:1032): the controls rg_batch_step holds for every tick. */
RG_API int rg_batch_upload_controls(rg_batch* b, const rg_car_controls* host, size_t count, void* stream);

/* BatchSim::step (rocketgpu.h:1063; src/rocketgpu.cpp:3237): advances every env by `ticks` 120 Hz ticks on `stream`
 * (asynchronous; no host synchronisation). */
RG_API int rg_batch_step(rg_batch* b, int32_t ticks, void* stream);
/* BatchSim::step_with_device_controls (rocketgpu.h:1075; checks src/rocketgpu.cpp:2412-2421): tick t reads car i's
 * controls at device_controls[t * control_stride + i]; control_stride 0 holds one row for every tick, otherwise it
 * must be at least the car capacity. ticks <= 0 does nothing. */
RG_API int rg_batch_step_with_device_controls(rg_batch* b, const rg_car_controls* device_controls, int32_t ticks,
                                              int32_t control_stride, void* stream);

/* BatchSim::apply_env_commands (rocketgpu.h:1066; src/rocketgpu.cpp:2136-2218; ApplyEnvCommand env_step.hpp:
 * 5672-5758): command i for env i, applied between steps. reset_to_kickoff resets the env to kickoff (with
 * reset_scoreboard = 0: scores and tick kept and, with no seed, the match's next kickoff order; keep_boost_pads keeps
 * the pads); reset_scoreboard / reset_tick_count then clear the score / tick (only together with a reset, as in the
 * reference); new_round_bodies takes every body out of the broadphase as the game does after a goal. The host array
 * is borrowed for the call (the call synchronises the stream). kickoff_countdown_ticks != 0 is the game's countdown
 * kickoff: cars appear at their spots a tick and a half later, driving stays off for that many ticks (0xFFFF: until
 * the game's countdown timers end it, about 482 ticks), the ball starts awake at the game's drop height. */
RG_API int rg_batch_apply_env_commands(rg_batch* b, const rg_env_command* host_commands, size_t count, void* stream);
/* BatchSim::apply_env_commands_device (rocketgpu.h:1067): as above with a device array, asynchronous. */
RG_API int rg_batch_apply_env_commands_device(rg_batch* b, const rg_env_command* device_commands, size_t count,
                                              void* stream);
/* BatchSim::step_with_device_commands (rocketgpu.h:1077; src/rocketgpu.cpp:2554-2575): as
 * rg_batch_step_with_device_controls, and at the start of tick t env e first applies
 * device_commands[t * command_stride + e] (StepEnvPreTickEnv, env_step.hpp:6701-6749); command_stride must be at
 * least env_count. Refused commands are reported as for rg_batch_apply_env_commands_device. */
RG_API int rg_batch_step_with_device_commands(rg_batch* b, const rg_car_controls* device_controls,
                                              int32_t control_stride, const rg_env_command* device_commands,
                                              int32_t command_stride, int32_t ticks, void* stream);
/* Episode resets for training loops, on the device. No counterpart in BatchSim: the reference's own benchmark makes
 * the same decisions on the host between steps (tools/bench_cpp.cpp:104-112). Writes device_commands[e] for every
 * env: a fresh-episode reset (reset_to_kickoff = reset_scoreboard = reset_tick_count = 1, kickoff_seed 0) when the
 * env's score is non-zero (a goal this episode) or no car has touched the ball for no_touch_ticks ticks, else an
 * all-zero command; pass the array to the next rg_batch_step_with_device_commands (stride env_count, first tick).
 * Touches are seen through each car's latest_touch_tick changing between calls. init != 0 starts the episode clocks
 * instead (writes all-zero commands): each env's clock starts at an age in [0, no_touch_ticks) drawn from
 * stagger_seed (0: age 0), so resets spread out over the ticks. The batch keeps the clocks (16 bytes per env). */
RG_API int rg_batch_episode_commands(rg_batch* b, int32_t no_touch_ticks, uint64_t stagger_seed, int32_t init,
                                     rg_env_command* device_commands, void* stream);

/* How steps launch (no counterpart in the reference, whose tick-loop graph cache is internal, src/rocketgpu_cuda.cu:
 * 3764-3876): threads per block of the per-arena kernels and of the per-car kernels (32, 64, 128 or 256; defaults
 * 32 and 64), and use_graphs != 0 to capture each distinct step (same controls and commands pointers, strides and
 * tick count) into a CUDA graph on first use and replay it after (up to 16 kept; a change of car counts, pads,
 * kickoff seed, meshes or launch config drops them). Results do not depend on any of these. rocketgpu_b200.autotune
 * picks them by timing. While phase timing is on, steps launch without graphs. */
typedef struct rg_launch_config {
    int32_t arena_threads, car_threads, use_graphs, reserved;
} rg_launch_config;
RG_API int rg_batch_set_launch_config(rg_batch* b, const rg_launch_config* config);
RG_API int rg_batch_get_launch_config(const rg_batch* b, rg_launch_config* config);

/* Per-kernel device time of the stepping path, for profiling (no counterpart in the reference). While enabled, every
 * tick of a car step records CUDA events on the step's stream around its six kernels (arena begin, car tick start,
 * car vehicle update, arena finish, car post-tick, arena tail). rg_batch_phase_times waits for the last event, returns
 * the device milliseconds of each kernel summed over the ticks since enabling or the previous call (out_ms[6]) and
 * the tick count, and starts a new sum. Enabling or disabling also starts a new sum. */
RG_API int rg_batch_phase_timing(rg_batch* b, int32_t enable);
RG_API int rg_batch_phase_times(rg_batch* b, float* out_ms, int64_t* out_ticks);

/* BatchSim::synchronize (rocketgpu.h:1083). Also reports a CUDA error from an earlier launch. */
RG_API int rg_batch_synchronize(rg_batch* b, void* stream);

/* BatchSim::set_physics_event_stream (rocketgpu.h:1015; src/rocketgpu.cpp:2896-2906, in the Python binding's form,
 * python/rocketgpu_bindings.cpp:832-845): device arrays records[env_count * capacity_per_env] and windows[env_count].
 * Every tick stamps each arena's window with its tick and appends that tick's events in the reference's order; a full
 * window sets overflow. The caller clears the counts between reads. goal_only keeps goals only. Null arrays and 0
 * turn the stream off. Synchronise before freeing the arrays (captured step graphs are dropped here). */
RG_API int rg_batch_set_physics_event_stream(rg_batch* b, rg_physics_event* records, rg_physics_event_window* windows,
                                             uint32_t capacity_per_env, int32_t goal_only);

/* Arenas on different geometries in one batch. The reference takes one geometry per BatchSim (ArenaLayout,
 * rocketgpu.h:943-959), so a mix of arenas needs one BatchSim per mesh there; here one batch holds up to 255 meshes.
 * rg_batch_add_mesh uploads another layout's mesh and returns its index (the create-time mesh is 0);
 * rg_batch_set_arena_meshes sets arena i's mesh to host_mesh_index[i] for i < count (initially every arena is on mesh
 * 0). An arena's results are those of the same arena in a batch created with its mesh. */
RG_API int rg_batch_add_mesh(rg_batch* b, const rg_arena_layout* layout, int32_t* mesh_index);
RG_API int rg_batch_set_arena_meshes(rg_batch* b, const uint8_t* host_mesh_index, size_t count, void* stream);

/* The arena tables rg_batch_create builds from a layout, for inspection: per triangle (caller order) 16 floats
 * a, b, c, normal (Bullet units, uu / 50), the three internal-edge angles and the edge flags (as a float), and the
 * BVH leaf order (caller triangle index of each leaf in the order queries visit them). Host only. Returns the
 * triangle count (tables written up to `cap` triangles) or -1 on error (rg_last_error). */
RG_API int64_t rg_arena_mesh_tables(const rg_arena_layout* layout, float* out_tri16, int32_t* out_leaf_order,
                                    int64_t cap);

/* The reference's single-precision transcendental routines as the tick evaluates them (reference
 * include/rocketgpu/detail/math.hpp:39-457: UCRT-compatible sinf, cosf, atan2f, powf), for host code that must
 * reproduce the tick's arithmetic (e.g. a config's cached drag factor). */
RG_API float rg_ucrt_sinf(float x);
RG_API float rg_ucrt_cosf(float x);
RG_API float rg_ucrt_atan2f(float y, float x);
RG_API float rg_ucrt_powf(float x, float y);

/* Device arrays (reference DeviceView, rocketgpu.h:961-986); non-owning, valid until rg_batch_destroy. */
typedef struct rg_device_view {
    void* ball_states;       /* rg_ball_state[env_count] */
    void* env_states;        /* rg_env_state[env_count] */
    int32_t* env_car_count;  /* [env_count] */
    void* car_states;        /* rg_car_state[car_capacity] */
    void* boost_pad_states;  /* rg_boost_pad_state[pad_capacity] */
    void* controls;          /* rg_car_controls[car_capacity] */
    void* car_configs;       /* rg_car_config[car_capacity] */
    uint8_t* teams;          /* [car_capacity], 0 blue / 1 orange */
    void* wheel_runtime;     /* per car slot, 292 B (the reference's WheelRuntimeState layout), read-only */
} rg_device_view;
RG_API int rg_batch_device_view(rg_batch* b, rg_device_view* out);

/* The internal state blob (reference BatchSim internal_state_layout / download_internal_state /
 * upload_internal_state, python/rocketgpu_bindings.cpp:1002-1060): the device state a batch keeps beyond the public
 * structs, as consecutive named sections (this build's own layout): wheel_runtime, ball_world, broadphase,
 * car_world, ball_car, car_pairs (the persistent contact state) and car_stages (the last tick's per-car stages, for
 * inspection). rg_batch_internal_state_layout gives section `index`'s name and bytes (out_of_range past the last);
 * the blob is their concatenation. Download then upload restores a batch's internal state exactly (with the public
 * arrays, a whole snapshot); both synchronise the stream. */
RG_API int rg_batch_internal_state_layout(rg_batch* b, int32_t index, const char** name, int64_t* bytes);
RG_API int rg_batch_download_internal_state(rg_batch* b, void* host, void* stream);
RG_API int rg_batch_upload_internal_state(rg_batch* b, const void* host, void* stream);

/* State arrays by name, as the reference's Python binding moves them (download_state_array / upload_state_array,
 * python/rocketgpu_bindings.cpp:958-1000): name is "car_states", "ball_states", "env_states", "boost_pad_states" or
 * (upload only) "controls"; host holds `count` raw structs. preserve_internal != 0 uploads cars and balls as they
 * are (the reference's StateUploadMode::PreserveInternal); 0 canonicalises them as rg_batch_upload_car_states /
 * rg_batch_upload_ball_states do (PublicState). An unknown name is invalid_argument. Both synchronise the stream. */
RG_API int rg_batch_upload_state_array(rg_batch* b, const char* name, const void* host, size_t count,
                                       int32_t preserve_internal, void* stream);
RG_API int rg_batch_download_state_array(rg_batch* b, const char* name, void* host, size_t count, void* stream);

/* ---- serving ------------------------------------------------------------------------------------------------------
 * A serving loop for many RL clients on one GPU. No counterpart in the reference (which steps one BatchSim per call
 * under a process-wide lock, src/rocketgpu_cuda.cu:2868-2916). The server owns a pool of arena slots sized at open
 * from an HBM budget; each client owns a contiguous range of slots, created at kickoff as a BatchSim of its own
 * (its arenas' RNG draws and car ids are numbered within the client), and submits step requests of 1 to 8 ticks
 * with the controls of every tick. A worker thread runs the pool in rounds of one tick over exactly the arenas whose
 * request has ticks left, admitting new requests between rounds (continuous batching; policy 1 admits a new batch
 * only when the previous one has finished: static batching, for comparison). A client's results are bitwise those
 * of its arenas stepped alone in a BatchSim with the same controls. Status 5 (RG_BUSY): no room for a client now. */
#define RG_BUSY 5
typedef struct rg_server rg_server;
typedef struct rg_server_config {
    int32_t max_arenas;        /* slot count ceiling (0: the budget alone decides) */
    int32_t policy;            /* 0 continuous batching, 1 static batching */
    int64_t hbm_budget_bytes;  /* device bytes the slots may take (0: max_arenas alone decides) */
} rg_server_config;
typedef struct rg_server_stats {
    int64_t capacity, used, slot_bytes, clients, rounds, arena_ticks, completed;
    double busy_s;             /* device-busy seconds of the rounds */
} rg_server_stats;
/* sim: the pool's config (env_count ignored; max_cars_per_env 1..6, kickoff_settled 0). */
RG_API int rg_server_open(const rg_server_config* server_config, const rg_sim_config* sim,
                          const rg_arena_layout* layout, int device, rg_server** out);
/* Stops the worker after the admitted requests finish, drops queued ones, frees everything. */
RG_API void rg_server_close(rg_server* s);
/* Creates `arenas` arenas for a client: car_counts[arenas], teams[arenas * max_cars] (null: all blue),
 * configs[arenas * max_cars] (null: default body), reset to kickoff with kickoff_seed. RG_BUSY when no free range. */
RG_API int rg_server_client_open(rg_server* s, int32_t arenas, const int32_t* car_counts, const uint8_t* teams,
                                 const rg_car_config* configs, uint64_t kickoff_seed, int32_t* client);
/* Waits for the client's admitted request (if any) to finish, drops its queued and unpolled requests, frees its
 * slots. */
RG_API int rg_server_client_close(rg_server* s, int32_t client);
/* Queues a request: `ticks` in [1, 8], host_controls[ticks][arenas * max_cars] (copied during the call). A client's
 * requests run in submission order. */
RG_API int rg_server_submit(rg_server* s, int32_t client, int32_t ticks, const rg_car_controls* host_controls,
                            int64_t* request);
/* Waits up to wait_ms for the request; *done = 1 once finished, and then the client's car states
 * [arenas * max_cars], ball states and env states [arenas] after its last tick are copied to the non-null outputs,
 * *latency_s (if non-null) is submit-to-finish seconds, and the request is released. */
RG_API int rg_server_poll(rg_server* s, int64_t request, int32_t wait_ms, rg_car_state* cars_out,
                          rg_ball_state* balls_out, rg_env_state* envs_out, int32_t* done, double* latency_s);
RG_API int rg_server_get_stats(rg_server* s, rg_server_stats* out);

/* Steps ball-only arenas whose states live in caller-owned device memory, without allocating any device memory.
 * No counterpart in the reference: an addition of this library.
 *
 * For callers that cannot call cudaMalloc when they step: a process whose device memory is owned by another
 * framework's pool, a loop that must not pay the implicit synchronisation an allocation can cause, or code stepping
 * while someone else captures a stream. The batch `b` (created beforehand, when allocation was allowed) supplies
 * the arena mesh and the config; dev_balls / dev_envs (rg_ball_state[env_count], rg_env_state[env_count], device
 * pointers, updated in place) are the arenas stepped, `ticks` ticks each, on `stream`.
 *
 * The contact manifolds the tick keeps between ticks go to one fixed array compiled into the library (capacity 4096
 * arenas, about 1.1 MB, held on every GPU that loads the library until the process exits); env_count above 4096 is
 * rejected (status 3). All calls share that array and it keeps what the last call left: reset_manifolds != 0 clears
 * the first env_count entries before stepping (do so whenever these arenas were not the ones stepped last); 0
 * continues from the previous call's manifolds. Calls that overlap on the GPU race on the array: serialise them
 * (one stream, or events). The first call on a device looks up the array's device address (cudaGetSymbolAddress)
 * with that device current; make that first call before any stream capture. */
RG_API int rg_batch_step_static_scratch(rg_batch* b, rg_ball_state* dev_balls, rg_env_state* dev_envs,
                                        int32_t env_count, int32_t ticks, int32_t reset_manifolds, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ROCKETGPU_B200_H */
