// Kickoff reset of one arena: the env's kickoff bookkeeping (the match's shuffled kickoff spots and respawn order),
// the ball at its kickoff rest, every pad active, controls cleared, and each car at its team's kickoff spot
// (reference ResetEnvToKickoff, include/rocketgpu/detail/step/arena_ball.hpp:2827-3085, as BatchSim::reset_to_kickoff
// runs it: kickoff seed mode 0, no platform respawn RNG, no settled-kickoff copy, score not preserved).
#pragma once

#include "rg_car.cuh"
#include "rg_pads.cuh"

namespace rg {

constexpr float kHalfPiF = 1.57079632679489661923f;
constexpr float kSqrtHalfF = 0.7071067811865475244f;

struct SpawnPos {
    float x, y, yaw;
};
// reference SoccarKickoffSpawn (constants.hpp:38-46)
RG_HDI SpawnPos soccar_kickoff_spawn(int i) {
    switch (i) {
        case 0: return {-2048.0f, -2560.0f, kPiF * 0.25f};
        case 1: return {2048.0f, -2560.0f, kPiF * 0.75f};
        case 2: return {-256.0f, -3840.0f, kPiF * 0.50f};
        case 3: return {256.0f, -3840.0f, kPiF * 0.50f};
        default: return {0.0f, -4608.0f, kPiF * 0.50f};
    }
}

RG_HDI uint32_t rng_advance(uint32_t s) { return s * 1664525u + 1013904223u; }
RG_HDI uint32_t mix_seed(uint64_t seed, int env_idx, int extra) {
    uint64_t x = seed;
    x ^= static_cast<uint64_t>(env_idx + 0x9e3779b9U) + (x << 6U) + (x >> 2U);
    x ^= static_cast<uint64_t>(extra + 0x85ebca6bU) + (x << 13U) + (x >> 7U);
    return static_cast<uint32_t>(x & 0xffffffffu);
}
// reference BuildKickoffOrder / BuildRespawnOrder (arena_ball.hpp:2606-2640)
RG_HDI void build_kickoff_order(uint64_t seed, int env_idx, int* order) {
    int left[5] = {0, 1, 2, 3, 4};
    uint32_t state = mix_seed(seed, env_idx, 0x6b1d4f2a);
    for (int n = 5; n > 0; --n) {
        state = rng_advance(state);
        const int idx =
            static_cast<int>(static_cast<float>((state >> 16) & 0x7fffu) * (1.0f / 32768.0f) * static_cast<float>(n));
        order[5 - n] = left[idx];
        for (int i = idx; i + 1 < n; ++i) left[i] = left[i + 1];
    }
}
RG_HDI uint8_t build_respawn_order(uint64_t seed, int env_idx) {
    uint32_t left = 0x3210u;
    uint32_t state = mix_seed(seed, env_idx, 0x3c6ef372);
    uint32_t packed = 0;
    for (int n = 4; n > 0; --n) {
        state = rng_advance(state);
        const int idx =
            static_cast<int>(static_cast<float>((state >> 16) & 0x7fffu) * (1.0f / 32768.0f) * static_cast<float>(n));
        packed |= ((left >> (4 * idx)) & 0xFu) << (2 * (4 - n));
        left = (left & ((1u << (4 * idx)) - 1u)) | ((left >> (4 * (idx + 1))) << (4 * idx));
    }
    return static_cast<uint8_t>(packed);
}

RG_HDI float wrap_angle(float a) {
    while (a > kPiF) a -= 2.0f * kPiF;
    while (a < -kPiF) a += 2.0f * kPiF;
    return a;
}
// reference FromYaw (math.hpp:838-863)
RG_HDI Q4 quat_from_yaw(float yaw) {
    constexpr float kEps = 1e-6f;
    constexpr float kSin8 = 0.38268343236508977173f;
    constexpr float kCos8 = 0.92387953251128675613f;
    if (fabs_(yaw - (kPiF * 0.25f)) <= kEps) return Q4{kCos8, 0.0f, 0.0f, kSin8};
    if (fabs_(yaw + (kPiF * 0.25f)) <= kEps) return Q4{kCos8, 0.0f, 0.0f, -kSin8};
    if (fabs_(yaw - (kPiF * 0.75f)) <= kEps) return Q4{kSin8, 0.0f, 0.0f, kCos8};
    if (fabs_(yaw + (kPiF * 0.75f)) <= kEps) return Q4{kSin8, 0.0f, 0.0f, -kCos8};
    if (fabs_(yaw - kHalfPiF) <= kEps) return Q4{kSqrtHalfF, 0.0f, 0.0f, kSqrtHalfF};
    if (fabs_(yaw + kHalfPiF) <= kEps) return Q4{kSqrtHalfF, 0.0f, 0.0f, -kSqrtHalfF};
    const float h = 0.5f * yaw;
    return Q4{game_cosf(h), 0.0f, 0.0f, game_sinf(h)};
}
RG_HDI int spawn_yaw_rotator_units(float yaw) { return static_cast<int>(yaw * (32768.0f / 3.14159274f) + 0.5f); }
// reference SeedCarBasisFromSpawnRotator (math.hpp:1478-1490)
RG_HDI void seed_car_basis_from_spawn(CarState& c, int blue_yaw, bool orange) {
    Q4 q = ue3_quat_from_yaw(blue_yaw);
    if (orange) {
        const Q4 h = ue3_quat_from_yaw(32768);
        q = Q4{((h.w * q.w - h.x * q.x) - h.y * q.y) - h.z * q.z, ((h.w * q.x + h.x * q.w) + h.y * q.z) - h.z * q.y,
               ((h.w * q.y + h.y * q.w) + h.z * q.x) - h.x * q.z, ((h.w * q.z + h.z * q.w) + h.x * q.y) - h.y * q.x};
    }
    game_basis_from_rot(q, c.basis_forward, c.basis_right, c.basis_up);
    c.basis_authoritative = 1;
}
// reference ResetCarCommonState (arena_ball.hpp:2478-2538)
RG_HDI void reset_car_common(CarState& c, float spawn_boost) {
    c.restored_inv_inertia_valid = 0;
    car_set_vel_bt(c, V3{0.0f, 0.0f, 0.0f});
    c.ang_vel = V3{0.0f, 0.0f, 0.0f};
    memset(&c.world_contact, 0, sizeof(c.world_contact));
    c.flip_rel_torque = V3{0.0f, 0.0f, 0.0f};
    c.boost = spawn_boost;
    c.boost_amount = spawn_boost / 100.0f;
    c.jump_time = c.flip_time = c.internal_jump_time = c.internal_flip_time = 0.0f;
    c.flip_timer_live = 1;
    c.air_time = c.air_time_since_jump = c.boosting_time = c.time_since_boosted = 0.0f;
    c.supersonic_time = c.handbrake_val = c.auto_flip_timer = c.auto_flip_torque_scale = 0.0f;
    c.demo_respawn_timer = 0.0f;
    c.tick_count_since_update = 0;
    c.is_on_ground = 1;
    c.air_state = 0;
    c.rlbotv5_dodged = 0;
    c.rlbotv5_boost_hold = 0;
    c.dodge_timeout = -1.0f;
    c.dodge_elapsed = c.dodge_dir_x = c.dodge_dir_y = 0.0f;
    for (int i = 0; i < 4; ++i) c.wheels_with_contact[i] = 0;
    c.has_jumped = c.has_double_jumped = c.has_flipped = c.is_flipping = c.is_jumping = 0;
    c.jump_hold_broken = c.is_boosting = c.is_supersonic = c.is_auto_flipping = c.is_demoed = c.just_respawned = 0;
    c.car_contact.other_car_id = 0;
    c.car_contact.cooldown_timer = 0.0f;
    c.vel_impulse_cache = c.vel_impulse_cache_bt = V3{0.0f, 0.0f, 0.0f};
    c.pending_bump_count = 0;
    memset(&c.ball_hit_info, 0, sizeof(c.ball_hit_info));
    memset(&c.last_controls, 0, sizeof(c.last_controls));
    c.boost_pad_touching = 0;
    c.driving_disabled = 0;
    c.respawn_slot_override_plus1 = 0;
    c.pad_frame_pos_valid = 0;
}
// reference PlaceCarAtKickoffSpawn (arena_ball.hpp:2540-2560); team 0 blue, 1 orange
RG_HDI void place_car_at_kickoff_spawn(CarState& c, int team, SpawnPos spawn, float z, float boost) {
    float x = spawn.x, y = spawn.y, yaw = spawn.yaw;
    if (team == 1) {
        x = -x;
        y = -y;
        yaw += kPiF;
    }
    car_set_pos_bt(c, V3{x, y, z} * kUuToBt);
    c.rot = quat_from_yaw(wrap_angle(yaw));
    seed_car_basis_from_spawn(c, spawn_yaw_rotator_units(spawn.yaw), team == 1);
    reset_car_common(c, boost);
}

// reference PendKickoffSpawn (arena_ball.hpp:2769-2773): at a game-spawn kickoff the car waits demolished for a tick
// and a half, then respawns at its kickoff spot
RG_HDI void pend_kickoff_spawn(CarState& c, int spot, float tick_dt) {
    c.is_demoed = 1;
    c.demo_respawn_timer = 1.5f * tick_dt;
    c.respawn_slot_override_plus1 = static_cast<uint8_t>(kKickoffSpawnOverridePlus1 + spot);
}

// reference PlaceCarAtWorldSpawn (arena_ball.hpp:2579-2585): a custom arena's spawn, pos.z the ground
RG_HDI void place_car_at_world_spawn(CarState& c, V3 pos, float yaw, float z, float boost) {
    car_set_pos_bt(c, V3{pos.x, pos.y, pos.z + z} * kUuToBt);
    c.rot = quat_from_yaw(wrap_angle(yaw));
    seed_car_basis_from_spawn(c, spawn_yaw_rotator_units(yaw), false);
    reset_car_common(c, boost);
}

// reference ResetBall(ball, Soccar, game_spawn, rules) (arena_ball.hpp:2775-2815): a game spawn (the countdown's
// kickoff) puts the ball at the height the game drops it from, awake
RG_HDI void reset_kickoff_ball(BallState& b, const ArenaRules* rules = nullptr, bool game_spawn = false) {
    b.pos_bt = V3{0.0f, 0.0f, 93.15f} * kUuToBt;
    b.pos = b.pos_bt * 50.0f;
    b.rot = Q4{1.0f, 0.0f, 0.0f, 0.0f};
    b.basis_forward = V3{1.0f, 0.0f, 0.0f};
    b.basis_right = V3{0.0f, 1.0f, 0.0f};
    b.basis_up = V3{0.0f, 0.0f, 1.0f};
    b.basis_authoritative = 1;
    b.vel_bt = V3{0.0f, 0.0f, 0.0f};
    b.vel = b.vel_bt * 50.0f;
    b.ang_vel = V3{0.0f, 0.0f, 0.0f};
    b.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
    b.vel_impulse_cache_bt = V3{0.0f, 0.0f, 0.0f};
    b.tick_count_when_extra_impulse_applied = 0;
    b.tick_count_since_update = 0;
    b.hs_y_target_dir = 0.0f;
    b.hs_cur_target_speed = 2900.0f;
    b.hs_time_since_hit = 0.0f;
    b.ds_charge_level = 1;
    b.ds_accumulated_hit_force = 0.0f;
    b.ds_y_target_dir = 0.0f;
    for (int i = 0; i < 4; ++i) b.ds_flags[i] = 0;
    b.ds_last_damage_tick = 0;
    b.sleeping = 0;
    b.deactivation_time = 0.0f;
    b.constrained_2d = 0;
    if (rules) {
        const V3 p = rules->ball_spawn;
        b.pos_bt = V3{p.x, p.y, game_spawn ? p.z + (100.487184524536f - 92.75f) : p.z} * kUuToBt;
        b.pos = b.pos_bt * 50.0f;
        b.sleeping = game_spawn ? 0 : 1;
    } else if (game_spawn) {
        b.pos_bt = V3{0.0f, 0.0f, 2.0097436904907227f};
        b.pos = b.pos_bt * 50.0f;
    } else {
        b.pos_bt = V3{0.0f, 0.0f, 92.75f} * kUuToBt;
        b.pos = b.pos_bt * 50.0f;
        b.sleeping = 1;
    }
}

// reference KickoffSpotPreferred / PreferKickoffSpotForShortTeam (arena_ball.hpp:2632-2653): a team with fewer cars
// than the other also gets the best of the spots a full team would take (nearest the ball, then the left diagonal,
// then the farther back).
RG_HDI bool kickoff_spot_preferred(SpawnPos a, SpawnPos b) {
    const float da = a.x * a.x + a.y * a.y;
    const float db = b.x * b.x + b.y * b.y;
    if (da != db) return da < db;
    const bool left_a = a.x * a.y < 0.0f;
    const bool left_b = b.x * b.y < 0.0f;
    if (left_a != left_b) return left_a;
    return (a.y < 0.0f ? -a.y : a.y) > (b.y < 0.0f ? -b.y : b.y);
}
// `spots`: the five kickoff spots of the blue side (a custom arena's blue kickoff positions, yaw unused)
RG_HDI void prefer_kickoff_spot_for_short_team(int* order, int team_count, const SpawnPos* spots) {
    constexpr int kMaxTeamSize = 4;
    if (team_count <= 0 || team_count >= kMaxTeamSize) return;
    int best = 0;
    for (int i = 1; i < kMaxTeamSize; ++i)
        if (kickoff_spot_preferred(spots[order[i]], spots[order[best]])) best = i;
    if (best < team_count) return;
    const int spot = order[best];
    order[best] = order[team_count - 1];
    order[team_count - 1] = spot;
}

// How a kickoff reset treats the match (the EnvCommand fields of the reference's ResetEnvToKickoff call,
// env_step.hpp:5735-5752). The defaults are BatchSim::reset_to_kickoff's: a new match.
// A car's state at its kickoff spot once the game's countdown has run, with its wheel record (reference
// KickoffSettledRow, arena_geometry.hpp:1580-1583).
struct KickoffSettledRow {
    CarState car;
    WheelRuntime wheels;
};
// A non-countdown kickoff puts each car (whose config and team have a recorded entry) into the recorded state of its
// spot, keeping the car's event and touch history (reference SettleKickoffCar and the kickoff history fields,
// arena_ball.hpp:2698-2767; the CPU build's word copy takes every other byte, driving_disabled included).
RG_HDI void settle_kickoff_car(CarState& c, WheelRuntime& w, int32_t entry, int spot, const TickConfig& tc) {
    if (tc.settled_rows == nullptr || spot >= tc.settled_spawns || entry < 0) return;
    const KickoffSettledRow& row = tc.settled_rows[static_cast<size_t>(entry) * tc.settled_spawns + spot];
    uint8_t bumps[7], demos[7];
    memcpy(bumps, c.bump_event_bumps, sizeof(bumps));
    memcpy(demos, c.bump_event_demos, sizeof(demos));
    const uint64_t prev_ball = c.previous_ball_contact_start, last_ball = c.last_ball_contact_start,
                   last_world = c.last_world_surface_contact, world_after_prev = c.first_world_after_previous_ball,
                   world_after_last = c.first_world_after_last_ball, flip_or_jump = c.last_flip_or_jump_start,
                   dir_flip = c.last_directional_flip_start, touch_tick = c.latest_touch_tick;
    const uint8_t started_with_world = c.last_ball_started_with_world, foj_last = c.flip_or_jump_last_tick;
    const V3 touch_loc = c.latest_touch_location, touch_normal = c.latest_touch_normal;
    c = row.car;
    memcpy(c.bump_event_bumps, bumps, sizeof(bumps));
    memcpy(c.bump_event_demos, demos, sizeof(demos));
    c.previous_ball_contact_start = prev_ball;
    c.last_ball_contact_start = last_ball;
    c.last_world_surface_contact = last_world;
    c.first_world_after_previous_ball = world_after_prev;
    c.first_world_after_last_ball = world_after_last;
    c.last_flip_or_jump_start = flip_or_jump;
    c.last_directional_flip_start = dir_flip;
    c.last_ball_started_with_world = started_with_world;
    c.flip_or_jump_last_tick = foj_last;
    c.latest_touch_tick = touch_tick;
    c.latest_touch_location = touch_loc;
    c.latest_touch_normal = touch_normal;
    w = row.wheels;
}

struct KickoffReset {
    bool preserve_score = false;  // keep scores, tick and last scorer; with seed 0, the match's next kickoff
    uint8_t seed_mode = 0;        // 0: spot order from the seed (0: from the reset count); 2: as 0 with seed 0;
                                  // 3: no shuffle, a team's nth car takes kickoff spot n
    bool keep_pads = false;       // keep the pads and their timers
    bool game_spawn = false;      // the countdown's kickoff: cars appear at their spots a tick and a half later
};

// The car slot visited k-th under `env`'s visit order (reference CarVisitSlot, rocketgpu.h:575-581).
RG_HD int reset_visit_slot(const EnvState& env, int k, int count) {
    if (env.car_visit_order_mode == 1 || env.car_visit_order_mode == 3)
        return static_cast<int>((env.car_visit_order_packed >> (4 * k)) & 0xFu);
    return env.car_visit_order_mode == 2 ? count - 1 - k : k;
}

// The whole arena (reference ResetEnvToKickoffState + ResetKickoffBall + ResetBoostPads + ResetKickoffCar,
// arena_ball.hpp:2846-3085, with no platform respawn RNG, no settled-kickoff copy and no countdown). `teams` are the
// arena's max_cars slot teams (0 blue, 1 orange); `scratch` is its persistent ball contact state, cleared as the
// reference clears its solver scratch.
// wheels and settled_entry (the arena's slots' settle entries, null when settling is off) are the arena's.
RG_HDI void reset_env_to_kickoff(int env_idx, uint64_t seed, EnvState& env, BallState& ball, BallWorldScratch& scratch,
                                 CarState* cars, WheelRuntime* wheels, const CarConfig* cfgs, CarControls* controls,
                                 PadState* pads, const PadLayout& L, const uint8_t* teams, int count, int max_cars,
                                 const TickConfig& tc, const int32_t* settled_entry,
                                 const KickoffReset& how = KickoffReset{}) {
    memset(&scratch, 0, sizeof(scratch));
    const EnvState saved = env;
    EnvState next;
    memset(&next, 0, sizeof(next));
    next.last_scored_team = -1;
    next.car_visit_order_mode = 3;
    next.car_visit_present_mask = 0xFF;
    next.car_visit_order_packed = 0x76543210u;
    next.frame_frac_prev = 0.5f;
    next.kickoff_resets = static_cast<uint8_t>(saved.kickoff_resets + 1);
    next.kickoff_match_order = saved.kickoff_match_order;
    next.kickoff_match_index = saved.kickoff_match_index;
    next.respawn_match_order = saved.respawn_match_order;
    const bool no_seed = how.seed_mode == 2 || (how.seed_mode == 0 && seed == 0);
    const bool next_kickoff = no_seed && how.preserve_score && (saved.kickoff_match_order & 0x8000u) != 0;
    if (no_seed) seed = saved.kickoff_resets * 0x9e3779b97f4a7c15ull;
    next.car_visit_order_mode = saved.car_visit_order_mode;
    next.car_visit_order_packed = saved.car_visit_order_packed;
    if (saved.car_visit_order_mode == 3) {
        next.car_visit_order_packed = 0x76543210u;
        next.car_visit_present_mask = 0xFFu;
    }
    next.frame_ticks = saved.frame_ticks;
    next.frame_frac_prev = saved.frame_frac_prev;
    if (how.preserve_score) {
        next.blue_score = saved.blue_score;
        next.orange_score = saved.orange_score;
        next.tick = saved.tick;
        next.last_scored_team = saved.last_scored_team;
    }
    int blue_count = 0, orange_count = 0;
    for (int k = 0; k < count; ++k) {
        if (teams[reset_visit_slot(next, k, count)] == 0)
            ++blue_count;
        else
            ++orange_count;
    }
    int kickoff_order[5] = {0, 1, 2, 3, 4};
    if (how.seed_mode == 3) {
    } else if (next_kickoff) {
        for (int j = 0; j < 5; ++j)
            kickoff_order[j] = (saved.kickoff_match_order >> (3 * ((saved.kickoff_match_index + j) % 5))) & 7;
    } else {
        build_kickoff_order(seed, env_idx, kickoff_order);
    }
    if (how.seed_mode != 3) {
        if (next_kickoff) {
            next.kickoff_match_index = static_cast<uint8_t>((saved.kickoff_match_index + 1) % 5);
        } else {
            uint32_t packed = 0x8000u;
            for (int j = 0; j < 5; ++j) packed |= static_cast<uint32_t>(kickoff_order[j]) << (3 * j);
            next.kickoff_match_order = static_cast<uint16_t>(packed);
            next.kickoff_match_index = 1;
            next.respawn_match_order = build_respawn_order(seed, env_idx);
        }
    }
    int team_order[2][5];
    for (int j = 0; j < 5; ++j) team_order[0][j] = team_order[1][j] = kickoff_order[j];
    const ArenaRules* rules = tc.rules;
    if (next_kickoff && blue_count != orange_count) {
        SpawnPos spots[5];
        for (int i = 0; i < 5; ++i)
            spots[i] = rules ? SpawnPos{rules->kickoff_pos[0][i].x, rules->kickoff_pos[0][i].y, 0.0f}
                             : soccar_kickoff_spawn(i);
        const int short_team = blue_count < orange_count ? 0 : 1;
        prefer_kickoff_spot_for_short_team(team_order[short_team], short_team == 0 ? blue_count : orange_count, spots);
    }
    env = next;
    uint32_t order_bits[2] = {0, 0};
    for (int t = 0; t < 2; ++t)
        for (int i = 0; i < 5; ++i) order_bits[t] |= static_cast<uint32_t>(team_order[t][i]) << (3 * i);

    reset_kickoff_ball(ball, rules, how.game_spawn);
    if (!how.game_spawn && tc.settled_rows != nullptr && tc.settled_ball != nullptr) ball = *tc.settled_ball;
    if (pads && !how.keep_pads) {
        for (int p = 0; p < L.count; ++p) {
            PadState& pad = pads[p];
            pad.cooldown = 0.0f;
            pad.is_active = 1;
            pad.is_big = L.is_big[p];
            pad.prev_locked_car_id = 0;
            pad.cur_locked_car_id = 0;
            pad.pickup_frac_q = 32768;
        }
    }
    for (int i = 0; i < max_cars; ++i) memset(&controls[i], 0, sizeof(CarControls));
    for (int i = 0; i < count; ++i) {
        // the car's place among its team's cars in visit order picks its kickoff spot (FindKickoffCarSpot)
        const int team = teams[i];
        int nth = 0;
        bool found = false;
        for (int k = 0; k < count && !found; ++k) {
            const int s = reset_visit_slot(env, k, count);
            if (s == i) {
                found = true;
            } else if (teams[s] == team) {
                ++nth;
            }
        }
        if (!found) continue;
        const int spot = nth < 5 ? static_cast<int>((order_bits[team == 0 ? 0 : 1] >> (3 * nth)) & 7u) : nth;
        if (rules) {
            // a custom arena's spots (reference PlaceKickoffCar with ArenaRules, arena_ball.hpp:2998-3007)
            const int t = team == 0 ? 0 : 1;
            const int r = (nth - 5) % 4;
            const float step = 250.0f * static_cast<float>((nth - 5) / 4);
            V3 pos = nth < 5 ? rules->kickoff_pos[t][spot] : rules->respawn_pos[t][r];
            const float yaw = nth < 5 ? rules->kickoff_yaw[t][spot] : rules->respawn_yaw[t][r];
            if (nth >= 5) pos = pos - V3{game_cosf(yaw), game_sinf(yaw), 0.0f} * step;
            place_car_at_world_spawn(cars[i], pos, yaw, cfgs[i].spawn_z, tc.boost_spawn_amount);
            if (how.game_spawn && nth < 5) pend_kickoff_spawn(cars[i], spot, tc.tick_dt);
            if (!how.game_spawn && settled_entry) settle_kickoff_car(cars[i], wheels[i], settled_entry[i], spot, tc);
            continue;
        }
        SpawnPos spawn;
        if (nth >= 5) {
            // a sixth car of a team takes a respawn spot, 250 uu further back per round of four
            // (reference PlaceKickoffCar, arena_ball.hpp:2998-3015; SoccarRespawnSpawn, constants.hpp:48-55)
            const int r = (nth - 5) % 4;
            const float step = 250.0f * static_cast<float>((nth - 5) / 4);
            const float xs[4] = {-2304.0f, -2688.0f, 2304.0f, 2688.0f};
            spawn = SpawnPos{xs[r], -4608.0f + step, kHalfPiF};
        } else {
            spawn = soccar_kickoff_spawn(spot);
        }
        place_car_at_kickoff_spawn(cars[i], team, spawn, cfgs[i].spawn_z, tc.boost_spawn_amount);
        if (how.game_spawn && nth < 5) pend_kickoff_spawn(cars[i], spot, tc.tick_dt);
        if (!how.game_spawn && settled_entry) settle_kickoff_car(cars[i], wheels[i], settled_entry[i], spot, tc);
    }
}

}  // namespace rg
