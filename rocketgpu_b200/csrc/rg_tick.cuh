// One 120 Hz tick of one arena (host+device): env commands and the tick-start env state (the game's car order,
// respawn-spot picks), each car's tick start and vehicle update, the world step (ball and cars against the arena mesh
// and each other, the unified velocity and split solves, integration), each car's post-tick and the tail (pads, the
// driving countdown, ball hits, goals, render-frame timers, tick counter).
//
// Phase order and arithmetic follow the reference's per-env tick, StepEnvGeneric
// (include/rocketgpu/detail/step/env_step.hpp:7048-7180), with WorldStepSoccar (env_step.hpp:4622-5623) and
// StepEnvTail (env_step.hpp:6968-7045).
#pragma once

#include "rg_ball_car.cuh"
#include "rg_ball_world.cuh"
#include "rg_broadphase.cuh"
#include "rg_car_car.cuh"
#include "rg_car_world.cuh"
#include "rg_math.cuh"
#include "rg_pads.cuh"
#include "rg_reset.cuh"
#include "rg_vehicle.cuh"
#include "rg_mesh.h"
#include "rg_state.cuh"

namespace rg {

// Bullet activation thresholds (reference env_step.hpp:3486-3488).
constexpr float kBallLinearSleepBt = 0.8f;
constexpr float kBallAngularSleep = 1.0f;
constexpr float kDeactivationTime = 2.0f;

RG_HD void ball_set_vel_bt(BallState& b, V3 v) {
    b.vel_bt = v;
    b.vel = v * 50.0f;
}
RG_HD void ball_set_pos_bt(BallState& b, V3 p) {
    b.pos_bt = p;
    b.pos = p * 50.0f;
}

// Tick start: speed caps in uu, then the game's replicated-state quantisation of position, velocity, angular velocity
// and rotation (reference CalTickStartLimitAndQuantizeBall / CapBallSpeeds / QuantizeBallStateV3Exact,
// raycast_wheels_and_contact_prep.hpp:3751-3783, 3873-3895, 4029-4031).
RG_HDI void ball_tick_start_quantize(BallState& b, const TickConfig& c) {
    V3 vel_uu = b.vel_bt * 50.0f;
    {
        const float l2 = len2(vel_uu);
        if (l2 > c.ball_max_speed * c.ball_max_speed) {
            vel_uu = (vel_uu * (1.0f / sqrtf(l2))) * c.ball_max_speed;
            ball_set_vel_bt(b, vel_uu * (1.0f / 50.0f));
        }
    }
    {
        const float l2 = len2(b.ang_vel);
        const float m2 = c.ball_max_ang_speed * c.ball_max_ang_speed;
        if (!(l2 <= m2)) b.ang_vel = (b.ang_vel * (1.0f / sqrtf(l2))) * c.ball_max_ang_speed;
    }
    constexpr float kUuToBt = 1.0f / 50.0f;
    const V3 p = b.pos_bt * 50.0f;
    const V3 qp{quant_round_pos(p.x, 100.0f), quant_round_pos(p.y, 100.0f), quant_round_pos(p.z, 100.0f)};
    ball_set_pos_bt(b, qp * kUuToBt);
    const V3 qv{quant_trunc_offset(vel_uu.x, 100.0f), quant_trunc_offset(vel_uu.y, 100.0f),
                quant_trunc_offset(vel_uu.z, 100.0f)};
    ball_set_vel_bt(b, qv * kUuToBt);
    b.pos = qp;
    b.vel = qv;
    b.ang_vel = V3{quant_trunc_offset(b.ang_vel.x, 10000.0f), quant_trunc_offset(b.ang_vel.y, 10000.0f),
                   quant_trunc_offset(b.ang_vel.z, 10000.0f)};
    if (!b.basis_authoritative) {
        upload_basis_from_rot(b.rot, b.basis_forward, b.basis_right, b.basis_up);
        b.basis_authoritative = 1;
    }
    b.inertia_basis_forward = b.basis_forward;
    b.inertia_basis_right = b.basis_right;
    b.inertia_basis_up = b.basis_up;
    b.inertia_basis_valid = 1;
    b.rot = game_quantize_basis(b.basis_forward, b.basis_right, b.basis_up);
}

// Rigid-body velocity clamp in Bullet units, then linear drag (reference BodyDampingClampBall, env_step.hpp:2941-2956;
// ApplyBulletLinearDampingBall with the drag factor cached per config, raycast_wheels_and_contact_prep.hpp:3784-3806).
RG_HDI void ball_clamp_and_drag(BallState& b, const TickConfig& c) {
    {
        const V3 v = b.vel_bt;
        const float max_lin = c.ball_max_speed * 0.02f;
        const float vsq = (v.x * v.x + v.y * v.y) + v.z * v.z;
        if (0.0f < max_lin && max_lin * max_lin < vsq) {
            const float s = 1.0f / sqrtf(vsq);
            ball_set_vel_bt(b, V3{(v.x * s) * max_lin, (v.y * s) * max_lin, (v.z * s) * max_lin});
        }
    }
    {
        const V3 w = b.ang_vel;
        const float max_ang = c.ball_max_ang_speed;
        const float lsq = (w.x * w.x + w.y * w.y) + w.z * w.z;
        if (0.0f < max_ang && max_ang * max_ang < lsq) {
            const float s = 1.0f / sqrtf(lsq);
            b.ang_vel = V3{(w.x * s) * max_ang, (w.y * s) * max_ang, (w.z * s) * max_ang};
        }
    }
    if (c.ball_drag > 0.0f) ball_set_vel_bt(b, b.vel_bt * c.ball_drag_scale);
}

// Sleeping state at the world step's start (reference BallWakeStateAtTickStart / ResolveBallActivationAtTickStart,
// env_step.hpp:3490-3524). State 2 (just uploaded) wakes on a custom-mesh arena.
RG_HDI bool ball_resolve_activation(BallState& b) {
    if (b.sleeping == 2) b.sleeping = 0;
    if (b.sleeping == 0 && b.deactivation_time > kDeactivationTime) {
        b.sleeping = 1;
        ball_set_vel_bt(b, V3{0.0f, 0.0f, 0.0f});
        b.ang_vel = V3{0.0f, 0.0f, 0.0f};
    }
    return b.sleeping == 1;
}

// The ball's integration step: origin += vel * dt; the basis becomes authoritative (ball rotation is off in soccar,
// SimConfig::no_ball_rot; reference IntegrateBallTransformOnly, raycast_wheels_and_contact_prep.hpp:3825-3846).
RG_HDI void ball_integrate(BallState& b, float dt) {
    if (!is_zero(b.vel_bt)) ball_set_pos_bt(b, b.pos_bt + b.vel_bt * dt);
    if (!b.basis_authoritative) {
        upload_basis_from_rot(b.rot, b.basis_forward, b.basis_right, b.basis_up);
        b.basis_authoritative = 1;
    }
    b.restored_inv_inertia_valid = 0;
}

// Ball finish: the velocity impulse cache, tick counters, the 2D constraint countdown (reference FinishBallTick,
// raycast_wheels_and_contact_prep.hpp:3897-3906 with ApplyBallVelocityImpulseCache :3848-3855).
RG_HDI void ball_finish(BallState& b) {
    if (len2(b.vel_impulse_cache_bt) > 0.0f || len2(b.vel_impulse_cache) > 0.0f) {
        ball_set_vel_bt(b, b.vel_bt + b.vel_impulse_cache_bt);
        b.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
        b.vel_impulse_cache_bt = V3{0.0f, 0.0f, 0.0f};
    }
    b.inertia_basis_valid = 0;
    b.tick_count_since_update += 1;
    if (b.constrained_2d) --b.constrained_2d;
}

// Goal test against the mouth planes and the render-frame bookkeeping (reference StepEnvTail, env_step.hpp:7006-7045;
// CountdownUpdateTimers :6516-6537). The countdown's end re-enables driving of the arena's first `count` car slots.
// event_env >= 0: a goal is a goal event of that arena.
RG_HDI void env_tail(EnvState& env, BallState& b, const TickConfig& c, CarState* cars = nullptr, int count = 0,
                     int event_env = -1) {
    ball_finish(b);
    if (c.enable_scoring && c.rules) {
        // a custom arena's goals (reference ScoreArenaRulesGoals, env_step.hpp:6951-6966)
        const ArenaRules& R = *c.rules;
        for (int t = 0; t < 2; ++t) {
            const V3 lo = R.goal_min[t], hi = R.goal_max[t];
            if (dot(b.pos - R.goal_point[t], R.goal_normal[t]) >= c.ball_radius && b.pos.x >= lo.x && b.pos.y >= lo.y &&
                b.pos.z >= lo.z && b.pos.x <= hi.x && b.pos.y <= hi.y && b.pos.z <= hi.z) {
                const int scorer = t == 0 ? 1 : 0;  // the blue goal (0) scores for orange
                env.last_scored_team = scorer;
                env.goal_scored_this_tick = 1;
                if (!env.goal_latched) {
                    if (scorer == 0)
                        env.blue_score += 1;
                    else
                        env.orange_score += 1;
                }
                break;
            }
        }
        env.goal_latched = env.goal_scored_this_tick;
    } else if (c.enable_scoring) {
        const float score_threshold = c.goal_base_threshold_y + c.ball_radius;
        if (b.pos.y >= score_threshold) {
            env.last_scored_team = 0;
            env.goal_scored_this_tick = 1;
            if (!env.goal_latched) env.blue_score += 1;
        } else if (b.pos.y <= -score_threshold) {
            env.last_scored_team = 1;
            env.goal_scored_this_tick = 1;
            if (!env.goal_latched) env.orange_score += 1;
        }
        env.goal_latched = env.goal_scored_this_tick;
    }
    if (env.goal_scored_this_tick && c.events.windows && event_env >= 0) {
        // reference StepEnvTail, env_step.hpp:7026-7033
        PhysicsEvent e = new_event(kEventGoal);
        e.team = env.last_scored_team;
        e.ball_position = b.pos;
        e.ball_velocity = b.vel;
        emit_event(c.events, static_cast<uint32_t>(event_env), e);
    }
    env.frame_ticks += 1;
    const float frame_frac = c.frame_frac;
    if (frame_frac >= 0.0f) {
        const float frame_dt = (static_cast<float>(env.frame_ticks) + frame_frac - env.frame_frac_prev) * c.tick_dt;
        env.frame_ticks = 0;
        env.frame_frac_prev = frame_frac;
        if (env.countdown_phase != 0) {
            env.countdown_count += frame_dt;
            if (env.countdown_count > 1.0f) {
                if (env.countdown_phase == 1) {
                    env.countdown_phase = 2;
                    env.countdown_count = 0.0f;
                } else {
                    env.countdown_count -= 1.0f;
                    if (++env.countdown_fires == 3) {
                        env.countdown_phase = 0;
                        env.countdown_fires = 0;
                        for (int i = 0; i < count; ++i) cars[i].driving_disabled = 0;
                        b.constrained_2d = 0;
                    }
                }
            }
        }
    }
    env.tick += 1;
}

// World step, ball-only arena (reference WorldStepSoccar with count == 0, env_step.hpp:4727-5623): activation,
// arena contacts, gravity, integration and Bullet's deactivation timer.
RG_HDI void ball_world_step(BallState& b, BallWorldScratch& s, const TickConfig& c, const MeshDevice& mesh,
                            int event_env = -1) {
    const float sub_dt = c.tick_dt;  // one world substep per tick
    const bool vehicle_woke = (b.sleeping & 4u) != 0;
    b.sleeping &= 3u;
    const bool ball_sleeping = ball_resolve_activation(b);
    if (vehicle_woke) b.deactivation_time = 0.0f;
    const V3 ext_delta = ball_sleeping ? V3{0.0f, 0.0f, 0.0f} : V3{0.0f, 0.0f, c.gravity_z * sub_dt};
    const V3 solver_vel_bt = b.vel_bt;
    const bool awake = !ball_sleeping || vehicle_woke;
    // predictive contact of this tick's motion (reference ComputePredictiveContactHits, env_step.hpp:4129-4168)
    V3 pred_n{0, 0, 0};
    float pred_dist = 0.0f;
    const bool pred_hit = !(ball_sleeping && !vehicle_woke) && ball_predictive_hit(b, mesh, sub_dt, pred_n, pred_dist);
    // the persistent manifold list: last tick's predictive entry leaves, a new one is appended, the ball/mesh pair
    // enters once the ball is awake (reference BuildBulletManifoldList, arena_geometry.hpp:4864-4930)
    for (int k = 0; k < s.list_count; ++k) {
        if (s.list[k] == kListPredictive) {
            s.list[k] = s.list[--s.list_count];
            break;
        }
    }
    if (pred_hit) s.list[s.list_count++] = kListPredictive;
    {
        bool has_mesh = false;
        for (int k = 0; k < s.list_count; ++k) has_mesh = has_mesh || s.list[k] == kListMesh;
        if (!has_mesh && !(ball_sleeping && !vehicle_woke)) s.list[s.list_count++] = kListMesh;
    }
    // island sort of the listed manifolds: two entries of the ball's island come out reversed (reference
    // SortBulletManifoldListByIsland, env_step.hpp:4269-4285)
    int32_t sorted_ids[2];
    const int n_sorted = s.list_count;
    for (int k = 0; k < n_sorted; ++k) {
        const uint8_t e = n_sorted == 2 ? s.list[1 - k] : s.list[k];
        sorted_ids[k] = e == kListPredictive ? kPredictiveStaticId : 0;
    }
    bool pred_listed = false;
    for (int k = 0; k < n_sorted; ++k) pred_listed = pred_listed || sorted_ids[k] == kPredictiveStaticId;
    // arena contacts: a sleeping ball keeps its manifold untouched
    BallContactRows rows;
    rows.split_count = rows.vel_count = rows.fric_count = 0;
    if (awake) ball_mesh_contacts(b, s, c, mesh, ext_delta, solver_vel_bt, sub_dt, rows, event_env);
    if (pred_hit) ball_predictive_rows(b, c, pred_n, pred_dist, ext_delta, solver_vel_bt, sub_dt, rows);
    if (rows.vel_count || rows.fric_count) {
        V3 dl, da;
        ball_solve_velocity(rows, pred_listed, dl, da);
        ball_set_vel_bt(b, solver_vel_bt + dl);
        b.ang_vel = b.ang_vel + da;
    }
    if (rows.split_count) {
        const V3 push = ball_solve_split(rows, sorted_ids, n_sorted);
        if (!is_zero(push)) ball_set_pos_bt(b, b.pos_bt + push * sub_dt);
    }
    if (!ball_sleeping) ball_set_vel_bt(b, b.vel_bt + uu_to_bt_div(ext_delta));
    if (awake) {
        ball_integrate(b, sub_dt);
        b.sleeping = 0;
        const bool below = len2(b.vel_bt) < kBallLinearSleepBt * kBallLinearSleepBt &&
                           len2(b.ang_vel) < kBallAngularSleep * kBallAngularSleep;
        b.deactivation_time = below && !ball_sleeping ? b.deactivation_time + sub_dt : 0.0f;
    }
}

// One tick of one ball-only arena (reference StepEnvGeneric, env_step.hpp:7088-7180).
// env_idx: the arena's index for physics events.
RG_HDI void arena_tick(EnvState& env, BallState& b, BallWorldScratch& s, const TickConfig& c,
                       const MeshDevice& mesh, int env_idx = -1) {
    if (c.events.windows && env_idx >= 0) c.events.windows[env_idx].tick = env.tick;
    env.goal_scored_this_tick = 0;
    ball_tick_start_quantize(b, c);
    ball_clamp_and_drag(b, c);
    ball_world_step(b, s, c, mesh, env_idx);
    env_tail(env, b, c, nullptr, 0, env_idx);
}

// ---- arenas with cars --------------------------------------------------------------------------------------------
// One arena's cars during a tick: its max_cars slots of car state, wheel records and configs, its pads (null when the
// batch never had a car, so every pad is still at its initial state) and this tick's control row.
struct ArenaCars {
    CarState* cars;
    WheelRuntime* wheels;
    const CarConfig* cfgs;
    PadState* pads;
    const CarControls* controls;
    const uint8_t* teams;
    CarCarManifold* pairs;  // the arena's retained car-car manifolds, slot car_pair_slot(lo, hi)
    const int32_t* settled_entry;  // the slots' kickoff-settle entries, or null (settling off)
    int count, max_cars, car_base;
};

// The slot visited k-th (reference CarVisitSlot, rocketgpu.h:575-581).
RG_HD int car_visit_slot(const EnvState& env, int k, int count) {
    if (env.car_visit_order_mode == 1 || env.car_visit_order_mode == 3)
        return static_cast<int>((env.car_visit_order_packed >> (4 * k)) & 0xFu);
    if (env.car_visit_order_mode == 2) return count - 1 - k;
    return k;
}
// The game's vehicle order kept across demolitions (reference UpdateGameCarVisitOrder, rocketgpu.h:592-634).
RG_HDI void update_game_visit_order(EnvState& env, const CarState* cars, int count) {
    if (env.car_visit_order_mode != 3) return;
    int order[8];
    for (int k = 0; k < 8; ++k) order[k] = static_cast<int>((env.car_visit_order_packed >> (4 * k)) & 0xFu);
    uint32_t present = env.car_visit_present_mask;
    auto is_present = [&](int slot) { return slot < count && ((present >> slot) & 1u) != 0u; };
    auto last_present = [&]() {
        int q = -1;
        for (int k = 0; k < 8; ++k)
            if (is_present(order[k])) q = k;
        return q;
    };
    for (int s = 0; s < count && s < 8; ++s) {
        if (((present >> s) & 1u) || cars[s].is_demoed) continue;
        int p = 0;
        while (order[p] != s) ++p;
        const int dst = last_present() + 1;
        for (int k = p; k > dst; --k) order[k] = order[k - 1];
        order[dst < p ? dst : p] = s;
        present |= 1u << s;
    }
    for (int s = 0; s < count && s < 8; ++s) {
        if (!((present >> s) & 1u) || !cars[s].is_demoed) continue;
        int p = 0;
        while (order[p] != s) ++p;
        const int q = last_present();
        order[p] = order[q];
        order[q] = s;
        present &= ~(1u << s);
    }
    uint32_t packed = 0;
    for (int k = 0; k < 8; ++k) packed |= (static_cast<uint32_t>(order[k]) & 0xFu) << (4 * k);
    env.car_visit_order_packed = packed;
    env.car_visit_present_mask = static_cast<uint8_t>(present);
}

// A car's tick start (reference StepEnvPreTickCar, env_step.hpp:6751-6873): working fields back from the report
// fields, internal clocks after a state set, the demolition timer, the tick-start quantization, the pre-physics
// control logic and the rigid-body speed clamp.
// Returns the car's uu velocity right after the tick-start quantisation.
// Where a demolished car comes back: the respawn spot chosen by the arena's respawn draw (reference
// RespawnStartIndex, RespawnPlace, RespawnCar, KickoffSpawnCar, arena_ball.hpp:3092-3177).
struct RespawnCtx {
    uint64_t seed;  // the batch's last kickoff seed
    int env_idx;
    uint32_t env_tick, car_id;
    uint8_t team;
};
RG_HDI int respawn_start_index(uint64_t seed, int env_idx, uint64_t tick, uint32_t car_id) {
    uint32_t st = mix_seed(seed ^ (tick * 0x9e3779b97f4a7c15ull), env_idx, static_cast<int>(car_id * 0x45d9f3bu));
    st = rng_advance(st);
    return static_cast<int>(static_cast<float>((st >> 16) & 0x7fffu) * (1.0f / 32768.0f) * 4.0f);
}
RG_HDI SpawnPos soccar_respawn_spawn(int i) {
    switch (i) {
        case 0: return SpawnPos{-2304.0f, -4608.0f, kPiF * 0.5f};
        case 1: return SpawnPos{-2688.0f, -4608.0f, kPiF * 0.5f};
        case 2: return SpawnPos{2304.0f, -4608.0f, kPiF * 0.5f};
        default: return SpawnPos{2688.0f, -4608.0f, kPiF * 0.5f};
    }
}
// The ground point and yaw of a team's respawn spot, moved 192 uu in one of eight directions around the spot's facing
// when dir >= 0 (reference RespawnPlace, arena_ball.hpp:3098-3122).
RG_HDI void respawn_place(int team, int spot, int dir, const ArenaRules* rules, V3& ground, float& yaw) {
    const bool blue = team == 0;
    float fx = 0.0f, fy = blue ? 1.0f : -1.0f;
    if (rules) {
        const int t = blue ? 0 : 1;
        ground = rules->respawn_pos[t][spot & 3];
        yaw = rules->respawn_yaw[t][spot & 3];
        const Q4 q = quat_from_yaw(wrap_angle(yaw));
        fx = q.w * q.w - q.z * q.z;
        fy = 2.0f * q.w * q.z;
    } else {
        const SpawnPos s = soccar_respawn_spawn(spot & 3);
        ground = V3{s.x, blue ? s.y : -s.y, 0.0f};
        yaw = s.yaw + (blue ? 0.0f : kPiF);
    }
    if (dir >= 0) {
        constexpr float k = 0.70710677f;
        const int d = dir & 7;
        const float ux = d == 0 ? 1.0f : (d == 1 || d == 7) ? k : (d == 2 || d == 6) ? 0.0f : (d == 3 || d == 5) ? -k : -1.0f;
        const float uy = (d == 0 || d == 4) ? 0.0f : (d == 1 || d == 3) ? k : d == 2 ? 1.0f : d == 6 ? -1.0f : -k;
        ground.x += 192.0f * (fx * ux - fy * uy);
        ground.y += 192.0f * (fx * uy + fy * ux);
    }
}

// Each car body's stored mesh bounds by CarConfig::body, unknown bodies reading the Octane's (reference
// CarBodyMeshBounds, env_step.hpp:6546-6553).
namespace body_bounds_host {
#define RG_BODY_BOUNDS_TABLE(name, n) static const float name[n][6]
#include "rg_body_bounds.inc"
#undef RG_BODY_BOUNDS_TABLE
}  // namespace body_bounds_host
#if defined(__CUDACC__)
namespace body_bounds_dev {
#define RG_BODY_BOUNDS_TABLE(name, n) __device__ static const float name[n][6]
#include "rg_body_bounds.inc"
#undef RG_BODY_BOUNDS_TABLE
}  // namespace body_bounds_dev
#endif
constexpr int kBodyCount = static_cast<int>(sizeof(body_bounds_host::kBodyMeshBounds) / sizeof(float[6]));
constexpr int kBodyOctane = 147;
RG_HDI const float* body_mesh_bounds(int body) {
    const int b = body >= 0 && body < kBodyCount ? body : kBodyOctane;
#if defined(__CUDA_ARCH__)
    return body_bounds_dev::kBodyMeshBounds[b];
#else
    return body_bounds_host::kBodyMeshBounds[b];
#endif
}

// Whether a spawn point lies within 48 uu of an axis-aligned box (reference SpawnSpotNearBox, env_step.hpp:6538-6543).
RG_HDI bool spawn_spot_near_box(V3 spot, V3 center, V3 half) {
    const float dx = fmax_(fabs_(spot.x - center.x) - half.x, 0.0f);
    const float dy = fmax_(fabs_(spot.y - center.y) - half.y, 0.0f);
    const float dz = fmax_(fabs_(spot.z - center.z) - half.z, 0.0f);
    return dx * dx + dy * dy + dz * dz <= 48.0f * 48.0f;
}
// ... of a car: a box at its origin, or its body's mesh bounds turned into a world-axis box (reference
// SpawnSpotNearCar, env_step.hpp:6556-6564).
RG_HDI bool spawn_spot_near_car(V3 spot, V3 pos, V3 fwd, V3 right, V3 up, const float* bounds) {
    if (spawn_spot_near_box(spot, pos, V3{48.0f, 48.0f, 32.0f})) return true;
    const V3 center = pos + fwd * bounds[0] + right * bounds[1] + up * bounds[2];
    return spawn_spot_near_box(spot, center,
                               V3{fabs_(fwd.x) * bounds[3] + fabs_(right.x) * bounds[4] + fabs_(up.x) * bounds[5],
                                  fabs_(fwd.y) * bounds[3] + fabs_(right.y) * bounds[4] + fabs_(up.y) * bounds[5],
                                  fabs_(fwd.z) * bounds[3] + fabs_(right.z) * bounds[4] + fabs_(up.z) * bounds[5]});
}
// Whether a respawn ground point is taken: near another car where it is now, or (a demolished car) where it comes
// back this tick or, for an earlier slot also due, where its spot was already picked; or near the ball (reference
// RespawnPlaceTaken, env_step.hpp:6566-6613).
RG_HDI bool respawn_place_taken(V3 ground, int self, const ArenaCars& A, uint32_t demoed, uint32_t due,
                                const TickConfig& tc, V3 ball_pos) {
    const V3 spot{ground.x, ground.y, ground.z + 83.0f};
    for (int j = 0; j < A.count && j < 32; ++j) {
        if (j == self) continue;
        const CarState& o = A.cars[j];
        V3 pos, fwd, right, up;
        if (((demoed >> j) & 1u) == 0u) {
            car_basis(o, fwd, right, up);
            pos = o.pos_bt * 50.0f;
        } else {
            const bool back_now = !(fmax_(0.0f, o.demo_respawn_timer - tc.tick_dt) > 0.0f);
            if (!back_now && (j > self || ((due >> j) & 1u) == 0u)) continue;
            const int code = o.respawn_slot_override_plus1;
            int s = -1, d = -1;
            if (code >= kRespawnOffsetOverridePlus1 && code < kRespawnOffsetOverridePlus1 + 32) {
                s = ((code - kRespawnOffsetOverridePlus1) >> 3) & 3;
                d = (code - kRespawnOffsetOverridePlus1) & 7;
            } else if (code != 0) {
                if (code >= kKickoffSpawnOverridePlus1) continue;
                s = code - 1;
            } else {
                continue;
            }
            float yaw;
            respawn_place(A.teams[j], s, d, tc.rules, pos, yaw);
            pos.z += A.cfgs[j].spawn_z;
            const Q4 q = quat_from_yaw(wrap_angle(yaw));
            fwd = V3{q.w * q.w - q.z * q.z, 2.0f * q.w * q.z, 0.0f};
            right = V3{-fwd.y, fwd.x, 0.0f};
            up = V3{0.0f, 0.0f, 1.0f};
        }
        if (spawn_spot_near_car(spot, pos, fwd, right, up, body_mesh_bounds(A.cfgs[j].body))) return true;
    }
    const float r = tc.ball_radius;
    return spawn_spot_near_box(spot, ball_pos, V3{r, r, r}) ||
           spawn_spot_near_box(spot, ball_pos, V3{34.0f, 34.0f, 78.0f});
}
// The respawn spots of the arena's demolished cars that come back within two ticks, picked one tick ahead: the
// arena's spot order from the draw's start, the first free spot, else its eight 192 uu neighbours one ring of spots at
// a time, else the drawn spot; stored as the car's respawn override (reference PickRespawnSpotsForEnv,
// env_step.hpp:6615-6650, called from StepEnvPreTickEnvState, env_step.hpp:6664-6693).
RG_HDI void pick_respawn_spots(const ArenaCars& A, const BallState& b, const EnvState& env, const TickConfig& tc,
                               uint64_t seed, int env_idx) {
    const int count = A.count;
    uint32_t demoed = 0;
    if (env.car_visit_order_mode == 3 && count <= 8) {
        demoed = ~static_cast<uint32_t>(env.car_visit_present_mask) & ((1u << count) - 1u);
    } else {
        for (int i = 0; i < count && i < 32; ++i) demoed |= static_cast<uint32_t>(A.cars[i].is_demoed != 0) << i;
    }
    if (demoed == 0) return;
    uint32_t due = 0;
    for (int i = 0; i < count && i < 32; ++i) {
        if (((demoed >> i) & 1u) == 0u) continue;
        const float left = fmax_(0.0f, A.cars[i].demo_respawn_timer - tc.tick_dt);
        if (!(fmax_(0.0f, left - tc.tick_dt) > 0.0f)) due |= 1u << i;
    }
    if (due == 0) return;
    const V3 ball_pos = b.pos_bt * 50.0f;
    const uint32_t order = env.respawn_match_order != 0 ? env.respawn_match_order : build_respawn_order(seed, env_idx);
    for (int i = 0; i < count && i < 32; ++i) {
        if (((due >> i) & 1u) == 0u) continue;
        CarState& car = A.cars[i];
        if (car.respawn_slot_override_plus1 != 0) continue;
        const int team = A.teams[i];
        const int start = respawn_start_index(seed, env_idx, static_cast<uint64_t>(env.tick),
                                              static_cast<uint32_t>(A.car_base + i + 1));
        const int flip = team == 0 ? 0 : 2;
        int spot = -1, dir = -1;
        for (int k = 0; k < 36 && spot < 0; ++k) {
            const int walk = k < 4 ? k : (k - 4) >> 3;
            const int d = k < 4 ? -1 : (k - 4) & 7;
            const int s = static_cast<int>((order >> (2 * ((start + walk) & 3))) & 3u) ^ flip;
            V3 ground;
            float yaw;
            respawn_place(team, s, d, tc.rules, ground, yaw);
            if (!respawn_place_taken(ground, i, A, demoed, due, tc, ball_pos)) {
                spot = s;
                dir = d;
            }
        }
        if (spot < 0) spot = static_cast<int>((order >> (2 * (start & 3))) & 3u) ^ flip;
        car.respawn_slot_override_plus1 =
            static_cast<uint8_t>(dir < 0 ? spot + 1 : kRespawnOffsetOverridePlus1 + 8 * spot + dir);
    }
}

RG_HDI void respawn_car(CarState& c, const CarConfig& cfg, const TickConfig& tc, const RespawnCtx& rc) {
    const int team = rc.team;
    int slot = -1, offset_dir = -1;
    if (c.respawn_slot_override_plus1 >= kRespawnOffsetOverridePlus1 &&
        c.respawn_slot_override_plus1 < kRespawnOffsetOverridePlus1 + 32) {
        offset_dir = (c.respawn_slot_override_plus1 - kRespawnOffsetOverridePlus1) & 7;
        slot = ((c.respawn_slot_override_plus1 - kRespawnOffsetOverridePlus1) >> 3) & 3;
        c.respawn_slot_override_plus1 = 0;
    } else if (c.respawn_slot_override_plus1 != 0) {
        slot = c.respawn_slot_override_plus1 - 1;
        c.respawn_slot_override_plus1 = 0;
    }
    if (slot < 0) slot = respawn_start_index(rc.seed, rc.env_idx, static_cast<uint64_t>(rc.env_tick), rc.car_id);
    if (tc.rules) {
        // a custom arena's spots (reference KickoffSpawnCar / RespawnCar / RespawnPlace with ArenaRules,
        // arena_ball.hpp:3098-3160)
        const ArenaRules& R = *tc.rules;
        const int t = team == 0 ? 0 : 1;
        if (offset_dir < 0 && slot >= kKickoffSpawnOverridePlus1 - 1) {
            const int spot = slot - (kKickoffSpawnOverridePlus1 - 1);
            const int ks = spot >= 0 && spot < 4 ? spot : 4;
            const uint16_t driving_disabled = c.driving_disabled;
            place_car_at_world_spawn(c, R.kickoff_pos[t][ks], R.kickoff_yaw[t][ks], cfg.spawn_z, tc.boost_spawn_amount);
            c.driving_disabled = driving_disabled;
            c.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
            return;
        }
        V3 ground;
        float yaw;
        respawn_place(team, slot % 4, offset_dir, tc.rules, ground, yaw);
        place_car_at_world_spawn(c, ground, yaw, cfg.spawn_z, tc.boost_spawn_amount);
        c.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
        c.is_on_ground = 0;
        return;
    }
    if (offset_dir < 0 && slot >= kKickoffSpawnOverridePlus1 - 1) {
        const uint16_t driving_disabled = c.driving_disabled;
        place_car_at_kickoff_spawn(c, team, soccar_kickoff_spawn(slot - (kKickoffSpawnOverridePlus1 - 1)), cfg.spawn_z,
                                   tc.boost_spawn_amount);
        c.driving_disabled = driving_disabled;
        c.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
        return;
    }
    SpawnPos spawn = soccar_respawn_spawn(slot % 4);
    if (offset_dir >= 0) {
        V3 ground;
        float yaw;
        respawn_place(team, slot % 4, offset_dir, nullptr, ground, yaw);
        spawn.x = ground.x;
        spawn.y = team == 0 ? ground.y : -ground.y;
    }
    // reference PlaceCarAtRespawnSpawn (arena_ball.hpp:2562-2577): x is not mirrored for orange
    const float y = team == 0 ? spawn.y : -spawn.y;
    const float yaw = spawn.yaw + (team == 0 ? 0.0f : kPiF);
    car_set_pos_bt(c, V3{spawn.x, y, cfg.spawn_z} * kUuToBt);
    c.rot = quat_from_yaw(wrap_angle(yaw));
    seed_car_basis_from_spawn(c, spawn_yaw_rotator_units(spawn.yaw), team == 1);
    reset_car_common(c, tc.boost_spawn_amount);
    c.vel_impulse_cache = V3{0.0f, 0.0f, 0.0f};
    c.is_on_ground = 0;
}

RG_HDI V3 car_pre_tick(CarState& c, const CarControls& k, const CarConfig& cfg, const TickConfig& tc, WheelRuntime& w,
                       const RespawnCtx& rc) {
    c.ball_contact_this_tick = 0;
    restore_step_fields(c);
    if (c.tick_count_since_update == 0) cal_internal_timers_from_set_state(c, tc);
    if (c.just_respawned) c.just_respawned = 0;
    bool respawned = false;
    if (c.is_demoed) {
        c.demo_respawn_timer = fmax_(0.0f, c.demo_respawn_timer - tc.tick_dt);
        if (c.demo_respawn_timer <= 0.0f) {
            respawn_car(c, cfg, tc, rc);
            respawned = true;
        } else if (!(fmax_(0.0f, c.demo_respawn_timer - tc.tick_dt) > 0.0f) &&
                   !(c.respawn_slot_override_plus1 >= kKickoffSpawnOverridePlus1 &&
                     c.respawn_slot_override_plus1 < kKickoffSpawnOverridePlus1 + 5)) {
            c.boost = tc.boost_spawn_amount;
            c.boost_amount = c.boost / 100.0f;
        }
    }
    const Q4 spawn_rot = c.rot;
    c.tick_start_pos_bt = c.pos_bt;
    car_tick_start_quantize(c, tc);
    if (respawned)
        spawn_inertia_basis(spawn_rot, c.tick_start_basis_forward, c.tick_start_basis_right, c.tick_start_basis_up);
    const Q4 snap_rot = c.rot;
    const V3 snap_vel = c.vel;
    cal_flip_z_damp_prepass(c, tc);
    c.cal_tick_start_ang_vel = c.ang_vel;
    const V3 before = c.vel_bt;
    car_pre_physics(c, k, cfg, tc, w, snap_rot, snap_vel);
    if (!c.is_demoed) {
        const bool impulsed = c.vel_bt.x != before.x || c.vel_bt.y != before.y || c.vel_bt.z != before.z;
        if ((car_body_damping_clamp(c, tc) & 1) && impulsed) car_set_vel_bt(c, c.vel_bt);
    }
    return snap_vel;
}

// ---- the world step of an arena with cars ------------------------------------------------------------------------
// Per-tick snapshots the world step needs from the tick start: the velocities the broadphase predicts motion with
// (reference car_predict_vel_bt / ball_predict_vel_bt, env_step.hpp:6847-6851, 6884).
struct TickSnap {
    V3 ball_vel_bt;
    V3 car_vel_bt[8], car_ang_vel[8];
    // uu velocities right after the tick-start quantisation, for the ball-hit impulse (reference cal_start_vel /
    // cal_ball_start_vel)
    V3 car_start_vel[8], ball_start_vel;
};

// The car's predictive (CCD) contact: its box centre's motion this tick (reference PredictiveContactRayForBody
// body > 0, env_step.hpp:3930-4060; the free-box shortcuts there only skip rays that cannot hit).
RG_HDI bool car_predictive_hit(const CarState& c, const CarConfig& cfg, const MeshDevice& m, float dt, V3& n,
                               float& dist) {
    V3 ax, ay, az;
    car_basis(c, ax, ay, az);
    const V3 child = cfg.hitbox_offset * (1.0f / 50.0f);
    const V3 cur{c.pos_bt.x + (ax.x * child.x + ay.x * child.y + az.x * child.z),
                 c.pos_bt.y + (ax.y * child.x + ay.y * child.y + az.y * child.z),
                 c.pos_bt.z + (ax.z * child.x + ay.z * child.y + az.z * child.z)};
    V3 f = c.basis_forward, r = c.basis_right, u = c.basis_up;
    Q4 rot = c.rot;
    game_integrate_orientation(f, r, u, rot, c.ang_vel, dt);
    const V3 po = c.pos_bt + c.vel_bt * dt;
    const V3 to{po.x + (f.x * child.x + r.x * child.y + u.x * child.z),
                po.y + (f.y * child.x + r.y * child.y + u.y * child.z),
                po.z + (f.z * child.x + r.z * child.y + u.z * child.z)};
    return predictive_ray(m, cur, to, n, dist);
}

// PGS at the velocity level over every contact row of the arena, in the order the sorted manifold list gives
// (reference SolveUnifiedVelocityContactRowsGeneral, arena_geometry.hpp:5527-5866): for each listed manifold its rows,
// then the unlisted car rows, then the unlisted ball rows; each normal row's friction row follows the normal order.
// The ball's rows are indexed car-ball rows first, then its arena rows, the order the world step appends them in.
// Rows act on their bodies' velocity deltas (a car-ball row on both, reference
// SolveBallVelocity{Normal,Friction}RowWithAccumulators, arena_geometry.hpp:2618-2750); one iteration count (stop
// when nothing changed) covers all.
RG_NOINL void unified_velocity_solve(BallContactRows& br, BallCarRows& bc, CarWorldRows& cr, CarCarRows& pr,
                                   const BpEntry* list, int n_list, V3& ball_dl, V3& ball_da, V3* car_dl, V3* car_da) {
    constexpr int kMax = kMaxBallVelRows + kMaxBallCarRows + kMaxCarWorldRows + kMaxPairRows;
    uint8_t nb[kMax], ni[kMax], fb[kMax], fi[kMax];
    int nn = 0, nf = 0;
    const int bcn = bc.nv, bcf = bc.nf;
    const int wn = cr.nv, bn = bcn + br.vel_count, wf = cr.nf, bf = bcf + br.fric_count;
    const int pn = pr.nv, pf = pr.nf;
    // combined ball index: car-ball rows first
    auto ball_fric_normal = [&](int f) { return f < bcf ? bc.fric[f].normal_row : br.fric[f - bcf].normal_row + bcn; };
    auto ball_applied = [&](int r) { return r < bcn ? bc.vel[r].applied : br.vel[r - bcn].applied; };
    if (wn + pn + bn <= 1 && wf + pf + bf <= 1) {
        if (wn == 1) {
            nb[0] = 0;
            ni[0] = 0;
            nn = 1;
        } else if (pn == 1) {
            nb[0] = 1;
            ni[0] = 0;
            nn = 1;
        } else if (bn == 1) {
            nb[0] = 2;
            ni[0] = 0;
            nn = 1;
        }
        if (wf == 1) {
            fb[0] = 0;
            fi[0] = 0;
            nf = 1;
        } else if (pf == 1) {
            fb[0] = 1;
            fi[0] = 0;
            nf = 1;
        } else if (bf == 1) {
            fb[0] = 2;
            fi[0] = 0;
            nf = 1;
        }
    } else {
        uint64_t wused = 0, bused = 0, pused = 0;
        for (int e = 0; e < n_list; ++e) {
            const uint32_t key = list[e].key;
            const int kind = bp_kind(key);
            if (kind == 2) {
                const int sid = bp_static(key);
                const int tag = sid >= 0 ? 100 + sid : -1;
                const int body = bp_body_a(key);
                for (int r = 0; r < wn; ++r) {
                    if ((wused >> r) & 1ull) continue;
                    if (cr.vel[r].body != body || cr.vel[r].tag != tag) continue;
                    wused |= 1ull << r;
                    nb[nn] = 0;
                    ni[nn++] = static_cast<uint8_t>(r);
                }
            } else if (kind == 3) {
                const int lo = bp_body_a(key), hi = bp_body_b(key);
                for (int r = 0; r < pn; ++r) {
                    const int ra = pr.vel[r].a, rb = pr.vel[r].b;
                    if (((pused >> r) & 1ull) || (ra < rb ? ra : rb) != lo || (ra < rb ? rb : ra) != hi) continue;
                    pused |= 1ull << r;
                    nb[nn] = 1;
                    ni[nn++] = static_cast<uint8_t>(r);
                }
            } else if (kind == 1) {
                const int car = bp_body_a(key);
                for (int r = 0; r < bcn; ++r) {
                    if (((bused >> r) & 1ull) || bc.vel[r].car != car) continue;
                    bused |= 1ull << r;
                    nb[nn] = 2;
                    ni[nn++] = static_cast<uint8_t>(r);
                }
            } else if (kind == 0 && bp_static(key) == kBpPredictiveId) {
                for (int r = bcn; r < bn; ++r) {
                    if (((bused >> r) & 1ull) || !br.vel[r - bcn].predictive) continue;
                    bused |= 1ull << r;
                    nb[nn] = 2;
                    ni[nn++] = static_cast<uint8_t>(r);
                }
            }
        }
        for (int r = 0; r < wn; ++r)
            if (!((wused >> r) & 1ull)) {
                nb[nn] = 0;
                ni[nn++] = static_cast<uint8_t>(r);
            }
        for (int r = 0; r < pn; ++r)
            if (!((pused >> r) & 1ull)) {
                nb[nn] = 1;
                ni[nn++] = static_cast<uint8_t>(r);
            }
        for (int r = 0; r < bn; ++r)
            if (!((bused >> r) & 1ull)) {
                nb[nn] = 2;
                ni[nn++] = static_cast<uint8_t>(r);
            }
        uint64_t wfu = 0, bfu = 0, pfu = 0;
        for (int k = 0; k < nn; ++k) {
            if (nb[k] == 0) {
                for (int f = 0; f < wf; ++f)
                    if (!((wfu >> f) & 1ull) && cr.fric[f].normal_row == ni[k]) {
                        wfu |= 1ull << f;
                        fb[nf] = 0;
                        fi[nf++] = static_cast<uint8_t>(f);
                    }
            } else if (nb[k] == 1) {
                for (int f = 0; f < pf; ++f)
                    if (!((pfu >> f) & 1ull) && pr.fric[f].normal_row == ni[k]) {
                        pfu |= 1ull << f;
                        fb[nf] = 1;
                        fi[nf++] = static_cast<uint8_t>(f);
                    }
            } else {
                for (int f = 0; f < bf; ++f)
                    if (!((bfu >> f) & 1ull) && ball_fric_normal(f) == ni[k]) {
                        bfu |= 1ull << f;
                        fb[nf] = 2;
                        fi[nf++] = static_cast<uint8_t>(f);
                    }
            }
        }
        for (int f = 0; f < wf; ++f)
            if (!((wfu >> f) & 1ull)) {
                fb[nf] = 0;
                fi[nf++] = static_cast<uint8_t>(f);
            }
        for (int f = 0; f < pf; ++f)
            if (!((pfu >> f) & 1ull)) {
                fb[nf] = 1;
                fi[nf++] = static_cast<uint8_t>(f);
            }
        for (int f = 0; f < bf; ++f)
            if (!((bfu >> f) & 1ull)) {
                fb[nf] = 2;
                fi[nf++] = static_cast<uint8_t>(f);
            }
    }
    // one normal / friction row against its body's accumulated velocity change
    auto solve_normal = [](V3 normal, V3 rel_cross, V3 ang, float inv_mass, float jac, float rhs, float& applied,
                           V3& dl, V3& da) {
        float di = rhs;
        const float dv = bt_dot(normal, dl) + bt_dot(rel_cross, da);
        di = di - dv * jac;
        const float before = applied;
        const float sum = before + di;
        if (sum < 0.0f) {
            di = -before;
            applied = 0.0f;
        } else {
            applied = sum;
        }
        if (di == 0.0f) return f2u(before) != f2u(applied);
        dl = dl + (normal * inv_mass) * di;
        da = da + ang * di;
        return true;
    };
    auto solve_friction = [](V3 tangent, V3 rel_cross, V3 ang, float inv_mass, float jac, float rhs, float maxi,
                             float& applied, V3& dl, V3& da) {
        float di = rhs;
        const float dv = bt_dot(tangent, dl) + bt_dot(rel_cross, da);
        di = di - dv * jac;
        const float before = applied;
        const float sum = before + di;
        if (sum < -maxi) {
            di = -maxi - before;
            applied = -maxi;
        } else if (sum > maxi) {
            di = maxi - before;
            applied = maxi;
        } else {
            applied = sum;
        }
        if (di == 0.0f) return f2u(before) != f2u(applied);
        dl = dl + (tangent * inv_mass) * di;
        da = da + ang * di;
        return true;
    };
    // a car-ball row: the car is Bullet's body 1 (direction -n), the ball body 2
    auto solve_pair = [](V3 n, V3 rel_ball_cross, V3 ball_ang, float ball_inv, V3 rel_car_cross, V3 car_ang,
                         float car_inv, float jac, float rhs, float lo, float hi, float& applied, V3& bdl, V3& bda,
                         V3& cdl, V3& cda) {
        float di = rhs;
        const float dv1 = bt_dot(-n, cdl) + bt_dot(rel_car_cross, cda);
        const float dv2 = bt_dot(n, bdl) + bt_dot(rel_ball_cross, bda);
        di = di - dv1 * jac;
        di = di - dv2 * jac;
        const float before = applied;
        const float sum = before + di;
        if (sum < lo) {
            di = lo - before;
            applied = lo;
        } else if (sum > hi) {
            di = hi - before;
            applied = hi;
        } else {
            applied = sum;
        }
        if (di == 0.0f) return f2u(before) != f2u(applied);
        bdl = bdl + (n * ball_inv) * di;
        bda = bda + ball_ang * di;
        cdl = cdl + ((-n) * car_inv) * di;
        cda = cda + car_ang * di;
        return true;
    };
    for (int iter = 0; iter < 10; ++iter) {
        bool changed = false;
        for (int k = 0; k < nn; ++k) {
            if (nb[k] == 2 && ni[k] < bcn) {
                BcVelRow& r = bc.vel[ni[k]];
                // the normal row's lower clamp: sum < 0 -> di = -before, applied = 0
                float di = r.rhs;
                const float dv1 = bt_dot(-r.normal, car_dl[r.car]) + bt_dot(r.rel_car_cross, car_da[r.car]);
                const float dv2 = bt_dot(r.normal, ball_dl) + bt_dot(r.rel_ball_cross, ball_da);
                di = di - dv1 * r.jac;
                di = di - dv2 * r.jac;
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
                ball_dl = ball_dl + (r.normal * r.ball_inv_mass) * di;
                ball_da = ball_da + r.ball_ang * di;
                car_dl[r.car] = car_dl[r.car] + ((-r.normal) * r.car_inv_mass) * di;
                car_da[r.car] = car_da[r.car] + r.car_ang * di;
                changed = true;
            } else if (nb[k] == 1) {
                // a pair row: car a along normal_a, car b along -normal_a (reference SolveSharedCarVelocityNormalRow)
                PairVelRow& r = pr.vel[ni[k]];
                const V3 nbv = -r.normal_a;
                const float dva = bt_dot(r.normal_a, car_dl[r.a]) + bt_dot(r.rel_a_cross, car_da[r.a]);
                const float dvb = bt_dot(nbv, car_dl[r.b]) + bt_dot(r.rel_b_cross, car_da[r.b]);
                const float before = r.applied;
                float di = r.rhs;
                di = di - dvb * r.jac;
                di = di - dva * r.jac;
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
                car_dl[r.a] = car_dl[r.a] + (r.normal_a * r.inv_mass) * di;
                car_da[r.a] = car_da[r.a] + r.ang_a * di;
                car_dl[r.b] = car_dl[r.b] + (nbv * r.inv_mass) * di;
                car_da[r.b] = car_da[r.b] + r.ang_b * di;
                changed = true;
            } else if (nb[k] == 2) {
                BallVelRow& r = br.vel[ni[k] - bcn];
                changed = solve_normal(r.normal, r.rel_cross, r.ang, r.inv_mass, r.jac_inv, r.rhs, r.applied, ball_dl,
                                       ball_da) || changed;
            } else {
                CarVelRow& r = cr.vel[ni[k]];
                changed = solve_normal(r.normal, r.rel_cross, r.ang, r.inv_mass, r.jac, r.rhs, r.applied,
                                       car_dl[r.body], car_da[r.body]) || changed;
            }
        }
        for (int k = 0; k < nf; ++k) {
            if (fb[k] == 2 && fi[k] < bcf) {
                BcFricRow& r = bc.fric[fi[k]];
                const float total = ball_applied(r.normal_row);
                if (total <= 0.0f) continue;
                const float maxi = r.friction * total;
                changed = solve_pair(r.tangent, r.rel_ball_cross, r.ball_ang, r.ball_inv_mass, r.rel_car_cross,
                                     r.car_ang, r.car_inv_mass, r.jac, r.rhs, -maxi, maxi, r.applied, ball_dl, ball_da,
                                     car_dl[r.car], car_da[r.car]) || changed;
            } else if (fb[k] == 1) {
                PairFricRow& r = pr.fric[fi[k]];
                const float total = pr.vel[r.normal_row].applied;
                if (total <= 0.0f) continue;
                const float maxi = r.friction * total;
                const V3 tb = -r.tangent_a;
                float di = r.rhs;
                const float dvb = bt_dot(tb, car_dl[r.b]) + bt_dot(r.rel_b_cross, car_da[r.b]);
                di = di - dvb * r.jac;
                const float dva = bt_dot(r.tangent_a, car_dl[r.a]) + bt_dot(r.rel_a_cross, car_da[r.a]);
                di = di - dva * r.jac;
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
                car_dl[r.a] = car_dl[r.a] + (r.tangent_a * r.inv_mass) * di;
                car_da[r.a] = car_da[r.a] + r.ang_a * di;
                car_dl[r.b] = car_dl[r.b] + (tb * r.inv_mass) * di;
                car_da[r.b] = car_da[r.b] + r.ang_b * di;
                changed = true;
            } else if (fb[k] == 2) {
                BallFricRow& r = br.fric[fi[k] - bcf];
                const float total = ball_applied(r.normal_row + bcn);
                if (total <= 0.0f) continue;
                changed = solve_friction(r.tangent, r.rel_cross, r.ang, r.inv_mass, r.jac_inv, r.rhs,
                                         r.friction * total, r.applied, ball_dl, ball_da) || changed;
            } else {
                CarFricRow& r = cr.fric[fi[k]];
                const float total = cr.vel[r.normal_row].applied;
                if (total <= 0.0f) continue;
                changed = solve_friction(r.tangent, r.rel_cross, r.ang, r.inv_mass, r.jac, r.rhs, r.friction * total,
                                         r.applied, car_dl[r.body], car_da[r.body]) || changed;
            }
        }
        if (!changed) break;
    }
}

// Split-impulse position correction over the arena's penetration rows, ordered like the velocity rows
// (reference SolveUnifiedSplitContactRows, arena_geometry.hpp:5035-5275; car-ball rows as in
// SolveUnifiedBallSplitRow, :3523-3600). Returns the ball's push velocity; the cars' push and turn velocities come
// back in `car_push` / `car_turn`, `car_bt` telling which cars had Bullet-unit rows (every row here carries Bullet
// units, so a car is in Bullet units when any of its arena or car-ball rows exists, MarkBtSplitAccumulators).
RG_NOINL V3 unified_split_solve(BallContactRows& br, BallCarRows& bc, CarWorldRows& cr, CarCarRows& pr,
                              const BpEntry* list, int n_list, V3* car_push, V3* car_turn, bool* car_bt, int count) {
    constexpr int kMax = kMaxBallSplitRows + kMaxBallCarRows + kMaxCarWorldRows + kMaxPairRows;
    // Bullet-unit accumulators (reference MarkBtSplitAccumulators, arena_geometry.hpp:3317-3431): a car is in
    // Bullet units when one of its split rows exists and none of the rows reaching it (through pair and car-ball rows)
    // lacks Bullet-unit terms; only a pair row whose Bullet-unit penetration rounds to zero lacks them.
    bool touched[8], blocked[8];
    for (int i = 0; i < 8; ++i) touched[i] = blocked[i] = false;
    for (int r = 0; r < cr.ns; ++r) touched[cr.split[r].body] = true;
    for (int r = 0; r < pr.ns; ++r) {
        touched[pr.split[r].a] = touched[pr.split[r].b] = true;
        if (!pr.split[r].has_bt) blocked[pr.split[r].a] = blocked[pr.split[r].b] = true;
    }
    for (int r = 0; r < bc.ns; ++r) touched[bc.split[r].car] = true;
    if (pr.ns > 0 || bc.ns > 0 || br.split_count > 0) {
        bool ball_blocked = false;
        for (int pass = 0; pass < 8; ++pass) {
            bool changed = false;
            for (int r = 0; r < pr.ns; ++r) {
                const int a = pr.split[r].a, b = pr.split[r].b;
                if (blocked[a] != blocked[b]) {
                    blocked[a] = blocked[b] = true;
                    changed = true;
                }
            }
            for (int r = 0; r < bc.ns; ++r) {
                const int o = bc.split[r].car;
                if (blocked[o] != ball_blocked) {
                    blocked[o] = ball_blocked = true;
                    changed = true;
                }
            }
            if (!changed) break;
        }
    }
    for (int i = 0; i < count && i < 8; ++i) car_bt[i] = touched[i] && !blocked[i];
    const int bcs = bc.ns;
    const int ws = cr.ns, ps = pr.ns, bs = bcs + br.split_count;
    uint8_t ob[kMax], oi[kMax];
    int no = 0;
    if (n_list > 0 && ws + ps + bs > 1) {
        uint64_t wused = 0, bused = 0, pused = 0;
        for (int e = 0; e < n_list; ++e) {
            const uint32_t key = list[e].key;
            const int kind = bp_kind(key);
            if (kind == 2) {
                const int sid = bp_static(key);
                const int tag = sid >= 0 ? 100 + sid : -1;
                const int body = bp_body_a(key);
                for (int r = 0; r < ws; ++r) {
                    if (((wused >> r) & 1ull) || cr.split[r].body != body || cr.split[r].tag != tag) continue;
                    wused |= 1ull << r;
                    ob[no] = 0;
                    oi[no++] = static_cast<uint8_t>(r);
                }
            } else if (kind == 3) {
                const int lo = bp_body_a(key), hi = bp_body_b(key);
                for (int r = 0; r < ps; ++r) {
                    const int ra = pr.split[r].a, rb = pr.split[r].b;
                    if (((pused >> r) & 1ull) || (ra < rb ? ra : rb) != lo || (ra < rb ? rb : ra) != hi) continue;
                    pused |= 1ull << r;
                    ob[no] = 1;
                    oi[no++] = static_cast<uint8_t>(r);
                }
            } else if (kind == 1) {
                const int car = bp_body_a(key);
                for (int r = 0; r < bcs; ++r) {
                    if (((bused >> r) & 1ull) || bc.split[r].car != car) continue;
                    bused |= 1ull << r;
                    ob[no] = 2;
                    oi[no++] = static_cast<uint8_t>(r);
                }
            } else if (kind == 0) {
                for (int r = bcs; r < bs; ++r) {
                    const BallSplitRow& row = br.split[r - bcs];
                    if (((bused >> r) & 1ull) || row.static_id < 0 || row.static_id != bp_static(key)) continue;
                    bused |= 1ull << r;
                    ob[no] = 2;
                    oi[no++] = static_cast<uint8_t>(r);
                }
            }
        }
        for (int r = 0; r < ws; ++r)
            if (!((wused >> r) & 1ull)) {
                ob[no] = 0;
                oi[no++] = static_cast<uint8_t>(r);
            }
        for (int r = 0; r < ps; ++r)
            if (!((pused >> r) & 1ull)) {
                ob[no] = 1;
                oi[no++] = static_cast<uint8_t>(r);
            }
        for (int r = 0; r < bs; ++r)
            if (!((bused >> r) & 1ull)) {
                ob[no] = 2;
                oi[no++] = static_cast<uint8_t>(r);
            }
    } else {
        for (int r = 0; r < ws; ++r) {
            ob[no] = 0;
            oi[no++] = static_cast<uint8_t>(r);
        }
        for (int r = 0; r < ps; ++r) {
            ob[no] = 1;
            oi[no++] = static_cast<uint8_t>(r);
        }
        for (int r = 0; r < bs; ++r) {
            ob[no] = 2;
            oi[no++] = static_cast<uint8_t>(r);
        }
    }
    V3 push{0, 0, 0}, turn{0, 0, 0};
    for (int i = 0; i < count; ++i) car_push[i] = car_turn[i] = V3{0.0f, 0.0f, 0.0f};
    for (int iter = 0; iter < 10; ++iter) {
        bool changed = false;
        for (int k = 0; k < no; ++k) {
            if (ob[k] == 2 && oi[k] < bcs) {
                BcSplitRow& r = bc.split[oi[k]];
                V3& p = car_push[r.car];
                V3& t = car_turn[r.car];
                const float before = r.applied;
                float di = r.rhs;
                const float ball_term = (bt_dot(r.normal, push) + bt_dot(r.rel_ball_cross, turn)) * r.jac;
                di -= (bt_dot(-r.normal, p) + bt_dot(r.rel_car_cross, t)) * r.jac;
                di -= ball_term;
                const float sum = r.applied + di;
                if (sum < 0.0f) {
                    di = -r.applied;
                    r.applied = 0.0f;
                } else {
                    r.applied = sum;
                }
                if (di == 0.0f) {
                    changed = (f2u(before) != f2u(r.applied)) || changed;
                    continue;
                }
                push = push + (r.normal * r.ball_inv_mass) * di;
                turn = turn + r.ball_ang * di;
                p = p + ((-r.normal) * r.car_inv_mass) * di;
                t = t + r.car_ang * di;
                changed = true;
            } else if (ob[k] == 1) {
                // a pair row in Bullet units (reference SolveSharedCarSplitRow)
                PairSplitRow& r = pr.split[oi[k]];
                if (r.rhs == 0.0f) continue;
                V3& pa = car_push[r.a];
                V3& ta = car_turn[r.a];
                V3& pb = car_push[r.b];
                V3& tb = car_turn[r.b];
                const V3 nbv = -r.normal_a;
                const float before = r.applied;
                float di = r.rhs;
                const float dva = bt_dot(r.normal_a, pa) + bt_dot(r.rel_a_cross, ta);
                di -= (bt_dot(nbv, pb) + bt_dot(r.rel_b_cross, tb)) * r.jac;
                di -= dva * r.jac;
                const float sum = r.applied + di;
                if (sum < 0.0f) {
                    di = 0.0f - r.applied;
                    r.applied = 0.0f;
                } else {
                    r.applied = sum;
                }
                if (di != 0.0f) {
                    pa = pa + (r.normal_a * r.inv_mass) * di;
                    ta = ta + r.ang_a * di;
                    pb = pb + (nbv * r.inv_mass) * di;
                    tb = tb + r.ang_b * di;
                }
                changed = di != 0.0f || f2u(before) != f2u(r.applied) || changed;
            } else if (ob[k] == 2) {
                BallSplitRow& r = br.split[oi[k] - bcs];
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
            } else {
                CarSplitRow& r = cr.split[oi[k]];
                if (r.rhs == 0.0f) continue;
                V3& p = car_push[r.body];
                V3& t = car_turn[r.body];
                const float before = r.applied;
                float di = r.rhs;
                di -= (bt_dot(r.normal, p) + bt_dot(r.rel_cross, t)) * r.jac;
                const float sum = r.applied + di;
                if (sum < 0.0f) {
                    di = 0.0f - r.applied;
                    r.applied = 0.0f;
                } else {
                    r.applied = sum;
                }
                if (di != 0.0f) {
                    p = p + (r.normal * r.inv_mass) * di;
                    t = t + r.ang * di;
                }
                changed = di != 0.0f || f2u(before) != f2u(r.applied) || changed;
            }
        }
        if (!changed) break;
    }
    return push;
}

// The car's hitbox AABB against the ball's (radius + 0.08 bt) in Bullet units (reference BallCarRetainedPairOverlaps).
RG_HDI bool ball_car_box_overlaps(const BallState& b, const CarState& car, const CarConfig& cfg, const TickConfig& c,
                                  bool allow_midtick_demo) {
    if ((!allow_midtick_demo && car.is_demoed) || car.just_respawned) return false;
    V3 ax{1.0f, 0.0f, 0.0f}, ay{0.0f, 1.0f, 0.0f}, az{0.0f, 0.0f, 1.0f};
    car_basis(car, ax, ay, az);
    const V3 half = car_box_half_bt(cfg);
    const V3 off = cfg.hitbox_offset * (1.0f / 50.0f);
    const V3 center = car.pos_bt + ax * off.x + ay * off.y + az * off.z;
    const V3 ext{fabs_(ax.x) * half.x + fabs_(ay.x) * half.y + fabs_(az.x) * half.z,
                 fabs_(ax.y) * half.x + fabs_(ay.y) * half.y + fabs_(az.y) * half.z,
                 fabs_(ax.z) * half.x + fabs_(ay.z) * half.y + fabs_(az.z) * half.z};
    const float r = c.ball_radius * (1.0f / 50.0f) + 0.08f;
    const V3 bmin = b.pos_bt - V3{r, r, r}, bmax = b.pos_bt + V3{r, r, r};
    const V3 cmin = center - ext, cmax = center + ext;
    return !(cmin.x > bmax.x || cmax.x < bmin.x || cmin.y > bmax.y || cmax.y < bmin.y || cmin.z > bmax.z ||
             cmax.z < bmin.z);
}

// ---- a car's part of the world step, staged ------------------------------------------------------------------
// What one car of an arena contributes to the world step before the arena's shared stages, computed by the per-car
// kernel right after the car's vehicle update (one thread per car instead of one per arena): the prestep, the car's
// predictive contact and its query against the arena mesh, with the retained manifold and the rows that query leaves
// (as if its manifold is listed, which the arena checks later). Exact: these read and write only the car, its wheel
// record and its car/mesh manifold (not the ball, the other cars or the broadphase), nothing the arena does between
// the vehicle update and their place in the world step changes what they read (car/car and car/ball contacts touch
// only the cars' contact bookkeeping), and their effects on the car (the world-surface record, the contact normal)
// are applied by the arena where the reference makes them. A car whose vehicle update must run in the arena's car
// order (arena_free_cars) has its stage computed by the arena thread after all those updates.
struct CarStage {
    PreContactCar pre;
    V3 pred_n;
    float pred_d;
    uint32_t pred_hit;  // the car has a predictive contact this tick
    uint32_t mesh_ran;  // the mesh query ran (the car is neither demolished at the step's start nor just respawned)
    CarWorldContactResult res;
    CarWorldScratch ws;  // the car/mesh manifold after the query
    CarStageRows rows;   // the query's rows, in the order it made them
    BpProxy proxy;       // the car's broadphase proxy (valid = 0 for a car demolished at the step's start)
    PadContacts pads;    // the car's pad contacts after its post-tick (pad_contacts_stage)
    uint32_t in_car_thread;  // this tick's vehicle update and stage ran in the car's own thread (arena_free_cars)
    RayHit wheel_mesh[4];    // the wheels' arena-mesh rays, cast ahead of the vehicle update (wheel_mesh_ray_ahead)
    uint8_t wheel_meets_car[4];  // the wheel's ray meets another car's box (0 for a demolished car)
    BallCarScratch ball_manifold;  // the car/ball manifold after this tick's geometry (car_ball_stage)
    uint32_t ball_staged;          // ball_manifold holds this tick's update
    MeshContactEvents mesh_events;  // the query's car-world events (when events are on)
};

// A car's broadphase proxy: its box now and at the pose this tick's tick-start velocities predict (reference
// ComputeBulletBodyProxy, arena_geometry.hpp:3873-4035).
RG_HDI void car_body_proxy(BpProxy& p, const CarState& car, const CarConfig& cfg, V3 vel_bt, V3 ang_vel, float dt) {
    V3 ax = car.basis_forward, ay = car.basis_right, az = car.basis_up;
    V3 px = ax, py = ay, pz = az;
    Q4 unused{};
    game_integrate_orientation(px, py, pz, unused, ang_vel, dt);
    car_proxy(p, car.pos_bt, ax, ay, az, px, py, pz, vel_bt, cfg.hitbox_offset * (1.0f / 50.0f), car_box_half_bt(cfg),
              dt);
}

// The car's ball contact geometry ahead of the world step (one thread per car). The manifold update reads only the
// two bodies' poses, and neither body moves between the tick start and the world step's car-ball stage (vehicle
// updates, wheel pushes, bumps and demolitions change velocities and flags only). Staged when the car's box or swept
// proxy meets the ball's, a superset of the world step's test; the world step takes it when its own test passes.
RG_HDI void car_ball_stage(const BallState& b, V3 ball_start_vel_bt, const CarState& car, const CarConfig& cfg,
                           const TickConfig& c, V3 start_vel_bt, V3 start_ang_vel, const BallCarScratch& m_in,
                           CarStage& st) {
    st.ball_staged = 0u;
    if (car.is_demoed || car.just_respawned) return;  // the world step's tests fail for both
    bool meet = ball_car_box_overlaps(b, car, cfg, c, true);
    if (!meet) {
        BpProxy pb, pc;
        ball_proxy(pb, b.pos_bt, ball_start_vel_bt, c.ball_radius, c.tick_dt);
        car_body_proxy(pc, car, cfg, start_vel_bt, start_ang_vel, c.tick_dt);
        meet = pc.valid != 0 && !(pc.child_min.x > pb.child_max.x || pc.child_max.x < pb.child_min.x ||
                                  pc.child_min.y > pb.child_max.y || pc.child_max.y < pb.child_min.y ||
                                  pc.child_min.z > pb.child_max.z || pc.child_max.z < pb.child_min.z);
    }
    if (!meet) return;
    st.ball_manifold = m_in;
    ball_car_manifold_update(st.ball_manifold, b, car, cfg, c);
    st.ball_staged = 1u;
}

RG_HDI void car_stage_compute(CarState& car, const CarConfig& cfg, WheelRuntime& w, const CarWorldScratch& ws_in,
                              const TickConfig& c, const MeshDevice& mesh, int slot, V3 start_vel_bt, V3 start_ang_vel,
                              CarStage& st) {
    const float sub_dt = c.tick_dt;
    car_world_prestep(car, cfg, w, c, sub_dt, st.pre);
    st.proxy.valid = 0;
    if (!st.pre.is_demoed) car_body_proxy(st.proxy, car, cfg, start_vel_bt, start_ang_vel, sub_dt);
    st.pred_hit = !st.pre.is_demoed && car_predictive_hit(car, cfg, mesh, sub_dt, st.pred_n, st.pred_d) ? 1u : 0u;
    st.mesh_ran = !(st.pre.is_demoed || car.just_respawned) ? 1u : 0u;
    st.rows.nv = st.rows.nf = st.rows.ns = 0;
    st.res.hit = false;
    st.res.latest_normal = V3{0.0f, 0.0f, 1.0f};
    st.mesh_events.count = 0;
    if (st.mesh_ran) {
        st.ws = ws_in;
        st.res = car_mesh_contacts(car, cfg, st.ws, true, mesh, c, slot, st.rows,
                                   c.events.windows ? &st.mesh_events : nullptr);
    }
}

// One arena's world step with cars (reference WorldStepSoccar, env_step.hpp:4727-5623, on the path a custom-mesh
// soccar arena takes): predictive rays, the broadphase's manifold list, the ball's and the cars' arena contacts, the
// unified velocity and position solves, then integration; car-ball contacts (reference env_step.hpp:5045-5133)
// with their ball-hit bookkeeping. Car/car contacts are not built yet: two cars whose boxes meet only shape the
// manifold list here.
RG_NOINL void world_step_cars(BallState& b, BallWorldScratch& s, Broadphase& bp, CarWorldScratch* cws,
                            BallCarScratch* bcs, const TickConfig& c, const MeshDevice& mesh, const ArenaCars& A,
                            PreContactCar* pre, const TickSnap& snap, uint64_t env_tick,
                            const CarStage* stages = nullptr) {
    const int count = A.count;
    const float sub_dt = c.tick_dt;
    const bool vehicle_woke = (b.sleeping & 4u) != 0;
    b.sleeping &= 3u;
    const bool ball_sleeping = ball_resolve_activation(b);
    if (vehicle_woke) b.deactivation_time = 0.0f;
    const V3 ext_delta = ball_sleeping ? V3{0.0f, 0.0f, 0.0f} : V3{0.0f, 0.0f, c.gravity_z * sub_dt};
    if (stages) {
        for (int i = 0; i < count; ++i) pre[i] = stages[i].pre;
    } else {
        for (int i = 0; i < count; ++i) car_world_prestep(A.cars[i], A.cfgs[i], A.wheels[i], c, sub_dt, pre[i]);
    }
    const V3 solver_vel_bt = b.vel_bt;
    // where the bodies stand at the step's start, for the ball-hit records (reference record_ball_car_info)
    const V3 hit_ball_pos = b.pos;
    V3 hit_car_pos[8];
    Q4 hit_car_rot[8];
    for (int i = 0; i < count && i < 8; ++i) {
        hit_car_pos[i] = A.cars[i].pos;
        hit_car_rot[i] = A.cars[i].rot;
    }
    const bool awake = !ball_sleeping || vehicle_woke;
    // predictive contacts (reference ComputePredictiveContactHits, env_step.hpp:4129-4168)
    const int body_count = count + 1 < kBpBodies ? count + 1 : kBpBodies;
    uint32_t pred_mask = 0u;
    V3 pred_n[kBpBodies];
    float pred_d[kBpBodies];
    if (!(ball_sleeping && !vehicle_woke) && ball_predictive_hit(b, mesh, sub_dt, pred_n[0], pred_d[0])) pred_mask |= 1u;
    for (int i = 0; i + 1 < body_count; ++i) {
        if (pre[i].is_demoed) continue;
        if (stages) {
            if (stages[i].pred_hit) {
                pred_n[i + 1] = stages[i].pred_n;
                pred_d[i + 1] = stages[i].pred_d;
                pred_mask |= 1u << (i + 1);
            }
        } else if (car_predictive_hit(A.cars[i], A.cfgs[i], mesh, sub_dt, pred_n[i + 1], pred_d[i + 1])) {
            pred_mask |= 1u << (i + 1);
        }
    }
    // broadphase proxies and the manifold list (reference BuildBulletManifoldList + SortBulletManifoldListByIsland)
    BpProxy proxies[kBpBodies];
    ball_proxy(proxies[0], b.pos_bt, snap.ball_vel_bt, c.ball_radius, sub_dt);
    for (int i = 0; i + 1 < body_count; ++i) {
        BpProxy& p = proxies[i + 1];
        if (pre[i].is_demoed) {
            p.valid = 0;
        } else if (stages) {
            p = stages[i].proxy;
        } else {
            car_body_proxy(p, A.cars[i], A.cfgs[i], snap.car_vel_bt[i], snap.car_ang_vel[i], sub_dt);
        }
    }
    BpEntry list[kBpMaxEntries];
    const int n_list = bp_build_manifold_list(bp, proxies, body_count, mesh.aabb_min, mesh.aabb_max, pred_mask,
                                              ball_sleeping && !vehicle_woke, list);
    // car/car contacts (reference env_step.hpp:4916-5042): pairs in the built manifold list's order, then the remaining
    // pairs in slot order; a pair whose retained manifold is empty and whose cars are apart or inactive is skipped
    uint32_t car_car_touched = 0u;
    CarCarRows pr;
    pr.nv = pr.nf = pr.ns = 0;
    if (c.enable_car_car && count >= 2 && A.pairs) {
        const uint32_t reject = car_car_reject_mask(A.cars, A.cfgs, A.pairs, count);
        const int pc = count < 8 ? count : 8;
        const uint32_t all = pc >= 2 ? (1u << (pc * (pc - 1) / 2)) - 1u : 0u;
        if ((reject & all) != all) {
            int8_t oi[28], oj[28];
            int no = 0;
            uint32_t listed = 0u;
            // the list as built, before its island sort (the reference sorts after the car pairs, env_step.hpp:5186)
            const int n_built = bp.manifold_count < kBpMaxEntries ? bp.manifold_count : kBpMaxEntries;
            for (int e = 0; e < n_built; ++e) {
                const uint32_t key = bp.manifolds[e];
                if (bp_kind(key) != 3) continue;
                const int x = bp_body_a(key), y = bp_body_b(key);
                const int pi = x < y ? x : y, pj = x < y ? y : x;
                if (pi < 0 || pj >= count || pj >= 8 || pi == pj) continue;
                const uint32_t bit = 1u << car_pair_slot(pi, pj);
                if (listed & bit) continue;
                listed |= bit;
                if (reject & bit) continue;
                oi[no] = static_cast<int8_t>(pi);
                oj[no] = static_cast<int8_t>(pj);
                ++no;
            }
            for (int pi = 0; pi < count && pi < 8; ++pi)
                for (int pj = pi + 1; pj < count && pj < 8; ++pj) {
                    const uint32_t bit = 1u << car_pair_slot(pi, pj);
                    if ((listed & bit) || (reject & bit)) continue;
                    if (no < 28) {
                        oi[no] = static_cast<int8_t>(pi);
                        oj[no] = static_cast<int8_t>(pj);
                        ++no;
                    }
                }
            for (int po = 0; po < no; ++po) {
                const int i = oi[po], j = oj[po];
                car_car_touched |= (1u << i) | (1u << j);
                // Bullet's body order in the pair: the car whose sweep handle is lower is body 0
                const bool i_body0 = bp.body_handle[i + 1] <= bp.body_handle[j + 1];
                const int a = i_body0 ? j : i, b2 = i_body0 ? i : j;
                car_car_resolve(A.cars[a], static_cast<uint32_t>(A.car_base + a + 1), A.teams[a], A.cfgs[a], A.cars[b2],
                                static_cast<uint32_t>(A.car_base + b2 + 1), A.teams[b2], A.cfgs[b2], c, pre[a], pre[b2],
                                snap.car_start_vel[a], snap.car_start_vel[b2], a, b2, A.pairs[car_pair_slot(i, j)], pr);
            }
        }
    }
    // car-ball contacts, in slot order: a car whose box AABB meets the ball's takes part (reference
    // env_step.hpp:5045-5133; a car with no valid proxy is demolished and never overlaps,
    // BallCarRetainedPairOverlaps)
    BallCarRows bc;
    bc.nv = bc.nf = bc.ns = 0;
    for (int i = 0; i < count && i < 8; ++i) {
        const BpProxy& pb = proxies[0];
        const BpProxy& pc = proxies[i + 1];
        CarState& car = A.cars[i];
        // a car touched by a car pair tests its current box instead of its swept proxy
        // (reference BallCarRetainedPairOverlaps, triangle_and_carcar.hpp:1658-1698)
        const bool overlaps =
            ((car_car_touched >> i) & 1u)
                ? ball_car_box_overlaps(b, car, A.cfgs[i], c, pre[i].is_demoed == 0)
                : (i + 1 < body_count && pc.valid != 0 && !car.just_respawned &&
                   !(pc.child_min.x > pb.child_max.x || pc.child_max.x < pb.child_min.x ||
                     pc.child_min.y > pb.child_max.y || pc.child_max.y < pb.child_min.y ||
                     pc.child_min.z > pb.child_max.z || pc.child_max.z < pb.child_min.z));
        if (!overlaps) {
            bcs[i].count = 0;
            continue;
        }
        if (stages && stages[i].ball_staged) {
            bcs[i] = stages[i].ball_manifold;
            ball_car_manifold_rows(bcs[i], b, car, A.cfgs[i], c, i, ext_delta, solver_vel_bt, sub_dt, bc);
        } else {
            ball_car_contacts(bcs[i], b, car, A.cfgs[i], c, i, ext_delta, solver_vel_bt, sub_dt, bc);
        }
        if (!pre[i].is_demoed && !car.just_respawned)
            commit_ball_hit_from_manifold(b, car, bcs[i], static_cast<uint32_t>(A.car_base + i + 1), env_tick,
                                          hit_car_pos[i], hit_car_rot[i], hit_ball_pos, snap.car_start_vel[i],
                                          snap.ball_start_vel, A.teams[i], c.events);
    }
    // the ball's arena contacts (reference env_step.hpp:5219-5290): a sleeping ball a car touched is awake now,
    // and looks at the arena when it still holds arena contact points
    const bool awake_after = awake || bc.nv > 0 || bc.nf > 0 || bc.ns > 0;
    BallContactRows rows;
    rows.split_count = rows.vel_count = rows.fric_count = 0;
    if (awake_after && (awake || s.count != 0))
        ball_mesh_contacts(b, s, c, mesh, ext_delta, solver_vel_bt, sub_dt, rows, A.car_base / A.max_cars);
    // the cars' arena contacts, in slot order
    CarWorldRows cr;
    cr.nv = cr.nf = cr.ns = 0;
    for (int i = 0; i < count; ++i) {
        CarState& car = A.cars[i];
        if (pre[i].is_demoed || car.just_respawned) {
            cws[i].count = 0;
            continue;
        }
        bool listed = false;
        for (int e = 0; e < n_list; ++e) {
            const uint32_t key = list[e].key;
            listed = listed || (bp_kind(key) == 2 && bp_body_a(key) == i && bp_static(key) == 0);
        }
        if (!listed && cws[i].count == 0) continue;
        CarWorldContactResult res;
        MeshContactEvents ev;
        const MeshContactEvents* events = nullptr;
        if (!stages) {
            res = car_mesh_contacts(car, A.cfgs[i], cws[i], listed, mesh, c, i, cr, c.events.windows ? &ev : nullptr);
            events = &ev;
        } else if (!listed) {
            cws[i].count = 0;  // what the query does for an unlisted manifold
            continue;
        } else {
            cws[i] = stages[i].ws;
            append_car_rows(cr, stages[i].rows);
            res = stages[i].res;
            events = &stages[i].mesh_events;
        }
        if (c.events.windows) {
            for (uint32_t k = 0; k < events->count; ++k) {
                PhysicsEvent e = new_event(kEventCarWorldContact);
                e.car_id = static_cast<uint32_t>(A.car_base + i + 1);
                e.position = car.pos;  // as the car stands here: a pair's rows may have rewritten its uu origin
                e.car_velocity = car.vel;
                e.car_on_ground = car.is_on_ground;
                e.normal = events->normal[k];
                emit_event_for_car(c.events, e.car_id, e);
            }
        }
        if (res.hit) {
            car_record_world_surface(car, true);
            car.world_contact.has_contact = 1;
            car.world_contact.contact_normal = res.latest_normal;
        }
    }
    // predictive rows, in the list's predictive order (reference AppendPredictiveContactRows)
    for (int k = 0; k < bp.predictive_count; ++k) {
        const uint32_t key = bp.predictive[k];
        const int body = bp_entry_body(key);
        if (((pred_mask >> body) & 1u) == 0u) continue;
        if (body == 0) {
            ball_predictive_rows(b, c, pred_n[0], pred_d[0], ext_delta, solver_vel_bt, sub_dt, rows);
            continue;
        }
        const int i = body - 1;
        const CarState& car = A.cars[i];
        const V3 zero{0.0f, 0.0f, 0.0f};
        const V3 n = pred_n[body];
        const V3 tangent = contact_tangent(n, car.vel_bt + car.ext_force_impulse_bt);
        car_contact_rows(cr, i, 100 + kBpPredictiveId, car, n, zero, pred_d[body], zero, zero, tangent, zero,
                         1.0f / c.car_mass, 0.0f, c.arena_friction, sub_dt);
    }
    // a car with a predictive contact takes the game normal of all its arena rows (reference
    // ApplyPredictiveCarWorldContactNormal, arena_ball.hpp:168-205)
    for (int i = 0; i < count && i < 8; ++i) {
        if (((pred_mask >> (i + 1)) & 1u) == 0u || !A.cars[i].world_contact.has_contact) continue;
        V3 sum{0.0f, 0.0f, 0.0f};
        bool any = false;
        for (int pass = 0; pass < 2; ++pass) {
            const int tag = pass == 0 ? 100 : 100 + kBpPredictiveId;
            for (int r = 0; r < cr.nv; ++r) {
                if (cr.vel[r].body != i || cr.vel[r].tag != tag) continue;
                sum += cr.vel[r].normal;
                any = true;
            }
        }
        const float l2 = dot(sum, sum);
        if (any && l2 >= 1e-8f) {
            const V3 nn = sum * (1.0f / sqrtf(l2));
            A.cars[i].world_contact.contact_normal = V3{0.0f + nn.x, 0.0f + nn.y, 0.0f + nn.z};
        }
    }
    // velocity solve
    if (rows.vel_count || rows.fric_count || cr.nv || cr.nf || bc.nv || bc.nf || pr.nv || pr.nf) {
        V3 dl{0, 0, 0}, da{0, 0, 0};
        V3 cdl[8], cda[8];
        for (int i = 0; i < count; ++i) cdl[i] = cda[i] = V3{0.0f, 0.0f, 0.0f};
        unified_velocity_solve(rows, bc, cr, pr, list, n_list, dl, da, cdl, cda);
        ball_set_vel_bt(b, solver_vel_bt + dl);
        b.ang_vel = b.ang_vel + da;
        for (int i = 0; i < count; ++i) {
            car_set_vel_bt(A.cars[i], A.cars[i].vel_bt + cdl[i]);
            A.cars[i].ang_vel = A.cars[i].ang_vel + cda[i];
        }
    }
    // position (split-impulse) solve
    if (rows.split_count || cr.ns || bc.ns || pr.ns) {
        V3 cpush[8], cturn[8];
        bool cbt[8];
        const V3 push = unified_split_solve(rows, bc, cr, pr, list, n_list, cpush, cturn, cbt, count);
        if (!is_zero(push)) ball_set_pos_bt(b, b.pos_bt + push * sub_dt);
        for (int i = 0; i < count; ++i) {
            CarState& car = A.cars[i];
            const bool nonzero = !is_zero(cpush[i]) || !is_zero(cturn[i]);
            bool turn;
            if (cbt[i]) {
                turn = nonzero;
                if (nonzero) car_set_pos_bt(car, car.pos_bt + cpush[i] * sub_dt);
            } else {
                turn = len2(cturn[i]) > 0.0f;
                car_set_pos_bt(car, car.pos_bt + uu_to_bt_div(cpush[i]) * sub_dt);
            }
            if (turn)
                game_integrate_orientation(car.basis_forward, car.basis_right, car.basis_up, car.rot,
                                           cturn[i] * 0.1f, sub_dt);
        }
    }
    // the ball's gravity, integration and deactivation clock
    if (!ball_sleeping) ball_set_vel_bt(b, b.vel_bt + uu_to_bt_div(ext_delta));
    if (awake_after) {
        ball_integrate(b, sub_dt);
        b.sleeping = 0;
        const bool below = len2(b.vel_bt) < kBallLinearSleepBt * kBallLinearSleepBt &&
                           len2(b.ang_vel) < kBallAngularSleep * kBallAngularSleep;
        b.deactivation_time = below && !ball_sleeping ? b.deactivation_time + sub_dt : 0.0f;
    }
    // each car's integration (car_world_finish) follows in car_tick_post, one thread per car
}

// The game's extra ball-hit impulses of this tick, as a velocity change of the ball (reference ApplyBallExtraHits,
// env_step.hpp:6929-6948).
RG_HDI void apply_ball_extra_hits(BallState& b, CarState* cars, int count, const TickConfig& c) {
    const float inv = 1.0f / c.ball_mass;
    const float mass_bt = 1.0f / inv;
    V3 v = b.vel_bt;
    bool any = false;
    for (int i = 0; i < count; ++i) {
        BallHitInfo& h = cars[i].ball_hit_info;
        if (!h.extra_pending) continue;
        const V3 a = h.extra_hit_vel;
        v = V3{v.x + ((a.x * 0.02f) * mass_bt) * inv, v.y + ((a.y * 0.02f) * mass_bt) * inv,
               v.z + ((a.z * 0.02f) * mass_bt) * inv};
        h.extra_pending = 0;
        any = true;
    }
    if (any) ball_set_vel_bt(b, v);
}

// A tick of an arena with cars runs in six parts, so that each car's own work runs one thread per car:
//   arena_tick_begin   (per arena)  this tick's env command, the game's vehicle order, the ball's tick start, pad timers;
//   car_tick_pre       (per car)    the car's tick start (demolition timer and respawn, quantisation, controls, jumps);
//   vehicle_update + car_stage_compute (per car, cars no other car's wheels can reach and whose wheels reach no other
//                                   car, arena_free_cars)
//                                   the vehicle update, then the car's prestep, predictive contact, broadphase proxy
//                                   and mesh contact query (CarStage);
//   arena_tick_finish  (per arena)  the other cars' vehicle updates in car order and their staged parts, the wheel
//                                   pushes on the ball in car order, the world step's shared stages (manifold list,
//                                   car/car, car/ball, ball/mesh contacts, the unified solves, the ball's
//                                   integration);
//   car_tick_post      (per car)    the car's integration and post-tick;
//   arena_tick_tail    (per arena)  pads in car order, the driving countdown, extra ball hits, goal and timers.
// Reordering is exact: each per-car part reads and writes only that car (the ball only through its position, which
// none of them moves), and the arena parts keep the reference's order for everything shared
// (reference StepEnvGeneric, env_step.hpp:7088-7180).

// What the world step needs from one car's tick start and vehicle update.
struct CarTickRecord {
    V3 start_vel;  // uu velocity right after the tick-start quantisation (ball-hit impulse)
    V3 vel_bt, ang_vel;  // velocities the broadphase predicts motion with
    WheelBallPushes pushes;
};
// The ball's velocities at the tick start.
struct ArenaTickSnap {
    V3 ball_start_vel, ball_vel_bt;
};

// respawn_seed and env_idx are the respawn draw's: the batch's last kickoff seed and the arena's logical index.
RG_HDI void arena_tick_begin(EnvState& env, BallState& b, const ArenaCars& A, const TickConfig& c,
                             const PadLayout& pads_layout, ArenaTickSnap& as, uint64_t respawn_seed, int env_idx) {
    const int count = A.count;
    update_game_visit_order(env, A.cars, count);
    pick_respawn_spots(A, b, env, c, respawn_seed, env_idx);
    if (c.events.windows) c.events.windows[env_idx].tick = env.tick;  // reference StepEnvPreTickEnvState, :6694-6696
    env.goal_scored_this_tick = 0;
    ball_tick_start_quantize(b, c);
    as.ball_start_vel = b.vel;
    ball_clamp_and_drag(b, c);
    as.ball_vel_bt = b.vel_bt;
    if (c.enable_boost_pads && count > 0 && A.pads)
        for (int p = 0; p < pads_layout.count; ++p) pad_pre_tick(A.pads[p], c.tick_dt);
}

RG_HDI void car_tick_pre(CarState& car, const CarControls& k, const CarConfig& cfg, const TickConfig& c,
                         WheelRuntime& w, const RespawnCtx& rc, CarTickRecord& r) {
    r.start_vel = car_pre_tick(car, k, cfg, c, w, rc);
    r.vel_bt = car.vel_bt;
    r.ang_vel = car.ang_vel;
    r.pushes.count = 0;
    r.pushes.world_event = 0u;
}

// The cars of an arena whose vehicle update is independent of the other cars': no other car can be under one of its
// wheel rays (each other car is demolished or excluded for its rays by the sweep-box rule, wheel_ray_excluded_bodies:
// the reference never tests those) and it is under no other car's rays. Their updates (and their staged world-step
// parts) run one thread per car; the other cars' updates run in the game's car order in the arena thread, because a
// wheel that lands on another car pushes that car at once. Every thread of the arena evaluates this alike from the
// cars' poses after their tick start, which no vehicle update changes.
RG_HDI uint32_t arena_free_cars(const CarState* cars, const CarConfig* cfgs, const Broadphase& bp, int count) {
    uint32_t reach[8];
    uint32_t under = 0u;
    for (int i = 0; i < count && i < 8; ++i) {
        reach[i] = 0u;
        if (cars[i].is_demoed) continue;
        const uint32_t ex = wheel_ray_excluded_bodies(cars[i], cfgs[i], &bp, i, count);
        for (int j = 0; j < count && j < 8; ++j)
            if (j != i && !cars[j].is_demoed && !((ex >> (j + 1)) & 1u)) reach[i] |= 1u << j;
        under |= reach[i];
    }
    uint32_t free = 0u;
    for (int i = 0; i < count && i < 8; ++i)
        if (reach[i] == 0u && !((under >> i) & 1u)) free |= 1u << i;
    return free;
}

// Whether any wheel ray of the arena's cars meets another car's box this tick (from the rays cast ahead). When none
// does, no vehicle update pushes another car or sees one, and every car's update depends on the car alone.
RG_HDI bool arena_wheels_meet_cars(const CarStage* stages, int count) {
    uint32_t any = 0u;
    for (int i = 0; i < count; ++i)
        any |= stages[i].wheel_meets_car[0] | stages[i].wheel_meets_car[1] | stages[i].wheel_meets_car[2] |
               stages[i].wheel_meets_car[3];
    return any != 0u;
}

RG_HDI void arena_tick_finish(EnvState& env, BallState& b, BallWorldScratch& s, Broadphase& bp, CarWorldScratch* cws,
                              BallCarScratch* bcs, const TickConfig& c, const MeshDevice& mesh, const ArenaCars& A,
                              CarTickRecord* recs, const ArenaTickSnap& as, CarStage* stages) {
    // stages[i].in_car_thread: car i's vehicle update and staged parts ran in its own thread this tick
    const int count = A.count;
    int order[8];
    TickSnap snap;
    for (int k = 0; k < count; ++k) order[k] = car_visit_slot(env, k, count);
    for (int i = 0; i < count && i < 8; ++i) {
        snap.car_start_vel[i] = recs[i].start_vel;
        snap.car_vel_bt[i] = recs[i].vel_bt;
        snap.car_ang_vel[i] = recs[i].ang_vel;
    }
    snap.ball_start_vel = as.ball_start_vel;
    snap.ball_vel_bt = as.ball_vel_bt;
    // cars whose wheels may land on other cars: vehicle updates in the game's car order, wheels seeing other cars,
    // then their staged world-step parts (after every update: a later car's wheel may push an earlier one)
    uint32_t left = 0u;
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        if (stages[i].in_car_thread) continue;
        left |= 1u << i;
        const uint32_t excluded = A.cars[i].is_demoed ? 0u : wheel_ray_excluded_bodies(A.cars[i], A.cfgs[i], &bp, i, count);
        vehicle_update(A.cars[i], A.controls[i], A.cfgs[i], c, A.wheels[i], b, mesh,
                       WheelOthers{A.cars, A.cfgs, count, i, excluded}, recs[i].pushes, stages[i].wheel_mesh);
    }
    for (int i = 0; i < count; ++i)
        if ((left >> i) & 1u)
            car_stage_compute(A.cars[i], A.cfgs[i], A.wheels[i], cws[i], c, mesh, i, recs[i].vel_bt, recs[i].ang_vel,
                              stages[i]);
    if (c.events.windows) {
        // the vehicle updates' car-world events, in the game's car order (each update emits its own in the reference)
        for (int k = 0; k < count; ++k) {
            const int i = order[k];
            const WheelBallPushes& p = recs[i].pushes;
            if (!p.world_event) continue;
            PhysicsEvent e = new_event(kEventCarWorldContact);
            e.car_id = static_cast<uint32_t>(A.car_base + i + 1);
            e.position = p.world_event_pos;
            e.car_velocity = p.world_event_vel;
            e.car_on_ground = p.world_event_on_ground;
            e.normal = p.world_event_normal;
            emit_event(c.events, static_cast<uint32_t>(A.car_base / A.max_cars), e);
        }
    }
    for (int k = 0; k < count; ++k) apply_wheel_ball_pushes(b, recs[order[k]].pushes, c);
    PreContactCar pre[8];
    world_step_cars(b, s, bp, cws, bcs, c, mesh, A, pre, snap, env.tick, stages);
    for (int i = 0; i < count; ++i) stages[i].pre = pre[i];  // for the car's own finish (car_tick_post)
}

// Tick part 5, per car: the car's integration, then its post-tick (reference WorldStepFinishCar + StepEnvPostCar,
// env_step.hpp:6902-6925). Each car reads and writes only itself, so the cars of an arena run in any order.
RG_HDI void car_tick_post(CarState& car, const PreContactCar& pre, const CarControls& k, const WheelRuntime& w,
                          const TickConfig& c, bool report_fields, const CarConfig& cfg, const PadState* pads,
                          const PadLayout& pads_layout, PadContacts& pad_contacts) {
    car_world_finish(car, pre, c.tick_dt);
    // a car demolished during this world step reports the rotation it had when the step began (reference
    // StepEnvPostCar, env_step.hpp:6915-6918)
    if (!pre.is_demoed && !car.just_respawned && car.is_demoed) car.rot = pre.rot;
    car_post_tick(car, k, c.tick_dt);
    car_finish_tick(car);
    if (report_fields) {
        report_rlbot_fields(car, w, c);
    } else {
        advance_rlbot_fields(car, w, c);
    }
    if (pads && c.enable_boost_pads && !(c.frame_frac < 0.0f))
        pad_contacts_stage(car, cfg, pads, pads_layout, c, pad_contacts);
}

// Tick part 6, per arena: pads in the game's car order, the driving countdown, the ball's extra hit impulses and the
// env tail (reference StepEnvTail, env_step.hpp:6968-7046).
RG_HDI void arena_tick_tail(EnvState& env, BallState& b, const ArenaCars& A, const PadLayout& pads_layout,
                            const TickConfig& c, const CarStage* stages) {
    const int count = A.count;
    int order[8];
    for (int k = 0; k < count; ++k) order[k] = car_visit_slot(env, k, count);
    if (A.pads)
        pads_tail(A.cars, A.car_base, A.max_cars, A.cfgs, count, order, A.pads, pads_layout, c, &stages[0].pads,
                  sizeof(CarStage));
    for (int k = 0; k < count; ++k) {
        CarState& car = A.cars[order[k]];
        if (!car.is_demoed && car.driving_disabled) --car.driving_disabled;
    }
    apply_ball_extra_hits(b, A.cars, count, c);
    env_tail(env, b, c, A.cars, count, A.car_base / A.max_cars);
}

// ---- env commands ------------------------------------------------------------------------------------------------
// One arena's command (byte-identical to rg_env_command / the reference's EnvCommand, rocketgpu.h:683-706).
constexpr uint16_t kKickoffCountdownTicks = 480;         // reference rocketgpu.h:632: driving off for 4 s
constexpr uint16_t kKickoffCountdownGameTimers = 0xFFFF;  // reference rocketgpu.h:635: until the game timers end it

struct EnvCommand {
    uint8_t reset_to_kickoff, reset_scoreboard, reset_tick_count, kickoff_seed_mode, new_round_bodies, keep_boost_pads;
    uint16_t kickoff_countdown_ticks;
    uint64_t kickoff_seed;
};
static_assert(sizeof(EnvCommand) == sizeof(rg_env_command), "EnvCommand layout");

RG_HD bool env_command_active(const EnvCommand& c) {
    return (c.reset_to_kickoff | c.reset_scoreboard | c.reset_tick_count | c.new_round_bodies) != 0;
}

// The persistent contact state of one arena an env command may clear.
struct ArenaContactState {
    BallWorldScratch* ball_world;
    Broadphase* bp;
    CarWorldScratch* car_world;  // max_cars entries
    BallCarScratch* ball_car;    // max_cars entries
    CarCarManifold* pairs;       // pair_slots entries (may be null)
    int pair_slots;
};

RG_HDI void clear_retained_car_contacts(const ArenaContactState& s, int max_cars) {
    for (int k = 0; k < max_cars; ++k) {
        s.car_world[k].count = 0;
        s.ball_car[k].count = 0;
    }
    for (int k = 0; s.pairs && k < s.pair_slots; ++k) s.pairs[k].count = 0;
}

// An arena's env command between ticks (reference ApplyEnvCommandBodies + ApplyEnvCommand + ApplyEnvCommandEnvState,
// env_step.hpp:5672-5758, as BatchSim applies them, src/rocketgpu.cpp:2136-2218 and the tick-start command of
// StepEnvPreTickEnv, env_step.hpp:6701-6749):
//   * the bodies: a reset with the scoreboard starts a fresh sweep; a reset without it, or new_round_bodies, takes
//     every body out of the sweep the way the game respawns them after a goal (demolished cars first), and the
//     ball's and the cars' retained contacts start over;
//   * reset_to_kickoff: the arena's kickoff (the match's next kickoff when the scoreboard is kept and no seed is
//     given), every retained contact cleared, then the scoreboard / tick counter / countdown fields of the env.
// A command without reset_to_kickoff changes no env field (the reference applies the env fields only with a reset).
// kickoff_countdown_ticks != 0 makes it the game's countdown kickoff (cars held and placed a tick and a half later,
// driving off for that many ticks or, at 0xFFFF, until the countdown timers end it, the ball dropped from the game's
// height).
RG_HDI void apply_env_command(const EnvCommand& cmd, int env_idx, EnvState& env, BallState& ball,
                              const ArenaContactState& cs, const ArenaCars& A, CarControls* controls,
                              const PadLayout& L, const TickConfig& tc) {
    if (!env_command_active(cmd)) return;
    const int count = A.count;
    if (cmd.reset_to_kickoff && cmd.reset_scoreboard) {
        memset(cs.bp, 0, sizeof(Broadphase));
    } else if (cmd.reset_to_kickoff || cmd.new_round_bodies) {
        uint8_t demoed[8];
        for (int i = 0; i < count && i < 8; ++i) demoed[i] = A.cars[i].is_demoed;
        bp_new_round(*cs.bp, count, demoed);
        memset(cs.ball_world, 0, sizeof(BallWorldScratch));
        clear_retained_car_contacts(cs, A.max_cars);
    }
    if (!cmd.reset_to_kickoff) return;
    KickoffReset how;
    how.preserve_score = cmd.reset_scoreboard == 0;
    how.seed_mode = cmd.kickoff_seed_mode;
    how.keep_pads = cmd.keep_boost_pads != 0;
    how.game_spawn = cmd.kickoff_countdown_ticks != 0;
    reset_env_to_kickoff(env_idx, cmd.kickoff_seed, env, ball, *cs.ball_world, A.cars, A.wheels, A.cfgs, controls,
                         A.pads, L, A.teams, count, A.max_cars, tc, A.settled_entry, how);
    clear_retained_car_contacts(cs, A.max_cars);
    // the countdown: driving off for its ticks (or until the game timers end it), the ball held in its plane
    // (reference ApplyEnvCommand, env_step.hpp:5747-5752)
    for (int k = 0; k < count; ++k) A.cars[car_visit_slot(env, k, count)].driving_disabled = cmd.kickoff_countdown_ticks;
    ball.constrained_2d = cmd.kickoff_countdown_ticks;
    if (cmd.reset_scoreboard) {
        env.blue_score = 0;
        env.orange_score = 0;
        env.last_scored_team = -1;
    }
    if (cmd.reset_tick_count) env.tick = 0;
    env.goal_scored_this_tick = 0;
    env.countdown_phase = cmd.kickoff_countdown_ticks == kKickoffCountdownGameTimers ? 1 : 0;
    env.countdown_fires = 0;
    env.countdown_count = 0.0f;
}

}  // namespace rg
