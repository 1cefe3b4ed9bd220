// One 120 Hz tick of one arena (host+device). Ball-only arenas in this build: the ball's pre-tick network
// quantisation, speed caps and drag, Bullet activation / sleeping, the world step (gravity, contacts with the arena
// mesh, integration) and the tail (ball finish, goal test, render-frame timers, tick counter).
//
// Phase order and arithmetic follow the reference's per-env tick, StepEnvGeneric
// (include/rocketgpu/detail/step/env_step.hpp:7048-7180), with the ball-only branches of WorldStepSoccar
// (env_step.hpp:4622-5623) and StepEnvTail (env_step.hpp:6968-7045).
#pragma once

#include "rg_ball_world.cuh"
#include "rg_math.cuh"
#include "rg_pads.cuh"
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
RG_HDI void env_tail(EnvState& env, BallState& b, const TickConfig& c, CarState* cars = nullptr, int count = 0) {
    ball_finish(b);
    if (c.enable_scoring) {
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
RG_HDI void ball_world_step(BallState& b, BallWorldScratch& s, const TickConfig& c, const MeshDevice& mesh) {
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
    if (awake) ball_mesh_contacts(b, s, c, mesh, ext_delta, solver_vel_bt, sub_dt, rows);
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
RG_HDI void arena_tick(EnvState& env, BallState& b, BallWorldScratch& s, const TickConfig& c,
                       const MeshDevice& mesh) {
    env.goal_scored_this_tick = 0;
    ball_tick_start_quantize(b, c);
    ball_clamp_and_drag(b, c);
    ball_world_step(b, s, c, mesh);
    env_tail(env, b, c);
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
RG_HDI void car_pre_tick(CarState& c, const CarControls& k, const CarConfig& cfg, const TickConfig& tc, WheelRuntime& w) {
    c.ball_contact_this_tick = 0;
    restore_step_fields(c);
    if (c.tick_count_since_update == 0) cal_internal_timers_from_set_state(c, tc);
    if (c.just_respawned) c.just_respawned = 0;
    if (c.is_demoed) {
        c.demo_respawn_timer = fmax_(0.0f, c.demo_respawn_timer - tc.tick_dt);
        if (!(c.demo_respawn_timer <= 0.0f) && !(fmax_(0.0f, c.demo_respawn_timer - tc.tick_dt) > 0.0f) &&
            !(c.respawn_slot_override_plus1 >= kKickoffSpawnOverridePlus1 &&
              c.respawn_slot_override_plus1 < kKickoffSpawnOverridePlus1 + 5)) {
            c.boost = tc.boost_spawn_amount;
            c.boost_amount = c.boost / 100.0f;
        }
    }
    c.tick_start_pos_bt = c.pos_bt;
    car_tick_start_quantize(c, tc);
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
}

// One tick of one arena with cars (reference StepEnvGeneric, env_step.hpp:7088-7180, and WorldStepSoccar for cars
// that touch nothing but the air: car contacts with the arena, the ball and each other are not built yet).
RG_HDI void arena_tick_cars(EnvState& env, BallState& b, BallWorldScratch& s, const TickConfig& c,
                            const MeshDevice& mesh, const ArenaCars& A, const PadLayout& pads_layout,
                            bool report_fields) {
    const int count = A.count;
    update_game_visit_order(env, A.cars, count);
    env.goal_scored_this_tick = 0;
    int order[8];
    for (int k = 0; k < count; ++k) order[k] = car_visit_slot(env, k, count);
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        car_pre_tick(A.cars[i], A.controls[i], A.cfgs[i], c, A.wheels[i]);
    }
    ball_tick_start_quantize(b, c);
    ball_clamp_and_drag(b, c);
    if (c.enable_boost_pads && count > 0 && A.pads)
        for (int p = 0; p < pads_layout.count; ++p) pad_pre_tick(A.pads[p], c.tick_dt);
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        vehicle_update(A.cars[i], A.controls[i], A.cfgs[i], c, A.wheels[i], b, mesh);
    }
    PreContactCar pre[8];
    for (int i = 0; i < count; ++i) car_world_prestep(A.cars[i], A.cfgs[i], A.wheels[i], c, c.tick_dt, pre[i]);
    ball_world_step(b, s, c, mesh);
    for (int i = 0; i < count; ++i) car_world_finish(A.cars[i], pre[i], c.tick_dt);
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        CarState& car = A.cars[i];
        car_post_tick(car, A.controls[i], c.tick_dt);
        car_finish_tick(car);
        if (report_fields) {
            report_rlbot_fields(car, A.wheels[i], c);
        } else {
            advance_rlbot_fields(car, A.wheels[i], c);
        }
    }
    if (A.pads) pads_tail(A.cars, A.car_base, A.max_cars, A.cfgs, count, order, A.pads, pads_layout, c);
    for (int k = 0; k < count; ++k) {
        CarState& car = A.cars[order[k]];
        if (!car.is_demoed && car.driving_disabled) --car.driving_disabled;
    }
    env_tail(env, b, c, A.cars, count);
}

}  // namespace rg
