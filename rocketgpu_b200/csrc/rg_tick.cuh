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
// CountdownUpdateTimers :6516-6537).
RG_HDI void env_tail(EnvState& env, BallState& b, const TickConfig& c) {
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

}  // namespace rg
