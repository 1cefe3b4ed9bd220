// rg_batch: the C ABI (include/rocketgpu_b200.h) and the sm_100a kernels behind it.
//
// Execution model. One CUDA thread owns one arena for the whole launch: it loads the arena's ball and env state from
// HBM once, runs `ticks` ticks with the state in registers, and stores it back once. Arenas are independent (the
// reference steps each env in isolation, include/rocketgpu/detail/step/env_step.hpp:7048), so a step is one launch
// of single-warp blocks with no inter-thread communication; at 16K arenas that is 512 blocks, about 3.5 per SM on the
// 148 SMs. Ticks per launch amortise the state load/store and launch latency.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "rg_mesh.h"
#include "rg_reset.cuh"
#include "rg_tick.cuh"
#include "rg_ucrt.cuh"
#include "rocketgpu_b200.h"

namespace {
thread_local std::string g_last_error;

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// A serving pool without room for a client's arenas (status 5, RG_BUSY): retry after other clients close.
struct ServerBusy : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F>
int guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_last_error = std::string("invalid_argument: ") + e.what();
        return 2;
    } catch (const std::out_of_range& e) {
        g_last_error = std::string("out_of_range: ") + e.what();
        return 3;
    } catch (const CudaError& e) {
        g_last_error = std::string("cuda: ") + e.what();
        return 4;
    } catch (const ServerBusy& e) {
        g_last_error = std::string("busy: ") + e.what();
        return 5;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 1;
    } catch (...) {
        g_last_error = "unknown error";
        return 1;
    }
}

template <class T>
struct DeviceArray {
    T* ptr = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        reset();
        n = count;
        if (count) check(cudaMalloc(&ptr, count * sizeof(T)), "cudaMalloc");
    }
    void reset() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        n = 0;
    }
    ~DeviceArray() {
        if (ptr) cudaFree(ptr);
    }
};

}  // namespace

struct rg_batch {
    int device = 0;
    rg_sim_config cfg{};
    rg::TickConfig tc{};
    int32_t env_count = 0;
    int32_t max_cars = 0;
    DeviceArray<rg::BallState> balls;
    DeviceArray<rg::EnvState> envs;
    DeviceArray<int32_t> env_car_count;
    DeviceArray<rg::BallWorldScratch> ball_world;
    DeviceArray<rg::CarState> cars;
    DeviceArray<rg::WheelRuntime> wheels;
    DeviceArray<rg::CarConfig> car_cfgs;
    DeviceArray<rg::CarControls> controls;
    DeviceArray<rg::PadState> pads;
    DeviceArray<uint8_t> teams;
    DeviceArray<rg::Broadphase> broadphase;    // per arena: sweep history and manifold list
    DeviceArray<rg::CarWorldScratch> car_world;  // per car slot: the car/mesh manifold
    DeviceArray<rg::BallCarScratch> ball_car;     // per car slot: the car/ball manifold
    DeviceArray<rg::CarCarManifold> car_pairs;   // per arena: max_cars * (max_cars - 1) / 2 retained car-car manifolds
    DeviceArray<rg::CarTickRecord> car_records;  // per car slot: this tick's record of the car's own update
    DeviceArray<rg::ArenaTickSnap> arena_snaps;  // per arena: the ball's velocities at this tick's start
    DeviceArray<rg::CarStage> car_stages;        // per car slot: its staged part of this tick's world step
    // Step order: arenas sorted by car count (so a warp's arenas take the same loops), and the active car slots of
    // those arenas in that order (one thread each in the per-car kernel). Rebuilt by set_env_car_count.
    DeviceArray<int32_t> arena_order;
    DeviceArray<int32_t> active_cars;
    int32_t active_car_count = 0;
    rg::PadLayout pad_layout{};
    DeviceArray<rg::ArenaRules> rules;  // a custom layout's spawns and goals (b->tc.rules points here), or empty
    // Pads stay at their initial state until a car exists or pads are uploaded; until then ball-only arenas skip them.
    bool pads_live = false;
    rg::MeshHost mesh_host;
    rg::MeshDevice mesh;
    // further geometries (rg_batch_add_mesh): all meshes, the create-time one first, and each arena's mesh index;
    // the table stays unallocated while the batch has one mesh
    std::vector<rg::MeshDevice> extra_meshes;
    DeviceArray<rg::MeshDevice> mesh_table;
    DeviceArray<uint8_t> mesh_of;
    std::vector<int32_t> host_car_count;
    std::vector<int32_t> host_arena_order, host_active_cars;
    int launch_threads = 32;      // threads per block of the per-arena kernels
    int car_threads = 64;         // threads per block of the per-car kernels
    int pair_slots = 0;
    // CUDA graphs of whole steps (rg_launch_config.use_graphs): one per (controls, stride, commands, stride, ticks),
    // captured on first use and replayed after; any change to what a step's launches capture (car counts, pads,
    // kickoff seed, meshes, launch config) moves graph_version on and drops them
    bool use_graphs = false;
    uint64_t graph_version = 0;
    cudaStream_t capture_stream = nullptr;
    struct StepGraph {
        const void *controls, *commands;
        int32_t control_stride, command_stride, ticks;
        uint64_t version, last_use;
        cudaGraphExec_t exec;
    };
    std::vector<StepGraph> graphs;
    uint64_t graph_clock = 0;
    DeviceArray<rg::EnvCommand> command_scratch;  // per arena: the host commands of rg_batch_apply_env_commands
    DeviceArray<uint32_t> device_status;          // reserved for device-side command errors (none today)
    DeviceArray<int64_t> episode_touch;           // per arena: the episode's latest ball touch (env ticks)
    DeviceArray<uint64_t> episode_seen;           // per car slot: latest_touch_tick at the previous episode check
    // Kickoff settling (cfg.kickoff_settled = 1): the create-time layout, kept to build the batch that records the
    // countdown; the (car config, team) entries recorded so far with their rows (settled_spawns per entry) and the
    // ball; the device copies b->tc.settled_* point at. New configs or teams record their entries before the next
    // reset (reference ensure_kickoff_settled, src/rocketgpu.cpp:1439-1500).
    std::vector<float> layout_vertices;
    std::vector<int32_t> layout_indices;
    bool layout_has_rules = false;
    rg_arena_rules layout_rules{};
    bool layout_has_pads = false;
    std::vector<rg_boost_pad_config> layout_pads;
    struct SettleEntry {
        rg::CarConfig config;
        uint8_t team;
    };
    std::vector<SettleEntry> settle_entries;
    std::vector<rg::KickoffSettledRow> settle_rows_host;
    std::vector<rg::BallState> settle_ball_host;
    bool settle_dirty = true;
    DeviceArray<rg::KickoffSettledRow> settle_rows;
    DeviceArray<int32_t> settle_entry;
    DeviceArray<rg::BallState> settle_ball;
    // Phase timing (rg_batch_phase_timing): events around the six kernels of every tick, seven per tick.
    bool timing = false;
    std::vector<cudaEvent_t> events;
    size_t events_used = 0;
    void drop_graphs() {
        for (StepGraph& g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
        ++graph_version;
    }
    ~rg_batch() {
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        drop_graphs();
        if (capture_stream) cudaStreamDestroy(capture_stream);
    }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) check(cudaSetDevice(dev), "cudaSetDevice");
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// Ball import: uu -> bt with the reference's one-ulp nudge so bt * 50 reproduces the uploaded uu value exactly, then
// uu recomputed from bt; the ball is marked "just uploaded" (sleeping = 2) (reference CanonicalizeImportedBallStates,
// src/rocketgpu.cpp:325-382).
__device__ float imported_linear_bt(float value) {
    const float bt = value * (1.0f / 50.0f);
    if (bt * 50.0f == value) return bt;
    const float up = nextafterf(bt, INFINITY);
    const float down = nextafterf(bt, -INFINITY);
    if (up * 50.0f == value) return up;
    if (down * 50.0f == value) return down;
    return bt;
}

__global__ void canonicalize_balls_kernel(rg::BallState* balls, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rg::BallState& b = balls[i];
    b.pos_bt = rg::V3{imported_linear_bt(b.pos.x), imported_linear_bt(b.pos.y), imported_linear_bt(b.pos.z)};
    b.vel_bt = rg::V3{imported_linear_bt(b.vel.x), imported_linear_bt(b.vel.y), imported_linear_bt(b.vel.z)};
    b.pos = b.pos_bt * 50.0f;
    b.vel = b.vel_bt * 50.0f;
    b.sleeping = 2;
    b.deactivation_time = 0.0f;
}

struct TickArgs {
    rg::BallState* balls;
    rg::EnvState* envs;
    const int32_t* env_car_count;
    rg::BallWorldScratch* ball_world;
    int32_t env_count;
    rg::TickConfig tc;
    rg::MeshDevice mesh;
    // arenas on more than one geometry (rg_batch_add_mesh / rg_batch_set_arena_meshes): arena e's mesh is
    // meshes[mesh_of[e]]; null: every arena on `mesh`
    const rg::MeshDevice* meshes;
    const uint8_t* mesh_of;
};

__device__ __forceinline__ const rg::MeshDevice& arena_mesh(const TickArgs& a, int e) {
    return a.meshes ? a.meshes[a.mesh_of[e]] : a.mesh;
}

__global__ void __launch_bounds__(256) tick_kernel(TickArgs a, int ticks) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.env_count) return;
    rg::BallState b = a.balls[e];
    rg::EnvState env = a.envs[e];
    rg::BallWorldScratch s = a.ball_world[e];
    const rg::MeshDevice& mesh = arena_mesh(a, e);
    for (int t = 0; t < ticks; ++t) {
        rg::arena_tick(env, b, s, a.tc, mesh, e);
    }
    a.balls[e] = b;
    a.envs[e] = env;
    a.ball_world[e] = s;
}

// Car import (reference CanonicalizeImportedCarStatesInPlace, src/rocketgpu.cpp:355-379): the working fields behind
// the report fields come back, training history resets, pos/vel go through the same uu -> bt nudge as the ball, and
// the orientation becomes Bullet's quaternion of the (authoritative) basis.
__global__ void canonicalize_cars_kernel(rg::CarState* cars, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rg::CarState& c = cars[i];
    c.pad_frame_pos_valid = 0;
    const uint8_t kept = c.tick_count_since_update != 0 ? rg::car_restore_working_fields(c) : 0;
    rg::car_reset_training_history(c);
    c.pos_bt = rg::V3{imported_linear_bt(c.pos.x), imported_linear_bt(c.pos.y), imported_linear_bt(c.pos.z)};
    c.vel_bt = rg::V3{imported_linear_bt(c.vel.x), imported_linear_bt(c.vel.y), imported_linear_bt(c.vel.z)};
    c.pos = c.pos_bt * 50.0f;
    c.vel = c.vel_bt * 50.0f;
    if (!c.basis_authoritative) {
        rg::upload_basis_from_rot(c.rot, c.basis_forward, c.basis_right, c.basis_up);
        c.basis_authoritative = 1;
    }
    c.rot = rg::bullet_quat_from_basis(c.basis_forward, c.basis_right, c.basis_up);
    rg::car_re_report_fields(c, kept);
}

// Per-arena tables of a serving pool (rg_server): ticks left in the arena's current request (0: idle this tick), the
// control row it reads next, its index among its client's arenas and its client's kickoff seed.
struct SlotTable {
    int32_t* remaining;
    int32_t* tick;
    const int32_t* logical;
    const uint64_t* seed;
};

struct CarTickArgs {
    TickArgs base;
    rg::CarState* cars;
    rg::WheelRuntime* wheels;
    const rg::CarConfig* car_cfgs;
    rg::PadState* pads;  // null while pads are not live
    const rg::CarControls* controls;
    int32_t control_stride;
    int32_t max_cars;
    rg::PadLayout pad_layout;
    rg::Broadphase* broadphase;
    rg::CarWorldScratch* car_world;
    rg::BallCarScratch* ball_car;
    rg::CarTickRecord* records;
    rg::ArenaTickSnap* snaps;
    rg::CarCarManifold* pairs;
    const uint8_t* teams;
    int32_t pair_slots;
    const int32_t* arena_order;
    const int32_t* active_cars;
    int32_t active_car_count;
    rg::CarStage* stages;
    const rg::EnvCommand* commands;  // step_with_device_commands: tick t's command for arena e at t * stride + e
    int32_t command_stride;
    rg::CarControls* reset_controls;  // the batch's held controls, cleared by a kickoff reset
    uint32_t* status;
    // Serving rounds (rg_server): a tick steps only arenas with ticks left, each reading its controls at its own row
    // and numbering its env and cars as in a batch of its own. Null: every arena steps, as a batch does.
    SlotTable slots;
};

// The control row arena e reads this tick: its own position in its request when serving, else the tick's.
__device__ __forceinline__ size_t control_row(const CarTickArgs& a, int e, int t) {
    return static_cast<size_t>(a.slots.remaining ? a.slots.tick[e] : t);
}
// The index the arena's RNG draws and car ids use (reference env_idx): its index in its client's arenas when serving.
__device__ __forceinline__ int logical_env(const CarTickArgs& a, int e) {
    return a.slots.remaining ? a.slots.logical[e] : e;
}
__device__ __forceinline__ bool arena_idle(const CarTickArgs& a, int e) {
    return a.slots.remaining && a.slots.remaining[e] <= 0;
}

__device__ __forceinline__ rg::ArenaCars arena_cars(const CarTickArgs& a, int e, int t) {
    const int car_base = e * a.max_cars;
    rg::ArenaCars A;
    A.cars = a.cars + car_base;
    A.wheels = a.wheels + car_base;
    A.cfgs = a.car_cfgs + car_base;
    A.pads = a.pads ? a.pads + static_cast<size_t>(e) * a.pad_layout.count : nullptr;
    A.controls = a.controls ? a.controls + control_row(a, e, t) * static_cast<size_t>(a.control_stride) + car_base
                            : nullptr;
    A.teams = a.teams + car_base;
    A.pairs = a.pair_slots ? a.pairs + static_cast<size_t>(e) * a.pair_slots : nullptr;
    A.settled_entry = a.base.tc.settled_entry ? a.base.tc.settled_entry + car_base : nullptr;
    A.count = a.base.env_car_count[e];
    A.max_cars = a.max_cars;
    A.car_base = logical_env(a, e) * a.max_cars;  // car ids are car_base + slot + 1
    return A;
}

__device__ __forceinline__ rg::ArenaContactState arena_contact_state(const CarTickArgs& a, int e) {
    rg::ArenaContactState cs;
    cs.ball_world = a.base.ball_world + e;
    cs.bp = a.broadphase + e;
    cs.car_world = a.car_world + static_cast<size_t>(e) * a.max_cars;
    cs.ball_car = a.ball_car + static_cast<size_t>(e) * a.max_cars;
    cs.pairs = a.pair_slots ? a.pairs + static_cast<size_t>(e) * a.pair_slots : nullptr;
    cs.pair_slots = a.pair_slots;
    return cs;
}

// Env commands between steps, one thread per arena (reference LaunchApplyEnvCommands / apply_env_commands_host,
// src/rocketgpu.cpp:2136-2218).
__global__ void apply_commands_kernel(CarTickArgs a, const rg::EnvCommand* cmds, int n, rg::CarControls* controls,
                                      uint32_t* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const rg::EnvCommand c = cmds[e];
    if (!rg::env_command_active(c)) return;
    rg::ArenaCars A = arena_cars(a, e, 0);
    rg::apply_env_command(c, e, a.base.envs[e], a.base.balls[e], arena_contact_state(a, e), A,
                          controls + static_cast<size_t>(e) * a.max_cars, a.pad_layout, a.base.tc);
}

// Tick part 1, one thread per arena in step order: this tick's env command (step_with_device_commands), vehicle
// order, the ball's tick start, pad timers.
__global__ void __launch_bounds__(256) arena_begin_kernel(CarTickArgs a, int t) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.base.env_count) return;
    const int e = a.arena_order[k];
    if (arena_idle(a, e)) return;
    if (a.commands) {
        const rg::EnvCommand c = a.commands[static_cast<size_t>(t) * static_cast<size_t>(a.command_stride) + e];
        if (rg::env_command_active(c))
            rg::apply_env_command(c, e, a.base.envs[e], a.base.balls[e], arena_contact_state(a, e),
                                  arena_cars(a, e, t), a.reset_controls + static_cast<size_t>(e) * a.max_cars,
                                  a.pad_layout, a.base.tc);
    }
    rg::BallState b = a.base.balls[e];
    rg::EnvState env = a.base.envs[e];
    rg::arena_tick_begin(env, b, arena_cars(a, e, t), a.base.tc, a.pad_layout, a.snaps[e],
                         a.slots.remaining ? a.slots.seed[e] : a.base.tc.kickoff_seed, logical_env(a, e));
    a.base.balls[e] = b;
    a.base.envs[e] = env;
}

// Tick part 2, one thread per active car: the car's tick start (demolition timer and respawn, quantisation, controls,
// jumps, dodges, boost) and the speed clamp.
__global__ void __launch_bounds__(256) car_pre_kernel(CarTickArgs a, int t) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.active_car_count) return;
    const int idx = a.active_cars[k];
    const int e = idx / a.max_cars;
    if (arena_idle(a, e)) return;
    const rg::CarControls& ctrl =
        a.controls[control_row(a, e, t) * static_cast<size_t>(a.control_stride) + static_cast<size_t>(idx)];
    const int le = logical_env(a, e);
    rg::RespawnCtx rc;
    rc.seed = a.slots.remaining ? a.slots.seed[e] : a.base.tc.kickoff_seed;
    rc.env_idx = le;
    rc.env_tick = a.base.envs[e].tick;
    rc.car_id = static_cast<uint32_t>(le * a.max_cars + (idx - e * a.max_cars) + 1);
    rc.team = a.teams[idx];
    // the car's structs are worked on in local copies: one burst of independent loads, after which the warp's
    // accesses to a field go to one interleaved local line instead of 32 lines of 880-byte-strided structs (measured:
    // faster here, where the tick start touches most of the car; slower in the post-tick, which touches little)
    rg::CarState car = a.cars[idx];
    rg::WheelRuntime wr = a.wheels[idx];
    const rg::CarConfig cfg = a.car_cfgs[idx];
    rg::car_tick_pre(car, ctrl, cfg, a.base.tc, wr, rc, a.records[idx]);
    a.cars[idx] = car;
    a.wheels[idx] = wr;
}

// Tick part 3, one thread per active car: the vehicle update (four suspension rays against the arena mesh and the
// ball, tyres, drive, air control) and the car's staged world-step parts, for cars whose wheels can land on no other
// car and under whose car no other wheel can land (rg::arena_free_cars); the others are left to part 4.
// Tick part 3a, one thread per wheel of an active car: the wheel's suspension ray against the arena mesh, cast ahead of
// the car's vehicle update (it reads only the car's pose and config, final once the car's tick start has run).
__global__ void __launch_bounds__(256) car_rays_kernel(CarTickArgs a, int t) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = g >> 2, wheel = g & 3;
    if (k >= a.active_car_count) return;
    const int idx = a.active_cars[k];
    const int e = idx / a.max_cars;
    if (arena_idle(a, e)) return;
    const rg::CarState& car = a.cars[idx];
    rg::CarStage& st = a.stages[idx];
    if (car.is_demoed) {  // a demolished car's vehicle update casts no rays
        st.wheel_meets_car[wheel] = 0;
        return;
    }
    const int base = e * a.max_cars, count = a.base.env_car_count[e], slot = idx - base;
    const uint32_t excluded = rg::wheel_ray_excluded_bodies(car, a.car_cfgs[idx], a.broadphase + e, slot, count);
    rg::wheel_mesh_ray_ahead(car, a.car_cfgs[idx], arena_mesh(a.base, e), wheel,
                             rg::WheelOthers{a.cars + base, a.car_cfgs + base, count, slot, excluded},
                             st.wheel_mesh[wheel], st.wheel_meets_car[wheel]);
}

__global__ void __launch_bounds__(256) car_vehicle_kernel(CarTickArgs a, int t) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.active_car_count) return;
    const int idx = a.active_cars[k];
    const int e = idx / a.max_cars;
    if (arena_idle(a, e)) return;
    const int base = e * a.max_cars;
    const int count = a.base.env_car_count[e];
    // the car's update runs here when no wheel of the arena meets another car, or when the sweep-box rule shows that
    // no other car can be under its wheels nor it under theirs
    const bool free =
        !rg::arena_wheels_meet_cars(a.stages + base, count) ||
        ((rg::arena_free_cars(a.cars + base, a.car_cfgs + base, a.broadphase[e], count) >> (idx - base)) & 1u);
    a.stages[idx].in_car_thread = free ? 1u : 0u;
    // every car's ball contact geometry, before its vehicle update (it reads poses only)
    rg::car_ball_stage(a.base.balls[e], a.snaps[e].ball_vel_bt, a.cars[idx], a.car_cfgs[idx], a.base.tc,
                       a.records[idx].vel_bt, a.records[idx].ang_vel, a.ball_car[idx], a.stages[idx]);
    if (!free) return;  // the arena thread updates this car in the game's car order
    const rg::CarControls& ctrl =
        a.controls[control_row(a, e, t) * static_cast<size_t>(a.control_stride) + static_cast<size_t>(idx)];
    const uint32_t excluded =
        a.cars[idx].is_demoed ? 0u
                              : rg::wheel_ray_excluded_bodies(a.cars[idx], a.car_cfgs[idx], a.broadphase + e, idx - base,
                                                              count);
    const rg::MeshDevice& mesh = arena_mesh(a.base, e);
    rg::vehicle_update(a.cars[idx], ctrl, a.car_cfgs[idx], a.base.tc, a.wheels[idx], a.base.balls[e], mesh,
                       rg::WheelOthers{nullptr, nullptr, 0, -1, excluded}, a.records[idx].pushes,
                       a.stages[idx].wheel_mesh);
    // the car's own part of the world step, while this thread has the car (rg::CarStage)
    rg::car_stage_compute(a.cars[idx], a.car_cfgs[idx], a.wheels[idx], a.car_world[idx], a.base.tc, mesh, idx - base,
                          a.records[idx].vel_bt, a.records[idx].ang_vel, a.stages[idx]);
}

// Tick part 4, one thread per arena in step order: the vehicle updates (and staged parts) of cars whose wheels may
// land on other cars, in the game's car order; wheel pushes on the ball; the world step's shared stages.
// One thread per arena fills a single wave at any batch this path runs, so these two kernels take the registers that
// remove most of their spills (measured at 16,384 mixed arenas: the finish 4.09 -> 3.91 ms per 8-tick step; the car
// kernels lost time under the same change, their spill-free register counts cost waves).
__global__ void __maxnreg__(255) arena_finish_kernel(CarTickArgs a, int t) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.base.env_count) return;
    const int e = a.arena_order[k];
    if (arena_idle(a, e)) return;
    rg::BallState b = a.base.balls[e];
    rg::BallWorldScratch s = a.base.ball_world[e];
    const int car_base = e * a.max_cars;
    rg::arena_tick_finish(a.base.envs[e], b, s, a.broadphase[e], a.car_world + car_base, a.ball_car + car_base,
                          a.base.tc, arena_mesh(a.base, e), arena_cars(a, e, t), a.records + car_base, a.snaps[e],
                          a.stages + car_base);
    a.base.balls[e] = b;
    a.base.ball_world[e] = s;
}

// Tick part 5, one thread per active car: its integration and post-tick.
__global__ void __launch_bounds__(256) car_post_kernel(CarTickArgs a, int t, int report_fields) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.active_car_count) return;
    const int idx = a.active_cars[k];
    const int e = idx / a.max_cars;
    if (arena_idle(a, e)) return;
    // serving: report fields after the request's last tick, as a batch reports them after a step's last tick
    const bool report = a.slots.remaining ? a.slots.remaining[e] == 1 : report_fields != 0;
    const rg::CarControls& ctrl =
        a.controls[control_row(a, e, t) * static_cast<size_t>(a.control_stride) + static_cast<size_t>(idx)];
    rg::car_tick_post(a.cars[idx], a.stages[idx].pre, ctrl, a.wheels[idx], a.base.tc, report, a.car_cfgs[idx],
                      a.pads ? a.pads + static_cast<size_t>(e) * a.pad_layout.count : nullptr, a.pad_layout,
                      a.stages[idx].pads);
}

// Tick part 6, one thread per arena in step order: pads, the driving countdown, extra ball hits, goal and timers.
__global__ void __maxnreg__(255) arena_tail_kernel(CarTickArgs a, int t) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.base.env_count) return;
    const int e = a.arena_order[k];
    if (arena_idle(a, e)) return;
    rg::BallState b = a.base.balls[e];
    rg::EnvState env = a.base.envs[e];
    rg::arena_tick_tail(env, b, arena_cars(a, e, t), a.pad_layout, a.base.tc, a.stages + static_cast<size_t>(e) * a.max_cars);
    a.base.balls[e] = b;
    a.base.envs[e] = env;
    if (a.slots.remaining) {
        --a.slots.remaining[e];
        ++a.slots.tick[e];
    }
}

CarTickArgs car_tick_args(rg_batch* b, const rg::CarControls* controls, int stride) {
    CarTickArgs a;
    a.base.balls = b->balls.ptr;
    a.base.envs = b->envs.ptr;
    a.base.env_car_count = b->env_car_count.ptr;
    a.base.ball_world = b->ball_world.ptr;
    a.base.env_count = b->env_count;
    a.base.tc = b->tc;
    a.base.mesh = b->mesh;
    a.base.meshes = b->mesh_table.ptr;
    a.base.mesh_of = b->mesh_table.ptr ? b->mesh_of.ptr : nullptr;
    a.cars = b->cars.ptr;
    a.wheels = b->wheels.ptr;
    a.car_cfgs = b->car_cfgs.ptr;
    a.pads = b->pads_live ? b->pads.ptr : nullptr;
    a.controls = controls;
    a.control_stride = stride;
    a.max_cars = b->max_cars;
    a.pad_layout = b->pad_layout;
    a.broadphase = b->broadphase.ptr;
    a.car_world = b->car_world.ptr;
    a.ball_car = b->ball_car.ptr;
    a.records = b->car_records.ptr;
    a.pairs = b->car_pairs.ptr;
    a.teams = b->teams.ptr;
    a.pair_slots = b->pair_slots;
    a.snaps = b->arena_snaps.ptr;
    a.arena_order = b->arena_order.ptr;
    a.active_cars = b->active_cars.ptr;
    a.active_car_count = b->active_car_count;
    a.stages = b->car_stages.ptr;
    a.commands = nullptr;
    a.command_stride = 0;
    a.reset_controls = b->controls.ptr;
    a.status = b->device_status.ptr;
    a.slots = SlotTable{};
    return a;
}

// Arenas with cars: four launches per tick (arena begin, per-car tick start, per-car vehicle update, arena finish).
void launch_car_tick(rg_batch* b, const rg::CarControls* controls, int stride, int ticks, cudaStream_t s,
                     const rg::EnvCommand* commands = nullptr, int command_stride = 0) {
    if (b->env_count == 0) return;
    CarTickArgs a = car_tick_args(b, controls, stride);
    a.commands = commands;
    a.command_stride = command_stride;
    if (commands) {
        // a reset may give pads their initial state and put cars on the field: pads take part from here on
        a.pads = b->pads.ptr;
        b->pads_live = true;
    }
    const int threads = b->launch_threads;
    const int blocks = (b->env_count + threads - 1) / threads;
    const int ct = b->car_threads;
    const int car_blocks = (b->active_car_count + ct - 1) / ct;
    const int wheel_blocks = (4 * b->active_car_count + ct - 1) / ct;
    auto mark = [&] {
        if (!b->timing) return;
        if (b->events_used == b->events.size()) {
            cudaEvent_t e;
            check(cudaEventCreate(&e), "cudaEventCreate");
            b->events.push_back(e);
        }
        check(cudaEventRecord(b->events[b->events_used++], s), "cudaEventRecord");
    };
    for (int t = 0; t < ticks; ++t) {
        mark();
        arena_begin_kernel<<<blocks, threads, 0, s>>>(a, t);
        mark();
        if (car_blocks) car_pre_kernel<<<car_blocks, ct, 0, s>>>(a, t);
        mark();
        // phase 2 (timing) is the wheel rays and the vehicle updates
        if (car_blocks) car_rays_kernel<<<wheel_blocks, ct, 0, s>>>(a, t);
        if (car_blocks) car_vehicle_kernel<<<car_blocks, ct, 0, s>>>(a, t);
        mark();
        arena_finish_kernel<<<blocks, threads, 0, s>>>(a, t);
        mark();
        // report fields after the last tick, and after every tick of a command stream (reference StepEnvGeneric,
        // env_step.hpp:7174: report_fields = last tick || has_commands)
        if (car_blocks) car_post_kernel<<<car_blocks, ct, 0, s>>>(a, t, (t + 1 == ticks || commands) ? 1 : 0);
        mark();
        arena_tail_kernel<<<blocks, threads, 0, s>>>(a, t);
        mark();
    }
    check(cudaGetLastError(), "car tick launch");
}

// A step through the batch's CUDA graphs when they are on (and phase timing is off): the launches of one step
// with these pointers are captured once and replayed after.
void step_car_path(rg_batch* b, const rg::CarControls* controls, int stride, int ticks, cudaStream_t s,
                   const rg::EnvCommand* commands, int command_stride) {
    if (!b->use_graphs || b->timing) {
        launch_car_tick(b, controls, stride, ticks, s, commands, command_stride);
        return;
    }
    if (commands && !b->pads_live) b->drop_graphs();  // the step turns pads on, which captured launches see
    if (commands) b->pads_live = true;
    rg_batch::StepGraph* hit = nullptr;
    for (rg_batch::StepGraph& g : b->graphs)
        if (g.controls == controls && g.commands == commands && g.control_stride == stride &&
            g.command_stride == command_stride && g.ticks == ticks && g.version == b->graph_version)
            hit = &g;
    if (!hit) {
        if (!b->capture_stream) check(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking), "capture");
        if (b->graphs.size() >= 16) {
            auto lru = std::min_element(b->graphs.begin(), b->graphs.end(),
                                        [](const auto& x, const auto& y) { return x.last_use < y.last_use; });
            cudaGraphExecDestroy(lru->exec);
            b->graphs.erase(lru);
        }
        check(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal), "graph capture");
        launch_car_tick(b, controls, stride, ticks, b->capture_stream, commands, command_stride);
        cudaGraph_t g = nullptr;
        check(cudaStreamEndCapture(b->capture_stream, &g), "graph capture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        check(e, "graph instantiate");
        b->graphs.push_back({controls, commands, stride, command_stride, ticks, b->graph_version, 0, exec});
        hit = &b->graphs.back();
    }
    hit->last_use = ++b->graph_clock;
    check(cudaGraphLaunch(hit->exec, s), "graph launch");
}

// reset_to_kickoff for every arena (reference BatchSim::reset_to_kickoff, src/rocketgpu.cpp:2085-2132).
// Arenas [first, first + n) reset; their RNG draws use their index within the range (the whole batch: first = 0).
__global__ void reset_kickoff_kernel(CarTickArgs a, const uint8_t* teams, rg::CarControls* controls, uint64_t seed,
                                     int first, int n) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int e = first + j;
    const int car_base = e * a.max_cars;
    // the reference resets the arena's whole solver scratch (src/rocketgpu.cpp:2107-2111): broadphase history,
    // manifold list and retained car manifolds start over
    memset(&a.broadphase[e], 0, sizeof(rg::Broadphase));
    for (int k = 0; k < a.max_cars; ++k) {
        a.car_world[car_base + k].count = 0;
        a.ball_car[car_base + k].count = 0;
    }
    for (int k = 0; k < a.pair_slots; ++k) a.pairs[static_cast<size_t>(e) * a.pair_slots + k].count = 0;
    rg::reset_env_to_kickoff(j, seed, a.base.envs[e], a.base.balls[e], a.base.ball_world[e], a.cars + car_base,
                             a.wheels + car_base, a.car_cfgs + car_base, controls + car_base,
                             a.pads ? a.pads + static_cast<size_t>(e) * a.pad_layout.count : nullptr, a.pad_layout,
                             teams + car_base, a.base.env_car_count[e], a.max_cars, a.base.tc,
                             a.base.tc.settled_entry ? a.base.tc.settled_entry + car_base : nullptr);
}

// Episode resets for training loops (no counterpart in BatchSim; the reference's benchmark makes these decisions on
// the host, tools/bench_cpp.cpp:104-112): an arena whose ball was scored (every reset clears the scoreboard, so a
// non-zero score is a goal this episode) or that no car touched for `no_touch_ticks` ticks gets a fresh-episode reset
// for the next step. Touches are noticed through each car's latest_touch_tick changing since the previous check, so a
// value left over from an earlier episode never counts. `stagger` != 0 starts every arena's clock at a seeded age in
// [0, no_touch_ticks) so that resets spread over the ticks instead of coming together.
__device__ __forceinline__ uint64_t episode_hash(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
__global__ void episode_commands_kernel(const rg::EnvState* envs, const rg::CarState* cars, const int32_t* counts,
                                        int64_t* touch, uint64_t* seen, rg::EnvCommand* out, int n, int max_cars,
                                        int32_t no_touch_ticks, uint64_t seed, int init) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const rg::EnvState& env = envs[e];
    const int count = counts[e];
    const size_t base = static_cast<size_t>(e) * max_cars;
    rg::EnvCommand c;
    memset(&c, 0, sizeof(c));
    if (init) {
        for (int i = 0; i < max_cars; ++i) seen[base + i] = cars[base + i].latest_touch_tick;
        touch[e] = static_cast<int64_t>(env.tick) -
                   (seed ? static_cast<int64_t>(episode_hash(seed ^ static_cast<uint64_t>(e)) %
                                                static_cast<uint64_t>(no_touch_ticks))
                         : 0);
        out[e] = c;
        return;
    }
    int64_t last = touch[e];
    for (int i = 0; i < count; ++i) {
        const uint64_t v = cars[base + i].latest_touch_tick;
        if (v != seen[base + i]) {
            seen[base + i] = v;
            if (v != ~0ull && static_cast<int64_t>(v) > last) last = static_cast<int64_t>(v);
        }
    }
    const bool scored = (env.blue_score | env.orange_score) != 0;
    if (scored || static_cast<int64_t>(env.tick) - last >= no_touch_ticks) {
        c.reset_to_kickoff = c.reset_scoreboard = c.reset_tick_count = 1;
        last = 0;
    }
    touch[e] = last;
    out[e] = c;
}

void call_ok(int status, const char* what) {
    if (status != 0) throw std::runtime_error(std::string("kickoff_settled: ") + what + ": " + rg_last_error());
}

// Records the settled kickoff of the entries first[] name (car slots whose config and team are new): one arena per
// entry, `spawns` cars of that config and team, the game's countdown kickoff with the spots in order, stepped through
// the countdown (480 ticks, then tick by tick until every arena's countdown has ended); car k's state and wheel record
// become the entry's row for spot k, and the first recording's ball the settled ball (reference
// record_kickoff_settled, src/rocketgpu.cpp:1538-1612).
void record_kickoff_settled(rg_batch* b, const std::vector<size_t>& first, const std::vector<rg::CarConfig>& configs,
                            const std::vector<uint8_t>& teams, int spawns) {
    const size_t envs = first.size();
    rg_sim_config rc = b->cfg;
    rc.env_count = static_cast<int32_t>(envs);
    rc.max_cars_per_env = spawns;
    rc.kickoff_settled = 0;
    rg_arena_layout L{};
    L.vertices_uu = b->layout_vertices.data();
    L.vertex_count = static_cast<int64_t>(b->layout_vertices.size() / 3);
    L.indices = b->layout_indices.data();
    L.index_count = static_cast<int64_t>(b->layout_indices.size());
    L.rules = b->layout_has_rules ? &b->layout_rules : nullptr;
    L.boost_pads = b->layout_has_pads ? b->layout_pads.data() : nullptr;
    L.boost_pad_count = b->layout_has_pads ? static_cast<int32_t>(b->layout_pads.size()) : 0;
    rg_batch* created = nullptr;
    call_ok(rg_batch_create(&rc, &L, b->device, &created), "create");
    std::unique_ptr<rg_batch, void (*)(rg_batch*)> run(created, rg_batch_destroy);
    const size_t m = envs * static_cast<size_t>(spawns);
    std::vector<int32_t> counts(envs, spawns);
    std::vector<rg_car_config> run_cfgs(m);
    std::vector<uint8_t> run_teams(m);
    for (size_t i = 0; i < m; ++i) {
        memcpy(&run_cfgs[i], &configs[first[i / spawns]], sizeof(rg_car_config));
        run_teams[i] = teams[first[i / spawns]];
    }
    call_ok(rg_batch_set_env_car_count(run.get(), counts.data(), envs, nullptr), "car counts");
    call_ok(rg_batch_set_teams(run.get(), run_teams.data(), m, nullptr), "teams");
    call_ok(rg_batch_set_car_configs(run.get(), run_cfgs.data(), m, nullptr), "car configs");
    rg_env_command cmd{};
    cmd.reset_to_kickoff = 1;
    cmd.reset_scoreboard = 1;
    cmd.kickoff_seed_mode = 3;
    cmd.kickoff_countdown_ticks = rg::kKickoffCountdownGameTimers;
    std::vector<rg_env_command> cmds(envs, cmd);
    call_ok(rg_batch_apply_env_commands(run.get(), cmds.data(), envs, nullptr), "countdown kickoff");
    call_ok(rg_batch_step(run.get(), rg::kKickoffCountdownTicks, nullptr), "countdown");
    std::vector<rg_env_state> env_out(envs);
    for (int k = 0;; ++k) {
        call_ok(rg_batch_download_env_states(run.get(), env_out.data(), envs, nullptr), "env states");
        bool ended = true;
        for (const rg_env_state& e : env_out) ended = ended && e.countdown_phase == 0;
        if (ended) break;
        if (k == 16) throw std::runtime_error("kickoff_settled: the countdown did not end");
        call_ok(rg_batch_step(run.get(), 1, nullptr), "countdown");
    }
    std::vector<rg::CarState> cars(m);
    std::vector<rg::WheelRuntime> wheels(m);
    rg::BallState ball;
    check(cudaMemcpy(cars.data(), run->cars.ptr, m * sizeof(rg::CarState), cudaMemcpyDeviceToHost), "settled cars");
    check(cudaMemcpy(wheels.data(), run->wheels.ptr, m * sizeof(rg::WheelRuntime), cudaMemcpyDeviceToHost),
          "settled wheels");
    check(cudaMemcpy(&ball, run->balls.ptr, sizeof(ball), cudaMemcpyDeviceToHost), "settled ball");
    for (size_t i = 0; i < m; ++i) b->settle_rows_host.push_back(rg::KickoffSettledRow{cars[i], wheels[i]});
    if (b->settle_ball_host.empty()) b->settle_ball_host.push_back(ball);
}

// Before a kickoff reset of a batch with kickoff_settled: every car slot's (config, team) entry, recording the new
// ones, and the device copies the resets read (reference ensure_kickoff_settled, src/rocketgpu.cpp:1439-1500).
void ensure_kickoff_settled(rg_batch* b, cudaStream_t s) {
    if (!b->cfg.kickoff_settled || !b->settle_dirty) return;
    const size_t n = static_cast<size_t>(b->env_count) * static_cast<size_t>(b->max_cars);
    std::vector<rg::CarConfig> configs(n);
    std::vector<uint8_t> teams(n);
    if (n) {
        check(cudaMemcpyAsync(configs.data(), b->car_cfgs.ptr, n * sizeof(rg::CarConfig), cudaMemcpyDeviceToHost, s),
              "kickoff_settled configs");
        check(cudaMemcpyAsync(teams.data(), b->teams.ptr, n, cudaMemcpyDeviceToHost, s), "kickoff_settled teams");
        check(cudaStreamSynchronize(s), "kickoff_settled configs");
    }
    const int spawns = b->max_cars > 5 ? b->max_cars : 5;
    std::vector<size_t> first;
    std::vector<int32_t> entry(n);
    const size_t old_entries = b->settle_entries.size(), old_rows = b->settle_rows_host.size(),
                 old_balls = b->settle_ball_host.size();
    try {
        for (size_t i = 0; i < n; ++i) {
            size_t e = 0;
            while (e < b->settle_entries.size() &&
                   !(b->settle_entries[e].team == teams[i] &&
                     memcmp(&b->settle_entries[e].config, &configs[i], sizeof(rg::CarConfig)) == 0))
                ++e;
            if (e == b->settle_entries.size()) {
                b->settle_entries.push_back(rg_batch::SettleEntry{configs[i], teams[i]});
                first.push_back(i);
            }
            entry[i] = static_cast<int32_t>(e);
        }
        if (!first.empty()) record_kickoff_settled(b, first, configs, teams, spawns);
    } catch (...) {
        b->settle_entries.resize(old_entries);
        b->settle_rows_host.resize(old_rows);
        b->settle_ball_host.resize(old_balls);
        throw;
    }
    const size_t m = b->settle_rows_host.size();
    if (b->settle_rows.n != m) b->settle_rows.alloc(m);
    check(cudaMemcpy(b->settle_rows.ptr, b->settle_rows_host.data(), m * sizeof(rg::KickoffSettledRow),
                     cudaMemcpyHostToDevice),
          "kickoff_settled rows");
    if (b->settle_entry.n != n) b->settle_entry.alloc(n);
    if (n) check(cudaMemcpy(b->settle_entry.ptr, entry.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice),
                 "kickoff_settled entries");
    if (!b->settle_ball_host.empty()) {
        if (b->settle_ball.n != 1) b->settle_ball.alloc(1);
        check(cudaMemcpy(b->settle_ball.ptr, b->settle_ball_host.data(), sizeof(rg::BallState),
                         cudaMemcpyHostToDevice),
              "kickoff_settled ball");
    }
    b->tc.settled_rows = b->settle_rows.ptr;
    b->tc.settled_entry = b->settle_entry.ptr;
    b->tc.settled_ball = b->settle_ball_host.empty() ? nullptr : b->settle_ball.ptr;
    b->tc.settled_spawns = spawns;
    b->settle_dirty = false;
    b->drop_graphs();  // every captured launch holds the tick config
}

void launch_reset(rg_batch* b, uint64_t seed, cudaStream_t s) {
    if (b->tc.kickoff_seed != seed) b->drop_graphs();  // the respawn seed is part of every captured launch
    b->tc.kickoff_seed = seed;  // demolished cars draw their respawn spot from the last kickoff seed
    CarTickArgs a = car_tick_args(b, nullptr, 0);
    a.pads = b->pads.ptr;
    reset_kickoff_kernel<<<(b->env_count + 63) / 64, 64, 0, s>>>(a, b->teams.ptr, b->controls.ptr, seed, 0,
                                                                  b->env_count);
    check(cudaGetLastError(), "reset_kickoff_kernel launch");
}

void launch_tick(rg_batch* b, int ticks, cudaStream_t s) {
    TickArgs a;
    a.balls = b->balls.ptr;
    a.envs = b->envs.ptr;
    a.env_car_count = b->env_car_count.ptr;
    a.ball_world = b->ball_world.ptr;
    a.env_count = b->env_count;
    a.tc = b->tc;
    a.mesh = b->mesh;
    a.meshes = b->mesh_table.ptr;
    a.mesh_of = b->mesh_table.ptr ? b->mesh_of.ptr : nullptr;
    // One warp per block: an arena is one thread, so 16K arenas are only 512 warps; single-warp blocks spread them
    // over all 148 SMs (128-thread blocks left 20 SMs idle at 16K arenas).
    const int threads = b->launch_threads;
    const int blocks = (b->env_count + threads - 1) / threads;
    tick_kernel<<<blocks, threads, 0, s>>>(a, ticks);
    check(cudaGetLastError(), "tick_kernel launch");
}

// The step order (reference set_env_car_count rebuilds its step order, src/rocketgpu.cpp:2920-2932): arenas stably
// sorted by car count, largest first (their warps run longest, so they start first and the short ones fill in behind
// them), and the active car slots of those arenas in that order. The host copies stay in the batch
// until the caller's stream has finished the upload (set_env_car_count synchronises it).
void rebuild_step_order(rg_batch* b, cudaStream_t s) {
    b->drop_graphs();
    std::vector<int32_t>& order = b->host_arena_order;
    order.resize(b->env_count);
    for (int32_t e = 0; e < b->env_count; ++e) order[e] = e;
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return b->host_car_count[x] > b->host_car_count[y]; });
    std::vector<int32_t>& cars = b->host_active_cars;
    cars.clear();
    for (int32_t e : order)
        for (int32_t i = 0; i < b->host_car_count[e]; ++i) cars.push_back(e * b->max_cars + i);
    if (b->env_count)
        check(cudaMemcpyAsync(b->arena_order.ptr, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                              s),
              "step order");
    if (!cars.empty())
        check(cudaMemcpyAsync(b->active_cars.ptr, cars.data(), cars.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                              s),
              "active cars");
    b->active_car_count = static_cast<int32_t>(cars.size());
}

rg::TickConfig resolve_tick_config(const rg_sim_config& c) {
    rg::TickConfig t{};
    t.tick_dt = c.tick_dt;
    t.gravity_z = c.gravity_z;
    t.ball_radius = c.ball_radius;
    t.ball_mass = c.ball_mass;
    t.ball_drag = c.ball_drag;
    // BatchSim caches the per-tick drag factor (1 - drag)^dt once per config (reference CacheBallDamping,
    // src/rocketgpu.cpp:259-270).
    t.ball_drag_scale = c.ball_drag <= 0.0f ? 1.0f : rg::ucrt_powf(rg::fmax_(0.0f, 1.0f - c.ball_drag), c.tick_dt);
    t.ball_friction = c.ball_friction;
    t.ball_restitution = c.ball_restitution;
    t.ball_max_speed = c.ball_max_speed;
    t.ball_max_ang_speed = c.ball_max_ang_speed;
    t.goal_base_threshold_y = c.goal_base_threshold_y;
    t.frame_frac = 0.5f;
    t.enable_scoring = c.enable_scoring;
    t.enable_boost_pads = c.enable_boost_pads;
    t.enable_car_car = c.enable_car_car_collisions;
    t.enable_demos = c.enable_demos;
    t.enable_team_demos = 0;
    t.bump_force_scale = 1.0f;
    t.bump_cooldown_time = 0.25f;
    t.kickoff_seed = 0;
    t.max_cars = c.max_cars_per_env;
    t.pad_count = 34;
    t.car_mass = c.car_mass;
    t.car_max_speed = c.car_max_speed;
    t.car_max_ang_speed = c.car_max_ang_speed;
    rg::fill_car_constants(t);
    t.arena_friction = c.arena_friction;
    t.arena_restitution = c.arena_restitution;
    return t;
}

}  // namespace

extern "C" {

RG_API const char* rg_last_error(void) { return g_last_error.c_str(); }
RG_API const char* rg_version(void) { return "rocketgpu_b200 0.1 (sm_100a)"; }

RG_API void rg_sim_config_default(rg_sim_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->env_count = 1;
    c->max_cars_per_env = 6;
    c->tick_dt = 1.0f / 120.0f;
    c->enable_boost_pads = 1;
    c->enable_car_car_collisions = 1;
    c->enable_demos = 1;
    c->enable_scoring = 1;
    c->gravity_z = -650.0f;
    c->ball_radius = 91.24999f;
    c->ball_mass = 30.000002f;
    c->car_mass = 180.0f;
    c->ball_drag = 0.03f;
    c->ball_friction = 0.35f;
    c->ball_restitution = 0.60f;
    c->ball_max_speed = 6000.0f;
    c->ball_max_ang_speed = 6.0f;
    c->car_max_speed = 2300.0f;
    c->car_max_ang_speed = 5.5f;
    c->arena_friction = 0.30f;
    c->arena_restitution = 0.30f;
    c->goal_base_threshold_y = 5124.2373046875f;
    // the reference defaults to 1 (rocketgpu.h:831); this build has no kickoff settling and refuses 1
    c->kickoff_settled = 1;
}

RG_API void rg_default_ball_state(rg_ball_state* o) {
    std::memset(o, 0, sizeof(*o));
    o->hs_info.cur_target_speed = 2900.0f;
    o->ds_info.charge_level = 1;
    o->pos = {0.0f, 0.0f, 93.15f};
    o->rot = {1.0f, 0.0f, 0.0f, 0.0f};
    o->pos_bt = {0.0f, 0.0f, 93.15f * (1.0f / 50.0f)};
    o->basis_forward = {1.0f, 0.0f, 0.0f};
    o->basis_right = {0.0f, 1.0f, 0.0f};
    o->basis_up = {0.0f, 0.0f, 1.0f};
    o->inertia_basis_forward = {1.0f, 0.0f, 0.0f};
    o->inertia_basis_right = {0.0f, 1.0f, 0.0f};
    o->inertia_basis_up = {0.0f, 0.0f, 1.0f};
}

RG_API void rg_default_env_state(rg_env_state* o) {
    std::memset(o, 0, sizeof(*o));
    o->last_scored_team = -1;
    o->car_visit_order_mode = 3;
    o->car_visit_present_mask = 0xFF;
    o->car_visit_order_packed = 0x76543210u;
    o->frame_frac_prev = 0.5f;
}

RG_API void rg_default_car_state(rg_car_state* o) {
    std::memset(o, 0, sizeof(*o));
    o->pos = {0.0f, 0.0f, 17.0f};
    o->rot = {1.0f, 0.0f, 0.0f, 0.0f};
    o->boost = 100.0f;
    o->boost_amount = 1.0f;
    o->is_on_ground = 1;
    for (int i = 0; i < 4; ++i) o->wheels_with_contact[i] = 1;
    o->pos_bt = {0.0f, 0.0f, 17.0f * (1.0f / 50.0f)};
    o->tick_start_pos_bt = o->pos_bt;
    o->pad_frame_pos_bt = o->pos_bt;
    o->vel_touched_solve_stage = 1;
    o->basis_forward = {1.0f, 0.0f, 0.0f};
    o->basis_right = {0.0f, 1.0f, 0.0f};
    o->basis_up = {0.0f, 0.0f, 1.0f};
    o->previous_ball_contact_start = o->last_ball_contact_start = o->last_world_surface_contact = ~0ull;
    o->first_world_after_previous_ball = o->first_world_after_last_ball = ~0ull;
    o->last_flip_or_jump_start = o->last_directional_flip_start = ~0ull;
    o->flip_or_jump_last_tick = 1;
    o->dodge_timeout = -1.0f;
    o->latest_touch_tick = ~0ull;
    o->double_jump_ticks = 255;
    o->cal_pre_pitchlock_restart_time = -1.0f;
    o->tick_start_basis_forward = {1.0f, 0.0f, 0.0f};
    o->tick_start_basis_right = {0.0f, 1.0f, 0.0f};
    o->tick_start_basis_up = {0.0f, 0.0f, 1.0f};
}

RG_API void rg_default_car_config(rg_car_config* o) {
    std::memset(o, 0, sizeof(*o));
    o->hitbox_size = {118.00738f + 2.5f, 84.19941f + 2.5f, 36.159073f + 2.5f};
    o->hitbox_published = {118.00738f, 84.19941f, 36.159073f};
    o->hitbox_offset = {13.87566f, 0.0f, 20.754988f};
    o->front_wheels_offset = {51.25f, 25.90f, 20.754988f};
    o->back_wheels_offset = {-33.75f, 29.50f, 20.754988f};
    o->front_wheel_radius = 12.50f;
    o->back_wheel_radius = 15.00f;
    o->front_suspension_rest = 38.75499f;
    o->back_suspension_rest = 37.054989f;
    o->dodge_deadzone = 0.5f;
    o->three_wheels = 0;
    o->body = 147;
    const float steer[6] = {30.570510864257812f, 18.294261932373047f, 10.429570198059082f,
                            6.0558881759643555f, 4.874049186706543f, 1.9791786670684814f};
    std::memcpy(o->steer_angle_curve_deg, steer, sizeof(steer));
    o->powerslide_steer_angle_curve_deg[0] = 22.478458404541016f;
    o->powerslide_steer_angle_curve_deg[1] = 7.224311351776123f;
    o->spawn_z = 36.02f;
}

// ---- the layout's rules and pads (reference ArenaLayout handling, src/rocketgpu.cpp:792-881, 1502-1536) ----------
namespace {
constexpr float kLayoutMaxCoord = 11500.0f;   // reference kArenaLayoutMaxCoord
constexpr float kLayoutMaxYaw = 25.132741f;   // reference kArenaLayoutMaxYaw (8 pi)
constexpr int kMaxLayoutPads = 48;            // reference kMaxBoostPads
void check_position(const rg_vec3& v, const char* what) {
    const bool ok = std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z) && std::fabs(v.x) <= kLayoutMaxCoord &&
                    std::fabs(v.y) <= kLayoutMaxCoord && std::fabs(v.z) <= kLayoutMaxCoord;
    if (!ok)
        throw std::invalid_argument(std::string("ArenaLayout: ") + what +
                                    " must be finite and within kArenaLayoutMaxCoord (11500 uu) of the origin on every axis");
}
bool same_vec(const rg_vec3& a, const rg_vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
// reference ValidateArenaLayout (rules and pads part) and SameArenaRules
void validate_rules(const rg_arena_rules& r) {
    for (int t = 0; t < 2; ++t) {
        const rg_arena_goal& g = r.goals[t];
        check_position(g.point, "a goal point");
        if (!(std::isfinite(g.normal.x) && std::isfinite(g.normal.y) && std::isfinite(g.normal.z)))
            throw std::invalid_argument("ArenaLayout: a goal normal must be finite");
        for (const float x : {g.min.x, g.min.y, g.min.z, g.max.x, g.max.y, g.max.z})
            if (std::isnan(x)) throw std::invalid_argument("ArenaLayout: a goal's min and max must not be NaN");
        for (const rg_arena_spawn& sp : r.kickoff_spawns[t]) {
            check_position(sp.pos, "a kickoff spawn position");
            if (!(std::fabs(sp.yaw) <= kLayoutMaxYaw))
                throw std::invalid_argument("ArenaLayout: a kickoff spawn yaw must be within 8 pi of zero");
        }
        for (const rg_arena_spawn& sp : r.respawn_spawns[t]) {
            check_position(sp.pos, "a respawn spawn position");
            if (!(std::fabs(sp.yaw) <= kLayoutMaxYaw))
                throw std::invalid_argument("ArenaLayout: a respawn spawn yaw must be within 8 pi of zero");
        }
    }
    check_position(r.ball_spawn, "the ball spawn");
}
bool same_rules(const rg_arena_rules& a, const rg_arena_rules& b) {
    bool same = same_vec(a.ball_spawn, b.ball_spawn);
    for (int t = 0; t < 2; ++t) {
        same = same && same_vec(a.goals[t].point, b.goals[t].point) && same_vec(a.goals[t].normal, b.goals[t].normal) &&
               same_vec(a.goals[t].min, b.goals[t].min) && same_vec(a.goals[t].max, b.goals[t].max);
        for (int k = 0; k < 5; ++k)
            same = same && same_vec(a.kickoff_spawns[t][k].pos, b.kickoff_spawns[t][k].pos) &&
                   a.kickoff_spawns[t][k].yaw == b.kickoff_spawns[t][k].yaw;
        for (int k = 0; k < 4; ++k)
            same = same && same_vec(a.respawn_spawns[t][k].pos, b.respawn_spawns[t][k].pos) &&
                   a.respawn_spawns[t][k].yaw == b.respawn_spawns[t][k].yaw;
    }
    return same;
}
// reference MakeArenaRules: goal normals normalized
rg::ArenaRules make_rules(const rg_arena_rules& in) {
    rg::ArenaRules r{};
    auto v3 = [](const rg_vec3& v) { return rg::V3{v.x, v.y, v.z}; };
    for (int t = 0; t < 2; ++t) {
        for (int k = 0; k < 5; ++k) {
            r.kickoff_pos[t][k] = v3(in.kickoff_spawns[t][k].pos);
            r.kickoff_yaw[t][k] = in.kickoff_spawns[t][k].yaw;
        }
        for (int k = 0; k < 4; ++k) {
            r.respawn_pos[t][k] = v3(in.respawn_spawns[t][k].pos);
            r.respawn_yaw[t][k] = in.respawn_spawns[t][k].yaw;
        }
        const rg_arena_goal& g = in.goals[t];
        const float len = std::sqrt((g.normal.x * g.normal.x + g.normal.y * g.normal.y) + g.normal.z * g.normal.z);
        if (!(len > 0.0f) || !std::isfinite(len)) throw std::invalid_argument("ArenaGoal normal must be nonzero");
        r.goal_point[t] = v3(g.point);
        r.goal_normal[t] = rg::V3{g.normal.x / len, g.normal.y / len, g.normal.z / len};
        r.goal_min[t] = v3(g.min);
        r.goal_max[t] = v3(g.max);
    }
    r.ball_spawn = v3(in.ball_spawn);
    return r;
}
}  // namespace

RG_API void rg_default_arena_rules(rg_arena_rules* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    rg_sim_config c;
    rg_sim_config_default(&c);
    const float thr = c.goal_base_threshold_y;
    o->goals[0] = rg_arena_goal{{0.0f, -thr, 0.0f}, {0.0f, -1.0f, 0.0f}, {-1.0e30f, -1.0e30f, -1.0e30f},
                                {1.0e30f, 1.0e30f, 1.0e30f}};
    o->goals[1] = rg_arena_goal{{0.0f, thr, 0.0f}, {0.0f, 1.0f, 0.0f}, {-1.0e30f, -1.0e30f, -1.0e30f},
                                {1.0e30f, 1.0e30f, 1.0e30f}};
    for (int k = 0; k < 5; ++k) {
        const rg::SpawnPos sp = rg::soccar_kickoff_spawn(k);
        o->kickoff_spawns[0][k] = rg_arena_spawn{{sp.x, sp.y, 0.0f}, sp.yaw};
        o->kickoff_spawns[1][k] = rg_arena_spawn{{-sp.x, -sp.y, 0.0f}, sp.yaw + rg::kPiF};
    }
    for (int k = 0; k < 4; ++k) {
        const rg::SpawnPos sp = rg::soccar_respawn_spawn(k);
        o->respawn_spawns[0][k] = rg_arena_spawn{{sp.x, sp.y, 0.0f}, sp.yaw};
        o->respawn_spawns[1][k] = rg_arena_spawn{{sp.x, -sp.y, 0.0f}, sp.yaw + rg::kPiF};
    }
    o->ball_spawn = rg_vec3{0.0f, 0.0f, 92.75f};
}

// The game's hitbox presets (reference OctaneConfig .. MercConfig, src/rocketgpu.cpp:417-490): hitbox (published size
// + 2.5 uu per axis), offsets, wheel radii and suspension rest lengths, steering curves, spawn height, body id. The
// numbers are the game's car data, the same in every implementation.
namespace {
struct PresetData {
    float hitbox[3], hitbox_offset[3];
    float front_radius, front_rest, front_offset[3];
    float back_radius, back_rest, back_offset[3];
    float steer[6], powerslide[2];
    bool own_steer;
    float spawn_z;
    uint16_t body;
};
constexpr PresetData kPresets[] = {
    // Dominus
    {{127.92678f, 83.27995f, 31.3f}, {9.0f, 0.0f, 15.75f}, 12.00f, 33.95f, {50.30f, 31.10f, 15.75f}, 13.50f, 33.85f,
     {-34.75f, 33.00f, 15.75f},
     {29.923809051513672f, 18.018766403198242f, 10.329229354858398f, 6.019903182983398f, 4.85035514831543f,
      1.9751166105270386f},
     {22.08690071105957f, 7.173928260803223f}, true, 36.01f, 132},
    // Plank
    {{128.81978f, 84.670364f, 29.394402f}, {9.008572f, 0.0f, 12.0942f}, 12.50f, 31.9242f, {49.97f, 27.799904f, 12.0942f},
     17.00f, 27.9242f, {-35.43f, 20.280005f, 12.0942f},
     {30.342710494995117f, 18.1981258392334f, 10.394840240478516f, 6.043498516082764f, 4.865903377532959f,
      1.9777874946594238f},
     {22.341325759887695f, 7.206938743591309f}, true, 38.84f, 150},
    // Breakout
    {{131.49236f, 80.521f, 30.3f}, {12.5f, 0.0f, 11.75f}, 13.50f, 29.7f, {51.50f, 26.67f, 11.75f}, 15.00f, 29.66f,
     {-35.75f, 35.00f, 11.75f},
     {30.55976104736328f, 18.289745330810547f, 10.42794418334961f, 6.055309772491455f, 4.873669147491455f,
      1.9791138172149658f},
     {22.472003936767578f, 7.2235002517700195f}, true, 36.00f, 64},
    // Hybrid
    {{127.01919f, 82.18787f, 34.159073f}, {13.87566f, 0.0f, 20.754988f}, 12.50f, 38.75499f, {51.25f, 25.90f, 20.754988f},
     15.00f, 37.054989f, {-34.00f, 29.50f, 20.754988f},
     {30.580455780029297f, 18.29843521118164f, 10.431071281433105f, 6.056422233581543f, 4.874399185180664f,
      1.9792383909225464f},
     {22.484424591064453f, 7.225060939788818f}, true, 37.53f, 56},
    // Merc (keeps the default steering curves)
    {{120.72023f, 76.71031f, 41.659073f}, {11.37566f, 0.0f, 21.504988f}, 15.00f, 39.50499f, {51.25f, 25.90f, 21.504988f},
     15.00f, 39.104988f, {-33.75f, 29.50f, 21.504988f}, {}, {}, false, 35.05f, 219},
};
}  // namespace

RG_API int rg_car_preset(int32_t preset, rg_car_config* out) {
    return guard([&] {
        if (!out) throw std::invalid_argument("null argument");
        if (preset < 0 || preset > 5) throw std::out_of_range("preset must be 0..5 (Octane .. Merc)");
        rg_default_car_config(out);
        if (preset == 0) return;
        const PresetData& d = kPresets[preset - 1];
        out->hitbox_published = {d.hitbox[0], d.hitbox[1], d.hitbox[2]};
        out->hitbox_size = {d.hitbox[0] + 2.5f, d.hitbox[1] + 2.5f, d.hitbox[2] + 2.5f};
        out->hitbox_offset = {d.hitbox_offset[0], d.hitbox_offset[1], d.hitbox_offset[2]};
        out->front_wheels_offset = {d.front_offset[0], d.front_offset[1], d.front_offset[2]};
        out->back_wheels_offset = {d.back_offset[0], d.back_offset[1], d.back_offset[2]};
        out->front_wheel_radius = d.front_radius;
        out->back_wheel_radius = d.back_radius;
        out->front_suspension_rest = d.front_rest;
        out->back_suspension_rest = d.back_rest;
        out->three_wheels = 0;
        if (d.own_steer) {
            std::memcpy(out->steer_angle_curve_deg, d.steer, sizeof(d.steer));
            std::memcpy(out->powerslide_steer_angle_curve_deg, d.powerslide, sizeof(d.powerslide));
        }
        out->spawn_z = d.spawn_z;
        out->body = d.body;
    });
}

RG_API int rg_batch_create(const rg_sim_config* cfg, const rg_arena_layout* layout, int device, rg_batch** out) {
    return guard([&] {
        if (!cfg || !layout || !out) throw std::invalid_argument("null argument");
        if (layout->boost_pads) {
            if (layout->boost_pad_count < 0 || layout->boost_pad_count > kMaxLayoutPads)
                throw std::invalid_argument("ArenaLayout::boost_pads holds at most kMaxBoostPads pads");
            for (int p = 0; p < layout->boost_pad_count; ++p) check_position(layout->boost_pads[p].pos, "a boost pad position");
        } else if (layout->boost_pad_count != 0) {
            throw std::invalid_argument("boost_pad_count without boost_pads");
        }
        if (layout->rules) validate_rules(*layout->rules);
        if (cfg->env_count <= 0) throw std::invalid_argument("env_count must be positive");
        // The car-car pair rows are sized for the 15 pairs of six cars (rg_car_car.cuh kMaxPairRows); 7- and 8-car
        // arenas would need more, so they are refused rather than run with rows dropped.
        if (cfg->max_cars_per_env < 0 || cfg->max_cars_per_env > 6)
            throw std::invalid_argument("max_cars_per_env must be in [0, 6]");
        if (cfg->kickoff_settled > 1) throw std::invalid_argument("kickoff_settled must be 0 or 1");
        if (!(cfg->tick_dt > 0.0f)) throw std::invalid_argument("tick_dt must be positive");
        std::unique_ptr<rg_batch> b(new rg_batch);
        b->device = device;
        b->cfg = *cfg;
        b->env_count = cfg->env_count;
        b->max_cars = cfg->max_cars_per_env;
        b->tc = resolve_tick_config(*cfg);
        b->mesh_host = rg::build_mesh_host(layout->vertices_uu, layout->vertex_count, layout->indices,
                                           layout->index_count);
        DeviceGuard dg(device);
        b->mesh = rg::upload_mesh(b->mesh_host);
        b->balls.alloc(b->env_count);
        b->envs.alloc(b->env_count);
        b->env_car_count.alloc(b->env_count);
        b->ball_world.alloc(b->env_count);
        check(cudaMemset(b->ball_world.ptr, 0, b->env_count * sizeof(rg::BallWorldScratch)), "clear ball manifolds");
        std::vector<rg_ball_state> balls(b->env_count);
        std::vector<rg_env_state> envs(b->env_count);
        for (auto& x : balls) rg_default_ball_state(&x);
        for (auto& x : envs) rg_default_env_state(&x);
        b->host_car_count.assign(b->env_count, 0);
        // cars, wheel records, configs, controls and pads at the reference's initial values
        // (src/rocketgpu.cpp:1085-1130; the layout's pads are the 34 soccar pads, rocketgpu.cpp:2754-2759)
        const size_t cap = static_cast<size_t>(b->env_count) * static_cast<size_t>(b->max_cars);
        {
            static const float kPads[34][3] = {
                {0, -4240, 70},    {-1792, -4184, 70}, {1792, -4184, 70},  {-940, -3308, 70},  {940, -3308, 70},
                {0, -2816, 70},    {-3584, -2484, 70}, {3584, -2484, 70},  {-1788, -2302, 70}, {1788, -2302, 70},
                {-2048, -1036, 70}, {0, -1024, 70},    {2048, -1036, 70},  {-1024, 0, 70},     {1024, 0, 70},
                {-2048, 1036, 70}, {0, 1024, 70},      {2048, 1036, 70},   {-1788, 2302, 70},  {1788, 2302, 70},
                {-3584, 2484, 70}, {3584, 2484, 70},   {0, 2816, 70},      {-940, 3308, 70},   {940, 3308, 70},
                {-1792, 4184, 70}, {1792, 4184, 70},   {0, 4240, 70},      {-3584, 0, 73},     {3584, 0, 73},
                {-3072, 4096, 73}, {3072, 4096, 73},   {-3072, -4096, 73}, {3072, -4096, 73}};
            b->pad_layout.count = 34;
            for (int p = 0; p < 34; ++p) {
                b->pad_layout.pos[p] = rg::V3{kPads[p][0], kPads[p][1], kPads[p][2]};
                b->pad_layout.is_big[p] = p >= 28 ? 1 : 0;
            }
            if (layout->boost_pads) {  // the layout's own pads
                b->pad_layout.count = layout->boost_pad_count;
                for (int p = 0; p < layout->boost_pad_count; ++p) {
                    const rg_boost_pad_config& pc = layout->boost_pads[p];
                    b->pad_layout.pos[p] = rg::V3{pc.pos.x, pc.pos.y, pc.pos.z};
                    b->pad_layout.is_big[p] = pc.is_big;
                }
            }
            b->tc.pad_count = b->pad_layout.count;
        }
        if (layout->rules) {
            rg_arena_rules official;
            rg_default_arena_rules(&official);
            if (!same_rules(*layout->rules, official)) {
                const rg::ArenaRules r = make_rules(*layout->rules);
                b->rules.alloc(1);
                check(cudaMemcpy(b->rules.ptr, &r, sizeof(r), cudaMemcpyHostToDevice), "arena rules");
                b->tc.rules = b->rules.ptr;
            }
        }
        b->cars.alloc(cap);
        b->wheels.alloc(cap);
        b->car_cfgs.alloc(cap);
        b->controls.alloc(cap);
        b->pads.alloc(static_cast<size_t>(b->env_count) * static_cast<size_t>(b->pad_layout.count));
        b->teams.alloc(cap);
        if (cap) check(cudaMemset(b->teams.ptr, 0, cap), "teams");
        b->broadphase.alloc(b->env_count);
        check(cudaMemset(b->broadphase.ptr, 0, b->env_count * sizeof(rg::Broadphase)), "broadphase");
        b->car_world.alloc(cap);
        if (cap) check(cudaMemset(b->car_world.ptr, 0, cap * sizeof(rg::CarWorldScratch)), "car manifolds");
        b->ball_car.alloc(cap);
        if (cap) check(cudaMemset(b->ball_car.ptr, 0, cap * sizeof(rg::BallCarScratch)), "car-ball manifolds");
        b->pair_slots = b->max_cars * (b->max_cars - 1) / 2;
        b->car_pairs.alloc(static_cast<size_t>(b->env_count) * b->pair_slots);
        if (b->pair_slots)
            check(cudaMemset(b->car_pairs.ptr, 0, static_cast<size_t>(b->env_count) * b->pair_slots *
                                                      sizeof(rg::CarCarManifold)),
                  "car-car manifolds");
        b->car_records.alloc(cap);
        b->car_stages.alloc(cap);
        b->arena_snaps.alloc(b->env_count);
        b->command_scratch.alloc(b->env_count);
        b->device_status.alloc(1);
        check(cudaMemset(b->device_status.ptr, 0, sizeof(uint32_t)), "device status");
        b->episode_touch.alloc(b->env_count);
        check(cudaMemset(b->episode_touch.ptr, 0, b->env_count * sizeof(int64_t)), "episode state");
        b->episode_seen.alloc(cap);
        if (cap) check(cudaMemset(b->episode_seen.ptr, 0xff, cap * sizeof(uint64_t)), "episode state");
        b->arena_order.alloc(b->env_count);
        b->active_cars.alloc(cap);
        rebuild_step_order(b.get(), nullptr);
        if (cap) {
            rg_car_state c0;
            rg_default_car_state(&c0);
            rg_car_config k0;
            rg_default_car_config(&k0);
            std::vector<rg_car_state> cars(cap, c0);
            std::vector<rg_car_config> cfgs(cap, k0);
            std::vector<rg::WheelRuntime> wheels(cap, rg::wheel_runtime_default());
            check(cudaMemcpy(b->cars.ptr, cars.data(), cap * sizeof(rg_car_state), cudaMemcpyHostToDevice), "cars");
            check(cudaMemcpy(b->car_cfgs.ptr, cfgs.data(), cap * sizeof(rg_car_config), cudaMemcpyHostToDevice),
                  "car configs");
            check(cudaMemcpy(b->wheels.ptr, wheels.data(), cap * sizeof(rg::WheelRuntime), cudaMemcpyHostToDevice),
                  "wheels");
            check(cudaMemset(b->controls.ptr, 0, cap * sizeof(rg::CarControls)), "controls");
        }
        {
            const size_t per = static_cast<size_t>(b->pad_layout.count);
            std::vector<rg::PadState> pads(static_cast<size_t>(b->env_count) * per);
            for (size_t i = 0; i < pads.size(); ++i) {
                pads[i] = rg::PadState{0.0f, 1, b->pad_layout.is_big[i % per], 32768, 0, 0};
            }
            check(cudaMemcpy(b->pads.ptr, pads.data(), pads.size() * sizeof(rg::PadState), cudaMemcpyHostToDevice),
                  "pads");
        }
        check(cudaMemcpy(b->balls.ptr, balls.data(), balls.size() * sizeof(rg_ball_state), cudaMemcpyHostToDevice),
              "upload balls");
        check(cudaMemcpy(b->envs.ptr, envs.data(), envs.size() * sizeof(rg_env_state), cudaMemcpyHostToDevice),
              "upload envs");
        check(cudaMemcpy(b->env_car_count.ptr, b->host_car_count.data(), b->env_count * sizeof(int32_t),
                         cudaMemcpyHostToDevice),
              "upload car counts");
        if (cfg->kickoff_settled) {
            // kept for the batches that record the settled kickoffs
            b->layout_vertices.assign(layout->vertices_uu, layout->vertices_uu + 3 * layout->vertex_count);
            b->layout_indices.assign(layout->indices, layout->indices + layout->index_count);
            b->layout_has_rules = layout->rules != nullptr;
            if (layout->rules) b->layout_rules = *layout->rules;
            b->layout_has_pads = layout->boost_pads != nullptr;
            if (layout->boost_pads)
                b->layout_pads.assign(layout->boost_pads, layout->boost_pads + layout->boost_pad_count);
        }
        // BatchSim's constructor ends with reset_to_kickoff(0) (src/rocketgpu.cpp:1281), which records the settled
        // kickoff of the default car first when settling is on
        ensure_kickoff_settled(b.get(), nullptr);
        launch_reset(b.get(), 0, nullptr);
        check(cudaDeviceSynchronize(), "initial kickoff reset");
        *out = b.release();
    });
}

RG_API void rg_batch_destroy(rg_batch* b) {
    if (!b) return;
    DeviceGuard dg(b->device);
    rg::free_mesh(b->mesh);
    for (rg::MeshDevice& m : b->extra_meshes) rg::free_mesh(m);
    delete b;
}

RG_API int64_t rg_batch_env_count(const rg_batch* b) { return b ? b->env_count : 0; }
RG_API int64_t rg_batch_car_capacity(const rg_batch* b) {
    return b ? static_cast<int64_t>(b->env_count) * b->max_cars : 0;
}

RG_API int rg_batch_set_env_car_count(rg_batch* b, const int32_t* counts, size_t count, void* stream) {
    return guard([&] {
        if (!b || (!counts && count)) throw std::invalid_argument("null argument");
        if (count > static_cast<size_t>(b->env_count))
            throw std::out_of_range("set_env_car_count count exceeds env_count");
        for (size_t i = 0; i < count; ++i) {
            if (counts[i] < 0 || counts[i] > b->max_cars)
                throw std::out_of_range("env car count out of range [0, max_cars_per_env]");
        }
        DeviceGuard dg(b->device);
        std::memcpy(b->host_car_count.data(), counts, count * sizeof(int32_t));
        b->settle_dirty = true;
        for (size_t i = 0; i < count; ++i) b->pads_live = b->pads_live || counts[i] > 0;
        rebuild_step_order(b, static_cast<cudaStream_t>(stream));
        check(cudaMemcpyAsync(b->env_car_count.ptr, counts, count * sizeof(int32_t), cudaMemcpyHostToDevice,
                              static_cast<cudaStream_t>(stream)),
              "set_env_car_count");
        check(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "set_env_car_count sync");
    });
}

RG_API int rg_batch_upload_ball_states(rg_batch* b, const rg_ball_state* host, size_t count, void* stream) {
    return guard([&] {
        if (!b || (!host && count)) throw std::invalid_argument("null argument");
        if (count > static_cast<size_t>(b->env_count))
            throw std::out_of_range("upload_ball_states count exceeds env_count");
        if (!count) return;
        DeviceGuard dg(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        check(cudaMemcpyAsync(b->balls.ptr, host, count * sizeof(rg_ball_state), cudaMemcpyHostToDevice, s),
              "upload_ball_states");
        canonicalize_balls_kernel<<<(static_cast<int>(count) + 127) / 128, 128, 0, s>>>(b->balls.ptr,
                                                                                        static_cast<int>(count));
        check(cudaGetLastError(), "canonicalize launch");
        check(cudaStreamSynchronize(s), "upload_ball_states sync");
    });
}

RG_API int rg_batch_download_ball_states(rg_batch* b, rg_ball_state* host, size_t count, void* stream) {
    return guard([&] {
        if (!b || (!host && count)) throw std::invalid_argument("null argument");
        if (count > static_cast<size_t>(b->env_count))
            throw std::out_of_range("download_ball_states count exceeds env_count");
        DeviceGuard dg(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        check(cudaMemcpyAsync(host, b->balls.ptr, count * sizeof(rg_ball_state), cudaMemcpyDeviceToHost, s),
              "download_ball_states");
        check(cudaStreamSynchronize(s), "download_ball_states sync");
    });
}

RG_API int rg_batch_upload_env_states(rg_batch* b, const rg_env_state* host, size_t count, void* stream) {
    return guard([&] {
        if (!b || (!host && count)) throw std::invalid_argument("null argument");
        if (count > static_cast<size_t>(b->env_count))
            throw std::out_of_range("upload_env_states count exceeds env_count");
        for (size_t i = 0; i < count; ++i) {
            const uint8_t m = host[i].car_visit_order_mode;
            if (m > 3) throw std::invalid_argument("upload_env_states: car_visit_order_mode must be 0, 1, 2 or 3");
        }
        DeviceGuard dg(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        check(cudaMemcpyAsync(b->envs.ptr, host, count * sizeof(rg_env_state), cudaMemcpyHostToDevice, s),
              "upload_env_states");
        check(cudaStreamSynchronize(s), "upload_env_states sync");
    });
}

RG_API int rg_batch_download_env_states(rg_batch* b, rg_env_state* host, size_t count, void* stream) {
    return guard([&] {
        if (!b || (!host && count)) throw std::invalid_argument("null argument");
        if (count > static_cast<size_t>(b->env_count))
            throw std::out_of_range("download_env_states count exceeds env_count");
        DeviceGuard dg(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        check(cudaMemcpyAsync(host, b->envs.ptr, count * sizeof(rg_env_state), cudaMemcpyDeviceToHost, s),
              "download_env_states");
        check(cudaStreamSynchronize(s), "download_env_states sync");
    });
}

}  // extern "C"

namespace {
template <class T, class D>
void upload_array(rg_batch* b, DeviceArray<D>& dst, const T* host, size_t count, size_t cap, const char* what,
                  void* stream) {
    static_assert(sizeof(T) == sizeof(D), "layout");
    if (!b || (!host && count)) throw std::invalid_argument("null argument");
    if (count > cap) throw std::out_of_range(std::string(what) + " count exceeds capacity");
    if (!count) return;
    DeviceGuard dg(b->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    check(cudaMemcpyAsync(dst.ptr, host, count * sizeof(T), cudaMemcpyHostToDevice, s), what);
    check(cudaStreamSynchronize(s), what);
}
template <class T, class D>
void download_array(rg_batch* b, const DeviceArray<D>& src, T* host, size_t count, size_t cap, const char* what,
                    void* stream) {
    static_assert(sizeof(T) == sizeof(D), "layout");
    if (!b || (!host && count)) throw std::invalid_argument("null argument");
    if (count > cap) throw std::out_of_range(std::string(what) + " count exceeds capacity");
    if (!count) return;
    DeviceGuard dg(b->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    check(cudaMemcpyAsync(host, src.ptr, count * sizeof(T), cudaMemcpyDeviceToHost, s), what);
    check(cudaStreamSynchronize(s), what);
}
}  // namespace

extern "C" {

RG_API int rg_batch_upload_car_states(rg_batch* b, const rg_car_state* host, size_t count, void* stream) {
    return guard([&] {
        upload_array(b, b->cars, host, count, static_cast<size_t>(rg_batch_car_capacity(b)), "upload_car_states",
                     stream);
        if (!count) return;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        canonicalize_cars_kernel<<<(static_cast<int>(count) + 127) / 128, 128, 0, s>>>(b->cars.ptr,
                                                                                       static_cast<int>(count));
        check(cudaGetLastError(), "canonicalize cars launch");
        check(cudaStreamSynchronize(s), "upload_car_states sync");
    });
}
RG_API int rg_batch_download_car_states(rg_batch* b, rg_car_state* host, size_t count, void* stream) {
    return guard([&] {
        download_array(b, b->cars, host, count, static_cast<size_t>(rg_batch_car_capacity(b)),
                       "download_car_states", stream);
    });
}
RG_API int64_t rg_batch_pad_capacity(const rg_batch* b) {
    return b ? static_cast<int64_t>(b->env_count) * b->pad_layout.count : 0;
}
RG_API int rg_batch_upload_pad_states(rg_batch* b, const rg_boost_pad_state* host, size_t count, void* stream) {
    return guard([&] {
        upload_array(b, b->pads, host, count, static_cast<size_t>(rg_batch_pad_capacity(b)), "upload_pad_states",
                     stream);
        if (count && !b->pads_live) {
            b->pads_live = true;
            b->drop_graphs();
        }
    });
}
RG_API int rg_batch_download_pad_states(rg_batch* b, rg_boost_pad_state* host, size_t count, void* stream) {
    return guard([&] {
        download_array(b, b->pads, host, count, static_cast<size_t>(rg_batch_pad_capacity(b)), "download_pad_states",
                       stream);
    });
}
RG_API int rg_batch_set_car_configs(rg_batch* b, const rg_car_config* host, size_t count, void* stream) {
    return guard([&] {
        for (size_t i = 0; host && i < count; ++i)
            if (host[i].three_wheels) throw std::invalid_argument("three-wheel car configs are not supported");
        upload_array(b, b->car_cfgs, host, count, static_cast<size_t>(rg_batch_car_capacity(b)), "set_car_configs",
                     stream);
        b->settle_dirty = true;
    });
}
RG_API int rg_batch_set_teams(rg_batch* b, const uint8_t* host, size_t count, void* stream) {
    return guard([&] {
        for (size_t i = 0; host && i < count; ++i)
            if (host[i] > 1) throw std::invalid_argument("team must be 0 (blue) or 1 (orange)");
        upload_array(b, b->teams, host, count, static_cast<size_t>(rg_batch_car_capacity(b)), "set_teams", stream);
        b->settle_dirty = true;
    });
}
RG_API int rg_batch_reset_to_kickoff(rg_batch* b, uint64_t seed, void* stream) {
    return guard([&] {
        if (!b) throw std::invalid_argument("null argument");
        DeviceGuard dg(b->device);
        ensure_kickoff_settled(b, static_cast<cudaStream_t>(stream));
        launch_reset(b, seed, static_cast<cudaStream_t>(stream));
    });
}
RG_API int rg_batch_upload_controls(rg_batch* b, const rg_car_controls* host, size_t count, void* stream) {
    return guard([&] {
        upload_array(b, b->controls, host, count, static_cast<size_t>(rg_batch_car_capacity(b)), "upload_controls",
                     stream);
    });
}

RG_API int rg_batch_step(rg_batch* b, int32_t ticks, void* stream) {
    return guard([&] {
        if (!b) throw std::invalid_argument("null argument");
        if (ticks < 0) throw std::invalid_argument("ticks must be >= 0");
        if (ticks == 0) return;
        DeviceGuard dg(b->device);
        if (b->pads_live) {
            step_car_path(b, b->controls.ptr, 0, ticks, static_cast<cudaStream_t>(stream), nullptr, 0);
        } else {
            launch_tick(b, ticks, static_cast<cudaStream_t>(stream));
        }
    });
}

RG_API int rg_batch_step_with_device_controls(rg_batch* b, const rg_car_controls* device_controls, int32_t ticks,
                                              int32_t control_stride, void* stream) {
    return guard([&] {
        if (!b) throw std::invalid_argument("null argument");
        if (ticks <= 0) return;
        if (!device_controls) throw std::invalid_argument("device_controls_by_tick must not be null");
        if (control_stride != 0 && static_cast<int64_t>(control_stride) < rg_batch_car_capacity(b))
            throw std::invalid_argument("control_stride must be zero or at least the total car capacity");
        if (control_stride < 0) throw std::invalid_argument("control_stride must be zero or at least the car capacity");
        DeviceGuard dg(b->device);
        step_car_path(b, reinterpret_cast<const rg::CarControls*>(device_controls), control_stride, ticks,
                      static_cast<cudaStream_t>(stream), nullptr, 0);
    });
}

RG_API int rg_batch_apply_env_commands(rg_batch* b, const rg_env_command* host, size_t count, void* stream) {
    return guard([&] {
        if (!b || !host) throw std::invalid_argument("host_commands must not be null");
        if (count > static_cast<size_t>(b->env_count))
            throw std::out_of_range("apply_env_commands count exceeds env_count");
        size_t active = 0;
        for (size_t i = 0; i < count; ++i) {
            const rg_env_command& c = host[i];
            active += (c.reset_to_kickoff | c.reset_scoreboard | c.reset_tick_count | c.new_round_bodies) != 0;
        }
        if (active == 0) return;
        DeviceGuard dg(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        ensure_kickoff_settled(b, s);
        check(cudaMemcpyAsync(b->command_scratch.ptr, host, count * sizeof(rg_env_command), cudaMemcpyHostToDevice, s),
              "apply_env_commands upload");
        CarTickArgs a = car_tick_args(b, nullptr, 0);
        a.pads = b->pads.ptr;
        apply_commands_kernel<<<(static_cast<int>(count) + 63) / 64, 64, 0, s>>>(
            a, b->command_scratch.ptr, static_cast<int>(count), b->controls.ptr, b->device_status.ptr);
        check(cudaGetLastError(), "apply_commands_kernel launch");
        // the host array is borrowed for the call only
        check(cudaStreamSynchronize(s), "apply_env_commands sync");
    });
}

RG_API int rg_batch_apply_env_commands_device(rg_batch* b, const rg_env_command* device_commands, size_t count,
                                              void* stream) {
    return guard([&] {
        if (!b || !device_commands) throw std::invalid_argument("device_commands must not be null");
        if (count > static_cast<size_t>(b->env_count))
            throw std::out_of_range("apply_env_commands_device count exceeds env_count");
        if (count == 0) return;
        DeviceGuard dg(b->device);
        ensure_kickoff_settled(b, static_cast<cudaStream_t>(stream));
        CarTickArgs a = car_tick_args(b, nullptr, 0);
        a.pads = b->pads.ptr;
        apply_commands_kernel<<<(static_cast<int>(count) + 63) / 64, 64, 0, static_cast<cudaStream_t>(stream)>>>(
            a, reinterpret_cast<const rg::EnvCommand*>(device_commands), static_cast<int>(count), b->controls.ptr,
            b->device_status.ptr);
        check(cudaGetLastError(), "apply_commands_kernel launch");
    });
}

RG_API int rg_batch_step_with_device_commands(rg_batch* b, const rg_car_controls* device_controls,
                                              int32_t control_stride, const rg_env_command* device_commands,
                                              int32_t command_stride, int32_t ticks, void* stream) {
    return guard([&] {
        if (!b) throw std::invalid_argument("null argument");
        if (ticks <= 0) return;
        if (!device_controls) throw std::invalid_argument("device_controls_by_tick must not be null");
        if (!device_commands) throw std::invalid_argument("device_env_commands_by_tick must not be null");
        if (control_stride < 0 || (control_stride != 0 && static_cast<int64_t>(control_stride) < rg_batch_car_capacity(b)))
            throw std::invalid_argument("control_stride must be zero or at least the total car capacity");
        if (command_stride < b->env_count) throw std::invalid_argument("env_command_stride must be at least env_count");
        DeviceGuard dg(b->device);
        ensure_kickoff_settled(b, static_cast<cudaStream_t>(stream));
        step_car_path(b, reinterpret_cast<const rg::CarControls*>(device_controls), control_stride, ticks,
                      static_cast<cudaStream_t>(stream), reinterpret_cast<const rg::EnvCommand*>(device_commands),
                      command_stride);
    });
}

RG_API int rg_batch_episode_commands(rg_batch* b, int32_t no_touch_ticks, uint64_t stagger_seed, int32_t init,
                                     rg_env_command* device_commands, void* stream) {
    return guard([&] {
        if (!b || !device_commands) throw std::invalid_argument("null argument");
        if (no_touch_ticks <= 0) throw std::invalid_argument("no_touch_ticks must be positive");
        DeviceGuard dg(b->device);
        episode_commands_kernel<<<(b->env_count + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
            b->envs.ptr, b->cars.ptr, b->env_car_count.ptr, b->episode_touch.ptr, b->episode_seen.ptr,
            reinterpret_cast<rg::EnvCommand*>(device_commands), b->env_count, b->max_cars, no_touch_ticks,
            stagger_seed, init);
        check(cudaGetLastError(), "episode_commands_kernel launch");
    });
}

RG_API int rg_batch_set_launch_config(rg_batch* b, const rg_launch_config* c) {
    return guard([&] {
        if (!b || !c) throw std::invalid_argument("null argument");
        auto ok = [](int t) { return t == 32 || t == 64 || t == 128 || t == 256; };
        if (!ok(c->arena_threads) || !ok(c->car_threads))
            throw std::invalid_argument("threads per block must be 32, 64, 128 or 256");
        DeviceGuard dg(b->device);
        b->launch_threads = c->arena_threads;
        b->car_threads = c->car_threads;
        b->use_graphs = c->use_graphs != 0;
        b->drop_graphs();
    });
}

RG_API int rg_batch_get_launch_config(const rg_batch* b, rg_launch_config* c) {
    return guard([&] {
        if (!b || !c) throw std::invalid_argument("null argument");
        c->arena_threads = b->launch_threads;
        c->car_threads = b->car_threads;
        c->use_graphs = b->use_graphs ? 1 : 0;
        c->reserved = 0;
    });
}

RG_API int rg_batch_phase_timing(rg_batch* b, int32_t enable) {
    return guard([&] {
        if (!b) throw std::invalid_argument("null argument");
        b->timing = enable != 0;
        b->events_used = 0;
    });
}

RG_API int rg_batch_phase_times(rg_batch* b, float* out_ms, int64_t* out_ticks) {
    return guard([&] {
        if (!b || !out_ms) throw std::invalid_argument("null argument");
        DeviceGuard dg(b->device);
        constexpr int kPhases = 6;
        for (int k = 0; k < kPhases; ++k) out_ms[k] = 0.0f;
        const size_t ticks = b->events_used / (kPhases + 1);
        if (ticks) check(cudaEventSynchronize(b->events[b->events_used - 1]), "phase timing sync");
        for (size_t t = 0; t < ticks; ++t)
            for (int k = 0; k < kPhases; ++k) {
                float ms = 0.0f;
                check(cudaEventElapsedTime(&ms, b->events[(kPhases + 1) * t + k], b->events[(kPhases + 1) * t + k + 1]),
                      "phase timing");
                out_ms[k] += ms;
            }
        if (out_ticks) *out_ticks = static_cast<int64_t>(ticks);
        b->events_used = 0;
    });
}

RG_API int rg_batch_synchronize(rg_batch* b, void* stream) {
    return guard([&] {
        if (!b) throw std::invalid_argument("null argument");
        DeviceGuard dg(b->device);
        check(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "synchronize");
    });
}

RG_API int rg_batch_set_physics_event_stream(rg_batch* b, rg_physics_event* records, rg_physics_event_window* windows,
                                             uint32_t capacity_per_env, int32_t goal_only) {
    return guard([&] {
        if (!b) throw std::invalid_argument("null argument");
        const bool off = !records && !windows && capacity_per_env == 0;
        if (!off && (!records || !windows || capacity_per_env == 0))
            throw std::invalid_argument("physics event stream must match the complete batch");
        DeviceGuard dg(b->device);
        rg::EventStream es{};
        if (!off) {
            es.records = reinterpret_cast<rg::PhysicsEvent*>(records);
            es.windows = reinterpret_cast<rg::PhysicsEventWindow*>(windows);
            es.capacity = capacity_per_env;
            es.env_count = static_cast<uint32_t>(b->env_count);
            es.cars_per_env = static_cast<uint32_t>(b->max_cars);
            es.goal_only = goal_only ? 1u : 0u;
        }
        b->tc.events = es;
        b->drop_graphs();  // every captured launch holds the tick config
    });
}

RG_API int rg_batch_add_mesh(rg_batch* b, const rg_arena_layout* layout, int32_t* mesh_index) {
    return guard([&] {
        if (!b || !layout || !mesh_index) throw std::invalid_argument("null argument");
        if (b->extra_meshes.size() + 1 >= 255) throw std::out_of_range("a batch holds at most 255 meshes");
        // the settled kickoffs are recorded on the batch's create-time geometry only
        if (b->cfg.kickoff_settled)
            throw std::invalid_argument("a batch with kickoff_settled = 1 takes no further geometry");
        rg::MeshHost h = rg::build_mesh_host(layout->vertices_uu, layout->vertex_count, layout->indices,
                                             layout->index_count);
        DeviceGuard dg(b->device);
        check(cudaDeviceSynchronize(), "add_mesh");
        b->extra_meshes.push_back(rg::upload_mesh(h));
        std::vector<rg::MeshDevice> table;
        table.push_back(b->mesh);
        for (const rg::MeshDevice& m : b->extra_meshes) table.push_back(m);
        b->drop_graphs();
        b->mesh_table.alloc(table.size());
        check(cudaMemcpy(b->mesh_table.ptr, table.data(), table.size() * sizeof(rg::MeshDevice), cudaMemcpyHostToDevice),
              "mesh table");
        if (!b->mesh_of.ptr) {
            b->mesh_of.alloc(b->env_count);
            check(cudaMemset(b->mesh_of.ptr, 0, b->env_count), "arena meshes");
        }
        *mesh_index = static_cast<int32_t>(table.size() - 1);
    });
}

RG_API int rg_batch_set_arena_meshes(rg_batch* b, const uint8_t* host_mesh_index, size_t count, void* stream) {
    return guard([&] {
        if (!b || (!host_mesh_index && count)) throw std::invalid_argument("null argument");
        if (count > static_cast<size_t>(b->env_count))
            throw std::out_of_range("set_arena_meshes count exceeds env_count");
        const size_t meshes = 1 + b->extra_meshes.size();
        for (size_t i = 0; i < count; ++i)
            if (host_mesh_index[i] >= meshes) throw std::out_of_range("mesh index out of range (rg_batch_add_mesh)");
        if (!count) return;
        if (meshes == 1) return;  // every index is 0: the batch's one mesh
        DeviceGuard dg(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        check(cudaMemcpyAsync(b->mesh_of.ptr, host_mesh_index, count, cudaMemcpyHostToDevice, s), "arena meshes");
        check(cudaStreamSynchronize(s), "arena meshes");
    });
}

RG_API int64_t rg_arena_mesh_tables(const rg_arena_layout* layout, float* out_tri16, int32_t* out_leaf_order,
                                    int64_t cap) {
    int64_t n = -1;
    const int rc = guard([&] {
        if (!layout) throw std::invalid_argument("null layout");
        const rg::MeshHost h = rg::build_mesh_host(layout->vertices_uu, layout->vertex_count, layout->indices,
                                                   layout->index_count);
        n = static_cast<int64_t>(h.tris.size());
        for (int64_t t = 0; t < n && t < cap; ++t) {
            const rg::HostTri& r = h.tris[t];
            const float f[16] = {r.a.x, r.a.y, r.a.z, r.b.x, r.b.y, r.b.z, r.c.x, r.c.y, r.c.z, r.normal.x,
                                 r.normal.y, r.normal.z, r.edge_angle[0], r.edge_angle[1], r.edge_angle[2],
                                 static_cast<float>(r.edge_flags)};
            if (out_tri16) std::memcpy(out_tri16 + 16 * t, f, sizeof(f));
            if (out_leaf_order) out_leaf_order[t] = h.leaf_order[t];
        }
    });
    return rc == 0 ? n : -1;
}

RG_API float rg_ucrt_sinf(float x) { return rg::game_sinf(x); }
RG_API float rg_ucrt_cosf(float x) { return rg::game_cosf(x); }
RG_API float rg_ucrt_atan2f(float y, float x) { return rg::ucrt_atan2f(y, x); }
RG_API float rg_ucrt_powf(float x, float y) { return rg::ucrt_powf(x, y); }

RG_API int rg_batch_device_view(rg_batch* b, rg_device_view* out) {
    return guard([&] {
        if (!b || !out) throw std::invalid_argument("null argument");
        out->ball_states = b->balls.ptr;
        out->env_states = b->envs.ptr;
        out->env_car_count = b->env_car_count.ptr;
        out->car_states = b->cars.ptr;
        out->boost_pad_states = b->pads.ptr;
        out->controls = b->controls.ptr;
        out->car_configs = b->car_cfgs.ptr;
        out->teams = b->teams.ptr;
        out->wheel_runtime = b->wheels.ptr;
    });
}

}  // extern "C"

namespace {
// The internal state blob: named sections of per-arena / per-car device state beyond the public structs (reference
// BatchSim internal_state_layout / download_internal_state / upload_internal_state, python/rocketgpu_bindings.cpp:
// 1002-1060, with this build's own sections).
struct InternalSection {
    const char* name;
    void* ptr;
    size_t bytes;
};
std::vector<InternalSection> internal_sections(rg_batch* b) {
    const size_t env = static_cast<size_t>(b->env_count), cap = env * static_cast<size_t>(b->max_cars);
    return {
        {"wheel_runtime", b->wheels.ptr, cap * sizeof(rg::WheelRuntime)},
        {"ball_world", b->ball_world.ptr, env * sizeof(rg::BallWorldScratch)},
        {"broadphase", b->broadphase.ptr, env * sizeof(rg::Broadphase)},
        {"car_world", b->car_world.ptr, cap * sizeof(rg::CarWorldScratch)},
        {"ball_car", b->ball_car.ptr, cap * sizeof(rg::BallCarScratch)},
        {"car_pairs", b->car_pairs.ptr, env * static_cast<size_t>(b->pair_slots) * sizeof(rg::CarCarManifold)},
        {"car_stages", b->car_stages.ptr, cap * sizeof(rg::CarStage)},
    };
}
}  // namespace

extern "C" {

RG_API int rg_batch_internal_state_layout(rg_batch* b, int32_t index, const char** name, int64_t* bytes) {
    return guard([&] {
        if (!b || !name || !bytes) throw std::invalid_argument("null argument");
        const auto secs = internal_sections(b);
        if (index < 0 || index >= static_cast<int32_t>(secs.size())) throw std::out_of_range("section index");
        *name = secs[index].name;
        *bytes = static_cast<int64_t>(secs[index].bytes);
    });
}

RG_API int rg_batch_download_internal_state(rg_batch* b, void* host, void* stream) {
    return guard([&] {
        if (!b || !host) throw std::invalid_argument("null argument");
        DeviceGuard dg(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        unsigned char* out = static_cast<unsigned char*>(host);
        for (const InternalSection& sec : internal_sections(b)) {
            if (sec.bytes) check(cudaMemcpyAsync(out, sec.ptr, sec.bytes, cudaMemcpyDeviceToHost, s), sec.name);
            out += sec.bytes;
        }
        check(cudaStreamSynchronize(s), "download_internal_state");
    });
}

RG_API int rg_batch_upload_internal_state(rg_batch* b, const void* host, void* stream) {
    return guard([&] {
        if (!b || !host) throw std::invalid_argument("null argument");
        DeviceGuard dg(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const unsigned char* in = static_cast<const unsigned char*>(host);
        for (const InternalSection& sec : internal_sections(b)) {
            if (sec.bytes) check(cudaMemcpyAsync(sec.ptr, in, sec.bytes, cudaMemcpyHostToDevice, s), sec.name);
            in += sec.bytes;
        }
        check(cudaStreamSynchronize(s), "upload_internal_state");
    });
}

RG_API int rg_batch_upload_state_array(rg_batch* b, const char* name, const void* host, size_t count,
                                       int32_t preserve_internal, void* stream) {
    if (!b || !name) return guard([] { throw std::invalid_argument("null argument"); });
    const std::string n(name);
    if (n == "car_states" || n == "ball_states") {
        if (!preserve_internal)
            return n == "car_states"
                       ? rg_batch_upload_car_states(b, static_cast<const rg_car_state*>(host), count, stream)
                       : rg_batch_upload_ball_states(b, static_cast<const rg_ball_state*>(host), count, stream);
        return guard([&] {
            if (n == "car_states")
                upload_array(b, b->cars, static_cast<const rg_car_state*>(host), count,
                             static_cast<size_t>(rg_batch_car_capacity(b)), "upload_state_array(car_states)", stream);
            else
                upload_array(b, b->balls, static_cast<const rg_ball_state*>(host), count,
                             static_cast<size_t>(b->env_count), "upload_state_array(ball_states)", stream);
        });
    }
    if (n == "env_states") return rg_batch_upload_env_states(b, static_cast<const rg_env_state*>(host), count, stream);
    if (n == "boost_pad_states")
        return rg_batch_upload_pad_states(b, static_cast<const rg_boost_pad_state*>(host), count, stream);
    if (n == "controls") return rg_batch_upload_controls(b, static_cast<const rg_car_controls*>(host), count, stream);
    return guard([&] { throw std::invalid_argument("unknown state array: " + n); });
}

RG_API int rg_batch_download_state_array(rg_batch* b, const char* name, void* host, size_t count, void* stream) {
    if (!b || !name) return guard([] { throw std::invalid_argument("null argument"); });
    const std::string n(name);
    if (n == "car_states") return rg_batch_download_car_states(b, static_cast<rg_car_state*>(host), count, stream);
    if (n == "ball_states") return rg_batch_download_ball_states(b, static_cast<rg_ball_state*>(host), count, stream);
    if (n == "env_states") return rg_batch_download_env_states(b, static_cast<rg_env_state*>(host), count, stream);
    if (n == "boost_pad_states")
        return rg_batch_download_pad_states(b, static_cast<rg_boost_pad_state*>(host), count, stream);
    return guard([&] { throw std::invalid_argument("unknown state array: " + n); });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------------
// Stepping without any device allocation.
//
// The per-arena contact manifolds a tick keeps between ticks normally live in memory rg_batch_create allocates, one
// entry per arena of the batch. For callers that may not allocate device memory at the point where they step (a
// process whose device memory belongs to another framework's pool, code that must not trigger the implicit
// synchronisation cudaMalloc can cause, or a step recorded while some other code is capturing a stream), this entry
// point keeps those manifolds in one fixed array compiled into the library instead. The array is a file-scope
// __device__ variable, so every GPU that loads the library holds it (kStaticScratchEnvs entries of
// sizeof(rg::BallWorldScratch) bytes, about 1.1 MB) until the process exits.
namespace {
constexpr int kStaticScratchEnvs = 4096;
static __device__ __align__(256) rg::BallWorldScratch g_static_ball_world[kStaticScratchEnvs];

constexpr int kMaxDevices = 64;
struct StaticScratchSlot {
    std::once_flag once;
    void* addr = nullptr;
    cudaError_t status = cudaSuccess;
};
StaticScratchSlot g_static_scratch[kMaxDevices];

// Device address of g_static_ball_world on the current device. In host code the symbol's name stands for a host-side
// shadow, not the device array, so the address comes from cudaGetSymbolAddress, once per device; the once_flag makes a
// first call from several host threads at the same time look it up once and all see the result.
rg::BallWorldScratch* static_scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device index out of range");
    StaticScratchSlot& slot = g_static_scratch[device];
    std::call_once(slot.once, [&] { slot.status = cudaGetSymbolAddress(&slot.addr, g_static_ball_world); });
    check(slot.status, "cudaGetSymbolAddress(static scratch)");
    return static_cast<rg::BallWorldScratch*>(slot.addr);
}
}  // namespace

extern "C" {

RG_API int rg_batch_step_static_scratch(rg_batch* b, rg_ball_state* dev_balls, rg_env_state* dev_envs,
                                        int32_t env_count, int32_t ticks, int32_t reset_manifolds, void* stream) {
    return guard([&] {
        if (!b || !dev_balls || !dev_envs) throw std::invalid_argument("null argument");
        if (env_count <= 0) throw std::invalid_argument("env_count must be positive");
        if (env_count > kStaticScratchEnvs)
            throw std::out_of_range("env_count exceeds the static scratch capacity (4096 arenas)");
        if (ticks < 0) throw std::invalid_argument("ticks must be >= 0");
        if (b->pads_live) throw std::invalid_argument("rg_batch_step_static_scratch steps ball-only batches");
        DeviceGuard dg(b->device);
        rg::BallWorldScratch* scratch = static_scratch_address(b->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (reset_manifolds) {
            check(cudaMemsetAsync(scratch, 0, static_cast<size_t>(env_count) * sizeof(rg::BallWorldScratch), s),
                  "clear static scratch");
        }
        if (ticks == 0) return;
        TickArgs a;
        a.balls = reinterpret_cast<rg::BallState*>(dev_balls);
        a.envs = reinterpret_cast<rg::EnvState*>(dev_envs);
        a.env_car_count = b->env_car_count.ptr;
        a.ball_world = scratch;
        a.env_count = env_count;
        a.tc = b->tc;
        a.mesh = b->mesh;
        a.meshes = b->mesh_table.ptr;
        a.mesh_of = b->mesh_table.ptr ? b->mesh_of.ptr : nullptr;
        const int threads = b->launch_threads;
        tick_kernel<<<(env_count + threads - 1) / threads, threads, 0, s>>>(a, ticks);
        check(cudaGetLastError(), "tick_kernel launch (static scratch)");
    });
}

}  // extern "C"

#include "rg_server.cuh"
