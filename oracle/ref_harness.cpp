// Oracle harness: a flat C ABI over the reference's own CPU BatchSim.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the reference's unmodified CPU sources
// (src/rocketgpu.cpp, src/arena/mesh_loader.cpp, read in place from the reference tree by oracle/Makefile) into
// oracle/_ref/librg_oracle.so. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, as the
// checker and the timed CPU baseline; the product (rocketgpu_b200) never links or calls it.
//
// Every entry point wraps one BatchSim method (include/rocketgpu/rocketgpu.h:988-1089) and turns C++ exceptions into
// a nonzero status plus orc_last_error(). The arena is a custom ArenaLayout whose only geometry is one triangle mesh
// given in uu (ArenaLayout::meshes, include/rocketgpu/rocketgpu.h:943-959); pads, goals and spawns keep the layout's
// defaults (the official soccar ones).
#include <rocketgpu/rocketgpu.h>
#include <rocketgpu/detail/arena/mesh_loader.hpp>
#include <rocketgpu/detail/step.hpp>

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

using namespace rocketgpu;

namespace {
thread_local std::string g_last_error;

template <class F>
int Guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 1;
    } catch (...) {
        g_last_error = "unknown C++ exception";
        return 1;
    }
}

struct OracleSim {
    std::unique_ptr<BatchSim> sim;
};
}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_last_error.c_str(); }

// Struct sizes, in this order: CarState, BallState, EnvState, BoostPadState, CarControls, CarConfig, EnvCommand,
// SimConfig, MutatorConfig.
int orc_struct_sizes(int64_t* out, int n) {
    const int64_t s[] = {(int64_t)sizeof(CarState),    (int64_t)sizeof(BallState),   (int64_t)sizeof(EnvState),
                         (int64_t)sizeof(BoostPadState), (int64_t)sizeof(CarControls), (int64_t)sizeof(CarConfig),
                         (int64_t)sizeof(EnvCommand),  (int64_t)sizeof(SimConfig),   (int64_t)sizeof(MutatorConfig)};
    const int k = (int)(sizeof(s) / sizeof(s[0]));
    for (int i = 0; i < n && i < k; ++i) out[i] = s[i];
    return k;
}

// Car hitbox presets (src/rocketgpu.cpp:417-499): 0 Octane, 1 Dominus, 2 Plank, 3 Breakout, 4 Hybrid, 5 Merc.
int orc_car_preset(int which, void* out) {
    return Guard([&] {
        CarConfig c;
        switch (which) {
            case 0: c = OctaneConfig(); break;
            case 1: c = DominusConfig(); break;
            case 2: c = PlankConfig(); break;
            case 3: c = BreakoutConfig(); break;
            case 4: c = HybridConfig(); break;
            case 5: c = MercConfig(); break;
            default: throw std::invalid_argument("preset out of range");
        }
        std::memcpy(out, &c, sizeof(c));
    });
}

// Default-constructed public state structs (the reference's initialisers), for layout tests.
int orc_default_states(void* car, void* ball, void* env, void* pad, void* cfg) {
    return Guard([&] {
        CarState c; BallState b; EnvState e; BoostPadState p; CarConfig k;
        if (car) std::memcpy(car, &c, sizeof(c));
        if (ball) std::memcpy(ball, &b, sizeof(b));
        if (env) std::memcpy(env, &e, sizeof(e));
        if (pad) std::memcpy(pad, &p, sizeof(p));
        if (cfg) std::memcpy(cfg, &k, sizeof(k));
    });
}

// flags bit0: kickoff_settled (MutatorConfig::kickoff_settled); bit1: enable_boost_pads; bit2: car-car collisions;
// bit3: demos; bit4: scoring.
// rules_f (optional): 99 floats, goals[2] (point, normal, min, max), kickoff_spawns[2][5] (pos, yaw),
// respawn_spawns[2][4] (pos, yaw), ball_spawn; pads_f (optional): pad_count x (x, y, z, is_big).
int orc_create_layout(int32_t env_count, int32_t max_cars, const float* verts_uu, int64_t vert_count,
                      const int32_t* indices, int64_t index_count, uint64_t respawn_seed, uint32_t flags,
                      const float* rules_f, const float* pads_f, int32_t pad_count, void** out);
int orc_create(int32_t env_count, int32_t max_cars, const float* verts_uu, int64_t vert_count, const int32_t* indices,
               int64_t index_count, uint64_t respawn_seed, uint32_t flags, void** out) {
    return orc_create_layout(env_count, max_cars, verts_uu, vert_count, indices, index_count, respawn_seed, flags,
                             nullptr, nullptr, 0, out);
}
int orc_create_layout(int32_t env_count, int32_t max_cars, const float* verts_uu, int64_t vert_count,
                      const int32_t* indices, int64_t index_count, uint64_t respawn_seed, uint32_t flags,
                      const float* rules_f, const float* pads_f, int32_t pad_count, void** out) {
    return Guard([&] {
        SimConfig cfg;
        cfg.env_count = env_count;
        cfg.max_cars_per_env = max_cars;
        cfg.respawn_rng_seed = respawn_seed;
        cfg.mutator.kickoff_settled = (flags & 1u) ? 1 : 0;
        cfg.enable_boost_pads = (flags & 2u) ? 1 : 0;
        cfg.enable_car_car_collisions = (flags & 4u) ? 1 : 0;
        cfg.enable_demos = (flags & 8u) ? 1 : 0;
        cfg.enable_scoring = (flags & 16u) ? 1 : 0;
        ArenaLayout layout;
        ArenaMesh mesh;
        mesh.vertices.resize((size_t)vert_count);
        for (int64_t i = 0; i < vert_count; ++i) {
            mesh.vertices[(size_t)i] = Vec3(verts_uu[3 * i], verts_uu[3 * i + 1], verts_uu[3 * i + 2]);
        }
        mesh.indices.assign(indices, indices + index_count);
        layout.meshes.push_back(std::move(mesh));
        if (rules_f) {
            const float* f = rules_f;
            auto v3 = [&]() { const Vec3 v(f[0], f[1], f[2]); f += 3; return v; };
            for (int t = 0; t < 2; ++t) {
                layout.goals[t].point = v3();
                layout.goals[t].normal = v3();
                layout.goals[t].min = v3();
                layout.goals[t].max = v3();
            }
            for (int t = 0; t < 2; ++t)
                for (int k = 0; k < 5; ++k) {
                    layout.kickoff_spawns[t][k].pos = v3();
                    layout.kickoff_spawns[t][k].yaw = *f++;
                }
            for (int t = 0; t < 2; ++t)
                for (int k = 0; k < 4; ++k) {
                    layout.respawn_spawns[t][k].pos = v3();
                    layout.respawn_spawns[t][k].yaw = *f++;
                }
            layout.ball_spawn = v3();
        }
        if (pads_f) {
            layout.boost_pads.resize((size_t)pad_count);
            for (int32_t p = 0; p < pad_count; ++p) {
                layout.boost_pads[(size_t)p].pos = Vec3(pads_f[4 * p], pads_f[4 * p + 1], pads_f[4 * p + 2]);
                layout.boost_pads[(size_t)p].is_big = pads_f[4 * p + 3] != 0.0f ? 1 : 0;
            }
        }
        auto* o = new OracleSim;
        o->sim.reset(new BatchSim(cfg, layout));
        *out = o;
    });
}

void orc_destroy(void* h) { delete static_cast<OracleSim*>(h); }

#define ORC_SIM static_cast<OracleSim*>(h)->sim

int64_t orc_car_capacity(void* h) { return (int64_t)ORC_SIM->car_capacity(); }
int64_t orc_pad_capacity(void* h) { return (int64_t)ORC_SIM->boost_pad_capacity(); }

int orc_set_env_car_count(void* h, const int32_t* counts, int64_t n) {
    return Guard([&] { ORC_SIM->set_env_car_count(counts, (size_t)n); });
}
int orc_set_teams(void* h, const uint8_t* teams, int64_t n) {
    return Guard([&] { ORC_SIM->set_teams(reinterpret_cast<const Team*>(teams), (size_t)n); });
}
int orc_set_car_configs(void* h, const void* cfgs, int64_t n) {
    return Guard([&] { ORC_SIM->set_car_configs(static_cast<const CarConfig*>(cfgs), (size_t)n); });
}
int orc_reset_to_kickoff(void* h, uint64_t seed) {
    return Guard([&] { ORC_SIM->reset_to_kickoff(seed); });
}
int orc_apply_env_commands(void* h, const void* cmds, int64_t n) {
    return Guard([&] { ORC_SIM->apply_env_commands(static_cast<const EnvCommand*>(cmds), (size_t)n); });
}
int orc_upload_controls(void* h, const void* ctrl, int64_t n) {
    return Guard([&] { ORC_SIM->upload_controls(static_cast<const CarControls*>(ctrl), (size_t)n); });
}
int orc_step(void* h, int32_t ticks) {
    return Guard([&] { ORC_SIM->step(ticks); });
}
// CPU builds take host pointers here (the controls of tick t for car slot c at ctrl[t * stride + c]).
int orc_step_with_controls(void* h, const void* ctrl, int32_t ticks, int32_t stride) {
    return Guard([&] {
        ORC_SIM->step_with_device_controls(static_cast<const CarControls*>(ctrl), ticks, stride);
    });
}
int orc_step_with_commands(void* h, const void* ctrl, int32_t ctrl_stride, const void* cmds, int32_t cmd_stride,
                           int32_t ticks) {
    return Guard([&] {
        ORC_SIM->step_with_device_commands(static_cast<const CarControls*>(ctrl), ctrl_stride,
                                           static_cast<const EnvCommand*>(cmds), cmd_stride, ticks);
    });
}

// BatchSim::set_physics_event_stream with host arrays (the CPU build writes them directly): records[env * capacity + k],
// windows[env]; capacity 0 and null arrays turn the stream off. Also reports the struct sizes the checker reads.
int orc_set_physics_event_stream(void* h, void* records, void* windows, uint32_t capacity, int goal_only) {
    return Guard([&] {
        PhysicsEventStream s;
        s.records = static_cast<PhysicsEvent*>(records);
        s.windows = static_cast<PhysicsEventWindow*>(windows);
        s.capacity_per_env = capacity;
        if (records || windows || capacity) {
            s.goal_only = goal_only != 0;
            s.env_count = static_cast<uint32_t>(ORC_SIM->env_count());
            s.cars_per_env = static_cast<uint32_t>(ORC_SIM->car_capacity() / ORC_SIM->env_count());
        }
        ORC_SIM->set_physics_event_stream(s);
    });
}
int orc_physics_event_sizes(int64_t* out) {
    out[0] = sizeof(PhysicsEvent);
    out[1] = sizeof(PhysicsEventWindow);
    out[2] = offsetof(PhysicsEvent, position);
    out[3] = offsetof(PhysicsEvent, boost_after);
    return 0;
}

int orc_download_cars(void* h, void* out, int64_t n) {
    return Guard([&] { ORC_SIM->download_car_states(static_cast<CarState*>(out), (size_t)n); });
}
int orc_download_balls(void* h, void* out, int64_t n) {
    return Guard([&] { ORC_SIM->download_ball_states(static_cast<BallState*>(out), (size_t)n); });
}
int orc_download_envs(void* h, void* out, int64_t n) {
    return Guard([&] { ORC_SIM->download_env_states(static_cast<EnvState*>(out), (size_t)n); });
}
int orc_download_pads(void* h, void* out, int64_t n) {
    return Guard([&] { ORC_SIM->download_boost_pad_states(static_cast<BoostPadState*>(out), (size_t)n); });
}
int orc_upload_cars(void* h, const void* in, int64_t n, int preserve_internal) {
    return Guard([&] {
        ORC_SIM->upload_car_states(static_cast<const CarState*>(in), (size_t)n, nullptr,
                                   preserve_internal ? BatchSim::StateUploadMode::PreserveInternal
                                                     : BatchSim::StateUploadMode::PublicState);
    });
}
int orc_upload_balls(void* h, const void* in, int64_t n, int preserve_internal) {
    return Guard([&] {
        ORC_SIM->upload_ball_states(static_cast<const BallState*>(in), (size_t)n, nullptr,
                                    preserve_internal ? BatchSim::StateUploadMode::PreserveInternal
                                                      : BatchSim::StateUploadMode::PublicState);
    });
}
int orc_upload_envs(void* h, const void* in, int64_t n) {
    return Guard([&] { ORC_SIM->upload_env_states(static_cast<const EnvState*>(in), (size_t)n); });
}
int orc_upload_pads(void* h, const void* in, int64_t n) {
    return Guard([&] { ORC_SIM->upload_boost_pad_states(static_cast<const BoostPadState*>(in), (size_t)n); });
}

// The reference's float transcendental routines (include/rocketgpu/detail/math.hpp:39-584), for checking the
// product's restatement of them.
float orc_ucrt_sinf(float x) { return RocketGpuSinf(x); }
float orc_ucrt_cosf(float x) { return RocketGpuCosf(x); }
float orc_ucrt_atan2f(float y, float x) { return RocketGpuUcrtAtan2f(y, x); }
float orc_ucrt_powf(float x, float y) { return RocketGpuUcrtPowf(x, y); }

// The reference's host-side mesh tables for a one-mesh custom arena (src/arena/mesh_loader.cpp:1263-1411): per
// triangle a, b, c, normal (bt) and the three internal-edge angles + flags (16 floats each, flags as float), and the
// triangle index of each BVH leaf in stackless-walk order. Returns the triangle count; leaf order via orc_mesh_leaves.
namespace {
std::vector<rocketgpu::detail::ArenaMeshTriangle> g_tris;
std::vector<rocketgpu::detail::ArenaMeshBvhNode> g_nodes;
std::vector<rocketgpu::detail::ArenaMeshBvhQuantization> g_quant;
}  // namespace

int64_t orc_mesh_tables(const float* verts_uu, int64_t vert_count, const int32_t* indices, int64_t index_count,
                        float* out_tri16, int64_t cap) {
    using namespace rocketgpu::detail;
    ArenaMeshSource src;
    for (int64_t i = 0; i < vert_count; ++i) {
        src.vertices.push_back(Vec3(verts_uu[3 * i] * (1.0f / 50.0f), verts_uu[3 * i + 1] * (1.0f / 50.0f),
                                    verts_uu[3 * i + 2] * (1.0f / 50.0f)));
    }
    src.indices.assign(indices, indices + index_count);
    std::vector<ArenaMeshSource> sources{src};
    std::vector<ArenaMeshBvhMeshInfo> infos;
    std::vector<ArenaMeshBvhSubtreeInfo> subtrees;
    std::vector<ArenaMeshTriangle> local;
    g_tris = LoadCustomArenaMeshTriangles(sources, g_quant, infos, g_nodes, subtrees, local);
    const int64_t n = (int64_t)g_tris.size();
    for (int64_t t = 0; t < n && t < cap; ++t) {
        const ArenaMeshTriangle& r = g_tris[(size_t)t];
        const float f[16] = {r.a.x, r.a.y, r.a.z, r.b.x, r.b.y, r.b.z, r.c.x, r.c.y, r.c.z, r.normal.x, r.normal.y,
                             r.normal.z, r.edge_v0v1_angle, r.edge_v1v2_angle, r.edge_v2v0_angle, (float)r.edge_flags};
        std::memcpy(out_tri16 + 16 * t, f, sizeof(f));
    }
    return n;
}

// After orc_mesh_tables: BVH node count, and per node (min xyz, max xyz as uint16, escape/triangle index).
int64_t orc_mesh_nodes(int32_t* out7, int64_t cap) {
    const int64_t n = (int64_t)g_nodes.size();
    for (int64_t i = 0; i < n && i < cap; ++i) {
        const auto& nd = g_nodes[(size_t)i];
        for (int a = 0; a < 3; ++a) {
            out7[7 * i + a] = nd.quantized_aabb_min[a];
            out7[7 * i + 3 + a] = nd.quantized_aabb_max[a];
        }
        out7[7 * i + 6] = nd.escape_index_or_triangle_index;
    }
    return n;
}

// After orc_mesh_tables: the BVH quantization (aabb min xyz, max xyz, scale xyz).
void orc_mesh_quantization(float* out9) {
    const auto& q = g_quant[0];
    const float f[9] = {q.bvh_aabb_min.x, q.bvh_aabb_min.y, q.bvh_aabb_min.z, q.bvh_aabb_max.x, q.bvh_aabb_max.y,
                        q.bvh_aabb_max.z, q.bvh_quantization.x, q.bvh_quantization.y, q.bvh_quantization.z};
    std::memcpy(out9, f, sizeof(f));
}

}  // extern "C"
