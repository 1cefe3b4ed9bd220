// rocketgpu_py_b200: a pybind11 module over the C ABI (include/rocketgpu_b200.h) with the method names, argument
// order and exceptions of the reference's Python binding `rocketgpu_py.BatchSim` (python/rocketgpu_bindings.cpp:
// 827-1000), so Python code written against the reference switches by changing the import.
//
// Differences, each forced by the C ABI: state arrays are passed as buffers of raw structs (numpy arrays or bytes of
// the reference's struct layouts, which the ABI keeps byte-identical) where the reference takes lists of bound
// struct objects; downloads return numpy uint8 arrays [count, sizeof(struct)]; the layout is one triangle mesh
// (ArenaLayout.meshes[0]); configs are the ABI's rg_sim_config fields. Errors map as in the reference: ValueError
// (std::invalid_argument), IndexError (std::out_of_range), RuntimeError (CUDA and other failures).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "rocketgpu_b200.h"

namespace py = pybind11;

namespace {

void check(int rc) {
    if (rc == 0) return;
    const std::string msg = rg_last_error();
    if (rc == 2) throw py::value_error(msg);
    if (rc == 3) throw py::index_error(msg);
    throw std::runtime_error(msg);
}

void* stream_of(uintptr_t s) { return reinterpret_cast<void*>(s); }

// A buffer of raw structs of `size` bytes each: returns the pointer and the struct count.
std::pair<const void*, size_t> structs(const py::buffer& b, size_t size, const char* what) {
    const py::buffer_info info = b.request();
    const size_t bytes = static_cast<size_t>(info.size) * static_cast<size_t>(info.itemsize);
    if (bytes % size) throw py::value_error(std::string(what) + ": buffer is not a whole number of structs");
    return {info.ptr, bytes / size};
}

struct ArenaMesh {
    std::vector<float> vertices;  // 3 per vertex, uu
    std::vector<int32_t> indices;
};

struct ArenaLayout {
    std::vector<ArenaMesh> meshes;
    std::vector<rg_boost_pad_config> boost_pads;  // empty: the 34 soccar pads
    rg_arena_rules rules;
    ArenaLayout() { rg_default_arena_rules(&rules); }
};

class BatchSim {
   public:
    BatchSim(const rg_sim_config& cfg, const ArenaLayout& layout, int device) {
        if (layout.meshes.size() != 1) throw py::value_error("the layout must hold exactly one mesh");
        const ArenaMesh& m = layout.meshes[0];
        rg_arena_layout l{m.vertices.data(), static_cast<int64_t>(m.vertices.size() / 3), m.indices.data(),
                          static_cast<int64_t>(m.indices.size())};
        l.rules = &layout.rules;
        if (!layout.boost_pads.empty()) {
            l.boost_pads = layout.boost_pads.data();
            l.boost_pad_count = static_cast<int32_t>(layout.boost_pads.size());
        }
        check(rg_batch_create(&cfg, &l, device, &b_));
        cfg_ = cfg;
    }
    ~BatchSim() { rg_batch_destroy(b_); }
    BatchSim(const BatchSim&) = delete;
    BatchSim& operator=(const BatchSim&) = delete;

    int64_t env_count() const { return rg_batch_env_count(b_); }
    int64_t car_capacity() const { return rg_batch_car_capacity(b_); }
    int64_t boost_pad_capacity() const { return rg_batch_pad_capacity(b_); }
    const rg_sim_config& config() const { return cfg_; }

    void set_env_car_count(const std::vector<int32_t>& counts, uintptr_t s) {
        check(rg_batch_set_env_car_count(b_, counts.data(), counts.size(), stream_of(s)));
    }
    void set_teams(const std::vector<uint8_t>& teams, uintptr_t s) {
        check(rg_batch_set_teams(b_, teams.data(), teams.size(), stream_of(s)));
    }
    void set_car_configs(const py::buffer& configs, uintptr_t s) {
        auto c = structs(configs, sizeof(rg_car_config), "set_car_configs");
        check(rg_batch_set_car_configs(b_, static_cast<const rg_car_config*>(c.first), c.second, stream_of(s)));
    }
    void upload(const std::string& name, const py::buffer& states, bool preserve_internal, uintptr_t s) {
        auto c = structs(states, struct_size(name), name.c_str());
        check(rg_batch_upload_state_array(b_, name.c_str(), c.first, c.second, preserve_internal ? 1 : 0,
                                          stream_of(s)));
    }
    py::array_t<uint8_t> download(const std::string& name, int64_t count, uintptr_t s) {
        const size_t size = struct_size(name);
        const int64_t n = count >= 0 ? count : default_count(name);
        py::array_t<uint8_t> out({static_cast<py::ssize_t>(n), static_cast<py::ssize_t>(size)});
        check(rg_batch_download_state_array(b_, name.c_str(), out.mutable_data(), static_cast<size_t>(n),
                                            stream_of(s)));
        return out;
    }
    void upload_state_array(const std::string& name, uintptr_t host_ptr, size_t count, bool preserve, uintptr_t s) {
        check(rg_batch_upload_state_array(b_, name.c_str(), reinterpret_cast<const void*>(host_ptr), count,
                                          preserve ? 1 : 0, stream_of(s)));
    }
    void download_state_array(const std::string& name, uintptr_t host_ptr, size_t count, uintptr_t s) {
        check(rg_batch_download_state_array(b_, name.c_str(), reinterpret_cast<void*>(host_ptr), count,
                                            stream_of(s)));
    }
    py::list internal_state_layout() const {
        py::list out;
        for (int32_t i = 0;; ++i) {
            const char* name = nullptr;
            int64_t bytes = 0;
            if (rg_batch_internal_state_layout(b_, i, &name, &bytes) != 0) break;
            out.append(py::make_tuple(std::string(name), static_cast<size_t>(bytes)));
        }
        return out;
    }
    void download_internal_state(uintptr_t host_ptr, uintptr_t s) {
        check(rg_batch_download_internal_state(b_, reinterpret_cast<void*>(host_ptr), stream_of(s)));
    }
    void upload_internal_state(uintptr_t host_ptr, uintptr_t s) {
        check(rg_batch_upload_internal_state(b_, reinterpret_cast<const void*>(host_ptr), stream_of(s)));
    }
    void upload_controls(const py::buffer& controls, uintptr_t s) {
        auto c = structs(controls, sizeof(rg_car_controls), "upload_controls");
        check(rg_batch_upload_controls(b_, static_cast<const rg_car_controls*>(c.first), c.second, stream_of(s)));
    }
    void apply_env_commands(const py::buffer& commands, uintptr_t s) {
        auto c = structs(commands, sizeof(rg_env_command), "apply_env_commands");
        check(rg_batch_apply_env_commands(b_, static_cast<const rg_env_command*>(c.first), c.second, stream_of(s)));
    }
    void apply_env_commands_device(uintptr_t ptr, size_t count, uintptr_t s) {
        check(rg_batch_apply_env_commands_device(b_, reinterpret_cast<const rg_env_command*>(ptr), count,
                                                 stream_of(s)));
    }
    void step(int32_t ticks, uintptr_t s) { check(rg_batch_step(b_, ticks, stream_of(s))); }
    void step_with_device_controls(uintptr_t ptr, int32_t ticks, int32_t stride, uintptr_t s) {
        check(rg_batch_step_with_device_controls(b_, reinterpret_cast<const rg_car_controls*>(ptr), ticks, stride,
                                                 stream_of(s)));
    }
    void step_with_device_commands(uintptr_t ctrl, int32_t ctrl_stride, uintptr_t cmds, int32_t cmd_stride,
                                   int32_t ticks, uintptr_t s) {
        check(rg_batch_step_with_device_commands(b_, reinterpret_cast<const rg_car_controls*>(ctrl), ctrl_stride,
                                                 reinterpret_cast<const rg_env_command*>(cmds), cmd_stride, ticks,
                                                 stream_of(s)));
    }
    void reset_to_kickoff(uint64_t seed, uintptr_t s) { check(rg_batch_reset_to_kickoff(b_, seed, stream_of(s))); }
    void synchronize(uintptr_t s) { check(rg_batch_synchronize(b_, stream_of(s))); }
    // reference binding set_physics_event_stream (python/rocketgpu_bindings.cpp:832-845): device addresses; zeros
    // turn the stream off
    void set_physics_event_stream(uintptr_t records, uintptr_t windows, uint32_t capacity, bool goal_only) {
        check(rg_batch_set_physics_event_stream(b_, reinterpret_cast<rg_physics_event*>(records),
                                                reinterpret_cast<rg_physics_event_window*>(windows), capacity,
                                                goal_only ? 1 : 0));
    }
    py::dict device_view() {
        rg_device_view v{};
        check(rg_batch_device_view(b_, &v));
        py::dict d;
        d["ball_states"] = reinterpret_cast<uintptr_t>(v.ball_states);
        d["env_states"] = reinterpret_cast<uintptr_t>(v.env_states);
        d["env_car_count"] = reinterpret_cast<uintptr_t>(v.env_car_count);
        d["car_states"] = reinterpret_cast<uintptr_t>(v.car_states);
        d["boost_pad_states"] = reinterpret_cast<uintptr_t>(v.boost_pad_states);
        d["controls"] = reinterpret_cast<uintptr_t>(v.controls);
        d["car_configs"] = reinterpret_cast<uintptr_t>(v.car_configs);
        d["teams"] = reinterpret_cast<uintptr_t>(v.teams);
        return d;
    }

   private:
    static size_t struct_size(const std::string& name) {
        if (name == "car_states") return sizeof(rg_car_state);
        if (name == "ball_states") return sizeof(rg_ball_state);
        if (name == "env_states") return sizeof(rg_env_state);
        if (name == "boost_pad_states") return sizeof(rg_boost_pad_state);
        if (name == "controls") return sizeof(rg_car_controls);
        throw py::value_error("unknown state array: " + name);
    }
    int64_t default_count(const std::string& name) const {
        if (name == "ball_states" || name == "env_states") return env_count();
        if (name == "boost_pad_states") return boost_pad_capacity();
        return car_capacity();
    }
    rg_batch* b_ = nullptr;
    rg_sim_config cfg_{};
};

}  // namespace

PYBIND11_MODULE(rocketgpu_py_b200, m) {
    m.doc() = "rocketgpu_b200 through the reference's rocketgpu_py BatchSim interface (C ABI underneath)";
    py::class_<rg_sim_config>(m, "SimConfig")
        .def(py::init([] {
            rg_sim_config c;
            rg_sim_config_default(&c);
            return c;
        }))
        .def_readwrite("env_count", &rg_sim_config::env_count)
        .def_readwrite("max_cars_per_env", &rg_sim_config::max_cars_per_env)
        .def_readwrite("tick_dt", &rg_sim_config::tick_dt)
        .def_readwrite("enable_boost_pads", &rg_sim_config::enable_boost_pads)
        .def_readwrite("enable_car_car_collisions", &rg_sim_config::enable_car_car_collisions)
        .def_readwrite("enable_demos", &rg_sim_config::enable_demos)
        .def_readwrite("enable_scoring", &rg_sim_config::enable_scoring)
        .def_readwrite("gravity_z", &rg_sim_config::gravity_z)
        .def_readwrite("ball_radius", &rg_sim_config::ball_radius)
        .def_readwrite("car_mass", &rg_sim_config::car_mass)
        .def_readwrite("kickoff_settled", &rg_sim_config::kickoff_settled);
    py::class_<ArenaMesh>(m, "ArenaMesh")
        .def(py::init<>())
        .def(py::init([](py::array_t<float, py::array::c_style | py::array::forcecast> v,
                         py::array_t<int32_t, py::array::c_style | py::array::forcecast> i) {
                 ArenaMesh a;
                 a.vertices.assign(v.data(), v.data() + v.size());
                 a.indices.assign(i.data(), i.data() + i.size());
                 return a;
             }),
             py::arg("vertices"), py::arg("indices"))
        .def_readwrite("vertices", &ArenaMesh::vertices)
        .def_readwrite("indices", &ArenaMesh::indices);
    py::class_<rg_vec3>(m, "Vec3")
        .def(py::init([](float x, float y, float z) { return rg_vec3{x, y, z}; }), py::arg("x") = 0.0f,
             py::arg("y") = 0.0f, py::arg("z") = 0.0f)
        .def_readwrite("x", &rg_vec3::x)
        .def_readwrite("y", &rg_vec3::y)
        .def_readwrite("z", &rg_vec3::z);
    py::class_<rg_arena_spawn>(m, "ArenaSpawn")
        .def(py::init([](rg_vec3 pos, float yaw) { return rg_arena_spawn{pos, yaw}; }), py::arg("pos") = rg_vec3{},
             py::arg("yaw") = 0.0f)
        .def_readwrite("pos", &rg_arena_spawn::pos)
        .def_readwrite("yaw", &rg_arena_spawn::yaw);
    py::class_<rg_arena_goal>(m, "ArenaGoal")
        .def(py::init([]() { rg_arena_rules r; rg_default_arena_rules(&r); return r.goals[1]; }))
        .def_readwrite("point", &rg_arena_goal::point)
        .def_readwrite("normal", &rg_arena_goal::normal)
        .def_readwrite("min", &rg_arena_goal::min)
        .def_readwrite("max", &rg_arena_goal::max);
    py::class_<rg_boost_pad_config>(m, "BoostPadConfig")
        .def(py::init([](rg_vec3 pos, bool is_big) {
                 rg_boost_pad_config c{};
                 c.pos = pos;
                 c.is_big = is_big ? 1 : 0;
                 return c;
             }),
             py::arg("pos") = rg_vec3{}, py::arg("is_big") = false)
        .def_readwrite("pos", &rg_boost_pad_config::pos)
        .def_readwrite("is_big", &rg_boost_pad_config::is_big);
    // the rules part is read and written whole (lists of copies), as the reference binding's arrays are
    py::class_<ArenaLayout>(m, "ArenaLayout")
        .def(py::init<>())
        .def_readwrite("meshes", &ArenaLayout::meshes)
        .def_readwrite("boost_pads", &ArenaLayout::boost_pads)
        .def_property(
            "goals", [](const ArenaLayout& l) { return std::vector<rg_arena_goal>{l.rules.goals[0], l.rules.goals[1]}; },
            [](ArenaLayout& l, const std::vector<rg_arena_goal>& g) {
                if (g.size() != 2) throw py::value_error("goals: two goals (blue, orange)");
                l.rules.goals[0] = g[0];
                l.rules.goals[1] = g[1];
            })
        .def_property(
            "kickoff_spawns",
            [](const ArenaLayout& l) {
                std::vector<std::vector<rg_arena_spawn>> out(2);
                for (int t = 0; t < 2; ++t) out[t].assign(l.rules.kickoff_spawns[t], l.rules.kickoff_spawns[t] + 5);
                return out;
            },
            [](ArenaLayout& l, const std::vector<std::vector<rg_arena_spawn>>& v) {
                if (v.size() != 2 || v[0].size() != 5 || v[1].size() != 5)
                    throw py::value_error("kickoff_spawns: 2 teams x 5 spawns");
                for (int t = 0; t < 2; ++t)
                    for (int k = 0; k < 5; ++k) l.rules.kickoff_spawns[t][k] = v[t][k];
            })
        .def_property(
            "respawn_spawns",
            [](const ArenaLayout& l) {
                std::vector<std::vector<rg_arena_spawn>> out(2);
                for (int t = 0; t < 2; ++t) out[t].assign(l.rules.respawn_spawns[t], l.rules.respawn_spawns[t] + 4);
                return out;
            },
            [](ArenaLayout& l, const std::vector<std::vector<rg_arena_spawn>>& v) {
                if (v.size() != 2 || v[0].size() != 4 || v[1].size() != 4)
                    throw py::value_error("respawn_spawns: 2 teams x 4 spawns");
                for (int t = 0; t < 2; ++t)
                    for (int k = 0; k < 4; ++k) l.rules.respawn_spawns[t][k] = v[t][k];
            })
        .def_property(
            "ball_spawn", [](const ArenaLayout& l) { return l.rules.ball_spawn; },
            [](ArenaLayout& l, rg_vec3 v) { l.rules.ball_spawn = v; });
    py::class_<BatchSim>(m, "BatchSim")
        .def(py::init<const rg_sim_config&, const ArenaLayout&, int>(), py::arg("config"), py::arg("layout"),
             py::arg("device") = 0)
        .def_property_readonly("config", &BatchSim::config)
        .def("env_count", &BatchSim::env_count)
        .def("car_capacity", &BatchSim::car_capacity)
        .def("boost_pad_capacity", &BatchSim::boost_pad_capacity)
        .def("device_view", &BatchSim::device_view)
        .def("set_env_car_count", &BatchSim::set_env_car_count, py::arg("counts"), py::arg("stream") = 0)
        .def("set_teams", &BatchSim::set_teams, py::arg("teams"), py::arg("stream") = 0)
        .def("set_car_configs", &BatchSim::set_car_configs, py::arg("configs"), py::arg("stream") = 0)
        .def("upload_car_states",
             [](BatchSim& s, const py::buffer& b, uintptr_t st) { s.upload("car_states", b, false, st); },
             py::arg("states"), py::arg("stream") = 0)
        .def("upload_ball_states",
             [](BatchSim& s, const py::buffer& b, uintptr_t st) { s.upload("ball_states", b, false, st); },
             py::arg("states"), py::arg("stream") = 0)
        .def("upload_env_states",
             [](BatchSim& s, const py::buffer& b, uintptr_t st) { s.upload("env_states", b, false, st); },
             py::arg("states"), py::arg("stream") = 0)
        .def("upload_boost_pad_states",
             [](BatchSim& s, const py::buffer& b, uintptr_t st) { s.upload("boost_pad_states", b, false, st); },
             py::arg("states"), py::arg("stream") = 0)
        .def("upload_controls", &BatchSim::upload_controls, py::arg("controls"), py::arg("stream") = 0)
        .def("download_car_states",
             [](BatchSim& s, int64_t n, uintptr_t st) { return s.download("car_states", n, st); },
             py::arg("count") = -1, py::arg("stream") = 0)
        .def("download_ball_states",
             [](BatchSim& s, int64_t n, uintptr_t st) { return s.download("ball_states", n, st); },
             py::arg("count") = -1, py::arg("stream") = 0)
        .def("download_env_states",
             [](BatchSim& s, int64_t n, uintptr_t st) { return s.download("env_states", n, st); },
             py::arg("count") = -1, py::arg("stream") = 0)
        .def("download_boost_pad_states",
             [](BatchSim& s, int64_t n, uintptr_t st) { return s.download("boost_pad_states", n, st); },
             py::arg("count") = -1, py::arg("stream") = 0)
        .def("upload_state_array", &BatchSim::upload_state_array, py::arg("name"), py::arg("host_ptr"),
             py::arg("count"), py::arg("preserve_internal") = false, py::arg("stream") = 0)
        .def("download_state_array", &BatchSim::download_state_array, py::arg("name"), py::arg("host_ptr"),
             py::arg("count"), py::arg("stream") = 0)
        .def("internal_state_layout", &BatchSim::internal_state_layout)
        .def("download_internal_state", &BatchSim::download_internal_state, py::arg("host_ptr"), py::arg("stream") = 0)
        .def("upload_internal_state", &BatchSim::upload_internal_state, py::arg("host_ptr"), py::arg("stream") = 0)
        .def("apply_env_commands", &BatchSim::apply_env_commands, py::arg("commands"), py::arg("stream") = 0)
        .def("apply_env_commands_device", &BatchSim::apply_env_commands_device, py::arg("device_commands"),
             py::arg("count"), py::arg("stream") = 0)
        .def("step", &BatchSim::step, py::arg("ticks") = 1, py::arg("stream") = 0)
        .def("step_with_device_controls", &BatchSim::step_with_device_controls, py::arg("device_controls_by_tick"),
             py::arg("ticks"), py::arg("control_stride"), py::arg("stream") = 0)
        .def("step_with_device_commands", &BatchSim::step_with_device_commands, py::arg("device_controls_by_tick"),
             py::arg("control_stride"), py::arg("device_env_commands_by_tick"), py::arg("env_command_stride"),
             py::arg("ticks"), py::arg("stream") = 0)
        .def("reset_to_kickoff", &BatchSim::reset_to_kickoff, py::arg("seed") = 0, py::arg("stream") = 0)
        .def("synchronize", &BatchSim::synchronize, py::arg("stream") = 0)
        .def("set_physics_event_stream", &BatchSim::set_physics_event_stream, py::arg("records"), py::arg("windows"),
             py::arg("capacity"), py::arg("goal_only") = false,
             "Pass zeros to disable; synchronise before freeing the buffers.");
    // reference physics_event_layout (python/rocketgpu_bindings.cpp:77-86)
    m.def("physics_event_layout", [] {
        py::dict d;
        d["record_size"] = sizeof(rg_physics_event);
        d["window_size"] = sizeof(rg_physics_event_window);
        d["type_offset"] = offsetof(rg_physics_event, type);
        d["velocity_offset"] = offsetof(rg_physics_event, ball_velocity);
        d["count_offset"] = offsetof(rg_physics_event_window, count);
        d["overflow_offset"] = offsetof(rg_physics_event_window, overflow);
        d["goal_type"] = 5;
        return d;
    });
}
