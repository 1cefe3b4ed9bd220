"""ctypes binding of include/rocketgpu_b200.h (the in-tree CUDA library rocketgpu_b200/_lib/librocketgpu_b200.so).

This is the binding a ctypes/cffi user of the C ABI writes; a pybind11 module or a Rust FFI crate binds the same
symbols.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "librocketgpu_b200.so")

# Every symbol include/rocketgpu_b200.h declares.
EXPORTS = [
    "rg_last_error", "rg_version", "rg_sim_config_default", "rg_default_ball_state", "rg_default_env_state",
    "rg_batch_create", "rg_batch_destroy", "rg_batch_env_count", "rg_batch_car_capacity",
    "rg_batch_set_env_car_count", "rg_batch_upload_ball_states", "rg_batch_download_ball_states",
    "rg_batch_upload_env_states", "rg_batch_download_env_states", "rg_batch_step", "rg_batch_synchronize",
    "rg_batch_set_physics_event_stream",
    "rg_batch_device_view", "rg_ucrt_sinf", "rg_ucrt_cosf", "rg_ucrt_atan2f", "rg_ucrt_powf",
    "rg_arena_mesh_tables", "rg_batch_step_static_scratch",
    "rg_default_car_state", "rg_default_car_config", "rg_batch_upload_car_states", "rg_batch_download_car_states",
    "rg_batch_pad_capacity", "rg_batch_upload_pad_states", "rg_batch_download_pad_states", "rg_batch_set_car_configs",
    "rg_batch_upload_controls", "rg_batch_step_with_device_controls", "rg_batch_set_teams",
    "rg_batch_reset_to_kickoff", "rg_batch_apply_env_commands", "rg_batch_apply_env_commands_device",
    "rg_batch_step_with_device_commands", "rg_batch_episode_commands", "rg_batch_phase_timing",
    "rg_batch_phase_times", "rg_server_open", "rg_server_close", "rg_server_client_open", "rg_server_client_close",
    "rg_server_submit", "rg_server_poll", "rg_server_get_stats", "rg_batch_add_mesh", "rg_batch_set_arena_meshes",
    "rg_batch_set_launch_config", "rg_batch_get_launch_config", "rg_batch_upload_state_array",
    "rg_batch_download_state_array", "rg_batch_internal_state_layout", "rg_batch_download_internal_state",
    "rg_batch_upload_internal_state", "rg_car_preset", "rg_default_arena_rules",
]


class rg_sim_config(ctypes.Structure):
    _fields_ = [
        ("env_count", ctypes.c_int32), ("max_cars_per_env", ctypes.c_int32), ("tick_dt", ctypes.c_float),
        ("enable_boost_pads", ctypes.c_uint8), ("enable_car_car_collisions", ctypes.c_uint8),
        ("enable_demos", ctypes.c_uint8), ("enable_scoring", ctypes.c_uint8),
        ("respawn_rng_seed", ctypes.c_uint64),
        ("gravity_z", ctypes.c_float), ("ball_radius", ctypes.c_float), ("ball_mass", ctypes.c_float),
        ("car_mass", ctypes.c_float), ("ball_drag", ctypes.c_float), ("ball_friction", ctypes.c_float),
        ("ball_restitution", ctypes.c_float), ("ball_max_speed", ctypes.c_float),
        ("ball_max_ang_speed", ctypes.c_float), ("car_max_speed", ctypes.c_float),
        ("car_max_ang_speed", ctypes.c_float), ("arena_friction", ctypes.c_float),
        ("arena_restitution", ctypes.c_float), ("goal_base_threshold_y", ctypes.c_float),
        ("kickoff_settled", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 7),
    ]


class rg_vec3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class rg_arena_spawn(ctypes.Structure):
    _fields_ = [("pos", rg_vec3), ("yaw", ctypes.c_float)]


class rg_arena_goal(ctypes.Structure):
    _fields_ = [("point", rg_vec3), ("normal", rg_vec3), ("min", rg_vec3), ("max", rg_vec3)]


class rg_boost_pad_config(ctypes.Structure):
    _fields_ = [("pos", rg_vec3), ("is_big", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 3)]


class rg_arena_rules(ctypes.Structure):
    _fields_ = [("goals", rg_arena_goal * 2), ("kickoff_spawns", (rg_arena_spawn * 5) * 2),
                ("respawn_spawns", (rg_arena_spawn * 4) * 2), ("ball_spawn", rg_vec3)]


class rg_arena_layout(ctypes.Structure):
    _fields_ = [("vertices_uu", ctypes.POINTER(ctypes.c_float)), ("vertex_count", ctypes.c_int64),
                ("indices", ctypes.POINTER(ctypes.c_int32)), ("index_count", ctypes.c_int64),
                ("rules", ctypes.POINTER(rg_arena_rules)), ("boost_pads", ctypes.POINTER(rg_boost_pad_config)),
                ("boost_pad_count", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class rg_device_view(ctypes.Structure):
    _fields_ = [("ball_states", ctypes.c_void_p), ("env_states", ctypes.c_void_p),
                ("env_car_count", ctypes.c_void_p), ("car_states", ctypes.c_void_p),
                ("boost_pad_states", ctypes.c_void_p), ("controls", ctypes.c_void_p),
                ("car_configs", ctypes.c_void_p), ("teams", ctypes.c_void_p), ("wheel_runtime", ctypes.c_void_p)]


class rg_launch_config(ctypes.Structure):
    _fields_ = [("arena_threads", ctypes.c_int32), ("car_threads", ctypes.c_int32), ("use_graphs", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class rg_server_config(ctypes.Structure):
    _fields_ = [("max_arenas", ctypes.c_int32), ("policy", ctypes.c_int32), ("hbm_budget_bytes", ctypes.c_int64)]


class rg_server_stats(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_int64), ("used", ctypes.c_int64), ("slot_bytes", ctypes.c_int64),
                ("clients", ctypes.c_int64), ("rounds", ctypes.c_int64), ("arena_ticks", ctypes.c_int64),
                ("completed", ctypes.c_int64), ("busy_s", ctypes.c_double)]


_lib = None


def lib():
    """Loads the CUDA library (raises if it is not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"rocketgpu_b200 CUDA library not built ({LIB_PATH}); run python -m rocketgpu_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, sz, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_size_t, ctypes.c_int32
        L.rg_last_error.restype = ctypes.c_char_p
        L.rg_version.restype = ctypes.c_char_p
        L.rg_sim_config_default.argtypes = [vp]
        L.rg_default_ball_state.argtypes = [vp]
        L.rg_default_env_state.argtypes = [vp]
        L.rg_batch_create.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(vp)]
        L.rg_batch_destroy.argtypes = [vp]
        L.rg_batch_env_count.argtypes = [vp]
        L.rg_batch_env_count.restype = i64
        L.rg_batch_car_capacity.argtypes = [vp]
        L.rg_batch_car_capacity.restype = i64
        for n in ("rg_batch_set_env_car_count", "rg_batch_upload_ball_states", "rg_batch_download_ball_states",
                  "rg_batch_upload_env_states", "rg_batch_download_env_states", "rg_batch_upload_car_states",
                  "rg_batch_download_car_states", "rg_batch_upload_pad_states", "rg_batch_download_pad_states",
                  "rg_batch_set_car_configs", "rg_batch_upload_controls", "rg_batch_set_teams"):
            getattr(L, n).argtypes = [vp, vp, sz, vp]
        L.rg_batch_step.argtypes = [vp, i32, vp]
        L.rg_batch_synchronize.argtypes = [vp, vp]
        L.rg_batch_set_physics_event_stream.argtypes = [vp, vp, vp, ctypes.c_uint32, i32]
        L.rg_batch_device_view.argtypes = [vp, vp]
        for n in ("rg_ucrt_sinf", "rg_ucrt_cosf"):
            getattr(L, n).argtypes = [ctypes.c_float]
            getattr(L, n).restype = ctypes.c_float
        for n in ("rg_ucrt_atan2f", "rg_ucrt_powf"):
            getattr(L, n).argtypes = [ctypes.c_float, ctypes.c_float]
            getattr(L, n).restype = ctypes.c_float
        L.rg_arena_mesh_tables.argtypes = [vp, vp, vp, i64]
        L.rg_arena_mesh_tables.restype = i64
        L.rg_batch_step_static_scratch.argtypes = [vp, vp, vp, i32, i32, i32, vp]
        L.rg_default_car_state.argtypes = [vp]
        L.rg_default_car_config.argtypes = [vp]
        L.rg_car_preset.argtypes = [i32, vp]
        L.rg_default_arena_rules.argtypes = [vp]
        L.rg_batch_pad_capacity.argtypes = [vp]
        L.rg_batch_pad_capacity.restype = i64
        L.rg_batch_step_with_device_controls.argtypes = [vp, vp, i32, i32, vp]
        L.rg_batch_reset_to_kickoff.argtypes = [vp, ctypes.c_uint64, vp]
        L.rg_batch_apply_env_commands.argtypes = [vp, vp, sz, vp]
        L.rg_batch_apply_env_commands_device.argtypes = [vp, vp, sz, vp]
        L.rg_batch_step_with_device_commands.argtypes = [vp, vp, i32, vp, i32, i32, vp]
        L.rg_batch_episode_commands.argtypes = [vp, i32, ctypes.c_uint64, i32, vp, vp]
        L.rg_batch_phase_timing.argtypes = [vp, i32]
        L.rg_batch_phase_times.argtypes = [vp, vp, vp]
        L.rg_batch_add_mesh.argtypes = [vp, vp, vp]
        L.rg_batch_set_launch_config.argtypes = [vp, vp]
        L.rg_batch_internal_state_layout.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(i64)]
        L.rg_batch_download_internal_state.argtypes = [vp, vp, vp]
        L.rg_batch_upload_internal_state.argtypes = [vp, vp, vp]
        L.rg_batch_upload_state_array.argtypes = [vp, ctypes.c_char_p, vp, sz, i32, vp]
        L.rg_batch_download_state_array.argtypes = [vp, ctypes.c_char_p, vp, sz, vp]
        L.rg_batch_get_launch_config.argtypes = [vp, vp]
        L.rg_batch_set_arena_meshes.argtypes = [vp, vp, sz, vp]
        L.rg_server_open.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.POINTER(vp)]
        L.rg_server_close.argtypes = [vp]
        L.rg_server_client_open.argtypes = [vp, i32, vp, vp, vp, ctypes.c_uint64, vp]
        L.rg_server_client_close.argtypes = [vp, i32]
        L.rg_server_submit.argtypes = [vp, i32, i32, vp, vp]
        L.rg_server_poll.argtypes = [vp, i64, i32, vp, vp, vp, vp, vp]
        L.rg_server_get_stats.argtypes = [vp, vp]
        _lib = L
    return _lib
