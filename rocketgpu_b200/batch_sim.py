"""Python mirror of the reference's BatchSim (include/rocketgpu/rocketgpu.h:988-1089) over the C ABI.

The methods keep the reference's names and argument meaning (state arrays are the byte-identical public structs, as
numpy uint8 rows or structured arrays); errors raise the reference's exception types: ValueError for
std::invalid_argument, IndexError for std::out_of_range, RuntimeError for CUDA errors.

There is no CPU fallback: loading fails loudly when the CUDA library is missing or no GPU is visible.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import abi

CAR_BYTES, BALL_BYTES, ENV_BYTES, PAD_BYTES, CONTROLS_BYTES, CAR_CONFIG_BYTES, ENV_COMMAND_BYTES = \
    880, 288, 44, 16, 24, 120, 16

# rg_env_command / the reference's EnvCommand (rocketgpu.h:683-706) as a numpy record
ENV_COMMAND_DTYPE = np.dtype([("reset_to_kickoff", "u1"), ("reset_scoreboard", "u1"), ("reset_tick_count", "u1"),
                              ("kickoff_seed_mode", "u1"), ("new_round_bodies", "u1"), ("keep_boost_pads", "u1"),
                              ("kickoff_countdown_ticks", "<u2"), ("kickoff_seed", "<u8")])
assert ENV_COMMAND_DTYPE.itemsize == ENV_COMMAND_BYTES


def _check(rc: int):
    if rc == 0:
        return
    msg = abi.lib().rg_last_error().decode()
    if rc == 2:
        raise ValueError(msg)
    if rc == 3:
        raise IndexError(msg)
    raise RuntimeError(msg)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


PRESETS = ("octane", "dominus", "plank", "breakout", "hybrid", "merc")


def car_preset(preset) -> np.ndarray:
    """One hitbox preset as a raw CarConfig row (120 bytes): index 0-5 or name (reference OctaneConfig() ..
    MercConfig(), src/rocketgpu.cpp:417-490)."""
    k = PRESETS.index(preset.lower()) if isinstance(preset, str) else int(preset)
    out = np.zeros(120, np.uint8)
    _check(abi.lib().rg_car_preset(k, _ptr(out)))
    return out


def arena_rules() -> "abi.rg_arena_rules":
    """The official goals, kickoff / respawn spawns and ball spawn (reference ArenaLayout()), to edit field by field:
    `r.goals[t].point.y`, `r.kickoff_spawns[t][k].pos`, `.yaw`, `r.respawn_spawns[t][k]`, `r.ball_spawn` (uu, rad)."""
    r = abi.rg_arena_rules()
    abi.lib().rg_default_arena_rules(ctypes.byref(r))
    return r


class SimConfig:
    """The reference SimConfig / MutatorConfig fields this path takes (defaults as the reference's)."""

    def __init__(self, env_count: int = 1, max_cars_per_env: int = 6, **kw):
        c = abi.rg_sim_config()
        abi.lib().rg_sim_config_default(ctypes.byref(c))
        c.env_count = env_count
        c.max_cars_per_env = max_cars_per_env
        for k, v in kw.items():
            if not hasattr(c, k):
                raise ValueError(f"unknown SimConfig field {k}")
            setattr(c, k, v)
        self.c = c


# rg_physics_event / rg_physics_event_window as numpy records (reference PhysicsEvent / PhysicsEventWindow).
_V3 = (np.float32, (3,))
PHYSICS_EVENT_DTYPE = np.dtype({
    "names": ["tick", "type", "car_id", "other_car_id", "team", "pad_index", "car_on_ground", "is_big_pad", "is_demo",
              "position", "normal", "car_velocity", "ball_position", "ball_velocity", "boost_before", "boost_after"],
    "formats": [np.uint64, np.uint8, np.uint32, np.uint32, np.int32, np.uint32, np.uint8, np.uint8, np.uint8,
                _V3, _V3, _V3, _V3, _V3, np.float32, np.float32],
    "offsets": [0, 8, 12, 16, 20, 24, 28, 29, 30, 32, 44, 56, 68, 80, 92, 96],
    "itemsize": 104})
PHYSICS_EVENT_WINDOW_DTYPE = np.dtype([("tick", np.uint64), ("count", np.uint32), ("overflow", np.uint32)])
EVENT_TYPES = ("ball_touch_start", "ball_world_contact", "car_world_contact", "boost_pickup", "car_bump", "goal")


class BatchSim:
    """N independent arenas on one GPU, stepped by whole 120 Hz ticks.

    `vertices` (float32 [V, 3], uu) and `indices` (int32 [3T]) are the arena's triangle mesh (ArenaLayout.meshes[0]).
    """

    def __init__(self, config: SimConfig, vertices: np.ndarray, indices: np.ndarray, device: int = 0,
                 rules: "abi.rg_arena_rules | None" = None, boost_pads=None):
        """`rules`: the layout's goals and spawns (arena_rules(), edited), None for the official ones;
        `boost_pads`: [(x, y, z, is_big)] (at most 48), None for the 34 soccar pads."""
        self._v = np.ascontiguousarray(vertices, np.float32)
        self._i = np.ascontiguousarray(indices, np.int32)
        lay = abi.rg_arena_layout()
        lay.vertices_uu = self._v.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        lay.vertex_count = len(self._v)
        lay.indices = self._i.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        lay.index_count = len(self._i)
        if rules is not None:
            self._rules = rules
            lay.rules = ctypes.pointer(rules)
        if boost_pads is not None:
            self._pads = (abi.rg_boost_pad_config * max(1, len(boost_pads)))()
            for k, (x, y, z, big) in enumerate(boost_pads):
                self._pads[k].pos = abi.rg_vec3(x, y, z)
                self._pads[k].is_big = int(big)
            lay.boost_pads = ctypes.cast(self._pads, ctypes.POINTER(abi.rg_boost_pad_config))
            lay.boost_pad_count = len(boost_pads)
        h = ctypes.c_void_p()
        _check(abi.lib().rg_batch_create(ctypes.byref(config.c), ctypes.byref(lay), device, ctypes.byref(h)))
        self._h = h
        self.config = config

    def add_mesh(self, vertices: np.ndarray, indices: np.ndarray) -> int:
        """Another arena geometry for this batch; returns its mesh index (the create-time mesh is 0)."""
        v = np.ascontiguousarray(vertices, np.float32)
        i = np.ascontiguousarray(indices, np.int32)
        lay = abi.rg_arena_layout()
        lay.vertices_uu = v.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        lay.vertex_count = len(v)
        lay.indices = i.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        lay.index_count = len(i)
        out = ctypes.c_int32()
        _check(abi.lib().rg_batch_add_mesh(self._h, ctypes.byref(lay), ctypes.byref(out)))
        return out.value

    def set_arena_meshes(self, mesh_index, stream: int = 0):
        m = np.ascontiguousarray(mesh_index, np.uint8)
        _check(abi.lib().rg_batch_set_arena_meshes(self._h, _ptr(m), len(m), stream))

    def close(self):
        if getattr(self, "_h", None):
            abi.lib().rg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def env_count(self) -> int:
        return abi.lib().rg_batch_env_count(self._h)

    def car_capacity(self) -> int:
        return abi.lib().rg_batch_car_capacity(self._h)

    def set_env_car_count(self, counts, stream: int = 0):
        c = np.ascontiguousarray(counts, np.int32)
        _check(abi.lib().rg_batch_set_env_car_count(self._h, _ptr(c), len(c), stream))

    def upload_ball_states(self, states: np.ndarray, stream: int = 0):
        s = np.ascontiguousarray(states, np.uint8).reshape(-1, BALL_BYTES)
        _check(abi.lib().rg_batch_upload_ball_states(self._h, _ptr(s), len(s), stream))

    def download_ball_states(self, count: int | None = None, stream: int = 0) -> np.ndarray:
        n = self.env_count() if count is None else count
        out = np.zeros((n, BALL_BYTES), np.uint8)
        _check(abi.lib().rg_batch_download_ball_states(self._h, _ptr(out), n, stream))
        return out

    def upload_env_states(self, states: np.ndarray, stream: int = 0):
        s = np.ascontiguousarray(states, np.uint8).reshape(-1, ENV_BYTES)
        _check(abi.lib().rg_batch_upload_env_states(self._h, _ptr(s), len(s), stream))

    def download_env_states(self, count: int | None = None, stream: int = 0) -> np.ndarray:
        n = self.env_count() if count is None else count
        out = np.zeros((n, ENV_BYTES), np.uint8)
        _check(abi.lib().rg_batch_download_env_states(self._h, _ptr(out), n, stream))
        return out

    def pad_capacity(self) -> int:
        return abi.lib().rg_batch_pad_capacity(self._h)

    def upload_car_states(self, states: np.ndarray, stream: int = 0):
        s = np.ascontiguousarray(states, np.uint8).reshape(-1, CAR_BYTES)
        _check(abi.lib().rg_batch_upload_car_states(self._h, _ptr(s), len(s), stream))

    def download_car_states(self, count: int | None = None, stream: int = 0) -> np.ndarray:
        n = self.car_capacity() if count is None else count
        out = np.zeros((n, CAR_BYTES), np.uint8)
        _check(abi.lib().rg_batch_download_car_states(self._h, _ptr(out), n, stream))
        return out

    def upload_boost_pad_states(self, states: np.ndarray, stream: int = 0):
        s = np.ascontiguousarray(states, np.uint8).reshape(-1, PAD_BYTES)
        _check(abi.lib().rg_batch_upload_pad_states(self._h, _ptr(s), len(s), stream))

    def download_boost_pad_states(self, count: int | None = None, stream: int = 0) -> np.ndarray:
        n = self.pad_capacity() if count is None else count
        out = np.zeros((n, PAD_BYTES), np.uint8)
        _check(abi.lib().rg_batch_download_pad_states(self._h, _ptr(out), n, stream))
        return out

    def set_car_configs(self, configs: np.ndarray, stream: int = 0):
        s = np.ascontiguousarray(configs, np.uint8).reshape(-1, CAR_CONFIG_BYTES)
        _check(abi.lib().rg_batch_set_car_configs(self._h, _ptr(s), len(s), stream))

    def set_teams(self, teams, stream: int = 0):
        t = np.ascontiguousarray(teams, np.uint8)
        _check(abi.lib().rg_batch_set_teams(self._h, _ptr(t), len(t), stream))

    def reset_to_kickoff(self, seed: int = 0, stream: int = 0):
        _check(abi.lib().rg_batch_reset_to_kickoff(self._h, seed, stream))

    def upload_controls(self, controls: np.ndarray, stream: int = 0):
        s = np.ascontiguousarray(controls, np.uint8).reshape(-1, CONTROLS_BYTES)
        _check(abi.lib().rg_batch_upload_controls(self._h, _ptr(s), len(s), stream))

    def step_with_device_controls(self, device_controls: int, ticks: int, control_stride: int, stream: int = 0):
        """`device_controls` is a device pointer to rg_car_controls rows (e.g. a torch uint8 tensor's data_ptr())."""
        _check(abi.lib().rg_batch_step_with_device_controls(self._h, ctypes.c_void_p(device_controls), ticks,
                                                            control_stride, stream))

    def apply_env_commands(self, commands: np.ndarray, stream: int = 0):
        """`commands`: ENV_COMMAND_DTYPE records (or uint8 rows of 16 bytes), one per env from env 0."""
        c = np.ascontiguousarray(commands).view(np.uint8).reshape(-1, ENV_COMMAND_BYTES)
        _check(abi.lib().rg_batch_apply_env_commands(self._h, _ptr(c), len(c), stream))

    def apply_env_commands_device(self, device_commands: int, count: int, stream: int = 0):
        _check(abi.lib().rg_batch_apply_env_commands_device(self._h, ctypes.c_void_p(device_commands), count, stream))

    def step_with_device_commands(self, device_controls: int, control_stride: int, device_commands: int,
                                  command_stride: int, ticks: int, stream: int = 0):
        _check(abi.lib().rg_batch_step_with_device_commands(self._h, ctypes.c_void_p(device_controls), control_stride,
                                                            ctypes.c_void_p(device_commands), command_stride, ticks,
                                                            stream))

    def episode_commands(self, no_touch_ticks: int, device_commands: int, stagger_seed: int = 0, init: bool = False,
                         stream: int = 0):
        _check(abi.lib().rg_batch_episode_commands(self._h, no_touch_ticks, stagger_seed, int(init),
                                                   ctypes.c_void_p(device_commands), stream))

    def step(self, ticks: int = 1, stream: int = 0):
        _check(abi.lib().rg_batch_step(self._h, ticks, stream))

    def synchronize(self, stream: int = 0):
        _check(abi.lib().rg_batch_synchronize(self._h, stream))

    def set_physics_event_stream(self, records: int, windows: int, capacity: int, goal_only: bool = False):
        """BatchSim::set_physics_event_stream (reference rocketgpu.h:1015, in the Python binding's form): device
        pointers to records[env_count * capacity] (PHYSICS_EVENT_DTYPE) and windows[env_count]
        (PHYSICS_EVENT_WINDOW_DTYPE); zeros turn the stream off."""
        _check(abi.lib().rg_batch_set_physics_event_stream(self._h, records or None, windows or None, capacity,
                                                           1 if goal_only else 0))

    def device_view(self) -> dict:
        v = abi.rg_device_view()
        _check(abi.lib().rg_batch_device_view(self._h, ctypes.byref(v)))
        return {name: getattr(v, name) for name, _ in v._fields_}

    def boost_pad_capacity(self) -> int:
        return self.pad_capacity()

    def device_arrays(self) -> dict:
        """Zero-copy views of the device state arrays (reference BatchSim.device_arrays,
        python/rocketgpu_bindings.cpp:846-898): per array a dict with a CUDA array interface (one record per element,
        typestr |V<itemsize>), itemsize, count, per_env and the element it indexes. torch.as_tensor / cupy.asarray
        take the interface; the views stay valid until the batch is closed."""
        v = self.device_view()
        envs, cars = self.env_count(), self.car_capacity()
        per = cars // envs if envs else 0
        pads = self.pad_capacity()
        spec = [("car_states", v["car_states"], cars, CAR_BYTES, per, "car slot", False),
                ("controls", v["controls"], cars, CONTROLS_BYTES, per, "car slot", False),
                ("car_configs", v["car_configs"], cars, CAR_CONFIG_BYTES, per, "car slot", False),
                ("teams", v["teams"], cars, 1, per, "car slot", False),
                ("ball_states", v["ball_states"], envs, BALL_BYTES, 1, "env", False),
                ("env_states", v["env_states"], envs, ENV_BYTES, 1, "env", False),
                ("boost_pad_states", v["boost_pad_states"], pads, PAD_BYTES, pads // envs if envs else 0,
                 "boost pad", False),
                ("env_car_count", v["env_car_count"], envs, 4, 1, "env", False),
                ("wheel_runtime", v["wheel_runtime"], cars, 292, per, "car slot", True)]
        out = {}
        for name, ptr, count, size, per_env, element, ro in spec:
            out[name] = {"__cuda_array_interface__": {"data": (int(ptr or 0), ro), "shape": (count,),
                                                      "typestr": f"|V{size}", "strides": None, "version": 3},
                         "itemsize": size, "count": count, "per_env": per_env, "element": element}
        return out

    def internal_state_layout(self) -> list:
        """[(section name, bytes)] of the internal state blob (reference BatchSim.internal_state_layout)."""
        out, k = [], 0
        while True:
            name, size = ctypes.c_char_p(), ctypes.c_int64()
            if abi.lib().rg_batch_internal_state_layout(self._h, k, ctypes.byref(name), ctypes.byref(size)) != 0:
                return out
            out.append((name.value.decode(), size.value))
            k += 1

    def download_internal_state(self, stream: int = 0) -> np.ndarray:
        total = sum(b for _, b in self.internal_state_layout())
        out = np.zeros(total, np.uint8)
        _check(abi.lib().rg_batch_download_internal_state(self._h, _ptr(out), stream))
        return out

    def upload_internal_state(self, blob: np.ndarray, stream: int = 0):
        b = np.ascontiguousarray(blob, np.uint8)
        assert b.size == sum(n for _, n in self.internal_state_layout())
        _check(abi.lib().rg_batch_upload_internal_state(self._h, _ptr(b), stream))

    def upload_state_array(self, name: str, host_ptr: int, count: int, preserve_internal: bool = False,
                           stream: int = 0):
        """Raw structs from host memory by array name (reference BatchSim.upload_state_array)."""
        _check(abi.lib().rg_batch_upload_state_array(self._h, name.encode(), ctypes.c_void_p(host_ptr), count,
                                                     int(preserve_internal), stream))

    def download_state_array(self, name: str, host_ptr: int, count: int, stream: int = 0):
        """Raw structs into host memory by array name (reference BatchSim.download_state_array)."""
        _check(abi.lib().rg_batch_download_state_array(self._h, name.encode(), ctypes.c_void_p(host_ptr), count,
                                                       stream))
