"""ctypes wrapper of the oracle: the reference's own CPU BatchSim built by oracle/Makefile into oracle/_ref.

Test infrastructure only (the checker): tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it; the
product never imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "_ref", "librg_oracle.so")

CAR_BYTES, BALL_BYTES, ENV_BYTES, PAD_BYTES, CTRL_BYTES, CFG_BYTES, CMD_BYTES = 880, 288, 44, 16, 24, 120, 16

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_create.argtypes = [i32, i32, vp, i64, vp, i64, ctypes.c_uint64, ctypes.c_uint32,
                                 ctypes.POINTER(vp)]
        L.orc_create_layout.argtypes = [i32, i32, vp, i64, vp, i64, ctypes.c_uint64, ctypes.c_uint32, vp, vp, i32, vp]
        L.orc_destroy.argtypes = [vp]
        L.orc_car_capacity.argtypes = [vp]
        L.orc_car_capacity.restype = i64
        L.orc_pad_capacity.argtypes = [vp]
        L.orc_pad_capacity.restype = i64
        for n in ("orc_set_env_car_count", "orc_set_teams", "orc_set_car_configs", "orc_apply_env_commands",
                  "orc_upload_controls", "orc_download_cars", "orc_download_balls", "orc_download_envs",
                  "orc_download_pads", "orc_upload_envs", "orc_upload_pads"):
            getattr(L, n).argtypes = [vp, vp, i64]
        for n in ("orc_upload_cars", "orc_upload_balls"):
            getattr(L, n).argtypes = [vp, vp, i64, ctypes.c_int]
        L.orc_reset_to_kickoff.argtypes = [vp, ctypes.c_uint64]
        L.orc_step.argtypes = [vp, i32]
        L.orc_step_with_controls.argtypes = [vp, vp, i32, i32]
        L.orc_step_with_commands.argtypes = [vp, vp, i32, vp, i32, i32]
        L.orc_car_preset.argtypes = [ctypes.c_int, vp]
        L.orc_set_physics_event_stream.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_int]
        L.orc_physics_event_sizes.argtypes = [vp]
        L.orc_default_states.argtypes = [vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def default_states():
    car = np.zeros(CAR_BYTES, np.uint8)
    ball = np.zeros(BALL_BYTES, np.uint8)
    env = np.zeros(ENV_BYTES, np.uint8)
    pad = np.zeros(PAD_BYTES, np.uint8)
    cfg = np.zeros(CFG_BYTES, np.uint8)
    _check(lib().orc_default_states(_ptr(car), _ptr(ball), _ptr(env), _ptr(pad), _ptr(cfg)))
    return car, ball, env, pad, cfg


def car_preset(which: int) -> np.ndarray:
    out = np.zeros(CFG_BYTES, np.uint8)
    _check(lib().orc_car_preset(which, _ptr(out)))
    return out


class OracleSim:
    """The reference BatchSim on a custom one-mesh ArenaLayout (uu vertices, int32 indices)."""

    def __init__(self, env_count: int, max_cars: int, vertices: np.ndarray, indices: np.ndarray,
                 respawn_seed: int = 0, kickoff_settled: bool = True, boost_pads: bool = True,
                 car_car: bool = True, demos: bool = True, scoring: bool = True, rules=None, pad_layout=None):
        """`rules`: 99 floats in rg_arena_rules order (goals, kickoff spawns, respawn spawns, ball spawn);
        `pad_layout`: [(x, y, z, is_big)] replacing the 34 soccar pads."""
        v = np.ascontiguousarray(vertices, np.float32)
        i = np.ascontiguousarray(indices, np.int32)
        flags = (1 if kickoff_settled else 0) | (2 if boost_pads else 0) | (4 if car_car else 0) | \
            (8 if demos else 0) | (16 if scoring else 0)
        h = ctypes.c_void_p()
        rf = None if rules is None else np.ascontiguousarray(rules, np.float32).reshape(99)
        pf = None if pad_layout is None else np.ascontiguousarray(pad_layout, np.float32).reshape(-1, 4)
        _check(lib().orc_create_layout(env_count, max_cars, _ptr(v), len(v), _ptr(i), len(i), respawn_seed, flags,
                                       None if rf is None else _ptr(rf), None if pf is None else _ptr(pf),
                                       0 if pf is None else len(pf), ctypes.byref(h)))
        self.h = h
        self.env_count = env_count
        self.max_cars = max_cars
        self.car_capacity = lib().orc_car_capacity(h)
        self.pad_capacity = lib().orc_pad_capacity(h)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_env_car_count(self, counts):
        c = np.ascontiguousarray(counts, np.int32)
        _check(lib().orc_set_env_car_count(self.h, _ptr(c), len(c)))

    def set_teams(self, teams):
        t = np.ascontiguousarray(teams, np.uint8)
        _check(lib().orc_set_teams(self.h, _ptr(t), len(t)))

    def set_car_configs(self, cfgs: np.ndarray):
        c = np.ascontiguousarray(cfgs, np.uint8).reshape(-1, CFG_BYTES)
        _check(lib().orc_set_car_configs(self.h, _ptr(c), len(c)))

    def reset_to_kickoff(self, seed: int = 0):
        _check(lib().orc_reset_to_kickoff(self.h, seed))

    def set_physics_event_stream(self, capacity: int, goal_only: bool = False):
        """The reference's event stream on host arrays the oracle writes: returns (records, windows), uint8 arrays of
        env_count * capacity * 104 and env_count * 16 bytes (capacity 0: off, returns None)."""
        if capacity == 0:
            _check(lib().orc_set_physics_event_stream(self.h, None, None, 0, 0))
            self._events = None
            return None
        n = self.env_count
        self._events = (np.zeros(n * capacity * 104, np.uint8), np.zeros(n * 16, np.uint8))
        _check(lib().orc_set_physics_event_stream(self.h, _ptr(self._events[0]), _ptr(self._events[1]), capacity,
                                                  1 if goal_only else 0))
        return self._events

    def apply_env_commands(self, cmds: np.ndarray):
        c = np.ascontiguousarray(cmds, np.uint8).reshape(-1, CMD_BYTES)
        _check(lib().orc_apply_env_commands(self.h, _ptr(c), len(c)))

    def step(self, ticks: int = 1):
        _check(lib().orc_step(self.h, ticks))

    def step_with_controls(self, ctrl: np.ndarray, ticks: int, stride: int):
        c = np.ascontiguousarray(ctrl, np.uint8)
        _check(lib().orc_step_with_controls(self.h, _ptr(c), ticks, stride))

    def step_with_commands(self, ctrl: np.ndarray, ctrl_stride: int, cmds: np.ndarray, cmd_stride: int, ticks: int):
        c = np.ascontiguousarray(ctrl, np.uint8)
        m = np.ascontiguousarray(cmds, np.uint8)
        _check(lib().orc_step_with_commands(self.h, _ptr(c), ctrl_stride, _ptr(m), cmd_stride, ticks))

    def step_with_device_commands(self, ctrl_ptr: int, ctrl_stride: int, cmd_ptr: int, cmd_stride: int, ticks: int):
        """Pointers passed through as they are: device pointers for the reference's CUDA build
        (librg_oracle_cuda.so), host pointers for its CPU build."""
        _check(lib().orc_step_with_commands(self.h, ctypes.c_void_p(ctrl_ptr), ctrl_stride, ctypes.c_void_p(cmd_ptr),
                                            cmd_stride, ticks))

    def _down(self, fn, n, nbytes):
        out = np.zeros((n, nbytes), np.uint8)
        _check(fn(self.h, _ptr(out), n))
        return out

    def cars(self):
        return self._down(lib().orc_download_cars, self.car_capacity, CAR_BYTES)

    def balls(self):
        return self._down(lib().orc_download_balls, self.env_count, BALL_BYTES)

    def envs(self):
        return self._down(lib().orc_download_envs, self.env_count, ENV_BYTES)

    def pads(self):
        return self._down(lib().orc_download_pads, self.env_count * self.pad_capacity // max(1, self.env_count)
                          if False else self.pad_capacity, PAD_BYTES)

    def upload_cars(self, cars: np.ndarray, preserve_internal=False):
        c = np.ascontiguousarray(cars, np.uint8)
        _check(lib().orc_upload_cars(self.h, _ptr(c), len(c), int(preserve_internal)))

    def upload_balls(self, balls: np.ndarray, preserve_internal=False):
        b = np.ascontiguousarray(balls, np.uint8)
        _check(lib().orc_upload_balls(self.h, _ptr(b), len(b), int(preserve_internal)))

    def upload_envs(self, envs: np.ndarray):
        e = np.ascontiguousarray(envs, np.uint8)
        _check(lib().orc_upload_envs(self.h, _ptr(e), len(e)))
