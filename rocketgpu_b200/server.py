"""Python binding of the serving loop (rg_server_* in include/rocketgpu_b200.h): many RL clients stepping their own
arenas on one GPU through one pool, with continuous batching between one-tick rounds.

No counterpart in the reference (whose BatchSim steps one batch per call under a process-wide lock,
src/rocketgpu_cuda.cu:2868-2916); every client's results are bitwise those of its arenas stepped alone in a BatchSim.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi
from .batch_sim import BALL_BYTES, CAR_BYTES, CAR_CONFIG_BYTES, CONTROLS_BYTES, ENV_BYTES, SimConfig, _check


class Busy(RuntimeError):
    """The pool has no free range for the client's arenas now (RG_BUSY); retry after other clients close."""


def _call(rc: int):
    if rc == 5:
        raise Busy(abi.lib().rg_last_error().decode())
    _check(rc)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Server:
    POLICIES = {"continuous": 0, "static": 1}

    def __init__(self, vertices: np.ndarray, indices: np.ndarray, max_arenas: int = 0, hbm_budget_bytes: int = 0,
                 policy: str = "continuous", max_cars_per_env: int = 6, device: int = 0, **sim_kw):
        self._v = np.ascontiguousarray(vertices, np.float32)
        self._i = np.ascontiguousarray(indices, np.int32)
        lay = abi.rg_arena_layout()
        lay.vertices_uu = self._v.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        lay.vertex_count = len(self._v)
        lay.indices = self._i.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        lay.index_count = len(self._i)
        cfg = abi.rg_server_config(max_arenas, self.POLICIES[policy], hbm_budget_bytes)
        sim = SimConfig(env_count=1, max_cars_per_env=max_cars_per_env, **{"kickoff_settled": 0, **sim_kw})
        h = ctypes.c_void_p()
        _call(abi.lib().rg_server_open(ctypes.byref(cfg), ctypes.byref(sim.c), ctypes.byref(lay), device,
                                       ctypes.byref(h)))
        self._h = h
        self.max_cars = max_cars_per_env
        self._arenas = {}

    def close(self):
        if getattr(self, "_h", None):
            abi.lib().rg_server_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def open_client(self, car_counts, teams=None, configs=None, kickoff_seed: int = 0) -> int:
        c = np.ascontiguousarray(car_counts, np.int32)
        t = None if teams is None else np.ascontiguousarray(teams, np.uint8)
        k = None if configs is None else np.ascontiguousarray(configs, np.uint8).reshape(-1, CAR_CONFIG_BYTES)
        out = ctypes.c_int32()
        _call(abi.lib().rg_server_client_open(self._h, len(c), _ptr(c), _ptr(t), _ptr(k), kickoff_seed,
                                              ctypes.byref(out)))
        self._arenas[out.value] = len(c)
        return out.value

    def close_client(self, client: int):
        _call(abi.lib().rg_server_client_close(self._h, client))
        self._arenas.pop(client, None)

    def submit(self, client: int, controls: np.ndarray) -> int:
        """`controls`: [ticks, arenas * max_cars, 24] bytes (rg_car_controls rows), 1 <= ticks <= 8."""
        c = np.ascontiguousarray(controls, np.uint8)
        ticks = c.shape[0]
        assert c.reshape(ticks, -1).shape[1] == self._arenas[client] * self.max_cars * CONTROLS_BYTES
        out = ctypes.c_int64()
        _call(abi.lib().rg_server_submit(self._h, client, ticks, _ptr(c), ctypes.byref(out)))
        return out.value

    def poll(self, request: int, client: int | None = None, wait_ms: int = 0):
        """Returns None while the request runs; then (latency_s, cars, balls, envs) with the states when `client` is
        given (else only the latency)."""
        done = ctypes.c_int32()
        lat = ctypes.c_double()
        cars = balls = envs = None
        if client is not None:
            n = self._arenas[client]
            cars = np.zeros((n * self.max_cars, CAR_BYTES), np.uint8)
            balls = np.zeros((n, BALL_BYTES), np.uint8)
            envs = np.zeros((n, ENV_BYTES), np.uint8)
        _call(abi.lib().rg_server_poll(self._h, request, wait_ms, _ptr(cars), _ptr(balls), _ptr(envs),
                                       ctypes.byref(done), ctypes.byref(lat)))
        if not done.value:
            return None
        return lat.value, cars, balls, envs

    def stats(self) -> dict:
        s = abi.rg_server_stats()
        _call(abi.lib().rg_server_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}
